// Filter-bank kernels: 8192-point tiles, 256 threads, chirp-z sizes.
#include "sk_fcfb_inst.cuh"

namespace sk {

const void* fcfb_ptr_8192_chirp(bool persistent) { return fcfb_ptr<8192, 256, 2, true>(persistent); }

}  // namespace sk
