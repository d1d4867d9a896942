// Filter-bank kernels: 8192-point tiles, 512 threads, chirp-z sizes.
#include "sk_fcfb_inst.cuh"

namespace sk {

const void* fcfb_ptr_8192x512_chirp(bool persistent) { return fcfb_ptr<8192, 512, 2, true>(persistent); }

}  // namespace sk
