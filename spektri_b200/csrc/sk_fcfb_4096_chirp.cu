// Filter-bank kernels: 4096-point tiles, 256 threads, chirp-z sizes.
#include "sk_fcfb_inst.cuh"

namespace sk {

const void* fcfb_ptr_4096_chirp(bool persistent) { return fcfb_ptr<4096, 256, 4, true>(persistent); }

}  // namespace sk
