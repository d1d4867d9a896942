// Filter-bank kernels: 4096-point tiles, 256 threads (16 elements each, 4 CTAs per SM), power-of-two sizes.
#include "sk_fcfb_inst.cuh"

namespace sk {

const void* fcfb_ptr_4096(bool persistent) { return fcfb_ptr<4096, 256, 4, false>(persistent); }

}  // namespace sk
