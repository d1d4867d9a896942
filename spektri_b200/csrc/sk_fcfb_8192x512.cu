// Filter-bank kernels: 8192-point tiles, 512 threads (16 elements each), power-of-two sizes.
#include "sk_fcfb_inst.cuh"

namespace sk {

const void* fcfb_ptr_8192x512(bool persistent) { return fcfb_ptr<8192, 512, 2, false>(persistent); }

}  // namespace sk
