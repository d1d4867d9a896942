// Filter-bank kernels: 8192-point tiles, 256 threads (32 elements each), power-of-two sizes.
#include "sk_fcfb_inst.cuh"

namespace sk {

const void* fcfb_ptr_8192(bool persistent) { return fcfb_ptr<8192, 256, 2, false>(persistent); }

}  // namespace sk
