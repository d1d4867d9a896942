// Filter-bank kernel for chirp-z tiles of M = 16384 points (IFFT sizes 4684 ..
// 9364): one tile per CTA, 1024 threads (16 elements each), one CTA per SM.
#include "sk_fcfb_inst.cuh"

namespace sk {

const void* fcfb_ptr_16384_chirp() { return (const void*)fcfb_kernel<16384, 1024, 1, false, true>; }

}  // namespace sk
