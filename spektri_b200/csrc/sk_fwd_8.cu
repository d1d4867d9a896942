// Forward-FFT kernels for the 8-bit input formats (inputformats.rs:65-155).
#include "sk_fwd_inst.cuh"

namespace sk {

cudaError_t fwd_prepare_8(int fmt) {
  switch (fmt) {
    case SK_FMT_S8: return fwd_prepare_one<SK_FMT_S8>();
    case SK_FMT_U8: return fwd_prepare_one<SK_FMT_U8>();
    case SK_FMT_CS8: return fwd_prepare_one<SK_FMT_CS8>();
    case SK_FMT_CU8: return fwd_prepare_one<SK_FMT_CU8>();
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_fwd_8(int fmt, int grid, const FwdArgs& a, cudaStream_t st) {
  switch (fmt) {
    case SK_FMT_S8: return fwd_launch_one<SK_FMT_S8>(grid, a, st);
    case SK_FMT_U8: return fwd_launch_one<SK_FMT_U8>(grid, a, st);
    case SK_FMT_CS8: return fwd_launch_one<SK_FMT_CS8>(grid, a, st);
    case SK_FMT_CU8: return fwd_launch_one<SK_FMT_CU8>(grid, a, st);
  }
  return cudaErrorInvalidValue;
}

const void* fwd_kernel_ptr_8(int fmt) {
  switch (fmt) {
    case SK_FMT_S8: return fwd_ptr_one<SK_FMT_S8>();
    case SK_FMT_U8: return fwd_ptr_one<SK_FMT_U8>();
    case SK_FMT_CS8: return fwd_ptr_one<SK_FMT_CS8>();
    case SK_FMT_CU8: return fwd_ptr_one<SK_FMT_CU8>();
  }
  return nullptr;
}

}  // namespace sk
