// Forward-FFT kernels for the 32-bit input formats (inputformats.rs:65-155).
#include "sk_fwd_inst.cuh"

namespace sk {

cudaError_t fwd_prepare_32(int fmt) {
  switch (fmt) {
    case SK_FMT_F32LE: return fwd_prepare_one<SK_FMT_F32LE>();
    case SK_FMT_F32BE: return fwd_prepare_one<SK_FMT_F32BE>();
    case SK_FMT_CF32LE: return fwd_prepare_one<SK_FMT_CF32LE>();
    case SK_FMT_CF32BE: return fwd_prepare_one<SK_FMT_CF32BE>();
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_fwd_32(int fmt, int grid, const FwdArgs& a, cudaStream_t st) {
  switch (fmt) {
    case SK_FMT_F32LE: return fwd_launch_one<SK_FMT_F32LE>(grid, a, st);
    case SK_FMT_F32BE: return fwd_launch_one<SK_FMT_F32BE>(grid, a, st);
    case SK_FMT_CF32LE: return fwd_launch_one<SK_FMT_CF32LE>(grid, a, st);
    case SK_FMT_CF32BE: return fwd_launch_one<SK_FMT_CF32BE>(grid, a, st);
  }
  return cudaErrorInvalidValue;
}

const void* fwd_kernel_ptr_32(int fmt) {
  switch (fmt) {
    case SK_FMT_F32LE: return fwd_ptr_one<SK_FMT_F32LE>();
    case SK_FMT_F32BE: return fwd_ptr_one<SK_FMT_F32BE>();
    case SK_FMT_CF32LE: return fwd_ptr_one<SK_FMT_CF32LE>();
    case SK_FMT_CF32BE: return fwd_ptr_one<SK_FMT_CF32BE>();
  }
  return nullptr;
}

}  // namespace sk
