// Forward-FFT kernels for the 16-bit input formats (inputformats.rs:65-155).
#include "sk_fwd_inst.cuh"

namespace sk {

cudaError_t fwd_prepare_16(int fmt) {
  switch (fmt) {
    case SK_FMT_S16LE: return fwd_prepare_one<SK_FMT_S16LE>();
    case SK_FMT_S16BE: return fwd_prepare_one<SK_FMT_S16BE>();
    case SK_FMT_CS16LE: return fwd_prepare_one<SK_FMT_CS16LE>();
    case SK_FMT_CS16BE: return fwd_prepare_one<SK_FMT_CS16BE>();
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_fwd_16(int fmt, int grid, const FwdArgs& a, cudaStream_t st) {
  switch (fmt) {
    case SK_FMT_S16LE: return fwd_launch_one<SK_FMT_S16LE>(grid, a, st);
    case SK_FMT_S16BE: return fwd_launch_one<SK_FMT_S16BE>(grid, a, st);
    case SK_FMT_CS16LE: return fwd_launch_one<SK_FMT_CS16LE>(grid, a, st);
    case SK_FMT_CS16BE: return fwd_launch_one<SK_FMT_CS16BE>(grid, a, st);
  }
  return cudaErrorInvalidValue;
}

const void* fwd_kernel_ptr_16(int fmt) {
  switch (fmt) {
    case SK_FMT_S16LE: return fwd_ptr_one<SK_FMT_S16LE>();
    case SK_FMT_S16BE: return fwd_ptr_one<SK_FMT_S16BE>();
    case SK_FMT_CS16LE: return fwd_ptr_one<SK_FMT_CS16LE>();
    case SK_FMT_CS16BE: return fwd_ptr_one<SK_FMT_CS16BE>();
  }
  return nullptr;
}

}  // namespace sk
