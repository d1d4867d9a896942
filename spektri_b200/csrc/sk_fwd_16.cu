// Forward-FFT kernels for the 16-bit input formats (inputformats.rs:65-155).
#include "sk_fwd_inst.cuh"

namespace sk {

#define SK_FOR_FORMATS(X) X(SK_FMT_S16LE) X(SK_FMT_S16BE) X(SK_FMT_CS16LE) X(SK_FMT_CS16BE)

cudaError_t fwd_prepare_16(int fmt) {
#define CASE(F) case F: return fwd_prepare_one<F>();
  switch (fmt) { SK_FOR_FORMATS(CASE) }
#undef CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_fwd_16(int fmt, int grid, const FwdArgs& a, cudaStream_t st) {
#define CASE(F) case F: return fwd_launch_one<F>(grid, a, st);
  switch (fmt) { SK_FOR_FORMATS(CASE) }
#undef CASE
  return cudaErrorInvalidValue;
}

cudaError_t launch_fwd_col_16(int fmt, int grid, const FwdArgs& a, float2* Y, cudaStream_t st) {
#define CASE(F) case F: return fwd_col_launch_one<F>(grid, a, Y, st);
  switch (fmt) { SK_FOR_FORMATS(CASE) }
#undef CASE
  return cudaErrorInvalidValue;
}

const void* fwd_kernel_ptr_16(int fmt, int kind, int R1) {
#define CASE(F) case F: return fwd_ptr_one<F>(kind, R1);
  switch (fmt) { SK_FOR_FORMATS(CASE) }
#undef CASE
  return nullptr;
}

}  // namespace sk
