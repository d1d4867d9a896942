// Kernel instances and launchers for the spectrum split, the fused Welch
// accumulation, the filter bank (plain and persistent) and its adjoint, plus
// the per-width dispatch of the forward FFT.
#include "sk_internal.h"
#include "sk_kernels.cuh"

namespace sk {

cudaError_t fwd_prepare(int fmt) {
  switch (format_bits(fmt)) {
    case 8: return fwd_prepare_8(fmt);
    case 16: return fwd_prepare_16(fmt);
    case 32: return fwd_prepare_32(fmt);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_fwd(int fmt, int grid, const FwdArgs& a, cudaStream_t st) {
  switch (format_bits(fmt)) {
    case 8: return launch_fwd_8(fmt, grid, a, st);
    case 16: return launch_fwd_16(fmt, grid, a, st);
    case 32: return launch_fwd_32(fmt, grid, a, st);
  }
  return cudaErrorInvalidValue;
}

const void* fwd_kernel_ptr(int fmt, bool col) {
  switch (format_bits(fmt)) {
    case 8: return fwd_kernel_ptr_8(fmt, col);
    case 16: return fwd_kernel_ptr_16(fmt, col);
    case 32: return fwd_kernel_ptr_32(fmt, col);
  }
  return nullptr;
}

cudaError_t launch_fwd_col(int fmt, int grid, const FwdArgs& a, float2* Y, cudaStream_t st) {
  switch (format_bits(fmt)) {
    case 8: return launch_fwd_col_8(fmt, grid, a, Y, st);
    case 16: return launch_fwd_col_16(fmt, grid, a, Y, st);
    case 32: return launch_fwd_col_32(fmt, grid, a, Y, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_fwd_rows(int grid, const FwdArgs& a, const float2* Y, cudaStream_t st) {
  fwd_row_kernel<TILE_S, TILE_T><<<grid, TILE_T, TILE_SMEM, st>>>(a, Y);
  return cudaGetLastError();
}

const void* welch_kernel_ptr(bool cplx) {
  return cplx ? (const void*)welch_kernel<false> : (const void*)welch_kernel<true>;
}

cudaError_t launch_split(bool cplx, int B, const SplitArgs& s, cudaStream_t st) {
  const dim3 g((s.K + 255) / 256, B);
  if (cplx) welch_split_kernel<false><<<g, 256, 0, st>>>(s);
  else welch_split_kernel<true><<<g, 256, 0, st>>>(s);
  return cudaGetLastError();
}

cudaError_t launch_welch(bool cplx, const WelchArgs& w, cudaStream_t st) {
  constexpr int bins_per_cta = WELCH_WARP_BINS;
  const int g = (w.s.K + bins_per_cta - 1) / bins_per_cta;
  if (cplx) welch_kernel<false><<<g, 32 * WELCH_WARPS, 0, st>>>(w);
  else welch_kernel<true><<<g, 32 * WELCH_WARPS, 0, st>>>(w);
  return cudaGetLastError();
}

// Filter-bank tile shapes: 8192-point tiles with 256 threads (32 elements
// each, 2 CTAs per SM) or 512 threads (16 elements each, radix <= 16 stages,
// twice the warps per SM).
template <int T>
const void* fcfb_fn(bool cplx, bool persistent) {
  if (persistent) return cplx ? (const void*)fcfb_kernel<TILE_S, T, true, false> : (const void*)fcfb_kernel<TILE_S, T, true, true>;
  return cplx ? (const void*)fcfb_kernel<TILE_S, T, false, false> : (const void*)fcfb_kernel<TILE_S, T, false, true>;
}

const void* fcfb_kernel_ptr(int tile_threads, bool cplx, bool persistent) {
  return tile_threads == 512 ? fcfb_fn<512>(cplx, persistent) : fcfb_fn<TILE_T>(cplx, persistent);
}

cudaError_t fcfb_prepare() {
  const void* fns[] = {fcfb_fn<TILE_T>(true, true), fcfb_fn<TILE_T>(true, false), fcfb_fn<TILE_T>(false, true),
                       fcfb_fn<TILE_T>(false, false), fcfb_fn<512>(true, true), fcfb_fn<512>(true, false),
                       fcfb_fn<512>(false, true), fcfb_fn<512>(false, false),
                       (const void*)fcfb_backward_kernel<TILE_S, TILE_T, true>,
                       (const void*)fcfb_backward_kernel<TILE_S, TILE_T, false>,
                       (const void*)fwd_row_kernel<TILE_S, TILE_T>};
  for (const void* f : fns) {
    const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TILE_SMEM);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t fcfb_occupancy(int tile_threads, int* per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fcfb_kernel_ptr(tile_threads, false, true),
                                                       tile_threads, TILE_SMEM);
}

cudaError_t launch_fcfb(bool cplx, bool persistent, int tile_threads, int grid, const FcfbArgs& a, int tile_base,
                        cudaStream_t st) {
  FcfbArgs args = a;
  int base = tile_base;
  void* params[] = {(void*)&args, (void*)&base};
  return cudaLaunchKernel(fcfb_kernel_ptr(tile_threads, cplx, persistent), dim3(grid), dim3(tile_threads), params,
                          TILE_SMEM, st);
}

cudaError_t launch_fcfb_backward(bool cplx, int grid, const BwdArgs& a, cudaStream_t st) {
  if (cplx) fcfb_backward_kernel<TILE_S, TILE_T, false><<<grid, TILE_T, TILE_SMEM, st>>>(a);
  else fcfb_backward_kernel<TILE_S, TILE_T, true><<<grid, TILE_T, TILE_SMEM, st>>>(a);
  return cudaGetLastError();
}

}  // namespace sk
