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

const void* fwd_kernel_ptr(int fmt, int kind, int R1) {
  switch (format_bits(fmt)) {
    case 8: return fwd_kernel_ptr_8(fmt, kind, R1);
    case 16: return fwd_kernel_ptr_16(fmt, kind, R1);
    case 32: return fwd_kernel_ptr_32(fmt, kind, R1);
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

cudaError_t launch_kernel(const void* fn, dim3 grid, dim3 block, void** params, size_t smem, cudaStream_t st,
                          bool pdl) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelExC(&cfg, fn, params);
}

cudaError_t launch_fwd_rows(int grid, const FwdArgs& a, const float2* Y, cudaStream_t st, bool pdl) {
  FwdArgs args = a;
  const float2* y = Y;
  void* params[] = {(void*)&args, (void*)&y};
  const bool mix = a.log2R1 < 0;
  const void* fn = mix ? (const void*)fwd_rowmix_kernel<TILE_S, TILE_T> : (const void*)fwd_row_kernel<TILE_T16>;
  return launch_kernel(fn, dim3(grid), dim3(mix ? TILE_T : TILE_T16), params, TILE_SMEM, st, pdl);
}

// Up to WELCH_BINS_MAX_B blocks per buffer each warp walks its own bins over
// all blocks; above that the warps of a CTA split the blocks.
template <bool P2>
const void* welch_ptr_t(bool cplx, int B) {
  if (B <= WELCH_BINS_MAX_B)
    return cplx ? (const void*)welch_bins_kernel<false, P2> : (const void*)welch_bins_kernel<true, P2>;
  return cplx ? (const void*)welch_kernel<false, P2> : (const void*)welch_kernel<true, P2>;
}
// Complex spectra of the power-of-two two-pass FFT with R1 >= 16 rows per
// block: the transposing kernel (its reads of the residue layout coalesce).
bool welch_transposed(bool cplx, bool pow2, int R1) { return cplx && pow2 && R1 >= 16; }
const void* welch_kernel_ptr(bool cplx, int B, bool pow2, int R1) {
  if (welch_transposed(cplx, pow2, R1)) return (const void*)welch_tr_kernel<256>;
  return pow2 ? welch_ptr_t<true>(cplx, B) : welch_ptr_t<false>(cplx, B);
}

cudaError_t launch_split(bool cplx, int B, const SplitArgs& s, cudaStream_t st) {
  const dim3 g((s.K + 255) / 256, B);
  const bool p2 = (s.N & (s.N - 1)) == 0;
  if (cplx) {
    if (p2) welch_split_kernel<false, true><<<g, 256, 0, st>>>(s);
    else welch_split_kernel<false, false><<<g, 256, 0, st>>>(s);
  } else {
    if (p2) welch_split_kernel<true, true><<<g, 256, 0, st>>>(s);
    else welch_split_kernel<true, false><<<g, 256, 0, st>>>(s);
  }
  return cudaGetLastError();
}

cudaError_t launch_extend(bool cplx, int B, const float2* X, int K, int N, float2* Xe, long long xs, int maxn,
                          cudaStream_t st) {
  const dim3 g((K + 255) / 256, B);
  if (cplx) extend_kernel<false><<<g, 256, 0, st>>>(X, K, N, Xe, xs, maxn);
  else extend_kernel<true><<<g, 256, 0, st>>>(X, K, N, Xe, xs, maxn);
  return cudaGetLastError();
}

cudaError_t launch_welch(bool cplx, const WelchArgs& w, cudaStream_t st, bool pdl) {
  const bool pow2 = (w.s.N & (w.s.N - 1)) == 0;
  WelchArgs args = w;
  void* params[] = {(void*)&args};
  if (welch_transposed(cplx, pow2, w.s.R1))
    return launch_kernel(welch_kernel_ptr(cplx, w.B, pow2, w.s.R1), dim3(w.s.K / WT_BINS), dim3(256), params, 0, st,
                         pdl);
  const int bins_per_cta = w.B <= WELCH_BINS_MAX_B ? WELCH_WARP_BINS * WELCH_WARPS : WELCH_WARP_BINS;
  const int g = (w.s.K + bins_per_cta - 1) / bins_per_cta;
  return launch_kernel(welch_kernel_ptr(cplx, w.B, pow2, w.s.R1), dim3(g), dim3(32 * WELCH_WARPS), params, 0, st,
                       pdl);
}

// Filter-bank tile shapes (tile size x threads, minimum CTAs per SM):
// 8192 x 256 (32 elements per thread, 2 CTAs/SM), 8192 x 512 (16 elements,
// radix <= 16 stages, 2 CTAs/SM), 4096 x 256 (16 elements, n = 8192 as two
// independent halves, 4 CTAs/SM).
// The instances live in sk_fcfb_<shape>[_chirp].cu, compiled in parallel.

bool fcfb_shape_ok(int tile_size, int tile_threads) {
  return (tile_size == 8192 && (tile_threads == 256 || tile_threads == 512)) ||
         (tile_size == 4096 && tile_threads == 256);
}

const void* fcfb_kernel_ptr(int tile_size, int tile_threads, bool persistent, bool chirp) {
  if (tile_size == 4096) return chirp ? fcfb_ptr_4096_chirp(persistent) : fcfb_ptr_4096(persistent);
  if (tile_threads == 512) return chirp ? fcfb_ptr_8192x512_chirp(persistent) : fcfb_ptr_8192x512(persistent);
  return chirp ? fcfb_ptr_8192_chirp(persistent) : fcfb_ptr_8192(persistent);
}

cudaError_t fcfb_prepare() {
  const int shapes[][2] = {{8192, 256}, {8192, 512}, {4096, 256}};
  for (const auto& sh : shapes)
    for (int k = 0; k < 4; ++k) {
      const cudaError_t e = cudaFuncSetAttribute(fcfb_kernel_ptr(sh[0], sh[1], k & 1, k & 2),
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fcfb_smem(sh[0]));
      if (e != cudaSuccess) return e;
    }
  {
    const cudaError_t e = cudaFuncSetAttribute(fcfb_ptr_16384_chirp(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)fcfb_smem(1 << CHIRP_LOGM_MAX));
    if (e != cudaSuccess) return e;
  }
  const void* fns[] = {(const void*)fcfb_bwd_fft_kernel<TILE_S, TILE_T>,
                       (const void*)fwd_row_kernel<TILE_T16>, (const void*)fwd_rowmix_kernel<TILE_S, TILE_T>};
  for (const void* f : fns) {
    const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TILE_SMEM);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_fcfb_chirp16k(int grid, const FcfbArgs& a, int tile_base, cudaStream_t st) {
  FcfbArgs args = a;
  int base = tile_base;
  void* params[] = {(void*)&args, (void*)&base};
  return launch_kernel(fcfb_ptr_16384_chirp(), dim3(grid), dim3(1024), params, fcfb_smem(1 << CHIRP_LOGM_MAX), st,
                       false);
}

cudaError_t fcfb_occupancy(int tile_size, int tile_threads, int* per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fcfb_kernel_ptr(tile_size, tile_threads, true, false),
                                                       tile_threads, fcfb_smem(tile_size));
}

cudaError_t launch_fcfb(bool persistent, bool chirp, int tile_size, int tile_threads, int grid, const FcfbArgs& a,
                        int tile_base, cudaStream_t st, bool pdl) {
  FcfbArgs args = a;
  int base = tile_base;
  void* params[] = {(void*)&args, (void*)&base};
  return launch_kernel(fcfb_kernel_ptr(tile_size, tile_threads, persistent, chirp), dim3(grid), dim3(tile_threads),
                       params, fcfb_smem(tile_size), st, pdl);
}

cudaError_t launch_fcfb_backward(bool cplx, int grid, int max_n, const BwdArgs& a, cudaStream_t st) {
  fcfb_bwd_fft_kernel<TILE_S, TILE_T><<<grid, TILE_T, TILE_SMEM, st>>>(a);
  const dim3 gw((max_n + 255) / 256, a.nchan);
  if (cplx) fcfb_bwd_dw_kernel<false><<<gw, 256, 0, st>>>(a);
  else fcfb_bwd_dw_kernel<true><<<gw, 256, 0, st>>>(a);
  if (a.dX) fcfb_bwd_dx_kernel<0><<<dim3((a.K + 255) / 256, a.B), 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace sk
