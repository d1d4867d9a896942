// Forward-FFT kernel instances per input format; included by the
// sk_fwd_{8,16,32}.cu units, which split the formats by sample width so the
// instances compile in parallel.
#pragma once
#include "spektri_b200.h"
#include "sk_kernels.cuh"

namespace sk {

template <int FMT>
cudaError_t fwd_launch_one(int grid, const FwdArgs& a, cudaStream_t st) {
  fwd_fft_kernel<TILE_S, TILE_T, FMT><<<grid, TILE_T, TILE_SMEM, st>>>(a);
  return cudaGetLastError();
}

// The mixed-radix column kernel for R1 = 3, 5, 6, 10, 12.
template <int FMT>
const void* fwd_colmix_ptr(int R1) {
  switch (R1) {
    case 3: return (const void*)fwd_colmix_kernel<3, 1, FMT>;
    case 6: return (const void*)fwd_colmix_kernel<3, 2, FMT>;
    case 12: return (const void*)fwd_colmix_kernel<3, 4, FMT>;
    case 5: return (const void*)fwd_colmix_kernel<5, 1, FMT>;
    case 10: return (const void*)fwd_colmix_kernel<5, 2, FMT>;
  }
  return nullptr;
}

// Column pass: mixed radix for R1 not a power of two (one thread per
// column), registers for R1 <= 8 (one thread per column), shared-memory
// R1-point transforms above (grid = B * R1 tiles).
template <int FMT>
cudaError_t fwd_col_launch_one(int grid, const FwdArgs& a, float2* Y, cudaStream_t st) {
  if (a.log2R1 < 0) {
    const void* fn = fwd_colmix_ptr<FMT>(a.R1);
    if (!fn) return cudaErrorInvalidValue;
    const long long cols = (long long)a.B << a.logM;
    FwdArgs args = a;
    float2* y = Y;
    void* params[] = {(void*)&args, (void*)&y};
    return cudaLaunchKernel(fn, dim3((unsigned)((cols + 255) / 256)), dim3(256), params, 0, st);
  }
  if (a.log2R1 <= 3) {
    const long long cols = (long long)a.B << TILE_LOGS;
    fwd_colreg_kernel<FMT><<<(unsigned)((cols + 255) / 256), 256, 0, st>>>(a, Y);
  } else {
    fwd_col_kernel<TILE_S, TILE_T16, FMT><<<grid, TILE_T16, TILE_SMEM_COL, st>>>(a, Y);
  }
  return cudaGetLastError();
}

template <int FMT>
cudaError_t fwd_prepare_one() {
  cudaError_t e = cudaFuncSetAttribute(fwd_fft_kernel<TILE_S, TILE_T, FMT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TILE_SMEM);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(fwd_col_kernel<TILE_S, TILE_T16, FMT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)TILE_SMEM_COL);
}

// kind 0: single-pass kernel; 1: shared-memory column pass; 2: register column
// pass; 3: mixed-radix column pass (R1 = 3, 5, 6, 10, 12).
template <int FMT>
const void* fwd_ptr_one(int kind, int R1) {
  if (kind == 3) return fwd_colmix_ptr<FMT>(R1);
  if (kind == 2) return (const void*)fwd_colreg_kernel<FMT>;
  return kind ? (const void*)fwd_col_kernel<TILE_S, TILE_T16, FMT> : (const void*)fwd_fft_kernel<TILE_S, TILE_T, FMT>;
}

}  // namespace sk
