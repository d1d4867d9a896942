// Device kernels of the filter-bank + Welch path.
//
// Per input buffer of B overlapped blocks (block b = samples [b*hop, b*hop+N)
// of [N/4 carried samples | 3N/4*B new samples], main.rs:162-181, dsp.rs:150-155):
//   fwd_fft_kernel       raw samples -> converted, scaled by scaling/N, forward
//                        FFT of size Nc (N/2 complex pairs for real input, N for
//                        complex) -> Z, whole blocks per tile (Nc <= 8192)  [multifft.rs]
//   fwd_colreg_kernel /  two-pass forward FFT for Nc = R1 * 8192: column pass
//   fwd_col_kernel       (registers for R1 <= 8, shared memory above) -> Y,
//   + fwd_row_kernel     then 8192-point rows -> Z in residue layout
//   welch_kernel /       Z -> X (K bins, real-input split) written as extended
//   welch_bins_kernel    rows for the filter bank, the Welch term
//                        |X[k] - (X[k-1]+X[k+1])/2|^2, its f32 accumulation in
//                        block order, emission and quantisation of records [spectrum.rs:82-163]
//   welch_split_kernel   Z -> X only, [B][K] (the differentiable stage, the allocation-free entry)
//   extend_kernel        [B][K] -> extended rows (the differentiable stage's filter bank)
//   fcfb_kernel          per channel and block: n contiguous bins of the extended row
//                        (get_bin's modulo and mirror already applied), times weights,
//                        inverse FFT, keep [n/8, 7n/8)                       [fcfb.rs:154-188]
//   fcfb_bwd_*_kernel    adjoint of fcfb_kernel for weight design (FFT of the output
//                        gradients, dW and dX sums in a fixed order)
#pragma once
#include "sk_types.h"
#include "sk_fft.cuh"
#include "sk_fcfb.cuh"
#include "sk_fcfb_ip.cuh"

namespace sk {

// Programmatic dependent launch.  In the batched graph the row pass, the Welch
// kernel and the filter bank are launched with programmatic stream
// serialization: their CTAs launch as soon as every CTA of the kernel ahead of
// them has exited (no early trigger: dependents that became resident early
// slowed the kernel they waited on), do what does not depend on it (tile
// claims, metadata) while that kernel's grid completes, and block in
// pdl_wait() until its writes are visible.  A no-op for a kernel launched
// without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// The first forward kernel of a batched call zeroes the filter bank's tile
// cursors (the previous call's filter bank has completed: graph launches are
// serialised).
__device__ __forceinline__ void reset_cursors(int* cursor) {
  if (cursor && blockIdx.x == 0 && threadIdx.x == 0) {
    cursor[0] = 0;
    cursor[1] = 0;
  }
}

// Stage trace (sk_types.h TRACE_SLOTS): one thread per CTA folds the global
// timer into a slot with an atomic min (stage start) or max (stage end).
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Only the first (start) or last (end) TRACE_EDGE CTAs of a grid record, so a
// kernel of thousands of CTAs adds a few hundred atomics, not thousands; CTAs
// are dispatched in index order, so the first to start and the last to end
// are among them.  No barrier: the recording thread stamps its own start or
// end.
constexpr int TRACE_EDGE = 512;
__device__ __forceinline__ void trace_start(unsigned long long* trace, int slot) {
  if (trace && threadIdx.x == 0 && blockIdx.x < TRACE_EDGE) atomicMin(trace + slot, global_ns());
}
__device__ __forceinline__ void trace_end(unsigned long long* trace, int slot) {
  if (trace && threadIdx.x == 0 && blockIdx.x + TRACE_EDGE >= gridDim.x) atomicMax(trace + slot, global_ns());
}

// ----------------------------------------------------------------- input formats
// One scalar component of a raw sample (inputformats.rs:65-155).  BASE is the
// format code without its complex bit.
template <int BASE>
__device__ __forceinline__ float load_comp(const uint8_t* __restrict__ p, long long ci) {
  if constexpr (BASE == 0x04) {
    return (float)(signed char)__ldg(reinterpret_cast<const signed char*>(p) + ci);
  } else if constexpr (BASE == 0x08) {
    return (float)__ldg(reinterpret_cast<const short*>(p) + ci);
  } else if constexpr (BASE == 0x09) {
    unsigned short u = __ldg(reinterpret_cast<const unsigned short*>(p) + ci);
    return (float)(short)(unsigned short)((u >> 8) | (u << 8));
  } else if constexpr (BASE == 0x1C) {
    return __ldg(reinterpret_cast<const float*>(p) + ci);
  } else if constexpr (BASE == 0x1D) {
    unsigned u = __ldg(reinterpret_cast<const unsigned*>(p) + ci);
    return __uint_as_float(__byte_perm(u, 0, 0x0123));
  } else {  // 0x24: u8 with the reference's -127.4 offset
    return (float)__ldg(p + ci) - 127.4f;
  }
}

// Sample source over [halo (converted, N/4 samples) | raw new samples].
// pair(p): real input -> (x[p], x[p+1]) for even p; complex -> sample p.
template <int FMT>
struct SampleSrc {
  const uint8_t* raw;
  const float* halo;
  long long overlap;
  // Component loads stay scalar: measured on B200, one 32-bit load per s16le
  // pair made the forward kernel 1.5x slower than two 16-bit loads.
  __device__ __forceinline__ float2 pair(long long p) const {
    constexpr int BASE = FMT & 0x3F;
    constexpr bool CPLX = (FMT & 0xC0) == 0x40;
    if (p < overlap) return *reinterpret_cast<const float2*>(halo + (CPLX ? 2 * p : p));
    const long long c = CPLX ? 2 * (p - overlap) : p - overlap;   // first component index
    return make_float2(load_comp<BASE>(raw, c), load_comp<BASE>(raw, c + 1));
  }
};

// ----------------------------------------------------------------- forward FFT

// Tile = S/Nc whole blocks (Nc <= S), or one residue class k1 of one block
// (Nc = R1*S): z'[j2] = W_Nc^{j2 k1} sum_j1 z[j1 S + j2] W_R1^{j1 k1}, whose
// S-point DFT is Z[k1 + R1 k2] (the last radix-R1 stage done first, as
// prototyping/parallel_fft.py:20-28 splits a 4-way FFT).
// Whole blocks: S/Nc blocks per tile, Nc = 2^LOGN.
template <int LOGN, int S, int T, int FMT>
__device__ __forceinline__ void fwd_tile_blocks(float2* sm, const FwdArgs& a, const SampleSrc<FMT>& src, int tile) {
  constexpr bool CPLX = (FMT & 0xC0) == 0x40;
  const int per = a.per > 0 ? a.per : S >> LOGN;
  const int b0 = tile * per;
  const int count = min(per, a.B - b0);
  using P = StagePlan<LOGN, S / T>;
  auto load = [&](int t, int q, int s) {
    const int j = q + (s << P::first_shift);
    float2 z = src.pair((long long)(b0 + t) * a.hop + (CPLX ? j : 2 * j));   // x * scaling/N
    return make_float2(z.x * a.wscale, z.y * a.wscale);
  };
  auto store = [&](int t, int q, int u, float2 v) { a.Z[((size_t)(b0 + t) << LOGN) + q + (u << P::last_shift)] = v; };
  tile_pipeline<LOGN, S, T, -1, false>(sm, count, a.tw_tile, load, store);
}

// One residue class k1 of one block (Nc = R1 S): element j2 of the tile is
// W_Nc^{j2 k1} sum_j1 z[j1 S + j2] W_R1^{j1 k1}.
template <int LOGR1, int S, int T, int FMT>
__device__ __forceinline__ void fwd_tile_split(float2* sm, const FwdArgs& a, const SampleSrc<FMT>& src, int tile) {
  constexpr bool CPLX = (FMT & 0xC0) == 0x40;
  constexpr int R1 = 1 << LOGR1, LOGS = ilog2c(S);
  const int b = tile >> LOGR1, k1 = tile & (R1 - 1);
  const int shR = a.log2N - LOGR1, shC = a.log2N - (LOGS + LOGR1);
  const long long p0 = (long long)b * a.hop;
  float2* Zb = a.Z + ((size_t)b << (LOGS + LOGR1)) + ((size_t)k1 << LOGS);
  float2 rot[R1];                                    // W_R1^{j1 k1}: fixed for the tile
#pragma unroll
  for (int j1 = 0; j1 < R1; ++j1) rot[j1] = __ldg(&a.tw_big[((j1 * k1) & (R1 - 1)) << shR]);
  using P = StagePlan<LOGS, S / T>;
  auto load = [&](int, int q, int s) {
    const int e = q + (s << P::first_shift);
    float2 z[R1];
#pragma unroll
    for (int j1 = 0; j1 < R1; ++j1) {
      const int jj = (j1 << LOGS) + e;
      z[j1] = src.pair(p0 + (CPLX ? jj : 2 * jj));
    }
    float2 acc = make_float2(z[0].x * a.wscale, z[0].y * a.wscale);
#pragma unroll
    for (int j1 = 1; j1 < R1; ++j1)
      acc = cadd(acc, cmul(make_float2(z[j1].x * a.wscale, z[j1].y * a.wscale), rot[j1]));
    if (k1) acc = cmul(acc, __ldg(&a.tw_big[(e * k1) << shC]));
    return acc;
  };
  auto store = [&](int, int q, int u, float2 v) { Zb[q + (u << P::last_shift)] = v; };
  tile_pipeline<LOGS, S, T, -1, false>(sm, 1, a.tw_tile, load, store);
}

template <int S, int T, int FMT>
__global__ void __launch_bounds__(T, 2) fwd_fft_kernel(FwdArgs a) {
  extern __shared__ float2 sm[];
  constexpr bool CPLX = (FMT & 0xC0) == 0x40;
  trace_start(a.trace, 0);
  reset_cursors(a.cursor);
  const SampleSrc<FMT> src{a.raw, a.halo, a.overlap};
  {  // carry: convert the last N/4 new samples for the next buffer (main.rs:173)
    const long long stride = (long long)gridDim.x * T;
    const long long ncomp = a.overlap * (CPLX ? 2 : 1);
    const long long base = (a.nnew - a.overlap) * (CPLX ? 2 : 1);
    for (long long h = (long long)blockIdx.x * T + threadIdx.x; h < ncomp; h += stride)
      a.halo_next[h] = load_comp<FMT & 0x3F>(a.raw, base + h);
  }
  const int tile = blockIdx.x;
  if (a.R1 == 1) {
    switch (a.log2Nc) {
      case 2: fwd_tile_blocks<2, S, T, FMT>(sm, a, src, tile); break;
      case 3: fwd_tile_blocks<3, S, T, FMT>(sm, a, src, tile); break;
      case 4: fwd_tile_blocks<4, S, T, FMT>(sm, a, src, tile); break;
      case 5: fwd_tile_blocks<5, S, T, FMT>(sm, a, src, tile); break;
      case 6: fwd_tile_blocks<6, S, T, FMT>(sm, a, src, tile); break;
      case 7: fwd_tile_blocks<7, S, T, FMT>(sm, a, src, tile); break;
      case 8: fwd_tile_blocks<8, S, T, FMT>(sm, a, src, tile); break;
      case 9: fwd_tile_blocks<9, S, T, FMT>(sm, a, src, tile); break;
      case 10: fwd_tile_blocks<10, S, T, FMT>(sm, a, src, tile); break;
      case 11: fwd_tile_blocks<11, S, T, FMT>(sm, a, src, tile); break;
      case 12: fwd_tile_blocks<12, S, T, FMT>(sm, a, src, tile); break;
      case 13: fwd_tile_blocks<13, S, T, FMT>(sm, a, src, tile); break;
    }
  } else {
    switch (a.log2R1) {
      case 1: fwd_tile_split<1, S, T, FMT>(sm, a, src, tile); break;
      case 2: fwd_tile_split<2, S, T, FMT>(sm, a, src, tile); break;
      case 3: fwd_tile_split<3, S, T, FMT>(sm, a, src, tile); break;
    }
  }
  trace_end(a.trace, 1);
}

// Two-pass forward FFT for Nc = R1 * S with R1 >= 16 (Nc up to 2^21).
// Pass A (columns): a tile holds C = S/R1 consecutive columns j2 of one block
// and computes Y[k1][j2] = W_Nc^{j2 k1} sum_j1 z[j1 S + j2] W_R1^{j1 k1} as
// two decimation-in-time stages: radix 16 straight from the samples (thread
// (col, q) loads z[(q + (R1/16) s) S + c0 + col], s < 16: lanes along
// consecutive columns, so every load is coalesced), its outputs down the
// column in shared memory (column stride R1 + 1, odd: conflict-free), then
// radix R1/16 on span 16 whose outputs k1 = j + 16 u go straight to Y (lanes
// along columns again, coalesced stores).  Shared memory is touched once each
// way per element (R1 = 16 needs none).
// Pass B (rows): S-point FFT of row k1 of Y gives Z[k1 + R1 k2], stored at
// k1 S + k2 — the residue layout the spectrum split reads.
template <int LOGR1, int T, int FMT>
__device__ __forceinline__ void fwd_col_tile(float2* sm, const FwdArgs& a, const SampleSrc<FMT>& src, float2* Y) {
  constexpr bool CPLX = (FMT & 0xC0) == 0x40;
  constexpr int LOGS = TILE_LOGS, R1 = 1 << LOGR1, LOGC = LOGS - LOGR1, C = 1 << LOGC;
  constexpr int LOGRB = LOGR1 - 4, RB = 1 << LOGRB, ROW = R1 + 1;
  static_assert(C * (R1 / 16) == T, "one radix-16 butterfly per thread");
  const int b = blockIdx.x >> LOGR1;
  const int c0 = (blockIdx.x & (R1 - 1)) << LOGC;
  const long long p0 = (long long)b * a.hop;
  const int shC = a.log2N - a.log2Nc;
  float2* Yb = Y + ((size_t)b << a.log2Nc) + c0;
  const int col = threadIdx.x & (C - 1), q = threadIdx.x >> LOGC;
  float2 v[16];
#pragma unroll
  for (int s = 0; s < 16; ++s) {
    const int jj = ((q + (s << LOGRB)) << LOGS) + c0 + col;
    const float2 z = src.pair(p0 + (CPLX ? jj : 2 * jj));
    v[s] = make_float2(z.x * a.wscale, z.y * a.wscale);
  }
  dft<16, -1>(v);
  if constexpr (RB == 1) {                                  // R1 = 16: k1 = u
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const float2 t = u ? cmul(v[u], __ldg(&a.tw_big[((c0 + col) * u) << shC])) : v[u];
      Yb[((size_t)u << LOGS) + col] = t;
    }
  } else {
    float2* p = sm + col * ROW + q * 16;                     // Stockham: y[q 16 + u]
#pragma unroll
    for (int u = 0; u < 16; ++u) p[u] = v[u];
    __syncthreads();
    constexpr int NB = 16 * C / T;                           // radix-RB butterflies per thread
    static_assert(C <= T, "a thread's butterflies share one column");
    // Output k1 = j + 16 u of column j2 = c0 + cl takes W_Nc^(j2 k1) =
    // W_Nc^(j2 j) (w16)^u, w16 = W_Nc^(16 j2): one gathered table read per
    // butterfly, the powers of w16 from w16 and w16^4 (as TwiddlePowers does)
    const int cl = threadIdx.x & (C - 1), j2 = c0 + cl;
    float2 pw[4] = {make_float2(1.f, 0.f), __ldg(&a.tw_big[(16 * j2) << shC]), {}, {}};
    pw[2] = cmul(pw[1], pw[1]);
    pw[3] = cmul(pw[2], pw[1]);
    float2 m[4] = {make_float2(1.f, 0.f), {}, {}, {}};
    if constexpr (RB > 4) {
      m[1] = __ldg(&a.tw_big[(64 * j2) << shC]);
      m[2] = cmul(m[1], m[1]);
      m[3] = cmul(m[2], m[1]);
    }
#pragma unroll
    for (int bb = 0; bb < NB; ++bb) {
      const int j = (threadIdx.x + bb * T) >> LOGC;          // span-16 index
      const float2* r = sm + cl * ROW + j;
      float2 w[RB];
#pragma unroll
      for (int s = 0; s < RB; ++s) w[s] = r[16 * s];
      twiddle_dft<RB, TILE_LOGS - LOGR1, -1>(w, a.tw_tile, j);   // W_R1^(j s), span 16
      const float2 base = __ldg(&a.tw_big[(j2 * j) << shC]);
#pragma unroll
      for (int u = 0; u < RB; ++u) {
        const int k1 = j + 16 * u;
        float2 tw = (u & 3) ? pw[u & 3] : m[u >> 2];
        if ((u & 3) && (u >> 2)) tw = cmul(tw, m[u >> 2]);
        tw = u ? cmul(base, tw) : base;
        Yb[((size_t)k1 << LOGS) + cl] = k1 ? cmul(w[u], tw) : w[u];
      }
    }
  }
}

template <int S, int T, int FMT>
__global__ void __launch_bounds__(T, 2) fwd_col_kernel(FwdArgs a, float2* Y) {   // T = 512
  extern __shared__ float2 sm[];
  constexpr bool CPLX = (FMT & 0xC0) == 0x40;
  static_assert(S == TILE_S && T == 512, "8192-point column tiles of 512 threads");
  trace_start(a.trace, 0);
  reset_cursors(a.cursor);
  const SampleSrc<FMT> src{a.raw, a.halo, a.overlap};
  {  // carry, as in fwd_fft_kernel
    const long long stride = (long long)gridDim.x * T;
    const long long ncomp = a.overlap * (CPLX ? 2 : 1);
    const long long base = (a.nnew - a.overlap) * (CPLX ? 2 : 1);
    for (long long h = (long long)blockIdx.x * T + threadIdx.x; h < ncomp; h += stride)
      a.halo_next[h] = load_comp<FMT & 0x3F>(a.raw, base + h);
  }
  switch (a.log2R1) {
    case 4: fwd_col_tile<4, T, FMT>(sm, a, src, Y); break;
    case 5: fwd_col_tile<5, T, FMT>(sm, a, src, Y); break;
    case 6: fwd_col_tile<6, T, FMT>(sm, a, src, Y); break;
    case 7: fwd_col_tile<7, T, FMT>(sm, a, src, Y); break;
    case 8: fwd_col_tile<8, T, FMT>(sm, a, src, Y); break;
  }
}

// Column pass for R1 = 2..8 (Nc = 16384..65536): one thread per column j2 of
// one block, the R1-point DFT in registers, no shared memory; the same Y as
// fwd_col_kernel.  Consecutive threads take consecutive columns, so every
// load of row j1 and every store of row k1 is coalesced.
template <int LOGR1, int FMT>
__device__ __forceinline__ void fwd_cols_reg(const FwdArgs& a, const SampleSrc<FMT>& src, float2* Y, long long g) {
  constexpr bool CPLX = (FMT & 0xC0) == 0x40;
  constexpr int R1 = 1 << LOGR1, LOGS = TILE_LOGS;
  const int b = (int)(g >> LOGS), j2 = (int)(g & ((1 << LOGS) - 1));
  const long long p0 = (long long)b * a.hop;
  float2 z[R1];
#pragma unroll
  for (int j1 = 0; j1 < R1; ++j1) {
    const int jj = (j1 << LOGS) + j2;
    const float2 v = src.pair(p0 + (CPLX ? jj : 2 * jj));
    z[j1] = make_float2(v.x * a.wscale, v.y * a.wscale);
  }
  dft<R1, -1>(z);
  const int shC = a.log2N - a.log2Nc;
  float2* Yb = Y + ((size_t)b << a.log2Nc) + j2;
  Yb[0] = z[0];
#pragma unroll
  for (int k1 = 1; k1 < R1; ++k1) Yb[(size_t)k1 << LOGS] = cmul(z[k1], __ldg(&a.tw_big[(j2 * k1) << shC]));
}

template <int FMT>
__global__ void __launch_bounds__(256) fwd_colreg_kernel(FwdArgs a, float2* Y) {
  constexpr bool CPLX = (FMT & 0xC0) == 0x40;
  trace_start(a.trace, 0);
  reset_cursors(a.cursor);
  const SampleSrc<FMT> src{a.raw, a.halo, a.overlap};
  {  // carry, as in fwd_fft_kernel
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long ncomp = a.overlap * (CPLX ? 2 : 1);
    const long long base = (a.nnew - a.overlap) * (CPLX ? 2 : 1);
    for (long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x; h < ncomp; h += stride)
      a.halo_next[h] = load_comp<FMT & 0x3F>(a.raw, base + h);
  }
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ((long long)a.B << TILE_LOGS)) return;
  switch (a.log2R1) {
    case 1: fwd_cols_reg<1, FMT>(a, src, Y, g); break;
    case 2: fwd_cols_reg<2, FMT>(a, src, Y, g); break;
    case 3: fwd_cols_reg<3, FMT>(a, src, Y, g); break;
  }
}

// Mixed-radix column pass, for the forward sizes that are not powers of two
// (the reference plans any size, multifft.rs:25-30): Nc = R1 M with
// R1 = R0 P (R0 = 3 or 5, P = 1, 2, 4) and M = 2^logM <= 8192.  One thread
// per column j2 < M of one block: the R1-point DFT of z[j1 M + j2] (j1 < R1)
// in registers, output k1 times W_Nc^(j2 k1), into row k1 of the block's Y
// (Y[(b R1 + k1) M + j2]); the row pass then gives Z[k1 + R1 k2] at
// (b R1 + k1) M + k2, the same residue layout as the power-of-two split.
//
// R-point DFT, R = R0 P, by Cooley-Tukey with input j = j0 P + j1 and output
// k = k0 + R0 k1:  X[k0 + R0 k1] = sum_j1 W_P^(j1 k1) W_R^(j1 k0)
// sum_j0 z[j0 P + j1] W_R0^(j0 k0): direct R0-point sums, twiddles, then the
// radix-2 Dft<P> per k0.  w[m] = W_R^m (forward sign) for m < R.
template <int R0, int P>
__device__ __forceinline__ void mixed_dft(float2* z, const float2* w) {
  constexpr int R = R0 * P;
  float2 t[R];
#pragma unroll
  for (int j1 = 0; j1 < P; ++j1) {
#pragma unroll
    for (int k0 = 0; k0 < R0; ++k0) {
      float2 acc = z[j1];
#pragma unroll
      for (int j0 = 1; j0 < R0; ++j0) {
        const float2 tw = w[((j0 * k0) % R0) * P];          // W_R0^(j0 k0) = W_R^(j0 k0 P)
        acc = k0 ? cadd(acc, cmul(z[j0 * P + j1], tw)) : cadd(acc, z[j0 * P + j1]);
      }
      t[k0 * P + j1] = (j1 && k0) ? cmul(acc, w[(j1 * k0) % R]) : acc;
    }
  }
#pragma unroll
  for (int k0 = 0; k0 < R0; ++k0) {
    dft<P, -1>(t + k0 * P);
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) z[k0 + R0 * k1] = t[k0 * P + k1];
  }
}

template <int R0, int P, int FMT>
__global__ void __launch_bounds__(256) fwd_colmix_kernel(FwdArgs a, float2* Y) {
  constexpr bool CPLX = (FMT & 0xC0) == 0x40;
  constexpr int R1 = R0 * P;
  trace_start(a.trace, 0);
  reset_cursors(a.cursor);
  const SampleSrc<FMT> src{a.raw, a.halo, a.overlap};
  {  // carry, as in fwd_fft_kernel
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long ncomp = a.overlap * (CPLX ? 2 : 1);
    const long long base = (a.nnew - a.overlap) * (CPLX ? 2 : 1);
    for (long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x; h < ncomp; h += stride)
      a.halo_next[h] = load_comp<FMT & 0x3F>(a.raw, base + h);
  }
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ((long long)a.B << a.logM)) return;
  const int M = 1 << a.logM;
  const int b = (int)(g >> a.logM), j2 = (int)(g & (M - 1));
  const long long p0 = (long long)b * a.hop;
  float2 w[R1];
  const int nr = a.N / R1;                                   // W_R1^m = W_N^(m N/R1)
#pragma unroll
  for (int m = 0; m < R1; ++m) w[m] = __ldg(&a.tw_big[m * nr]);
  float2 z[R1];
#pragma unroll
  for (int j1 = 0; j1 < R1; ++j1) {
    const int jj = j1 * M + j2;
    const float2 v = src.pair(p0 + (CPLX ? jj : 2 * jj));
    z[j1] = make_float2(v.x * a.wscale, v.y * a.wscale);
  }
  mixed_dft<R0, P>(z, w);
  const int step = a.N / a.Nc;                               // W_Nc^k = W_N^(k N/Nc)
  float2* Yb = Y + (size_t)b * R1 * M + j2;
  Yb[0] = z[0];
#pragma unroll
  for (int k1 = 1; k1 < R1; ++k1) Yb[(size_t)k1 * M] = cmul(z[k1], __ldg(&a.tw_big[j2 * k1 * step]));
}

// Row pass: the M-point FFT of every row of Y (row r = b R1 + k1 at r M),
// S/M rows per tile, into Z at the same place (the residue layout).
template <int LOGM, int S, int T>
__device__ __forceinline__ void fwd_rows_tile(float2* sm, const FwdArgs& a, const float2* Y, int tile) {
  constexpr int rpt = S >> LOGM;
  const int r0 = tile * rpt, count = min(rpt, a.B * a.R1 - r0);
  const float2* Yr = Y + ((size_t)r0 << LOGM);
  float2* Zr = a.Z + ((size_t)r0 << LOGM);
  using P = StagePlan<LOGM, S / T>;
  auto load = [&](int t, int q, int s) { return __ldg(&Yr[((size_t)t << LOGM) + q + (s << P::first_shift)]); };
  auto store = [&](int t, int q, int u, float2 v) { Zr[((size_t)t << LOGM) + q + (u << P::last_shift)] = v; };
  tile_pipeline<LOGM, S, T, -1, false>(sm, count, a.tw_tile, load, store);
}

// Rows of 8192 points (the power-of-two two-pass FFT): one row per tile, on
// the in-place 16-16-16-2 pipeline with 512 threads (16 elements each, two
// CTAs per SM at 64 registers).
template <int T>
__global__ void __launch_bounds__(T, 2) fwd_row_kernel(FwdArgs a, const float2* Y) {
  extern __shared__ float2 sm[];
  pdl_wait();                                               // Y from the column pass
  const float2* Yr = Y + ((size_t)blockIdx.x << TILE_LOGS);
  float2* Zr = a.Z + ((size_t)blockIdx.x << TILE_LOGS);
  auto load = [&](int, int q, int s) { return __ldg(&Yr[q + (s << 9)]); };
  auto store = [&](int, int kk, int u, float2 v) { Zr[kk + (u << 12)] = v; };
  ip_pipeline_8k<T, -1>(sm, a.tw_tile, load, store);
  trace_end(a.trace, 1);
}

// ... and rows of M = 2^logM points, S/M per tile (the mixed-radix FFT).
template <int S, int T>
__global__ void __launch_bounds__(T, 2) fwd_rowmix_kernel(FwdArgs a, const float2* Y) {
  extern __shared__ float2 sm[];
  pdl_wait();
  switch (a.logM) {
    case 4: fwd_rows_tile<4, S, T>(sm, a, Y, blockIdx.x); break;
    case 5: fwd_rows_tile<5, S, T>(sm, a, Y, blockIdx.x); break;
    case 6: fwd_rows_tile<6, S, T>(sm, a, Y, blockIdx.x); break;
    case 7: fwd_rows_tile<7, S, T>(sm, a, Y, blockIdx.x); break;
    case 8: fwd_rows_tile<8, S, T>(sm, a, Y, blockIdx.x); break;
    case 9: fwd_rows_tile<9, S, T>(sm, a, Y, blockIdx.x); break;
    case 10: fwd_rows_tile<10, S, T>(sm, a, Y, blockIdx.x); break;
    case 11: fwd_rows_tile<11, S, T>(sm, a, Y, blockIdx.x); break;
    case 12: fwd_rows_tile<12, S, T>(sm, a, Y, blockIdx.x); break;
    case 13: fwd_rows_tile<13, S, T>(sm, a, Y, blockIdx.x); break;
  }
  trace_end(a.trace, 1);
}

// ----------------------------------------------------------------- Welch split

// Packed spectrum element m (the residue layout for R1 > 1).  POW2: N (so Nc
// and R1) is a power of two: masks and shifts; else R1 = 3, 5, 6, 10, 12 and
// divisions.  Kernels are instantiated for both, so the power-of-two sizes
// pay nothing for the others.
template <bool POW2>
__device__ __forceinline__ int z_index(const SplitArgs& a, int m) {
  if (a.R1 == 1) return m;
  if constexpr (POW2) return ((m & (a.R1 - 1)) << a.logM) + (m >> a.log2R1);
  const int k2 = m / a.R1;
  return ((m - k2 * a.R1) << a.logM) + k2;
}
template <bool POW2>
__device__ __forceinline__ float2 z_at(const SplitArgs& a, const float2* Zb, int m) {
  return __ldg(&Zb[z_index<POW2>(a, m)]);
}
// Real-input bin k in [0, N/2] from the N/2-point complex FFT of the packed
// pairs: X = (A + B)/2 - i W_N^k (A - B)/2 with A = Z[k mod Nc], B = conj(Z[(Nc-k) mod Nc]).
template <bool POW2>
__device__ __forceinline__ float2 xr_at(const SplitArgs& a, const float2* Zb, int k) {
  float2 za, zb;
  if constexpr (POW2) {
    za = z_at<true>(a, Zb, k & (a.Nc - 1));
    zb = cconj(z_at<true>(a, Zb, (a.Nc - k) & (a.Nc - 1)));
  } else {
    za = z_at<false>(a, Zb, k == a.Nc ? 0 : k);
    zb = cconj(z_at<false>(a, Zb, k == 0 ? 0 : a.Nc - k));
  }
  const float2 s = cadd(za, zb), d = csub(za, zb);
  const float2 u = cmul(__ldg(&a.tw_big[k]), d);
  return make_float2(0.5f * s.x + 0.5f * u.y, 0.5f * s.y - 0.5f * u.x);
}
// get_bin (fftutil.rs:8-22) on the spectrum being formed, any kk.
template <bool REAL, bool POW2>
__device__ __forceinline__ float2 x_at(const SplitArgs& a, const float2* Zb, int kk) {
  int m;
  if constexpr (POW2) {
    m = kk & (a.N - 1);
  } else {
    m = kk % a.N;
    m += m < 0 ? a.N : 0;
  }
  if constexpr (!REAL) return z_at<POW2>(a, Zb, m);
  return m < a.K ? xr_at<POW2>(a, Zb, m) : cconj(xr_at<POW2>(a, Zb, a.N - m));
}

template <bool REAL, bool POW2>
__global__ void __launch_bounds__(256) welch_split_kernel(SplitArgs a) {
  __shared__ float2 xs[258];
  const int b = blockIdx.y;
  const int k0 = blockIdx.x * 256;
  const float2* Zb = a.Z + (size_t)b * a.Nc;
  for (int idx = threadIdx.x; idx < 258; idx += 256) xs[idx] = x_at<REAL, POW2>(a, Zb, k0 - 1 + idx);
  __syncthreads();
  const int k = k0 + threadIdx.x;
  if (k < a.K) {
    const float2 x0 = xs[threadIdx.x], x1 = xs[threadIdx.x + 1], x2 = xs[threadIdx.x + 2];
    a.X[(size_t)b * a.K + k] = x1;
    if (a.P) {
      const float cr = x1.x - (x0.x + x2.x) * 0.5f, ci = x1.y - (x0.y + x2.y) * 0.5f;
      a.P[(size_t)b * a.K + k] = __fadd_rn(__fmul_rn(cr, cr), __fmul_rn(ci, ci));
    }
  }
}

// ----------------------------------------------------------------- extended spectra
// Bin k of a block (k < K: all N bins for complex input, 0..N/2 for real)
// written into its extended row at every m < N + maxn with m = k mod N, and
// for real input its conjugate at every m = N - k mod N (0 < k < N/2): the
// row then holds get_bin(X, N, m) (fftutil.rs:8-22) for each m it has.
template <bool REAL>
__device__ __forceinline__ void store_ext(float2* __restrict__ row, int N, int maxn, int k, float2 x) {
  const int end = N + maxn;
  for (int m = k; m < end; m += N) row[m] = x;
  if constexpr (REAL) {
    if (k > 0 && k < N / 2) {
      const float2 c = cconj(x);
      for (int m = N - k; m < end; m += N) row[m] = c;
    }
  }
}

// One bin kk of the spectrum being formed, resolved once for every block of
// a buffer (the Welch kernels' lanes keep their bin across blocks):
// get_bin(X, N, kk) is the packed element at ia for complex input, and for
// real input the split of the elements at ia and ib with twiddle tw,
// conjugated (sg = -1) when kk mod N mirrors a bin of [0, N/2].  Its
// extended-row slots: kk, kk + N when below end = N + maxn, and for real
// 0 < kk < N/2 the conjugate at N - kk and 2N - kk when below end; more
// copies (maxn > N) take the general loops.
struct LaneBin {
  int ia, ib;
  float2 tw;
  float sg;
  bool wrap, mir1, mir2, more;
};

template <bool REAL, bool POW2>
__device__ __forceinline__ LaneBin lane_bin(const SplitArgs& a, int maxn, int kk) {
  int m;
  if constexpr (POW2) {
    m = kk & (a.N - 1);
  } else {
    m = kk % a.N;
    m += m < 0 ? a.N : 0;
  }
  LaneBin L;
  L.ib = 0;
  L.tw = make_float2(0.f, 0.f);
  L.sg = 1.f;
  if constexpr (!REAL) {
    L.ia = z_index<POW2>(a, m);
  } else {
    const bool mirror = m >= a.K;
    const int k = mirror ? a.N - m : m;                      // k in [0, N/2]
    if constexpr (POW2) {
      L.ia = z_index<true>(a, k & (a.Nc - 1));
      L.ib = z_index<true>(a, (a.Nc - k) & (a.Nc - 1));
    } else {
      L.ia = z_index<false>(a, k == a.Nc ? 0 : k);
      L.ib = z_index<false>(a, k == 0 ? 0 : a.Nc - k);
    }
    L.tw = __ldg(&a.tw_big[k]);
    L.sg = mirror ? -1.f : 1.f;
  }
  const int end = a.N + maxn;
  L.wrap = kk + a.N < end;
  L.mir1 = REAL && kk > 0 && 2 * kk < a.N;
  L.mir2 = L.mir1 && 2 * a.N - kk < end;
  L.more = kk + 2 * a.N < end || (L.mir1 && 3 * a.N - kk < end);
  return L;
}

// The lane's bin of one block, the same arithmetic as xr_at / x_at.
template <bool REAL>
__device__ __forceinline__ float2 lane_x(const LaneBin& L, const float2* __restrict__ Zb) {
  const float2 za = __ldg(&Zb[L.ia]);
  if constexpr (!REAL) return za;
  const float2 zb = cconj(__ldg(&Zb[L.ib]));
  const float2 s = cadd(za, zb), d = csub(za, zb);
  const float2 u = cmul(L.tw, d);
  return make_float2(0.5f * s.x + 0.5f * u.y, L.sg * (0.5f * s.y - 0.5f * u.x));
}

// store_ext for the lane's bin kk (kk < K) with its slots resolved.
template <bool REAL>
__device__ __forceinline__ void lane_store(const LaneBin& L, float2* __restrict__ row, int N, int end, int kk,
                                           float2 x) {
  row[kk] = x;
  if (L.wrap) row[kk + N] = x;
  if constexpr (REAL) {
    const float2 c = cconj(x);
    if (L.mir1) row[N - kk] = c;
    if (L.mir2) row[2 * N - kk] = c;
  }
  if (L.more) {
    for (int m = kk + 2 * N; m < end; m += N) row[m] = x;
    if (REAL && L.mir1)
      for (int m = 3 * N - kk; m < end; m += N) row[m] = cconj(x);
  }
}

template <bool REAL>
__global__ void __launch_bounds__(256) extend_kernel(const float2* __restrict__ X, int K, int N, float2* Xe,
                                                     long long xs, int maxn) {
  const int b = blockIdx.y, k = blockIdx.x * 256 + threadIdx.x;
  if (k < K) store_ext<REAL>(Xe + (size_t)b * xs, N, maxn, k, __ldg(&X[(size_t)b * K + k]));
}

// ----------------------------------------------------------------- split + Welch
// Each warp owns WELCH_WARP_BINS consecutive bins for all B blocks of the
// buffer: lane l forms X[k0 - 1 + l] (lanes 0 and 31 are the neighbours'
// halo), takes its neighbours by shuffle, writes X for the filter bank and
// adds the Hann-by-convolution term |X[k] - (X[k-1]+X[k+1])/2|^2 to the bin's
// f32 accumulator in block order, exactly as spectrum.rs:90-111 does.  No
// barrier separates the blocks, so their loads overlap.  Every `averages`
// blocks a record is written (spectrum.rs:116-161) and the accumulator
// restarts.  fmt: 0 u8, 1 u16 big-endian, 2 f32 mean power.  The u8/u16
// arithmetic is rounded per operation (no fused multiply-add) like the
// reference; only log10f may differ from the host libm in the last place.
__device__ __forceinline__ void emit_record(const WelchArgs& a, int r, int k, float s, int cnt) {
  const size_t o = (size_t)r * a.s.K + k;
  if (a.fmt == 2) {
    reinterpret_cast<float*>(a.out)[o] = __fdiv_rn(s, (float)cnt);
    return;
  }
  const float db = __fadd_rn(__fmul_rn(log10f(s), 10.0f), a.db_plus);
  if (a.fmt == 1) {
    const float q = fminf(fmaxf(__fadd_rn(__fmul_rn(db, 20.0f), 4000.0f), 0.0f), 4095.0f);
    const unsigned v = (unsigned)q;
    a.out[2 * o] = (uint8_t)(v >> 8);
    a.out[2 * o + 1] = (uint8_t)(v & 0xFF);
  } else {
    const float q = fminf(fmaxf(__fadd_rn(__fmul_rn(db, 2.0f), 250.0f), 0.0f), 255.0f);
    a.out[o] = (uint8_t)(unsigned)q;
  }
}

template <bool REAL, bool POW2>
__global__ void __launch_bounds__(32 * WELCH_WARPS) welch_kernel(WelchArgs a) {
  constexpr int CB = WELCH_WARP_BINS;                        // bins per CTA (every warp covers them)
  __shared__ float terms[WELCH_CHUNK][CB];
  pdl_wait();                                               // Z from the forward FFT
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int k0 = blockIdx.x * CB;
  const int kk = k0 - 1 + lane;                              // bin this lane forms
  const bool owner = lane >= 1 && lane <= CB && kk < a.s.K;
  const int slot = lane - 1;                                 // owner's column in `terms`
  const int N = a.s.N, end = N + a.maxn;
  const long long zs = a.s.Nc, xs = a.xs;
  const float2* __restrict__ Z = a.s.Z;
  float2* __restrict__ X = a.s.X;
  const LaneBin lb = lane_bin<REAL, POW2>(a.s, a.maxn, kk);
  // Phase B state: thread t sums bin k0 + t.
  const int kb = k0 + threadIdx.x;
  const bool summer = threadIdx.x < CB && kb < a.s.K;
  float acc = summer ? a.acc[kb] : 0.0f;
  int cnt = a.accn0, r = 0;
  for (int b0 = 0; b0 < a.B; b0 += WELCH_CHUNK) {
    const int nb = min(WELCH_CHUNK, a.B - b0);
    // Phase A: warp w forms blocks w, w + WARPS, ... (independent loads).
#pragma unroll 4
    for (int i = wid; i < nb; i += WELCH_WARPS) {
      const float2 x1 = lane_x<REAL>(lb, Z + (b0 + i) * zs);
      const float2 x0 = make_float2(__shfl_up_sync(0xffffffffu, x1.x, 1), __shfl_up_sync(0xffffffffu, x1.y, 1));
      const float2 x2 = make_float2(__shfl_down_sync(0xffffffffu, x1.x, 1), __shfl_down_sync(0xffffffffu, x1.y, 1));
      if (owner) {
        lane_store<REAL>(lb, X + (b0 + i) * xs, N, end, kk, x1);
        const float cr = x1.x - (x0.x + x2.x) * 0.5f, ci = x1.y - (x0.y + x2.y) * 0.5f;
        terms[i][slot] = __fadd_rn(__fmul_rn(cr, cr), __fmul_rn(ci, ci));
      }
    }
    __syncthreads();
    // Phase B: accumulate in block order, one run of additions per record.
    if (summer) {
      for (int i = 0; i < nb;) {
        const int stop = min(nb, i + (a.averages - cnt));
        cnt += stop - i;
#pragma unroll 8
        for (; i < stop; ++i) acc += terms[i][threadIdx.x];
        if (cnt >= a.averages) {
          emit_record(a, r, kb, acc, cnt);
          acc = 0.0f;
          cnt = 0;
          ++r;
        }
      }
    }
    __syncthreads();
  }
  if (summer) a.acc[kb] = acc;
  trace_end(a.trace, 2);
}

// The same records for few blocks per buffer: each warp owns its own 30 bins
// (+ a 1-bin halo each side) and walks every block in order, accumulating in
// registers -- the same additions in the same order as welch_kernel's
// phase B, with no shared memory and no barrier.
template <bool REAL, bool POW2>
__global__ void __launch_bounds__(32 * WELCH_WARPS) welch_bins_kernel(WelchArgs a) {
  constexpr int CB = WELCH_WARP_BINS;
  pdl_wait();                                               // Z from the forward FFT
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int k0 = (blockIdx.x * WELCH_WARPS + wid) * CB;
  if (k0 >= a.s.K) return;                                   // whole warp: no shuffle partner left behind
  const int kk = k0 - 1 + lane;
  const bool owner = lane >= 1 && lane <= CB && kk < a.s.K;
  const int N = a.s.N, end = N + a.maxn;
  const long long zs = a.s.Nc, xs = a.xs;
  const float2* __restrict__ Z = a.s.Z;
  float2* __restrict__ X = a.s.X;
  const LaneBin lb = lane_bin<REAL, POW2>(a.s, a.maxn, kk);
  float acc = owner ? a.acc[kk] : 0.0f;
  int cnt = a.accn0, r = 0;
#pragma unroll 4
  for (int b = 0; b < a.B; ++b) {
    const float2 x1 = lane_x<REAL>(lb, Z + b * zs);
    const float2 x0 = make_float2(__shfl_up_sync(0xffffffffu, x1.x, 1), __shfl_up_sync(0xffffffffu, x1.y, 1));
    const float2 x2 = make_float2(__shfl_down_sync(0xffffffffu, x1.x, 1), __shfl_down_sync(0xffffffffu, x1.y, 1));
    if (owner) {
      lane_store<REAL>(lb, X + b * xs, N, end, kk, x1);
      const float cr = x1.x - (x0.x + x2.x) * 0.5f, ci = x1.y - (x0.y + x2.y) * 0.5f;
      acc += __fadd_rn(__fmul_rn(cr, cr), __fmul_rn(ci, ci));
    }
    if (++cnt >= a.averages) {
      if (owner) emit_record(a, r, kk, acc, cnt);
      acc = 0.0f;
      cnt = 0;
      ++r;
    }
  }
  if (owner) a.acc[kk] = acc;
  trace_end(a.trace, 2);
}

// The same records for complex input whose spectra come from the two-pass
// FFT (R1 = Nc / M >= 16, powers of two): element m = k1 + R1 k2 sits at
// k1 M + k2, so the bins of a warp in welch_bins_kernel would read 32
// different rows.  Here a CTA owns WT_BINS consecutive bins m0 .. m0 +
// WT_BINS - 1, i.e. k2 in [k20, k20 + W) of every row k1 (W = WT_BINS / R1):
// per block it reads the R1 row segments of W elements (lanes along a
// segment: coalesced), transposes them through shared memory into bin order
// (one pad slot per R1 bins against bank conflicts), and each thread then
// forms, accumulates and emits its bins (tid + i T) exactly as
// welch_bins_kernel does, with coalesced spectrum, accumulator and record
// accesses.  Blocks run in order through two shared-memory buffers: block
// b + 1 is copied in asynchronously (cp.async, no registers held) while
// block b is formed, one barrier per block.
constexpr int WT_BINS = 1024;
constexpr int WT_SLOTS = WT_BINS + WT_BINS / 16 + 2;        // bins m0 - 1 .. m0 + WT_BINS, padded

__device__ __forceinline__ void cp_async8(float2* smem, const float2* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <int T>
__global__ void __launch_bounds__(T) welch_tr_kernel(WelchArgs a) {
  constexpr int PER = WT_BINS / T;
  __shared__ float2 zs[2][WT_SLOTS];
  pdl_wait();                                               // Z from the forward FFT
  const SplitArgs& s = a.s;
  const int logR1 = s.log2R1, logW = ilog2c(WT_BINS) - logR1, W = 1 << logW;
  const int m0 = blockIdx.x * WT_BINS, k20 = m0 >> logR1;
  // bin offset o (o = -1 .. WT_BINS) -> slot; one pad slot after every R1 bins
  auto slot = [&](int o) { return 1 + o + ((o + 1) >> logR1); };
  // Block b's R1 row segments and the two halo bins into buf, asynchronously.
  auto fetch = [&](int b, float2* buf) {
    const float2* Zb = s.Z + (size_t)b * s.Nc;
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = threadIdx.x + i * T, k1 = e >> logW, j = e & (W - 1);
      cp_async8(&buf[slot(k1 + (j << logR1))], &Zb[((size_t)k1 << s.logM) + k20 + j]);
    }
    if (threadIdx.x == 0) cp_async8(&buf[slot(-1)], &Zb[z_index<true>(s, (m0 - 1) & (s.N - 1))]);
    if (threadIdx.x == 1) cp_async8(&buf[slot(WT_BINS)], &Zb[z_index<true>(s, (m0 + WT_BINS) & (s.N - 1))]);
    cp_async_commit();
  };
  float acc[PER];
#pragma unroll
  for (int i = 0; i < PER; ++i) acc[i] = a.acc[m0 + threadIdx.x + i * T];
  int cnt = a.accn0, r = 0;
  if (a.B > 0) fetch(0, zs[0]);
  for (int b = 0; b < a.B; ++b) {
    cp_async_wait_all();
    __syncthreads();            // block b is in zs[b & 1]; every thread is done reading zs[(b + 1) & 1]
    if (b + 1 < a.B) fetch(b + 1, zs[(b + 1) & 1]);
    const float2* z = zs[b & 1];
    float2* Xb = s.X + (size_t)b * a.xs;
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = threadIdx.x + i * T;
      const float2 x0 = z[slot(e - 1)], x1 = z[slot(e)], x2 = z[slot(e + 1)];
      store_ext<false>(Xb, s.N, a.maxn, m0 + e, x1);
      const float cr = x1.x - (x0.x + x2.x) * 0.5f, ci = x1.y - (x0.y + x2.y) * 0.5f;
      acc[i] += __fadd_rn(__fmul_rn(cr, cr), __fmul_rn(ci, ci));
    }
    if (++cnt >= a.averages) {
#pragma unroll
      for (int i = 0; i < PER; ++i) {
        emit_record(a, r, m0 + threadIdx.x + i * T, acc[i], cnt);
        acc[i] = 0.0f;
      }
      cnt = 0;
      ++r;
    }
  }
#pragma unroll
  for (int i = 0; i < PER; ++i) a.acc[m0 + threadIdx.x + i * T] = acc[i];
  trace_end(a.trace, 2);
}

// ----------------------------------------------------------------- filter bank
// CHIRP: the chirp-z tiles of the list (their own launch); else the
// power-of-two tiles.
template <int S, int T, int MINB, bool PERSIST, bool CHIRP>
__global__ void __launch_bounds__(T, MINB) fcfb_kernel(FcfbArgs a, int tile_base) {
  extern __shared__ float2 sm[];
  __shared__ TileMeta s_meta[MAX_TILE_TRANSFORMS];
  __shared__ int s_tile[2];
  static_assert(MAX_TILE_TRANSFORMS <= T, "one thread stages one transform's metadata");
  // Persistent: thread 0 claims tile it+1 while tile it is being transformed
  // (the claim's latency hides behind the FFT), publishing it in s_tile[(it+1)&1]
  // just before the barrier that starts iteration it+1.
  if constexpr (PERSIST) {
    if (threadIdx.x == 0) s_tile[0] = atomicAdd(a.cursor, 1);
  }
  for (int it = 0;; ++it) {
    const FcfbTileConst c{a.tw, a.tw_split, a.log_split};
    int tile, next = 0;
    if constexpr (PERSIST) {
      __syncthreads();               // also orders the previous tile's reads before this tile's writes
      tile = s_tile[it & 1];
      if (tile >= a.ntiles) {
        trace_end(a.trace, 3);
        return;
      }
      if (threadIdx.x == 0) next = atomicAdd(a.cursor, 1);
    } else {
      if (it) {
        trace_end(a.trace, 3);
        return;
      }
      tile = tile_base + blockIdx.x;
    }
    const TileDesc td = a.tiles[tile];
    if (threadIdx.x < td.count) {
      const int2 cb = __ldg(&a.list[td.list_off + threadIdx.x]);
      const ChanDev& ch = a.chans[cb.x];
      const int keep = 6 * ((CHIRP ? a.blu[td.pad].n : 1 << td.log2n) >> 3);
      const int logp = CHIRP ? 0 : max(0, td.log2n - ilog2c(S));   // split into 2^logp parts: entry (channel, P block + part)
      const int b = cb.y >> logp;
      TileMeta m;
      m.X = a.X + (size_t)b * a.xs + ch.first;                // first is already modulo N
      m.w = ch.w;
      m.out = ch.out + (size_t)b * keep;
      m.pad = cb.y & ((1 << logp) - 1);
      m.unused = 0;
      s_meta[threadIdx.x] = m;
    }
    __syncthreads();
    if (it == 0) pdl_wait();                                  // X from the Welch kernel
    fcfb_tile_dispatch<S, T, CHIRP>(td.log2n, sm, s_meta, td.count, c, CHIRP ? a.blu + td.pad : nullptr);
    if constexpr (PERSIST) {
      if (threadIdx.x == 0) s_tile[(it + 1) & 1] = next;
    }
  }
}

// Adjoint of fcfb_kernel, deterministic (no atomics: every sum runs in a
// fixed order, so two runs give the same bits).  With g = FFT_n(dy zero-padded
// to [n/8, 7n/8)) (the forward transform is the adjoint of the unnormalised
// inverse) and v = w * G, G = get_bin(X, first + j):
//   dW[j] = sum over blocks, in block order, of conj(G[j]) g[j]
//   dX[bin] += sum over the (channel, j) that gather the bin, in channel
//              order, of conj(w[j]) g[j] (conjugated for mirror bins).
// Step 1: g of every (channel, block) transform on the staged tile pipeline
// (forward FFT, load = padded dy, store = the channel's g scratch).
struct BwdMeta {
  const float2* dy;     // block's output gradients, 6(n/8)
  float2* g;            // block's row of the channel's g scratch, n, indexed by weight index j
};

template <int LOGN, int S, int T>
__device__ __forceinline__ void bwd_tile(float2* sm, const BwdMeta* meta, int count, const float2* tw) {
  constexpr int n = 1 << LOGN, lo = n >> 3, keep = 6 * lo;
  using P = StagePlan<LOGN, S / T>;
  auto load = [&](int t, int q, int s) {
    const int i = q + (s << P::first_shift) - lo;
    if constexpr (keep == 0) return make_float2(0.f, 0.f);  // n = 4 keeps no outputs
    else return (unsigned)i < (unsigned)keep ? __ldg(&meta[t].dy[i]) : make_float2(0.f, 0.f);
  };
  // FFT output o pairs with IFFT input o, whose weight index is j = (o + n/2) mod n
  // (fcfb.rs:166-169): g is stored by j, so g[j] multiplies conj(G[j]) and conj(w[j]).
  auto store = [&](int t, int q, int u, float2 v) {
    meta[t].g[(q + (u << P::last_shift) + n / 2) & (n - 1)] = v;
  };
  tile_pipeline<LOGN, S, T, -1, true>(sm, count, tw, load, store);
}

template <int S, int T>
__global__ void __launch_bounds__(T, 2) fcfb_bwd_fft_kernel(BwdArgs a) {
  extern __shared__ float2 sm[];
  __shared__ BwdMeta s_meta[MAX_TILE_TRANSFORMS];
  static_assert(MAX_TILE_TRANSFORMS <= T, "one thread stages one transform's metadata");
  const TileDesc td = a.tiles[blockIdx.x];
  if (threadIdx.x < td.count) {
    const int2 cb = __ldg(&a.list[td.list_off + threadIdx.x]);
    const BwdChan& ch = a.chans[cb.x];
    const int n = 1 << td.log2n;
    s_meta[threadIdx.x] = BwdMeta{ch.dy + (size_t)cb.y * (6 * (n >> 3)), ch.g + (size_t)cb.y * n};
  }
  __syncthreads();
  switch (td.log2n) {
    case 2: bwd_tile<2, S, T>(sm, s_meta, td.count, a.tw); break;
    case 3: bwd_tile<3, S, T>(sm, s_meta, td.count, a.tw); break;
    case 4: bwd_tile<4, S, T>(sm, s_meta, td.count, a.tw); break;
    case 5: bwd_tile<5, S, T>(sm, s_meta, td.count, a.tw); break;
    case 6: bwd_tile<6, S, T>(sm, s_meta, td.count, a.tw); break;
    case 7: bwd_tile<7, S, T>(sm, s_meta, td.count, a.tw); break;
    case 8: bwd_tile<8, S, T>(sm, s_meta, td.count, a.tw); break;
    case 9: bwd_tile<9, S, T>(sm, s_meta, td.count, a.tw); break;
    case 10: bwd_tile<10, S, T>(sm, s_meta, td.count, a.tw); break;
    case 11: bwd_tile<11, S, T>(sm, s_meta, td.count, a.tw); break;
    case 12: bwd_tile<12, S, T>(sm, s_meta, td.count, a.tw); break;
    case 13: bwd_tile<13, S, T>(sm, s_meta, td.count, a.tw); break;
  }
}

// get_bin on the [B][K] spectra: bin (first + j) mod N of block b, and
// whether it is the conjugate mirror (real input, m >= K).
template <bool REAL>
__device__ __forceinline__ float2 bwd_bin(const BwdArgs& a, int b, long long first, int j) {
  const int m = (int)((first + j) % a.N);
  const bool mirror = REAL && m >= a.K;
  const float2 x = __ldg(&a.X[(size_t)b * a.K + (mirror ? a.N - m : m)]);
  return mirror ? cconj(x) : x;
}

// Step 2: dW[c][j] = sum_b conj(G_b[j]) g_b[j], one thread per (channel, j).
template <bool REAL>
__global__ void __launch_bounds__(256) fcfb_bwd_dw_kernel(BwdArgs a) {
  const int c = blockIdx.y, j = blockIdx.x * 256 + threadIdx.x;
  const BwdChan& ch = a.chans[c];
  const int n = 1 << ch.log2n;
  if (j >= n) return;
  float2 acc = make_float2(0.f, 0.f);
  for (int b = 0; b < a.B; ++b) {
    const float2 G = bwd_bin<REAL>(a, b, ch.first, j);
    acc = cadd(acc, cmul(cconj(G), __ldg(&ch.g[(size_t)b * n + j])));
  }
  ch.dw[j] = acc;
}

// Step 3: dX[b][k] += sum over bin k's gather list (channel order) of
// conj(w[j]) g_b[j], conjugated for mirror entries; one thread per (b, k).
template <int V = 0>   // a template, so that every translation unit including this header shares one instance
__global__ void __launch_bounds__(256) fcfb_bwd_dx_kernel(BwdArgs a) {
  const int b = blockIdx.y, k = blockIdx.x * 256 + threadIdx.x;
  if (k >= a.K) return;
  float2 acc = make_float2(0.f, 0.f);
  const int e1 = __ldg(&a.bin_off[k + 1]);
  for (int e = __ldg(&a.bin_off[k]); e < e1; ++e) {
    const int2 ent = __ldg(&a.bin_ent[e]);
    const BwdChan& ch = a.chans[ent.x];
    const int j = ent.y >> 1;
    const int n = 1 << ch.log2n;
    float2 d = cmul(cconj(__ldg(&ch.w[j])), __ldg(&ch.g[(size_t)b * n + j]));
    if (ent.y & 1) d = cconj(d);
    acc = cadd(acc, d);
  }
  float2* x = a.dX + (size_t)b * a.K + k;
  *x = cadd(*x, acc);
}

}  // namespace sk
