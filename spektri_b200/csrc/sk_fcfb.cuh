// Filter-bank tile pipeline (fcfb.rs:154-188 for many channels and blocks).
//
// A tile holds `count` n-point inverse transforms (one per (channel, block)
// pair).  Each transform's metadata (spectrum row, weights, output row, first
// bin modulo N) is staged in shared memory once per tile.  The FFT runs as 1-3
// Stockham stages with the IFFT size fixed at compile time:
//   first stage : gathers its inputs straight from the spectrum
//                 (get_bin with modulo and conjugate mirror, fftutil.rs:8-22),
//                 multiplies by the weights, DFT_R, writes shared memory
//   middle stage: shared -> twiddle -> DFT_R -> shared (in place)
//   last stage  : shared -> twiddle -> DFT_R -> the kept samples [n/8, 7(n/8))
//                 straight to the channel's output (fcfb.rs:177-187)
// so shared memory is touched twice per element per middle/last stage and the
// gather and discard need no extra pass.
#pragma once
#include "sk_fft.cuh"

namespace sk {

constexpr int MAX_TILE_TRANSFORMS = 256;

struct TileMeta {
  const float2* X;     // spectrum row of the block, K bins
  const float2* w;     // weights, natural order
  float2* out;         // output row of the block: 6(n/8) samples
  int first;           // first bin modulo N
  int pad;
};

struct FcfbTileConst {
  int N, K;
  const float2* tw;    // W_S^k
};

// log2 radices of the stages for a 2^LOGN-point transform.
template <int LOGN> struct FcfbPlan;
template <> struct FcfbPlan<2> { static constexpr int ns = 1, r0 = 2, r1 = 0, r2 = 0; };
template <> struct FcfbPlan<3> { static constexpr int ns = 1, r0 = 3, r1 = 0, r2 = 0; };
template <> struct FcfbPlan<4> { static constexpr int ns = 1, r0 = 4, r1 = 0, r2 = 0; };
template <> struct FcfbPlan<5> { static constexpr int ns = 2, r0 = 3, r1 = 2, r2 = 0; };
template <> struct FcfbPlan<6> { static constexpr int ns = 2, r0 = 3, r1 = 3, r2 = 0; };
template <> struct FcfbPlan<7> { static constexpr int ns = 2, r0 = 4, r1 = 3, r2 = 0; };
template <> struct FcfbPlan<8> { static constexpr int ns = 2, r0 = 4, r1 = 4, r2 = 0; };
template <> struct FcfbPlan<9> { static constexpr int ns = 2, r0 = 4, r1 = 5, r2 = 0; };
template <> struct FcfbPlan<10> { static constexpr int ns = 3, r0 = 4, r1 = 3, r2 = 3; };
template <> struct FcfbPlan<11> { static constexpr int ns = 3, r0 = 4, r1 = 3, r2 = 4; };
template <> struct FcfbPlan<12> { static constexpr int ns = 3, r0 = 4, r1 = 4, r2 = 4; };
template <> struct FcfbPlan<13> { static constexpr int ns = 3, r0 = 4, r1 = 4, r2 = 5; };

// get_bin for the gather: bin m (already reduced modulo N) of one block.
template <bool REAL>
__device__ __forceinline__ float2 spectrum_bin(const float2* __restrict__ X, int m, int N, int K) {
  if (REAL && m >= K) {
    const float2 v = __ldg(&X[N - m]);
    return make_float2(v.x, -v.y);
  }
  return __ldg(&X[m]);
}

// Stage 1 (L = 1): butterfly q of transform t reads elements q + s n/R.
template <int LOGN, int R, int S, int T, bool REAL, bool LAST>
__device__ __forceinline__ void fcfb_first(float2* sm, const TileMeta* meta, int count, const FcfbTileConst& c) {
  constexpr int n = 1 << LOGN, LOGR = ilog2c(R), LOGNR = LOGN - LOGR, NB = S / (R * T);
  static_assert(NB >= 1, "radix too large for the tile");
  constexpr int lo = n >> 3, keep = 6 * lo;
  // Inputs come from global memory, so each butterfly is stored as soon as
  // it is done (no in-place hazard): only R values are live at a time.
#pragma unroll
  for (int bb = 0; bb < NB; ++bb) {
    const int beta = threadIdx.x + bb * T;
    const int t = beta >> LOGNR, q = beta & ((1 << LOGNR) - 1);
    float2 v[R];
    if (t < count) {
      const float2* X = meta[t].X;
      const float2* w = meta[t].w;
      const int first = meta[t].first;
#pragma unroll
      for (int s = 0; s < R; ++s) {
        const int i = q + (s << LOGNR);
        const int j = (i + n / 2) & (n - 1);                  // fcfb.rs:166-169
        const int m = (first + j) & (c.N - 1);
        v[s] = cmul(__ldg(&w[j]), spectrum_bin<REAL>(X, m, c.N, c.K));
      }
    } else {
#pragma unroll
      for (int s = 0; s < R; ++s) v[s] = make_float2(0.f, 0.f);
    }
    dft<R, +1>(v);
    if constexpr (LAST) {                                    // n = R: q = 0, output u
      if (t < count) {
        float2* out = meta[t].out;
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (u >= lo && u < lo + keep) out[u - lo] = v[u];
      }
    } else {
#pragma unroll
      for (int u = 0; u < R; ++u) sm[padx((t << LOGN) + q * R + u)] = v[u];
    }
  }
}

// Stages 2..: span L = 2^LOGL, shared-memory input.  LAST writes the kept
// outputs to global memory (g = 0 there), otherwise in place to shared memory.
template <int LOGN, int R, int LOGL, int S, int T, bool LAST>
__device__ __forceinline__ void fcfb_next(float2* sm, const TileMeta* meta, int count, const FcfbTileConst& c) {
  constexpr int n = 1 << LOGN, LOGR = ilog2c(R), LOGNR = LOGN - LOGR, NB = S / (R * T);
  constexpr int LOGS = ilog2c(S), SH = LOGS - LOGL - LOGR;
  static_assert(NB >= 1 && SH >= 0, "bad stage");
  constexpr int lo = n >> 3, keep = 6 * lo;
  if constexpr (LAST) {
    // Outputs go to global memory: one butterfly live at a time.
#pragma unroll
    for (int bb = 0; bb < NB; ++bb) {
      const int beta = threadIdx.x + bb * T;
      const int t = beta >> LOGNR, q = beta & ((1 << LOGNR) - 1);
      const int j = q & ((1 << LOGL) - 1);
      const int base = t << LOGN;
      float2 v[R];
#pragma unroll
      for (int s = 0; s < R; ++s) v[s] = sm[padx(base + q + (s << LOGNR))];
#pragma unroll
      for (int s = 1; s < R; ++s) {
        const float2 w = __ldg(&c.tw[(j * s) << SH]);
        v[s] = cmul(v[s], make_float2(w.x, -w.y));           // inverse: conj of W_S
      }
      dft<R, +1>(v);
      if (t < count) {
        float2* out = meta[t].out;
#pragma unroll
        for (int u = 0; u < R; ++u) {
          const int o = q + (u << LOGNR) - lo;               // q + u L with L = n/R
          if ((unsigned)o < (unsigned)keep) out[o] = v[u];
        }
      }
    }
  } else {
    float2 v[NB][R];
#pragma unroll
    for (int bb = 0; bb < NB; ++bb) {
      const int beta = threadIdx.x + bb * T;
      const int t = beta >> LOGNR, q = beta & ((1 << LOGNR) - 1);
      const int j = q & ((1 << LOGL) - 1);
      const int base = t << LOGN;
#pragma unroll
      for (int s = 0; s < R; ++s) v[bb][s] = sm[padx(base + q + (s << LOGNR))];
#pragma unroll
      for (int s = 1; s < R; ++s) {
        const float2 w = __ldg(&c.tw[(j * s) << SH]);
        v[bb][s] = cmul(v[bb][s], make_float2(w.x, -w.y));
      }
      dft<R, +1>(v[bb]);
    }
    __syncthreads();
#pragma unroll
    for (int bb = 0; bb < NB; ++bb) {
      const int beta = threadIdx.x + bb * T;
      const int t = beta >> LOGNR, q = beta & ((1 << LOGNR) - 1);
      const int j = q & ((1 << LOGL) - 1), g = q >> LOGL;
      const int ob = (t << LOGN) + (g << (LOGL + LOGR)) + j;
#pragma unroll
      for (int u = 0; u < R; ++u) sm[padx(ob + (u << LOGL))] = v[bb][u];
    }
  }
}

template <int LOGN, int S, int T, bool REAL>
__device__ __forceinline__ void fcfb_tile(float2* sm, const TileMeta* meta, int count, const FcfbTileConst& c) {
  using P = FcfbPlan<LOGN>;
  if constexpr (P::ns == 1) {
    fcfb_first<LOGN, 1 << P::r0, S, T, REAL, true>(sm, meta, count, c);
  } else if constexpr (P::ns == 2) {
    fcfb_first<LOGN, 1 << P::r0, S, T, REAL, false>(sm, meta, count, c);
    __syncthreads();
    fcfb_next<LOGN, 1 << P::r1, P::r0, S, T, true>(sm, meta, count, c);
  } else {
    fcfb_first<LOGN, 1 << P::r0, S, T, REAL, false>(sm, meta, count, c);
    __syncthreads();
    fcfb_next<LOGN, 1 << P::r1, P::r0, S, T, false>(sm, meta, count, c);
    __syncthreads();
    fcfb_next<LOGN, 1 << P::r2, P::r0 + P::r1, S, T, true>(sm, meta, count, c);
  }
}

template <int S, int T, bool REAL>
__device__ __forceinline__ void fcfb_tile_dispatch(int log2n, float2* sm, const TileMeta* meta, int count,
                                                   const FcfbTileConst& c) {
  switch (log2n) {
    case 2: fcfb_tile<2, S, T, REAL>(sm, meta, count, c); break;
    case 3: fcfb_tile<3, S, T, REAL>(sm, meta, count, c); break;
    case 4: fcfb_tile<4, S, T, REAL>(sm, meta, count, c); break;
    case 5: fcfb_tile<5, S, T, REAL>(sm, meta, count, c); break;
    case 6: fcfb_tile<6, S, T, REAL>(sm, meta, count, c); break;
    case 7: fcfb_tile<7, S, T, REAL>(sm, meta, count, c); break;
    case 8: fcfb_tile<8, S, T, REAL>(sm, meta, count, c); break;
    case 9: fcfb_tile<9, S, T, REAL>(sm, meta, count, c); break;
    case 10: fcfb_tile<10, S, T, REAL>(sm, meta, count, c); break;
    case 11: fcfb_tile<11, S, T, REAL>(sm, meta, count, c); break;
    case 12: fcfb_tile<12, S, T, REAL>(sm, meta, count, c); break;
    case 13: fcfb_tile<13, S, T, REAL>(sm, meta, count, c); break;
  }
}

}  // namespace sk
