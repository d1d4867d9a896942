// In-place tile FFTs for the filter bank's large transforms, 16 elements per
// thread (tile shapes 4096 x 256 and 8192 x 512): n = 512 .. 4096 in three
// stages, n = 8192 in four (ip_pipeline_8k below), decimation in time with the
// leaf outputs kept in place:
//
//   n = 16 R2 R1, input index i = i1 + R1 i2 + R1 R2 i3 (i1 < R1, i2 < R2, i3 < 16)
//   leaf   : for each q = i1 + R1 i2 (NL = n/16 leaves), Y[q][k3] = DFT_16 over
//            i3 of x[q + NL i3]  (input stride NL: one gather per element)
//   middle : for each (i1, k3), Z[i1][k3 + 16 u2] =
//            DFT_R2 over i2 of W_{16 R2}^(i2 k3) Y[i1 + R1 i2][k3]
//   last   : for each k'' < n/R1, X[k'' + (n/R1) u1] =
//            DFT_R1 over i1 of W_n^(i1 k'') Z[i1][k'']
//
// Y[q][k3] sits at row k3, column q of a transform's region: position
// q + (NL + 1) k3 (one pad slot per row).  The middle stage writes
// Z[i1][k3 + 16 u2] where it read Y[i1 + R1 u2][k3], so each thread writes
// exactly the positions it read: no barrier between its reads and writes,
// one barrier per stage.  Every address of a stage is one base register plus
// compile-time offsets, and with the odd row stride NL + 1:
//   leaf stores   : lanes at consecutive q            -> consecutive words
//   middle        : lanes at consecutive k3 (row)     -> stride NL + 1 (odd)
//   last loads    : lanes at consecutive k'' (k3 fastest) -> stride NL + 1
// so a warp's 256 bytes take the minimum two shared-memory wavefronts, and
// the last stage's global stores (output k'' + (n/R1) u1) are coalesced.
// Twiddles: the same per-stage tables as the Stockham stages (sk_fcfb.cuh,
// TwiddlePowers): W_{16 R2}^(k3 s) is the span-16 table of P = 16 R2, and
// W_n^(k'' s) the span-n/R1 table of P = n.
#pragma once
#include "sk_fcfb.cuh"

namespace sk {

// log2 of the middle (R2) and last (R1) radices for n = 2^LOGN.
template <int LOGN>
struct IpPlan {
  static_assert(LOGN >= 9 && LOGN <= 12, "in-place plan: 512 .. 4096 points");
  static constexpr int r_last = LOGN == 9 ? 3 : LOGN == 10 ? 3 : 4;   // R1 >= 8: output window on digit edges
  static constexpr int r_mid = LOGN - 4 - r_last;
  static constexpr int n = 1 << LOGN, NL = n >> 4, ROW = NL + 1, SPAN = n + 16;
};

// load(t, q, s): input i = q + NL s of transform t.  store(t, kk, u, v):
// output o = kk + (n/R1) u (the Stockham stores' convention).  count
// transforms (t < count); the caller syncs before (shared memory free).
template <int LOGN, int S, int T, class Load, class Store, class Ctx = CtaCtx>
__device__ __forceinline__ void ip_pipeline(float2* sm, int count, const float2* __restrict__ tw, Load& load,
                                            Store& store, const Ctx& ctx = Ctx()) {
  using P = IpPlan<LOGN>;
  constexpr int R2 = 1 << P::r_mid, R1 = 1 << P::r_last, LOGNL = LOGN - 4;
  constexpr int NB0 = S / (16 * T), NB1 = S / (R2 * T), NB2 = S / (R1 * T);
  static_assert(NB0 >= 1 && NB1 >= 1 && NB2 >= 1, "tile too small for the radices");
  // leaf: 16-point DFTs straight from the loads, stored down a column
#pragma unroll
  for (int bb = 0; bb < NB0; ++bb) {
    const int beta = ctx.tid() + bb * T;
    const int t = beta >> LOGNL, q = beta & (P::NL - 1);
    float2 v[16];
    if (t < count) {
#pragma unroll
      for (int s = 0; s < 16; ++s) v[s] = load(t, q, s);
    } else {
#pragma unroll
      for (int s = 0; s < 16; ++s) v[s] = make_float2(0.f, 0.f);
    }
    dft<16, +1>(v);
    float2* p = sm + t * P::SPAN + q;
#pragma unroll
    for (int k = 0; k < 16; ++k) p[k * P::ROW] = v[k];
  }
  ctx.sync();
  // middle: (i1, k3) per butterfly, k3 fastest across lanes; in place
  {
    constexpr int SH = TILE_LOGS - 4 - P::r_mid;           // table of P = 16 R2, span 16
    float2 v[NB1][R2];
    float2* base[NB1];
#pragma unroll
    for (int bb = 0; bb < NB1; ++bb) {
      const int beta = ctx.tid() + bb * T;
      const int k3 = beta & 15, i1 = (beta >> 4) & (R1 - 1), t = beta >> (4 + P::r_last);
      base[bb] = sm + t * P::SPAN + i1 + P::ROW * k3;
#pragma unroll
      for (int s = 0; s < R2; ++s) v[bb][s] = base[bb][R1 * s];
      twiddle_dft<R2, SH, +1>(v[bb], tw, k3);
    }
#pragma unroll
    for (int bb = 0; bb < NB1; ++bb) {
#pragma unroll
      for (int u = 0; u < R2; ++u) base[bb][R1 * u] = v[bb][u];
    }
  }
  ctx.sync();
  // last: k'' per butterfly (k3 fastest), reads a row segment, stores outputs
  {
    constexpr int SH = TILE_LOGS - LOGN;                    // table of P = n, span n/R1
    constexpr int LOGK = LOGN - P::r_last;
#pragma unroll
    for (int bb = 0; bb < NB2; ++bb) {
      const int beta = ctx.tid() + bb * T;
      const int kk = beta & ((1 << LOGK) - 1), t = beta >> LOGK;
      const float2* p = sm + t * P::SPAN + R1 * (kk >> 4) + P::ROW * (kk & 15);
      float2 v[R1];
#pragma unroll
      for (int s = 0; s < R1; ++s) v[s] = p[s];
      twiddle_dft<R1, SH, +1>(v, tw, kk);
      if (t < count) {
#pragma unroll
        for (int u = 0; u < R1; ++u) store(t, kk, u, v[u]);
      }
    }
  }
}

// The filter-bank tile of n = 512 .. 4096 points on the in-place pipeline:
// input buf[i] = W[j] bin(first + j), j = (i + n/2) mod n (fcfb.rs:166-172),
// outputs [n/8, 7(n/8)) kept (fcfb.rs:177).
template <int LOGN, int S, int T, class Ctx = CtaCtx>
__device__ __forceinline__ void fcfb_tile_ip(float2* sm, const TileMeta* meta, int count, const FcfbTileConst& c,
                                             const Ctx& ctx = Ctx()) {
  constexpr int R1 = 1 << IpPlan<LOGN>::r_last;
  auto load = [&](int t, int q, int s) { return fcfb_input<LOGN, 16>(meta[t], q, s); };
  auto store = [&](int t, int kk, int u, float2 v) {
    fcfb_keep<LOGN, R1>(kk, u, [&](int k) { meta[t].out[k] = v; });
  };
  ip_pipeline<LOGN, S, T>(sm, count, c.tw, load, store, ctx);
}

// The same in-place scheme for n = 8192 = 16 * 16 * 16 * 2 (one transform
// per 8192-point tile, 512 threads), input i = i1 + 2 i2 + 32 i3 + 512 i4:
//   leaf : Y[q][k4]               = DFT_16 over i4 of x[q + 512 i4]     (q = i1 + 2 i2 + 32 i3)
//   A    : Z1[o][k4 + 16 u3]       = DFT_16 over i3 of W_256^(i3 k4) Y[o + 32 i3][k4]      (o = i1 + 2 i2)
//   B    : Z2[i1][k'' + 256 u2]    = DFT_16 over i2 of W_4096^(i2 k'') Z1[i1 + 2 i2][k'']  (k'' = k4 + 16 u3)
//   last : X[k''' + 4096 u1]       = DFT_2 over i1 of W_8192^(i1 k''') Z2[i1][k''']         (k''' = k'' + 256 u2)
// Y[q][k4] at q + 513 k4; A and B write in place, so Z2[i1][k4 + 16 u3 + 256 u2]
// sits at i1 + 2 u2 + 32 u3 + 513 k4.  Lanes run k4 fastest in A, B and the
// last stage (odd stride 513), consecutive q in the leaf.  DIR = +1 is the
// inverse transform (the filter bank), -1 the forward one (the row pass of
// the two-pass forward FFT).
constexpr int IP8K_ROW = 513;                // 8192 + 16 elements of shared memory

template <int T, int DIR = +1, class Load, class Store>
__device__ __forceinline__ void ip_pipeline_8k(float2* sm, const float2* __restrict__ tw, Load& load, Store& store) {
  static_assert(T == 512, "one 16-point leaf, A and B butterfly per thread");
  const int tid = threadIdx.x;
  {
    float2 v[16];
#pragma unroll
    for (int s = 0; s < 16; ++s) v[s] = load(0, tid, s);
    dft<16, DIR>(v);
    float2* p = sm + tid;
#pragma unroll
    for (int k = 0; k < 16; ++k) p[k * IP8K_ROW] = v[k];
  }
  __syncthreads();
  {
    const int k4 = tid & 15, o = tid >> 4;
    float2* p = sm + o + IP8K_ROW * k4;
    float2 v[16];
#pragma unroll
    for (int s = 0; s < 16; ++s) v[s] = p[32 * s];
    twiddle_dft<16, TILE_LOGS - 8, DIR>(v, tw, k4);          // P = 256, span 16
#pragma unroll
    for (int u = 0; u < 16; ++u) p[32 * u] = v[u];
  }
  __syncthreads();
  {
    const int k4 = tid & 15, u3 = (tid >> 4) & 15, i1 = tid >> 8;
    float2* p = sm + i1 + 32 * u3 + IP8K_ROW * k4;
    float2 v[16];
#pragma unroll
    for (int s = 0; s < 16; ++s) v[s] = p[2 * s];
    twiddle_dft<16, TILE_LOGS - 12, DIR>(v, tw, tid & 255);  // P = 4096, span 256: k'' = k4 + 16 u3
#pragma unroll
    for (int u = 0; u < 16; ++u) p[2 * u] = v[u];
  }
  __syncthreads();
#pragma unroll
  for (int bb = 0; bb < 8; ++bb) {
    const int kk = tid + bb * T;                             // k''' < 4096
    const float2* p = sm + 2 * (kk >> 8) + 32 * ((kk >> 4) & 15) + IP8K_ROW * (kk & 15);
    float2 v[2] = {p[0], p[1]};
    twiddle_dft<2, 0, DIR>(v, tw, kk);                        // P = 8192, span 4096
    store(0, kk, 0, v[0]);
    store(0, kk, 1, v[1]);
  }
}

// The filter bank's 8192-point transform on ip_pipeline_8k.
template <int T>
__device__ __forceinline__ void fcfb_tile_8k(float2* sm, const TileMeta* meta, const FcfbTileConst& c) {
  auto load = [&](int, int q, int s) { return fcfb_input<13, 16>(meta[0], q, s); };
  auto store = [&](int, int kk, int u, float2 v) {
    fcfb_keep<13, 2>(kk, u, [&](int k) { meta[0].out[k] = v; });
  };
  ip_pipeline_8k<T>(sm, c.tw, load, store);
}

// One part of an n = P S transform (P = 2, 4, 8; fcfb_tile_part's split)
// on the in-place pipeline of S points.
template <int S, int T, int LOGP>
__device__ __forceinline__ void fcfb_tile_part_ip(float2* sm, const TileMeta* meta, const FcfbTileConst& c) {
  constexpr int LOGS = ilog2c(S), P = 1 << LOGP, NL = S >> 4;
  const TileMeta& m = meta[0];
  auto load = [&](int, int q, int s) { return part_input<S, LOGP>(m, c, q + s * NL); };
  if constexpr (LOGS == 13) {
    auto store = [&](int, int kk, int u, float2 v) {
      fcfb_keep<13, 2>(kk, u, [&](int k) { m.out[P * k + m.pad] = v; });
    };
    ip_pipeline_8k<T>(sm, c.tw, load, store);
  } else {
    constexpr int RL = 1 << IpPlan<LOGS>::r_last;
    auto store = [&](int, int kk, int u, float2 v) {
      fcfb_keep<LOGS, RL>(kk, u, [&](int k) { m.out[P * k + m.pad] = v; });
    };
    ip_pipeline<LOGS, S, T>(sm, 1, c.tw, load, store);
  }
}

// An 8192-point tile of n <= 4096 points in a 512-thread CTA: each 256-thread
// half runs the first or second half of the tile's transforms as a 4096-point
// tile of its own, in its own half of shared memory, synchronised by its own
// named barrier, so that barriers span 8 warps as in the 4096 x 256 shape
// while 8192-point transforms still run on the whole CTA.
template <int LOGN>
__device__ __forceinline__ void fcfb_tile_halves(float2* sm, const TileMeta* meta, int count, const FcfbTileConst& c) {
  constexpr int HALF = 4096 >> LOGN;                         // transforms per half
  const int h = threadIdx.x >> 8;
  const int cnt = min(HALF, count - h * HALF);
  if (cnt <= 0) return;                                      // this half has nothing (a short tile)
  const HalfCtx ctx{(int)(threadIdx.x & 255), 1 + h};
  float2* smh = sm + h * (4096 + 256);
  if constexpr (LOGN >= 9) fcfb_tile_ip<LOGN, 4096, 256>(smh, meta + h * HALF, cnt, c, ctx);
  else fcfb_tile<LOGN, 4096, 256>(smh, meta + h * HALF, cnt, c, ctx);
}

// Filter-bank tile of log2 size log2n (or a chirp-z tile).  With 16 elements
// per thread, n = 512 .. 4096 run on the in-place pipeline (in the 8192 x 512
// shape as two independent 256-thread halves), n = 8192 natively
// in an 8192-point tile (as two parts in a 4096-point one) and n > S as parts
// of S points on the in-place pipeline; smaller n, the 32-element shape and
// the chirp-z tiles run on the Stockham stages (M = 16384 chirp-z tiles in a
// kernel of their own: one 16384-point tile per CTA, 1024 threads).
template <int S, int T, bool CHIRP>
__device__ __forceinline__ void fcfb_tile_dispatch(int log2n, float2* sm, const TileMeta* meta, int count,
                                                   const FcfbTileConst& c, const BluDesc* bd) {
  constexpr int LOGS = ilog2c(S);
  constexpr bool IP = S / T == 16;
  if constexpr (CHIRP && LOGS == CHIRP_LOGM_MAX) {
    fcfb_tile_chirp<CHIRP_LOGM_MAX, S, T>(sm, meta, count, c, bd);   // the 16384-point tiles' own kernel
  } else if constexpr (CHIRP) {
    switch (log2n - BLU_TAG) {
      case 4: fcfb_tile_chirp<4, S, T>(sm, meta, count, c, bd); break;
      case 5: fcfb_tile_chirp<5, S, T>(sm, meta, count, c, bd); break;
      case 6: fcfb_tile_chirp<6, S, T>(sm, meta, count, c, bd); break;
      case 7: fcfb_tile_chirp<7, S, T>(sm, meta, count, c, bd); break;
      case 8: fcfb_tile_chirp<8, S, T>(sm, meta, count, c, bd); break;
      case 9: fcfb_tile_chirp<9, S, T>(sm, meta, count, c, bd); break;
      case 10: fcfb_tile_chirp<10, S, T>(sm, meta, count, c, bd); break;
      case 11: fcfb_tile_chirp<11, S, T>(sm, meta, count, c, bd); break;
      case 12: if constexpr (LOGS >= 12) fcfb_tile_chirp<12, S, T>(sm, meta, count, c, bd); break;
      case 13: if constexpr (LOGS >= 13) fcfb_tile_chirp<13, S, T>(sm, meta, count, c, bd); break;
    }
  } else {
    if (log2n > LOGS) {
      switch (log2n - LOGS) {
        case 1: if constexpr (IP) fcfb_tile_part_ip<S, T, 1>(sm, meta, c); else fcfb_tile_part<S, T, 1>(sm, meta, c); break;
        case 2: if constexpr (IP) fcfb_tile_part_ip<S, T, 2>(sm, meta, c); else fcfb_tile_part<S, T, 2>(sm, meta, c); break;
        case 3: if constexpr (IP) fcfb_tile_part_ip<S, T, 3>(sm, meta, c); else fcfb_tile_part<S, T, 3>(sm, meta, c); break;
      }
      return;
    }
    if constexpr (S == 8192 && T == 512) {                 // n <= 4096: two independent halves
      switch (log2n) {
        case 2: fcfb_tile_halves<2>(sm, meta, count, c); return;
        case 3: fcfb_tile_halves<3>(sm, meta, count, c); return;
        case 4: fcfb_tile_halves<4>(sm, meta, count, c); return;
        case 5: fcfb_tile_halves<5>(sm, meta, count, c); return;
        case 6: fcfb_tile_halves<6>(sm, meta, count, c); return;
        case 7: fcfb_tile_halves<7>(sm, meta, count, c); return;
        case 8: fcfb_tile_halves<8>(sm, meta, count, c); return;
        case 9: fcfb_tile_halves<9>(sm, meta, count, c); return;
        case 10: fcfb_tile_halves<10>(sm, meta, count, c); return;
        case 11: fcfb_tile_halves<11>(sm, meta, count, c); return;
        case 12: fcfb_tile_halves<12>(sm, meta, count, c); return;
      }
    }
    switch (log2n) {
      case 2: fcfb_tile<2, S, T>(sm, meta, count, c); break;
      case 3: fcfb_tile<3, S, T>(sm, meta, count, c); break;
      case 4: fcfb_tile<4, S, T>(sm, meta, count, c); break;
      case 5: fcfb_tile<5, S, T>(sm, meta, count, c); break;
      case 6: fcfb_tile<6, S, T>(sm, meta, count, c); break;
      case 7: fcfb_tile<7, S, T>(sm, meta, count, c); break;
      case 8: fcfb_tile<8, S, T>(sm, meta, count, c); break;
      case 9: if constexpr (IP) fcfb_tile_ip<9, S, T>(sm, meta, count, c); else fcfb_tile<9, S, T>(sm, meta, count, c); break;
      case 10: if constexpr (IP) fcfb_tile_ip<10, S, T>(sm, meta, count, c); else fcfb_tile<10, S, T>(sm, meta, count, c); break;
      case 11: if constexpr (IP) fcfb_tile_ip<11, S, T>(sm, meta, count, c); else fcfb_tile<11, S, T>(sm, meta, count, c); break;
      case 12:
        if constexpr (LOGS >= 12) {
          if constexpr (IP) fcfb_tile_ip<12, S, T>(sm, meta, count, c); else fcfb_tile<12, S, T>(sm, meta, count, c);
        }
        break;
      case 13:
        if constexpr (LOGS >= 13) {
          if constexpr (IP) fcfb_tile_8k<T>(sm, meta, c); else fcfb_tile<13, S, T>(sm, meta, count, c);
        }
        break;
    }
  }
}

}  // namespace sk
