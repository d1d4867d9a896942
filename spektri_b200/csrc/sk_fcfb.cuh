// Tile pipelines: batched power-of-two FFTs whose first stage loads straight
// from global memory and whose last stage stores straight to it.
//
// A tile holds `count` transforms of n = 2^LOGN points (S/n at most).  The
// FFT runs as 1-3 Stockham stages (decimation in time, sk_fft.cuh) with the
// size fixed at compile time:
//   first stage : load(t, q, s) supplies input i = q + s n/R of transform t
//                 (a gather, a format conversion, ...), DFT_R, then shared
//                 memory (or the store directly when it is the only stage)
//   middle stage: shared -> twiddle -> DFT_R -> shared (in place)
//   last stage  : shared -> twiddle -> DFT_R -> store(t, q, u, v) for output
//                 o = q + u n/R
// The radix-digit index s (u) is a compile-time constant after unrolling, so a
// caller can turn index arithmetic on it (the filter bank's n/2 rotation of
// the inputs, its [n/8, 7n/8) output window) into immediate offsets and
// statically dropped stores.
// Shared memory is touched twice per element per middle/last stage; the first
// and last stages have global memory on their other side, so there is no
// in-place hazard: the last stage stays rolled over butterflies (one live at a
// time), the first is unrolled where the caller asks (UNROLL: all gathers of
// a thread in flight at once) and rolled otherwise.
//
// Users: fcfb_tile (filter bank: gather x weights, inverse FFT, keep
// [n/8, 7(n/8)), fcfb.rs:154-188) and the forward FFT kernel.
#pragma once
#include "sk_fft.cuh"
#include "sk_types.h"

namespace sk {

// log2 radices of the stages for a 2^LOGN-point transform.
// log2 radix of stage p (0 = none) for a 2^logn-point transform with E
// elements per thread: a stage of radix R needs R <= E, the first stage keeps
// R <= 16 (its R gathered inputs are live at once).
__host__ __device__ constexpr int stage_log_radix(int logn, int e, int p) {
  if (e >= 32) {
    // 4:[4] 8:[8] 16:[16] 32:[8,4] 64:[8,8] 128:[16,8] 256:[16,16] 512:[16,32]
    // 1024:[16,8,8] 2048:[16,8,16] 4096:[16,16,16] 8192:[16,16,32]
    constexpr int t[12][3] = {{2, 0, 0}, {3, 0, 0}, {4, 0, 0}, {3, 2, 0}, {3, 3, 0}, {4, 3, 0},
                              {4, 4, 0}, {4, 5, 0}, {4, 3, 3}, {4, 3, 4}, {4, 4, 4}, {4, 4, 5}};
    return p < 3 ? t[logn - 2][p] : 0;
  }
  // radix <= 16: ... 512:[8,8,8] 1024:[16,8,8] 2048:[16,16,8] 4096:[16,16,16] 8192:[16,16,16,2]
  // 16384:[16,16,16,4] (the chirp-z tiles of M = 16384)
  constexpr int u[13][4] = {{2, 0, 0, 0}, {3, 0, 0, 0}, {4, 0, 0, 0}, {3, 2, 0, 0}, {3, 3, 0, 0}, {4, 3, 0, 0},
                            {4, 4, 0, 0}, {3, 3, 3, 0}, {4, 3, 3, 0}, {4, 4, 3, 0}, {4, 4, 4, 0}, {4, 4, 4, 1},
                            {4, 4, 4, 2}};
  return u[logn - 2][p];
}

template <int LOGN, int E>
struct StagePlan {
  static constexpr int r0 = stage_log_radix(LOGN, E, 0), r1 = stage_log_radix(LOGN, E, 1),
                       r2 = stage_log_radix(LOGN, E, 2), r3 = stage_log_radix(LOGN, E, 3);
  static constexpr int ns = (r0 > 0) + (r1 > 0) + (r2 > 0) + (r3 > 0);
  static_assert(r0 + r1 + r2 + r3 == LOGN, "stages must cover the transform");
  // log2 radix of the last stage, and of the stride n/R between the outputs
  // q + u n/R that one butterfly of the last stage stores.
  static constexpr int last = ns == 1 ? r0 : ns == 2 ? r1 : ns == 3 ? r2 : r3;
  static constexpr int last_shift = LOGN - last;
  static constexpr int first_shift = LOGN - r0;   // the same stride for the first stage's inputs
};

// Powers w^s (s = 1..R-1) of a stage twiddle w = W_P^j, P = 2^(13 - SH) (the
// stage's span times radix), conjugated for DIR > 0.  Only w^1, w^4 and w^16
// come from the stage's table (consecutive j at consecutive entries); the
// other powers are products of at most three of them (w^(16a + 4b + c) =
// w^16a w^4b w^c), which keeps each twiddle within a few ulps while cutting
// the table reads of a radix-R stage from R-1 to at most 3.
template <int R, int SH, int DIR>
struct TwiddlePowers {
  float2 lo[4], mid[4], hi;                              // w^c (c < 4), w^4b (b < 4), w^16
  __device__ __forceinline__ TwiddlePowers(const float2* __restrict__ tw, int j) {
    constexpr int p = TILE_LOGS - SH;
    auto ld = [&](int si) {
      float2 w = __ldg(&tw[stage_tw_offset(p, si) + j]);  // forward W_P^(j s); inverse uses its conjugate
      if (DIR > 0) w.y = -w.y;
      return w;
    };
    lo[1] = ld(0);
    if constexpr (R > 2) lo[2] = cmul(lo[1], lo[1]);
    if constexpr (R > 3) lo[3] = cmul(lo[2], lo[1]);
    if constexpr (R > 4) mid[1] = ld(1);
    if constexpr (R > 8) mid[2] = cmul(mid[1], mid[1]);
    if constexpr (R > 12) mid[3] = cmul(mid[2], mid[1]);
    hi = make_float2(1.f, 0.f);
    if constexpr (R > 16) hi = ld(2);
  }
  // w^s for 1 <= s < R (s compile-time after unrolling).
  __device__ __forceinline__ float2 pow(int s) const {
    const int a = s >> 4, b = (s >> 2) & 3, c = s & 3;
    if (b == 0 && a == 0) return lo[c];
    float2 w = b ? mid[b] : hi;
    if (a && b) w = cmul(hi, w);
    if (c) w = cmul(w, lo[c]);
    return w;
  }
};

// v <- DFT_R(v[s] w^s) with the powers of TwiddlePowers.  Each first-level
// butterfly (inputs i0 and i1 = i0 + R/2) scales x0 by w^i0 and folds x1 w^i1
// into two FMAs per component, the difference as 2 p - u: 10 instructions
// per pair instead of 12 (6 instead of 8 for i0 = 0).
template <int R, int SH, int DIR>
__device__ __forceinline__ void twiddle_dft(float2* v, const float2* __restrict__ tw, int j) {
  const TwiddlePowers<R, SH, DIR> w(tw, j);
  auto leaf = [&](int i0, int i1, float2 x0, float2 x1, float2& u, float2& d) {
    const float2 p = i0 ? cmul(x0, w.pow(i0)) : x0;
    const float2 w1 = w.pow(i1);
    u = make_float2(__fmaf_rn(x1.x, w1.x, __fmaf_rn(-x1.y, w1.y, p.x)),
                    __fmaf_rn(x1.x, w1.y, __fmaf_rn(x1.y, w1.x, p.y)));
    d = make_float2(__fmaf_rn(2.0f, p.x, -u.x), __fmaf_rn(2.0f, p.y, -u.y));
  };
  DftLeaf<R, DIR>::run(v, leaf);
}

// The threads and the barrier a tile pipeline runs on: the whole CTA
// (threadIdx.x, __syncthreads), or one 256-thread half of a 512-thread CTA
// (named barrier 1 + half), so that two halves run independent tiles.
struct CtaCtx {
  __device__ __forceinline__ int tid() const { return threadIdx.x; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};
struct HalfCtx {
  int t, bar;                                    // thread index in the half; named barrier id
  __device__ __forceinline__ int tid() const { return t; }
  __device__ __forceinline__ void sync() const { asm volatile("bar.sync %0, 256;" ::"r"(bar) : "memory"); }
};

// Stage 1 (span L = 1): butterfly q of transform t takes inputs
// i = q + s n/R (load(t, q, s), s = 0..R-1 compile-time after unrolling) and
// writes y[q R + u]; as the only stage (n = R, q = 0) it stores output u
// through store(t, 0, u).
template <int LOGN, int R, int S, int T, int DIR, bool LAST, bool UNROLL, class Load, class Store,
          class Ctx = CtaCtx>
__device__ __forceinline__ void stage_first(float2* sm, int count, Load& load, Store& store, const Ctx& ctx = Ctx()) {
  constexpr int LOGR = ilog2c(R), LOGNR = LOGN - LOGR, NB = S / (R * T);
  static_assert(NB >= 1, "radix too large for the tile");
#pragma unroll (UNROLL ? NB : 1)
  for (int bb = 0; bb < NB; ++bb) {
    const int beta = ctx.tid() + bb * T;
    const int t = beta >> LOGNR, q = beta & ((1 << LOGNR) - 1);
    float2 v[R];
    if (t < count) {
#pragma unroll
      for (int s = 0; s < R; ++s) v[s] = load(t, q, s);
    } else {
#pragma unroll
      for (int s = 0; s < R; ++s) v[s] = make_float2(0.f, 0.f);
    }
    dft<R, DIR>(v);
    if constexpr (LAST) {
      if (t < count) {
#pragma unroll
        for (int u = 0; u < R; ++u) store(t, 0, u, v[u]);
      }
    } else {
#pragma unroll
      for (int u = 0; u < R; ++u) sm[padx((t << LOGN) + q * R + u)] = v[u];
    }
  }
}

// Stages 2..: span L = 2^LOGL (LOGL = 0: a first stage run from shared
// memory, in place).  LAST: q < L, g = 0, output o = q + u L stored through
// store(t, q, u, v) (u compile-time after unrolling).
template <int LOGN, int R, int LOGL, int S, int T, int DIR, bool LAST, class Store, class Pad = PadX,
          class Ctx = CtaCtx>
__device__ __forceinline__ void stage_next(float2* sm, int count, const float2* __restrict__ tw, Store& store,
                                           const Pad& pad = Pad(), const Ctx& ctx = Ctx()) {
  constexpr int LOGR = ilog2c(R), LOGNR = LOGN - LOGR, NB = S / (R * T);
  constexpr int SH = TILE_LOGS - LOGL - LOGR;            // stage tables: P = 2^(LOGL + LOGR)
  // SH = -1: the span-4096 radix-4 stage of a 16384-point transform, whose
  // twiddle powers come from the appended p = 14 table (w^1 only)
  static_assert(NB >= 1 && (SH >= 0 || (SH == -1 && R <= 4)), "bad stage");
  auto twiddled_dft = [&](float2* v, int j) {            // DFT_R(v[s] w^s); no twiddle for LOGL = 0
    if constexpr (LOGL > 0) twiddle_dft<R, SH, DIR>(v, tw, j);
    else dft<R, DIR>(v);
  };
  if constexpr (LAST) {
#pragma unroll 1
    for (int bb = 0; bb < NB; ++bb) {
      const int beta = ctx.tid() + bb * T;
      const int t = beta >> LOGNR, q = beta & ((1 << LOGNR) - 1);
      const int base = t << LOGN;
      float2 v[R];
#pragma unroll
      for (int s = 0; s < R; ++s) v[s] = sm[pad(base + q + (s << LOGNR))];
      twiddled_dft(v, q);
      if (t < count) {
#pragma unroll
        for (int u = 0; u < R; ++u) store(t, q, u, v[u]);
      }
    }
  } else {
    float2 v[NB][R];
#pragma unroll
    for (int bb = 0; bb < NB; ++bb) {
      const int beta = ctx.tid() + bb * T;
      const int t = beta >> LOGNR, q = beta & ((1 << LOGNR) - 1);
      const int base = t << LOGN;
#pragma unroll
      for (int s = 0; s < R; ++s) v[bb][s] = sm[pad(base + q + (s << LOGNR))];
      twiddled_dft(v[bb], q & ((1 << LOGL) - 1));
    }
    ctx.sync();
#pragma unroll
    for (int bb = 0; bb < NB; ++bb) {
      const int beta = ctx.tid() + bb * T;
      const int t = beta >> LOGNR, q = beta & ((1 << LOGNR) - 1);
      const int j = q & ((1 << LOGL) - 1), g = q >> LOGL;
      const int ob = (t << LOGN) + (g << (LOGL + LOGR)) + j;
#pragma unroll
      for (int u = 0; u < R; ++u) sm[pad(ob + (u << LOGL))] = v[bb][u];
    }
  }
}

// The whole transform of every tile entry.  The caller syncs before (shared
// memory free) and after (if it reuses shared memory).
template <int LOGN, int S, int T, int DIR, bool UNROLL, class Load, class Store, class Ctx = CtaCtx>
__device__ __forceinline__ void tile_pipeline(float2* sm, int count, const float2* __restrict__ tw, Load& load,
                                              Store& store, const Ctx& ctx = Ctx()) {
  using P = StagePlan<LOGN, S / T>;
  if constexpr (P::ns == 1) {
    stage_first<LOGN, 1 << P::r0, S, T, DIR, true, UNROLL>(sm, count, load, store, ctx);
  } else if constexpr (P::ns == 2) {
    stage_first<LOGN, 1 << P::r0, S, T, DIR, false, UNROLL>(sm, count, load, store, ctx);
    ctx.sync();
    stage_next<LOGN, 1 << P::r1, P::r0, S, T, DIR, true>(sm, count, tw, store, PadX(), ctx);
  } else if constexpr (P::ns == 3) {
    stage_first<LOGN, 1 << P::r0, S, T, DIR, false, UNROLL>(sm, count, load, store, ctx);
    ctx.sync();
    stage_next<LOGN, 1 << P::r1, P::r0, S, T, DIR, false>(sm, count, tw, store, PadX(), ctx);
    ctx.sync();
    stage_next<LOGN, 1 << P::r2, P::r0 + P::r1, S, T, DIR, true>(sm, count, tw, store, PadX(), ctx);
  } else {
    stage_first<LOGN, 1 << P::r0, S, T, DIR, false, UNROLL>(sm, count, load, store, ctx);
    ctx.sync();
    stage_next<LOGN, 1 << P::r1, P::r0, S, T, DIR, false>(sm, count, tw, store, PadX(), ctx);
    ctx.sync();
    stage_next<LOGN, 1 << P::r2, P::r0 + P::r1, S, T, DIR, false>(sm, count, tw, store, PadX(), ctx);
    ctx.sync();
    stage_next<LOGN, 1 << P::r3, P::r0 + P::r1 + P::r2, S, T, DIR, true>(sm, count, tw, store, PadX(), ctx);
  }
}

// Forward M-point FFT of load() left in shared memory in natural order, each
// element e of a transform times H[e] in place, then the inverse M-point FFT
// stored through store().  The inverse's first stage reads shared memory
// (LOGL = 0), so every stage but the very last writes in place.
template <int LOGM, int S, int T, class Load, class Store>
__device__ __forceinline__ void tile_chirp(float2* sm, int count, const float2* __restrict__ tw, Load& load,
                                           const float2* __restrict__ H, Store& store) {
  using P = StagePlan<LOGM, S / T>;
  stage_first<LOGM, 1 << P::r0, S, T, -1, false, true>(sm, count, load, store);
  __syncthreads();
  if constexpr (P::ns >= 2) {
    stage_next<LOGM, 1 << P::r1, P::r0, S, T, -1, false>(sm, count, tw, store);
    __syncthreads();
  }
  if constexpr (P::ns >= 3) {
    stage_next<LOGM, 1 << P::r2, P::r0 + P::r1, S, T, -1, false>(sm, count, tw, store);
    __syncthreads();
  }
  if constexpr (P::ns >= 4) {
    stage_next<LOGM, 1 << P::r3, P::r0 + P::r1 + P::r2, S, T, -1, false>(sm, count, tw, store);
    __syncthreads();
  }
#pragma unroll 4
  for (int k = 0; k < S / T; ++k) {                     // pointwise product, element by element in place
    const int e = threadIdx.x + k * T;
    const int i = padx(e);
    sm[i] = cmul(sm[i], __ldg(&H[e & ((1 << LOGM) - 1)]));
  }
  __syncthreads();
  if constexpr (P::ns == 1) {
    stage_next<LOGM, 1 << P::r0, 0, S, T, +1, true>(sm, count, tw, store);
  } else {
    stage_next<LOGM, 1 << P::r0, 0, S, T, +1, false>(sm, count, tw, store);
    __syncthreads();
    if constexpr (P::ns == 2) {
      stage_next<LOGM, 1 << P::r1, P::r0, S, T, +1, true>(sm, count, tw, store);
    } else if constexpr (P::ns == 3) {
      stage_next<LOGM, 1 << P::r1, P::r0, S, T, +1, false>(sm, count, tw, store);
      __syncthreads();
      stage_next<LOGM, 1 << P::r2, P::r0 + P::r1, S, T, +1, true>(sm, count, tw, store);
    } else {
      stage_next<LOGM, 1 << P::r1, P::r0, S, T, +1, false>(sm, count, tw, store);
      __syncthreads();
      stage_next<LOGM, 1 << P::r2, P::r0 + P::r1, S, T, +1, false>(sm, count, tw, store);
      __syncthreads();
      stage_next<LOGM, 1 << P::r3, P::r0 + P::r1 + P::r2, S, T, +1, true>(sm, count, tw, store);
    }
  }
}

// ------------------------------------------------------------------ filter bank
// The filter bank reads the spectra in an extended layout: per block a row of
// xs >= N + maxn bins holding get_bin(X, N, m) (fftutil.rs:8-22) at every
// m < xs, i.e. bin m mod N, conjugate-mirrored for real input.  A channel's n
// bins (first + j) mod N, j < n, are then the contiguous run starting at
// first mod N, with no modulo, mirror test or select per element.
struct TileMeta {
  const float2* X;     // extended spectrum row of the block, from bin first mod N
  const float2* w;     // weights, natural order
  float2* out;         // output row of the block: 6(n/8) samples
  int pad;             // split transforms (n > S): the part, i.e. the output residue mod n/S
  int unused;
};

struct FcfbTileConst {
  const float2* tw;        // tile twiddle table (W_8192^k, then the stage tables)
  const float2* tw_split;  // W_Ns^k, k < Ns = 2^log_split: the twiddles of split transforms (n > S)
  int log_split;
};

// Weighted input of the IFFT (fcfb.rs:166-172): buf[i] = W[j] bin(first + j),
// j = (i + n/2) mod n.  With i = q + s n/R (first-stage digit s, q < n/R),
// j = q + ((s + R/2) mod R) n/R: a compile-time offset from q once s is.
template <int LOGN, int R>
__device__ __forceinline__ float2 fcfb_input(const TileMeta& m, int q, int s) {
  constexpr int LOGNR = LOGN - ilog2c(R);
  const int j = q + (((s + R / 2) & (R - 1)) << LOGNR);
  return cmul(__ldg(&m.w[j]), __ldg(&m.X[j]));
}

// Output o = q + u n/R of the last stage lands at o - n/8 when kept
// ([n/8, 7n/8), fcfb.rs:177).  For R >= 8 the window edges fall on digit
// boundaries (n/8 = (R/8) n/R), so kept-or-not depends on the compile-time u
// alone: the dropped quarter costs no test and no store.
template <int LOGN, int RL, class Emit>
__device__ __forceinline__ void fcfb_keep(int q, int u, Emit emit) {
  constexpr int n = 1 << LOGN, lo = n >> 3, keep = 6 * lo, SHL = LOGN - ilog2c(RL);
  if constexpr (keep > 0) {                                 // n = 4 keeps nothing
    if constexpr (RL >= 8) {
      if (u >= RL / 8 && u < 7 * RL / 8) emit(q + ((u - RL / 8) << SHL));
    } else {
      const int k = q + (u << SHL) - lo;
      if ((unsigned)k < (unsigned)keep) emit(k);
    }
  }
}

template <int LOGN, int S, int T, class Ctx = CtaCtx>
__device__ __forceinline__ void fcfb_tile(float2* sm, const TileMeta* meta, int count, const FcfbTileConst& c,
                                          const Ctx& ctx = Ctx()) {
  using P = StagePlan<LOGN, S / T>;
  constexpr int R0 = 1 << P::r0, RL = 1 << P::last;
  auto load = [&](int t, int q, int s) { return fcfb_input<LOGN, R0>(meta[t], q, s); };
  auto store = [&](int t, int q, int u, float2 v) {
    fcfb_keep<LOGN, RL>(q, u, [&](int k) { meta[t].out[k] = v; });
  };
  tile_pipeline<LOGN, S, T, +1, true>(sm, count, c.tw, load, store, ctx);
}

// v times e^{+2 pi i k/P} for a runtime k < P (P <= 8): exact swaps and
// negations for multiples of a quarter turn, one product otherwise.
template <int P>
__device__ __forceinline__ float2 rot_inv(float2 v, int k) {
  constexpr int Q = P / 4;                                  // k = Q: a quarter turn (P >= 4)
  if constexpr (P == 2) return k ? make_float2(-v.x, -v.y) : v;
  if constexpr (P >= 4) {
    if constexpr (P == 8) {
      if (k & 1) {                                          // odd eighth turns: times (1 + i)/sqrt(2), then quarter turns
        const float h = 0.70710678118654752440f;
        v = make_float2(h * (v.x - v.y), h * (v.x + v.y));
        k -= 1;
      }
    }
    const int qt = (k / Q) & 3;
    if (qt == 1) return make_float2(-v.y, v.x);
    if (qt == 2) return make_float2(-v.x, -v.y);
    if (qt == 3) return make_float2(v.y, -v.x);
  }
  return v;
}

// One part r of an n = P S transform in an S-point tile (count = 1,
// meta.pad = r; P = 2, 4, 8).  With buf the shifted, weighted input
// (buf[i] = W[j] bin(first + j), j = (i + n/2) mod n), the inverse DFT
// splits by output residue mod P:
//   y[P k + r] = IDFT_S(z_r)[k],
//   z_r[i]     = e^{+2 pi i i r/n} sum_m buf[i + m S] e^{+2 pi i m r/P}
// so the P parts are independent S-point transforms; each gathers all n
// inputs (buf[i + m S] has j = i + ((m + P/2) mod P) S) and keeps its
// residue of [n/8, 7(n/8)): y[P k + r] is kept iff k is in [S/8, 7S/8), the
// same digit window as an S-point transform's, at P (k - S/8) + r.  The
// twiddle e^{+2 pi i i r/n} is the conjugate of W_n^(i r) from the split
// table (W_Ns^k, Ns the largest such n of the plan).
template <int S, int LOGP>
__device__ __forceinline__ float2 part_input(const TileMeta& m, const FcfbTileConst& c, int i) {
  constexpr int LOGS = ilog2c(S), P = 1 << LOGP, LOGN = LOGS + LOGP;
  const int r = m.pad;
  // W_n^k: the tile table itself when n = 8192 (compile-time offsets), else
  // the split table at k << shn
  const float2* __restrict__ twn = LOGN == TILE_LOGS ? c.tw : c.tw_split;
  const int shn = LOGN == TILE_LOGS ? 0 : c.log_split - LOGN;
  float2 z;
  if constexpr (P == 2) {                                   // y[2k] from buf[i] + buf[i + S], y[2k+1] from the difference
    const float2 a = cmul(__ldg(&m.w[i + S]), __ldg(&m.X[i + S]));
    const float2 b = cmul(__ldg(&m.w[i]), __ldg(&m.X[i]));
    if (r == 0) return cadd(a, b);
    z = csub(a, b);
  } else {
#pragma unroll
    for (int mm = 0; mm < P; ++mm) {
      const int j = i + (((mm + P / 2) & (P - 1)) << LOGS);
      const float2 b = cmul(__ldg(&m.w[j]), __ldg(&m.X[j]));
      z = mm ? cadd(z, rot_inv<P>(b, (mm * r) & (P - 1))) : b;
    }
    if (r == 0) return z;
  }
  const float2 t = __ldg(&twn[(i * r) << shn]);
  return cmul(z, make_float2(t.x, -t.y));
}

template <int S, int T, int LOGP>
__device__ __forceinline__ void fcfb_tile_part(float2* sm, const TileMeta* meta, const FcfbTileConst& c) {
  constexpr int LOGS = ilog2c(S), P = 1 << LOGP;
  using PL = StagePlan<LOGS, S / T>;
  constexpr int RL = 1 << PL::last;
  const TileMeta& m = meta[0];
  auto load = [&](int, int q, int s) { return part_input<S, LOGP>(m, c, q + (s << PL::first_shift)); };
  auto store = [&](int, int q, int u, float2 v) {
    fcfb_keep<LOGS, RL>(q, u, [&](int k) { m.out[P * k + m.pad] = v; });
  };
  tile_pipeline<LOGS, S, T, +1, true>(sm, 1, c.tw, load, store);
}

// A chirp-z tile: count transforms of one size n (not a power of two).  With
// buf the shifted, weighted input and c[i] = exp(+i pi i^2/n),
//   y[k] = c[k] sum_i (buf[i] c[i]) conj(c[k - i])        (fcfb.rs:171-177)
// is a convolution, done as IFFT_M(FFT_M(buf c) * H) with H the 1/M-scaled
// transform of conj(c[d]) wrapped modulo M; only the kept outputs
// [n/8, 7(n/8)) are formed (times c[k]) and stored.  These tiles run in a
// kernel of their own, so the power-of-two tiles' register allocation is
// not shaped by them.
template <int LOGM, int S, int T>
__device__ __forceinline__ void fcfb_tile_chirp(float2* sm, const TileMeta* meta, int count, const FcfbTileConst& c,
                                                const BluDesc* __restrict__ bd) {
  using P = StagePlan<LOGM, S / T>;
  const int n = bd->n, half = n >> 1, lo = n >> 3, keep = 6 * lo;
  const float2* __restrict__ chirp = bd->chirp;
  const float2* __restrict__ H = bd->H;
  auto load = [&](int t, int q, int s) {
    const int i = q + (s << P::first_shift);
    if (i >= n) return make_float2(0.f, 0.f);
    const int j = i < n - half ? i + half : i - (n - half);  // (i + n/2) mod n, fcfb.rs:166-169
    const float2 x = cmul(__ldg(&meta[t].w[j]), __ldg(&meta[t].X[j]));
    return cmul(x, __ldg(&chirp[i]));
  };
  auto store = [&](int t, int q, int u, float2 v) {
    const int o = q + (u << P::last_shift), k = o - lo;
    if ((unsigned)k < (unsigned)keep) meta[t].out[k] = cmul(v, __ldg(&chirp[o]));
  };
  tile_chirp<LOGM, S, T>(sm, count, c.tw, load, H, store);
}

}  // namespace sk
