// FP32 FFT building blocks for sm_100a: complex helpers, in-register DFTs of
// 2..32 points, and the shared-memory "tile" engine that runs S/n independent
// n-point transforms (n a power of two, 4 <= n <= S) with T threads.
//
// Tile engine (Stockham autosort, decimation in time).  A stage of radix R on
// sub-transforms of span L maps, inside each n-point transform,
//   q in [0, n/R):  j = q mod L,  g = q div L,
//   a_s = x[q + s n/R] * W_{LR}^{j s}            (s = 0..R-1)
//   y[g L R + j + t L] = sum_s a_s W_R^{s t}     (t = 0..R-1)
// and after the last stage (L R = n) y holds the DFT in natural order.
// W_m = exp(DIR 2 pi i / m): DIR = -1 forward, +1 inverse (both unnormalised,
// the conventions of the reference's FFT library).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sk {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

__host__ __device__ constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v >> 1); }

// cos(pi m / 16) for m = 0..8 (first quadrant of W_32).
__host__ __device__ constexpr float kC32(int m) {
  return m == 0 ? 1.0f : m == 1 ? 0.98078528040323044912f : m == 2 ? 0.92387953251128675613f
       : m == 3 ? 0.83146961230254523708f : m == 4 ? 0.70710678118654752440f
       : m == 5 ? 0.55557023301960222474f : m == 6 ? 0.38268343236508977173f
       : m == 7 ? 0.19509032201612826785f : 0.0f;
}
__host__ __device__ constexpr float cos32(int m) {
  return m <= 8 ? kC32(m) : m <= 16 ? -kC32(16 - m) : m <= 24 ? -kC32(m - 16) : kC32(32 - m);
}
__host__ __device__ constexpr float sin32(int m) {
  return m <= 8 ? kC32(8 - m) : m <= 16 ? kC32(m - 8) : m <= 24 ? -kC32(24 - m) : -kC32(m - 24);
}

// v * W_32^m for a compile-time m (after unrolling); exact for m = 0, 8, 16, 24.
template <int DIR>
__device__ __forceinline__ float2 twmul32(float2 v, int m) {
  if (m == 0) return v;
  if (m == 16) return make_float2(-v.x, -v.y);
  if (m == 8) return DIR < 0 ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);    // * (DIR i)
  if (m == 24) return DIR < 0 ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);   // * (-DIR i)
  const float c = cos32(m), s = DIR * sin32(m);
  return make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
}

// Radix-2 butterfly (e + W_32^m o, e - W_32^m o) for a compile-time m, with
// the twiddle folded into fused multiply-adds: 6 instructions instead of 8
// where W_32^m is not a multiple of i.  For |cos| = |sin| (m = 4, 12, 20, 28)
// both outputs are c (o.x -/+ o.y, ...) + e and -c (...) + e; otherwise
// u = e + W o is two FMAs per component and e - W o = 2e - u.
template <int DIR>
__device__ __forceinline__ void bfly32(float2 e, float2 o, int m, float2& u, float2& v) {
  if ((m & 7) == 0) {
    const float2 t = twmul32<DIR>(o, m);
    u = cadd(e, t);
    v = csub(e, t);
  } else if ((m & 3) == 0) {
    const float c = cos32(m), r = DIR * sin32(m) / cos32(m);   // r = +-1, exact
    const float dx = o.x - r * o.y, dy = r * o.x + o.y;
    u = make_float2(__fmaf_rn(c, dx, e.x), __fmaf_rn(c, dy, e.y));
    v = make_float2(__fmaf_rn(-c, dx, e.x), __fmaf_rn(-c, dy, e.y));
  } else {
    const float c = cos32(m), s = DIR * sin32(m);
    u = make_float2(__fmaf_rn(o.x, c, __fmaf_rn(-o.y, s, e.x)), __fmaf_rn(o.x, s, __fmaf_rn(o.y, c, e.y)));
    v = make_float2(__fmaf_rn(2.0f, e.x, -u.x), __fmaf_rn(2.0f, e.y, -u.y));
  }
}

// In-register R-point DFT (R = 1..32), recursive radix-2 decimation in time:
// DFT_R(a) from DFT_{R/2} of the even and odd samples.  Every index is affine
// in unrolled loop counters, so the whole transform stays in registers.
template <int R, int DIR>
struct Dft {
  static __device__ __forceinline__ void run(float2* a) {
    constexpr int H = R / 2;
    float2 e[H], o[H];
#pragma unroll
    for (int i = 0; i < H; ++i) { e[i] = a[2 * i]; o[i] = a[2 * i + 1]; }
    Dft<H, DIR>::run(e);
    Dft<H, DIR>::run(o);
#pragma unroll
    for (int k = 0; k < H; ++k) bfly32<DIR>(e[k], o[k], k * (32 / R), a[k], a[k + H]);
  }
};
template <int DIR>
struct Dft<1, DIR> {
  static __device__ __forceinline__ void run(float2*) {}
};
template <int DIR>
struct Dft<2, DIR> {
  static __device__ __forceinline__ void run(float2* a) {
    const float2 u = a[0], v = a[1];
    a[0] = cadd(u, v);
    a[1] = csub(u, v);
  }
};
template <int R, int DIR>
__device__ __forceinline__ void dft(float2* a) { Dft<R, DIR>::run(a); }

// The same DFT with its first radix-2 level left to the caller: element i of
// `a` is input OFF + i STRIDE of the whole transform, and each two-point leaf
// calls leaf(i0, i1, x0, x1, u, v), i1 = i0 + R/2, which must set u = x0' + x1'
// and v = x0' - x1' for its own scaled inputs x' (e.g. x times a twiddle).
template <int R, int DIR, int STRIDE = 1, int OFF = 0>
struct DftLeaf {
  template <class Leaf>
  static __device__ __forceinline__ void run(float2* a, Leaf& leaf) {
    constexpr int H = R / 2;
    float2 e[H], o[H];
#pragma unroll
    for (int i = 0; i < H; ++i) { e[i] = a[2 * i]; o[i] = a[2 * i + 1]; }
    DftLeaf<H, DIR, 2 * STRIDE, OFF>::run(e, leaf);
    DftLeaf<H, DIR, 2 * STRIDE, OFF + STRIDE>::run(o, leaf);
#pragma unroll
    for (int k = 0; k < H; ++k) bfly32<DIR>(e[k], o[k], k * (32 / R), a[k], a[k + H]);
  }
};
template <int DIR, int STRIDE, int OFF>
struct DftLeaf<2, DIR, STRIDE, OFF> {
  template <class Leaf>
  static __device__ __forceinline__ void run(float2* a, Leaf& leaf) {
    const float2 x0 = a[0], x1 = a[1];
    leaf(OFF, OFF + STRIDE, x0, x1, a[0], a[1]);
  }
};

// Shared-memory index with one pad slot per 16 float2: radix-R scatters at
// stride R (R <= 16) then land in distinct 8-byte banks of a half warp.
__device__ __forceinline__ int padx(int a) { return a + (a >> 4); }
template <int S>
struct TileShape {
  static constexpr int LOGS = ilog2c(S);
  static constexpr int SMEM_ELEMS = S + S / 16;
  static constexpr size_t SMEM_BYTES = sizeof(float2) * (size_t)SMEM_ELEMS;
};

// Shared-memory index policies: padx, and padx plus one slot per transform
// (for tiles written column-wise, one transform per column: with 2^logn-point
// transforms the column stride n + n/16 + 1 is odd in 8-byte slots for
// n >= 32, so a warp writing 32 consecutive columns hits every bank pair).
struct PadX {
  __device__ __forceinline__ int operator()(int e) const { return padx(e); }
};
struct PadCols {
  int logn;
  __device__ __forceinline__ int operator()(int e) const { return padx(e) + (e >> logn); }
};

// One Stockham stage of radix R over the whole tile (S/n transforms).
// Reads, sync, writes, sync: the caller syncs before the first stage.
// tw: forward table W_S^k, k in [0, S).
template <int R, int DIR, int S, int T, class Pad = PadX>
__device__ __forceinline__ void tile_stage(float2* sm, const float2* __restrict__ tw, int log2n, int log2L,
                                           const Pad& pad = Pad()) {
  constexpr int NB = S / (R * T);
  static_assert(NB >= 1, "radix larger than elements per thread");
  constexpr int LOGR = ilog2c(R);
  constexpr int LOGS = ilog2c(S);
  const int log2nR = log2n - LOGR;
  float2 v[NB][R];
  int ob[NB];
#pragma unroll
  for (int bb = 0; bb < NB; ++bb) {
    const int beta = threadIdx.x + bb * T;
    const int t = beta >> log2nR;
    const int q = beta & ((1 << log2nR) - 1);
    const int j = q & ((1 << log2L) - 1);
    const int g = q >> log2L;
    const int base = t << log2n;
#pragma unroll
    for (int s = 0; s < R; ++s) v[bb][s] = sm[pad(base + q + (s << log2nR))];
    if (log2L > 0) {
      const int sh = LOGS - log2L - LOGR;       // S / (L R) = 2^sh
#pragma unroll
      for (int s = 1; s < R; ++s) {
        float2 w = __ldg(&tw[(j * s) << sh]);
        if (DIR > 0) w.y = -w.y;
        v[bb][s] = cmul(v[bb][s], w);
      }
    }
    dft<R, DIR>(v[bb]);
    ob[bb] = base + (g << (log2L + LOGR)) + j;
  }
  __syncthreads();
#pragma unroll
  for (int bb = 0; bb < NB; ++bb) {
#pragma unroll
    for (int u = 0; u < R; ++u) sm[pad(ob[bb] + (u << log2L))] = v[bb][u];
  }
  __syncthreads();
}

// log2 of the radix of stage p for a 2^log2n-point transform (0 = no stage).
__device__ __forceinline__ int stage_radix(int log2n, int p) {
  // 4:[4] 8:[8] 16:[16] 32:[32] 64:[8,8] 128:[16,8] 256:[16,16] 512:[16,32]
  // 1024:[32,32] 2048:[16,16,8] 4096:[16,16,16] 8192:[16,16,32]
  switch (log2n) {
    case 2: return p == 0 ? 2 : 0;
    case 3: return p == 0 ? 3 : 0;
    case 4: return p == 0 ? 4 : 0;
    case 5: return p == 0 ? 5 : 0;
    case 6: return p < 2 ? 3 : 0;
    case 7: return p == 0 ? 4 : p == 1 ? 3 : 0;
    case 8: return p < 2 ? 4 : 0;
    case 9: return p == 0 ? 4 : p == 1 ? 5 : 0;
    case 10: return p < 2 ? 5 : 0;
    case 11: return p < 2 ? 4 : p == 2 ? 3 : 0;
    case 12: return p < 3 ? 4 : 0;
    case 13: return p < 2 ? 4 : p == 2 ? 5 : 0;
  }
  return 0;
}

// All stages of a batched 2^log2n-point FFT over the tile in shared memory.
template <int DIR, int S, int T, class Pad = PadX>
__device__ __forceinline__ void tile_fft(float2* sm, const float2* __restrict__ tw, int log2n, const Pad& pad = Pad()) {
  int log2L = 0;
#pragma unroll 1
  for (int p = 0; p < 3; ++p) {
    const int lr = stage_radix(log2n, p);
    if (lr == 0) break;
    switch (lr) {
      case 2: tile_stage<4, DIR, S, T>(sm, tw, log2n, log2L, pad); break;
      case 3: tile_stage<8, DIR, S, T>(sm, tw, log2n, log2L, pad); break;
      case 4: tile_stage<16, DIR, S, T>(sm, tw, log2n, log2L, pad); break;
      case 5: tile_stage<32, DIR, S, T>(sm, tw, log2n, log2L, pad); break;
    }
    log2L += lr;
  }
}

}  // namespace sk
