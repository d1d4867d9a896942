// FP32 FFT building blocks for sm_100a: complex helpers and in-register DFTs
// of 2..32 points, used by the tile pipelines (sk_fcfb.cuh: Stockham stages;
// sk_fcfb_ip.cuh: in-place stages).  A Stockham stage of radix R on
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

// Shared-memory index policy of the Stockham stages (sk_fcfb.cuh).
struct PadX {
  __device__ __forceinline__ int operator()(int e) const { return padx(e); }
};

}  // namespace sk
