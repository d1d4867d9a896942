// Device kernels of the filter-bank + Welch path.
//
// Per input buffer of B overlapped blocks (block b = samples [b*hop, b*hop+N)
// of [N/4 carried samples | 3N/4*B new samples], main.rs:162-181, dsp.rs:150-155):
//   fwd_fft_kernel      raw samples -> converted, scaled by scaling/N, forward
//                       FFT of size Nc (N/2 complex pairs for real input, N for
//                       complex) -> Z                                       [multifft.rs]
//   welch_split_kernel  Z -> X (K bins, real-input split), and the Welch term
//                       |X[k] - (X[k-1]+X[k+1])/2|^2 per block -> P        [spectrum.rs:90-111]
//   welch_accum_kernel  P -> running f32 accumulator in block order, emits and
//                       quantises records                                  [spectrum.rs:112-161]
//   fcfb_kernel         per channel and block: gather n bins (modulo/mirror),
//                       times weights, inverse FFT, keep [n/8, 7n/8)        [fcfb.rs:154-188]
//   fcfb_backward_kernel adjoint of fcfb_kernel for weight design
#pragma once
#include "sk_fft.cuh"
#include "sk_fcfb.cuh"

namespace sk {

constexpr int TILE_S = 8192;   // complex elements per tile (64 KB + padding in shared memory)
constexpr int TILE_T = 256;    // threads per tile CTA (32 elements per thread)

struct ChanDev {               // one filter-bank channel, as the kernels see it
  const float2* w;             // weights, natural order: w[j] scales bin first+j
  float2* out;                 // B * 3n/4 outputs
  long long first;
  int log2n;
  int pad;
};
struct BwdChan {
  const float2* w;
  const float2* dy;            // B * 3n/4 output gradients
  float2* dw;                  // n weight gradients (accumulated)
  long long first;
  int log2n;
  int pad;
};
struct TileDesc {              // S/n transforms of one size
  int log2n;
  int list_off;                // first entry in the (channel, block) list
  int count;                   // transforms in this tile (<= S/n)
  int pad;
};

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
  __device__ __forceinline__ float2 pair(long long p) const {
    constexpr int BASE = FMT & 0x3F;
    constexpr bool CPLX = (FMT & 0xC0) == 0x40;
    if (p < overlap) return *reinterpret_cast<const float2*>(halo + (CPLX ? 2 * p : p));
    const long long q = p - overlap;
    if constexpr (CPLX) return make_float2(load_comp<BASE>(raw, 2 * q), load_comp<BASE>(raw, 2 * q + 1));
    return make_float2(load_comp<BASE>(raw, q), load_comp<BASE>(raw, q + 1));
  }
};

// ----------------------------------------------------------------- forward FFT
struct FwdArgs {
  const uint8_t* raw;          // new samples of this buffer
  const float* halo;           // converted last N/4 samples of the previous buffer
  float* halo_next;            // receives the converted last N/4 samples of this one
  long long overlap, nnew;
  int hop, B;
  int log2N, log2Nc;           // N (window length) and Nc (complex FFT length)
  int R1, log2R1;              // Nc = R1 * S when Nc > S (R1 = 1 otherwise)
  float wscale;                // rectangular window value scaling/N (dsp.rs:70-73)
  const float2* tw_tile;       // W_S^k
  const float2* tw_big;        // W_N^k, k < N
  float2* Z;                   // [B][Nc]; for R1 > 1 element k1 + R1*k2 sits at k1*S + k2
};

// Tile = S/Nc whole blocks (Nc <= S), or one residue class k1 of one block
// (Nc = R1*S): z'[j2] = W_Nc^{j2 k1} sum_j1 z[j1 S + j2] W_R1^{j1 k1}, whose
// S-point DFT is Z[k1 + R1 k2] (the last radix-R1 stage done first, as
// prototyping/parallel_fft.py:20-28 splits a 4-way FFT).
template <int S, int T, int FMT>
__global__ void __launch_bounds__(T, 2) fwd_fft_kernel(FwdArgs a) {
  extern __shared__ float2 sm[];
  constexpr bool CPLX = (FMT & 0xC0) == 0x40;
  constexpr int E = S / T;
  constexpr int LOGS = ilog2c(S);
  const SampleSrc<FMT> src{a.raw, a.halo, a.overlap};
  {  // carry: convert the last N/4 new samples for the next buffer (main.rs:173)
    const long long stride = (long long)gridDim.x * T;
    const long long ncomp = a.overlap * (CPLX ? 2 : 1);
    const long long base = (a.nnew - a.overlap) * (CPLX ? 2 : 1);
    for (long long h = (long long)blockIdx.x * T + threadIdx.x; h < ncomp; h += stride)
      a.halo_next[h] = load_comp<FMT & 0x3F>(a.raw, base + h);
  }
  const int tile = blockIdx.x;
  const int Nc = 1 << a.log2Nc;
  if (a.R1 == 1) {
    const int per = S >> a.log2Nc;
    const int b0 = tile * per;
#pragma unroll 4
    for (int k = 0; k < E; ++k) {
      const int e = threadIdx.x + k * T;
      const int b = b0 + (e >> a.log2Nc);
      const int j = e & (Nc - 1);
      float2 z = make_float2(0.f, 0.f);
      if (b < a.B) {
        z = src.pair((long long)b * a.hop + (CPLX ? j : 2 * j));
        z.x *= a.wscale;
        z.y *= a.wscale;
      }
      sm[padx(e)] = z;
    }
    __syncthreads();
    tile_fft<-1, S, T>(sm, a.tw_tile, a.log2Nc);
#pragma unroll 4
    for (int k = 0; k < E; ++k) {
      const int e = threadIdx.x + k * T;
      const int b = b0 + (e >> a.log2Nc);
      if (b < a.B) a.Z[((size_t)b << a.log2Nc) + (e & (Nc - 1))] = sm[padx(e)];
    }
  } else {
    const int b = tile >> a.log2R1;
    const int k1 = tile & (a.R1 - 1);
    const int shR = a.log2N - a.log2R1, shC = a.log2N - a.log2Nc;
    const long long p0 = (long long)b * a.hop;
#pragma unroll 2
    for (int k = 0; k < E; ++k) {
      const int e = threadIdx.x + k * T;
      float2 acc = make_float2(0.f, 0.f);
      for (int j1 = 0; j1 < a.R1; ++j1) {
        const int jj = (j1 << LOGS) + e;
        float2 z = src.pair(p0 + (CPLX ? jj : 2 * jj));
        z.x *= a.wscale;
        z.y *= a.wscale;
        const int m = (j1 * k1) & (a.R1 - 1);
        acc = cadd(acc, m == 0 ? z : cmul(z, __ldg(&a.tw_big[m << shR])));
      }
      if (k1) acc = cmul(acc, __ldg(&a.tw_big[(e * k1) << shC]));
      sm[padx(e)] = acc;
    }
    __syncthreads();
    tile_fft<-1, S, T>(sm, a.tw_tile, LOGS);
    float2* Zb = a.Z + ((size_t)b << a.log2Nc) + ((size_t)k1 << LOGS);
#pragma unroll 4
    for (int k = 0; k < E; ++k) {
      const int e = threadIdx.x + k * T;
      Zb[e] = sm[padx(e)];
    }
  }
}

// ----------------------------------------------------------------- Welch split
struct SplitArgs {
  const float2* Z;
  float2* X;                   // [B][K]
  float* P;                    // [B][K] Welch terms
  int log2N, log2Nc, K, R1, log2R1, logS;
  const float2* tw_big;        // W_N^k
};

__device__ __forceinline__ float2 z_at(const SplitArgs& a, const float2* Zb, int m) {
  return __ldg(&Zb[a.R1 == 1 ? m : ((m & (a.R1 - 1)) << a.logS) + (m >> a.log2R1)]);
}
// Real-input bin k in [0, N/2] from the N/2-point complex FFT of the packed
// pairs: X = (A + B)/2 - i W_N^k (A - B)/2 with A = Z[k], B = conj(Z[Nc-k]).
__device__ __forceinline__ float2 xr_at(const SplitArgs& a, const float2* Zb, int k) {
  const int Nc = 1 << a.log2Nc;
  const float2 za = z_at(a, Zb, k & (Nc - 1));
  const float2 zb = cconj(z_at(a, Zb, (Nc - k) & (Nc - 1)));
  const float2 s = cadd(za, zb), d = csub(za, zb);
  const float2 u = cmul(__ldg(&a.tw_big[k]), d);
  return make_float2(0.5f * s.x + 0.5f * u.y, 0.5f * s.y - 0.5f * u.x);
}
// get_bin (fftutil.rs:8-22) on the spectrum being formed.
template <bool REAL>
__device__ __forceinline__ float2 x_at(const SplitArgs& a, const float2* Zb, int kk) {
  const int N = 1 << a.log2N;
  const int m = kk & (N - 1);
  if constexpr (!REAL) return z_at(a, Zb, m);
  return m < a.K ? xr_at(a, Zb, m) : cconj(xr_at(a, Zb, N - m));
}

template <bool REAL>
__global__ void __launch_bounds__(256) welch_split_kernel(SplitArgs a) {
  __shared__ float2 xs[258];
  const int b = blockIdx.y;
  const int k0 = blockIdx.x * 256;
  const float2* Zb = a.Z + ((size_t)b << a.log2Nc);
  for (int idx = threadIdx.x; idx < 258; idx += 256) xs[idx] = x_at<REAL>(a, Zb, k0 - 1 + idx);
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

// ----------------------------------------------------------------- Welch accumulate
// acc[k] += P[b][k] in block order; every `averages` blocks a record is
// written (spectrum.rs:116-161) and the accumulator restarts.  fmt: 0 u8,
// 1 u16 big-endian, 2 f32 mean power.  The u8/u16 arithmetic is rounded per
// operation (no fused multiply-add) like the reference.
static __global__ void __launch_bounds__(256) welch_accum_kernel(const float* __restrict__ P, float* acc, int K, int B,
                                                          int accn0, int averages, int fmt, float db_plus,
                                                          uint8_t* out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  float s = acc[k];
  int cnt = accn0, r = 0;
  for (int b = 0; b < B; ++b) {
    s += __ldg(&P[(size_t)b * K + k]);
    if (++cnt >= averages) {
      const size_t o = (size_t)r * K + k;
      if (fmt == 2) {
        reinterpret_cast<float*>(out)[o] = __fdiv_rn(s, (float)cnt);
      } else {
        const float db = __fadd_rn(__fmul_rn(log10f(s), 10.0f), db_plus);
        if (fmt == 1) {
          const float q = fminf(fmaxf(__fadd_rn(__fmul_rn(db, 20.0f), 4000.0f), 0.0f), 4095.0f);
          const unsigned v = (unsigned)q;
          out[2 * o] = (uint8_t)(v >> 8);
          out[2 * o + 1] = (uint8_t)(v & 0xFF);
        } else {
          const float q = fminf(fmaxf(__fadd_rn(__fmul_rn(db, 2.0f), 250.0f), 0.0f), 255.0f);
          out[o] = (uint8_t)(unsigned)q;
        }
      }
      s = 0.0f;
      cnt = 0;
      ++r;
    }
  }
  acc[k] = s;
}

// ----------------------------------------------------------------- filter bank
struct FcfbArgs {
  const TileDesc* tiles;
  int ntiles;
  int* cursor;                 // persistent mode: next tile to claim
  const int2* list;            // (channel, block) per transform
  const ChanDev* chans;
  const float2* X;             // [B][K]
  int K, log2N;
  const float2* tw;            // W_S^k
};

template <int S, int T, bool PERSIST, bool REAL>
__global__ void __launch_bounds__(T, 2) fcfb_kernel(FcfbArgs a, int tile_base) {
  extern __shared__ float2 sm[];
  __shared__ TileMeta s_meta[MAX_TILE_TRANSFORMS];
  __shared__ int s_tile;
  static_assert(MAX_TILE_TRANSFORMS <= T, "one thread stages one transform's metadata");
  for (int it = 0;; ++it) {
    const FcfbTileConst c{1 << a.log2N, a.K, a.tw};
    int tile;
    if constexpr (PERSIST) {
      if (threadIdx.x == 0) s_tile = atomicAdd(a.cursor, 1);
      __syncthreads();               // also orders the previous tile's reads before this tile's writes
      tile = s_tile;
      if (tile >= a.ntiles) return;
    } else {
      if (it) return;
      tile = tile_base + blockIdx.x;
    }
    const TileDesc td = a.tiles[tile];
    if (threadIdx.x < td.count) {
      const int2 cb = __ldg(&a.list[td.list_off + threadIdx.x]);
      const ChanDev& ch = a.chans[cb.x];
      const int keep = 6 * ((1 << td.log2n) >> 3);
      TileMeta m;
      m.X = a.X + (size_t)cb.y * a.K;
      m.w = ch.w;
      m.out = ch.out + (size_t)cb.y * keep;
      m.first = (int)(ch.first & (long long)(c.N - 1));
      m.pad = 0;
      s_meta[threadIdx.x] = m;
    }
    __syncthreads();
    fcfb_tile_dispatch<S, T, REAL>(td.log2n, sm, s_meta, td.count, c);
  }
}

// Adjoint of fcfb_kernel.  With g = FFT_n(dy zero-padded to [n/8, 7n/8)) (the
// forward transform is the adjoint of the unnormalised inverse), v = w * G:
//   dW[j] += conj(G[j]) g,  dX[bin] += conj(w[j]) g  (conjugated for mirror bins).
struct BwdArgs {
  const TileDesc* tiles;
  const int2* list;
  const BwdChan* chans;
  const float2* X;
  float2* dX;                  // may be null
  int K, log2N;
  const float2* tw;
};

template <int S, int T, bool REAL>
__global__ void __launch_bounds__(T, 2) fcfb_backward_kernel(BwdArgs a) {
  extern __shared__ float2 sm[];
  constexpr int E = S / T;
  const int N = 1 << a.log2N;
  const TileDesc td = a.tiles[blockIdx.x];
  const int log2n = td.log2n, n = 1 << log2n, half = n >> 1;
  const int lo = n >> 3, keep = 6 * lo;
  for (int k = 0; k < E; ++k) {
    const int e = threadIdx.x + k * T;
    const int t = e >> log2n, i = e & (n - 1);
    float2 v = make_float2(0.f, 0.f);
    if (t < td.count && i >= lo && i < lo + keep) {
      const int2 cb = a.list[td.list_off + t];
      v = a.chans[cb.x].dy[(size_t)cb.y * keep + (i - lo)];
    }
    sm[padx(e)] = v;
  }
  __syncthreads();
  tile_fft<-1, S, T>(sm, a.tw, log2n);
  for (int k = 0; k < E; ++k) {
    const int e = threadIdx.x + k * T;
    const int t = e >> log2n, i = e & (n - 1);
    if (t >= td.count) continue;
    const int2 cb = a.list[td.list_off + t];
    const BwdChan& ch = a.chans[cb.x];
    const float2 g = sm[padx(e)];
    const int j = (i + half) & (n - 1);
    const int m = (int)((ch.first + j) & (long long)(N - 1));
    const bool mirror = REAL && m >= a.K;
    const size_t xi = (size_t)cb.y * a.K + (mirror ? N - m : m);
    const float2 G = mirror ? cconj(a.X[xi]) : a.X[xi];
    const float2 dw = cmul(cconj(G), g);
    atomicAdd(&ch.dw[j].x, dw.x);
    atomicAdd(&ch.dw[j].y, dw.y);
    if (a.dX) {
      float2 dg = cmul(cconj(ch.w[j]), g);
      if (mirror) dg = cconj(dg);
      atomicAdd(&a.dX[xi].x, dg.x);
      atomicAdd(&a.dX[xi].y, dg.y);
    }
  }
}

}  // namespace sk
