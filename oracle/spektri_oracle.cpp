// FP32 CPU restatement of the spektri filter-bank + Welch spectrum path.
//
// TEST INFRASTRUCTURE ONLY.  The product library and host never link, load or
// run this file; tests, the smoke check and the benchmark's CPU-baseline leg
// use it as the checker ("port" baseline: the Rust reference cannot be built
// without a Rust toolchain).
//
// Follows the reference (tejeez/spektri) step by step, in f32 like the reference:
//   main.rs:113-193         stream loop: N/4 zero prefix, overlap carry, drop a short tail
//   inputformats.rs:12-155  the 12 input formats
//   dsp.rs:70-79,114-160    rectangular window scaling/N, block slicing, stage order
//   multifft.rs:34-95       complex FFTs; two real blocks packed in one complex FFT
//   spectrum.rs:82-163      Hann-by-convolution, f32 accumulation in block order,
//                           u8 / u16-BE dB quantisation, emission rule
//   fftutil.rs:8-22         modulo / conjugate-mirror bin access
//   fcfb.rs:66-203,225-285  gather x weights, inverse FFT, keep [n/8, 7n/8), bin maths
//   data.rs:110-171         24-byte metadata and topics
// The FFT arithmetic of the reference lives in rustfft 6.0.1 (crates.io, not in
// the reference tree); it is restated here from the DFT definition
// (unnormalised, exponent sign -1 forward / +1 inverse, any size) as a
// mixed-radix Stockham FFT with f64-computed twiddles rounded to f32.
// Threads split the work as rayon does in the reference: block pairs for the
// forward FFTs (multifft.rs:57), filters for the filter bank (fcfb.rs:74).
// The reference's fixed 100000-byte per-filter output buffer (fcfb.rs:51) is
// not restated: records of any size are produced.
//
// Extensions beside the reference behaviour (off unless asked for):
//   spectrum format 2 = f32 mean power acc/accn; filter keys tw=<bins> (Tukey
//   weights) and w=<file> (complex64 weights); --fake-clock=<secs>,<step_ns>.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

struct cf { float re, im; };
static inline cf cadd(cf a, cf b) { return {a.re + b.re, a.im + b.im}; }
static inline cf csub(cf a, cf b) { return {a.re - b.re, a.im - b.im}; }
static inline cf cmul(cf a, cf b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

// ------------------------------------------------------------------ FFT plan
// Stockham autosort: stage (radix R, span L): for q in [0,n/R): j=q%L, g=q/L,
// a_s = x[q + s n/R] * W_{LR}^{j s};  y[g L R + j + t L] = sum_s a_s W_R^{s t}.
struct FftPlan {
  int n = 0, sign = -1;
  std::vector<int> radices;
  std::vector<std::vector<cf>> tw;   // per stage: [s-1][j], s in 1..R-1, j in 0..L-1
  std::vector<std::vector<cf>> wr;   // per stage: W_R^k for generic radices
  std::vector<std::vector<float>> twr, twi;   // the same twiddles split into real and imaginary parts
  bool soa = false;                  // every radix 4 or 2: the structure-of-arrays path

  FftPlan() {}
  FftPlan(int n_, int sign_) : n(n_), sign(sign_) {
    int m = n;
    while (m % 4 == 0 && m > 0) { radices.push_back(4); m /= 4; }
    while (m % 2 == 0 && m > 0) { radices.push_back(2); m /= 2; }
    for (int p = 3; m > 1; p += 2) while (m % p == 0) { radices.push_back(p); m /= p; }
    int L = 1;
    for (int R : radices) {
      std::vector<cf> t((size_t)(R - 1) * L);
      for (int s = 1; s < R; ++s)
        for (int j = 0; j < L; ++j) {
          long long e = (long long)j * s % ((long long)L * R);
          double a = sign * 2.0 * M_PI * (double)e / ((double)L * R);
          t[(size_t)(s - 1) * L + j] = {(float)std::cos(a), (float)std::sin(a)};
        }
      tw.push_back(std::move(t));
      std::vector<cf> w(R);
      for (int k = 0; k < R; ++k) {
        double a = sign * 2.0 * M_PI * k / R;
        w[k] = {(float)std::cos(a), (float)std::sin(a)};
      }
      wr.push_back(std::move(w));
      std::vector<float> tr(tw.back().size()), ti(tw.back().size());
      for (size_t k = 0; k < tr.size(); ++k) { tr[k] = tw.back()[k].re; ti[k] = tw.back()[k].im; }
      twr.push_back(std::move(tr));
      twi.push_back(std::move(ti));
      L *= R;
    }
    soa = n > 1;
    for (int R : radices) soa = soa && (R == 4 || R == 2);
  }

  // One radix-4 (R = 4) or radix-2 stage of span L on split real/imaginary
  // arrays, with exactly the arithmetic of the generic butterfly below (the
  // same products and sums in the same order, so the same bits); for L >= 8
  // the inner loop runs along j, contiguous on both sides, which the compiler
  // vectorises.
  template <int R, int SIGN>
  static inline void bfly_soa(int q, int o, int j, int L, int stride, const float* __restrict__ sr,
                              const float* __restrict__ si, float* __restrict__ dr, float* __restrict__ di,
                              const float* __restrict__ tr, const float* __restrict__ ti) {
    const float x0r = sr[q], x0i = si[q];
    if (R == 2) {
      const float ar = sr[q + stride], ai = si[q + stride], wr_ = tr[j], wi_ = ti[j];
      const float x1r = ar * wr_ - ai * wi_, x1i = ar * wi_ + ai * wr_;
      dr[o] = x0r + x1r; di[o] = x0i + x1i;
      dr[o + L] = x0r - x1r; di[o + L] = x0i - x1i;
    } else {
      const float a1r = sr[q + stride], a1i = si[q + stride];
      const float a2r = sr[q + 2 * stride], a2i = si[q + 2 * stride];
      const float a3r = sr[q + 3 * stride], a3i = si[q + 3 * stride];
      const float w1r = tr[j], w1i = ti[j], w2r = tr[L + j], w2i = ti[L + j], w3r = tr[2 * L + j], w3i = ti[2 * L + j];
      const float x1r = a1r * w1r - a1i * w1i, x1i = a1r * w1i + a1i * w1r;
      const float x2r = a2r * w2r - a2i * w2i, x2i = a2r * w2i + a2i * w2r;
      const float x3r = a3r * w3r - a3i * w3i, x3i = a3r * w3i + a3i * w3r;
      const float s02r = x0r + x2r, s02i = x0i + x2i, d02r = x0r - x2r, d02i = x0i - x2i;
      const float s13r = x1r + x3r, s13i = x1i + x3i, d13r = x1r - x3r, d13i = x1i - x3i;
      const float r13r = SIGN < 0 ? d13i : -d13i, r13i = SIGN < 0 ? -d13r : d13r;   // d13 * (sign i)
      dr[o] = s02r + s13r;         di[o] = s02i + s13i;
      dr[o + L] = d02r + r13r;     di[o + L] = d02i + r13i;
      dr[o + 2 * L] = s02r - s13r; di[o + 2 * L] = s02i - s13i;
      dr[o + 3 * L] = d02r - r13r; di[o + 3 * L] = d02i - r13i;
    }
  }

  // One radix-4 (R = 4) or radix-2 stage of span L on split real/imaginary
  // arrays, with exactly the arithmetic of the generic butterfly below (the
  // same products and sums in the same order, so the same bits); for L >= 8
  // the inner loop runs along j, contiguous on both sides, which the compiler
  // vectorises.
  template <int R, int SIGN>
  void stage_soa(int st, int L, const float* __restrict__ sr, const float* __restrict__ si, float* __restrict__ dr,
                 float* __restrict__ di) const {
    const int stride = n / R, groups = n / (L * R);
    const float* __restrict__ tr = twr[st].data();
    const float* __restrict__ ti = twi[st].data();
    if (L >= 8) {
      for (int g = 0; g < groups; ++g) {
        const float* __restrict__ s0r = sr + g * L;
        const float* __restrict__ s0i = si + g * L;
        float* __restrict__ d0r = dr + g * L * R;
        float* __restrict__ d0i = di + g * L * R;
#pragma GCC ivdep
        for (int j = 0; j < L; ++j) bfly_soa<R, SIGN>(j, j, j, L, stride, s0r, s0i, d0r, d0i, tr, ti);
      }
    } else if (L == 1) {
      stage_short<R, SIGN, 1>(groups, stride, sr, si, dr, di, tr, ti);
    } else if (L == 2) {
      stage_short<R, SIGN, 2>(groups, stride, sr, si, dr, di, tr, ti);
    } else {
      stage_short<R, SIGN, 4>(groups, stride, sr, si, dr, di, tr, ti);
    }
  }

  // Short spans (L = 1, 2, 4) with L a compile-time constant, so the loop over
  // groups has constant strides (interleaved stores the compiler can vectorise).
  template <int R, int SIGN, int LC>
  static void stage_short(int groups, int stride, const float* __restrict__ sr, const float* __restrict__ si,
                          float* __restrict__ dr, float* __restrict__ di, const float* __restrict__ tr,
                          const float* __restrict__ ti) {
#pragma GCC ivdep
    for (int g = 0; g < groups; ++g)
      for (int j = 0; j < LC; ++j) bfly_soa<R, SIGN>(g * LC + j, g * LC * R + j, j, LC, stride, sr, si, dr, di, tr, ti);
  }

  void run_soa(cf* x) const {
    thread_local std::vector<float> buf;
    if (buf.size() < 4 * (size_t)n) buf.resize(4 * (size_t)n);
    float *ar = buf.data(), *ai = ar + n, *br = ai + n, *bi = br + n;
    for (int k = 0; k < n; ++k) { ar[k] = x[k].re; ai[k] = x[k].im; }
    int L = 1;
    for (size_t st = 0; st < radices.size(); ++st) {
      const int R = radices[st];
      if (R == 4) { if (sign < 0) stage_soa<4, -1>((int)st, L, ar, ai, br, bi); else stage_soa<4, 1>((int)st, L, ar, ai, br, bi); }
      else        { if (sign < 0) stage_soa<2, -1>((int)st, L, ar, ai, br, bi); else stage_soa<2, 1>((int)st, L, ar, ai, br, bi); }
      std::swap(ar, br);
      std::swap(ai, bi);
      L *= R;
    }
    for (int k = 0; k < n; ++k) x[k] = {ar[k], ai[k]};
  }

  // In place on x (n values) using scratch y (n values).
  void run(cf* x, cf* y) const {
    if (n <= 1) return;
    if (soa) { run_soa(x); return; }
    cf* src = x; cf* dst = y;
    int L = 1;
    for (size_t st = 0; st < radices.size(); ++st) {
      const int R = radices[st];
      const int stride = n / R;
      const int groups = n / (L * R);
      const cf* t = tw[st].data();
      const cf* w = wr[st].data();
      auto bfly = [&](int g, int j) {
        const int q = g * L + j;
        cf a[64];
        cf* av = R <= 64 ? a : nullptr;
        std::vector<cf> big;
        if (!av) { big.resize(R); av = big.data(); }
        av[0] = src[q];
        for (int s = 1; s < R; ++s) av[s] = cmul(src[q + s * stride], t[(size_t)(s - 1) * L + j]);
        cf* o = dst + (size_t)g * L * R + j;
        if (R == 4) {
          cf s02 = cadd(av[0], av[2]), d02 = csub(av[0], av[2]);
          cf s13 = cadd(av[1], av[3]), d13 = csub(av[1], av[3]);
          // W_4 = sign*i: d13 * (sign*i)
          cf r13 = sign < 0 ? cf{d13.im, -d13.re} : cf{-d13.im, d13.re};
          o[0] = cadd(s02, s13);
          o[L] = cadd(d02, r13);
          o[2 * L] = csub(s02, s13);
          o[3 * L] = csub(d02, r13);
        } else if (R == 2) {
          o[0] = cadd(av[0], av[1]);
          o[L] = csub(av[0], av[1]);
        } else {
          for (int tt = 0; tt < R; ++tt) {
            cf acc = av[0];
            for (int s = 1; s < R; ++s) acc = cadd(acc, cmul(av[s], w[(long long)s * tt % R]));
            o[(size_t)tt * L] = acc;
          }
        }
      };
      if (L >= 8) { for (int g = 0; g < groups; ++g) for (int j = 0; j < L; ++j) bfly(g, j); }
      else        { for (int j = 0; j < L; ++j) for (int g = 0; g < groups; ++g) bfly(g, j); }
      std::swap(src, dst);
      L *= R;
    }
    if (src != x) std::memcpy(x, src, sizeof(cf) * (size_t)n);
  }
};

// ------------------------------------------------------------------ threads
template <class F>
void parallel_for(int count, int nthreads, F f) {
  if (nthreads <= 1 || count <= 1) { for (int i = 0; i < count; ++i) f(i); return; }
  std::atomic<int> next{0};
  int nt = std::min(nthreads, count);
  std::vector<std::thread> th;
  th.reserve(nt);
  for (int k = 0; k < nt; ++k)
    th.emplace_back([&] { for (int i; (i = next.fetch_add(1)) < count;) f(i); });
  for (auto& t : th) t.join();
}

// ------------------------------------------------------------------ formats
// inputformats.rs:12-62 (format codes from data.rs:79-96)
bool fmt_complex(int c) { return (c & 0xC0) == 0x40; }
int fmt_bits(int c) { int b = (c >> 1) & 7; return b == 2 ? 8 : b == 4 ? 16 : b == 6 ? 32 : 0; }
bool fmt_valid(int c) {
  switch (c) {
    case 0x04: case 0x08: case 0x09: case 0x1C: case 0x1D: case 0x24:
    case 0x44: case 0x48: case 0x49: case 0x5C: case 0x5D: case 0x64: return true;
  }
  return false;
}
int fmt_bytes(int c) { return fmt_bits(c) / 8 * (fmt_complex(c) ? 2 : 1); }
float fmt_scaling(int c) {
  int b = fmt_bits(c);
  if (b == 8) return 1.0f / 127.0f;
  if (b == 16) return 1.0f / 32767.0f;
  return 1.0f;
}
// One scalar component (inputformats.rs:65-155).
inline float conv1(const uint8_t* p, int c) {
  int base = c & 0x3F;   // strip the complex bit
  switch (base) {
    case 0x04: return (float)(int8_t)p[0];
    case 0x08: { int16_t v = (int16_t)(p[0] | (p[1] << 8)); return (float)v; }
    case 0x09: { int16_t v = (int16_t)(p[1] | (p[0] << 8)); return (float)v; }
    case 0x1C: { uint32_t u = p[0] | (p[1] << 8) | (p[2] << 16) | ((uint32_t)p[3] << 24); float f; std::memcpy(&f, &u, 4); return f; }
    case 0x1D: { uint32_t u = p[3] | (p[2] << 8) | (p[1] << 16) | ((uint32_t)p[0] << 24); float f; std::memcpy(&f, &u, 4); return f; }
    case 0x24: return (float)p[0] - 127.4f;
  }
  return 0.0f;
}

// ------------------------------------------------------------------ bins
// fcfb.rs:225-285
long long nearest_multiple(double value, long long multiple) {
  double r = std::round(value / (double)multiple) * (double)multiple;
  if (std::isnan(r)) return 0;                       // Rust `as isize` saturates, NaN -> 0
  if (r >= 9.2233720368547758e18) return INT64_MAX;
  if (r <= -9.2233720368547758e18) return INT64_MIN;
  return (long long)r;
}
bool freq_to_bins(double fs, double fc, long long N, double fs_out, double fc_out, long long* bins, long long* first) {
  double spacing = fs / (double)N;
  long long b = nearest_multiple(fs_out / spacing, 4);
  long long center = nearest_multiple((fc_out - fc) / spacing, 4);
  if (b > 0) { *bins = b; *first = center - b / 2; return true; }
  return false;
}
void bins_to_freq(double fs, double fc, long long N, long long bins, long long first, double* fs_out, double* fc_out) {
  double spacing = fs / (double)N;
  *fs_out = spacing * (double)bins;
  *fc_out = fc + spacing * (double)(first + bins / 2);
}
bool freq_to_bins_exact(double fs, double fc, long long N, double fs_out, double fc_out, long long* bins, long long* first) {
  if (!freq_to_bins(fs, fc, N, fs_out, fc_out, bins, first)) return false;
  double a, b;
  bins_to_freq(fs, fc, N, *bins, *first, &a, &b);
  return a == fs_out && b == fc_out;
}

// fcfb.rs:197-203 in f32
std::vector<cf> raised_cosine(int n) {
  const float PI = 3.14159265358979323846f;
  float f = (2.0f * PI) / (float)n;
  std::vector<cf> w(n);
  for (int i = 0; i < n; ++i) w[i] = {0.5f - 0.5f * std::cos((float)i * f), 0.0f};
  return w;
}
// Periodic Tukey window, tw taper bins per side (prototyping/fcfb.py:122).
std::vector<cf> tukey(int n, int tw) {
  std::vector<cf> w(n);
  if (tw <= 0) { for (auto& v : w) v = {1.0f, 0.0f}; return w; }
  double alpha = 2.0 * tw / n;
  int m = n + 1;
  if (alpha >= 1.0) {
    for (int k = 0; k < n; ++k) w[k] = {(float)(0.5 - 0.5 * std::cos(2.0 * M_PI * k / n)), 0.0f};
    return w;
  }
  int width = (int)std::floor(alpha * (m - 1) / 2.0);
  for (int k = 0; k < n; ++k) {
    double v = 1.0;
    if (k <= width) v = 0.5 * (1 + std::cos(M_PI * (-1 + 2.0 * k / alpha / (m - 1))));
    else if (k >= m - width - 1) v = 0.5 * (1 + std::cos(M_PI * (-2.0 / alpha + 1 + 2.0 * k / alpha / (m - 1))));
    w[k] = {(float)v, 0.0f};
  }
  return w;
}

// fftutil.rs:8-22
inline cf get_bin(const cf* X, long long N, long long K, long long i) {
  long long m = ((i % N) + N) % N;
  if (m < K) return X[m];
  cf v = X[N - m];
  return {v.re, -v.im};
}

// data.rs:110-132
void put_u64(uint8_t* p, uint64_t v) { for (int i = 0; i < 8; ++i) p[i] = (uint8_t)(v >> (8 * i)); }
void put_u32(uint8_t* p, uint32_t v) { for (int i = 0; i < 4; ++i) p[i] = (uint8_t)(v >> (8 * i)); }
void put_f64(uint8_t* p, double v) { uint64_t u; std::memcpy(&u, &v, 8); put_u64(p, u); }
void metadata24(uint8_t* p, uint64_t seq, uint64_t secs, uint32_t nanos) {
  put_u64(p, seq); put_u64(p + 8, secs); put_u32(p + 16, nanos); put_u32(p + 20, 0);
}
void topic24(uint8_t* p, uint8_t type, uint8_t fmt, double a, double b) {
  std::memset(p, 0, 24); p[0] = 2; p[1] = type; p[2] = fmt; put_f64(p + 8, a); put_f64(p + 16, b);
}

}  // namespace

// ====================================================================== state
struct orc_params {
  double fs_in, fc_in;
  int32_t fft_size, ffts_per_buf, averages, input_format, spectrum_format, n_threads;
};
struct orc_filter {
  double fs_out, fc_out;
  const float* weights;      // complex64 [bins], natural order; NULL -> reference raised cosine
  int32_t transition;        // >0 and weights NULL: Tukey with that taper width
};

struct Chan {
  long long bins, first;
  std::vector<cf> w;
  FftPlan ifft;
  std::vector<long long> gi;   // get_bin's modulo and mirror (fftutil.rs:8-22) for IFFT input i:
  std::vector<uint8_t> gc;     // spectrum index and whether to conjugate
};

struct orc_state {
  orc_params p;
  bool cplx;
  long long N, overlap, hop, nnew, total, K;
  float window;
  std::vector<float> rbuf;          // real input buffer [total]
  std::vector<cf> cbuf;             // complex input buffer [total]
  std::vector<cf> X;                // [B][K]
  std::vector<float> acc;
  uint32_t accn = 0;
  uint64_t spec_seq = 0;
  FftPlan fft;
  std::vector<Chan> ch;
};

static int spec_bytes(int f) { return f == 0 ? 1 : f == 1 ? 2 : 4; }

extern "C" {

orc_state* orc_create(const orc_params* p, const orc_filter* f, int32_t nf, int32_t* status) {
  if (!fmt_valid(p->input_format) || p->fft_size < 4 || p->ffts_per_buf < 1 || p->averages < 1) return nullptr;
  auto* s = new orc_state();
  s->p = *p;
  s->cplx = fmt_complex(p->input_format);
  if (!s->cplx && (p->ffts_per_buf % 2)) { delete s; return nullptr; }   // multifft.rs:57-61 pairs blocks
  s->N = p->fft_size;
  s->overlap = s->N / 4;                 // dsp.rs:77
  s->hop = s->N - s->overlap;            // dsp.rs:78
  s->nnew = s->hop * p->ffts_per_buf;    // dsp.rs:107-110
  s->total = s->nnew + s->overlap;
  s->K = s->cplx ? s->N : s->N / 2 + 1;  // dsp.rs:79
  s->window = fmt_scaling(p->input_format) / (float)s->N;   // dsp.rs:70-73
  if (s->cplx) s->cbuf.assign(s->total, {0, 0}); else s->rbuf.assign(s->total, 0.0f);
  s->X.assign((size_t)s->K * p->ffts_per_buf, {0, 0});
  s->acc.assign(s->K, 0.0f);
  s->fft = FftPlan((int)s->N, -1);
  for (int i = 0; i < nf; ++i) {
    long long bins, first;
    bool ok = freq_to_bins_exact(p->fs_in, p->fc_in, s->N, f[i].fs_out, f[i].fc_out, &bins, &first);
    if (status) status[i] = ok ? 0 : -2;
    if (!ok) continue;                   // fcfb.rs:58-61 drops invalid filters
    Chan c;
    c.bins = bins; c.first = first;
    if (f[i].weights) {
      c.w.resize(bins);
      std::memcpy(c.w.data(), f[i].weights, sizeof(cf) * bins);
    } else if (f[i].transition > 0) {
      c.w = tukey((int)bins, f[i].transition);
    } else {
      c.w = raised_cosine((int)bins);
    }
    c.ifft = FftPlan((int)bins, +1);
    const long long shift = bins / 2, NN = s->N, KK = s->K;
    c.gi.resize(bins);
    c.gc.resize(bins);
    for (long long i = 0; i < (long long)bins; ++i) {
      const long long m = (((c.first + (i + shift) % bins) % NN) + NN) % NN;
      c.gi[i] = m < KK ? m : NN - m;
      c.gc[i] = m < KK ? 0 : 1;
    }
    s->ch.push_back(std::move(c));
  }
  return s;
}

void orc_destroy(orc_state* s) { delete s; }

int32_t orc_info(const orc_state* s, int64_t* nnew, int64_t* overlap, int32_t* K, int32_t* nch) {
  if (nnew) *nnew = s->nnew;
  if (overlap) *overlap = s->overlap;
  if (K) *K = (int32_t)s->K;
  if (nch) *nch = (int32_t)s->ch.size();
  return 0;
}

int32_t orc_channel(const orc_state* s, int32_t i, int64_t* bins, int64_t* first) {
  if (i < 0 || i >= (int)s->ch.size()) return -1;
  *bins = s->ch[i].bins; *first = s->ch[i].first;
  return 0;
}

int32_t orc_max_spectra(const orc_state* s) {
  return (int32_t)((s->p.ffts_per_buf + s->p.averages - 1) / s->p.averages + 1);
}

// One buffer of `new` raw samples.  chan_out[c] receives B*3n/4 complex64.
// spec_out receives n_spec records of K values each in the spectrum format
// (u8, u16 big-endian, or f32 = acc/accn), without metadata.
int32_t orc_process(orc_state* s, const uint8_t* raw, float* const* chan_out, void* spec_out,
                    int32_t* n_spec, uint64_t* spec_seq0) {
  const long long N = s->N, K = s->K, B = s->p.ffts_per_buf, I = s->hop;
  const int fmt = s->p.input_format, nth = std::max(1, s->p.n_threads);
  const int bps = fmt_bytes(fmt);
  // main.rs:173 then main.rs:181
  const long long nchunk = 64, chunk = (s->nnew + nchunk - 1) / nchunk;
  if (s->cplx) {
    std::memmove(s->cbuf.data(), s->cbuf.data() + s->nnew, sizeof(cf) * s->overlap);
    int half = bps / 2;
    parallel_for((int)nchunk, nth, [&](int c) {
      for (long long i = c * chunk; i < std::min(s->nnew, (c + 1) * chunk); ++i)
        s->cbuf[s->overlap + i] = {conv1(raw + i * bps, fmt), conv1(raw + i * bps + half, fmt)};
    });
  } else {
    std::memmove(s->rbuf.data(), s->rbuf.data() + s->nnew, sizeof(float) * s->overlap);
    parallel_for((int)nchunk, nth, [&](int c) {
      for (long long i = c * chunk; i < std::min(s->nnew, (c + 1) * chunk); ++i)
        s->rbuf[s->overlap + i] = conv1(raw + i * bps, fmt);
    });
  }
  const float w = s->window;
  // multifft.rs:34-95
  if (s->cplx) {
    parallel_for((int)B, nth, [&](int b) {
      std::vector<cf> y(N);
      cf* o = s->X.data() + (size_t)b * K;
      const cf* in = s->cbuf.data() + b * I;
      for (long long j = 0; j < N; ++j) o[j] = {in[j].re * w, in[j].im * w};   // apply_window
      s->fft.run(o, y.data());
    });
  } else {
    parallel_for((int)(B / 2), nth, [&](int pr) {
      std::vector<cf> buf(N), y(N);
      const float* in0 = s->rbuf.data() + (2 * pr) * I;
      const float* in1 = s->rbuf.data() + (2 * pr + 1) * I;
      for (long long j = 0; j < N; ++j) buf[j] = {in0[j] * w, in1[j] * w};
      s->fft.run(buf.data(), y.data());
      cf* o0 = s->X.data() + (size_t)(2 * pr) * K;
      cf* o1 = s->X.data() + (size_t)(2 * pr + 1) * K;
      for (long long i = 0; i < K; ++i) {
        cf r = buf[i], m = buf[i == 0 ? 0 : N - i];
        o0[i] = {0.5f * (r.re + m.re), 0.5f * (r.im - m.im)};
        o1[i] = {0.5f * (r.im + m.im), 0.5f * (-r.re + m.re)};
      }
    });
  }
  // spectrum.rs:82-163.  Records complete at fixed blocks of the buffer, so
  // the bins run in parallel ranges, each bin's terms summed in block order
  // (the same additions as a loop over blocks outside, bins inside).
  if (spec_seq0) *spec_seq0 = s->spec_seq;
  const int sb = spec_bytes(s->p.spectrum_format);
  std::vector<long long> emit_at;                  // blocks after which a record completes
  {
    uint32_t a = s->accn;
    for (long long b = 0; b < B; ++b)
      if (++a >= (uint32_t)s->p.averages) { emit_at.push_back(b); a = 0; }
  }
  const uint32_t accn0 = s->accn;
  const long long kchunk = 4096, nk = (K + kchunk - 1) / kchunk;
  parallel_for((int)nk, nth, [&](int kc) {
    const long long k0 = kc * kchunk, k1 = std::min(K, k0 + kchunk);
    for (long long k = k0; k < k1; ++k) {
      float a = s->acc[k];
      uint32_t cnt = accn0;
      int r = 0;
      const bool edge = k == 0 || k == K - 1;
      for (long long b = 0; b < B; ++b) {
        const cf* Xb = s->X.data() + (size_t)b * K;
        cf c0, cm, cp;
        if (edge) { c0 = get_bin(Xb, N, K, k); cm = get_bin(Xb, N, K, k - 1); cp = get_bin(Xb, N, K, k + 1); }
        else { c0 = Xb[k]; cm = Xb[k - 1]; cp = Xb[k + 1]; }
        cf c = {c0.re - (cm.re + cp.re) * 0.5f, c0.im - (cm.im + cp.im) * 0.5f};
        a += c.re * c.re + c.im * c.im;
        if (++cnt >= (uint32_t)s->p.averages) {
          uint8_t* out = (uint8_t*)spec_out + (size_t)r * K * sb;
          if (s->p.spectrum_format == 2) {
            float v = a / (float)cnt;
            std::memcpy(out + 4 * k, &v, 4);
          } else {
            float db_plus = std::log10((float)cnt) * -10.0f;
            float db = std::log10(a) * 10.0f + db_plus;
            if (s->p.spectrum_format == 1) {
              float q = std::fmin(std::fmax(db * 20.0f + 4000.0f, 0.0f), 4095.0f);   // fmax(NaN,0)=0 like f32::max
              uint16_t o = (uint16_t)q;
              out[2 * k] = (uint8_t)(o >> 8); out[2 * k + 1] = (uint8_t)(o & 0xFF);
            } else {
              float q = std::fmin(std::fmax(db * 2.0f + 250.0f, 0.0f), 255.0f);
              out[k] = (uint8_t)q;
            }
          }
          a = 0.0f;
          cnt = 0;
          ++r;
        }
      }
      s->acc[k] = a;
    }
  });
  const int ns = (int)emit_at.size();
  s->accn = emit_at.empty() ? accn0 + (uint32_t)B : (uint32_t)(B - 1 - emit_at.back());
  s->spec_seq += ns;
  if (n_spec) *n_spec = ns;
  // fcfb.rs:66-100 / 154-188.  Work items of (channel, run of blocks), the
  // largest IFFT sizes first, so that threads finish together.
  constexpr long long BRUN = 8;
  std::vector<std::pair<int, long long>> items;
  for (size_t ci = 0; ci < s->ch.size(); ++ci)
    for (long long b0 = 0; b0 < B; b0 += BRUN) items.push_back({(int)ci, b0});
  std::stable_sort(items.begin(), items.end(), [&](const auto& x, const auto& y) {
    return s->ch[x.first].bins > s->ch[y.first].bins;
  });
  parallel_for((int)items.size(), nth, [&](int it) {
    const int ci = items[it].first;
    const Chan& c = s->ch[ci];
    const long long n = c.bins, shift = n / 2, keep = n / 8 * 6;
    thread_local std::vector<cf> buf, y;
    if ((long long)buf.size() < n) { buf.resize(n); y.resize(n); }
    const long long b1 = std::min(B, items[it].second + BRUN);
    for (long long b = items[it].second; b < b1; ++b) {
      const cf* Xb = s->X.data() + (size_t)b * K;
      for (long long i = 0; i < n; ++i) {
        const long long j = i + shift < n ? i + shift : i + shift - n;
        cf v = Xb[c.gi[i]];
        if (c.gc[i]) v.im = -v.im;
        cf wj = c.w[j];
        buf[i] = (wj.im == 0.0f) ? cf{wj.re * v.re, wj.re * v.im} : cmul(wj, v);
      }
      c.ifft.run(buf.data(), y.data());
      if (chan_out) std::memcpy(chan_out[ci] + 2 * b * keep, buf.data() + n / 8, sizeof(cf) * (size_t)keep);
    }
  });
  return 0;
}

// KAT hooks: multifft.rs:65-95 on one pair, and a bare FFT.
int32_t orc_two_real_ffts(int32_t n, const float* window, const float* in0, const float* in1, float* out0, float* out1) {
  FftPlan plan(n, -1);
  std::vector<cf> buf(n), y(n);
  for (int j = 0; j < n; ++j) buf[j] = {in0[j] * window[j], in1[j] * window[j]};
  plan.run(buf.data(), y.data());
  for (int i = 0; i < n / 2 + 1; ++i) {
    cf r = buf[i], m = buf[i == 0 ? 0 : n - i];
    out0[2 * i] = 0.5f * (r.re + m.re); out0[2 * i + 1] = 0.5f * (r.im - m.im);
    out1[2 * i] = 0.5f * (r.im + m.im); out1[2 * i + 1] = 0.5f * (-r.re + m.re);
  }
  return 0;
}
int32_t orc_fft(int32_t n, int32_t sign, float* data) {
  FftPlan plan(n, sign);
  std::vector<cf> y(n);
  plan.run((cf*)data, y.data());
  return 0;
}
int32_t orc_freq_to_bins(double fs, double fc, int64_t N, double fs_out, double fc_out, int32_t exact,
                         int64_t* bins, int64_t* first) {
  long long b = 0, f = 0;
  bool ok = exact ? freq_to_bins_exact(fs, fc, N, fs_out, fc_out, &b, &f) : freq_to_bins(fs, fc, N, fs_out, fc_out, &b, &f);
  *bins = b; *first = f;
  return ok ? 0 : -2;
}
void orc_bins_to_freq(double fs, double fc, int64_t N, int64_t bins, int64_t first, double* fs_out, double* fc_out) {
  bins_to_freq(fs, fc, N, bins, first, fs_out, fc_out);
}
void orc_tukey(int32_t n, int32_t tw, float* out) {
  auto w = tukey(n, tw);
  std::memcpy(out, w.data(), sizeof(cf) * n);
}
void orc_raised_cosine(int32_t n, float* out) {
  auto w = raised_cosine(n);
  std::memcpy(out, w.data(), sizeof(cf) * n);
}

}  // extern "C"

// ====================================================================== CLI
// Same command line as main.rs:15-91 (no ZeroMQ: this checker writes the
// per-filter file= outputs and the spectrum records to stdout only).
#ifdef ORACLE_MAIN
#include <unistd.h>

static int parse_format(const std::string& s) {
  static const struct { const char* n; int c; } t[] = {
    {"s8", 0x04}, {"s16le", 0x08}, {"s16be", 0x09}, {"f32le", 0x1C}, {"f32be", 0x1D}, {"u8", 0x24},
    {"cs8", 0x44}, {"cs16le", 0x48}, {"cs16be", 0x49}, {"cf32le", 0x5C}, {"cf32be", 0x5D}, {"cu8", 0x64}};
  for (auto& e : t) if (strcasecmp(s.c_str(), e.n) == 0) return e.c;
  return -1;
}

static bool read_exact(uint8_t* p, size_t n) {
  size_t got = 0;
  while (got < n) {
    ssize_t r = read(0, p + got, n - got);
    if (r <= 0) return false;
    got += (size_t)r;
  }
  return true;
}

static void write_all(FILE* f, const void* p, size_t n) { if (f) fwrite(p, 1, n, f); }

int main(int argc, char** argv) {
  orc_params p{};
  p.fc_in = 0; p.fft_size = 16384; p.ffts_per_buf = 8; p.averages = 2000; p.spectrum_format = 0;
  p.n_threads = (int)std::thread::hardware_concurrency();
  bool have_fs = false; int fmt = -1;
  std::vector<std::string> filters;
  uint64_t clk_secs = 0, clk_step = 0; bool fake = false;
  auto val = [&](int& i, const std::string& a, const char* lng, const char* sht, std::string& out) -> bool {
    std::string L = std::string("--") + lng;
    if (a == L || (sht && a == std::string("-") + sht)) { if (i + 1 >= argc) { fprintf(stderr, "missing value for %s\n", a.c_str()); exit(1); } out = argv[++i]; return true; }
    if (a.rfind(L + "=", 0) == 0) { out = a.substr(L.size() + 1); return true; }
    if (sht && a.rfind(std::string("-") + sht, 0) == 0 && a.size() > 2) { out = a.substr(2); if (!out.empty() && out[0] == '=') out = out.substr(1); return true; }
    return false;
  };
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i], v;
    if (val(i, a, "samplerate", "s", v)) { p.fs_in = atof(v.c_str()); have_fs = true; }
    else if (val(i, a, "centerfreq", "f", v)) p.fc_in = atof(v.c_str());
    else if (val(i, a, "fftsize", "n", v)) p.fft_size = atoi(v.c_str());
    else if (val(i, a, "fftbuf", nullptr, v)) p.ffts_per_buf = atoi(v.c_str());
    else if (val(i, a, "averages", "a", v)) p.averages = atoi(v.c_str());
    else if (val(i, a, "inputformat", "I", v)) fmt = parse_format(v);
    else if (val(i, a, "spectrumformat", nullptr, v)) p.spectrum_format = strcasecmp(v.c_str(), "u16") == 0 ? 1 : strcasecmp(v.c_str(), "f32") == 0 ? 2 : 0;
    else if (val(i, a, "threads", nullptr, v)) p.n_threads = atoi(v.c_str());
    else if (val(i, a, "fake-clock", nullptr, v)) { fake = true; sscanf(v.c_str(), "%lu,%lu", &clk_secs, &clk_step); }
    else if (val(i, a, "zmqbind", nullptr, v)) { while (i + 1 < argc && argv[i + 1][0] != '-') ++i; }
    else if (val(i, a, "filters", nullptr, v)) {
      filters.push_back(v);
      while (i + 1 < argc && argv[i + 1][0] != '-') filters.push_back(argv[++i]);
    } else { fprintf(stderr, "unknown argument %s\n", a.c_str()); return 1; }
  }
  if (!have_fs || fmt < 0) { fprintf(stderr, "--samplerate and --inputformat are required\n"); return 1; }
  p.input_format = fmt;
  std::vector<orc_filter> fl;
  std::vector<std::vector<float>> wstore;
  std::vector<std::string> files;
  for (auto& fs : filters) {
    orc_filter f{}; std::string file, wpath;
    size_t pos = 0;
    while (pos <= fs.size()) {
      size_t e = fs.find(':', pos); if (e == std::string::npos) e = fs.size();
      std::string kv = fs.substr(pos, e - pos);
      size_t eq = kv.find('=');
      if (eq == std::string::npos) { fprintf(stderr, "malformed filter parameter '%s'\n", kv.c_str()); return 101; }
      std::string k = kv.substr(0, eq), v = kv.substr(eq + 1);
      if (k == "fs") f.fs_out = atof(v.c_str());
      else if (k == "fc") f.fc_out = atof(v.c_str());
      else if (k == "file") file = v;
      else if (k == "tw") f.transition = atoi(v.c_str());
      else if (k == "w") wpath = v;
      pos = e + 1;
    }
    if (!wpath.empty()) {
      FILE* wf = fopen(wpath.c_str(), "rb");
      if (!wf) { fprintf(stderr, "cannot read weights %s\n", wpath.c_str()); return 101; }
      std::vector<float> w; float buf[1024]; size_t r;
      while ((r = fread(buf, 4, 1024, wf)) > 0) w.insert(w.end(), buf, buf + r);
      fclose(wf);
      wstore.push_back(std::move(w));
      f.weights = wstore.back().data();
    }
    fl.push_back(f); files.push_back(file);
  }
  std::vector<int32_t> st(fl.size());
  // Weight pointers must stay valid: wstore is not resized after this point.
  orc_state* s = orc_create(&p, fl.data(), (int32_t)fl.size(), st.data());
  if (!s) { fprintf(stderr, "invalid parameters\n"); return 1; }
  std::vector<FILE*> fouts;
  std::vector<uint8_t> ftopic;
  for (size_t i = 0; i < fl.size(); ++i) {
    if (st[i] != 0) { fprintf(stderr, "Invalid filter parameters\n"); continue; }
    FILE* fo = nullptr;
    if (!files[i].empty()) { fo = fopen(files[i].c_str(), "wb"); if (!fo) fprintf(stderr, "Could not create file: %s\n", files[i].c_str()); }
    fouts.push_back(fo);
  }
  int64_t nnew, ov; int32_t K, nch;
  orc_info(s, &nnew, &ov, &K, &nch);
  std::vector<uint8_t> raw((size_t)nnew * fmt_bytes(fmt));
  std::vector<std::vector<float>> co(nch);
  std::vector<float*> cptr(nch);
  std::vector<int64_t> nout(nch);
  for (int c = 0; c < nch; ++c) {
    int64_t b = 0, f0 = 0; orc_channel(s, c, &b, &f0);
    nout[c] = (int64_t)p.ffts_per_buf * (b / 8 * 6);
    co[c].resize(2 * nout[c]); cptr[c] = co[c].data();
  }
  const int sb = spec_bytes(p.spectrum_format);
  std::vector<uint8_t> spec((size_t)orc_max_spectra(s) * K * sb);
  std::vector<uint8_t> rec;
  uint64_t seq = 0;
  while (read_exact(raw.data(), raw.size())) {          // main.rs:176-178
    uint64_t secs = 0; uint32_t nanos = 0;
    if (fake) { uint64_t t = clk_secs * 1000000000ull + seq * clk_step; secs = t / 1000000000ull; nanos = (uint32_t)(t % 1000000000ull); }
    else { timespec ts; clock_gettime(CLOCK_REALTIME, &ts); secs = ts.tv_sec; nanos = (uint32_t)ts.tv_nsec; }
    int32_t ns; uint64_t sseq;
    orc_process(s, raw.data(), cptr.data(), spec.data(), &ns, &sseq);
    for (int r = 0; r < ns; ++r) {
      rec.assign(24 + (size_t)K * sb, 0);
      metadata24(rec.data(), sseq + r, secs, nanos);
      std::memcpy(rec.data() + 24, spec.data() + (size_t)r * K * sb, (size_t)K * sb);
      write_all(stdout, rec.data(), rec.size());
    }
    for (int c = 0; c < nch; ++c) {
      rec.assign(24 + (size_t)nout[c] * 8, 0);
      metadata24(rec.data(), seq, secs, nanos);
      std::memcpy(rec.data() + 24, co[c].data(), (size_t)nout[c] * 8);
      write_all(fouts[c], rec.data(), rec.size());
    }
    ++seq;
  }
  fflush(stdout);
  for (auto* f : fouts) if (f) fclose(f);
  orc_destroy(s);
  return 0;
}
#endif
