// Rational downconverter on the GPU: the reference's RationalDdc
// (tools/ddc.py:51-145), the stage that runs after the filter bank on one
// channel's complex output stream (mixing, polyphase resampling).
//
// Per input sample s the reference mixes x[s] with a repeating oscillator
// table lo[s mod L] (ddc.py:20-34, L = den), pushes it into its FIR history
// and advances the polyphase phase by `interpolation`; each time the phase
// reaches `decimation` it drops by `decimation` and one output is formed
// from the firlen newest mixed samples with that phase's taps
// (ddc.py:113-141).  The same outputs in closed form, one thread each: with
// the phase starting at 0, T(S) = floor(S * interpolation / decimation)
// outputs exist after S samples; output o comes from sample
// s_o = ceil((o + 1) * decimation / interpolation) - 1 with phase
// p_o = (s_o + 1) * interpolation - (o + 1) * decimation, and
//   y[o] = sum_j taps[p_o + j * interpolation] * mixed[s_o - firlen + 1 + j]
// summed in j order in float32 as the reference does.  The last firlen - 1
// mixed samples of a call are kept on the device for the next one (zeros
// before the stream starts, as the reference's buffer, ddc.py:84).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "spektri_b200.h"
#include "sk_internal.h"

using namespace sk;

namespace {

struct DdcArgs {
  const float2* x;            // this call's input, n_in samples
  long long s0, n_in;         // global index of x[0]; samples in this call
  long long o0, n_out;        // global index of the first output; outputs in this call
  const float* taps;          // firlen * interp
  int firlen, interp, decim;
  const float2* lo;           // L oscillator values
  int L;
  const float2* hist;         // mixed samples [s0 - firlen + 1, s0)
  float2* hist_next;          // receives the mixed samples [s0 + n_in - firlen + 1, s0 + n_in)
  float2* y;                  // n_out outputs
};

// x times the oscillator, in float32 with separate products and sums like the
// reference's complex64 arithmetic.
__device__ __forceinline__ float2 mix(const DdcArgs& a, long long s) {
  const float2 v = __ldg(&a.x[s - a.s0]);
  const float2 l = __ldg(&a.lo[s % a.L]);
  return make_float2(__fsub_rn(__fmul_rn(v.x, l.x), __fmul_rn(v.y, l.y)),
                     __fadd_rn(__fmul_rn(v.x, l.y), __fmul_rn(v.y, l.x)));
}

__device__ __forceinline__ float2 mixed_at(const DdcArgs& a, long long s) {
  return s >= a.s0 ? mix(a, s) : __ldg(&a.hist[s - (a.s0 - (a.firlen - 1))]);
}

__global__ void __launch_bounds__(256) ddc_kernel(DdcArgs a) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.n_out) {
    const long long o = a.o0 + i;
    const long long so = ((o + 1) * a.decim + a.interp - 1) / a.interp - 1;
    const int p = (int)((so + 1) * a.interp - (o + 1) * a.decim);
    float2 acc = make_float2(0.f, 0.f);
    const long long s_first = so - a.firlen + 1;
    for (int j = 0; j < a.firlen; ++j) {
      const float t = __ldg(&a.taps[p + j * a.interp]);
      const float2 m = mixed_at(a, s_first + j);
      acc = make_float2(__fadd_rn(acc.x, __fmul_rn(t, m.x)), __fadd_rn(acc.y, __fmul_rn(t, m.y)));
    }
    a.y[i] = acc;
  }
}

// The history for the next call: the last firlen - 1 mixed samples.
__global__ void __launch_bounds__(256) ddc_history_kernel(DdcArgs a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < a.firlen - 1) a.hist_next[k] = mixed_at(a, a.s0 + a.n_in - (a.firlen - 1) + k);
}

}  // namespace

struct sk_ddc {
  int device = 0;
  int firlen = 1, interp = 1, decim = 1, L = 1;
  float* d_taps = nullptr;
  float2* d_lo = nullptr;
  float2* d_hist[2] = {nullptr, nullptr};
  int cur = 0;
  long long n_in = 0;         // samples consumed so far
};

namespace {

long long outputs_after(const sk_ddc* d, long long samples) {
  return samples * d->interp / d->decim;
}

void ddc_free(sk_ddc* d) {
  if (!d) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(d->device);
  for (void* p : {(void*)d->d_taps, (void*)d->d_lo, (void*)d->d_hist[0], (void*)d->d_hist[1]})
    if (p) cudaFree(p);
  if (prev >= 0) cudaSetDevice(prev);
  delete d;
}

}  // namespace

extern "C" {

int sk_ddc_create(const float* taps, uint32_t n_taps, uint32_t interpolation, uint32_t decimation, int64_t freq_num,
                  int64_t freq_den, int32_t device, sk_ddc** out) {
  clear_error();
  if (!taps || !out) return fail(SK_ERR_ARG, "sk_ddc_create: null argument");
  *out = nullptr;
  if (interpolation == 0 || decimation == 0 || n_taps == 0 || n_taps % interpolation)
    return fail(SK_ERR_ARG, "sk_ddc_create: the tap count must be a positive multiple of the interpolation (ddc.py:65)");
  if (freq_den <= 0 || freq_den > (1 << 24))
    return fail(SK_ERR_ARG, "sk_ddc_create: oscillator denominator must be 1 .. 2^24");
  if (interpolation > (1u << 20) || decimation > (1u << 20))
    return fail(SK_ERR_ARG, "sk_ddc_create: interpolation and decimation must be at most 2^20");
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return fail(SK_ERR_CUDA, "no CUDA device available");
  if (cudaSetDevice(device) != cudaSuccess) return fail(SK_ERR_ARG, "sk_ddc_create: device %d unavailable", device);
  sk_ddc* d = new sk_ddc();
  d->device = device;
  d->interp = (int)interpolation;
  d->decim = (int)decimation;
  d->firlen = (int)(n_taps / interpolation);
  // ddc.py:20-34: phases (k num mod den) * float32(2 pi / den) in float32, then cos + i sin
  std::vector<float2> lo;
  if (freq_num == 0) {
    lo.push_back(make_float2(1.f, 0.f));
  } else {
    const float step = (float)(2.0 * M_PI / (double)freq_den);
    lo.resize((size_t)freq_den);
    for (int64_t k = 0; k < freq_den; ++k) {
      const int64_t r = ((k * (freq_num % freq_den)) % freq_den + freq_den) % freq_den;
      const float ph = (float)r * step;
      lo[(size_t)k] = make_float2((float)std::cos((double)ph), (float)std::sin((double)ph));
    }
  }
  d->L = (int)lo.size();
  const size_t hist_n = (size_t)std::max(1, d->firlen - 1);
  cudaError_t e = cudaMalloc((void**)&d->d_taps, sizeof(float) * n_taps);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d->d_lo, sizeof(float2) * lo.size());
  if (e == cudaSuccess) e = cudaMalloc((void**)&d->d_hist[0], sizeof(float2) * hist_n);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d->d_hist[1], sizeof(float2) * hist_n);
  if (e == cudaSuccess) e = cudaMemcpy(d->d_taps, taps, sizeof(float) * n_taps, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d->d_lo, lo.data(), sizeof(float2) * lo.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(d->d_hist[0], 0, sizeof(float2) * hist_n);   // ddc.py:84: zeros
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess) {
    ddc_free(d);
    return fail(SK_ERR_NOMEM, "sk_ddc_create: %s", cudaGetErrorString(e));
  }
  *out = d;
  return SK_OK;
}

int sk_ddc_outputs(const sk_ddc* d, uint64_t n_in, uint64_t* n_out) {
  if (!d || !n_out) return fail(SK_ERR_ARG, "sk_ddc_outputs: null argument");
  *n_out = (uint64_t)(outputs_after(d, d->n_in + (long long)n_in) - outputs_after(d, d->n_in));
  return SK_OK;
}

int sk_ddc_process_device(sk_ddc* d, const float* in_c64, uint64_t n_in, float* out_c64, uint64_t* n_out,
                          void* stream) {
  if (!d || (n_in && !in_c64) || !n_out) return fail(SK_ERR_ARG, "sk_ddc_process_device: null argument");
  const long long o0 = outputs_after(d, d->n_in), o1 = outputs_after(d, d->n_in + (long long)n_in);
  *n_out = (uint64_t)(o1 - o0);
  if (o1 > o0 && !out_c64) return fail(SK_ERR_ARG, "sk_ddc_process_device: null output");
  if (n_in == 0) return SK_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  if (cudaSetDevice(d->device) != cudaSuccess) return fail(SK_ERR_CUDA, "cudaSetDevice(%d) failed", d->device);
  DdcArgs a{};
  a.x = (const float2*)in_c64;
  a.s0 = d->n_in;
  a.n_in = (long long)n_in;
  a.o0 = o0;
  a.n_out = o1 - o0;
  a.taps = d->d_taps;
  a.firlen = d->firlen;
  a.interp = d->interp;
  a.decim = d->decim;
  a.lo = d->d_lo;
  a.L = d->L;
  a.hist = d->d_hist[d->cur];
  a.hist_next = d->d_hist[d->cur ^ 1];
  a.y = (float2*)out_c64;
  cudaStream_t st = (cudaStream_t)stream;
  if (a.n_out > 0) ddc_kernel<<<(unsigned)((a.n_out + 255) / 256), 256, 0, st>>>(a);
  if (d->firlen > 1) ddc_history_kernel<<<(d->firlen - 1 + 255) / 256, 256, 0, st>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess) return fail(SK_ERR_CUDA, "DDC kernels: %s", cudaGetErrorString(e));
  if (d->firlen > 1) d->cur ^= 1;
  d->n_in += (long long)n_in;
  return SK_OK;
}

void sk_ddc_destroy(sk_ddc* d) { ddc_free(d); }

}  // extern "C"
