// Post-detection stages of the reference's demodulators on the GPU
// (tools/demodulator.py): the SSB automatic gain control SsbAgc (:16-65),
// the AM one AmAgc (:68-103) and the AM envelope |s| (:162).
//
// Both controls follow one scalar, the average amplitude pa, through the
// stream; every output sample depends on the pa after its own update:
//   SsbAgc: p = |s|, pd = p - pa, pa += pd * (pd >= 0 ? 0.002 : 0.0002),
//           s *= 0.25 / pa (0 when pa <= 0), and if |s|^2 > 0.9,
//           s *= sqrt(0.9 / |s|^2)
//   AmAgc : pd = s - pa, pa += pd * 0.0002,
//           s = s * (0.25 / pa) - 0.25 (0 when pa <= 0)
// all in float32 with separate products and sums.  The recurrence on pa is
// the only serial part, so a CTA takes the stream in segments of SEG
// samples: every thread forms the amplitudes p of its samples in shared
// memory, one thread runs the recurrence over the segment and leaves pa
// after each sample in place of p, and every thread then writes its
// outputs.  pa lives on the device between calls (0 at the start, as the
// reference's constructors set it).
#include <cmath>
#include <cstdint>

#include <cuda_runtime.h>

#include "spektri_b200.h"
#include "sk_internal.h"

using namespace sk;

namespace {

constexpr int AGC_T = 256;
constexpr int AGC_SEG = 4096;

struct AgcArgs {
  const void* x;              // float2 (SSB, envelopes) or float (AM) samples
  long long n;
  void* y;                    // float2 (SSB) or float outputs
  float* pa;                  // the carried average amplitude
};

// |s| of a complex64 sample, as numpy's absolute value of complex64 (hypot).
__device__ __forceinline__ float amplitude_of(float2 s) { return hypotf(s.x, s.y); }

template <int KIND>
__device__ __forceinline__ float detect(const AgcArgs& a, long long i) {
  if constexpr (KIND == SK_AGC_AM) return static_cast<const float*>(a.x)[i];
  else return amplitude_of(static_cast<const float2*>(a.x)[i]);
}

template <int KIND>
__device__ __forceinline__ float update(float pa, float p) {
  const float pd = __fsub_rn(p, pa);
  if constexpr (KIND == SK_AGC_SSB) {
    const float up = __fadd_rn(pa, __fmul_rn(pd, 0.002f));
    const float down = __fadd_rn(pa, __fmul_rn(pd, 0.0002f));
    return pd >= 0.f ? up : down;
  } else {
    return __fadd_rn(pa, __fmul_rn(pd, 0.0002f));
  }
}

template <int KIND>
__global__ void __launch_bounds__(AGC_T) agc_kernel(AgcArgs a) {
  __shared__ float seg[AGC_SEG];
  __shared__ float pa_carry;
  if (threadIdx.x == 0) pa_carry = *a.pa;
  for (long long base = 0; base < a.n; base += AGC_SEG) {
    const int len = (int)min((long long)AGC_SEG, a.n - base);
    for (int k = threadIdx.x; k < len; k += AGC_T) seg[k] = detect<KIND>(a, base + k);
    __syncthreads();
    if (KIND != SK_ENVELOPE && threadIdx.x == 0) {
      float pa = pa_carry;
      int k = 0;
      for (; k + 8 <= len; k += 8) {
        float p[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) p[u] = seg[k + u];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          pa = update<KIND>(pa, p[u]);
          seg[k + u] = pa;
        }
      }
      for (; k < len; ++k) {
        pa = update<KIND>(pa, seg[k]);
        seg[k] = pa;
      }
      pa_carry = pa;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < len; k += AGC_T) {
      const long long i = base + k;
      const float v = seg[k];
      if constexpr (KIND == SK_AGC_SSB) {
        float2 s = static_cast<const float2*>(a.x)[i];
        if (v > 0.f) {
          const float g = __fdiv_rn(0.25f, v);
          s = make_float2(__fmul_rn(s.x, g), __fmul_rn(s.y, g));
        } else {
          s = make_float2(0.f, 0.f);
        }
        const float p2 = __fadd_rn(__fmul_rn(s.x, s.x), __fmul_rn(s.y, s.y));
        if (p2 > 0.9f) {
          const float c = __fsqrt_rn(__fdiv_rn(0.9f, p2));
          s = make_float2(__fmul_rn(s.x, c), __fmul_rn(s.y, c));
        }
        static_cast<float2*>(a.y)[i] = s;
      } else if constexpr (KIND == SK_ENVELOPE) {
        static_cast<float*>(a.y)[i] = v;
      } else {
        const float s = detect<KIND>(a, i);
        static_cast<float*>(a.y)[i] = v > 0.f ? __fsub_rn(__fmul_rn(s, __fdiv_rn(0.25f, v)), 0.25f) : 0.f;
      }
    }
    __syncthreads();                                       // seg is rewritten by the next segment
  }
  if (threadIdx.x == 0 && KIND != SK_ENVELOPE) *a.pa = pa_carry;
}

}  // namespace

struct sk_agc {
  int device = 0;
  int kind = 0;
  float* d_pa = nullptr;
};

extern "C" {

int sk_agc_create(int32_t kind, int32_t device, sk_agc** out) {
  clear_error();
  if (!out) return fail(SK_ERR_ARG, "sk_agc_create: null argument");
  *out = nullptr;
  if (kind != SK_AGC_SSB && kind != SK_AGC_AM && kind != SK_AGC_AM_ENVELOPE && kind != SK_ENVELOPE)
    return fail(SK_ERR_ARG, "sk_agc_create: unknown kind %d", kind);
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return fail(SK_ERR_CUDA, "no CUDA device available");
  if (cudaSetDevice(device) != cudaSuccess) return fail(SK_ERR_ARG, "sk_agc_create: device %d unavailable", device);
  sk_agc* g = new sk_agc();
  g->device = device;
  g->kind = kind;
  cudaError_t e = cudaMalloc((void**)&g->d_pa, sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(g->d_pa, 0, sizeof(float));      // pa = 0 (demodulator.py:21, :73)
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess) {
    if (g->d_pa) cudaFree(g->d_pa);
    delete g;
    return fail(SK_ERR_NOMEM, "sk_agc_create: %s", cudaGetErrorString(e));
  }
  *out = g;
  return SK_OK;
}

int sk_agc_process_device(sk_agc* g, const float* in, uint64_t n, float* out, void* stream) {
  if (!g || (n && (!in || !out))) return fail(SK_ERR_ARG, "sk_agc_process_device: null argument");
  if (n == 0) return SK_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  if (cudaSetDevice(g->device) != cudaSuccess) return fail(SK_ERR_CUDA, "cudaSetDevice(%d) failed", g->device);
  const AgcArgs a{in, (long long)n, out, g->d_pa};
  cudaStream_t st = (cudaStream_t)stream;
  switch (g->kind) {
    case SK_AGC_SSB: agc_kernel<SK_AGC_SSB><<<1, AGC_T, 0, st>>>(a); break;
    case SK_AGC_AM: agc_kernel<SK_AGC_AM><<<1, AGC_T, 0, st>>>(a); break;
    case SK_AGC_AM_ENVELOPE: agc_kernel<SK_AGC_AM_ENVELOPE><<<1, AGC_T, 0, st>>>(a); break;
    default: agc_kernel<SK_ENVELOPE><<<1, AGC_T, 0, st>>>(a); break;
  }
  const cudaError_t e = cudaGetLastError();
  if (prev >= 0) cudaSetDevice(prev);
  if (e != cudaSuccess) return fail(SK_ERR_CUDA, "AGC kernel: %s", cudaGetErrorString(e));
  return SK_OK;
}

void sk_agc_destroy(sk_agc* g) {
  if (!g) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(g->device);
  if (g->d_pa) cudaFree(g->d_pa);
  if (prev >= 0) cudaSetDevice(prev);
  delete g;
}

}  // extern "C"
