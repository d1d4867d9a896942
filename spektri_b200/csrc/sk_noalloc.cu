// Allocation-free forward spectra: sk_spectra_noalloc.
//
// Who needs this.  Some programs that embed the filter bank may not call
// cudaMalloc at all: an SDR receive callback that must never stall (a device
// allocation can synchronise the whole GPU and take milliseconds, long enough
// to drop samples), or a host application that hands its entire device
// memory budget to its own pool at start-up and forbids libraries from
// allocating behind its back.  The plan-based API allocates its scratch when
// a plan is created, so those callers cannot use it.  This entry point gives
// them the forward FFT stage with no allocation: the caller passes the raw
// input and the output spectra, and the intermediate FFT results and twiddle
// tables live in one fixed array compiled into the library.
//
// The array is g_noalloc_scratch below: SK_NOALLOC_SCRATCH_ELEMS complex
// floats (8 MiB), reserved on every GPU that loads the library until the
// process exits.  All calls on a device share it and it keeps whatever the
// last call left there.  Its head holds the twiddle tables: the tile tables
// (the same for every call) are written by the first call on a device, the
// window table W_N^k again whenever N differs from the previous call's; the
// FFT results after them are rewritten by every call, so nothing has to
// start at zero.  Two calls whose work overlaps on the GPU (different
// streams, or different host threads on the same device) race on the array
// and corrupt each other.
//
// Host code cannot use the array's name as a device address (in host code it
// names a host-side shadow), so the first call on each device looks up the
// real address with cudaGetSymbolAddress, with that device current, and sets
// the kernels' shared-memory limits.  That first call therefore makes
// synchronous runtime calls; make it before any stream capture begins.  The
// looked-up address and the table flags are kept per device for the life of
// the process: do not use this entry point on a device after cudaDeviceReset
// (the module may load again at another address, and the kernel attributes
// set here are gone).
#include <algorithm>
#include <cmath>
#include <deque>
#include <mutex>

#include <cuda_runtime.h>

#include "spektri_b200.h"
#include "sk_internal.h"
#include "sk_types.h"

using namespace sk;

namespace {

constexpr int S = TILE_S;
constexpr size_t kScratchElems = SK_NOALLOC_SCRATCH_ELEMS;

static __device__ __align__(256) float2 g_noalloc_scratch[kScratchElems];

struct DeviceSetup {
  bool ready = false;
  float2* base = nullptr;     // device address of g_noalloc_scratch on this device
  bool tile_tables = false;   // the tile twiddle tables have been written
  long long window_n = 0;     // N of the window table W_N^k written last (0: none)
};
std::mutex g_mu;
std::deque<DeviceSetup> g_setup;      // one per device ordinal; growing it keeps earlier elements in place

// W_n^k = exp(-2 pi i k / n) for the tile table (n = S, then the per-stage
// tables W_P^(j s), layout stage_tw_offset; skipped when tile == false) and
// the window table (skipped when n_big == 0).
__global__ void noalloc_twiddles(float2* tw_tile, float2* tw_big, int n_big, bool tile) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double s, c;
  if (!tile) {
  } else if (i < S) {
    sincospi(-2.0 * (double)i / (double)S, &s, &c);
    tw_tile[i] = make_float2((float)c, (float)s);
  } else if (i < TILE_TW_ELEMS) {
    int p = 1;
    while (p < TILE_LOGS && i >= stage_tw_offset(p + 1, 0)) ++p;
    const int h = 1 << (p - 1), r = i - stage_tw_offset(p, 0), si = r / h, j = r - si * h;
    const long long P = 2ll * h, e = ((long long)j * (si == 0 ? 1 : si == 1 ? 4 : 16)) % P;
    sincospi(-2.0 * (double)e / (double)P, &s, &c);
    tw_tile[i] = make_float2((float)c, (float)s);
  }
  if (i < n_big) {
    sincospi(-2.0 * (double)i / (double)n_big, &s, &c);
    tw_big[i] = make_float2((float)c, (float)s);
  }
}

int log2_exact(long long v) {
  if (v <= 0 || (v & (v - 1))) return -1;
  int r = 0;
  while ((1ll << r) < v) ++r;
  return r;
}

// Once per device, with that device current: the array's device address and
// the kernels' dynamic shared-memory limit.
DeviceSetup* setup_device(int dev) {
  std::lock_guard<std::mutex> lk(g_mu);
  if ((int)g_setup.size() <= dev) g_setup.resize(dev + 1);
  DeviceSetup& d = g_setup[dev];
  if (!d.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      fail(SK_ERR_CUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(e));
      return nullptr;
    }
    static const int fmts[] = {SK_FMT_S8, SK_FMT_S16LE, SK_FMT_S16BE, SK_FMT_F32LE, SK_FMT_F32BE, SK_FMT_U8,
                               SK_FMT_CS8, SK_FMT_CS16LE, SK_FMT_CS16BE, SK_FMT_CF32LE, SK_FMT_CF32BE, SK_FMT_CU8};
    for (int f : fmts) {
      e = fwd_prepare(f);
      if (e != cudaSuccess) {
        fail(SK_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
        return nullptr;
      }
    }
    d.base = (float2*)p;
    d.ready = true;
  }
  return &d;
}

}  // namespace

extern "C" int sk_spectra_noalloc(const void* raw, int32_t input_format, uint32_t fft_size, uint32_t n_blocks,
                                  float* X, void* stream) {
  if (!raw || !X) return fail(SK_ERR_ARG, "sk_spectra_noalloc: null raw input or output");
  if (!format_valid(input_format)) return fail(SK_ERR_ARG, "sk_spectra_noalloc: unknown input format 0x%02x", input_format);
  if (n_blocks == 0) return fail(SK_ERR_ARG, "sk_spectra_noalloc: n_blocks must be positive");
  const bool cplx = format_complex(input_format);
  const int log2N = log2_exact(fft_size);
  const int log2Nc = log2N - (cplx ? 0 : 1);
  if (log2N < 3 || log2Nc < 2 || log2Nc > TILE_LOGS + 3)
    return fail(SK_ERR_UNSUPPORTED, "sk_spectra_noalloc: FFT size %u not supported (power of two, 8 .. %d complex points)",
                fft_size, 1 << (TILE_LOGS + 3));
  if ((uintptr_t)raw % (format_bits(input_format) / 8))
    return fail(SK_ERR_ARG, "sk_spectra_noalloc: raw input misaligned for its sample format");
  const long long N = fft_size, Nc = 1ll << log2Nc;
  const unsigned long long need = (unsigned long long)TILE_TW_ELEMS + (unsigned long long)N + (unsigned long long)n_blocks * Nc;
  if (need > kScratchElems)
    return fail(SK_ERR_ARG,
                "sk_spectra_noalloc: %u blocks of FFT size %u need %llu complex scratch elements; the static "
                "scratch holds %zu (%zu MiB): at most %lld blocks at this size",
                n_blocks, fft_size, need, kScratchElems, kScratchElems * sizeof(float2) >> 20,
                (long long)((kScratchElems - TILE_TW_ELEMS - N) / Nc));
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(SK_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  DeviceSetup* d = setup_device(dev);
  if (!d) return SK_ERR_CUDA;
  float2* base = d->base;
  cudaStream_t st = (cudaStream_t)stream;
  float2* tw_tile = base;
  float2* tw_big = base + TILE_TW_ELEMS;
  float2* Z = base + TILE_TW_ELEMS + N;

  {
    std::lock_guard<std::mutex> lk(g_mu);
    const bool tile = !d->tile_tables, window = d->window_n != N;
    if (tile || window) {               // tables this call reads that the array does not hold yet
      const int nt = (int)std::max<long long>(tile ? TILE_TW_ELEMS : 0, window ? N : 0);
      noalloc_twiddles<<<(nt + 255) / 256, 256, 0, st>>>(tw_tile, tw_big, window ? (int)N : 0, tile);
      e = cudaGetLastError();
      if (e != cudaSuccess) return fail(SK_ERR_CUDA, "twiddle kernel: %s", cudaGetErrorString(e));
      d->tile_tables = true;
      d->window_n = N;
    }
  }

  // The caller's window holds every sample: [N/4 carried | 3N/4 * n_blocks new].
  const long long hop = N - N / 4;
  FwdArgs a{};
  a.raw = (const uint8_t*)raw;
  a.halo = nullptr;
  a.halo_next = nullptr;
  a.overlap = 0;                       // no carry: the window starts at sample 0 of block 0
  a.nnew = hop * n_blocks + N / 4;
  a.hop = (int)hop;
  a.B = (int)n_blocks;
  a.log2N = log2N;
  a.log2Nc = log2Nc;
  a.N = (int)N;
  a.Nc = (int)Nc;
  a.logM = TILE_LOGS;
  a.R1 = 1;
  a.log2R1 = 0;
  if (log2Nc > TILE_LOGS) {
    a.log2R1 = log2Nc - TILE_LOGS;
    a.R1 = 1 << a.log2R1;
  }
  a.wscale = format_scaling(input_format) / (float)N;
  a.tw_tile = tw_tile;
  a.tw_big = tw_big;
  a.Z = Z;
  int grid;
  if (a.R1 == 1) {
    const int per = S >> log2Nc;
    grid = (int)((n_blocks + per - 1) / per);
  } else {
    grid = (int)n_blocks * a.R1;
  }
  e = launch_fwd(input_format, grid, a, st);
  if (e != cudaSuccess) return fail(SK_ERR_CUDA, "forward FFT kernel: %s", cudaGetErrorString(e));

  SplitArgs s{};
  s.Z = Z;
  s.X = (float2*)X;
  s.P = nullptr;
  s.N = (int)N;
  s.Nc = (int)Nc;
  s.K = cplx ? (int)N : (int)(N / 2 + 1);
  s.R1 = a.R1;
  s.log2R1 = a.log2R1;
  s.logM = TILE_LOGS;
  s.tw_big = tw_big;
  e = launch_split(cplx, (int)n_blocks, s, st);
  if (e != cudaSuccess) return fail(SK_ERR_CUDA, "spectrum split kernel: %s", cudaGetErrorString(e));
  return SK_OK;
}
