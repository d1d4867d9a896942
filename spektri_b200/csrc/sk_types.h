// Kernel argument structures, tile constants and the launchers that the host
// code calls.  Host-compilable: the kernels themselves live in the .cu files
// that include sk_kernels.cuh (one instantiation each).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace sk {

constexpr int TILE_S = 8192;              // complex elements per FFT tile
constexpr int TILE_T = 256;               // threads per tile CTA (32 elements each)
constexpr int TILE_T16 = 512;             // threads of the 16-element kernels (two-pass column and row passes)
constexpr int TILE_LOGS = 13;
constexpr int MAX_TILE_TRANSFORMS = 128;  // transforms per filter-bank tile
constexpr int MAX_SPLIT_LOG = 3;          // an IFFT of up to 2^3 tiles runs as independent parts (n = P S, P <= 8)
constexpr int MAX_IFFT_LOG = 16;          // power-of-two IFFT sizes up to 2^16
// The tile twiddle array: W_S^k for k < S, then per-stage tables.  A tile FFT
// stage of span L and radix R (P = L R = 2^p) multiplies by w^s, w = W_P^j,
// j < L <= P/2; its table holds W_P^(j s) for s = 1, 4, 16 (si = 0, 1, 2) at
// stage_tw_offset(p, si) + j, so lane-consecutive j read consecutive entries.
__host__ __device__ constexpr int stage_tw_offset(int p, int si) {
  return TILE_S + 3 * ((1 << (p - 1)) - 1) + si * (1 << (p - 1));
}
constexpr int TILE_TW_ELEMS = TILE_S + 3 * ((1 << TILE_LOGS) - 1);   // p = 1 .. 13
// The filter bank's array appends the p = 14 table for si = 0 (W_16384^j,
// j < 8192, at stage_tw_offset(14, 0) = TILE_TW_ELEMS): the last radix-4
// stage of the 16384-point chirp-z tiles reads only it.
constexpr int TILE_TW_ELEMS_X = TILE_TW_ELEMS + (1 << TILE_LOGS);
constexpr int CHIRP_LOGM_MAX = TILE_LOGS + 1;   // chirp-z transforms up to M = 16384 (IFFT sizes up to 9364)
// Tile in shared memory: S complex values with one pad slot per 16.
constexpr size_t TILE_SMEM = sizeof(float2) * (size_t)(TILE_S + TILE_S / 16);
// The column pass's tile adds one slot per transform (at most S/16 of them).
constexpr size_t TILE_SMEM_COL = sizeof(float2) * (size_t)(TILE_S + TILE_S / 8);
constexpr int WELCH_WARP_BINS = 30;       // bins per Welch CTA (a warp plus a 1-bin halo each side)
constexpr int WELCH_WARPS = 4;            // warps per Welch CTA (they split the blocks; 4 measured best of 1..32)
constexpr int WELCH_BINS_MAX_B = 16;      // blocks per buffer up to which a warp walks its own bins
constexpr int WELCH_CHUNK = 64;           // blocks whose Welch terms a CTA stages at once

struct ChanDev {               // one filter-bank channel, as the kernels see it
  const float2* w;             // weights, natural order: w[j] scales bin first+j
  float2* out;                 // B * 6(n/8) outputs
  long long first;             // first bin modulo N (in [0, N))
  int log2n;
  int pad;
};
struct BwdChan {
  const float2* w;
  const float2* dy;            // B * 6(n/8) output gradients
  float2* dw;                  // n weight gradients (written)
  float2* g;                   // scratch, B * n: per block the forward FFT of dy zero-padded to [n/8, 7n/8)
  long long first;             // first bin modulo N
  int log2n;
  int pad;
};
struct TileDesc {              // transforms of one size
  int log2n;                   // log2 n, or BLU_TAG + log2 M for a chirp-z tile
  int list_off;                // first entry in the (channel, block) list
  int count;                   // transforms in this tile
  int pad;                     // chirp-z tiles: index of their BluDesc
};

// Chirp-z (Bluestein) channels: an IFFT size n that is a multiple of 4 but
// not a power of two runs as a forward and an inverse M-point FFT, M = 2^logm
// the smallest power of two >= n + 6(n/8) - 1 (what the kept outputs
// [n/8, 7(n/8)) need of the circular convolution).
struct BluDesc {
  const float2* chirp;         // c[i] = exp(+i pi i^2 / n), i < n
  const float2* H;             // forward M-point FFT of the kernel conj(c[d]) (d wrapped mod M), times 1/M
  int n, logm;
};
constexpr int BLU_TAG = 16;

// Stage trace: global-timer nanoseconds, per call, of [0] the first forward
// CTA's start (minimum), [1] the last forward CTA's end, [2] the last Welch
// CTA's end, [3] the last filter-bank CTA's end (maxima).  Recorded by one
// thread per CTA inside the kernels (also inside the captured graph); the
// host resets the slots between traced calls.
constexpr int TRACE_SLOTS = 4;

struct FwdArgs {
  const uint8_t* raw;          // new samples of this buffer
  const float* halo;           // converted last N/4 samples of the previous buffer
  float* halo_next;            // receives the converted last N/4 samples of this one
  long long overlap, nnew;
  int hop, B;
  int log2N, log2Nc;           // N (window length) and Nc (complex FFT length), powers of two (else -1)
  int N, Nc;                   // the same lengths (any supported size)
  int R1, log2R1;              // two-pass FFTs: Nc = R1 * M (R1 = 1: single pass); log2R1 = -1 when R1
                               // is not a power of two (R1 = 3, 5, 6, 10, 12: the mixed-radix column pass)
  int logM;                    // two-pass FFTs: log2 of the row length M (8192 when R1 is a power of two)
  float wscale;                // rectangular window value scaling/N (dsp.rs:70-73)
  const float2* tw_tile;       // W_S^k
  const float2* tw_big;        // W_N^k, k < N
  float2* Z;                   // [B][Nc]; for R1 > 1 element k1 + R1*k2 sits at k1*S + k2
  int per;                     // Nc <= S: blocks per tile (0: S / Nc, a full tile)
  int* cursor;                 // non-null: the filter bank's two tile cursors, zeroed by the
                               // first forward kernel (the batched graph, in place of a memset)
  unsigned long long* trace;   // stage trace slots (may be null)
};

struct SplitArgs {
  const float2* Z;             // [B][Nc] packed spectra; residue layout for R1 > 1 (k1 + R1 k2 at k1 M + k2)
  float2* X;                   // [B][K]
  float* P;                    // [B][K] Welch terms (may be null)
  int N, Nc, K, R1, log2R1, logM;   // log2R1 = -1: R1 not a power of two
  const float2* tw_big;        // W_N^k
};

struct WelchArgs {
  SplitArgs s;                 // Z -> s.X in the filter bank's extended layout (s.P unused)
  long long xs;                // extended row stride: >= N + maxn bins per block
  int maxn;                    // largest IFFT size of the plan (the wrap margin past bin N - 1)
  float* acc;                  // [K] running accumulator (carried across buffers)
  int B, accn0, averages, fmt;
  float db_plus;               // -10 log10(averages), computed on the host in f32
  uint8_t* out;                // records, K bins each
  unsigned long long* trace;   // stage trace slots (may be null)
};

struct FcfbArgs {
  const TileDesc* tiles;
  int ntiles;
  int* cursor;                 // persistent mode: next tile to claim
  const int2* list;            // (channel, block) per transform
  const ChanDev* chans;
  const float2* X;             // [B][xs] extended spectra: bin m mod N (mirrored for real input) at every m < xs
  long long xs;
  int log2N;
  const float2* tw;            // W_8192^k, k < 8192
  const float2* tw_split;      // W_Ns^k, k < Ns = 2^log_split (IFFTs larger than a tile)
  int log_split;
  const BluDesc* blu;          // chirp-z sizes (may be null)
  unsigned long long* trace;   // stage trace slots (may be null)
};

struct BwdArgs {
  const TileDesc* tiles;       // the 8192-point tiles of the plan (power-of-two sizes <= 8192)
  const int2* list;            // (channel, block) per transform
  const BwdChan* chans;
  int nchan;
  const float2* X;             // [B][K] spectra of the forward pass
  float2* dX;                  // [B][K], accumulated into (may be null)
  const int* bin_off;          // dX gather lists: bin k's entries are bin_ent[bin_off[k] .. bin_off[k+1])
  const int2* bin_ent;         // (channel, 2 j + mirror): get_bin(first + j) is bin k (conjugated if mirror)
  int K, N, B;
  const float2* tw;
};

// Launchers (sk_fwd_*.cu, sk_kern.cu).  Each returns the launch status.
cudaError_t fwd_prepare(int fmt);                         // shared-memory limit of the format's kernel
cudaError_t launch_fwd(int fmt, int grid, const FwdArgs& a, cudaStream_t st);
cudaError_t fwd_prepare_8(int fmt);
cudaError_t fwd_prepare_16(int fmt);
cudaError_t fwd_prepare_32(int fmt);
cudaError_t launch_fwd_8(int fmt, int grid, const FwdArgs& a, cudaStream_t st);
cudaError_t launch_fwd_16(int fmt, int grid, const FwdArgs& a, cudaStream_t st);
cudaError_t launch_fwd_32(int fmt, int grid, const FwdArgs& a, cudaStream_t st);
// Two-pass forward FFT (R1 >= 2): column pass from the raw samples into Y,
// then the row pass from Y into Z.
cudaError_t launch_fwd_col(int fmt, int grid, const FwdArgs& a, float2* Y, cudaStream_t st);
cudaError_t launch_fwd_col_8(int fmt, int grid, const FwdArgs& a, float2* Y, cudaStream_t st);
cudaError_t launch_fwd_col_16(int fmt, int grid, const FwdArgs& a, float2* Y, cudaStream_t st);
cudaError_t launch_fwd_col_32(int fmt, int grid, const FwdArgs& a, float2* Y, cudaStream_t st);
// pdl: launched with programmatic stream serialization (the kernel's CTAs may
// start as those of the kernel ahead of it in the stream exit, before that
// grid has completed; it waits for that grid in pdl_wait()).
cudaError_t launch_kernel(const void* fn, dim3 grid, dim3 block, void** params, size_t smem, cudaStream_t st,
                          bool pdl);
cudaError_t launch_fwd_rows(int grid, const FwdArgs& a, const float2* Y, cudaStream_t st, bool pdl = false);
cudaError_t launch_split(bool cplx, int B, const SplitArgs& s, cudaStream_t st);
cudaError_t launch_welch(bool cplx, const WelchArgs& w, cudaStream_t st, bool pdl = false);
// [B][K] spectra (the differentiable stage's layout) -> [B][xs] extended rows.
cudaError_t launch_extend(bool cplx, int B, const float2* X, int K, int N, float2* Xe, long long xs, int maxn,
                          cudaStream_t st);
cudaError_t fcfb_prepare();
// Filter-bank tile shapes (tile_size, tile_threads): (8192, 256), (8192, 512)
// and (4096, 256); a 4096-point tile runs an 8192-point transform as two halves.
bool fcfb_shape_ok(int tile_size, int tile_threads);
constexpr size_t fcfb_smem(int tile_size) { return sizeof(float2) * (size_t)(tile_size + tile_size / 16); }
cudaError_t fcfb_occupancy(int tile_size, int tile_threads, int* ctas_per_sm);
// chirp: the kernel for chirp-z tiles (else power-of-two tiles).
cudaError_t launch_fcfb(bool persistent, bool chirp, int tile_size, int tile_threads, int grid, const FcfbArgs& a,
                        int tile_base, cudaStream_t st, bool pdl = false);
const void* fcfb_kernel_ptr(int tile_size, int tile_threads, bool persistent, bool chirp);
// Per-shape instance tables (sk_fcfb_*.cu).
const void* fcfb_ptr_8192(bool persistent);
const void* fcfb_ptr_8192_chirp(bool persistent);
const void* fcfb_ptr_8192x512(bool persistent);
const void* fcfb_ptr_8192x512_chirp(bool persistent);
const void* fcfb_ptr_4096(bool persistent);
const void* fcfb_ptr_4096_chirp(bool persistent);
const void* fcfb_ptr_16384_chirp();                       // non-persistent, M = 16384 chirp-z tiles only
// One launch of that kernel: grid = tiles (one transform each) from tile_base.
cudaError_t launch_fcfb_chirp16k(int grid, const FcfbArgs& a, int tile_base, cudaStream_t st);
// Adjoint in three deterministic launches: the per-transform forward FFTs of
// the padded output gradients (grid = tiles), dW summed over blocks in block
// order (grid = channels x n_max/256), dX gathered per bin in channel order.
cudaError_t launch_fcfb_backward(bool cplx, int grid, int max_n, const BwdArgs& a, cudaStream_t st);
// Kernel entry addresses (to recognise the nodes of a captured graph).
// kind 0: single-pass forward kernel; 1: shared-memory column pass (R1 >= 16);
// 2: register column pass (R1 = 2..8); 3: mixed-radix column pass (R1 = 3, 5, 6, 10, 12).
const void* fwd_kernel_ptr(int fmt, int kind, int R1);
const void* fwd_kernel_ptr_8(int fmt, int kind, int R1);
const void* fwd_kernel_ptr_16(int fmt, int kind, int R1);
const void* fwd_kernel_ptr_32(int fmt, int kind, int R1);
// Mixed-radix column factors: R1 = R0 * P with R0 = 3 or 5 and P a power of two.
constexpr bool mixed_r1_ok(int r1) { return r1 == 3 || r1 == 5 || r1 == 6 || r1 == 10 || r1 == 12; }
const void* welch_kernel_ptr(bool cplx, int B, bool pow2, int R1);   // pow2: the FFT size is a power of two

}  // namespace sk
