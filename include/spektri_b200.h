/*
 * spektri_b200 — C ABI of the B200 (sm_100a) fast-convolution filter bank and
 * Welch spectrum.
 *
 * The reference (tejeez/spektri) is a single Rust binary; the seam this ABI
 * replaces is its DSP state machine:
 *
 *   DspState::init(DspParams) -> (DspState, InputBufferSize)   spektri/src/dsp.rs:76-111
 *   DspState::process_real / process_complex                   spektri/src/dsp.rs:114-160
 *   MultiFft::process_real / process_complex                   spektri/src/dsp/multifft.rs:34-95
 *   SpectrumAccumulator::accumulate                            spektri/src/dsp/spectrum.rs:82-163
 *   Fcfb::add_filter / Fcfb::process / FilterDsp::process      spektri/src/dsp/fcfb.rs:41-188
 *   freq_to_bins / bins_to_freq / freq_to_bins_exact           spektri/src/dsp/fcfb.rs:225-285
 *   serialize_metadata / serialize_*_topic                     spektri/src/dsp/data.rs:110-171
 *   convert_to_f32 / convert_to_cf32 (fused into the FFT load)  spektri/src/inputformats.rs:65-155
 *
 * Conventions.  Every function returns an int status (SK_OK = 0, negative =
 * error, positive = warning) and never aborts; sk_last_error() gives the
 * message of the last failure on the calling thread.  A plan is driven by one
 * host thread at a time (the reference keeps all I/O on its main thread,
 * spektri/src/dsp/output.rs:1-6).  The caller owns raw input and output
 * buffers; the plan owns all device state (the N/4 sample halo, the Welch
 * accumulator, twiddles, weights and scratch).  Complex samples are
 * interleaved float32 (re, im) — the complex64 wire format of fcfb.rs:180-187.
 */
#ifndef SPEKTRI_B200_H
#define SPEKTRI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define SK_OK               0
#define SK_WARN_FILTER      1   /* plan made; some filters were dropped, as fcfb.rs:58-61 does */
#define SK_ERR_ARG         -1   /* invalid argument (the reference would panic or clap would exit) */
#define SK_ERR_FILTER      -2   /* filter parameters not exactly representable (fcfb.rs:274-285) */
#define SK_ERR_CUDA        -3   /* a CUDA runtime call failed */
#define SK_ERR_NOMEM       -4   /* device or pinned host allocation failed */
#define SK_ERR_TIMEOUT     -5   /* a bounded device wait gave up */
#define SK_ERR_UNSUPPORTED -6   /* valid for the reference, not implemented on the device path */
#define SK_ERR_STATE       -7   /* call out of order */

/* ------------------------------------------------------------ enums */
/* Input sample formats: the DataFormat codes of spektri/src/dsp/data.rs:79-96. */
enum {
  SK_FMT_S8 = 0x04, SK_FMT_S16LE = 0x08, SK_FMT_S16BE = 0x09, SK_FMT_F32LE = 0x1C,
  SK_FMT_F32BE = 0x1D, SK_FMT_U8 = 0x24, SK_FMT_CS8 = 0x44, SK_FMT_CS16LE = 0x48,
  SK_FMT_CS16BE = 0x49, SK_FMT_CF32LE = 0x5C, SK_FMT_CF32BE = 0x5D, SK_FMT_CU8 = 0x64
};
/* Spectrum record formats: SpectrumFormat of spectrum.rs:29-32 (u8 at
 * 0.5 dB/LSB, u16 big-endian at 0.05 dB/LSB) plus f32 mean power acc/accn. */
enum { SK_SPEC_U8 = 0, SK_SPEC_U16 = 1, SK_SPEC_F32 = 2 };
/* Filter-bank execution: one launch per channel, or every channel in one
 * persistent size-ordered launch per buffer, replayed from a CUDA graph. */
enum { SK_MODE_PLAIN = 0, SK_MODE_BATCHED = 1 };

/* ------------------------------------------------------------ structures */
/* DspParams (dsp.rs:22-33) plus device selection. */
typedef struct {
  double   fs_in;            /* --samplerate */
  double   fc_in;            /* --centerfreq */
  uint32_t fft_size;         /* --fftsize, N */
  uint32_t ffts_per_buf;     /* --fftbuf, B (even for real input: multifft.rs:57-61) */
  uint32_t averages;         /* --averages */
  int32_t  input_format;     /* --inputformat, SK_FMT_* */
  int32_t  spectrum_format;  /* --spectrumformat, SK_SPEC_* */
  int32_t  mode;             /* SK_MODE_* */
  int32_t  device;           /* CUDA device ordinal */
  uint32_t flags;            /* reserved, must be 0 */
} sk_params;

/* FilterParams (fcfb.rs:206-210) plus weight design. */
typedef struct {
  double       fs_out;       /* fs= : output sample rate */
  double       fc_out;       /* fc= : output centre frequency */
  const float* weights;      /* w= : complex64[bins] on the host, W[j] scales bin first+j;
                                NULL selects designed real weights (below) */
  uint32_t     transition;   /* tw= : with weights==NULL, Tukey taper of this many bins per
                                side; 0 keeps the reference's raised cosine (fcfb.rs:197-203) */
  uint32_t     reserved;
} sk_filter;

/* InputBufferSize (dsp.rs:36-40) plus output sizing. */
typedef struct {
  uint64_t new_samples;      /* samples consumed per sk_process call: 3N/4 * B */
  uint64_t overlap;          /* N/4, carried inside the plan */
  uint64_t total;            /* new + overlap */
  uint64_t raw_bytes;        /* bytes of raw input per call */
  uint32_t result_bins;      /* K: N/2+1 (real) or N (complex) */
  uint32_t n_channels;       /* filters that passed validation, in their given order */
  uint32_t max_spectra;      /* upper bound on spectrum records per call */
  uint32_t spectrum_bytes;   /* payload bytes of one spectrum record (no metadata) */
} sk_plan_info;

typedef struct {
  uint32_t bins;             /* IFFT size n (BinNumbers.bins) */
  int32_t  filter_index;     /* position in the sk_filter array given at creation */
  int64_t  first;            /* first bin (BinNumbers.first) */
  double   fs_out, fc_out;
  uint64_t out_samples;      /* complex64 samples per call: B * 3n/4 */
} sk_channel_info;

typedef struct {
  uint32_t n_spectra;        /* spectrum records completed in this call */
  uint32_t reserved;
  uint64_t spectrum_seq0;    /* sequence number of the first one (spectrum.rs:36,160) */
} sk_result;

typedef struct sk_plan sk_plan;

/* ------------------------------------------------------------ host-only helpers
 * These need no GPU.  Bit-exact with the reference's f64 arithmetic. */

/* freq_to_bins (fcfb.rs:225-252).  SK_ERR_FILTER when bins <= 0. */
int sk_freq_to_bins(double fs_in, double fc_in, uint64_t fft_size, double fs_out, double fc_out,
                    uint32_t* bins, int64_t* first);
/* freq_to_bins_exact (fcfb.rs:274-285).  SK_ERR_FILTER unless the round trip is exact. */
int sk_freq_to_bins_exact(double fs_in, double fc_in, uint64_t fft_size, double fs_out, double fc_out,
                          uint32_t* bins, int64_t* first);
/* bins_to_freq (fcfb.rs:257-268). */
int sk_bins_to_freq(double fs_in, double fc_in, uint64_t fft_size, uint32_t bins, int64_t first,
                    double* fs_out, double* fc_out);
/* raised_cosine_weights (fcfb.rs:197-203) as complex64 with zero imaginary parts. */
int sk_raised_cosine_weights(uint32_t n, float* out_c64);
/* Periodic Tukey weights, tw taper bins per side (prototyping/fcfb.py:122). */
int sk_tukey_weights(uint32_t n, uint32_t tw, float* out_c64);
/* serialize_metadata (data.rs:110-132): 24 bytes <u64 seq, u64 secs, u32 nanos, u32 0>. */
int sk_serialize_metadata(uint8_t out[24], uint64_t seq, uint64_t secs, uint32_t nanos);
/* serialize_signal_topic (data.rs:137-153): [2, 0x40, 0x5C, 0 x5, f64 fs, f64 fc]. */
int sk_signal_topic(uint8_t out[24], double fs, double fc);
/* serialize_spectrum_topic (data.rs:157-171): [2, 0x60, fmt, 0 x5, f64 fd, f64 f0].
 * fmt is 0x24 (U8) for the u8 and u16 formats, as the reference writes, and
 * 0x1C (F32le) for the f32 extension. */
int sk_spectrum_topic(uint8_t out[24], int32_t spectrum_format, double fd, double f0);
/* bytes_per_input_sample / is_input_format_complex (inputformats.rs:12-44);
 * negative for an unknown format. */
int sk_format_bytes(int32_t input_format);
int sk_format_is_complex(int32_t input_format);

const char* sk_last_error(void);
const char* sk_version(void);

/* ------------------------------------------------------------ plans
 * DspState::init + Fcfb::add_filter per filter.  filter_status (optional,
 * n_filters entries) receives SK_OK or the reason each filter was dropped.
 * Sizes: fft_size a power of two (8 .. 2^21 complex points, 2^22 real
 * samples) or 3 * 2^k, 5 * 2^k whose complex length is R1 M with R1 = 3, 5,
 * 6, 10 or 12 and M = 16 .. 8192, else SK_ERR_UNSUPPORTED; filter IFFT sizes powers of
 * two from 4 to 65536 or other multiples of 4 up to 9364 (chirp-z), others
 * dropped with SK_ERR_UNSUPPORTED in filter_status. */
int sk_plan_create(const sk_params* params, const sk_filter* filters, int32_t n_filters,
                   int32_t* filter_status, sk_plan** out);
int sk_plan_info_get(const sk_plan* plan, sk_plan_info* info);
int sk_plan_channel(const sk_plan* plan, int32_t channel, sk_channel_info* info);
void sk_plan_destroy(sk_plan* plan);

/* Replace one channel's complex64 weights (natural order, `bins` values). */
int sk_set_weights(sk_plan* plan, int32_t channel, const float* weights_c64);
/* Copy one channel's current weights out (host memory). */
int sk_get_weights(const sk_plan* plan, int32_t channel, float* weights_c64);

/* One input buffer — DspState::process_real/process_complex with the
 * reference main loop's overlap carry (main.rs:171-191).
 *   raw        : info.raw_bytes of new samples in the plan's input format
 *   chan_out[c]: channel c's B*3n/4 complex64 output samples (payload of its
 *                record, fcfb.rs:84-87), c in [0, n_channels)
 *   spec_out   : room for info.max_spectra * info.spectrum_bytes; receives the
 *                payloads of the spectrum records completed by this call
 * sk_process takes host pointers (copies in, computes, copies out, returns
 * when done).  sk_process_device takes device pointers and only enqueues on
 * `stream` (a cudaStream_t; NULL = the plan's own stream, which is non-blocking:
 * work on the legacy default stream is not ordered with it, so a caller whose
 * buffers belong to the legacy default stream passes cudaStreamLegacy). */
int sk_process(sk_plan* plan, const void* raw, void* const* chan_out, void* spec_out, sk_result* result);
int sk_process_device(sk_plan* plan, const void* raw, void* const* chan_out, void* spec_out,
                      sk_result* result, void* stream);
/* Set the carried samples (main.rs:173): raw holds info.overlap samples in the
 * plan's input format, the last N/4 samples before the next buffer.  A fresh
 * plan carries zeros, as the reference's first buffer does (main.rs:165);
 * setting the carry lets a plan start in the middle of a stream (a time
 * shard on another GPU, or a restart). */
int sk_plan_set_carry(sk_plan* plan, const void* raw);

/* Wait for all work the plan enqueued. */
int sk_synchronize(sk_plan* plan);
/* Number of device kernels one sk_process_device call launches. */
int sk_launches_per_call(const sk_plan* plan);

/* ------------------------------------------------------------ differentiable filter bank
 * The filter-bank stage y_c = keep(IFFT_n(W'_c * gather(X, first_c))) as a
 * separate forward / adjoint pair on device spectra, for gradient-based
 * weight design.  X is [B][K] complex64 (the forward FFT of B blocks).
 *   sk_spectra_device : raw -> X for one buffer (advances the halo and the
 *                       Welch state exactly like sk_process_device)
 *   sk_fcfb_forward_device : X, W -> y (W_dev[c] = complex64[n_c] natural order);
 *                       X is first expanded into the plan's own extended
 *                       spectrum rows (bin m mod N at every m < N + max n,
 *                       the filter bank's gather layout), so calls on one plan
 *                       must stay ordered (one stream, or synchronised)
 *   sk_fcfb_backward_device: X, W, dy -> dW (summed over blocks) and dX
 *                       (accumulated into dX when not NULL); gradients follow
 *                       torch's convention for real losses of complex tensors
 *                       (dL/d conj(z)). */
int sk_spectra_device(sk_plan* plan, const void* raw, float* X, void* stream);
/* Stateless variant: raw holds the whole window, overlap + new samples
 * (N/4 + 3N/4 * B), so the same window always gives the same spectra and the
 * plan's carry is untouched; used to recompute spectra in backward passes. */
int sk_spectra_window_device(sk_plan* plan, const void* raw_window, float* X, void* stream);
int sk_fcfb_forward_device(sk_plan* plan, const float* X, const float* const* W, float* const* y, void* stream);
int sk_fcfb_backward_device(sk_plan* plan, const float* X, const float* const* W, const float* const* dy,
                            float* const* dW, float* dX, void* stream);

/* Per-stage device timing with CUDA events recorded on the launching stream
 * (off by default).  Stages: 0 forward FFT, 1 spectrum split + Welch
 * accumulation, 2 filter bank.  sk_plan_timing waits for the recorded work,
 * returns the summed milliseconds per stage and the number of calls
 * measured, and resets the totals. */
#define SK_N_STAGES 3
int sk_plan_set_timing(sk_plan* plan, int enable);
int sk_plan_timing(sk_plan* plan, double* ms_per_stage, uint64_t* calls);

/* Stage trace of the production path (the batched CUDA graph included):
 * every kernel folds the GPU's global timer into per-call slots (first
 * forward CTA start, last forward / Welch / filter-bank CTA end), which
 * cost one atomic per CTA and are always recorded.  With tracing enabled,
 * each sk_process_device call also copies its slots to pinned host memory
 * and resets them (two small copies after the call on its stream; up to
 * 4096 calls between reads).  sk_plan_trace waits for the device and
 * returns, per stage, the summed milliseconds of [forward start, forward
 * end], [forward end, Welch end] and [Welch end, filter-bank end] (each
 * stage's span as it runs back to back in the graph, launch gaps
 * included), the number of calls traced, and resets.  Reference
 * counterpart: none (the reference has no tracing; scripts wrap runs in
 * `time`, test/benchmark_spektri.sh:5-6). */
int sk_plan_set_trace(sk_plan* plan, int enable);
int sk_plan_trace(sk_plan* plan, double* ms_per_stage, uint64_t* calls);

/* ------------------------------------------------------------ tuning
 * The filter bank runs tiles of tile_size points and tile_threads threads:
 * 8192 x 256 (32 elements per thread), 8192 x 512 (16) or 4096 x 256 (16; an
 * 8192-point IFFT then runs as two independent 4096-point halves, one per
 * output parity), with ctas_per_sm persistent CTAs per SM.
 * sk_plan_autotune times every shape on the plan's own buffers (CUDA events,
 * 5 launches after 2 warm-ups), applies the fastest and appends it to the
 * JSON-lines file cache_path (when not NULL) under a key of device, FFT size,
 * input kind, blocks per buffer and channel mix; a later call with the same
 * key reads the cache instead of measuring.  Reference counterpart: none (the
 * reference uses rustfft's planner per size, fcfb.rs:143-150). */
int sk_plan_autotune(sk_plan* plan, const char* cache_path, double* best_us);
int sk_plan_set_tuning(sk_plan* plan, int32_t tile_size, int32_t tile_threads, int32_t ctas_per_sm);
int sk_plan_get_tuning(const sk_plan* plan, int32_t* tile_size, int32_t* tile_threads, int32_t* ctas_per_sm);

/* ------------------------------------------------------------ allocation-free spectra
 * No counterpart in the reference: an addition for callers that may not
 * allocate device memory — a real-time receive callback that must never
 * stall on cudaMalloc (it can synchronise the GPU for milliseconds and drop
 * samples), or a host application whose own pool owns the whole device
 * budget.  Same forward spectra as sk_spectra_device, with no plan and no
 * allocation: the FFT intermediates and twiddles live in one static device
 * array of SK_NOALLOC_SCRATCH_ELEMS complex floats (8 MiB) that every GPU
 * loading the library keeps until exit.
 *   raw : device, fft_size/4 + 3*fft_size/4 * n_blocks samples of
 *         input_format: the last N/4 samples of the previous window, then
 *         3N/4 * n_blocks new ones; block b is samples [b 3N/4, b 3N/4 + N)
 *   X   : device, n_blocks * K complex64 spectra, K = N/2+1 (real) or N
 * Limit: 32765 + N + n_blocks * Nc <= SK_NOALLOC_SCRATCH_ELEMS (32765 twiddles; Nc = N/2 for
 * real input, N for complex); larger requests return SK_ERR_ARG.  All calls
 * share the array: calls whose work overlaps on the GPU race.  The first call
 * on each device looks up the array's address and makes synchronous runtime
 * calls, so make it before any stream capture; the address is kept for the
 * process's life, so do not call this on a device after cudaDeviceReset. */
#define SK_NOALLOC_SCRATCH_ELEMS 1048576
int sk_spectra_noalloc(const void* raw, int32_t input_format, uint32_t fft_size, uint32_t n_blocks,
                       float* X, void* stream);

/* ------------------------------------------------------------ rational downconverter
 * The stage after the filter bank on one channel's complex64 output stream:
 * mixing with an exact rational oscillator and polyphase resampling by
 * interpolation / decimation.  Replaces RationalDdc (tools/ddc.py:51-145):
 * sk_ddc_create is RationalDdc.__init__ (taps designed for input rate x
 * interpolation, n_taps a multiple of the interpolation; the oscillator is
 * exp(2 pi i freq_num / freq_den) per sample, freq_den <= 2^24), and
 * sk_ddc_process_device is RationalDdc.execute: it consumes n_in device
 * samples and writes the outputs they complete (sk_ddc_outputs tells how many
 * beforehand: floor(S interpolation / decimation) exist after S samples).
 * State (FIR history, oscillator and polyphase phases) carries across calls;
 * one caller thread per object.  DesignDdc (ddc.py:148-177) is
 * spektri_b200/ddc.py's design_ddc. */
typedef struct sk_ddc sk_ddc;
int sk_ddc_create(const float* taps, uint32_t n_taps, uint32_t interpolation, uint32_t decimation, int64_t freq_num,
                  int64_t freq_den, int32_t device, sk_ddc** out);
int sk_ddc_outputs(const sk_ddc* ddc, uint64_t n_in, uint64_t* n_out);
int sk_ddc_process_device(sk_ddc* ddc, const float* in_c64, uint64_t n_in, float* out_c64, uint64_t* n_out,
                          void* stream);
void sk_ddc_destroy(sk_ddc* ddc);

/* ------------------------------------------------------------ post-detection stages
 * The demodulators' last stages after the downconverters, on one stream of
 * device samples (tools/demodulator.py):
 *   SK_AGC_SSB          complex64 in, complex64 out: SsbAgc.execute (:16-65)
 *   SK_AGC_AM           float32 in, float32 out: AmAgc.execute (:68-103)
 *   SK_AGC_AM_ENVELOPE  complex64 in, float32 out: |s| (AmDemodulator.execute,
 *                       :162) followed by AmAgc
 *   SK_ENVELOPE         complex64 in, float32 out: |s| alone (the AM
 *                       demodulator without its gain control)
 * sk_agc_process_device writes n outputs for n inputs; the gain control's
 * average amplitude carries across calls (0 at creation, as the reference's
 * constructors set it).  One caller thread per object. */
#define SK_AGC_SSB 1
#define SK_AGC_AM 2
#define SK_AGC_AM_ENVELOPE 3
#define SK_ENVELOPE 4
typedef struct sk_agc sk_agc;
int sk_agc_create(int32_t kind, int32_t device, sk_agc** out);
int sk_agc_process_device(sk_agc* agc, const float* in, uint64_t n, float* out, void* stream);
void sk_agc_destroy(sk_agc* agc);

/* Pinned host memory for staging (cudaHostAlloc); NULL on failure. */
void* sk_host_alloc(size_t bytes);
void sk_host_free(void* p);

#ifdef __cplusplus
}
#endif
#endif /* SPEKTRI_B200_H */
