// Host-only parts of the C ABI: bin arithmetic, weight design, wire framing,
// format tables and error reporting.  Compiled with -ffp-contract=off so the
// f64 arithmetic rounds exactly like the reference's (no fused multiply-add).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "spektri_b200.h"
#include "sk_internal.h"

namespace sk {

static thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

void clear_error() { g_last_error.clear(); }

bool format_valid(int c) {
  switch (c) {
    case SK_FMT_S8: case SK_FMT_S16LE: case SK_FMT_S16BE: case SK_FMT_F32LE: case SK_FMT_F32BE:
    case SK_FMT_U8: case SK_FMT_CS8: case SK_FMT_CS16LE: case SK_FMT_CS16BE: case SK_FMT_CF32LE:
    case SK_FMT_CF32BE: case SK_FMT_CU8: return true;
  }
  return false;
}
// The format code packs complex (bits 7-6), number kind (5-4), width (3-1)
// and endianness (bit 0): data.rs:55-78.
bool format_complex(int c) { return (c & 0xC0) == 0x40; }
int format_bits(int c) { int b = (c >> 1) & 7; return b == 2 ? 8 : b == 4 ? 16 : b == 6 ? 32 : 0; }
int format_bytes(int c) { return format_bits(c) / 8 * (format_complex(c) ? 2 : 1); }
// input_format_scaling (inputformats.rs:47-62), evaluated in f32.
float format_scaling(int c) {
  int b = format_bits(c);
  if (b == 8) return 1.0f / 127.0f;
  if (b == 16) return 1.0f / 32767.0f;
  return 1.0f;
}

// nearest_multiple (fcfb.rs:233-235): f64 round half away from zero, then a
// saturating cast like Rust's `as isize` (NaN -> 0).
static long long nearest_multiple(double value, long long multiple) {
  double r = std::round(value / (double)multiple) * (double)multiple;
  if (std::isnan(r)) return 0;
  if (r >= 9.2233720368547758e18) return INT64_MAX;
  if (r <= -9.2233720368547758e18) return INT64_MIN;
  return (long long)r;
}

bool freq_to_bins(double fs, double fc, long long N, double fs_out, double fc_out, long long* bins, long long* first) {
  const long long multiple = 4;    // 25 % overlap needs IFFT sizes in multiples of 4 (fcfb.rs:230-232)
  double spacing = fs / (double)N;
  long long b = nearest_multiple(fs_out / spacing, multiple);
  long long center = nearest_multiple((fc_out - fc) / spacing, multiple);
  if (b <= 0) return false;
  *bins = b;
  *first = center - b / 2;
  return true;
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

void raised_cosine(uint32_t n, float* out) {
  // fcfb.rs:197-203: 0.5 - 0.5 cos(i * 2pi/n), all in f32 (libm cosf).
  const float pi = 3.14159265358979323846f;
  const float f = (2.0f * pi) / (float)n;
  for (uint32_t i = 0; i < n; ++i) {
    out[2 * i] = 0.5f - 0.5f * std::cos((float)i * f);
    out[2 * i + 1] = 0.0f;
  }
}

void tukey(uint32_t n, uint32_t tw, float* out) {
  // Periodic Tukey: the symmetric window of length n+1 (cosine tapers of
  // tw bins rising from 0 and falling back) with its last sample dropped.
  for (uint32_t k = 0; k < n; ++k) { out[2 * k] = 1.0f; out[2 * k + 1] = 0.0f; }
  if (tw == 0) return;
  const double alpha = 2.0 * tw / n;
  if (alpha >= 1.0) {
    for (uint32_t k = 0; k < n; ++k) out[2 * k] = (float)(0.5 - 0.5 * std::cos(2.0 * M_PI * k / n));
    return;
  }
  const int m = (int)n + 1;
  const int width = (int)std::floor(alpha * (m - 1) / 2.0);
  for (int k = 0; k < (int)n; ++k) {
    double v = 1.0;
    if (k <= width) v = 0.5 * (1.0 + std::cos(M_PI * (-1.0 + 2.0 * k / alpha / (m - 1))));
    else if (k >= m - width - 1) v = 0.5 * (1.0 + std::cos(M_PI * (-2.0 / alpha + 1.0 + 2.0 * k / alpha / (m - 1))));
    out[2 * k] = (float)v;
  }
}

static void le64(uint8_t* p, uint64_t v) { for (int i = 0; i < 8; ++i) p[i] = (uint8_t)(v >> (8 * i)); }
static void le32(uint8_t* p, uint32_t v) { for (int i = 0; i < 4; ++i) p[i] = (uint8_t)(v >> (8 * i)); }
static void lef64(uint8_t* p, double v) { uint64_t u; std::memcpy(&u, &v, 8); le64(p, u); }

}  // namespace sk

using namespace sk;

extern "C" {

const char* sk_last_error(void) { return g_last_error.c_str(); }
const char* sk_version(void) { return "spektri_b200 1.0 (sm_100a)"; }

int sk_format_bytes(int32_t f) { return format_valid(f) ? format_bytes(f) : SK_ERR_ARG; }
int sk_format_is_complex(int32_t f) { return format_valid(f) ? (format_complex(f) ? 1 : 0) : SK_ERR_ARG; }

int sk_freq_to_bins(double fs_in, double fc_in, uint64_t N, double fs_out, double fc_out, uint32_t* bins, int64_t* first) {
  long long b = 0, f = 0;
  if (!bins || !first || N == 0) return fail(SK_ERR_ARG, "sk_freq_to_bins: null output or zero FFT size");
  if (!freq_to_bins(fs_in, fc_in, (long long)N, fs_out, fc_out, &b, &f)) return fail(SK_ERR_FILTER, "Invalid filter parameters");
  if (b > UINT32_MAX) return fail(SK_ERR_UNSUPPORTED, "IFFT size %lld too large", b);
  *bins = (uint32_t)b; *first = f;
  return SK_OK;
}

int sk_freq_to_bins_exact(double fs_in, double fc_in, uint64_t N, double fs_out, double fc_out, uint32_t* bins, int64_t* first) {
  long long b = 0, f = 0;
  if (!bins || !first || N == 0) return fail(SK_ERR_ARG, "sk_freq_to_bins_exact: null output or zero FFT size");
  if (!freq_to_bins_exact(fs_in, fc_in, (long long)N, fs_out, fc_out, &b, &f)) return fail(SK_ERR_FILTER, "Invalid filter parameters");
  if (b > UINT32_MAX) return fail(SK_ERR_UNSUPPORTED, "IFFT size %lld too large", b);
  *bins = (uint32_t)b; *first = f;
  return SK_OK;
}

int sk_bins_to_freq(double fs_in, double fc_in, uint64_t N, uint32_t bins, int64_t first, double* fs_out, double* fc_out) {
  if (!fs_out || !fc_out || N == 0) return fail(SK_ERR_ARG, "sk_bins_to_freq: null output or zero FFT size");
  bins_to_freq(fs_in, fc_in, (long long)N, bins, first, fs_out, fc_out);
  return SK_OK;
}

int sk_raised_cosine_weights(uint32_t n, float* out) {
  if (!out || n == 0) return fail(SK_ERR_ARG, "sk_raised_cosine_weights: bad arguments");
  raised_cosine(n, out);
  return SK_OK;
}

int sk_tukey_weights(uint32_t n, uint32_t tw, float* out) {
  if (!out || n == 0) return fail(SK_ERR_ARG, "sk_tukey_weights: bad arguments");
  tukey(n, tw, out);
  return SK_OK;
}

int sk_serialize_metadata(uint8_t out[24], uint64_t seq, uint64_t secs, uint32_t nanos) {
  if (!out) return fail(SK_ERR_ARG, "null buffer");
  le64(out, seq); le64(out + 8, secs); le32(out + 16, nanos); le32(out + 20, 0);
  return SK_OK;
}

int sk_signal_topic(uint8_t out[24], double fs, double fc) {
  if (!out) return fail(SK_ERR_ARG, "null buffer");
  std::memset(out, 0, 24);
  out[0] = 2; out[1] = 0x40; out[2] = SK_FMT_CF32LE;   // PROTOCOL_VERSION, Waveform, Cf32le
  lef64(out + 8, fs); lef64(out + 16, fc);
  return SK_OK;
}

int sk_spectrum_topic(uint8_t out[24], int32_t spectrum_format, double fd, double f0) {
  if (!out) return fail(SK_ERR_ARG, "null buffer");
  std::memset(out, 0, 24);
  out[0] = 2; out[1] = 0x60;
  out[2] = spectrum_format == SK_SPEC_F32 ? SK_FMT_F32LE : SK_FMT_U8;
  lef64(out + 8, fd); lef64(out + 16, f0);
  return SK_OK;
}

}  // extern "C"
