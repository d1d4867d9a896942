// testsignal — the reference's sweep generator (testsignal/src/main.rs),
// the integration stimulus for the filter bank: a complex (or real) tone
// whose frequency sweeps the whole band from -pi to pi rad/sample over the
// run, written to stdout in s16le, f32le, cs16le or cf32le.
//
// Same options (main.rs:27-34): -f/--format=<FORMAT>, -n/--samples=<NUMBER>.
// Same arithmetic, in float32 like the reference (main.rs:40-76): buffers of
// 1024 samples, nsamples / 1024 of them; per sample I = cos(phase) (and
// Q = sin(phase) for IQ), s16 as (v * 32767) truncated toward zero;
// freq = -pi + step * counter with step = 2 pi / (1024 * nbufs), and
// phase = fmod(phase + freq, 2 pi).  Built with -ffp-contract=off so no
// multiply-add is fused, as in the reference.
#include <cmath>
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <strings.h>
#include <vector>

namespace {

[[noreturn]] void usage(const std::string& msg) {
  fprintf(stderr, "error: %s\n\nUSAGE:\n    testsignal [OPTIONS]\n\nOPTIONS:\n"
          "    -f, --format <FORMAT>     Data format (s16le, f32le, cs16le or cf32le)\n"
          "    -n, --samples <NUMBER>    Number of samples to produce\n", msg.c_str());
  exit(1);
}

// main.rs:33-37: value_t!(...).unwrap() panics on a missing or bad value
[[noreturn]] void panic(const std::string& msg) {
  fprintf(stderr, "thread 'main' panicked: %s\n", msg.c_str());
  exit(101);
}

void put_f32(std::vector<uint8_t>& b, size_t& o, float v) {
  std::memcpy(&b[o], &v, 4);   // little-endian host
  o += 4;
}
void put_i16(std::vector<uint8_t>& b, size_t& o, float v) {
  const int16_t s = (int16_t)v;   // |v| <= 32767: truncation toward zero, as Rust's `as i16`
  std::memcpy(&b[o], &s, 2);
  o += 2;
}

}  // namespace

int main(int argc, char** argv) {
  signal(SIGPIPE, SIG_IGN);   // a closed stdout is a write error, as for the reference
  std::string fmt, samples;
  bool have_fmt = false, have_n = false;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    auto value = [&](const char* lng, const char* sht, std::string& out) {
      const std::string L = std::string("--") + lng, S = std::string("-") + sht;
      if (a == L || a == S) {
        if (i + 1 >= argc) usage("The argument '" + L + "' requires a value but none was supplied");
        out = argv[++i];
        return true;
      }
      if (a.rfind(L + "=", 0) == 0) { out = a.substr(L.size() + 1); return true; }
      if (a.rfind(S, 0) == 0 && a.size() > 2) { out = a.substr(2); return true; }
      return false;
    };
    if (value("format", "f", fmt)) have_fmt = true;
    else if (value("samples", "n", samples)) have_n = true;
    else usage("Found argument '" + a + "' which wasn't expected");
  }
  if (!have_fmt) panic("called `Result::unwrap()` on an `Err` value: the argument 'format' was not supplied");
  int code = 0;
  if (!strcasecmp(fmt.c_str(), "s16le")) code = 0x08;
  else if (!strcasecmp(fmt.c_str(), "f32le")) code = 0x1C;
  else if (!strcasecmp(fmt.c_str(), "cs16le")) code = 0x48;
  else if (!strcasecmp(fmt.c_str(), "cf32le")) code = 0x5C;
  else panic("called `Result::unwrap()` on an `Err` value: '" + fmt + "' isn't a valid value for 'format'");
  if (!have_n) panic("called `Result::unwrap()` on an `Err` value: the argument 'samples' was not supplied");
  char* end = nullptr;
  const long long nsamples = strtoll(samples.c_str(), &end, 10);
  if (samples.empty() || *end) panic("called `Result::unwrap()` on an `Err` value: invalid digit found in string");

  const bool is_iq = (code & 0xC0) == 0x40;
  const bool is_s16 = (code & 0x1F) == 0x08;
  const size_t buflen = 1024;
  const long long nbufs = nsamples / (long long)buflen;
  const float PI = 3.14159265358979323846f;
  const float init_freq = -PI;
  const float freq_step = 2.0f * PI / ((float)buflen * (float)nbufs);
  float phase = 0.0f;
  std::vector<uint8_t> buf(buflen * (is_iq ? 2 : 1) * (is_s16 ? 2 : 4));
  long long counter = 0;
  for (long long j = 0; j < nbufs; ++j) {
    size_t o = 0;
    for (size_t i = 0; i < buflen; ++i) {
      const float si = cosf(phase);
      if (is_s16) put_i16(buf, o, si * 32767.0f); else put_f32(buf, o, si);
      if (is_iq) {
        const float sq = sinf(phase);
        if (is_s16) put_i16(buf, o, sq * 32767.0f); else put_f32(buf, o, sq);
      }
      const float freq = init_freq + freq_step * (float)counter;
      phase = fmodf(phase + freq, 2.0f * PI);
      ++counter;
    }
    if (fwrite(buf.data(), 1, buf.size(), stdout) != buf.size())           // main.rs:75: write_all(..).unwrap()
      panic("called `Result::unwrap()` on an `Err` value: Broken pipe");
  }
  return 0;
}
