// spektri — drop-in replacement for the reference binary (spektri/src/main.rs)
// with the filter bank and spectrum on a B200 through libspektri_b200.
//
// Same command line (main.rs:15-66), filter grammar (main.rs:70-91), stdin
// framing (main.rs:113-193) and outputs: every record is published on a
// ZeroMQ PUB socket as (topic24, metadata24 + payload) (output.rs:49-60),
// filter records are appended to their file= (header + payload), spectrum
// records are also written to stdout (spectrum.rs:73-78).  Per buffer the
// spectrum records come first, then the filters in their configured order
// (dsp.rs:157-158, fcfb.rs:93-95).
//
// Additions, all off by default: --spectrumformat=f32, filter keys tw= and w=,
// --mode=plain|batched (default batched), --device=N,
// --fake-clock=<secs>,<step_ns> (deterministic timestamps for tests) and
// --stats (at exit, one stderr line with the run's throughput, each
// pipeline stage's busy time and the device stage spans per buffer).
#include <cerrno>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <cstring>
#include <ctime>
#include <mutex>
#include <string>
#include <thread>
#include <strings.h>
#include <unistd.h>
#include <vector>

#include "spektri_b200.h"
#include "zmq_pub.h"

namespace {

struct FilterArg {
  double fs = 0, fc = 0;
  std::string file, wpath;
  uint32_t tw = 0;
  std::vector<float> weights;
};

[[noreturn]] void usage_error(const std::string& msg) {
  fprintf(stderr, "error: %s\n", msg.c_str());
  exit(1);   // clap's Error::exit
}

[[noreturn]] void panic(const std::string& msg) {
  fprintf(stderr, "thread 'main' panicked: %s\n", msg.c_str());
  exit(101); // Rust panic exit code
}

int parse_format(const std::string& s) {
  static const struct { const char* n; int c; } t[] = {
      {"s8", SK_FMT_S8}, {"s16le", SK_FMT_S16LE}, {"s16be", SK_FMT_S16BE}, {"f32le", SK_FMT_F32LE},
      {"f32be", SK_FMT_F32BE}, {"u8", SK_FMT_U8}, {"cs8", SK_FMT_CS8}, {"cs16le", SK_FMT_CS16LE},
      {"cs16be", SK_FMT_CS16BE}, {"cf32le", SK_FMT_CF32LE}, {"cf32be", SK_FMT_CF32BE}, {"cu8", SK_FMT_CU8}};
  for (auto& e : t)
    if (strcasecmp(s.c_str(), e.n) == 0) return e.c;
  return -1;
}

double parse_f64(const std::string& v, const char* what, bool is_panic) {
  char* end = nullptr;
  errno = 0;
  double d = strtod(v.c_str(), &end);
  if (v.empty() || *end != 0) {
    std::string m = std::string("invalid value '") + v + "' for " + what;
    if (is_panic) panic(m);
    usage_error(m);
  }
  return d;
}

long long parse_int(const std::string& v, const char* what) {
  char* end = nullptr;
  long long d = strtoll(v.c_str(), &end, 10);
  if (v.empty() || *end != 0 || d < 0) usage_error(std::string("invalid value '") + v + "' for " + what);
  return d;
}

// main.rs:70-91
FilterArg parse_filter(const std::string& s) {
  FilterArg f;
  bool have_fs = false, have_fc = false;
  size_t pos = 0;
  while (true) {
    size_t e = s.find(':', pos);
    std::string kv = s.substr(pos, e == std::string::npos ? std::string::npos : e - pos);
    size_t eq = kv.find('=');
    if (eq == std::string::npos) panic("called `Option::unwrap()` on a `None` value (filter parameter '" + kv + "')");
    std::string k = kv.substr(0, eq), v = kv.substr(eq + 1);
    if (k == "fs") { f.fs = parse_f64(v, "fs", true); have_fs = true; }
    else if (k == "fc") { f.fc = parse_f64(v, "fc", true); have_fc = true; }
    else if (k == "file") f.file = v;
    else if (k == "tw") f.tw = (uint32_t)parse_f64(v, "tw", true);
    else if (k == "w") f.wpath = v;
    if (e == std::string::npos) break;
    pos = e + 1;
  }
  if (!have_fs || !have_fc) panic("called `Option::unwrap()` on a `None` value (filter needs fs= and fc=)");
  if (!f.wpath.empty()) {
    FILE* wf = fopen(f.wpath.c_str(), "rb");
    if (!wf) panic("cannot read weights file " + f.wpath);
    float buf[4096];
    size_t r;
    while ((r = fread(buf, sizeof(float), 4096, wf)) > 0) f.weights.insert(f.weights.end(), buf, buf + r);
    fclose(wf);
  }
  return f;
}

bool read_exact(uint8_t* p, size_t n) {
  size_t got = 0;
  while (got < n) {
    ssize_t r = read(0, p + got, n - got);
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) return false;
    got += (size_t)r;
  }
  return true;
}

void write_all(FILE* f, const void* p, size_t n) {
  if (f && n) fwrite(p, 1, n, f);
}

}  // namespace

int main(int argc, char** argv) {
  sk_params p{};
  p.fc_in = 0;
  p.fft_size = 16384;         // main.rs:44
  p.ffts_per_buf = 8;         // main.rs:49
  p.averages = 2000;          // main.rs:55
  p.spectrum_format = SK_SPEC_U8;
  p.mode = SK_MODE_BATCHED;
  p.device = 0;
  bool have_fs = false;
  int fmt = -1;
  std::vector<std::string> filter_strs, binds;
  bool fake = false, stats = false;
  unsigned long long clk_secs = 0, clk_step = 0;

  auto take = [&](int& i, const std::string& a, const char* lng, const char* sht, std::string& out) -> bool {
    const std::string L = std::string("--") + lng;
    if (a == L || (sht && a == std::string("-") + sht)) {
      if (i + 1 >= argc) usage_error("The argument '" + L + "' requires a value but none was supplied");
      out = argv[++i];
      return true;
    }
    if (a.rfind(L + "=", 0) == 0) { out = a.substr(L.size() + 1); return true; }
    if (sht && a.size() > 2 && a.rfind(std::string("-") + sht, 0) == 0) {
      out = a.substr(2);
      if (!out.empty() && out[0] == '=') out = out.substr(1);
      return true;
    }
    return false;
  };
  auto more_values = [&](int& i, std::vector<std::string>& dst) {
    while (i + 1 < argc && argv[i + 1][0] != '-') dst.push_back(argv[++i]);
  };
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i], v;
    if (a == "--stats") { stats = true; continue; }
    if (take(i, a, "samplerate", "s", v)) { p.fs_in = parse_f64(v, "samplerate", false); have_fs = true; }
    else if (take(i, a, "centerfreq", "f", v)) p.fc_in = parse_f64(v, "centerfreq", false);
    else if (take(i, a, "fftsize", "n", v)) p.fft_size = (uint32_t)parse_int(v, "fftsize");
    else if (take(i, a, "fftbuf", nullptr, v)) p.ffts_per_buf = (uint32_t)parse_int(v, "fftbuf");
    else if (take(i, a, "averages", "a", v)) p.averages = (uint32_t)parse_int(v, "averages");
    else if (take(i, a, "inputformat", "I", v)) {
      fmt = parse_format(v);
      if (fmt < 0) usage_error("'" + v + "' isn't a valid value for '--inputformat <FORMAT>'");
    } else if (take(i, a, "spectrumformat", nullptr, v)) {
      if (strcasecmp(v.c_str(), "u8") == 0) p.spectrum_format = SK_SPEC_U8;
      else if (strcasecmp(v.c_str(), "u16") == 0) p.spectrum_format = SK_SPEC_U16;
      else if (strcasecmp(v.c_str(), "f32") == 0) p.spectrum_format = SK_SPEC_F32;
      else usage_error("'" + v + "' isn't a valid value for '--spectrumformat <FORMAT>'");
    } else if (take(i, a, "filters", nullptr, v)) { filter_strs.push_back(v); more_values(i, filter_strs); }
    else if (take(i, a, "zmqbind", nullptr, v)) { binds.push_back(v); more_values(i, binds); }
    else if (take(i, a, "mode", nullptr, v)) p.mode = (v == "plain") ? SK_MODE_PLAIN : SK_MODE_BATCHED;
    else if (take(i, a, "device", nullptr, v)) p.device = (int32_t)parse_int(v, "device");
    else if (take(i, a, "fake-clock", nullptr, v)) {
      fake = true;
      if (sscanf(v.c_str(), "%llu,%llu", &clk_secs, &clk_step) != 2) usage_error("--fake-clock=<secs>,<step_ns>");
    } else usage_error("Found argument '" + a + "' which wasn't expected");
  }
  if (!have_fs) usage_error("The argument '--samplerate <HZ>' is required");
  if (fmt < 0) usage_error("The argument '--inputformat <FORMAT>' is required");
  p.input_format = fmt;
  if (binds.empty()) binds.push_back("ipc:///tmp/spektri.zmq");   // main.rs:65

  std::vector<FilterArg> fa;
  for (auto& s : filter_strs) fa.push_back(parse_filter(s));

  // main.rs:97-102
  ZmqPub zmq;
  std::string err;
  if (!zmq.load(&err)) panic(err);
  for (auto& b : binds)
    if (!zmq.bind(b, &err)) panic(err);

  std::vector<sk_filter> sf(fa.size());
  for (size_t i = 0; i < fa.size(); ++i) {
    sf[i].fs_out = fa[i].fs;
    sf[i].fc_out = fa[i].fc;
    sf[i].transition = fa[i].tw;
    sf[i].weights = fa[i].weights.empty() ? nullptr : fa[i].weights.data();
  }
  std::vector<int32_t> status(fa.size(), 0);
  sk_plan* plan = nullptr;
  int rc = sk_plan_create(&p, sf.data(), (int32_t)sf.size(), status.data(), &plan);
  if (rc < 0) {
    fprintf(stderr, "spektri: %s\n", sk_last_error());
    return rc == SK_ERR_ARG ? 101 : 1;
  }
  sk_plan_info info{};
  sk_plan_info_get(plan, &info);

  // One output per surviving filter (output.rs:24-46: a file that cannot be
  // created only prints a message).
  struct Out { uint8_t topic[24]; FILE* file = nullptr; uint64_t n = 0; };
  std::vector<Out> outs(info.n_channels);
  for (uint32_t c = 0; c < info.n_channels; ++c) {
    sk_channel_info ci{};
    sk_plan_channel(plan, (int32_t)c, &ci);
    const FilterArg& f = fa[ci.filter_index];
    sk_signal_topic(outs[c].topic, f.fs, f.fc);
    outs[c].n = ci.out_samples;
    if (!f.file.empty()) {
      outs[c].file = fopen(f.file.c_str(), "wb");
      if (!outs[c].file) fprintf(stderr, "Could not create file: %s\n", strerror(errno));
    }
  }
  uint8_t spec_topic[24];
  sk_spectrum_topic(spec_topic, p.spectrum_format, p.fs_in / (double)p.fft_size, p.fc_in);   // spectrum.rs:57-65

  // Three pipelined stages over a ring of pinned slots, so reading stdin,
  // the GPU call (copy in, process, copy out) and the output I/O of
  // consecutive buffers overlap; records still leave in buffer order.  A slot
  // holds the raw input, one record buffer per channel (24-byte header then
  // payload) and the spectrum payloads.
  const int bps = sk_format_bytes(fmt);
  const size_t raw_bytes = info.new_samples * (size_t)bps;
  constexpr int NSLOT = 3;
  struct Slot {
    uint8_t* raw = nullptr;
    std::vector<uint8_t*> rec;
    std::vector<void*> payload;
    uint8_t* spec = nullptr;
    sk_result r{};
    uint64_t seq = 0, secs = 0;
    uint32_t nanos = 0;
    int state = 0;        // 0 free, 1 read, 2 processed, 3 end of stream
  } slots[NSLOT];
  for (auto& sl : slots) {
    sl.raw = (uint8_t*)sk_host_alloc(raw_bytes);
    sl.rec.resize(info.n_channels);
    sl.payload.resize(info.n_channels);
    for (uint32_t c = 0; c < info.n_channels; ++c) {
      sl.rec[c] = (uint8_t*)sk_host_alloc(32 + outs[c].n * 8);
      if (!sl.rec[c]) { fprintf(stderr, "spektri: %s\n", sk_last_error()); return 1; }
      sl.payload[c] = sl.rec[c] + 32;   // 16-byte aligned payload; the header goes at +8
    }
    sl.spec = (uint8_t*)sk_host_alloc((size_t)info.max_spectra * info.spectrum_bytes);
    if (!sl.raw || !sl.spec) { fprintf(stderr, "spektri: %s\n", sk_last_error()); return 1; }
  }
  std::mutex mu;
  std::condition_variable cv;
  bool failed = false;
  // --stats: busy seconds of each pipeline stage, device stage spans
  using clk = std::chrono::steady_clock;
  auto secs_since = [](clk::time_point t0) { return std::chrono::duration<double>(clk::now() - t0).count(); };
  double t_read = 0, t_gpu = 0, t_write = 0, dev_ms[SK_N_STAGES] = {};
  uint64_t n_done = 0, dev_calls = 0;
  const clk::time_point t_start = clk::now();
  auto drain_trace = [&] {
    double ms[SK_N_STAGES];
    uint64_t n = 0;
    if (sk_plan_trace(plan, ms, &n) == SK_OK) {
      for (int s = 0; s < SK_N_STAGES; ++s) dev_ms[s] += ms[s];
      dev_calls += n;
    }
  };
  if (stats) sk_plan_set_trace(plan, 1);
  auto wait_state = [&](Slot& sl, int want) {
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [&] { return failed || sl.state == want || (want == 1 && sl.state == 3); });
    return !failed;
  };
  auto set_state = [&](Slot& sl, int st) {
    { std::lock_guard<std::mutex> lk(mu); sl.state = st; }
    cv.notify_all();
  };

  // Stage 1: stdin (main.rs:176-178: a short read ends the stream).
  std::thread reader([&] {
    for (uint64_t seq = 0;; ++seq) {
      Slot& sl = slots[seq % NSLOT];
      if (!wait_state(sl, 0)) return;
      const clk::time_point t0 = clk::now();
      const bool full = read_exact(sl.raw, raw_bytes);
      t_read += secs_since(t0);
      if (!full) { set_state(sl, 3); return; }
      sl.seq = seq;
      if (fake) {
        const unsigned long long t = clk_secs * 1000000000ull + seq * clk_step;
        sl.secs = t / 1000000000ull;
        sl.nanos = (uint32_t)(t % 1000000000ull);
      } else {
        timespec ts;
        clock_gettime(CLOCK_REALTIME, &ts);   // main.rs:180
        sl.secs = (uint64_t)ts.tv_sec;
        sl.nanos = (uint32_t)ts.tv_nsec;
      }
      set_state(sl, 1);
    }
  });
  // Stage 3: framing and output, in buffer order.
  uint8_t spec_topic_copy[24];
  std::memcpy(spec_topic_copy, spec_topic, 24);
  std::thread writer([&] {
    std::vector<uint8_t> srec(24 + info.spectrum_bytes);
    for (uint64_t k = 0;; ++k) {
      Slot& sl = slots[k % NSLOT];
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return failed || sl.state == 2 || sl.state == 3; });
        if (failed || sl.state == 3) return;
      }
      const clk::time_point t0 = clk::now();
      for (uint32_t s = 0; s < sl.r.n_spectra; ++s) {
        sk_serialize_metadata(srec.data(), sl.r.spectrum_seq0 + s, sl.secs, sl.nanos);
        std::memcpy(srec.data() + 24, sl.spec + (size_t)s * info.spectrum_bytes, info.spectrum_bytes);
        zmq.send2(spec_topic_copy, 24, srec.data(), srec.size());
        write_all(stdout, srec.data(), srec.size());
      }
      for (uint32_t c = 0; c < info.n_channels; ++c) {
        uint8_t* h = sl.rec[c] + 8;
        sk_serialize_metadata(h, sl.seq, sl.secs, sl.nanos);     // fcfb.rs:84: seq of the buffer
        const size_t len = 24 + outs[c].n * 8;
        zmq.send2(outs[c].topic, 24, h, len);
        write_all(outs[c].file, h, len);
      }
      t_write += secs_since(t0);
      set_state(sl, 0);
    }
  });
  // Stage 2: the GPU call.
  int exit_code = 0;
  for (uint64_t k = 0;; ++k) {
    Slot& sl = slots[k % NSLOT];
    if (!wait_state(sl, 1)) break;
    if (sl.state == 3) {
      // end of stream: let the writer drain and stop at this slot
      std::unique_lock<std::mutex> lk(mu);
      cv.notify_all();
      break;
    }
    const clk::time_point t0 = clk::now();
    rc = sk_process(plan, sl.raw, sl.payload.data(), sl.spec, &sl.r);
    t_gpu += secs_since(t0);
    ++n_done;
    if (stats && n_done % 1024 == 0) drain_trace();
    if (rc < 0) {
      fprintf(stderr, "spektri: %s\n", sk_last_error());
      exit_code = 1;
      { std::lock_guard<std::mutex> lk(mu); failed = true; }
      cv.notify_all();
      break;
    }
    set_state(sl, 2);
  }
  if (exit_code) {
    // stdin may still block the reader: leave without joining it
    fflush(stdout);
    _exit(exit_code);
  }
  writer.join();
  reader.join();
  fflush(stdout);
  if (stats) {
    drain_trace();
    const double wall = secs_since(t_start), per = dev_calls ? 1e3 / (double)dev_calls : 0.0;
    const double samples = (double)n_done * (double)info.new_samples;
    fprintf(stderr,
            "spektri stats: %llu buffers, %.0f samples in %.3f s = %.2f Msamples/s; busy: stdin %.3f s, "
            "GPU calls %.3f s, output %.3f s; device per buffer: forward FFT %.1f us, Welch %.1f us, "
            "filter bank %.1f us\n",
            (unsigned long long)n_done, samples, wall, wall > 0 ? samples / wall / 1e6 : 0.0, t_read, t_gpu, t_write,
            dev_ms[0] * per, dev_ms[1] * per, dev_ms[2] * per);
  }
  for (auto& o : outs)
    if (o.file) fclose(o.file);
  sk_plan_destroy(plan);
  return 0;
}
