// Minimal ZeroMQ PUB socket over a dlopen'd libzmq (C API of libzmq 4.x:
// zmq_ctx_new, zmq_socket, zmq_bind, zmq_send, zmq_close, zmq_ctx_term).
// The reference publishes every record as a 2-part message: the 24-byte topic
// with ZMQ_SNDMORE, then header + payload (spektri/src/dsp/output.rs:49-60).
#pragma once
#include <dlfcn.h>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

class ZmqPub {
 public:
  static constexpr int kPub = 1;       // ZMQ_PUB
  static constexpr int kSndMore = 2;   // ZMQ_SNDMORE

  ~ZmqPub() {
    if (sock_) close_(sock_);
    if (ctx_) term_(ctx_);
  }

  // Loads libzmq: $SPEKTRI_LIBZMQ first, then the usual sonames.
  bool load(std::string* err) {
    std::vector<std::string> names;
    if (const char* e = std::getenv("SPEKTRI_LIBZMQ")) names.push_back(e);
    names.push_back("libzmq.so.5");
    names.push_back("libzmq.so");
    for (auto& n : names) {
      h_ = dlopen(n.c_str(), RTLD_NOW | RTLD_LOCAL);
      if (h_) break;
    }
    if (!h_) { *err = "cannot load libzmq (set SPEKTRI_LIBZMQ to its path)"; return false; }
    ctx_new_ = (void* (*)())dlsym(h_, "zmq_ctx_new");
    socket_ = (void* (*)(void*, int))dlsym(h_, "zmq_socket");
    bind_ = (int (*)(void*, const char*))dlsym(h_, "zmq_bind");
    send_ = (int (*)(void*, const void*, size_t, int))dlsym(h_, "zmq_send");
    close_ = (int (*)(void*))dlsym(h_, "zmq_close");
    term_ = (int (*)(void*))dlsym(h_, "zmq_ctx_term");
    errno_ = (int (*)())dlsym(h_, "zmq_errno");
    strerror_ = (const char* (*)(int))dlsym(h_, "zmq_strerror");
    if (!ctx_new_ || !socket_ || !bind_ || !send_ || !close_ || !term_) { *err = "libzmq lacks the C API"; return false; }
    ctx_ = ctx_new_();
    if (!ctx_) { *err = "zmq_ctx_new failed"; return false; }
    sock_ = socket_(ctx_, kPub);
    if (!sock_) { *err = "zmq_socket failed"; return false; }
    return true;
  }

  bool bind(const std::string& addr, std::string* err) {
    if (bind_(sock_, addr.c_str()) != 0) {
      *err = "zmq_bind(" + addr + "): " + (strerror_ && errno_ ? strerror_(errno_()) : "failed");
      return false;
    }
    return true;
  }

  // Errors are ignored, as the reference drops the send Result (fcfb.rs:94).
  void send2(const void* topic, size_t tn, const void* msg, size_t mn) {
    send_(sock_, topic, tn, kSndMore);
    send_(sock_, msg, mn, 0);
  }

 private:
  void* h_ = nullptr;
  void* ctx_ = nullptr;
  void* sock_ = nullptr;
  void* (*ctx_new_)() = nullptr;
  void* (*socket_)(void*, int) = nullptr;
  int (*bind_)(void*, const char*) = nullptr;
  int (*send_)(void*, const void*, size_t, int) = nullptr;
  int (*close_)(void*) = nullptr;
  int (*term_)(void*) = nullptr;
  int (*errno_)() = nullptr;
  const char* (*strerror_)(int) = nullptr;
};
