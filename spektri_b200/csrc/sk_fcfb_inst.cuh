// Filter-bank kernel instances for one tile shape; included by the
// sk_fcfb_<shape>[_chirp].cu units so the shapes compile in parallel.
#pragma once
#include "sk_kernels.cuh"

namespace sk {

// The kernels read the extended spectrum layout, the same for real and
// complex input, so one instance serves both.
template <int S, int T, int MINB, bool CHIRP>
const void* fcfb_ptr(bool persistent) {
  return persistent ? (const void*)fcfb_kernel<S, T, MINB, true, CHIRP>
                    : (const void*)fcfb_kernel<S, T, MINB, false, CHIRP>;
}

}  // namespace sk
