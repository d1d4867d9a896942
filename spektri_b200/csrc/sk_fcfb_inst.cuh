// Filter-bank kernel instances for one tile shape; included by the
// sk_fcfb_<shape>[_chirp].cu units so the shapes compile in parallel.
#pragma once
#include "sk_kernels.cuh"

namespace sk {

template <int S, int T, int MINB, bool CHIRP>
const void* fcfb_ptr(bool cplx, bool persistent) {
  if (persistent)
    return cplx ? (const void*)fcfb_kernel<S, T, MINB, true, false, CHIRP>
                : (const void*)fcfb_kernel<S, T, MINB, true, true, CHIRP>;
  return cplx ? (const void*)fcfb_kernel<S, T, MINB, false, false, CHIRP>
              : (const void*)fcfb_kernel<S, T, MINB, false, true, CHIRP>;
}

}  // namespace sk
