"""Python face of a filter-bank plan (the reference's DspState, dsp.rs:42-160).

``Plan`` owns an ``sk_plan``.  ``process`` is the host-pointer path
(DspState::process_real / process_complex with main.rs's overlap carry);
``process_device`` takes torch CUDA tensors and only enqueues work.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

from . import _lib
from ._lib import check, lib

FORMATS = {
    "s8": 0x04, "s16le": 0x08, "s16be": 0x09, "f32le": 0x1C, "f32be": 0x1D, "u8": 0x24,
    "cs8": 0x44, "cs16le": 0x48, "cs16be": 0x49, "cf32le": 0x5C, "cf32be": 0x5D, "cu8": 0x64,
}
SPECTRUM_FORMATS = {"u8": _lib.SPEC_U8, "u16": _lib.SPEC_U16, "f32": _lib.SPEC_F32}
SPECTRUM_DTYPES = {_lib.SPEC_U8: np.dtype(np.uint8), _lib.SPEC_U16: np.dtype(">u2"), _lib.SPEC_F32: np.dtype(np.float32)}
MODES = {"plain": _lib.MODE_PLAIN, "batched": _lib.MODE_BATCHED}


def format_code(fmt) -> int:
    """DataFormat code (data.rs:79-96) from a name (case-insensitive) or a code."""
    if isinstance(fmt, str):
        try:
            return FORMATS[fmt.lower()]
        except KeyError:
            raise ValueError(f"unknown input format {fmt!r}") from None
    return int(fmt)


def pinned_empty(shape, dtype) -> np.ndarray:
    """A numpy array in page-locked host memory (fast DMA to and from the GPU)."""
    dtype = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dtype.itemsize
    ptr = lib().sk_host_alloc(max(nbytes, 1))
    if not ptr:
        raise MemoryError(_lib.last_error())
    buf = (C.c_uint8 * max(nbytes, 1)).from_address(ptr)
    arr = np.frombuffer(buf, dtype=np.uint8, count=nbytes).view(dtype).reshape(shape)
    weakref.finalize(buf, lib().sk_host_free, ptr)
    return arr


def _ptr(x) -> int:
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    return int(x)


class Plan:
    """One GPU filter bank + Welch spectrum (DspState::init, dsp.rs:76-111).

    filters: sequence of dicts with ``fs_out``, ``fc_out`` and optionally
    ``weights`` (complex64[bins], natural order) or ``transition`` (Tukey
    taper bins).  Filters whose parameters are not exact are dropped with a
    message, as Fcfb::add_filter does (fcfb.rs:58-61); ``filter_status``
    tells which.
    """

    def __init__(self, fs_in, fft_size, input_format, filters=(), fc_in=0.0, ffts_per_buf=8,
                 averages=2000, spectrum_format="u8", mode="batched", device=0):
        L = lib()
        self.input_format = format_code(input_format)
        self.spectrum_format = SPECTRUM_FORMATS[spectrum_format] if isinstance(spectrum_format, str) else int(spectrum_format)
        self.mode = MODES[mode] if isinstance(mode, str) else int(mode)
        p = _lib.Params(float(fs_in), float(fc_in), int(fft_size), int(ffts_per_buf), int(averages),
                        self.input_format, self.spectrum_format, self.mode, int(device), 0)
        filters = list(filters)
        arr = (_lib.Filter * max(1, len(filters)))()
        self._wkeep = []
        for i, f in enumerate(filters):
            w = f.get("weights")
            wp = None
            if w is not None:
                w = np.ascontiguousarray(np.asarray(w, dtype=np.complex64))
                self._wkeep.append(w)
                wp = w.ctypes.data
            arr[i] = _lib.Filter(float(f["fs_out"]), float(f["fc_out"]), wp, int(f.get("transition", 0)), 0)
        status = (C.c_int32 * max(1, len(filters)))()
        h = C.c_void_p()
        rc = L.sk_plan_create(C.byref(p), arr, len(filters), status, C.byref(h))
        check(rc, "sk_plan_create")
        self._h = h
        self.device = int(device)
        self.filter_status = list(status)[: len(filters)]
        info = _lib.PlanInfo()
        check(L.sk_plan_info_get(h, C.byref(info)))
        self.new_samples = info.new_samples
        self.overlap = info.overlap
        self.total = info.total
        self.raw_bytes = info.raw_bytes
        self.result_bins = info.result_bins
        self.n_channels = info.n_channels
        self.max_spectra = info.max_spectra
        self.spectrum_bytes = info.spectrum_bytes
        self.ffts_per_buf = int(ffts_per_buf)
        self.averages = int(averages)
        self.fft_size = int(fft_size)
        self.fs_in, self.fc_in = float(fs_in), float(fc_in)
        self.channels = []
        for c in range(self.n_channels):
            ci = _lib.ChannelInfo()
            check(L.sk_plan_channel(h, c, C.byref(ci)))
            self.channels.append(dict(bins=ci.bins, first=ci.first, fs_out=ci.fs_out, fc_out=ci.fc_out,
                                      out_samples=ci.out_samples, filter_index=ci.filter_index))
        self.spectrum_dtype = SPECTRUM_DTYPES[self.spectrum_format]
        self.launches_per_call = L.sk_launches_per_call(h)
        self._out_tables = {}

    # ----------------------------------------------------------- lifecycle
    def close(self):
        if getattr(self, "_h", None):
            lib().sk_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ----------------------------------------------------------- weights
    def set_weights(self, channel: int, weights) -> None:
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.complex64))
        assert w.shape == (self.channels[channel]["bins"],)
        check(lib().sk_set_weights(self._h, channel, w.ctypes.data), "sk_set_weights")

    def get_weights(self, channel: int) -> np.ndarray:
        w = np.empty(self.channels[channel]["bins"], np.complex64)
        check(lib().sk_get_weights(self._h, channel, w.ctypes.data), "sk_get_weights")
        return w

    # ----------------------------------------------------------- processing
    def empty_outputs(self, pinned: bool = False):
        """Host buffers for one call: (channel outputs, spectrum buffer).  The
        channel outputs are views of one block in channel order, which the
        host path fills with a single copy."""
        mk = pinned_empty if pinned else (lambda s, d: np.empty(s, d))
        sizes = [c["out_samples"] for c in self.channels]
        block = mk((max(1, sum(sizes)),), np.complex64)
        offs = np.concatenate([[0], np.cumsum(sizes)]).astype(int)
        outs = [block[offs[i]:offs[i + 1]] for i in range(len(sizes))]
        spec = mk((self.max_spectra * self.spectrum_bytes,), np.uint8)
        return outs, spec

    def _table(self, ptrs):
        key = tuple(ptrs)
        t = self._out_tables.get(key)
        if t is None:
            if len(self._out_tables) > 64:
                self._out_tables.clear()
            t = (C.c_void_p * max(1, len(ptrs)))(*ptrs)
            self._out_tables[key] = t
        return t

    def process_into(self, raw, outs, spec) -> _lib.Result:
        """Host path into caller buffers (numpy arrays, ideally pinned)."""
        raw = np.ascontiguousarray(raw) if isinstance(raw, np.ndarray) else np.frombuffer(raw, np.uint8)
        if raw.nbytes != self.raw_bytes:
            raise ValueError(f"raw input must be {self.raw_bytes} bytes, got {raw.nbytes}")
        r = _lib.Result()
        tbl = self._table([_ptr(o) for o in outs])
        check(lib().sk_process(self._h, raw.ctypes.data, tbl, _ptr(spec), C.byref(r)), "sk_process")
        return r

    def process(self, raw):
        """One buffer: returns (spectra, outputs); spectra = [(seq, values)]."""
        outs, spec = self.empty_outputs()
        r = self.process_into(raw, outs, spec)
        return self.split_spectra(spec, r), outs

    def split_spectra(self, spec, r):
        sb = self.spectrum_bytes
        spec = np.asarray(spec).view(np.uint8)
        return [(r.spectrum_seq0 + i, spec[i * sb:(i + 1) * sb].view(self.spectrum_dtype).copy())
                for i in range(r.n_spectra)]

    def process_device(self, raw, outs, spec, stream=None) -> _lib.Result:
        """Device path: torch CUDA tensors (or raw device pointers).  Enqueues
        on ``stream`` (torch stream / handle; default: torch's current stream)."""
        stream = _stream(stream, self.device)
        r = _lib.Result()
        tbl = self._table([_ptr(o) for o in outs])
        check(lib().sk_process_device(self._h, _ptr(raw), tbl, _ptr(spec) if spec is not None else None,
                                      C.byref(r), stream), "sk_process_device")
        return r

    def autotune(self, cache_path=None):
        """Pick the filter-bank tile shape and persistent grid by timing (or
        from the JSON-lines cache).  Returns (tile_size, tile_threads, ctas_per_sm, us)."""
        if cache_path is None:
            cache_path = os.environ.get("SPEKTRI_TUNE_CACHE") or os.path.join(
                os.path.expanduser("~"), ".cache", "spektri_b200", "tune.jsonl")
        if cache_path:
            os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        us = C.c_double()
        check(lib().sk_plan_autotune(self._h, cache_path.encode() if cache_path else None, C.byref(us)), "sk_plan_autotune")
        return self.tuning() + (us.value,)

    def set_tuning(self, tile_size: int, tile_threads: int, ctas_per_sm: int):
        """Filter-bank tile shape: 8192 x 256, 8192 x 512 or 4096 x 256, and
        persistent CTAs per SM."""
        check(lib().sk_plan_set_tuning(self._h, int(tile_size), int(tile_threads), int(ctas_per_sm)),
              "sk_plan_set_tuning")

    def tuning(self):
        z, t, c = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().sk_plan_get_tuning(self._h, C.byref(z), C.byref(t), C.byref(c)))
        return z.value, t.value, c.value

    def set_timing(self, enable: bool = True):
        check(lib().sk_plan_set_timing(self._h, int(bool(enable))))

    def timing(self):
        """(ms per stage [fwd_fft, welch, fcfb], calls) since the last read."""
        ms = (C.c_double * 3)()
        n = C.c_uint64()
        check(lib().sk_plan_timing(self._h, ms, C.byref(n)), "sk_plan_timing")
        return list(ms), n.value

    def set_trace(self, enable: bool = True):
        """Trace every following call's stage spans from device timestamps
        (also inside the batched CUDA graph)."""
        check(lib().sk_plan_set_trace(self._h, int(bool(enable))))

    def trace(self):
        """(ms per stage [fwd_fft, welch, fcfb] summed over the traced calls,
        calls) since the last read: each stage's span in the production path."""
        ms = (C.c_double * 3)()
        n = C.c_uint64()
        check(lib().sk_plan_trace(self._h, ms, C.byref(n)), "sk_plan_trace")
        return list(ms), n.value

    def set_carry(self, raw):
        """Carried samples (the N/4 raw samples before the next buffer), so a
        plan can start mid-stream: a time shard or a restart."""
        raw = np.ascontiguousarray(raw).view(np.uint8)
        need = self.overlap * (self.raw_bytes // self.new_samples)
        if raw.nbytes != need:
            raise ValueError(f"carry must be {need} bytes, got {raw.nbytes}")
        check(lib().sk_plan_set_carry(self._h, raw.ctypes.data), "sk_plan_set_carry")

    def synchronize(self):
        check(lib().sk_synchronize(self._h))

    # ----------------------------------------------------------- differentiable stage
    def spectra_device(self, raw, X, stream=None):
        stream = _stream(stream, self.device)
        check(lib().sk_spectra_device(self._h, _ptr(raw), _ptr(X), stream), "sk_spectra_device")

    def spectra_window_device(self, raw_window, X, stream=None):
        """Stateless spectra of a window of N/4 + new samples (carry untouched)."""
        stream = _stream(stream, self.device)
        check(lib().sk_spectra_window_device(self._h, _ptr(raw_window), _ptr(X), stream), "sk_spectra_window_device")

    def fcfb_forward_device(self, X, W, y, stream=None):
        stream = _stream(stream, self.device)
        wt = (C.c_void_p * max(1, len(W)))(*[_ptr(w) for w in W])
        yt = (C.c_void_p * max(1, len(y)))(*[_ptr(v) for v in y])
        check(lib().sk_fcfb_forward_device(self._h, _ptr(X), wt, yt, stream), "sk_fcfb_forward_device")

    def fcfb_backward_device(self, X, W, dy, dW, dX=None, stream=None):
        stream = _stream(stream, self.device)
        wt = (C.c_void_p * max(1, len(W)))(*[_ptr(w) for w in W])
        dyt = (C.c_void_p * max(1, len(dy)))(*[_ptr(v) for v in dy])
        dwt = (C.c_void_p * max(1, len(dW)))(*[_ptr(v) for v in dW])
        check(lib().sk_fcfb_backward_device(self._h, _ptr(X), wt, dyt, dwt, _ptr(dX) if dX is not None else None,
                                            stream), "sk_fcfb_backward_device")


CUDA_STREAM_LEGACY = 1        # cudaStreamLegacy: the legacy default stream, named explicitly


def _stream(stream, device):
    """The cudaStream_t handle for a torch stream (default: torch's current
    stream) or a raw handle.  Torch's default stream has handle 0, which the
    C ABI reads as "the plan's own stream" (non-blocking, unordered with
    torch's work), so it is passed as cudaStreamLegacy instead."""
    if stream is None:
        import torch
        stream = torch.cuda.current_stream(device)
    h = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
    return h if h else CUDA_STREAM_LEGACY
