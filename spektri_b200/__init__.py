"""spektri_b200: the fast-convolution filter bank and Welch spectrum of
tejeez/spektri on NVIDIA B200 (sm_100a).

The compute path is libspektri_b200.so (hand-written CUDA kernels behind a C
ABI, include/spektri_b200.h); this package is its Python face: ``Plan`` (the
device filter bank), the reference-shaped ``dsp`` module, the differentiable
filter-bank stage (``autograd``), the workload generators, and the stages
downstream of a channel (``ddc``: the rational downconverter, ``demod``: the
SSB / AM / IQ demodulators).
"""
from .plan import Plan, FORMATS, format_code, pinned_empty
from . import dsp
from ._lib import SpektriError, lib

__all__ = ["Plan", "FORMATS", "format_code", "pinned_empty", "dsp", "SpektriError", "lib"]
