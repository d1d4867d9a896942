"""Checker for the spektri filter-bank + Welch path (test infrastructure only).

``oracle64``: float64 numpy restatement (error floor).
``oracle32``: ctypes wrapper of the FP32 C++ restatement (CPU baseline, "port").
Only tests, the smoke check and the benchmark's CPU-baseline leg may use this
package; the product path never imports it.
"""
