"""The sweep generator (spektri_b200/bin/testsignal) against the float32
restatement of testsignal/src/main.rs:27-77 (oracle/testsignal.py): the same
bytes for every format, whole buffers of 1024 samples only, and the
reference's exit codes for option errors.  No GPU needed."""
import os
import subprocess

import pytest

from oracle import testsignal as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "spektri_b200", "bin", "testsignal")


@pytest.mark.parametrize("fmt", ["s16le", "f32le", "cs16le", "cf32le"])
@pytest.mark.parametrize("n", [100000, 1024, 1000, 0])
def test_sweep_bytes_match_restatement(fmt, n):
    assert os.path.exists(BIN), "build spektri_b200/bin/testsignal first"
    r = subprocess.run([BIN, "--format", fmt, f"--samples={n}"], capture_output=True, timeout=60)
    assert r.returncode == 0
    want = T.testsignal(fmt, n)
    assert len(r.stdout) == len(want) == (n // 1024) * 1024 * (2 if fmt.startswith("c") else 1) * \
        (2 if "16" in fmt else 4)
    assert r.stdout == want


def test_option_errors():
    assert subprocess.run([BIN, "-f", "s16le"], capture_output=True).returncode == 101         # samples missing
    assert subprocess.run([BIN, "-f", "u8", "-n", "10"], capture_output=True).returncode == 101  # not a format
    assert subprocess.run([BIN, "-x"], capture_output=True).returncode == 1                     # unknown option
