"""Time shards of one stream across GPUs (one process per GPU, no collective
on the data path).

Blocks are independent once their N/4-sample carry is known (main.rs:173),
so a stream splits into contiguous runs of buffers: rank r takes buffers
[first_r, first_r + count_r) and starts from the N/4 raw samples that precede
its first buffer (``Plan.set_carry``; rank 0 starts from zeros as the
reference does, main.rs:165).  Shard boundaries fall on Welch-window
boundaries (lcm(B, averages) blocks), so every spectrum record completes on
one rank; spectrum sequence numbers continue across ranks
(``spectrum_seq_offsets``), channel records keep the global buffer number as
their sequence number (fcfb.rs:84), and concatenating the ranks' records in
rank order gives the single-GPU stream.
"""
from __future__ import annotations

import math


def window_buffers(ffts_per_buf: int, averages: int) -> int:
    """Buffers per Welch window boundary: lcm(B, averages) / B."""
    a = max(1, int(averages))
    return math.lcm(int(ffts_per_buf), a) // int(ffts_per_buf)


def plan_shards(n_buffers: int, world: int, ffts_per_buf: int, averages: int):
    """[(first_buffer, count)] per rank: contiguous, in rank order, whole
    Welch windows each (the last rank also takes the trailing partial window)."""
    unit = window_buffers(ffts_per_buf, averages)
    units = n_buffers // unit
    base, extra = divmod(units, world)
    out, first = [], 0
    for r in range(world):
        count = (base + (1 if r < extra else 0)) * unit
        if r == world - 1:
            count = n_buffers - first
        out.append((first, count))
        first += count
    return out


def spectrum_seq_offsets(shards, ffts_per_buf: int, averages: int):
    """First spectrum sequence number of each rank."""
    a = max(1, int(averages))
    offs, done = [], 0
    for first, count in shards:
        offs.append(done)
        done += count * ffts_per_buf // a
    return offs


def carry_bytes(raw_stream, first_buffer: int, new_samples: int, overlap: int, bytes_per_sample: int):
    """The raw bytes of the `overlap` samples before buffer `first_buffer`
    (zeros for buffer 0).  raw_stream: bytes-like / uint8 array of the stream."""
    import numpy as np
    if first_buffer == 0:
        return None
    end = first_buffer * new_samples * bytes_per_sample
    start = end - overlap * bytes_per_sample
    return np.asarray(raw_stream[start:end], dtype=np.uint8)
