"""Multi-process (world size 2, gloo on CPU) check of time sharding: each
rank processes its contiguous shard of one stream, primed with the N/4
samples before it, and rank 0 checks that the concatenated channel records
and spectrum records equal one unsharded run.  The per-rank processor here is
the FP64 oracle; on GPUs it is a Plan primed with Plan.set_carry."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle64
from spektri_b200 import shard

N, B, AVG, NBUF = 256, 4, 8, 11
I = N * 3 // 4
CHANS = [(32, 20), (64, -40), (16, 100)]


def _stream():
    rng = np.random.default_rng(17)
    return np.clip(np.round(rng.normal(0, 2000, NBUF * B * I)), -32768, 32767).astype("<i2")


def _oracle():
    return oracle64.Oracle64("s16le", N, B, AVG, [oracle64.Channel(n, f, oracle64.raised_cosine_weights(n).astype(np.complex128))
                                                  for n, f in CHANS])


def _worker(rank, world, port, result_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        raw = _stream()
        shards = shard.plan_shards(NBUF, world, B, AVG)
        seq0 = shard.spectrum_seq_offsets(shards, B, AVG)[rank]
        first, count = shards[rank]
        o = _oracle()
        carry = shard.carry_bytes(raw.view(np.uint8), first, B * I, N // 4, 2)
        if carry is not None:                     # what Plan.set_carry does on a GPU
            o.buf[o.new:] = oracle64.convert(carry, "s16le")
        spectra, outs = [], []
        for b in range(first, first + count):
            sp, oc = o.process(raw[b * B * I:(b + 1) * B * I].tobytes())
            spectra += [(s + seq0, v) for s, v in sp]
            outs.append((b, oc))
        gathered = [None] * world
        dist.all_gather_object(gathered, (spectra, outs))
        if rank == 0:
            result_q.put(gathered)
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_plan_shards_align_to_welch_windows():
    assert shard.window_buffers(64, 256) == 4
    assert shard.window_buffers(64, 100) == 25
    sh = shard.plan_shards(341, 8, 64, 256)
    assert sh[0] == (0, 44) and sum(c for _, c in sh) == 341
    assert all(c % 4 == 0 for _, c in sh[:-1])
    assert [f for f, _ in sh] == [sum(c for _, c in sh[:i]) for i in range(8)]
    assert shard.spectrum_seq_offsets(sh, 64, 256)[1] == 44 * 64 // 256


def test_two_rank_shards_reproduce_single_stream():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    gathered = q.get(timeout=300)
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    # single run
    raw = _stream()
    o = _oracle()
    ref_sp, ref_out = [], []
    for b in range(NBUF):
        sp, oc = o.process(raw[b * B * I:(b + 1) * B * I].tobytes())
        ref_sp += sp
        ref_out.append(oc)
    got_sp = [x for g in gathered for x in g[0]]
    got_out = [x for g in gathered for x in g[1]]
    assert [s for s, _ in got_sp] == [s for s, _ in ref_sp]
    for (_, a), (_, r) in zip(got_sp, ref_sp):
        assert np.allclose(a, r, rtol=1e-12, atol=0)
    assert [b for b, _ in got_out] == list(range(NBUF))
    for (_, a), r in zip(got_out, ref_out):
        for x, y in zip(a, r):
            assert np.allclose(x, y, rtol=1e-10, atol=1e-15)
