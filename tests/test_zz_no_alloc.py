"""The allocation-free entry point, swe_score_pairs_noalloc.

It is for callers that cannot allocate device memory - code running during a
CUDA graph capture, real-time hosts that must not call the allocator after
start-up, programs whose device memory belongs to a pool the library cannot
see - so the test hands it only device buffers it already owns (made with
torch here) and checks, on two calls in a row, that its distances equal those
of the existing explicit-pair entry point (swe_score_pairs), exactly: the
work is integer.  This file is collected last on purpose.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import swgpu
from swgpu import workloads as W

pytestmark = pytest.mark.gpu


def _sequences():
    rng = np.random.default_rng(77)
    seqs = []
    for _ in range(60):  # short and medium DNA, some with N runs
        s = bytearray(W.BASES[rng.integers(0, 4, size=int(rng.integers(20, 400)))].tobytes())
        if rng.random() < 0.3:
            p = int(rng.integers(0, len(s)))
            s[p:p + 15] = b"N" * len(s[p:p + 15])
        seqs.append(bytes(s))
    for _ in range(12):  # longer than one 512-column chunk: these use the scratch column
        base = W.BASES[rng.integers(0, 4, size=int(rng.integers(600, 2600)))]
        seqs.append(base.tobytes())
        seqs.append(W._mutate(rng, base.copy(), 0.05, 0.01).tobytes())
    seqs += [b"ACGTRYKMSW" * 9, b"", b"A", b"acgtACGT" * 20]
    return seqs


def _device_buffers(torch, seqs):
    host = bytearray()
    offs, lens = [], []
    for s in seqs:
        offs.append(len(host))
        host += s + b"\0"
        lens.append(len(s))
    dev = torch.device("cuda:0")
    d_seqs = torch.frombuffer(bytearray(host), dtype=torch.uint8).to(dev)
    d_off = torch.tensor(offs, dtype=torch.int64, device=dev)
    d_len = torch.tensor(lens, dtype=torch.int32, device=dev)
    return d_seqs, d_off, d_len, max(lens)


def _call(torch, bufs, a, b):
    d_seqs, d_off, d_len, max_len = bufs
    dev = d_seqs.device
    pairs = torch.tensor(np.stack([a, b], axis=1).reshape(-1), dtype=torch.int32, device=dev)
    out = torch.zeros(len(a), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    st = swgpu.lib().swe_score_pairs_noalloc(d_seqs.data_ptr(), d_off.data_ptr(), d_len.data_ptr(),
                                             pairs.data_ptr(), len(a), out.data_ptr(), max_len,
                                             C.c_void_p(stream.cuda_stream))
    assert st == 0, swgpu.STATUS.get(st, st)
    torch.cuda.synchronize(dev)
    return out.cpu().numpy().view(np.uint32)


def test_noalloc_matches_pairs_entry_point_twice():
    torch = pytest.importorskip("torch")
    seqs = _sequences()
    n = len(seqs)
    rng = np.random.default_rng(5)
    eng = swgpu.Engine(device=0)
    eng.upload(seqs)
    bufs = _device_buffers(torch, seqs)
    for call in range(2):
        a = rng.integers(0, n, size=700).astype(np.int32)
        b = rng.integers(0, n, size=700).astype(np.int32)
        a[:n] = np.arange(n)  # every sequence at least once, long ones against long ones too
        b[:n] = np.roll(np.arange(n), 1 + call)
        want = eng.score_pairs(a, b)
        got = _call(torch, bufs, a, b)
        assert np.array_equal(got, want), (call, np.nonzero(got != want)[0][:10])
    eng.close()


def test_noalloc_rejects_sizes_beyond_its_limit():
    lib = swgpu.lib()
    # checked on the host before anything is enqueued
    st = lib.swe_score_pairs_noalloc(C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), 1,
                                     C.c_void_p(1), 65536, None)
    assert st == 1  # SWE_ERR_INVALID
