"""The allocation-free entry point, swe_score_pairs_noalloc.

It is for callers that cannot allocate device memory - real-time hosts that
must not call the allocator once they have started, programs whose device
memory is all owned by their own pool, which the library cannot see - so the
tests hand it only device buffers they already own (made with torch here).
They check, on two calls in a row, that its distances equal those of the
existing explicit-pair entry point (swe_score_pairs) and of the oracle,
exactly (the work is integer); that it reproduces the reference's own golden
pairs; that an over-length pair is reported by status; and that free device
memory does not move across calls.  This file is collected last on purpose.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
import swgpu
from conftest import load_golden
from swgpu import workloads as W

pytestmark = pytest.mark.gpu

SWE_ERR_INVALID = 1


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


def _device_buffers(torch, seqs, lens=None):
    host = bytearray()
    offs = []
    for s in seqs:
        offs.append(len(host))
        host += s + b"\0"
    lens = [len(s) for s in seqs] if lens is None else list(lens)
    dev = torch.device("cuda:0")
    d_seqs = torch.frombuffer(bytearray(host), dtype=torch.uint8).to(dev)
    d_off = torch.tensor(offs, dtype=torch.int64, device=dev)
    d_len = torch.tensor(lens, dtype=torch.int32, device=dev)
    torch.cuda.synchronize(dev)
    return d_seqs, d_off, d_len, max(lens)


def _call(torch, bufs, a, b, max_len=None, expect=0):
    d_seqs, d_off, d_len, longest = bufs
    dev = d_seqs.device
    pairs = torch.tensor(np.stack([a, b], axis=1).reshape(-1), dtype=torch.int32, device=dev)
    out = torch.zeros(len(a), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    st = swgpu.lib().swe_score_pairs_noalloc(d_seqs.data_ptr(), d_off.data_ptr(), d_len.data_ptr(),
                                             pairs.data_ptr(), len(a), out.data_ptr(),
                                             longest if max_len is None else max_len,
                                             C.c_void_p(stream.cuda_stream))
    assert st == expect, swgpu.STATUS.get(st, st)
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
        sample = rng.choice(len(a), size=120, replace=False)
        ref = np.array([O.score(seqs[a[k]], seqs[b[k]]) for k in sample], dtype=np.uint32)
        assert np.array_equal(got[sample], ref), (call, sample[np.nonzero(got[sample] != ref)[0][:10]])
    eng.close()


def test_noalloc_reproduces_reference_golden_pairs():
    """The 641 pairs the reference's own score() produced (KATs, N runs, rare
    symbols, reverse complements, 480-1,300 bp, claimed lengths below the
    string length), scored in two calls of half the pairs each."""
    torch = pytest.importorskip("torch")
    pairs = load_golden("score_pairs.json.gz")
    P = len(pairs)
    seqs = [a.encode("latin-1") for a, b, la, lb, d in pairs] + [b.encode("latin-1") for a, b, la, lb, d in pairs]
    lens = [la for a, b, la, lb, d in pairs] + [lb for a, b, la, lb, d in pairs]
    bufs = _device_buffers(torch, seqs, lens)
    want = np.array([d for a, b, la, lb, d in pairs], dtype=np.uint32)
    idx = np.arange(P)
    for half in (idx[: P // 2], idx[P // 2:]):
        got = _call(torch, bufs, half.astype(np.int32), (half + P).astype(np.int32))
        assert np.array_equal(got, want[half]), half[np.nonzero(got != want[half])[0][:10]]


def test_noalloc_reports_pairs_longer_than_max_len():
    torch = pytest.importorskip("torch")
    seqs = _sequences()
    bufs = _device_buffers(torch, seqs)
    lens = np.array([len(s) for s in seqs])
    long_i = int(np.argmax(lens))
    a = np.array([0, long_i, 1, 2], dtype=np.int32)
    b = np.array([1, 0, 2, long_i], dtype=np.int32)
    limit = int(lens[long_i]) - 1
    assert max(lens[[0, 1, 2]]) <= limit
    got = _call(torch, bufs, a, b, max_len=limit, expect=SWE_ERR_INVALID)
    assert got[1] == 0xFFFFFFFF and got[3] == 0xFFFFFFFF
    assert got[0] == O.score(seqs[0], seqs[1]) and got[2] == O.score(seqs[1], seqs[2])
    # the next call starts from a cleared counter
    got = _call(torch, bufs, a[[0, 2]], b[[0, 2]], max_len=limit)
    assert list(got) == [O.score(seqs[0], seqs[1]), O.score(seqs[1], seqs[2])]


def test_noalloc_leaves_free_device_memory_unchanged():
    torch = pytest.importorskip("torch")
    seqs = _sequences()
    n = len(seqs)
    bufs = _device_buffers(torch, seqs)
    rng = np.random.default_rng(9)
    a = rng.integers(0, n, size=400).astype(np.int32)
    b = rng.integers(0, n, size=400).astype(np.int32)
    dev = bufs[0].device
    d_pairs = torch.tensor(np.stack([a, b], axis=1).reshape(-1), dtype=torch.int32, device=dev)
    d_out = torch.zeros(len(a), dtype=torch.int32, device=dev)
    lib = swgpu.lib()

    def call():
        return lib.swe_score_pairs_noalloc(bufs[0].data_ptr(), bufs[1].data_ptr(), bufs[2].data_ptr(),
                                           d_pairs.data_ptr(), len(a), d_out.data_ptr(), bufs[3], None)

    torch.cuda.synchronize(dev)
    assert call() == 0  # the first call on the device loads the module and looks up the array
    first = d_out.cpu().numpy().copy()
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(2):
        assert call() == 0
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    assert np.array_equal(d_out.cpu().numpy(), first)


def test_noalloc_rejects_sizes_beyond_its_limit():
    lib = swgpu.lib()
    # checked on the host before anything is enqueued
    st = lib.swe_score_pairs_noalloc(C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), C.c_void_p(1), 1,
                                     C.c_void_p(1), 65536, None)
    assert st == SWE_ERR_INVALID
