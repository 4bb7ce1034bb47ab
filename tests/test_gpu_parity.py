"""GPU engine parity: every distance, neighbour list, cluster label, log line
and file must equal the reference's (golden vectors produced by the
reference itself) or the oracle's on the same seeded inputs.  Integer work:
the bar is bit-exact."""
from __future__ import annotations

import base64
import hashlib
import math
import subprocess
import zlib
from pathlib import Path

import numpy as np
import pytest

import oracle as O
import swgpu
from conftest import load_golden
from swgpu import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = swgpu.Engine()
    yield e
    e.close()


def _matrix(eng, seqs):
    eng.upload(seqs)
    eng.score_all_pairs()
    return eng.distances()


def _row_diag(D, golden):
    D16 = D.astype("<u2")
    bad = [i for i in range(D.shape[0]) if zlib.crc32(D16[i].tobytes()) != golden["row_crc32"][i]]
    return bad[:10]


# ---------------------------------------------------------------------------
# single pairs
# ---------------------------------------------------------------------------
def test_dropin_score_matches_reference_pairs():
    pairs = load_golden("score_pairs.json.gz")
    bad = []
    for a, b, la, lb, d in pairs:
        got = swgpu.score(a.encode("latin-1"), b.encode("latin-1"), la, lb)
        if got != d:
            bad.append((a[:20], b[:20], la, lb, d, got))
    assert not bad, bad[:5]


def test_engine_pairs_and_matrix_match_reference_pairs(eng):
    """The golden pairs scored as one dataset: explicit pairs (32-bit kernel)
    and the all-pairs matrix (16x2 kernel plus the 32-bit path for rare
    symbols, empty and long sequences) agree with the reference."""
    import ctypes as C
    pairs = load_golden("score_pairs.json.gz")
    P = len(pairs)
    # full strings with their claimed lengths: the engine reads s[1..len], so a
    # claimed length below the string length keeps the character at s[len]
    seqs = [a.encode("latin-1") for a, b, la, lb, d in pairs] + [b.encode("latin-1") for a, b, la, lb, d in pairs]
    lens = [la for a, b, la, lb, d in pairs] + [lb for a, b, la, lb, d in pairs]
    bufs = [C.create_string_buffer(s, len(s) + 1) for s in seqs]
    ptrs = (C.c_char_p * len(bufs))(*[C.addressof(x) for x in bufs])
    lens_c = (C.c_size_t * len(bufs))(*lens)
    swgpu._check(swgpu.lib().swe_upload(eng.ctx, ptrs, lens_c, len(bufs)), eng.ctx)
    eng.n = len(bufs)
    want = np.array([d for a, b, la, lb, d in pairs], dtype=np.uint32)
    got = eng.score_pairs(np.arange(P), np.arange(P) + P)
    assert np.array_equal(got, want), np.nonzero(got != want)[0][:10]
    eng.score_all_pairs()
    D = eng.distances()
    diag = D[np.arange(P), np.arange(P) + P]
    assert np.array_equal(diag, want), np.nonzero(diag != want)[0][:10]
    assert np.array_equal(D, D.T)


# ---------------------------------------------------------------------------
# full matrices against the reference
# ---------------------------------------------------------------------------
def test_config1_matrix_bit_exact(eng):
    seqs, _ = W.config1()
    g = load_golden("config1_golden.json")
    D = _matrix(eng, seqs)
    assert hashlib.sha256(D.astype("<u2").tobytes()).hexdigest() == g["sha256"], _row_diag(D, g)
    st = eng.stats()
    assert st["reruns"] == 0 and st["n_fast"] == 2000


@pytest.mark.parametrize("name,gen", [("config2_head1500_golden", lambda: W.config2()[0][:1500]),
                                      ("config3_head1500_golden", lambda: W.config3()[0][:1500])])
def test_subset_matrices_bit_exact(eng, name, gen):
    seqs = gen()
    g = load_golden(name + ".json")
    D = _matrix(eng, seqs)
    assert hashlib.sha256(D.astype("<u2").tobytes()).hexdigest() == g["sha256"], _row_diag(D, g)


def test_forced_saturation_rerun_is_exact():
    """With the saturation guard lowered, pairs whose 16-bit maximum reaches it
    are rescored by the 32-bit kernel; the matrix must not change."""
    seqs, _ = W.config1()
    seqs = seqs[:600]
    ref = O.all_pairs(seqs)
    e = swgpu.Engine(sat_limit=400)
    D = _matrix(e, seqs)
    st = e.stats()
    e.close()
    assert st["reruns"] > 1000
    assert np.array_equal(D, ref)


def _mixed_set(rng):
    seqs = []
    for L in list(range(1, 40)) + [63, 64, 65, 127, 128, 129, 191, 192, 193, 255, 256, 383, 384, 385,
                                   511, 512, 513, 700, 767, 768, 769, 900, 1030, 1600]:
        seqs.append(W.BASES[rng.integers(0, 4, size=L)].tobytes())
    base = seqs[-5]
    seqs += [base, base[:300] + b"N" * 40 + base[340:], base.lower(), b"", b"", b"A", b"N",
             b"ACGTRYKMACGT" * 5, b"-" * 30, b"ACGT" * 50 + b"Z"]
    for _ in range(40):
        s = bytearray(W.BASES[rng.integers(0, 4, size=int(rng.integers(80, 400)))].tobytes())
        for _ in range(int(rng.integers(0, 4))):
            p = int(rng.integers(0, len(s)))
            s[p:p + 12] = b"N" * len(s[p:p + 12])
        seqs.append(bytes(s))
    return seqs


@pytest.mark.parametrize("ppb,threads", [(32, 256), (1, 32), (3, 96), (7, 128)])
def test_mixed_lengths_symbols_and_tile_shapes(ppb, threads):
    rng = np.random.default_rng(21)
    seqs = _mixed_set(rng)
    ref = O.all_pairs(seqs)
    e = swgpu.Engine(packs_per_block=ppb, threads=threads)
    D = _matrix(e, seqs)
    st = e.stats()
    e.close()
    assert st["n_exceptional"] > 0 and st["n_fast"] > 0
    bad = np.argwhere(D != ref)
    assert len(bad) == 0, [(int(i), int(j), int(D[i, j]), int(ref[i, j])) for i, j in bad[:5]]


def test_long_sequences_need_uint32_matrix():
    rng = np.random.default_rng(5)
    seqs = [W.BASES[rng.integers(0, 4, size=17000)].tobytes()]
    seqs.append(W._mutate(rng, np.frombuffer(seqs[0], dtype=np.uint8).copy(), 0.02, 0.0).tobytes())
    seqs.append(W.BASES[rng.integers(0, 4, size=300)].tobytes())
    seqs += [W.BASES[rng.integers(0, 4, size=int(rng.integers(50, 300)))].tobytes() for _ in range(70)]
    e = swgpu.Engine()
    D = _matrix(e, seqs)
    assert e.stats()["dist_bytes"] == 4
    for i in range(3):
        for k in range(3):
            assert D[i, k] == O.score(seqs[k], seqs[i]), (i, k)
    ref = O.all_pairs(seqs)
    assert np.array_equal(D, ref)
    for eps in [500.0, 1200.0, 70000.0]:
        assert e.dbscan(eps, 2) == O.dbscan(ref, eps, 2), eps
    e.close()


@pytest.mark.parametrize("threshold_path", [0, 1, 2, 3, 4, 5, 6])
def test_many_sets_in_one_upload_match_one_by_one(threshold_path):
    """Independent sets scored in one pass: each set's matrix equals the oracle's
    for that set alone (no pair across sets), and per-set neighbourhoods and
    DBSCAN equal the single-set results.  Sizes include empty and one-sequence
    sets and sets with 32-bit-path sequences only.  Every path of the threshold
    pass (the transposed two-pass one with 32-, 16- and 8-row blocks, global
    gather, bulk-copied rows with and without staged positions, one or two
    row buffers) gives the same bits."""
    rng = np.random.default_rng(31)
    mixed = _mixed_set(rng)
    pool, _ = W.config1()
    sets = [pool[:150], [], [pool[200]], mixed[:20], [b"", b"N" * 3, b"ACGT" * 300], pool[300:301] * 5,
            mixed, pool[400:1000], [pool[1100], pool[1101]]]
    e = swgpu.Engine(threshold_path=threshold_path)
    e.upload_sets(sets)
    assert e.set_count() == len(sets)
    e.score_all_pairs()
    with pytest.raises(swgpu.SwgpuError):
        e.distances()
    with pytest.raises(swgpu.SwgpuError):
        e.dbscan(100.0, 5)
    for k, st in enumerate(sets):
        D = e.distances(set=k)
        ref = O.all_pairs(st) if st else np.zeros((0, 0), dtype=np.uint32)
        bad = np.argwhere(D != ref)
        assert len(bad) == 0, (k, [(int(i), int(j), int(D[i, j]), int(ref[i, j])) for i, j in bad[:5]])
        for eps, mp in [(130.0, 5), (600.0, 2), (-1.0, 3)]:
            assert e.dbscan(eps, mp, set=k) == O.dbscan(ref, 0.015 if eps == -1 else eps, mp), (k, eps)
        rp, cols = e.neighbors(90.0, set=k)
        for i in range(len(st)):
            want = np.nonzero(ref[i].astype(np.float32) <= np.float32(90.0))[0]
            assert np.array_equal(cols[rp[i]:rp[i + 1]], want), (k, i)
    # many thresholds of many sets in one launch
    res = e.adaptive_sets(100.0, 37.0, 3, max_steps=12)
    for k, st in enumerate(sets):
        if len(st) >= 3 and len(set(st)) > 1:
            D = O.all_pairs(st)
            text, kept = O.adaptive(D, 100.0, 37.0, 3, max_steps=12, truncate=True)
            assert res[k]["log"] == text and res[k]["layers"] == kept, k
    e.close()


def test_aligned_sets_take_the_vector_threshold_pass():
    """Sets whose sizes are multiples of 8 (so every matrix row starts on a
    16-byte boundary) go through the vector pack kernel of the default
    threshold pass; its neighbour lists and DBSCAN runs equal those of the
    bulk-copy pass and the oracle's, one threshold and many per launch."""
    pool, _ = W.config1()
    rng = np.random.default_rng(12)
    sets = [pool[:64], pool[100:108], pool[200:400], pool[500:1500]]
    sets.append([pool[int(i)] for i in rng.integers(0, 2000, size=48)])
    runs = {}
    for path in (0, 4):
        e = swgpu.Engine(threshold_path=path)
        e.upload_sets(sets)
        e.score_all_pairs()
        out = []
        for k, st in enumerate(sets):
            for eps in (130.0, 260.0, 700.0):
                rp, cols = e.neighbors(eps, set=k)
                out.append((rp.tolist(), cols.tolist(), e.dbscan(eps, 5, set=k)))
        out.append([(r["log"], r["layers"]) for r in e.adaptive_sets(100.0, 60.0, 5, max_steps=12)])
        runs[path] = out
        e.close()
    assert runs[0] == runs[4]
    for k, st in enumerate(sets):
        D = O.all_pairs(st)
        for j, eps in enumerate((130.0, 260.0, 700.0)):
            assert runs[0][3 * k + j][2] == O.dbscan(D, eps, 5), (k, eps)


def test_adaptive_per_set_matches_single_set_runs(tmp_path):
    sets, _ = W.config5(n_sets=6, lo=50, hi=400)
    e = swgpu.Engine()
    e.upload_sets(sets)
    e.score_all_pairs()
    runs = [e.adaptive(150.0, 50.0, 5, set=k) for k in range(len(sets))]
    e.close()
    e1 = swgpu.Engine()
    for k, st in enumerate(sets):
        e1.upload(st)
        e1.score_all_pairs()
        assert e1.adaptive(150.0, 50.0, 5) == runs[k], k
    e1.close()


def _sweep_sets():
    sets, _ = W.config5(seed=15, n_sets=10, lo=30, hi=300)
    pool, _ = W.config1()
    rng = np.random.default_rng(8)
    sets.append(_mixed_set(rng)[:60])          # 32-bit-path sequences inside a set
    sets.append([pool[7]] * 12)                 # one cluster at every eps: the start search fails
    sets.append(pool[:3])                       # fewer points than minpts: never one cluster
    sets.append([pool[0]])
    return sets


@pytest.mark.parametrize("eps_start,eps_inc,minpts,max_steps", [(150.0, 50.0, 5, 0), (100.0, 60.0, 5, 12),
                                                                 (150.0, 50.0, 3, 2), (20.0, 35.0, 4, 5)])
def test_adaptive_sets_match_oracle(tmp_path, eps_start, eps_inc, minpts, max_steps):
    """All sets' sweeps advanced together (one threshold launch per round):
    each set's log text, kept layers and split-set files equal the oracle's
    sweep of that set alone; max_steps bounds the sweep (layers found so far
    are kept)."""
    sets = _sweep_sets()
    e = swgpu.Engine()
    e.upload_sets(sets)
    e.score_all_pairs()
    res = e.adaptive_sets(eps_start, eps_inc, minpts, max_steps=max_steps, prefix=str(tmp_path / "L"))
    st = e.stats()
    assert st["last_neighbor_launches"] >= 1
    singles = {}
    if max_steps == 0:  # the single-set call on the same upload
        for k in range(len(sets)):
            try:
                singles[k] = e.adaptive(eps_start, eps_inc, minpts, set=k)
            except swgpu.SwgpuError as err:
                singles[k] = err.status
    e.close()
    for k, st in enumerate(sets):
        r = res[k]
        D = O.all_pairs(st)
        if len(set(st)) == 1 and len(st) >= minpts:
            assert r["status"] == 9 and r["layers"] == [], k  # SWE_ERR_SWEEP
            assert r["log"].endswith("Error did not find a sufficient starting position in 20 tries \n")
            continue
        if len(st) < minpts and max_steps == 0:
            assert r["status"] == 9, k
            continue
        text, kept = O.adaptive(D, eps_start, eps_inc, minpts, max_steps=max_steps or 100000,
                                truncate=max_steps > 0)
        assert r["status"] == 0, (k, r["log"][-300:])
        assert r["log"] == text, k
        assert r["layers"] == kept, k
        for i, layer in enumerate(kept):
            assert (tmp_path / f"L{k}_{i:04d}").read_bytes() == O.split_set_bytes(layer), (k, i)
        if max_steps == 0:
            assert singles[k] == (text, kept), k
        else:
            assert r["steps"] <= max_steps


def _bitmap_instance(rng, n):
    """Eps-neighbour bitmap rows and counts of n random points on a line in
    a few families (ascending or shuffled order)."""
    x = rng.normal(0, 1, n)
    if rng.random() < 0.3:
        x = np.sort(x)
    x = x + rng.integers(0, int(rng.integers(1, 6)), n) * 3.0
    A = np.abs(x[:, None] - x[None, :]) <= rng.uniform(0.01, 0.6)
    wpr = (n + 63) // 64
    padded = np.zeros((n, wpr * 64), dtype=bool)
    padded[:, :n] = A
    words = np.packbits(padded.reshape(n, wpr, 64)[:, :, ::-1], axis=2).reshape(n, wpr * 8)
    words = np.ascontiguousarray(words).view(">u8").astype(np.uint64).reshape(n, wpr)
    return words, A.sum(axis=1).astype(np.int32)


def _host_bitmap_dbscan(words, counts, minpts):
    import ctypes as C
    s = swgpu.SplitSet()
    n, wpr = words.shape if len(counts) else (0, 0)
    w = np.ascontiguousarray(words, dtype=np.uint64)
    c = np.ascontiguousarray(counts, dtype=np.int32)
    assert swgpu.lib().swe_dbscan_bitmap(n, w.ctypes.data, max(wpr, 1), c.ctypes.data, minpts, C.byref(s)) == 0
    out = swgpu.split_set_to_lists(s)
    swgpu.lib().free_split_set_and_associated_clusters(s)
    return out


def test_device_bitmap_replays_equal_host_replay(eng):
    """Many DBSCAN instances on caller bitmaps in one device launch (one warp
    each) against the host replay of each: the same clusters, members in the
    same order.  Sizes 1-300 points (shared-memory state) plus one of 17,000
    (global scratch); minpts 0, 1, 3, 5, 10."""
    rng = np.random.default_rng(5)
    inst = [_bitmap_instance(rng, int(rng.integers(1, 300))) for _ in range(80)]
    inst.append(_bitmap_instance(rng, 17000))
    for minpts in (0, 1, 3, 5, 10):
        got = eng.dbscan_bitmaps_device(inst, minpts)
        for k, (words, counts) in enumerate(inst):
            assert got[k] == _host_bitmap_dbscan(words, counts, minpts), (k, len(counts), minpts)


@pytest.mark.parametrize("eps_start,eps_inc,minpts", [(300.0, 100.0, 5), (150.0, 50.0, 0), (60.0, 45.0, 2)])
def test_device_replays_equal_host_replays(tmp_path, eps_start, eps_inc, minpts):
    """The multi-set sweeps' DBSCAN runs replayed on the device (one launch
    per round, one warp per (set, eps) instance) and on host threads over the
    bitmaps copied back: the same status, steps, log text, kept layers and
    split-set files for every set, including one above 16,384 points (its
    traversal state in global scratch instead of shared memory) and the edge
    sets of the oracle sweep test."""
    sets, _ = W.config5(seed=21, n_sets=24, lo=50, hi=3000)
    big, _ = W.config2(seed=9, n=17000)
    sets = sets + [big] + _sweep_sets()
    out = {}
    for mode in (1, 2):
        e = swgpu.Engine(dbscan_replay=mode)
        e.upload_sets(sets)
        e.score_all_pairs()
        out[mode] = e.adaptive_sets(eps_start, eps_inc, minpts, max_steps=12, prefix=str(tmp_path / f"m{mode}_"))
        e.close()
    for k in range(len(sets)):
        a, b = out[1][k], out[2][k]
        for key in ("status", "steps", "truncated", "log", "layers"):
            assert a[key] == b[key], (k, key)
    host_files = sorted(p.name[3:] for p in tmp_path.glob("m1_*"))
    assert host_files == sorted(p.name[3:] for p in tmp_path.glob("m2_*"))
    for name in host_files:
        assert (tmp_path / f"m1_{name}").read_bytes() == (tmp_path / f"m2_{name}").read_bytes(), name
    assert sum(len(r["layers"]) for r in out[2]) > 0


# ---------------------------------------------------------------------------
# neighbourhoods, DBSCAN, adaptive sweep
# ---------------------------------------------------------------------------
def test_neighbors_csr_matches_threshold(eng):
    seqs, _ = W.config1()
    seqs = seqs[:700]
    D = _matrix(eng, seqs)
    for eps in [130.0, 0.0, 0.5, 90.0, 129.99, 1e9, -0.5, float("nan"), -1.0]:
        rp, cols = eng.neighbors(eps)
        for i in range(0, 700, 37):
            want = np.nonzero(D[i].astype(np.float32) <= np.float32(eps))[0]
            assert np.array_equal(cols[rp[i]:rp[i + 1]], want), (eps, i)


def test_dbscan_matches_reference_small(eng):
    doc = load_golden("dbscan_small.json")
    seqs = [s.encode() for s in doc["seqs"]]
    _matrix(eng, seqs)
    for case in doc["cases"]:
        assert eng.dbscan(case["eps"], case["minpts"]) == case["clusters"], case["eps"]


def test_dbscan_config1_matches_oracle(eng):
    seqs, _ = W.config1()
    D = _matrix(eng, seqs)
    for eps, mp in [(130.0, 5), (250.0, 10), (700.0, 5), (60.0, 2)]:
        assert eng.dbscan(eps, mp) == O.dbscan(D, eps, mp), (eps, mp)


def test_adaptive_matches_reference_small(eng, tmp_path):
    doc = load_golden("adaptive_small.json")
    seqs = [s.encode() for s in doc["seqs"]]
    _matrix(eng, seqs)
    for k, run in enumerate(doc["runs"]):
        d = tmp_path / f"r{k}"
        d.mkdir()
        text, kept = eng.adaptive(run["eps_start"], run["eps_inc"], run["minpts"], prefix=str(d / "layer"))
        assert "Dataset read!\n" + text == run["stdout"]
        got = {p.name: base64.b64encode(p.read_bytes()).decode() for p in sorted(d.glob("layer*"))}
        assert got == run["files"]


def test_sweep_that_cannot_end_returns_error(eng):
    seqs, _ = W.config1()
    _matrix(eng, seqs[:5])  # 5 points, minpts 5: never one cluster
    with pytest.raises(swgpu.SwgpuError) as e:
        eng.adaptive(10.0, 50.0, 5)
    assert e.value.status == 9


def test_bounded_wait_timeout_is_reported_and_context_survives():
    seqs, _ = W.config1()
    seqs = seqs[:300]
    e = swgpu.Engine(inject_timeout=1)
    e.upload(seqs)
    with pytest.raises(swgpu.SwgpuError) as err:
        e.score_all_pairs()
    assert err.value.status == 5
    e.close()
    ok = swgpu.Engine()
    D = _matrix(ok, seqs)
    ok.close()
    assert np.array_equal(D, O.all_pairs(seqs))


def test_one_to_many_and_query_length_quirk(eng):
    rng = np.random.default_rng(9)
    seqs, _ = W.config1()
    db = seqs[:500] + [W.BASES[rng.integers(0, 4, size=900)].tobytes()]
    eng.upload(db)
    q = W._mutate(rng, np.frombuffer(db[7], dtype=np.uint8).copy(), 0.05, 0.01).tobytes()
    want = np.array([O.score(s, q) for s in db], dtype=np.uint32)
    assert np.array_equal(eng.one_to_many(q), want)
    want = np.array([O.score(s, q, len(s), 120) for s in db], dtype=np.uint32)
    assert np.array_equal(eng.one_to_many(q, 120), want)


# ---------------------------------------------------------------------------
# drop-in command-line tools against the reference tools
# ---------------------------------------------------------------------------
def _tool(name, args, cwd):
    r = subprocess.run([str(swgpu.BIN_DIR / name)] + [str(a) for a in args], cwd=cwd, capture_output=True,
                       timeout=1200)
    return r.returncode, r.stdout.decode("latin-1"), r.stderr.decode("latin-1")


def test_cluster_dbscan_tool_config1(tmp_path):
    seqs, _ = W.config1()
    g = load_golden("config1_golden.json")["dbscan"]
    W.write_fasta(tmp_path / "c1.fa", seqs)
    rc, out, err = _tool("cluster_dbscan_SW", ["c1.fa", g["eps"], g["minpts"], "c1"], tmp_path)
    assert rc == g["rc"] == 0, err
    assert out == g["stdout"]
    got = {p.name: hashlib.sha256(p.read_bytes()).hexdigest() for p in sorted(tmp_path.glob("c1-*"))}
    assert got == g["files_sha256"]


def test_adaptive_tool_config1(tmp_path):
    seqs, _ = W.config1()
    g = load_golden("config1_golden.json")["adaptive"]
    W.write_fasta(tmp_path / "c1.fa", seqs)
    rc, out, err = _tool("adaptive_clustering_SW", ["c1.fa", g["eps_start"], g["eps_inc"], g["minpts"], "lay", 1],
                         tmp_path)
    assert rc == g["rc"] == 0, err
    assert out == g["stdout"]
    got = {p.name: hashlib.sha256(p.read_bytes()).hexdigest() for p in sorted(tmp_path.glob("lay*"))}
    assert got == g["files_sha256"]


def test_cluster_tool_small(tmp_path):
    doc = load_golden("cluster_tool_small.json")
    W.write_fasta(tmp_path / "in.fa", [s.encode() for s in doc["seqs"]])
    rc, out, err = _tool("cluster_dbscan_SW", ["in.fa", doc["eps"], doc["minpts"], "cl"], tmp_path)
    assert rc == 0, err
    assert out == doc["stdout"]
    got = {p.name: base64.b64encode(p.read_bytes()).decode() for p in sorted(tmp_path.glob("cl-*"))}
    assert got == doc["files"]


def test_find_closest_tool(tmp_path):
    doc = load_golden("find_closest_small.json")
    W.write_fasta(tmp_path / "db.fa", [s.encode() for s in doc["db"]])
    W.write_fasta(tmp_path / "q.fa", [s.encode() for s in doc["queries"]])
    for run in doc["runs"]:
        rc, out, err = _tool("find_closest_sequence_SW", ["db.fa", "q.fa", run["idx"], 4, "o.fa"], tmp_path)
        assert rc == 0, err
        assert out == run["stdout"]
        assert (tmp_path / "o.fa").read_text() == run["out"]


def test_adaptive_tool_small(tmp_path):
    doc = load_golden("adaptive_small.json")
    W.write_fasta(tmp_path / "in.fa", [s.encode() for s in doc["seqs"]])
    for k, run in enumerate(doc["runs"]):
        d = tmp_path / f"r{k}"
        d.mkdir()
        rc, out, err = _tool("adaptive_clustering_SW", [tmp_path / "in.fa", run["eps_start"], run["eps_inc"],
                                                        run["minpts"], "layer", 1], d)
        assert rc == run["rc"], err
        assert out == run["stdout"]
        got = {p.name: base64.b64encode(p.read_bytes()).decode() for p in sorted(d.glob("layer*"))}
        assert got == run["files"]


def _ref_main(name):
    exe = O.REF_DIR / f"{name}_on_swgpu"
    if not exe.exists():
        pytest.skip("reference mains relinked on libswgpu were not built (make -C oracle ref-dropin)")
    return exe


def test_reference_mains_linked_on_libswgpu(tmp_path):
    """The reference's own cluster_dbscan_SW.c / adaptive_clustering.c /
    find_closest_sequence_SW.c, compiled with the reference headers and linked
    against libswgpu, reproduce the reference tools' outputs."""
    seqs, _ = W.config1()
    W.write_fasta(tmp_path / "c1.fa", seqs)
    g = load_golden("config1_golden.json")
    r = subprocess.run([str(_ref_main("cluster_dbscan_SW")), "c1.fa", "130", "5", "c1"], cwd=tmp_path,
                       capture_output=True, timeout=1200)
    assert r.returncode == 0 and r.stdout.decode() == g["dbscan"]["stdout"]
    got = {p.name: hashlib.sha256(p.read_bytes()).hexdigest() for p in sorted(tmp_path.glob("c1-*"))}
    assert got == g["dbscan"]["files_sha256"]
    a = g["adaptive"]
    r = subprocess.run([str(_ref_main("adaptive_clustering_SW")), "c1.fa", str(a["eps_start"]), str(a["eps_inc"]),
                        str(a["minpts"]), "lay", "1"], cwd=tmp_path, capture_output=True, timeout=1200)
    assert r.returncode == 0 and r.stdout.decode() == a["stdout"]
    got = {p.name: hashlib.sha256(p.read_bytes()).hexdigest() for p in sorted(tmp_path.glob("lay*"))}
    assert got == a["files_sha256"]
    doc = load_golden("find_closest_small.json")
    W.write_fasta(tmp_path / "db.fa", [s.encode() for s in doc["db"]])
    W.write_fasta(tmp_path / "q.fa", [s.encode() for s in doc["queries"]])
    for run in doc["runs"]:
        r = subprocess.run([str(_ref_main("find_closest_sequence_SW")), "db.fa", "q.fa", str(run["idx"]), "4",
                            "o.fa"], cwd=tmp_path, capture_output=True, timeout=600)
        assert r.returncode == 0 and r.stdout.decode() == run["stdout"]
        assert (tmp_path / "o.fa").read_text() == run["out"]


def test_score_callers_linked_on_libswgpu(tmp_path):
    """The reference's compareSW.c, silhouette.c, compare_norms.c and
    find_satellite.c (the other callers of score(): comparison.c, filter.c),
    linked against libswgpu, print byte for byte what the reference tools
    print (golden stdout, one thread)."""
    doc = load_golden("score_callers.json")
    W.write_fasta(tmp_path / "one.fa", [s.encode("latin-1") for s in doc["one"]])
    W.write_fasta(tmp_path / "two.fa", [s.encode("latin-1") for s in doc["two"]])
    W.write_fasta(tmp_path / "target.fa", [doc["target"].encode("latin-1")])
    (tmp_path / "proj.txt").write_text(doc["proj"])
    for run in doc["runs"]:
        r = subprocess.run([str(_ref_main(run["tool"]))] + run["args"], cwd=tmp_path, capture_output=True,
                           timeout=600)
        assert r.returncode == 0, (run["tool"], r.stderr.decode()[-500:])
        assert r.stdout.decode("latin-1") == run["stdout"], (run["tool"], run["args"])


def test_comparison_statistics_match_oracle(eng):
    """mean / sigma / silhouette / matrix through the C ABI against the same
    quantities computed from the oracle's distances (larger sets than the
    golden case, uneven sizes)."""
    import ctypes as C
    pool, _ = W.config2(n=900, seed=40)
    one, two = pool[:530], pool[530:]
    D = O.all_pairs(pool)
    cross = D[:530, 530:].astype(np.float64)
    L = swgpu.lib()
    for name in ("mean_from_smith_waterman_datasets", "silhouette_from_smith_waterman_datasets"):
        getattr(L, name).restype = C.c_double
        getattr(L, name).argtypes = [swgpu.Dataset, swgpu.Dataset, C.c_size_t]
    L.sigma_from_smith_waterman_datasets.restype = C.c_double
    L.sigma_from_smith_waterman_datasets.argtypes = [C.c_double, swgpu.Dataset, swgpu.Dataset, C.c_size_t]
    L.smith_waterman_distances_matrix.restype = C.POINTER(C.c_ulong)
    L.smith_waterman_distances_matrix.argtypes = [swgpu.Dataset, swgpu.Dataset]
    b1, b2 = swgpu.SeqBuffer(one), swgpu.SeqBuffer(two)
    mean = L.mean_from_smith_waterman_datasets(b1.dataset(), b2.dataset(), 4)
    assert mean == cross.sum() / (530.0 * 370.0)
    sigma = L.sigma_from_smith_waterman_datasets(mean, b1.dataset(), b2.dataset(), 4)
    want = np.sqrt(np.floor((cross - mean) * (cross - mean)).sum()) / 900
    assert sigma == pytest.approx(want, rel=1e-12)
    sil = L.silhouette_from_smith_waterman_datasets(b1.dataset(), b2.dataset(), 4)
    a = D[:530, :530].sum(axis=1) / 529.0
    b = cross.sum(axis=1) / 370.0
    s = np.where(a < b, 1 - a / b, np.where(a > b, b / a - 1, 0.0))
    assert sil == pytest.approx(s.sum() / 530, rel=1e-12)
    m = L.smith_waterman_distances_matrix(b1.dataset(), b2.dataset())
    got = np.ctypeslib.as_array(m, shape=(530 * 370,)).reshape(530, 370).copy()
    swgpu.lib().swe_free(C.cast(m, C.c_void_p))
    assert np.array_equal(got, D[:530, 530:])


# ---------------------------------------------------------------------------
# size-independent properties at the full config-2 size
# ---------------------------------------------------------------------------
@pytest.mark.slow
def test_config2_full_properties_and_sampled_rows(eng):
    seqs, _ = W.config2()
    D = _matrix(eng, seqs)
    L = np.array([len(s) for s in seqs])
    assert np.array_equal(D, D.T)
    assert not D.diagonal().any()
    assert (D <= 4 * np.maximum(L[:, None], L[None, :])).all()
    rows = list(range(0, 20000, 1999))
    R = O.score_rows(seqs, rows)
    assert np.array_equal(D[rows], R)


@pytest.mark.gpu
def test_partitioned_tile_exchange_rebuilds_the_full_matrix():
    """The exchange sized to the result on one GPU: three tile groups scored
    one after the other (as three ranks would), each packing only its own
    tile rectangles; a context holding group 0's pass unpacks the other two
    payloads (in chunks that cut through tiles) and then holds the whole
    pass's matrix, with DBSCAN matching."""
    import torch
    import swgpu
    seqs, _ = W.config2(n=1500)
    seqs = list(seqs) + [b"ACGTRYNNNNACGT" * 3, b"", b"A" * 900]  # 32-bit path rows too
    eng = swgpu.Engine()
    eng.upload(seqs)
    eng.score_all_pairs()
    full = eng.distances()
    whole = eng.partition_bytes(0)
    payload = []
    for p in range(3):
        eng.set_partition(p, 3)
        eng.score_all_pairs()
        sizes = [eng.partition_bytes(q) for q in range(3)]
        buf = torch.empty(max(sizes[p], 16), dtype=torch.uint8, device="cuda:0")
        eng.partition_pack(buf.data_ptr())
        payload.append((sizes, buf))
    assert payload[0][0] == payload[1][0] == payload[2][0]
    assert sum(payload[0][0]) == whole  # the groups' tiles cover the layout once
    eng.set_partition(0, 3)
    eng.score_all_pairs()
    assert not np.array_equal(eng.distances(), full)
    chunk = 1 << 16
    for p in (1, 2):
        size = payload[p][0][p]
        for off in range(0, size, chunk):
            n = min(chunk, size - off)
            eng.partition_unpack(p, payload[p][1][off:off + n].data_ptr(), off, n)
    assert np.array_equal(eng.distances(), full)
    assert eng.dbscan(300.0, 5) == O.dbscan(full, 300.0, 5)
    with pytest.raises(swgpu.SwgpuError):
        eng.partition_unpack(1, payload[1][1].data_ptr(), 2, 3)  # not whole distances
    eng.close()


def test_partitioned_score_passes_combine_to_the_full_matrix():
    """Three tile groups scored one after the other on one GPU (as three ranks
    would), each leaving 0xFF bytes outside its tiles; their bytewise minimum,
    copied back into the engine, is the whole pass's matrix, and DBSCAN on it
    matches."""
    import torch
    import swgpu
    seqs, _ = W.config2(n=1500)
    seqs = list(seqs) + [b"ACGTRYNNNNACGT" * 3, b"", b"A" * 900]  # 32-bit path rows too
    eng = swgpu.Engine()
    eng.upload(seqs)
    eng.score_all_pairs()
    full = eng.distances()
    cells_full = eng.stats()["tile_cells"]
    nbytes = eng.distance_bytes()
    parts, cells = [], 0.0
    for p in range(3):
        eng.set_partition(p, 3)
        eng.score_all_pairs()
        cells += eng.stats()["tile_cells"]
        buf = torch.empty(nbytes, dtype=torch.uint8, device="cuda:0")
        eng.distance_copy(buf.data_ptr(), to_engine=False)
        parts.append(buf)
    assert cells == pytest.approx(cells_full)
    combined = torch.minimum(torch.minimum(parts[0], parts[1]), parts[2])
    eng.distance_copy(combined.data_ptr(), to_engine=True)
    assert np.array_equal(eng.distances(), full)
    assert eng.dbscan(300.0, 5) == O.dbscan(full, 300.0, 5)
    eng.set_partition(0, 1)
    eng.score_all_pairs()
    assert np.array_equal(eng.distances(), full)
    eng.close()
