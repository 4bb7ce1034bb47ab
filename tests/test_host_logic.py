"""Host logic of libswgpu.so that runs without a GPU: the C ABI's exports,
the FASTA loader, split-set and cluster-file formats, layer relations, the
order-faithful DBSCAN replay and the adaptive driver.  No kernel is launched
here; where distances are needed they come from the oracle."""
from __future__ import annotations

import base64
import ctypes as C
import json
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import oracle as O
import swgpu
from conftest import ROOT, gpu_available, load_golden


def _declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", text, flags=re.M):
            name = m.group(1)
            if m.group(0).startswith("typedef"):  # function-pointer types
                continue
            if name not in {"if", "while", "for", "return", "sizeof"}:
                names.add(name)
    return names


def test_library_exports_every_declared_symbol():
    L = swgpu.lib()
    declared = _declared_functions()
    assert set(swgpu.EXPORTS) <= declared | {"adaptive_dbscan"}
    for name in sorted(declared):
        assert hasattr(L, name), f"{name} declared in include/ but not exported"
    out = subprocess.run(["nm", "-D", "--defined-only", str(swgpu.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert declared <= exported


def test_cli_tools_built():
    for t in ("cluster_dbscan_SW", "adaptive_clustering_SW", "find_closest_sequence_SW", "fasta2kmer",
              "cluster_dbscan_kmerL1", "cluster_dbscan_kmerL2", "cluster_dbscan_pca", "adaptive_clustering_kmer_L1",
              "adaptive_clustering_kmer_L2", "adaptive_clustering_PCA", "split_sets_to_newick", "tree_pureness",
              "filter_split_sets_by_min", "split_set_to_fasta", "kmer2pca"):
        assert (swgpu.BIN_DIR / t).exists()


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_create_fails_loudly_without_gpu():
    with pytest.raises(swgpu.SwgpuError) as e:
        swgpu.Engine()
    assert e.value.status == 4  # SWE_ERR_NO_DEVICE


def _load_with_lib(path):
    L = swgpu.lib()
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    L.dataset_from_fasta.restype = swgpu.Dataset
    L.dataset_from_fasta.argtypes = [C.c_void_p]
    L.free_sequences_from_dataset.argtypes = [swgpu.Dataset]
    f = libc.fopen(str(path).encode(), b"r")
    ds = L.dataset_from_fasta(f)
    libc.fclose(f)
    out = [C.string_at(ds.sequences[k], ds.sequence_lengths[k]).decode("latin-1") for k in range(ds.n_values)]
    mx = ds.max_sequence_length
    L.free_sequences_from_dataset(ds)
    return out, mx


def test_fasta_loader_matches_reference(tmp_path):
    cases = load_golden("fasta_cases.json")
    for name, case in cases.items():
        p = tmp_path / f"{name}.fa"
        p.write_bytes(case["text"].encode("latin-1"))
        got, mx = _load_with_lib(p)
        assert got == case["expected"], name
        assert mx == max((len(s) for s in got), default=0)


def _make_split_set(clusters):
    arr = (swgpu.Cluster * max(1, len(clusters)))()
    keep = []
    for i, cl in enumerate(clusters):
        m = (C.c_int * max(1, len(cl)))(*cl)
        keep.append(m)
        arr[i] = swgpu.Cluster(C.cast(m, C.POINTER(C.c_int)), len(cl), i)
    return swgpu.SplitSet(len(clusters), C.cast(arr, C.POINTER(swgpu.Cluster))), (arr, keep)


def test_split_set_bytes_and_roundtrip(tmp_path):
    rng = np.random.default_rng(3)
    clusters = [sorted(rng.choice(500, size=int(rng.integers(1, 40)), replace=False).tolist())
                for _ in range(7)]
    s, _keep = _make_split_set(clusters)
    p = tmp_path / "ss"
    swgpu.lib().store_split_set(str(p).encode(), s)
    assert p.read_bytes() == O.split_set_bytes(clusters)
    back = swgpu.lib().read_split_set(str(p).encode())
    assert swgpu.split_set_to_lists(back) == clusters
    swgpu.lib().free_split_set_and_associated_clusters(back)


def test_store_split_set_keeps_tail_like_reference(tmp_path):
    # cluster_io.c:644-645 opens without O_TRUNC
    p = tmp_path / "ss"
    p.write_bytes(b"X" * 200)
    s, _keep = _make_split_set([[1, 2, 3]])
    swgpu.lib().store_split_set(str(p).encode(), s)
    body = O.split_set_bytes([[1, 2, 3]])
    assert p.read_bytes() == body + b"X" * (200 - len(body))


def test_relation_sorts_in_place_like_reference():
    L = swgpu.lib()

    class Conn(C.Structure):
        _fields_ = [("connections", C.POINTER(C.c_int)), ("n_connections", C.c_int)]

    L.generate_split_set_relation.restype = C.POINTER(Conn)
    L.generate_split_set_relation.argtypes = [swgpu.SplitSet, swgpu.SplitSet]
    rng = np.random.default_rng(5)
    for trial in range(20):
        n = 300
        perm = rng.permutation(n).tolist()
        cuts = sorted(rng.choice(np.arange(1, n), size=5, replace=False).tolist())
        anc = [perm[a:b] for a, b in zip([0] + cuts, cuts + [n])]
        perm2 = rng.permutation(n).tolist()
        cuts2 = sorted(rng.choice(np.arange(1, n), size=3, replace=False).tolist())
        new = [perm2[a:b] for a, b in zip([0] + cuts2, cuts2 + [n])]
        # mix: some new clusters are unions of ancient ones
        new[0] = anc[0] + anc[1][: len(anc[1]) // 2]
        sa, ka = _make_split_set(anc)
        sn, kn = _make_split_set(new)
        conns = L.generate_split_set_relation(sa, sn)
        got = [[conns[i].connections[k] for k in range(conns[i].n_connections)] for i in range(len(new))]
        anc_py = [list(c) for c in anc]
        new_py = [list(c) for c in new]
        want = O.relation(anc_py, new_py)
        assert got == want
        # the in-place sorts are visible in the member arrays
        assert [list(ka[1][i][: len(anc[i])]) for i in range(len(anc))] == anc_py
        assert [list(kn[1][i][: len(new[i])]) for i in range(len(new))] == new_py


def test_relation_on_partitions_matches_pairwise_reference():
    """Partitions (every DBSCAN result) take the one-pass relation; connections
    and the in-place sorts must equal the reference's pairwise computation."""
    L = swgpu.lib()

    class Conn(C.Structure):
        _fields_ = [("connections", C.POINTER(C.c_int)), ("n_connections", C.c_int)]

    L.generate_split_set_relation.restype = C.POINTER(Conn)
    L.generate_split_set_relation.argtypes = [swgpu.SplitSet, swgpu.SplitSet]
    rng = np.random.default_rng(9)
    for trial in range(40):
        n = int(rng.integers(30, 900))

        def partition(k, cover):
            pts = rng.permutation(n)[: max(k, int(n * cover))]
            cuts = sorted(rng.choice(np.arange(1, len(pts)), size=k - 1, replace=False).tolist())
            return [pts[a:b].tolist() for a, b in zip([0] + cuts, cuts + [len(pts)])]

        anc = partition(int(rng.integers(1, 25)), rng.uniform(0.3, 1.0))
        if trial % 3 == 0:  # new layer = unions of ancient clusters plus strays
            new, cur = [], []
            for cl in anc:
                cur = cur + cl
                if rng.random() < 0.4:
                    new.append(cur)
                    cur = []
            if cur:
                new.append(cur)
        else:
            new = partition(int(rng.integers(1, 20)), rng.uniform(0.3, 1.0))
        sa, ka = _make_split_set(anc)
        sn, kn = _make_split_set(new)
        conns = L.generate_split_set_relation(sa, sn)
        got = [[conns[i].connections[k] for k in range(conns[i].n_connections)] for i in range(len(new))]
        anc_py = [list(c) for c in anc]
        new_py = [list(c) for c in new]
        assert got == O.relation(anc_py, new_py), trial
        assert [list(ka[1][i][: len(anc[i])]) for i in range(len(anc))] == anc_py, trial
        assert [list(kn[1][i][: len(new[i])]) for i in range(len(new))] == new_py, trial


def test_replay_matches_oracle_dbscan():
    doc = load_golden("dbscan_small.json")
    seqs = [s.encode() for s in doc["seqs"]]
    D = O.all_pairs(seqs)
    for case in doc["cases"]:
        eps = 0.015 if case["eps"] == -1 else case["eps"]
        got = swgpu.dbscan_from_matrix(D, eps, case["minpts"])
        assert got == case["clusters"], case


def test_replay_random_graphs():
    rng = np.random.default_rng(11)
    for trial in range(30):
        n = int(rng.integers(1, 400))
        pts = rng.normal(size=(n, 2)) * rng.uniform(0.5, 5)
        D = np.round(np.sqrt(((pts[:, None] - pts[None]) ** 2).sum(-1)) * 10).astype(np.uint32)
        eps = float(rng.uniform(0, 15))
        mp = int(rng.integers(0, 8))
        assert swgpu.dbscan_from_matrix(D, eps, mp) == O.dbscan(D, eps, mp), (trial, n, eps, mp)


def test_replay_rows_of_many_words():
    """Rows of more than 8 bitmap words (n > 512): the replay tests words in
    blocks of 8 before walking them; clusters spread over every block."""
    rng = np.random.default_rng(12)
    for n in (513, 777, 1600, 2100):
        centres = rng.normal(size=(int(rng.integers(3, 9)), 2)) * 20
        pts = centres[rng.integers(0, len(centres), size=n)] + rng.normal(size=(n, 2)) * 2
        D = np.round(np.sqrt(((pts[:, None] - pts[None]) ** 2).sum(-1)) * 10).astype(np.uint32)
        for eps, mp in ((15.0, 4), (40.0, 10), (4.0, 2)):
            assert swgpu.dbscan_from_matrix(D, eps, mp) == O.dbscan(D, eps, mp), (n, eps, mp)


@pytest.fixture(scope="module")
def host_driver(tmp_path_factory):
    exe = tmp_path_factory.mktemp("drv") / "adaptive_host_driver"
    subprocess.run(["gcc", "-O1", "-std=c11", "-I", str(ROOT / "include"),
                    str(ROOT / "tests/c/adaptive_host_driver.c"), "-o", str(exe),
                    "-L", str(swgpu.LIB_PATH.parent), "-lswgpu", f"-Wl,-rpath,{swgpu.LIB_PATH.parent}"],
                   check=True)
    return exe


def test_adaptive_driver_matches_reference(tmp_path, host_driver):
    """libswgpu's adaptive_dbscan driving a caller-supplied dbscanner (the
    function-pointer seam of dbscan.h:72-81) reproduces the reference's log and
    split-set files byte for byte."""
    from swgpu import workloads as W
    doc = load_golden("adaptive_small.json")
    seqs = [s.encode() for s in doc["seqs"]]
    D = O.all_pairs(seqs)
    W.write_fasta(tmp_path / "in.fa", seqs)
    O.write_dist_file(tmp_path / "d.swd", D)
    for k, run in enumerate(doc["runs"]):
        d = tmp_path / f"run{k}"
        d.mkdir()
        r = subprocess.run([str(host_driver), str(tmp_path / "in.fa"), str(tmp_path / "d.swd"),
                            repr(run["eps_start"]), repr(run["eps_inc"]), str(run["minpts"]), "layer"],
                           cwd=d, capture_output=True, timeout=600)
        assert r.returncode == 0, r.stderr.decode()[-2000:]
        assert r.stdout.decode("latin-1") == run["stdout"]
        got = {p.name: base64.b64encode(p.read_bytes()).decode() for p in sorted(d.glob("layer*"))}
        assert got == run["files"]


def test_cluster_files_match_reference(tmp_path):
    doc = load_golden("cluster_tool_small.json")
    seqs = [s.encode() for s in doc["seqs"]]
    D = O.all_pairs(seqs)
    cl = swgpu.dbscan_from_matrix(D, doc["eps"], doc["minpts"])
    s, _keep = _make_split_set(cl)
    buf = swgpu.SeqBuffer(seqs)
    L = swgpu.lib()
    L.create_cluster_files.argtypes = [C.c_char_p, swgpu.SplitSet, swgpu.Dataset]
    L.create_cluster_files(str(tmp_path / "cl").encode(), s, buf.dataset())
    got = {p.name: base64.b64encode(p.read_bytes()).decode() for p in sorted(tmp_path.glob("cl-*"))}
    assert got == doc["files"]


@pytest.mark.parametrize("speculate,batch", [(False, 1), (True, 1), (True, 3), (True, 8)])
def test_sweep_batches_and_speculation_match_reference(tmp_path, speculate, batch):
    """The sweep state machine the engine drives (rounds of `batch` eps values,
    and the starting eps evaluated together with the batch after it) over the
    oracle's matrix reproduces the reference's adaptive_clustering_SW log and
    split-set files for every golden run, halving starts included."""
    doc = load_golden("adaptive_small.json")
    seqs = [s.encode() for s in doc["seqs"]]
    D = O.all_pairs(seqs)
    for k, run in enumerate(doc["runs"]):
        prefix = str(tmp_path / f"s{int(speculate)}b{batch}r{k}_layer")
        text, kept = swgpu.adaptive_from_matrix(D, run["eps_start"], run["eps_inc"], run["minpts"],
                                                speculate=speculate, batch=batch, prefix=prefix)
        assert "Dataset read!\n" + text == run["stdout"], (k, speculate, batch)
        got = {p.name.split("_", 1)[1]: base64.b64encode(p.read_bytes()).decode()
               for p in sorted(tmp_path.glob(f"s{int(speculate)}b{batch}r{k}_layer*"))}
        assert got == run["files"], (k, speculate, batch)


def test_sweep_speculation_through_halving():
    # a start with one cluster: the speculative batch is discarded and the start halved
    rng = np.random.default_rng(4)
    pts = np.concatenate([rng.normal(c, 1.0, size=(40, 2)) for c in (0, 12, 30)])
    D = np.round(np.sqrt(((pts[:, None] - pts[None]) ** 2).sum(-1)) * 10).astype(np.uint32)
    for start in (400.0, 900.0):
        want = O.adaptive(D, start, 7.0, 4)
        for batch in (1, 5):
            got = swgpu.adaptive_from_matrix(D, start, 7.0, 4, speculate=True, batch=batch)
            assert got[0] == want[0] and got[1] == want[1], (start, batch)


def _load_kmer_file_with_lib(path):
    import os as _os
    L = swgpu.lib()

    class Shape(C.Structure):
        _fields_ = [("n_features", C.c_size_t), ("n_samples", C.c_size_t)]

    L.shape_from_kmer_file.restype = Shape
    L.shape_from_kmer_file.argtypes = [C.c_int]
    L.load_kmer_from_file_into_dataset.restype = swgpu.Dataset
    L.load_kmer_from_file_into_dataset.argtypes = [C.c_void_p, Shape]
    L.free_values_from_dataset.argtypes = [swgpu.Dataset]
    libc = C.CDLL(None)
    libc.fdopen.restype = C.c_void_p
    libc.fdopen.argtypes = [C.c_int, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    fd = _os.open(str(path), _os.O_RDONLY)
    shape = L.shape_from_kmer_file(fd)
    f = libc.fdopen(fd, b"r")
    ds = L.load_kmer_from_file_into_dataset(f, shape)
    libc.fclose(f)
    vals = C.cast(ds.values, C.POINTER(C.POINTER(C.c_float)))
    V = np.array([[vals[d][i] for i in range(ds.n_values)] for d in range(ds.n_dimensions)], dtype=np.float32)
    L.free_values_from_dataset(ds)
    return (shape.n_features, shape.n_samples), V


def test_kmer_file_loader_matches_reference_semantics(tmp_path):
    """shape_from_kmer_file + load_kmer_from_file_into_dataset (dataset.c:
    346-425) on the reference fasta2kmer's own tables, and on a 3 MB table
    with scattered whitespace and numbers in several notations (the threaded
    tokenizer's pieces): the same floats as the reference's fscanf stream."""
    doc = load_golden("points.json")
    for k, text in doc["kmer"].items():
        p = tmp_path / f"k{k}.tsv"
        p.write_text(text)
        shape, V = _load_kmer_file_with_lib(p)
        want = O.load_kmer_text(text)
        assert shape == (want.shape[0], want.shape[1]) and np.array_equal(V, want), k
    rng = np.random.default_rng(3)
    rows = []
    for i in range(3000):
        vals = rng.normal(0, 50, size=64)
        toks = [("%d" % int(v)) if j % 3 == 0 else ("%.6f" % v) if j % 3 == 1 else ("%.3e" % v)
                for j, v in enumerate(vals)]
        sep = ["\t" if rng.random() < 0.9 else " \t " for _ in toks]
        rows.append("sequence_%d\t" % i + "".join(t + s for t, s in zip(toks[:-1], sep)) + toks[-1] + "\n")
    text = "".join(rows)
    p = tmp_path / "big.tsv"
    p.write_text(text)
    shape, V = _load_kmer_file_with_lib(p)
    want = O.load_kmer_text(text)
    assert shape == (want.shape[0], want.shape[1])
    assert np.array_equal(V, want)
    # integer tokens take a shortcut: the same float bits, signed zero included
    text = "a\t-0\t+5\t1234567\t16777217\t-007\nb\t0\t-1\t9999999\t12345678\t3\n"
    p.write_text(text)
    _, V = _load_kmer_file_with_lib(p)
    assert np.array_equal(V.view(np.uint32), O.load_kmer_text(text).view(np.uint32))


def _linkage_reference(n, pairs, cap):
    """Union-find with path halving, root = the group's smallest index: the
    grouping rule of the prefiltered pass written out directly."""
    parent = list(range(n))
    size = [1] * n

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in pairs:
        x, y = find(int(a)), find(int(b))
        if x == y or size[x] + size[y] > cap:
            continue
        if x > y:
            x, y = y, x
        parent[y] = x
        size[x] += size[y]
    return np.array([find(i) for i in range(n)], dtype=np.int32)


@pytest.mark.parametrize("cap", [1, 2, 3, 7, 128, 100000])
def test_capped_linkage_matches_union_find(cap):
    """The prefiltered layout's grouping (relabelling form) against a plain
    union-find: random pairs, pairs within planted families in a random
    order, repeated and self pairs."""
    rng = np.random.default_rng(cap)
    for n, m, fam in [(1, 3, 1), (50, 400, 5), (2000, 30000, 40), (3000, 60000, 300)]:
        a = rng.integers(0, n, size=m)
        b = rng.integers(0, n, size=m)
        owner = rng.integers(0, fam, size=n)
        same = [(i, j) for i, j in zip(rng.integers(0, n, size=4 * m), rng.integers(0, n, size=4 * m))
                if owner[i] == owner[j]][:m]
        for pairs in (np.stack([a, b], 1), np.array(same, dtype=np.int64).reshape(-1, 2),
                      np.concatenate([np.stack([a, a], 1)[:10], np.stack([a, b], 1), np.stack([b, a], 1)])):
            got = swgpu.capped_linkage(n, pairs, cap)
            want = _linkage_reference(n, pairs, cap)
            assert np.array_equal(got, want), (n, m, cap)
            sizes = np.bincount(got, minlength=n)
            assert sizes.max() <= max(cap, 1)


def test_tile_cost_order_is_a_stable_descending_sort():
    """The score pass's tile order (radix sort of integer costs) equals a
    stable sort by descending cost, ties in index order; non-integral costs
    take the comparison sort."""
    rng = np.random.default_rng(3)
    cases = [np.zeros(0), np.array([5.0]), np.full(1000, 7.0),
             rng.integers(0, 4, size=5000).astype(np.float64),  # many ties
             (rng.integers(1, 3, size=200000) * rng.integers(8, 25, size=200000) *
              rng.integers(4000, 12000, size=200000) * 16.0),  # tile-like products
             rng.integers(0, 2**52, size=3000).astype(np.float64),  # wide keys: five passes
             rng.random(2000) * 1e6]  # not integral
    for c in cases:
        want = np.argsort(-c, kind="stable").astype(np.int32)
        got = swgpu.cost_order(c)
        assert np.array_equal(got, want), len(c)

