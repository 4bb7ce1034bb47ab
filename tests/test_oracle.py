"""The oracle (oracle/sw_oracle.c + oracle/oracle.py) pinned against golden
vectors that the reference itself produced (tests/golden/make_golden.py)."""
from __future__ import annotations

import base64
import hashlib
import tempfile
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from conftest import load_golden


def test_score_kats():
    # smith-waterman.c quirks: first base ignored, terminator counts, N == N
    assert O.score(b"ACGT", b"ACGT") == 0
    assert O.score(b"ACGT", b"TCGT") == 0
    assert O.score(b"ACGT", b"ACGA") == 8
    assert O.score(b"ACGT", b"GGGG") == 11
    assert O.score(b"NNNN", b"NNNN") == 0
    assert O.score(b"ACGTACGTAC", b"ACGTAC") == 16 == O.score(b"ACGTAC", b"ACGTACGTAC")


def test_score_golden_pairs():
    pairs = load_golden("score_pairs.json.gz")
    bad = [(a, b, la, lb, d) for a, b, la, lb, d in pairs
           if O.score(a.encode("latin-1"), b.encode("latin-1"), la, lb) != d]
    assert not bad, bad[:3]


def test_fasta_golden(tmp_path):
    cases = load_golden("fasta_cases.json")
    for name, case in cases.items():
        p = tmp_path / f"{name}.fa"
        p.write_bytes(case["text"].encode("latin-1"))
        got = [s.decode("latin-1") for s in O.fasta_load(p)]
        assert got == case["expected"], name


def _small_matrix(doc):
    seqs = [s.encode() for s in doc["seqs"]]
    return seqs, O.all_pairs(seqs)


def test_dbscan_golden():
    doc = load_golden("dbscan_small.json")
    seqs, D = _small_matrix(doc)
    assert hashlib.sha256(D.astype("<u2").tobytes()).hexdigest() == doc["dist_sha256"]
    for case in doc["cases"]:
        assert O.dbscan(D, case["eps"], case["minpts"]) == case["clusters"], case["eps"]


def test_adaptive_golden():
    doc = load_golden("adaptive_small.json")
    seqs, D = _small_matrix(doc)
    for run in doc["runs"]:
        text, kept = O.adaptive(D, run["eps_start"], run["eps_inc"], run["minpts"])
        assert "Dataset read!\n" + text == run["stdout"]
        files = {f"layer{i:04d}": O.split_set_bytes(s) for i, s in enumerate(kept)}
        assert set(files) == set(run["files"])
        for k, v in files.items():
            assert v == base64.b64decode(run["files"][k]), k


def test_cluster_tool_golden():
    doc = load_golden("cluster_tool_small.json")
    seqs, D = _small_matrix(doc)
    cl = O.dbscan(D, doc["eps"], doc["minpts"])
    assert doc["stdout"] == "%u clusters obtained \n" % len(cl)
    for i, c in enumerate(cl):
        assert base64.b64decode(doc["files"][f"cl-{i:03d}"]).decode() == O.cluster_fasta_text(c, seqs)


def test_find_closest_golden():
    doc = load_golden("find_closest_small.json")
    db = [s.encode() for s in doc["db"]]
    qs = [s.encode() for s in doc["queries"]]
    for run in doc["runs"]:
        d, i = O.find_closest(db, qs, run["idx"])
        assert run["stdout"] == "Smith Waterman distance = %i \n" % d
        assert run["out"] == O.cluster_fasta_text([i], db)


def test_config_generators_are_seeded():
    from swgpu import workloads as W
    a, _ = W.config1()
    b, _ = W.config1()
    assert a == b and len(a) == 2000
    g = load_golden("config1_golden.json")
    assert g["n"] == 2000 and g["cells"] == W.cells(a)


@pytest.mark.slow
def test_config1_rows_match_reference_golden():
    """Sampled rows of the oracle's config-1 matrix against the reference's row CRCs."""
    import zlib
    from swgpu import workloads as W
    seqs, _ = W.config1()
    g = load_golden("config1_golden.json")
    rows = list(range(0, 2000, 97))
    R = O.score_rows(seqs, rows).astype("<u2")
    for k, r in enumerate(rows):
        assert zlib.crc32(R[k].tobytes()) == g["row_crc32"][r], r


def test_score_substitution_forms_match_reference_tool(tmp_path):
    """The score-substitution build of cluster_dbscan_SW (oracle/score_subst.c)
    answers score() from a file.  Given the distances of 200 config-1 reads,
    as a matrix ("SWD1") and as the neighbour bits of the one eps ("SWB1"), it
    prints and writes byte for byte what the real reference tool does."""
    if not (O.REF_DIR / "cluster_dbscan_SW_subst").exists():
        pytest.skip("reference build (oracle/_ref) not present")
    from swgpu import workloads as W
    seqs, _ = W.config1()
    seqs = seqs[::10][:200]
    D = O.all_pairs(seqs)
    eps, minpts = 200.0, 5
    runs = {}
    for name in ("real", "matrix", "bits"):
        d = tmp_path / name
        d.mkdir()
        W.write_fasta(d / "r.fa", seqs)
        env = None
        if name == "matrix":
            O.write_dist_file(d / "d.bin", D)
            env = {"SWGPU_SUBST_DIST": str(d / "d.bin")}
        elif name == "bits":
            n = O.write_neighbor_bitmap_file(d / "d.bin", len(seqs), [(0, D)], eps)
            assert n == int((D <= eps).sum())
            env = {"SWGPU_SUBST_DIST": str(d / "d.bin")}
        tool = "cluster_dbscan_SW" if name == "real" else "cluster_dbscan_SW_subst"
        p = O.run_ref_tool(tool, ["r.fa", eps, minpts, "c"], d, env)
        assert p.returncode == 0, p.stderr
        files = {f.name: f.read_bytes() for f in sorted(d.glob("c-*"))}
        runs[name] = (p.stdout, files)
    assert runs["real"][0].startswith(b"16 clusters")
    assert runs["matrix"] == runs["real"]
    assert runs["bits"] == runs["real"]


def test_kmer_table_oracle_matches_reference_fasta2kmer(tmp_path):
    """The oracle's frequency table + text (kmers.c:157-389) reproduces the
    reference fasta2kmer's stdout byte for byte (sha256) on every golden run:
    DNA k = 1..9, protein k = 1..4, each alphabet over the other's input, and
    repeats whose counts pass 32767 and 65535."""
    from conftest import fasta2kmer_input
    from swgpu import workloads as W
    doc = load_golden("fasta2kmer.json")
    loaded = {}
    for run in doc["runs"]:
        name = run["input"]
        if name not in loaded:
            p = tmp_path / f"{name}.fa"
            W.write_fasta(p, fasta2kmer_input(doc, name))
            loaded[name] = O.fasta_load(p)
        text = O.kmer_tsv(O.kmer_table(loaded[name], run["k"], bool(run["protein"])))
        assert len(text) == run["bytes"], run
        assert hashlib.sha256(text).hexdigest() == run["sha256"], run


def test_kmer_table_short_wrap():
    # counts live in a short (kmers.c:171): 65999 A's -> 463, 32999 C's -> -32537
    t = O.kmer_table([b"A" * 66000, b"C" * 33000], 1)
    assert t[0, 0] == 65999 - 65536 and t[1, 1] == 32999 - 65536
    assert O.kmer_table([b"ACGT"], 4).sum() == 0     # the window ending at the last symbol is skipped
    assert O.kmer_table([b"ACGTA"], 4)[0, 0b11100100] == 1
