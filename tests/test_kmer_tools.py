"""fasta2kmer on the GPU (kmers.c:157-389): frequency tables and their text
against the oracle (itself pinned to the reference's fasta2kmer output), the
reference's own fasta2kmer main() relinked on libswgpu.so, and every counting
and formatting path (shared-memory and global tables, 16-bit carry rows,
batches, rows split into several text segments)."""
from __future__ import annotations

import hashlib
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import swgpu
from conftest import fasta2kmer_input, load_golden
from swgpu import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = swgpu.Engine()
    yield e
    e.close()


@pytest.fixture(scope="module")
def small_batches():
    # 64 KB device batches: many count batches, one text segment per batch
    e = swgpu.Engine(kmer_batch_kb=64)
    yield e
    e.close()


def _loaded(doc, name, tmp_path):
    p = tmp_path / f"{name}.fa"
    W.write_fasta(p, fasta2kmer_input(doc, name))
    return O.fasta_load(p)


def test_golden_inputs_match_oracle(eng, tmp_path):
    doc = load_golden("fasta2kmer.json")
    loaded = {}
    for run in doc["runs"]:
        name = run["input"]
        if name not in loaded:
            loaded[name] = _loaded(doc, name, tmp_path)
        want = O.kmer_table(loaded[name], run["k"], bool(run["protein"]))
        got = eng.kmer_counts(loaded[name], run["k"], bool(run["protein"]))
        assert np.array_equal(got, want), run
        text = eng.kmer_tsv(got)
        assert len(text) == run["bytes"] and hashlib.sha256(text).hexdigest() == run["sha256"], run


def _random_reads(seed, n, lo, hi, alphabet=b"ACGT", junk=b"NRYX"):
    rng = np.random.default_rng(seed)
    a = np.frombuffer(alphabet, dtype=np.uint8)
    out = []
    for _ in range(n):
        L = int(rng.integers(lo, hi + 1))
        s = a[rng.integers(0, len(a), size=L)]
        for q in rng.integers(0, max(L, 1), size=int(rng.poisson(L / 200))):
            s[q] = junk[int(rng.integers(0, len(junk)))]
        out.append(s.tobytes())
    return out


@pytest.mark.parametrize("k,protein", [(5, False), (7, False), (8, False), (9, False), (3, True), (4, True)])
def test_random_reads_match_oracle(eng, small_batches, k, protein):
    alpha = b"ACDEFGHIKLMNPQRSTVWY" if protein else b"ACGT"
    n = 300 if k < 9 else 60
    seqs = _random_reads(100 + k, n, 0, 700, alpha)
    want = O.kmer_table(seqs, k, protein)
    assert np.array_equal(eng.kmer_counts(seqs, k, protein), want)
    assert np.array_equal(small_batches.kmer_counts(seqs, k, protein), want)


def test_long_sequences_keep_the_short_wrap(eng, small_batches):
    # >= 65536 windows go through 32-bit counters; the table keeps the low 16
    # bits, as the reference's short does
    seqs = [b"A" * 66000, b"ACGT" * 17000, b"C" * 33000, b"ACGTN" * 3, b"G" * 65537, b"G" * 65536]
    for k, protein in [(1, False), (2, False), (5, False), (9, False), (1, True), (2, True), (5, True)]:
        want = O.kmer_table(seqs, k, protein)
        assert np.array_equal(eng.kmer_counts(seqs, k, protein), want), (k, protein)
        assert np.array_equal(small_batches.kmer_counts(seqs, k, protein), want), (k, protein)
    t = eng.kmer_counts([b"A" * 66000], 1)
    assert t[0, 0] == 65999 - 65536


@pytest.mark.parametrize("nk", [1, 4, 20, 400, 1024, 65536, 70001])
def test_tsv_matches_oracle(eng, small_batches, nk):
    rng = np.random.default_rng(nk)
    n = max(1, min(40, 400000 // nk))
    t = rng.integers(-32768, 32768, size=(n, nk)).astype(np.int16)
    t[:, 0] = 0
    t.flat[rng.integers(0, t.size, size=min(t.size, 50))] = -32768
    t.flat[rng.integers(0, t.size, size=min(t.size, 50))] = 32767
    want = O.kmer_tsv(t)
    assert eng.kmer_tsv(t) == want
    assert small_batches.kmer_tsv(t) == want


def test_empty_and_invalid(eng):
    assert eng.kmer_counts([], 5).shape == (0, 1024)
    assert eng.kmer_tsv(np.zeros((0, 16), dtype=np.int16)) == b""
    assert np.array_equal(eng.kmer_counts([b"", b"A", b"ACGTA"], 5), np.zeros((3, 1024), dtype=np.int16))
    for k, protein in [(0, False), (16, False), (8, True)]:
        with pytest.raises(swgpu.SwgpuError):
            eng.kmer_counts([b"ACGT"], k, protein)


@pytest.mark.parametrize("build", ["reference_main", "cli"])
def test_fasta2kmer_main_relinked_on_libswgpu(tmp_path, build):
    """The reference's own fasta2kmer.c main() linked against libswgpu.so, and
    this package's fasta2kmer CLI, print the reference's stdout byte for
    byte."""
    exe = O.REF_DIR / "fasta2kmer_on_swgpu" if build == "reference_main" else swgpu.BIN_DIR / "fasta2kmer"
    if not exe.exists():
        pytest.skip("drop-in build not present")
    doc = load_golden("fasta2kmer.json")
    for name in doc["inputs"]:
        W.write_fasta(tmp_path / f"{name}.fa", fasta2kmer_input(doc, name))
    env = dict(os.environ)
    for run in doc["runs"]:
        r = subprocess.run([str(exe), f"{run['input']}.fa", str(run["k"]), "4", str(run["protein"])],
                           cwd=tmp_path, env=env, capture_output=True, timeout=600)
        assert r.returncode == 0, r.stderr[-400:]
        assert len(r.stdout) == run["bytes"] and hashlib.sha256(r.stdout).hexdigest() == run["sha256"], run


def test_dropin_frequencies_and_text(tmp_path):
    """frequencies_from_dataset / write_kmer_base / free_kmer_frequencies
    through ctypes: the table rows and the file text equal the oracle's."""
    import ctypes as C
    L = swgpu.lib()
    seqs = _random_reads(7, 120, 1, 400)
    buf = swgpu.SeqBuffer(seqs)
    f = L.frequencies_from_dataset(buf.dataset(), 6, 8, 0)
    assert L.swgpu_last_dropin_status() == 0 and f.n_seq == len(seqs) and f.n_kmers == 4096
    want = O.kmer_table(seqs, 6)
    got = np.array([np.ctypeslib.as_array(f.frequencies[i], shape=(4096,)) for i in range(len(seqs))])
    assert np.array_equal(got, want)
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    path = tmp_path / "out.tsv"
    fp = libc.fopen(str(path).encode(), b"w")
    L.write_kmer_base(fp, f)
    libc.fclose(fp)
    assert path.read_bytes() == O.kmer_tsv(want)
    L.free_kmer_frequencies(f)
    bad = L.frequencies_from_dataset(buf.dataset(), 0, 1, 0)
    assert not bad.frequencies and bad.n_seq == 0 and L.swgpu_last_dropin_status() != 0
