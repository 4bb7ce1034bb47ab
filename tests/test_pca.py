"""kmer2pca (kmer2pca.c): the covariance matrix and the projections on the GPU,
the eigen-decomposition on the host, and the drop-in tool, against the oracle
and against the reference's own kmer2pca.c (built into oracle/_ref on the
LAPACK inside scipy's OpenBLAS, oracle/lapack_shim.c; its outputs on seeded
tables are the golden file kmer2pca.json).

Tolerances.  Eigenvectors are defined up to sign, so projections are compared
column by column up to sign.  The reference prints "%lf" (six decimals): its
files are compared with 1.5e-6 (a unit and a half in the last place).  The
integer route's covariance is compared bit for bit with the oracle's exact
evaluation; the float64 route's with 1e-12 of the matrix's largest entry.
The host eigen-solver is compared with numpy's LAPACK solver with 1e-12 of
the largest eigenvalue, its vectors with 1e-9 where eigenvalues are apart."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import swgpu
from conftest import load_golden

PRINT_TOL = 1.5e-6


def _columns_match_up_to_sign(a: np.ndarray, b: np.ndarray, tol: float) -> bool:
    a, b = np.atleast_2d(a), np.atleast_2d(b)
    if a.shape != b.shape:
        return False
    for i in range(a.shape[1]):
        if min(np.abs(a[:, i] - b[:, i]).max(), np.abs(a[:, i] + b[:, i]).max()) > tol:
            return False
    return True


def _proj(text: str, dims: int) -> np.ndarray:
    return np.array([float(t) for t in text.split()]).reshape(-1, dims)


# ---------------------------------------------------------------- CPU: oracle

def test_golden_reference_outputs_match_oracle():
    """The oracle's restatement (means over all samples, centred sums over the
    first n - n % 4 samples, numpy's eigen-solver, FMA projections) prints
    what the reference's kmer2pca printed, up to the last printed digit."""
    doc = load_golden("kmer2pca.json")
    for case in doc["cases"]:
        X = O.read_feature_table(case["table"])
        w, P = O.kmer2pca(X, case["dims"])
        ev = np.array([float(t) for t in case["ev"].split()])
        assert np.abs(w - ev).max() <= PRINT_TOL, case["name"]
        assert _columns_match_up_to_sign(P, _proj(case["proj"], case["dims"]), PRINT_TOL), case["name"]
        assert case["stdout"] == ("Read in data complete: shape: features %d samples %d\nMeans complete \n"
                                  "Covariance complete\nEigenspace obtained\n" % (X.shape[1], X.shape[0]))


def test_host_eigen_on_golden_tables():
    """The library's host solver (swe_pca_eigen) on the oracle's covariance of
    each golden table prints the reference's eigenvalue file and projections
    (through the oracle's FMA projection) to the last printed digit."""
    for case in load_golden("kmer2pca.json")["cases"]:
        X = O.read_feature_table(case["table"])
        w, V = swgpu.pca_eigen(O.pca_covariance(X), case["dims"])
        ev = np.array([float(t) for t in case["ev"].split()])
        assert np.abs(w - ev).max() <= PRINT_TOL, case["name"]
        P = O.pca_project(X, V)
        assert _columns_match_up_to_sign(P, _proj(case["proj"], case["dims"]), PRINT_TOL), case["name"]


def test_reference_skips_the_last_samples():
    """The reference's covariance leaves out the last n % 4 samples: with all
    samples summed the golden eigenvalues are not reproduced."""
    case = next(c for c in load_golden("kmer2pca.json")["cases"] if c["name"] == "k3_n203")
    X = O.read_feature_table(case["table"])
    ev = np.array([float(t) for t in case["ev"].split()])
    m = X.mean(0)
    full = np.linalg.eigvalsh((X - m).T @ (X - m) / len(X))
    assert np.abs(full - ev).max() > 1e-3
    assert np.abs(np.linalg.eigvalsh(O.pca_covariance(X)) - ev).max() <= PRINT_TOL


def test_reference_tool_matches_oracle_on_more_tables(tmp_path):
    """The reference's kmer2pca (oracle/_ref, run here on the host) against the
    oracle on tables the golden file does not hold: a protein 2-mer table
    (400 features), a DNA 5-mer table (1,024 features, 1,203 reads) and a
    table of negative and large counts with n % 4 == 2."""
    ref = O.REF_DIR / "kmer2pca"
    if not ref.exists():
        pytest.skip("reference kmer2pca not built")
    rng = np.random.default_rng(8)
    dna = np.frombuffer(b"ACGT", dtype=np.uint8)
    aa = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY", dtype=np.uint8)
    prot = [aa[rng.integers(0, 20, size=int(rng.integers(200, 600)))].tobytes() for _ in range(450)]
    reads = [dna[rng.integers(0, 4, size=int(rng.integers(80, 300)))].tobytes() for _ in range(1203)]
    wide = rng.integers(-3000, 30000, size=(130, 12))
    tables = [("protein_k2", O.kmer_tsv(O.kmer_table(prot, 2, True)).decode(), 6),
              ("dna_k5", O.kmer_tsv(O.kmer_table(reads, 5)).decode(), 7),
              ("wide_n130", "".join("r%d\t" % i + "\t".join(str(v) for v in row) + "\n"
                                     for i, row in enumerate(wide)), 4)]
    for name, text, dims in tables:
        (tmp_path / "in.tsv").write_text(text)
        r = subprocess.run([str(ref), "in.tsv", "p.txt", "e.txt", str(dims), "4"], cwd=tmp_path,
                           capture_output=True, timeout=600)
        assert r.returncode == 0, name
        X = O.read_feature_table(text)
        w, P = O.kmer2pca(X, dims)
        ev = np.array([float(t) for t in (tmp_path / "e.txt").read_text().split()])
        assert np.abs(w - ev).max() <= PRINT_TOL * max(1.0, np.abs(w).max() / 1e6), name
        tol = PRINT_TOL * max(1.0, np.abs(P).max() / 1e6)
        assert _columns_match_up_to_sign(P, _proj((tmp_path / "p.txt").read_text(), dims), tol), name


def test_exact_covariance_is_the_reference_sum():
    rng = np.random.default_rng(3)
    for n, nf in [(1, 3), (4, 2), (7, 5), (64, 9), (203, 16)]:
        X = rng.integers(-40, 300, size=(n, nf))
        a, b = O.pca_covariance_exact(X), O.pca_covariance(X.astype(float))
        assert np.abs(a - b).max() <= 1e-12 * max(1.0, np.abs(b).max()), (n, nf)


# ---------------------------------------------------------------- CPU: host code

@pytest.mark.parametrize("n,d", [(1, 1), (2, 2), (3, 3), (6, 6), (17, 7), (64, 10), (300, 7)])
def test_host_eigen_matches_numpy(n, d):
    rng = np.random.default_rng(n)
    X = rng.poisson(2.5, size=(max(3 * n, 40), n)).astype(float)
    cov = O.pca_covariance(X)
    w, V = swgpu.pca_eigen(cov, d)
    wr, Vr = O.pca_eigen(cov, d)
    scale = max(np.abs(wr).max(), 1e-300)
    assert np.abs(w - wr).max() <= 1e-12 * scale
    top = wr[::-1][:d + 1]
    for i in range(d):
        gap = min(abs(top[i] - top[i - 1]) if i > 0 else np.inf, abs(top[i] - top[i + 1]) if i + 1 < len(top) else np.inf)
        if gap > 1e-6 * scale:
            assert np.abs(V[i] - Vr[i]).max() <= 1e-9, (n, i)
    assert np.abs(V @ V.T - np.eye(d)).max() <= 1e-12
    assert np.abs(cov @ V.T - V.T * w[::-1][:d]).max() <= 1e-11 * scale


def test_host_eigen_rank_deficient_and_clustered():
    rng = np.random.default_rng(11)
    X = rng.poisson(1.0, size=(60, 120)).astype(float)
    X[:, :25] = 0
    X[:, 40] = X[:, 41]
    cov = O.pca_covariance(X)
    w, V = swgpu.pca_eigen(cov, 6)
    assert np.abs(w - np.linalg.eigvalsh(cov)).max() <= 1e-12 * np.abs(w).max()
    assert np.abs(cov @ V.T - V.T * w[::-1][:6]).max() <= 1e-11 * np.abs(w).max()
    # an eigenvalue of multiplicity 3 at the top: any orthonormal basis of its space
    Q, _ = np.linalg.qr(rng.normal(size=(30, 30)))
    lam = np.concatenate([np.linspace(0.1, 1.0, 27), [5.0, 5.0, 5.0]])
    A = (Q * lam) @ Q.T
    A = (A + A.T) / 2
    w, V = swgpu.pca_eigen(A, 4)
    assert np.abs(w - np.sort(lam)).max() <= 1e-12 * 5
    assert np.abs(V @ V.T - np.eye(4)).max() <= 1e-10
    assert np.abs(A @ V.T - V.T * np.array([5.0, 5.0, 5.0, 1.0])).max() <= 1e-10


def test_host_eigen_diagonal_matrices_follow_dsyev():
    """Diagonal matrices (the zero matrix of fewer than four samples among
    them) give unit vectors in the order dsyev's final selection sort leaves."""
    w, V = swgpu.pca_eigen(np.diag([3.0, 1.0, 2.0]), 3)
    assert list(w) == [1.0, 2.0, 3.0]
    assert np.array_equal(V, np.eye(3)[[0, 2, 1]])
    w, V = swgpu.pca_eigen(np.zeros((4, 4)), 4)
    assert list(w) == [0.0] * 4 and np.array_equal(V, np.eye(4)[::-1])
    w, V = swgpu.pca_eigen(np.diag([0.0, 0.0, -1.0]), 3)  # selection sort: -1 swapped to the front
    assert list(w) == [-1.0, 0.0, 0.0] and np.array_equal(V, np.eye(3)[[0, 1, 2]])


def test_host_eigen_rejects_bad_input():
    L = swgpu.lib()
    w = np.zeros(3)
    V = np.zeros((4, 3))
    A = np.eye(3)
    assert L.swe_pca_eigen(A.ctypes.data, 3, 4, w.ctypes.data, V.ctypes.data) != 0
    A[1, 1] = np.nan
    assert L.swe_pca_eigen(A.ctypes.data, 3, 1, w.ctypes.data, V.ctypes.data) != 0
    assert L.swe_pca_eigen(None, 0, 0, None, None) == 0


def _read_with_lib(tmp_path, text):
    p = tmp_path / "t.tsv"
    p.write_text(text)
    L = swgpu.lib()
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    L.shape_from_kmer_file.restype = swgpu.DataShape
    L.shape_from_kmer_file.argtypes = [C.c_int]
    L.swe_read_feature_table.restype = C.c_int
    L.swe_read_feature_table.argtypes = [C.c_void_p, swgpu.DataShape, C.c_void_p]
    fd = os.open(str(p), os.O_RDONLY)
    shape = L.shape_from_kmer_file(fd)
    os.close(fd)
    out = np.zeros((shape.n_samples, shape.n_features))
    fp = libc.fopen(str(p).encode(), b"r")
    st = L.swe_read_feature_table(fp, shape, out.ctypes.data)
    libc.fclose(fp)
    return st, out


def test_read_feature_table_matches_oracle(tmp_path):
    for case in load_golden("kmer2pca.json")["cases"]:
        st, X = _read_with_lib(tmp_path, case["table"])
        assert st == 0 and np.array_equal(X, O.read_feature_table(case["table"])), case["name"]
    text = "a\t-0\t+5\t007\nb 1e3 3.5 -12\nc\t-0.0\t123456789012345\t1234567890123456789\n"
    st, X = _read_with_lib(tmp_path, text)
    assert st == 0 and np.array_equal(X.view(np.uint64), O.read_feature_table(text).view(np.uint64))
    st, _ = _read_with_lib(tmp_path, "a\t1\t2\nb\t3\n")  # file ends early
    assert st != 0
    st, _ = _read_with_lib(tmp_path, "a\t1\t2\nb\t3\tx\n")  # not a number
    assert st != 0


# ---------------------------------------------------------------- GPU

@pytest.fixture(scope="module")
def eng():
    e = swgpu.Engine()
    yield e
    e.close()


def _kmer_tables():
    rng = np.random.default_rng(42)
    A = np.frombuffer(b"ACGT", dtype=np.uint8)

    def reads(n, lo, hi):
        return [A[rng.integers(0, 4, size=int(rng.integers(lo, hi + 1)))].tobytes() for _ in range(n)]

    yield "k3_n1", O.kmer_table(reads(1, 20, 40), 3)
    yield "k3_n3", O.kmer_table(reads(3, 20, 40), 3)
    yield "k2_n4", O.kmer_table(reads(4, 20, 40), 2)
    yield "k3_n5", O.kmer_table(reads(5, 60, 90), 3)
    yield "k3_n203", O.kmer_table(reads(203, 50, 400), 3)
    yield "k4_n1002", O.kmer_table(reads(1002, 50, 300), 4)
    yield "k5_n1501", O.kmer_table(reads(1501, 100, 300), 5)
    yield "wide_values", rng.integers(-32768, 32768, size=(301, 70)).astype(np.int16)
    yield "nf1", rng.integers(0, 50, size=(37, 1)).astype(np.int16)
    yield "nf65", rng.integers(0, 9, size=(4099, 65)).astype(np.int16)


@pytest.mark.gpu
def test_covariance_integer_tables_bit_exact(eng):
    for name, T in _kmer_tables():
        cov, info = eng.pca_covariance(T)
        assert info["exact"] == 1, name
        assert np.array_equal(cov, O.pca_covariance_exact(T)), name


@pytest.mark.gpu
def test_covariance_float_tables(eng):
    rng = np.random.default_rng(9)
    for n, nf in [(5, 3), (41, 6), (1000, 64), (2003, 130)]:
        X = rng.normal(size=(n, nf)) * rng.uniform(0.1, 10, size=nf) + rng.uniform(-5, 50, size=nf)
        cov, info = eng.pca_covariance(X)
        assert info["exact"] == 0
        want = O.pca_covariance(X)
        assert np.abs(cov - want).max() <= 1e-12 * np.abs(want).max(), (n, nf)
    X = rng.integers(0, 40000, size=(99, 7)).astype(float)  # integers outside int16: the float64 route
    cov, info = eng.pca_covariance(X)
    assert info["exact"] == 0
    want = O.pca_covariance(X)
    assert np.abs(cov - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.gpu
def test_projection_bit_exact(eng):
    rng = np.random.default_rng(5)
    for name, T in list(_kmer_tables())[3:8]:
        nf = T.shape[1]
        V = rng.normal(size=(min(7, nf), nf))
        V /= np.linalg.norm(V, axis=1, keepdims=True)
        want = O.pca_project(T.astype(float), V)
        assert np.array_equal(eng.pca_project(T, V), want), name
        eng.pca_covariance(T)
        assert np.array_equal(eng.pca_project(None, V), want), name
    X = rng.normal(size=(333, 19)) * 7.0
    V = rng.normal(size=(4, 19))
    assert np.array_equal(eng.pca_project(X, V), O.pca_project(X, V))


@pytest.mark.gpu
def test_pca_matches_oracle(eng):
    for name, T in _kmer_tables():
        nf = T.shape[1]
        d = min(nf, 5)
        w, P, info = eng.pca(T, d)
        wr, Vr = O.pca_eigen(O.pca_covariance_exact(T), d)
        scale = max(np.abs(wr).max(), 1.0)
        assert np.abs(w - wr).max() <= 1e-11 * scale, name
        top = np.sort(wr)[::-1]
        if len(T) >= 4 and all(top[i] - top[i + 1] > 1e-6 * scale for i in range(min(d, nf - 1))):
            Pr = O.pca_project(T.astype(float), Vr)
            assert _columns_match_up_to_sign(P, Pr, 1e-8 * max(1.0, np.abs(Pr).max())), name
        if len(T) < 4:  # zero covariance: dsyev's unit vectors, projections are raw columns
            assert np.array_equal(P, T[:, ::-1][:, :d].astype(float)), name
        assert info["ms_gram"] >= 0 and info["ms_project"] >= 0


@pytest.mark.gpu
def test_gpu_eigen_matches_host_eigen(eng):
    """swe_pca_eigen_gpu (reduction and bisection on the GPU) against the host
    solver and numpy: eigenvalues to 1e-12 of the largest, eigenvectors where
    eigenvalues are apart, eigen-residuals and orthonormality everywhere."""
    rng = np.random.default_rng(21)
    mats = []
    for n, rows in [(64, 300), (65, 40), (256, 97), (300, 2000), (1024, 3000)]:
        X = rng.poisson(1.5, size=(rows, n)).astype(float)
        X[:, : n // 10] = 0  # features that never occur: exact zero rows and columns
        mats.append(O.pca_covariance(X))
    Q, _ = np.linalg.qr(rng.normal(size=(80, 80)))
    lam = np.concatenate([np.linspace(0.1, 1.0, 77), [5.0, 5.0, 5.0]])
    mats.append((Q * lam) @ Q.T)
    mats[-1] = (mats[-1] + mats[-1].T) / 2
    mats.append(np.diag(rng.normal(size=70)))
    for A in mats:
        n = A.shape[0]
        d = min(7, n)
        w, V = eng.pca_eigen(A, d)
        wh, Vh = swgpu.pca_eigen(A, d)
        scale = np.abs(wh).max()
        assert np.abs(w - wh).max() <= 1e-12 * scale, n
        assert np.abs(w - np.linalg.eigvalsh(A)).max() <= 1e-12 * scale, n
        assert np.abs(V @ V.T - np.eye(d)).max() <= 1e-10, n
        assert np.abs(A @ V.T - V.T * w[::-1][:d]).max() <= 1e-10 * scale, n
        top = np.sort(wh)[::-1][:d + 1]
        for i in range(d):
            gaps = [abs(top[i] - top[j]) for j in (i - 1, i + 1) if 0 <= j < len(top)]
            if min(gaps) > 1e-6 * scale:
                assert np.abs(V[i] - Vh[i]).max() <= 1e-9, (n, i)


@pytest.mark.gpu
def test_pca_rejects_bad_arguments(eng):
    T = np.ones((8, 4), dtype=np.int16)
    for d in (0, 5):
        with pytest.raises(swgpu.SwgpuError):
            eng.pca(T, d)
    with pytest.raises(swgpu.SwgpuError):
        eng.pca(np.zeros((0, 4)), 1)
    eng.pca_covariance(T)
    with pytest.raises(swgpu.SwgpuError):  # resident table has 8 rows, not 9
        swgpu._check(swgpu.lib().swe_pca_project(eng.ctx, None, 9, 4, np.ones((1, 4)).ctypes.data, 1,
                                                 np.zeros(9).ctypes.data, None), eng.ctx)


@pytest.mark.gpu
@pytest.mark.parametrize("build", ["golden", "reference"])
def test_kmer2pca_tool_matches_reference(tmp_path, build):
    """bin/kmer2pca against the reference's kmer2pca outputs: the golden
    files, and a run of oracle/_ref/kmer2pca on the same input (a larger
    5-mer table)."""
    exe = swgpu.BIN_DIR / "kmer2pca"
    if build == "golden":
        cases = [(c["name"], c["table"], c["dims"], c["stdout"], c["ev"], c["proj"])
                 for c in load_golden("kmer2pca.json")["cases"]]
    else:
        ref = O.REF_DIR / "kmer2pca"
        if not ref.exists():
            pytest.skip("reference kmer2pca not built")
        rng = np.random.default_rng(77)
        A = np.frombuffer(b"ACGT", dtype=np.uint8)
        seqs = [A[rng.integers(0, 4, size=int(rng.integers(80, 300)))].tobytes() for _ in range(1203)]
        text = O.kmer_tsv(O.kmer_table(seqs, 5)).decode()
        (tmp_path / "in.tsv").write_text(text)
        r = subprocess.run([str(ref), "in.tsv", "p.txt", "e.txt", "7", "8"], cwd=tmp_path, capture_output=True,
                           timeout=900)
        assert r.returncode == 0
        cases = [("k5_n1203", text, 7, r.stdout.decode(), (tmp_path / "e.txt").read_text(),
                  (tmp_path / "p.txt").read_text())]
    for name, text, dims, stdout, ev, proj in cases:
        (tmp_path / "in.tsv").write_text(text)
        r = subprocess.run([str(exe), "in.tsv", "proj.txt", "ev.txt", str(dims), "4"], cwd=tmp_path,
                           capture_output=True, timeout=600)
        assert r.returncode == 0, r.stdout[-400:]
        assert r.stdout.decode() == stdout, name
        got_ev = np.array([float(t) for t in (tmp_path / "ev.txt").read_text().split()])
        want_ev = np.array([float(t) for t in ev.split()])
        assert np.abs(got_ev - want_ev).max() <= PRINT_TOL, name
        got = _proj((tmp_path / "proj.txt").read_text(), dims)
        assert _columns_match_up_to_sign(got, _proj(proj, dims), PRINT_TOL), name
        if name.endswith(("_n3", "_n1")):  # no sample in the sums: the same files byte for byte
            assert (tmp_path / "ev.txt").read_text() == ev and (tmp_path / "proj.txt").read_text() == proj


def test_kmer2pca_tool_rejects_bad_arguments_before_the_gpu(tmp_path):
    """The CLI's argument and file errors come before it opens the GPU: usage
    text for fewer than five arguments (the reference reads argv[5] with
    four), exit 1 for dimensions outside 1 .. n_features, a missing or
    unreadable table."""
    exe = swgpu.BIN_DIR / "kmer2pca"
    (tmp_path / "t.tsv").write_text("s0\t1\t2\t3\ns1\t4\t5\t6\n")
    (tmp_path / "bad.tsv").write_text("s0\t1\t2\t3\ns1\t4\tx\t6\n")
    runs = [["t.tsv", "p", "e", "2"], ["t.tsv", "p", "e", "0", "1"], ["t.tsv", "p", "e", "4", "1"],
            ["missing.tsv", "p", "e", "1", "1"], ["bad.tsv", "p", "e", "1", "1"]]
    for args in runs:
        r = subprocess.run([str(exe), *args], cwd=tmp_path, capture_output=True, timeout=60)
        assert r.returncode == 1, args
    r = subprocess.run([str(exe), "t.tsv"], cwd=tmp_path, capture_output=True, timeout=60)
    assert r.stdout.decode().startswith("Arguments are: \n [FILE-in ] kmer file to apply PCA on")
    assert not (tmp_path / "p").exists() and not (tmp_path / "e").exists()
