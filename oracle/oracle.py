"""ORACLE - test infrastructure only.

Python side of the CPU checkers for the all-pairs Smith-Waterman neighbourhood
engine.  Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline leg of
``bench.py`` import this module; the product library never does.

Two kinds of checker live here:

* ``liboracle.so`` - the plain-C restatement in ``sw_oracle.c`` (score,
  all-pairs, DBSCAN, FASTA loader, k-mer counts, point distances, kmer2pca's
  projections), wrapped with ctypes;
* the reference itself, compiled from its own sources into ``_ref/`` by
  ``make -C oracle ref`` (``libref.so`` and the reference command-line tools,
  plus ``*_subst`` builds whose score() reads a precomputed matrix, see
  ``score_subst.c``, and kmer2pca linked to scipy's OpenBLAS LAPACK through
  ``lapack_shim.c``).

The adaptive-eps driver and the split-set helpers are restated below in
Python (small inputs only); each cites the reference lines it follows.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
_lib = None
_ref = None


# --------------------------------------------------------------------------
# loading
# --------------------------------------------------------------------------

def reference_dir() -> str:
    """The reference's source tree: $MNHN_REFERENCE_DIR, else the default
    mount point /root/reference."""
    return os.environ.get("MNHN_REFERENCE_DIR") or "/root/reference"


def build(ref_src: str | None = None) -> None:
    """Compile liboracle.so (and the reference into _ref/ when its sources exist)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    src = ref_src or reference_dir()
    if os.path.isdir(src):
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={src}"], check=True)


def lib():
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        L = C.CDLL(str(path))
        L.orc_score.restype = C.c_uint
        L.orc_score.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t, C.c_size_t]
        L.orc_score_rows.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                                     C.c_void_p, C.c_int]
        L.orc_all_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        L.orc_dbscan.restype = C.c_int
        L.orc_dbscan.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_fasta_load.restype = C.c_int
        L.orc_fasta_load.argtypes = [C.c_char_p, C.POINTER(C.c_void_p),
                                     C.POINTER(C.c_void_p), C.POINTER(C.c_int)]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_kmer_counts.argtypes = [C.c_char_p, C.c_size_t, C.c_int, C.c_void_p]
        L.orc_kmer_frequencies.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p]
        L.orc_points_dist.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.orc_dbscan_points.restype = C.c_int
        L.orc_dbscan_points.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_int, C.c_int, C.c_void_p,
                                        C.c_void_p]
        L.orc_pca_project.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return (REF_DIR / "libref.so").exists()


class _Dataset(C.Structure):
    # field layout of the reference's dataset (dataset.h:27-35)
    _fields_ = [("sequences", C.POINTER(C.c_char_p)), ("sequence_lengths", C.POINTER(C.c_size_t)),
                ("binary_sequences", C.c_void_p), ("n_values", C.c_int),
                ("values", C.c_void_p), ("n_dimensions", C.c_int),
                ("max_sequence_length", C.c_size_t)]


def ref_lib():
    """The reference's own score()/dataset_from_fasta() compiled from its sources."""
    global _ref
    if _ref is None:
        R = C.CDLL(str(REF_DIR / "libref.so"))
        R.score.restype = C.c_uint
        R.score.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t, C.c_size_t, C.c_void_p]
        R.dataset_from_fasta.restype = _Dataset
        R.dataset_from_fasta.argtypes = [C.c_void_p]
        _ref = R
    return _ref


class _SeqArray:
    """Sequences kept alive as NUL-terminated buffers plus pointer/length arrays."""

    def __init__(self, seqs):
        self.bufs = [C.create_string_buffer(bytes(s), len(s) + 1) for s in seqs]
        self.ptrs = (C.c_void_p * max(1, len(seqs)))(*[C.addressof(b) for b in self.bufs])
        self.lens = (C.c_size_t * max(1, len(seqs)))(*[len(s) for s in seqs])
        self.n = len(seqs)


# --------------------------------------------------------------------------
# restatement (liboracle.so)
# --------------------------------------------------------------------------

def score(a: bytes, b: bytes, la: int | None = None, lb: int | None = None) -> int:
    """Distance of smith-waterman.c:16-80 (C restatement).  la/lb default to len()."""
    la = len(a) if la is None else la
    lb = len(b) if lb is None else lb
    ab = C.create_string_buffer(bytes(a), max(len(a), la) + 1)
    bb = C.create_string_buffer(bytes(b), max(len(b), lb) + 1)
    return lib().orc_score(ab, bb, la, lb)


def all_pairs(seqs, threads: int = 0) -> np.ndarray:
    """n x n distances, D[i][k] = score(seq[k], seq[i]) as region_query calls it."""
    sa = _SeqArray(seqs)
    out = np.zeros((sa.n, sa.n), dtype=np.uint32)
    lib().orc_all_pairs(sa.ptrs, sa.lens, sa.n, out.ctypes.data, threads or os.cpu_count())
    return out


def score_rows(seqs, rows, threads: int = 0) -> np.ndarray:
    sa = _SeqArray(seqs)
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    out = np.zeros((len(rows), sa.n), dtype=np.uint32)
    lib().orc_score_rows(sa.ptrs, sa.lens, sa.n, rows.ctypes.data, len(rows), out.ctypes.data,
                         threads or os.cpu_count())
    return out


def dbscan(D: np.ndarray, eps: float, minpts: int):
    """dbscan.c:950-1047 over a distance matrix; list of member lists in id order."""
    D = np.ascontiguousarray(D, dtype=np.uint32)
    n = D.shape[0]
    members = np.zeros(max(1, n), dtype=np.int32)
    sizes = np.zeros(max(1, n), dtype=np.int32)
    nc = lib().orc_dbscan(D.ctypes.data, n, C.c_float(eps), minpts, members.ctypes.data,
                          sizes.ctypes.data)
    out, pos = [], 0
    for c in range(nc):
        out.append(members[pos:pos + sizes[c]].tolist())
        pos += sizes[c]
    return out


def points_dist(values: np.ndarray, metric: int) -> np.ndarray:
    """dbscan_L1 (metric 1) / dbscan_L2 (metric 2) pair distances
    (dbscan.c:563-779) of points values[dim][point]: float32 n x n, row =
    query point."""
    V = np.ascontiguousarray(values, dtype=np.float32)
    dims, n = V.shape
    D = np.zeros((n, n), dtype=np.float32)
    lib().orc_points_dist(V.ctypes.data, dims, n, metric, D.ctypes.data)
    return D


_libc = None


def _strtof(tok: str) -> float:
    """C strtof (what fscanf "%f" stores for a number token)."""
    global _libc
    if _libc is None:
        _libc = C.CDLL(None)
        _libc.strtof.restype = C.c_float
        _libc.strtof.argtypes = [C.c_char_p, C.c_void_p]
    return _libc.strtof(tok.encode(), None)


def load_kmer_text(text: str) -> np.ndarray:
    """load_kmer_from_file_into_dataset over shape_from_kmer_file (dataset.c:
    346-425): n_features = tabs of the first line, n_samples = newlines from
    the end of the first line on; the token stream is a label then n_features
    numbers per sample.  Returns values[feature][sample] as float32."""
    first_nl = text.index("\n") if "\n" in text else len(text)
    nf = text[:first_nl].count("\t")
    ns = text[first_nl:].count("\n")
    toks = text.split()
    V = np.zeros((nf, ns), dtype=np.float32)
    for s in range(ns):
        for f in range(nf):
            V[f, s] = _strtof(toks[s * (nf + 1) + 1 + f])
    return V


def load_projection_text(text: str, dims: int, n: int) -> np.ndarray:
    """load_projections_from_file_into_dataset (dataset.c:427-469): n samples
    of `dims` numbers, values[dim][sample] as float32."""
    toks = text.split()
    V = np.zeros((dims, n), dtype=np.float32)
    for i in range(n):
        for j in range(dims):
            V[j, i] = _strtof(toks[i * dims + j])
    return V


def cluster_values_text(members, V: np.ndarray) -> str:
    """create_single_cluster_file_with_values (cluster_io.c:343-356)."""
    return "".join("\t".join("%f" % float(V[k, m]) for k in range(V.shape[0])) + "\n" for m in members)


def dbscan_points(D: np.ndarray, eps: float, minpts: int, metric: int):
    """dbscan_L1 / dbscan_L2 (dbscan.c:950-1047) over points_dist's matrix."""
    D = np.ascontiguousarray(D, dtype=np.float32)
    n = D.shape[0]
    members = np.zeros(max(1, n), dtype=np.int32)
    sizes = np.zeros(max(1, n), dtype=np.int32)
    nc = lib().orc_dbscan_points(D.ctypes.data, n, C.c_float(eps), minpts, metric, members.ctypes.data,
                                 sizes.ctypes.data)
    out, pos = [], 0
    for c in range(nc):
        out.append(members[pos:pos + sizes[c]].tolist())
        pos += sizes[c]
    return out


def fasta_load(path) -> list[bytes]:
    buf, lens, n = C.c_void_p(), C.c_void_p(), C.c_int()
    rc = lib().orc_fasta_load(str(path).encode(), C.byref(buf), C.byref(lens), C.byref(n))
    if rc != 0:
        raise ValueError(f"orc_fasta_load({path}) failed with {rc}")
    L = np.ctypeslib.as_array(C.cast(lens, C.POINTER(C.c_size_t)), shape=(max(1, n.value),))
    out, pos = [], 0
    for k in range(n.value):
        out.append(C.string_at(buf.value + pos, int(L[k])))
        pos += int(L[k]) + 1
    lib().orc_free(buf)
    lib().orc_free(lens)
    return out


def kmer_counts(seq: bytes, k: int) -> np.ndarray:
    out = np.zeros(4 ** k, dtype=np.int16)
    lib().orc_kmer_counts(bytes(seq), len(seq), k, out.ctypes.data)
    return out


def kmer_table(seqs, k: int, protein: bool = False) -> np.ndarray:
    """frequencies_from_dataset (kmers.c:292-371) over NUL-terminated
    sequences: one int16 row of 4^k (or 20^k) counts per sequence."""
    nk = (20 if protein else 4) ** k
    out = np.zeros((len(seqs), nk), dtype=np.int16)
    for i, s in enumerate(seqs):
        lib().orc_kmer_frequencies(bytes(s), k, int(bool(protein)), out[i].ctypes.data)
    return out


def kmer_tsv(table: np.ndarray) -> bytes:
    """write_kmer_base (kmers.c:373-385): "sequence_%i" then "%hi" counts,
    tab separated, one line per row."""
    lines = []
    for i, row in enumerate(np.asarray(table, dtype=np.int16)):
        lines.append("sequence_%d\t" % i + "\t".join(str(int(v)) for v in row) + "\n")
    return "".join(lines).encode()


# --------------------------------------------------------------------------
# kmer2pca (kmer2pca.c)
# --------------------------------------------------------------------------

def read_feature_table(text: str) -> np.ndarray:
    """shape_from_input_file + data_from_file (kmer2pca.c:43-89, 255-268):
    n_features = tabs of the first line, n_samples = newlines from the end of
    the first line on, then per sample a label and n_features numbers of the
    whitespace token stream ("%lf").  Returns (samples, features) float64."""
    first_nl = text.index("\n") if "\n" in text else len(text)
    nf = text[:first_nl].count("\t")
    ns = text[first_nl:].count("\n")
    toks = text.split()
    X = np.zeros((ns, nf))
    for s in range(ns):
        X[s] = [float(t) for t in toks[s * (nf + 1) + 1:(s + 1) * (nf + 1)]]
    return X


def pca_covariance(X: np.ndarray) -> np.ndarray:
    """means_from_data + feature_covariance_matrix (kmer2pca.c:466-481,
    337-463) in float64: means over all n samples; the centred products summed
    over the first n - n % 4 samples only (the AVX loop's scalar tail is
    guarded by `!n_samples%4`, which is 0 for n > 0); divided by n.  The sums
    run in numpy's order, the reference's are 4-lane Kahan sums: equal up to
    rounding."""
    X = np.asarray(X, dtype=np.float64)
    n = X.shape[0]
    m = X.sum(0) / n
    n4 = n - n % 4
    Xc = X[:n4] - m
    return Xc.T @ Xc / n


def pca_covariance_exact(table: np.ndarray) -> np.ndarray:
    """The quantity pca_covariance estimates, computed exactly for an integer
    table and rounded as the GPU's integer route does: with P = X4^T X4, T the
    column sums of X4 (X4 = the first n4 = n - n % 4 rows) and S those of X,
    C = float(n^2 P - n (S T^T + T S^T) + n4 S S^T) / n / n / n, the numerator
    an exact (Python) integer converted to the nearest double."""
    X = np.asarray(table, dtype=np.int64)
    n, nf = X.shape
    n4 = n - n % 4
    P = (X[:n4].T @ X[:n4]).astype(object)
    T = X[:n4].sum(0).astype(object)
    S = X.sum(0).astype(object)
    Q = n * n * P - n * (np.outer(S, T) + np.outer(T, S)) + n4 * np.outer(S, S)
    out = np.empty((nf, nf))
    for i in range(nf):
        for j in range(nf):
            out[i, j] = float(Q[i, j]) / n / n / n
    return out


def pca_eigen(cov: np.ndarray, n_vectors: int):
    """eigen_from_corr (kmer2pca.c:107-138): numpy's LAPACK symmetric solver
    in place of the reference's dsyev: every eigenvalue ascending, and the
    eigenvectors of the n_vectors largest as rows, largest first, each signed
    so that its largest-magnitude entry is positive."""
    w, V = np.linalg.eigh(np.asarray(cov, dtype=np.float64))
    vec = V[:, ::-1][:, :n_vectors].T.copy()
    for v in vec:
        if v[np.argmax(np.abs(v))] < 0:
            v *= -1
    return w, vec


def pca_project(X: np.ndarray, vectors: np.ndarray) -> np.ndarray:
    """obtain_projections (kmer2pca.c:141-168) through orc_pca_project: one
    fused multiply-add per feature, in order."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    V = np.ascontiguousarray(vectors, dtype=np.float64)
    n, nf = X.shape
    d = V.shape[0]
    P = np.zeros((n, d))
    lib().orc_pca_project(X.ctypes.data, n, nf, V.ctypes.data, d, P.ctypes.data)
    return P


def kmer2pca(X: np.ndarray, dimensions: int):
    """kmer2pca's computation after reading its file (kmer2pca.c:540-586):
    eigenvalues ascending and the (samples, dimensions) projections."""
    w, V = pca_eigen(pca_covariance(X), dimensions)
    return w, pca_project(X, V)


def kmer2pca_texts(eigenvalues, projections) -> tuple[str, str]:
    """print_eigenvalues / print_projections (kmer2pca.c:226-253): "%lf" per
    line, and "%lf" tab separated per sample."""
    ev = "".join("%f\n" % v for v in eigenvalues)
    pr = "".join("\t".join("%f" % v for v in row) + "\n" for row in np.asarray(projections))
    return ev, pr


# --------------------------------------------------------------------------
# the reference itself (oracle/_ref)
# --------------------------------------------------------------------------

def ref_score(a: bytes, b: bytes, la: int | None = None, lb: int | None = None) -> int:
    la = len(a) if la is None else la
    lb = len(b) if lb is None else lb
    ab = C.create_string_buffer(bytes(a), max(len(a), la) + 1)
    bb = C.create_string_buffer(bytes(b), max(len(b), lb) + 1)
    return ref_lib().score(ab, bb, la, lb, None)


def ref_fasta_load(path) -> list[bytes]:
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    f = libc.fopen(str(path).encode(), b"r")
    if not f:
        raise FileNotFoundError(path)
    ds = ref_lib().dataset_from_fasta(f)
    libc.fclose(f)
    return [C.string_at(ds.sequences[k], ds.sequence_lengths[k]) for k in range(ds.n_values)]


_harness = None


def ref_harness():
    """pthreads row driver around the reference's own score() (ref_harness.c)."""
    global _harness
    if _harness is None:
        ref_lib()  # the harness resolves score() from libref.so's objects it was linked with
        H = C.CDLL(str(REF_DIR / "libref_harness.so"))
        H.refh_score_rows.restype = C.c_int
        H.refh_score_rows.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                      C.c_int]
        H.refh_score_block.restype = C.c_int
        H.refh_score_block.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                       C.c_int, C.c_void_p, C.c_int]
        H.refh_score_pairs.restype = C.c_int
        H.refh_score_pairs.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_longlong,
                                       C.c_void_p, C.c_int]
        _harness = H
    return _harness


def ref_score_rows(seqs, rows=None, threads: int = 0) -> np.ndarray:
    """Reference score() of the listed query rows against every sequence
    (rows x n, D[r][k] = score(seq[k], seq[rows[r]]) as region_query calls it)."""
    sa = _SeqArray(seqs)
    if rows is None:
        rows_arr, nrows, rp = None, sa.n, None
    else:
        rows_arr = np.ascontiguousarray(rows, dtype=np.int32)
        nrows, rp = len(rows_arr), rows_arr.ctypes.data
    out = np.zeros((nrows, sa.n), dtype=np.uint32)
    ref_harness().refh_score_rows(sa.ptrs, sa.lens, sa.n, rp, nrows, out.ctypes.data,
                                  threads or os.cpu_count())
    return out


def ref_dbscan(seqs, eps: float, minpts: int):
    """The reference's dbscan_SW (real score(), O(n^2) per call) on in-memory sequences."""
    R = ref_lib()

    class Cl(C.Structure):
        _fields_ = [("members", C.POINTER(C.c_int)), ("n_members", C.c_int), ("id", C.c_int)]

    class SS(C.Structure):
        _fields_ = [("n_clusters", C.c_int), ("clusters", C.POINTER(Cl))]

    R.dbscan_SW.restype = SS
    R.dbscan_SW.argtypes = [_Dataset, C.c_float, C.c_int]
    sa = _SeqArray(seqs)
    mx = max((len(s) for s in seqs), default=0)
    ds = _Dataset(C.cast(sa.ptrs, C.POINTER(C.c_char_p)), C.cast(sa.lens, C.POINTER(C.c_size_t)), None,
                  sa.n, None, 0, mx)
    s = R.dbscan_SW(ds, C.c_float(eps), minpts)
    return [[s.clusters[c].members[k] for k in range(s.clusters[c].n_members)] for c in range(s.n_clusters)]


def ref_score_block(seqs, rows, cols, threads: int = 0) -> np.ndarray:
    """Reference score() on rows x cols (D[r][c] = score(seq[cols[c]],
    seq[rows[r]]), region_query's argument order) on all host cores."""
    sa = _SeqArray(seqs)
    rows_arr = np.ascontiguousarray(rows, dtype=np.int32)
    cols_arr = np.ascontiguousarray(cols, dtype=np.int32)
    out = np.zeros((len(rows_arr), len(cols_arr)), dtype=np.uint32)
    ref_harness().refh_score_block(sa.ptrs, sa.lens, sa.n, rows_arr.ctypes.data, len(rows_arr),
                                   cols_arr.ctypes.data, len(cols_arr), out.ctypes.data,
                                   threads or os.cpu_count())
    return out


def ref_score_pairs(seqs, a, b, threads: int = 0) -> np.ndarray:
    """Reference score(seq[a[k]], seq[b[k]]) for every k, on all host cores."""
    sa = _SeqArray(seqs)
    a = np.ascontiguousarray(a, dtype=np.int32)
    b = np.ascontiguousarray(b, dtype=np.int32)
    out = np.zeros(len(a), dtype=np.uint32)
    ref_harness().refh_score_pairs(sa.ptrs, sa.lens, sa.n, a.ctypes.data, b.ctypes.data, len(a),
                                   out.ctypes.data, threads or os.cpu_count())
    return out


def write_neighbor_bitmap_file(path, n: int, row_blocks, eps: float) -> int:
    """Neighbour bits of one eps in the "SWB1" form score_subst.c reads: bit j
    of row i is (float)D[i][j] <= eps, the test of region_query
    (dbscan.c:548-551), evaluated here in float32 on the distances of each
    (row0, uint32 rows) block that `row_blocks` yields in row order.  Returns
    the number of neighbour pairs (ordered, self included)."""
    words = (n + 63) // 64
    e = np.float32(eps)
    total = 0
    nxt = 0
    with open(path, "wb") as f:
        f.write(b"SWB1" + struct.pack("<II", n, words))
        for r0, block in row_blocks:
            assert r0 == nxt and block.shape[1] == n
            bits = block.astype(np.float32) <= e
            total += int(bits.sum())
            packed = np.packbits(bits, axis=1, bitorder="little")
            out = np.zeros((block.shape[0], words * 8), dtype=np.uint8)
            out[:, :packed.shape[1]] = packed
            f.write(out.tobytes())
            nxt += block.shape[0]
    assert nxt == n
    return total


def read_split_set_file(path) -> list[list[int]]:
    """Clusters (member lists in stored order) of a split-set file
    (cluster_io.c:638-669: "SPLIT_SET", int32 count, per cluster int32
    n_members, int32 id, members)."""
    b = Path(path).read_bytes()
    assert b[:9] == b"SPLIT_SET"
    (nc,) = struct.unpack_from("<i", b, 9)
    pos, out = 13, []
    for _ in range(nc):
        nm, _cid = struct.unpack_from("<ii", b, pos)
        pos += 8
        out.append(list(struct.unpack_from(f"<{nm}i", b, pos)))
        pos += 4 * nm
    return out


def write_dist_file(path, D: np.ndarray) -> None:
    """Distance matrix in the format score_subst.c reads."""
    D = np.ascontiguousarray(D)
    elem = 2 if D.max(initial=0) < 65536 else 4
    arr = D.astype(np.uint16 if elem == 2 else np.uint32)
    with open(path, "wb") as f:
        f.write(b"SWD1" + struct.pack("<II", D.shape[0], elem))
        f.write(arr.tobytes())


def run_ref_tool(name: str, args, cwd, env=None, timeout=3600) -> subprocess.CompletedProcess:
    exe = REF_DIR / name
    e = dict(os.environ)
    if env:
        e.update(env)
    return subprocess.run([str(exe)] + [str(a) for a in args], cwd=cwd, env=e,
                          capture_output=True, timeout=timeout)


# --------------------------------------------------------------------------
# host-logic restatements (pure Python; small inputs)
# --------------------------------------------------------------------------

f32 = np.float32


def not_covered(split, n: int) -> int:
    """data_not_in_clusters, cluster_io.c:564-593 (count only)."""
    seen = np.zeros(n, dtype=bool)
    for cl in split:
        seen[cl] = True
    return int(n - seen.sum())


def intersection_count(a: list, b: list) -> int:
    """intersection_of_clusters, cluster_io.c:446-501.  The larger cluster (a on
    ties) is sorted IN PLACE when it has more than 20 members (cluster_io.c:467-469)."""
    big, small = (a, b) if len(a) >= len(b) else (b, a)
    if len(big) > 20:
        big.sort()
        s = set(big)
        return sum(1 for x in small if x in s)
    return sum(1 for x in small for y in big if x == y)


def relation(ancient, new):
    """generate_split_set_relation, cluster_io.c:407-444: new cluster i links to
    ancient cluster j when |j ∩ i| > 0.8 |j|."""
    out = []
    for i in range(len(new)):
        conn = []
        for j in range(len(ancient)):
            inter = intersection_count(ancient[j], new[i])
            if float(inter) > float(len(ancient[j])) * 0.8:
                conn.append(j)
        out.append(conn)
    return out


def split_set_bytes(split) -> bytes:
    """store_split_set byte format, cluster_io.c:638-669 (ids = position)."""
    parts = [b"SPLIT_SET", struct.pack("<i", len(split))]
    for cid, cl in enumerate(split):
        parts.append(struct.pack("<ii", len(cl), cid))
        parts.append(np.asarray(cl, dtype="<i4").tobytes())
    return b"".join(parts)


def cluster_fasta_text(members, seqs) -> str:
    """create_single_cluster_file, cluster_io.c:672-699: '>sequence_<idx>' and
    50 characters per line."""
    out = []
    for m in members:
        s = seqs[m].decode("latin-1")
        out.append(">sequence_%i\n" % m)
        out.append("\n".join(s[k:k + 50] for k in range(0, len(s), 50)))
        out.append("\n")
    return "".join(out)


def adaptive(D: np.ndarray, eps_start: float, eps_inc: float, minpts: int, max_steps: int = 100000,
             truncate: bool = False, dbscan_fn=None):
    """adaptive_dbscan, dbscan.c:1117-1380, single thread, over a distance matrix.

    Returns (stdout text, kept split sets).  Float semantics follow the
    reference: eps_{k+1} = eps_k + inc in float (dbscan.c:1079-1080, 1267),
    halving eps_start while the first result has one cluster (dbscan.c:1211-1231),
    and the logged eps is eps_start + (i+1)*inc (dbscan.c:1323-1324).

    The reference's sweep is unbounded.  With truncate=True a sweep that has
    not reached one cluster after max_steps DBSCAN runs keeps the layers found
    so far (the engine's bounded sweep for many sets); otherwise it raises.
    dbscan_fn(eps, minpts) replaces the Smith-Waterman DBSCAN over D (the
    dbscan_L1 / dbscan_L2 builds of the same driver).
    """
    n = D.shape[0]
    out = []
    out.append("Performing adaptive clustering with parameters: \nminpts: %i\nepsilon_start: %f\n"
               "epsilon_inc: %f\n" % (minpts, float(f32(eps_start)), float(f32(eps_inc))))
    start = f32(eps_start)
    inc = f32(eps_inc)

    def run(eps):
        if f32(eps) == f32(-1):
            out.append("Warning @dbscan: epsilon value is: %f\n" % float(f32(eps)))
            out.append("Warning @dbscan: epsilon was changed to: %f\n" % float(f32(0.015)))
        if dbscan_fn is not None:
            return dbscan_fn(float(f32(eps)), minpts)
        return dbscan(D, float(f32(eps)), minpts)

    first = run(start)
    out.append("Initial set obtained with %i clusters\n" % len(first))
    counter = 0
    while len(first) == 1:
        if counter == 20 or start == 0:
            out.append("Error did not find a sufficient starting position in 20 tries \n")
            return "".join(out), None
        start = f32(start / f32(2))
        out.append("Trying new starting point \n")
        first = run(start)
        counter += 1
    out.append("Sarting with %i clusters\n" % len(first))
    nc = not_covered(first, n)
    out.append("Coverage at initial point: %f\n" % float(f32(1) - f32(nc) / f32(n)))
    sets = [first]
    eps_now = f32(start + inc)
    stop = None
    for _ in range(max_steps):
        eps = eps_now
        eps_now = f32(eps_now + inc)
        s = run(eps)
        sets.append(s)
        if len(s) == 1:
            stop = len(sets) - 1
            break
    if stop is None:
        if not truncate:
            raise RuntimeError("sweep did not reach one cluster")
        stop = len(sets) - 1
    kept = [first]
    conns = []
    for i in range(1, stop + 1):
        new = sets[i]
        if len(new) < len(kept[-1]):
            count = len(kept)
            nc = not_covered(new, n)
            out.append("Layer %i has %i clusters\n" % (count, len(new)))
            out.append("  Coverage at layer %i: %f\n" % (count, float(f32(1) - f32(nc) / f32(n))))
            # the reference build rounds start + (i+1)*inc once (a fused multiply-add);
            # in float64 the product and the sum are exact, so one rounding to float32 matches
            out.append("  Epsilon at layer %i: %f\n" % (count, float(f32(np.float64(start) + np.float64(i + 1) * np.float64(inc)))))
            conns.append(relation(kept[-1], new))
            kept.append(new)
    out.append("Connections found: \n")
    for i in range(len(kept) - 1, 0, -1):
        out.append("Layer %i:\n" % i)
        for j in range(len(kept[i])):
            out.append("  Cluster %i connected to: \n  " % j)
            for k in conns[i - 1][j]:
                out.append("%i " % k)
            out.append("\n")
    return "".join(out), kept


def find_closest(db, queries, idx: int):
    """find_closest_sequence_SW.c:26-153: query record idx-1 with the length of
    record 0 (find_closest_sequence_SW.c:49-53); strict '<', lowest index wins."""
    q = queries[idx - 1]
    lq = len(queries[0])
    best, best_i = 2 ** 31 - 1, -1
    for i, s in enumerate(db):
        d = score(s, q, len(s), lq)
        if d < best:
            best, best_i = d, i
    return best, best_i
