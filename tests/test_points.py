"""The k-mer / PCA DBSCAN path (dbscan_L1 / dbscan_L2, dbscan.c:563-779 and
950-1047; cluster_dbscan_kmer.c, cluster_dbscan_pca.c, adaptive_clustering.c
in its PCA and k-mer builds): the oracle against the outputs of the reference
tools themselves, the GPU point distances bit for bit against the oracle, the
DBSCAN and sweep on them, and the reference mains relinked on libswgpu."""
from __future__ import annotations

import base64
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import load_golden
from swgpu import workloads as W

METRIC = {"cluster_dbscan_kmerL1": 1, "cluster_dbscan_kmerL2": 2, "cluster_dbscan_pca": 2,
          "adaptive_clustering_kmer_L1": 1, "adaptive_clustering_kmer_L2": 2, "adaptive_clustering_PCA": 2}


def _inputs(doc):
    seqs = [s.encode("latin-1") for s in doc["seqs"]]
    return seqs


def _points_of(doc, run):
    """values[dim][point] the tool reads, and the FASTA it writes clusters from."""
    tool, args = run["tool"], run["args"]
    if tool.startswith("cluster_dbscan_kmer"):
        return O.load_kmer_text(doc["kmer"][args[1][1]])
    if tool.startswith("adaptive_clustering_kmer"):
        return O.load_kmer_text(doc["kmer"][args[0][1]])
    if tool == "cluster_dbscan_pca":
        return O.load_projection_text(doc["proj"], int(args[2]), len(doc["seqs"]))
    return O.load_projection_text(doc["proj"], int(args[6]), len(doc["seqs"]))


def _expected(doc, run, clusters_fn, adaptive_fn):
    """stdout and files of one golden run, from a DBSCAN and a sweep."""
    tool, args = run["tool"], run["args"]
    seqs = _inputs(doc)
    V = _points_of(doc, run)
    files = {}
    if tool.startswith("cluster_dbscan"):
        if tool == "cluster_dbscan_pca":
            eps, mp, pre, vpre = float(args[3]), int(args[4]), args[5], args[6]
        else:
            eps, mp, pre, vpre = float(args[2]), int(args[3]), args[4], None
        cl = clusters_fn(V, eps, mp, METRIC[tool])
        out = "%u clusters obtained \n" % len(cl)
        if len(cl) < 500:
            for c, m in enumerate(cl):
                files["%s-%03d" % (pre, c)] = O.cluster_fasta_text(m, seqs).encode()
                if vpre:
                    files["%s-%03d" % (vpre, c)] = O.cluster_values_text(m, V).encode()
        return out, files
    eps_start, eps_inc, mp, pre = float(args[1]), float(args[2]), int(args[3]), args[4]
    text, kept = adaptive_fn(V, eps_start, eps_inc, mp, METRIC[tool])
    for i, layer in enumerate(kept or []):
        files["%s%04d" % (pre, i)] = O.split_set_bytes(layer)
    return "Dataset read!\n" + text, files


def _oracle_clusters(V, eps, mp, metric):
    return O.dbscan_points(O.points_dist(V, metric), eps, mp, metric)


def _oracle_adaptive(V, es, ei, mp, metric):
    D = O.points_dist(V, metric)
    return O.adaptive(D, es, ei, mp, dbscan_fn=lambda e, m: O.dbscan_points(D, e, m, metric))


def _decode(files):
    return {k: base64.b64decode(v) for k, v in files.items()}


def test_points_oracle_matches_reference_tools():
    """Every golden run of the reference's six point tools (stdout and files,
    byte for byte) from the oracle's distances, DBSCAN and sweep."""
    doc = load_golden("points.json")
    for run in doc["runs"]:
        out, files = _expected(doc, run, _oracle_clusters, _oracle_adaptive)
        assert out == run["stdout"], run["tool"]
        assert files == _decode(run["files"]), run["tool"]


def test_points_dist_order_is_the_references():
    # an FMA chain in dimension order from +0 (dbscan.c:661-665), not a pairwise sum
    V = np.array([[1e8, 0.0], [1.0, 0.0], [-1e8, 0.0]], dtype=np.float32)
    D2 = O.points_dist(V, 2)
    acc = np.float32(0)
    for k in range(3):
        d = np.float32(V[k, 0] - V[k, 1])
        acc = np.float32(np.float64(d) * np.float64(d) + np.float64(acc))
    assert D2[0, 1] == acc == D2[1, 0]
    D1 = O.points_dist(V, 1)
    assert D1[0, 1] == np.float32(np.float32(np.float32(1e8) + np.float32(1)) + np.float32(1e8))


# ---------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def eng():
    import swgpu
    e = swgpu.Engine()
    yield e
    e.close()


def _rand_points(seed, dims, n, kind="normal"):
    rng = np.random.default_rng(seed)
    if kind == "normal":
        V = rng.normal(0, 3, size=(dims, n))
    elif kind == "counts":
        V = rng.poisson(2.0, size=(dims, n))
    else:  # wide dynamic range, denormals, zeros, negative zero
        V = rng.normal(0, 1, size=(dims, n)) * 10.0 ** rng.integers(-42, 30, size=(dims, n))
        V[:, ::7] = 0.0
        V[:, 3::11] = -0.0
    return V.astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,n,kind", [(1, 5, "normal"), (3, 257, "normal"), (17, 300, "wide"),
                                         (64, 512, "counts"), (256, 130, "wide"), (1024, 301, "counts"),
                                         (0, 10, "normal")])
@pytest.mark.parametrize("metric", [1, 2])
def test_point_distances_bit_exact(eng, dims, n, kind, metric):
    V = _rand_points(dims * 1000 + n, dims, n, kind)
    eng.upload_points(V, metric)
    got = eng.distances().view(np.uint32)
    want = O.points_dist(V, metric).view(np.uint32)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_point_distances_nan_inf(eng):
    V = _rand_points(5, 8, 64)
    V[2, 5] = np.inf
    V[3, 9] = np.inf
    V[4, 9] = -np.inf
    V[1, 20] = np.nan
    for metric in (1, 2):
        eng.upload_points(V, metric)
        got = eng.distances().view(np.uint32)
        want = O.points_dist(V, metric)
        nan = np.isnan(want)
        assert np.array_equal(np.isnan(got.view(np.float32)), nan)
        assert np.array_equal(got[~nan], want.view(np.uint32)[~nan])
        cl = eng.dbscan(4.0, 3)
        assert cl == O.dbscan_points(want, 4.0, 3, metric)


@pytest.mark.gpu
@pytest.mark.parametrize("metric", [1, 2])
def test_point_dbscan_and_sweep_match_oracle(eng, metric):
    rng = np.random.default_rng(metric)
    centres = rng.normal(0, 10, size=(6, 5))
    V = np.concatenate([centres[i % 6] + rng.normal(0, 1.0, size=(1, 5)) for i in range(600)]).T.astype(np.float32)
    eng.upload_points(V, metric)
    D = O.points_dist(V, metric)
    scale = float(np.median(D)) if metric == 1 else float(np.sqrt(np.median(D)))
    for f, mp in [(0.05, 4), (0.1, 10), (0.3, 5), (-1, -1), (0.0, 2)]:
        eps = -1.0 if f == -1 else f * scale
        assert eng.dbscan(eps, mp) == O.dbscan_points(D, eps, mp, metric), (f, mp)
    es, ei = 0.02 * scale, 0.03 * scale
    text, kept = eng.adaptive(es, ei, 4, prefix=None, log_path=None)
    want_text, want_kept = O.adaptive(D, es, ei, 4, dbscan_fn=lambda e, m: O.dbscan_points(D, e, m, metric))
    assert text == want_text and kept == want_kept


@pytest.mark.gpu
@pytest.mark.parametrize("build", ["reference_main", "cli"])
def test_point_tools_relinked_on_libswgpu(tmp_path, build):
    """The reference's cluster_dbscan_kmer (L1, L2), cluster_dbscan_pca and
    adaptive_clustering (kmer L1, L2, PCA) mains on libswgpu, and this
    package's own CLIs of the same names, reproduce the reference tools'
    stdout and files byte for byte."""
    import swgpu
    doc = load_golden("points.json")
    exe = {r["tool"]: (O.REF_DIR / (r["tool"] + "_on_swgpu") if build == "reference_main" else
                       swgpu.BIN_DIR / r["tool"]) for r in doc["runs"]}
    if not all(p.exists() for p in exe.values()):
        pytest.skip("drop-in builds not present")
    W.write_fasta(tmp_path / "in.fa", _inputs(doc))
    (tmp_path / "proj.txt").write_text(doc["proj"])
    for k, text in doc["kmer"].items():
        (tmp_path / f"k{k}.tsv").write_text(text)
    for run in doc["runs"]:
        for old in tmp_path.glob("out_*"):
            old.unlink()
        r = subprocess.run([str(exe[run["tool"]])] + run["args"], cwd=tmp_path, capture_output=True, timeout=600)
        assert r.returncode == 0, (run["tool"], r.stderr[-300:])
        assert r.stdout.decode() == run["stdout"], run["tool"]
        got = {p.name: p.read_bytes() for p in sorted(tmp_path.glob("out_*"))}
        assert got == _decode(run["files"]), run["tool"]


@pytest.mark.gpu
def test_point_distances_at_scale(eng):
    """4,000 points of 64 dimensions (k-mer-like counts): every distance bit
    for bit against the oracle, and DBSCAN against the oracle."""
    V = _rand_points(77, 64, 4000, "counts")
    eng.upload_points(V, 2)
    got = eng.distances().view(np.uint32)
    want = O.points_dist(V, 2)
    assert np.array_equal(got, want.view(np.uint32))
    eps = float(np.sqrt(np.quantile(want, 0.01)))
    assert eng.dbscan(eps, 5) == O.dbscan_points(want, eps, 5, 2)
