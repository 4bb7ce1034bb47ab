"""Generates the golden fixtures in tests/golden/ from the REFERENCE itself.

Every expected value below comes from the reference's own C code, compiled
from its sources into oracle/_ref by ``make -C oracle ref`` (score(),
dataset_from_fasta(), dbscan_SW(), the cluster_dbscan_SW /
adaptive_clustering_SW / find_closest_sequence_SW tools, and the
score-substitution builds of those tools).  Inputs are seeded synthetic data.

Run from the repository root (needs the reference sources, i.e. this
container, not the GPU box):

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import base64
import gzip
import hashlib
import json
import os
import sys
import tempfile
import zlib
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "mnhn-tree-tools_b200"))
import oracle as O  # noqa: E402
from swgpu import workloads as W  # noqa: E402

OUT = Path(__file__).resolve().parent
IUPAC = b"RYKMSWBDHV"


def rand_seq(rng, n, alphabet=b"ACGT"):
    a = np.frombuffer(alphabet, dtype=np.uint8)
    return a[rng.integers(0, len(a), size=n)].tobytes()


def with_n_runs(rng, s, frac=0.05):
    b = bytearray(s)
    for _ in range(rng.poisson(frac * len(b) / 8 + 0.5)):
        st = int(rng.integers(0, max(1, len(b))))
        ln = int(rng.geometric(0.15))
        b[st:st + ln] = b"N" * len(b[st:st + ln])
    return bytes(b)


def revcomp(s):
    return s[::-1].translate(bytes.maketrans(b"ACGTN", b"TGCAN"))


def mutate(rng, s, sub=0.05, indel=0.02):
    arr = np.frombuffer(s, dtype=np.uint8).copy()
    return W._mutate(rng, arr, sub, indel).tobytes()


def score_pairs():
    rng = np.random.default_rng(1234)
    pairs = []
    kat = [(b"ACGT", b"ACGT"), (b"ACGT", b"TCGT"), (b"ACGT", b"ACGA"), (b"ACGT", b"GGGG"),
           (b"NNNN", b"NNNN"), (b"ACGTACGTAC", b"ACGTAC"), (b"ACGTAC", b"ACGTACGTAC"), (b"", b""),
           (b"", b"ACG"), (b"ACG", b""), (b"A", b"A"), (b"A", b"C"), (b"AC", b"CA"), (b"acgt", b"ACGT"),
           (b"ACGT", b"acgt"), (b"RYKM", b"RYKM"), (b"ACGTRYACGT", b"ACGTRYACGT"), (b"A-C-G", b"A-C-G"),
           (b"NNNNACGTNNNN", b"ACGT"), (b"GATTACA" * 20, b"GATTACA" * 20), (b"T" * 100, b"T" * 99)]
    for a, b in kat:
        pairs.append((a, b, len(a), len(b)))
    for _ in range(300):  # plain DNA, related and unrelated
        la = int(rng.integers(1, 300))
        a = rand_seq(rng, la)
        b = mutate(rng, a, rng.uniform(0, 0.3), rng.uniform(0, 0.05)) if rng.random() < 0.6 else \
            rand_seq(rng, int(rng.integers(1, 300)))
        pairs.append((a, b, len(a), len(b)))
    for _ in range(150):  # N masking runs
        a = with_n_runs(rng, rand_seq(rng, int(rng.integers(20, 400))))
        b = with_n_runs(rng, mutate(rng, a, 0.1, 0.02))
        pairs.append((a, b, len(a), len(b)))
    for _ in range(80):  # other IUPAC letters and rare symbols
        a = rand_seq(rng, int(rng.integers(10, 200)), b"ACGT" * 6 + IUPAC + b"-*")
        b = mutate(rng, a.replace(b"-", b"A").replace(b"*", b"C"), 0.1, 0.0) if rng.random() < 0.5 else \
            rand_seq(rng, int(rng.integers(10, 200)), b"ACGTN" * 4 + IUPAC)
        pairs.append((a, b, len(a), len(b)))
    for _ in range(40):  # reverse complements
        a = rand_seq(rng, int(rng.integers(50, 300)))
        pairs.append((a, revcomp(mutate(rng, a, 0.05, 0.01)), 0, 0))
    for _ in range(30):  # long pairs across 512/768-column boundaries
        la = int(rng.integers(480, 1300))
        a = rand_seq(rng, la)
        b = mutate(rng, a, 0.08, 0.02) if rng.random() < 0.7 else rand_seq(rng, int(rng.integers(480, 1300)))
        pairs.append((a, b, len(a), len(b)))
    for _ in range(20):  # claimed length below the string length (find_closest's record-0 length)
        a = rand_seq(rng, int(rng.integers(20, 200)))
        b = rand_seq(rng, int(rng.integers(20, 200)))
        pairs.append((a, b, len(a), int(rng.integers(1, len(b) + 1))))
    out = []
    for a, b, la, lb in pairs:
        la = la or len(a)
        lb = lb or len(b)
        out.append([a.decode("latin-1"), b.decode("latin-1"), la, lb, O.ref_score(a, b, la, lb)])
    with gzip.open(OUT / "score_pairs.json.gz", "wt") as f:
        json.dump(out, f)
    print("score_pairs", len(out))


FASTA_CASES = {
    "simple": ">a\nACGT\n>b\nGGCCTA\n",
    "multiline": ">a\nACGTACGT\nTTGA\nCC\n>b\nA\n",
    "blank_middle": ">a\nACGT\n\nTTT\n>b\nGG\n",
    "trailing_blank": ">a\nACGT\n>b\nGGCC\n\n",
    "blank_after_header": ">a\nACG\n>b\n\nTT\n",
    "lowercase": ">a\nacgtNn\n>b\nAcGt\n",
    "crlf": ">a\r\nACGT\r\nTT\r\n>b\r\nGG\r\n",
    "leading_space": ">a\n  ACGT\n\tTT\n",
    "two_tokens": ">a\nACGT TTTT\nGG\n",
    "empty_record": ">a\n>b\nACGT\n>c\n",
    "no_final_newline": ">a\nACGT\n>b\nTTGG",
    "long_line": ">a\n" + "ACGT" * 375 + "\n>b\nA\n",
    "iupac": ">a\nACGTRYKMSWBDHVN\n>b\n-*.\n",
}


def fasta_cases():
    out = {}
    with tempfile.TemporaryDirectory() as td:
        for name, text in FASTA_CASES.items():
            p = Path(td) / f"{name}.fa"
            p.write_bytes(text.encode())
            out[name] = {"text": text, "expected": [s.decode("latin-1") for s in O.ref_fasta_load(p)]}
    (OUT / "fasta_cases.json").write_text(json.dumps(out, indent=1))
    print("fasta_cases", len(out))


def small_family_set(seed, n_fam, per_fam, root_len, sub=(0.01, 0.10), indel=0.01):
    rng = np.random.default_rng(seed)
    roots = [rng.integers(0, 4, size=root_len) for _ in range(n_fam)]
    seqs = []
    for f in range(n_fam):
        r = W.BASES[roots[f]]
        for _ in range(per_fam):
            seqs.append(W._mutate(rng, r, rng.uniform(*sub), indel).tobytes())
    order = rng.permutation(len(seqs))
    return [seqs[i] for i in order]


def hier_set(seed, n_top=2, n_sub=3, per_sub=30, root_len=120):
    """Two-level families: sub-roots are 15% mutants of a top root, reads are
    1-8% mutants of a sub-root, so an eps sweep merges in several layers."""
    rng = np.random.default_rng(seed)
    seqs = []
    for _ in range(n_top):
        top = W.BASES[rng.integers(0, 4, size=root_len)]
        for _ in range(n_sub):
            sub = W._mutate(rng, top, 0.15, 0.01)
            for _ in range(per_sub):
                seqs.append(W._mutate(rng, sub, rng.uniform(0.01, 0.08), 0.01).tobytes())
    order = rng.permutation(len(seqs))
    return [seqs[i] for i in order]


def dbscan_small():
    seqs = small_family_set(7, 4, 60, 150)
    D = O.ref_score_rows(seqs)
    cases = []
    for eps, minpts in [(60.0, 5), (60.0, 3), (95.5, 10), (150.0, 5), (-1.0, -1), (30.0, 2)]:
        cl = O.ref_dbscan(seqs, eps, minpts)
        cases.append({"eps": eps, "minpts": minpts, "clusters": cl})
    doc = {"seqs": [s.decode() for s in seqs], "cases": cases,
           "dist_sha256": hashlib.sha256(D.astype("<u2").tobytes()).hexdigest()}
    (OUT / "dbscan_small.json").write_text(json.dumps(doc))
    print("dbscan_small", [len(c["clusters"]) for c in cases])


def run_tool(name, args, cwd, env=None):
    r = O.run_ref_tool(name, args, cwd, env)
    return r.returncode, r.stdout.decode("latin-1")


def files_b64(d: Path, prefix: str):
    return {p.name: base64.b64encode(p.read_bytes()).decode() for p in sorted(d.glob(prefix + "*"))}


def adaptive_small():
    seqs = hier_set(11)
    doc = {"seqs": [s.decode() for s in seqs], "runs": []}
    for eps_start, inc, minpts in [(20.0, 15.0, 5), (400.0, 25.0, 4), (30.0, 12.5, 5), (45.0, 7.3, 3)]:
        with tempfile.TemporaryDirectory() as td:
            W.write_fasta(Path(td) / "in.fa", seqs)
            rc, out = run_tool("adaptive_clustering_SW", ["in.fa", eps_start, inc, minpts, "layer", 1], td)
            doc["runs"].append({"eps_start": eps_start, "eps_inc": inc, "minpts": minpts, "rc": rc,
                                "stdout": out, "files": files_b64(Path(td), "layer")})
    (OUT / "adaptive_small.json").write_text(json.dumps(doc))
    print("adaptive_small", [r["rc"] for r in doc["runs"]])


def cluster_tool_small():
    seqs = small_family_set(13, 3, 40, 100)
    with tempfile.TemporaryDirectory() as td:
        W.write_fasta(Path(td) / "in.fa", seqs)
        rc, out = run_tool("cluster_dbscan_SW", ["in.fa", 45.0, 4, "cl"], td)
        doc = {"seqs": [s.decode() for s in seqs], "eps": 45.0, "minpts": 4, "rc": rc, "stdout": out,
               "files": files_b64(Path(td), "cl-")}
    (OUT / "cluster_tool_small.json").write_text(json.dumps(doc))
    print("cluster_tool_small", out.strip())


def find_closest_small():
    rng = np.random.default_rng(17)
    db = [rand_seq(rng, int(rng.integers(60, 160))) for _ in range(120)]
    q1 = mutate(rng, db[37], 0.05, 0.01)[:90]
    q2 = mutate(rng, db[81], 0.1, 0.02) + rand_seq(rng, 10)
    q3 = db[5]
    queries = [q1, q2, q3]
    runs = []
    with tempfile.TemporaryDirectory() as td:
        W.write_fasta(Path(td) / "db.fa", db)
        W.write_fasta(Path(td) / "q.fa", queries)
        for idx in (1, 2, 3):
            if len(queries[idx - 1]) < len(queries[0]):
                continue  # the reference reads past the string there
            rc, out = run_tool("find_closest_sequence_SW", ["db.fa", "q.fa", idx, 4, f"out{idx}.fa"], td)
            runs.append({"idx": idx, "rc": rc, "stdout": out, "out": (Path(td) / f"out{idx}.fa").read_text()})
    doc = {"db": [s.decode() for s in db], "queries": [s.decode() for s in queries], "runs": runs}
    (OUT / "find_closest_small.json").write_text(json.dumps(doc))
    print("find_closest_small", [r["stdout"].strip() for r in runs])


def row_crcs(D16):
    return [zlib.crc32(D16[i].tobytes()) for i in range(D16.shape[0])]


def matrix_golden(name, seqs, extra=None):
    D = O.ref_score_rows(seqs)
    D16 = D.astype("<u2")
    doc = {"n": len(seqs), "sha256": hashlib.sha256(D16.tobytes()).hexdigest(), "row_crc32": row_crcs(D16),
           "max": int(D.max()), "cells": W.cells(seqs)}
    if extra:
        doc.update(extra(D))
    (OUT / f"{name}.json").write_text(json.dumps(doc))
    print(name, doc["sha256"][:16], doc["max"])
    return D


def config1_golden():
    seqs, _ = W.config1()

    def extra(D):
        out = {}
        with tempfile.TemporaryDirectory() as td:
            td = Path(td)
            W.write_fasta(td / "c1.fa", seqs)
            O.write_dist_file(td / "d.bin", D)
            env = {"SWGPU_SUBST_DIST": str(td / "d.bin")}
            rc, so = run_tool("cluster_dbscan_SW_subst", ["c1.fa", 130.0, 5, "c1"], td, env)
            files = sorted(td.glob("c1-*"))
            out["dbscan"] = {"eps": 130.0, "minpts": 5, "rc": rc, "stdout": so,
                             "files_sha256": {p.name: hashlib.sha256(p.read_bytes()).hexdigest() for p in files}}
            rc, so = run_tool("adaptive_clustering_SW_subst", ["c1.fa", 100.0, 60.0, 5, "lay", 1], td, env)
            files = sorted(td.glob("lay*"))
            out["adaptive"] = {"eps_start": 100.0, "eps_inc": 60.0, "minpts": 5, "rc": rc, "stdout": so,
                               "files_sha256": {p.name: hashlib.sha256(p.read_bytes()).hexdigest() for p in files}}
        return out

    matrix_golden("config1_golden", seqs, extra)


def subset_goldens():
    s2, _ = W.config2()
    matrix_golden("config2_head1500_golden", s2[:1500])
    s3, _ = W.config3()
    matrix_golden("config3_head1500_golden", s3[:1500])


def kmer_golden():
    """5-mer counts from the reference's own frequence_of_kmer_in_sequence()
    (kmers.c:157-229) over the k-mer strings of gen_dna_kmers() (kmers.c:87-107),
    so index b of the table is the reference's own k-mer order."""
    import ctypes as C
    R = O.ref_lib()
    R.gen_dna_kmers.restype = C.POINTER(C.c_char_p)
    R.gen_dna_kmers.argtypes = [C.c_size_t]
    R.frequence_of_kmer_in_sequence.restype = C.c_short
    R.frequence_of_kmer_in_sequence.argtypes = [C.c_char_p, C.c_char_p, C.c_size_t]
    rng = np.random.default_rng(77)
    seqs = [b"", b"A", b"ACGT", b"ACGTA", b"ACGTAC", b"AAAAAA", b"AAAAAAAAAAAAAAAAAAAA", b"ACGTN" * 6,
            b"acgtacgtacgt", b"ACGTRYACGTACGTAAA"]
    for L in [15, 16, 17, 20, 21, 22, 63, 100, 250, 600]:
        seqs.append(rand_seq(rng, L))
    for L in [40, 120, 300]:
        seqs.append(with_n_runs(rng, rand_seq(rng, L), 0.08))
    cases = []
    for k in (5, 3):
        km = R.gen_dna_kmers(k)
        for sq in seqs:
            counts = {}
            for b in range(4 ** k):
                c = R.frequence_of_kmer_in_sequence(km[b], sq, k)
                if c:
                    counts[str(b)] = int(c)
            cases.append({"k": k, "seq": sq.decode("latin-1"), "counts": counts})
    (OUT / "kmer_counts.json").write_text(json.dumps(cases))


def kmer_inputs(doc):
    """Sequences of one fasta2kmer_golden input: literal strings, or
    {"unit": u, "length": n} for u repeated to n symbols."""
    out = []
    for x in doc:
        if isinstance(x, str):
            out.append(x.encode("latin-1"))
        else:
            u = x["unit"]
            out.append((u * (x["length"] // len(u) + 1))[:x["length"]].encode("latin-1"))
    return out


def fasta2kmer_golden():
    """stdout of the reference's fasta2kmer (fasta2kmer.c, kmers.c, built from
    its sources into oracle/_ref) as sha256 + size, on seeded DNA and protein
    reads (lengths 1..300, N runs, IUPAC and lower-case symbols, symbols outside
    the alphabet) and on long repeats whose counts pass 32767 and 65535 (the
    reference keeps them in a short)."""
    rng = np.random.default_rng(123)
    dna = [b"A", b"AC", b"ACG", b"ACGT", b"ACGTA", b"ACGTAC", b"ACGTACGT", b"TTTTTTTTT", b"ACGTN" * 7,
           b"acgtacgtaaccggtt", b"ACGTRYKMACGTACGTAAA"]
    for L in [15, 16, 17, 31, 33, 64, 100, 180, 300]:
        dna.append(rand_seq(rng, L))
    for L in [50, 140, 290]:
        dna.append(with_n_runs(rng, rand_seq(rng, L), 0.08))
    for L in [80, 200]:
        b = bytearray(rand_seq(rng, L))
        for _ in range(6):
            b[int(rng.integers(0, L))] = IUPAC[int(rng.integers(0, len(IUPAC)))]
        dna.append(bytes(b))
    aa = b"ACDEFGHIKLMNPQRSTVWY"
    prot = [b"M", b"MK", b"MKV", b"WWWW", b"ACDEFGHIKLMNPQRSTVWY", b"mkvlaagg", b"MXBZU*MKV"]
    for L in [10, 19, 20, 21, 40, 90, 160, 200]:
        prot.append(rand_seq(rng, L, aa))
    for L in [60, 150]:
        b = bytearray(rand_seq(rng, L, aa))
        for _ in range(5):
            b[int(rng.integers(0, L))] = b"XBZJOU"[int(rng.integers(0, 6))]
        prot.append(bytes(b))
    long_doc = [{"unit": "A", "length": 66000}, {"unit": "C", "length": 33000},
                {"unit": "ACGT", "length": 68000}, {"unit": "ACGTTGCA", "length": 70001}]
    inputs = {"dna": [x.decode("latin-1") for x in dna], "protein": [x.decode("latin-1") for x in prot],
              "long": long_doc}
    runs = [("dna", k, 0) for k in (1, 2, 3, 5, 6, 7, 8, 9)] + [("protein", k, 1) for k in (1, 2, 3, 4)] + \
           [("dna", 3, 1), ("protein", 2, 0)] + [("long", k, 0) for k in (1, 2, 4, 8)] + [("long", 2, 1)]
    doc = {"inputs": inputs, "runs": []}
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        for name in inputs:
            seqs = kmer_inputs(inputs[name]) if name == "long" else [x.encode("latin-1") for x in inputs[name]]
            W.write_fasta(d / (name + ".fa"), seqs)
        for name, k, protein in runs:
            r = O.run_ref_tool("fasta2kmer", [name + ".fa", str(k), "4", str(protein)], d)
            assert r.returncode == 0, (name, k, r.stdout[-300:])
            doc["runs"].append({"input": name, "k": k, "protein": protein, "bytes": len(r.stdout),
                                "sha256": hashlib.sha256(r.stdout).hexdigest()})
            print("fasta2kmer", name, k, protein, len(r.stdout))
    (OUT / "fasta2kmer.json").write_text(json.dumps(doc, indent=0))


STALE_ENV = {"GLIBC_TUNABLES": "glibc.malloc.tcache_count=0:glibc.malloc.perturb=165"}


def points_golden():
    """The reference's k-mer / PCA DBSCAN tools (cluster_dbscan_kmerL1/L2,
    cluster_dbscan_pca, adaptive_clustering_kmer_L1/L2, adaptive_clustering_PCA,
    built from its sources into oracle/_ref): stdout and every file they write,
    on two-level read families (hier_set), their 3-mer and 4-mer tables from
    the reference's own fasta2kmer, and 3-D projections of three groups of two
    Gaussian blobs printed with six decimals (so sweeps keep several layers).

    The tools run with glibc's malloc cache off and fresh blocks filled with a
    byte pattern (STALE_ENV): expand_cluster reads right_in_left one slot past
    its filled length (dbscan.c:896), i.e. memory malloc did not initialise,
    and when that stale word equals a later neighbour the neighbour is dropped
    from the frontier.  With the pattern the word is never a point index, so
    the outputs are the reference's intended set difference; without it they
    depend on heap history (this data set's adaptive_clustering_PCA run keeps
    its first layer one eps step later)."""
    seqs = hier_set(31, n_top=2, n_sub=3, per_sub=15, root_len=160)
    n = len(seqs)
    rng = np.random.default_rng(31)
    sup = rng.normal(0, 8, size=(3, 3))
    sub = sup[:, None, :] + rng.normal(0, 2.5, size=(3, 2, 3))
    proj = np.array([sub[i % 3, (i // 3) % 2] + rng.normal(0, 0.5, size=3) for i in range(n)])
    proj_text = "".join(" ".join(f"{v:.6f}" for v in row) + "\n" for row in proj)
    doc = {"seqs": [s.decode("latin-1") for s in seqs], "proj": proj_text, "kmer": {}, "runs": [],
           "env": STALE_ENV}
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        W.write_fasta(d / "in.fa", seqs)
        (d / "proj.txt").write_text(proj_text)
        for k in (3, 4):
            r = O.run_ref_tool("fasta2kmer", ["in.fa", str(k), "1", "0"], d)
            assert r.returncode == 0
            (d / f"k{k}.tsv").write_bytes(r.stdout)
            doc["kmer"][str(k)] = r.stdout.decode()
        # eps values from the distance distributions (float64, only to pick parameters)
        def dists(X, p):
            diff = X[:, None, :] - X[None, :, :]
            return np.abs(diff).sum(-1) if p == 1 else np.sqrt((diff ** 2).sum(-1))
        k3 = np.loadtxt(d / "k3.tsv", usecols=range(1, 65))
        k4 = np.loadtxt(d / "k4.tsv", usecols=range(1, 257))
        q = lambda D, f: float(np.quantile(D[np.triu_indices(n, 1)], f))
        cases = []
        for name, X, p in (("k3", k3, 1), ("k4", k4, 2)):
            D = dists(X, p)
            tool = "cluster_dbscan_kmerL1" if p == 1 else "cluster_dbscan_kmerL2"
            for f, mp in ((0.02, 4), (0.08, 5), (0.3, 3)):
                cases.append((tool, ["in.fa", f"{name}.tsv", f"{q(D, f):.3f}", str(mp), "out_cl"], "out_"))
            atool = "adaptive_clustering_kmer_L1" if p == 1 else "adaptive_clustering_kmer_L2"
            cases.append((atool, [f"{name}.tsv", f"{q(D, 0.02):.3f}", f"{q(D, 0.03) - q(D, 0.02):.3f}", "4",
                                  "out_layer", "1"], "out_"))
        Dp = dists(proj, 2)
        for f, mp in ((0.03, 4), (0.3, 5)):
            cases.append(("cluster_dbscan_pca", ["in.fa", "proj.txt", "3", f"{q(Dp, f):.4f}", str(mp), "out_pc",
                                                 "out_pv"], "out_"))
        cases.append(("adaptive_clustering_PCA", ["in.fa", f"{q(Dp, 0.02):.4f}", f"{q(Dp, 0.04) - q(Dp, 0.02):.4f}",
                                                  "4", "out_player", "1", "3", "proj.txt"], "out_"))
        for tool, args, prefix in cases:
            for old in d.glob(prefix + "*"):
                old.unlink()
            rc, out = run_tool(tool, args, d, env=STALE_ENV)
            assert rc == 0, (tool, out[-400:])
            doc["runs"].append({"tool": tool, "args": args, "stdout": out, "files": files_b64(d, prefix)})
            print(tool, args, [ln for ln in out.splitlines() if "clusters" in ln][-3:], len(doc["runs"][-1]["files"]))
    (OUT / "points.json").write_text(json.dumps(doc))


def tree_golden():
    """The reference's split-set tree tools (split_sets_to_newick, tree_pureness,
    filter_split_sets_by_min, split_set_to_fasta, built from its sources into
    oracle/_ref) on the layers and logs of two adaptive_clustering_SW golden
    runs (adaptive_small.json): stdout and files.  filter_split_sets_by_min
    stores cluster ids the reference never sets (cluster_io.c:191-215); they
    come from malloc'd memory, i.e. the STALE_ENV pattern here, and are not
    compared."""
    src = json.loads((OUT / "adaptive_small.json").read_text())
    doc = {"source": "adaptive_small.json", "runs": []}
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        W.write_fasta(d / "in.fa", [s.encode() for s in src["seqs"]])
        for ri in (1, 3):
            run = src["runs"][ri]
            names = sorted(run["files"])
            for nm in names:
                (d / f"r{ri}_{nm}").write_bytes(base64.b64decode(run["files"][nm]))
            (d / f"r{ri}.log").write_text(run["stdout"])
            layers = [f"r{ri}_{nm}" for nm in names]
            cases = [("split_sets_to_newick", ["0", "0"] + layers),
                     ("split_sets_to_newick", ["3", "0"] + layers),
                     ("split_sets_to_newick", ["0", "1", "2", f"r{ri}.log", "5"] + layers),
                     ("split_sets_to_newick", ["2", "2", "3", f"r{ri}.log", "5"] + layers),
                     ("tree_pureness", ["in.fa", layers[1]] + layers),
                     ("filter_split_sets_by_min", ["4", "out_f"] + layers),
                     ("split_set_to_fasta", ["in.fa", layers[-2], "out_s"])]
            for tool, args in cases:
                for old in d.glob("out_*"):
                    old.unlink()
                rc, out = run_tool(tool, args, d, env=STALE_ENV)
                assert rc == 0, (tool, args, out[-300:])
                doc["runs"].append({"source_run": ri, "tool": tool, "args": args, "stdout": out,
                                    "files": files_b64(d, "out_")})
                print(tool, args[:3], out[:80].replace("\n", "|"), len(doc["runs"][-1]["files"]))
    (OUT / "trees.json").write_text(json.dumps(doc))


def score_callers_golden():
    """stdout of the reference's compareSW, silhouette, compare_norms and
    find_satellite (built from its sources into oracle/_ref, one thread) on
    seeded inputs: two families sets for the comparisons, projections with six
    decimals, a satellite filter with a size window and a distance bound."""
    rng = np.random.default_rng(91)
    one = small_family_set(91, 3, 20, 180)
    two = small_family_set(92, 2, 15, 200)
    one += [rand_seq(rng, int(rng.integers(60, 260))) for _ in range(5)]
    two += [with_n_runs(rng, rand_seq(rng, int(rng.integers(60, 260)))) for _ in range(5)]
    proj = rng.normal(0, 3, size=(len(one), 3))
    proj_text = "".join(" ".join(f"{v:.6f}" for v in row) + "\n" for row in proj)
    target = one[0]
    runs = []
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        W.write_fasta(d / "one.fa", one)
        W.write_fasta(d / "two.fa", two)
        W.write_fasta(d / "target.fa", [target])
        (d / "proj.txt").write_text(proj_text)
        cases = [("compareSW", ["one.fa", "two.fa", "1"]), ("silhouette", ["one.fa", "two.fa", "1"]),
                 ("silhouette", ["two.fa", "one.fa", "1"]), ("compare_norms", ["one.fa", "proj.txt", "3"]),
                 ("find_satellite", ["one.fa", "target.fa", "180", "30", "40", "400", "1"]),
                 ("find_satellite", ["one.fa", "target.fa", "100", "500", "90", "5000", "1"])]
        for tool, args in cases:
            rc, out = run_tool(tool, args, d)
            assert rc == 0, (tool, out[-500:])
            runs.append({"tool": tool, "args": args, "stdout": out})
    doc = {"one": [s.decode("latin-1") for s in one], "two": [s.decode("latin-1") for s in two],
           "target": target.decode("latin-1"), "proj": proj_text, "runs": runs}
    (OUT / "score_callers.json").write_text(json.dumps(doc))


def kmer2pca_tables():
    """The seeded input tables of kmer2pca.json, as the text kmer2pca reads:
    5-mer, 3-mer and 2-mer tables of random reads (fasta2kmer's format, made by
    the oracle's frequencies_from_dataset restatement), a table of fractions
    with spaces, tabs and exponents in its token stream, and tables of fewer
    than four samples (no sample enters the reference's covariance sums)."""
    rng = np.random.default_rng(2024)
    out = []

    def reads(n, lo, hi):
        return [rand_seq(rng, int(rng.integers(lo, hi + 1))) for _ in range(n)]

    out.append(("k3_n203", O.kmer_tsv(O.kmer_table(reads(203, 50, 400), 3)).decode(), 5))
    out.append(("k2_n50", O.kmer_tsv(O.kmer_table(reads(50, 20, 120), 2)).decode(), 16))
    out.append(("k4_n97", O.kmer_tsv(O.kmer_table(reads(97, 100, 300), 4)).decode(), 7))
    lines = []
    for i in range(41):
        vals = rng.normal(size=6) * np.array([5.0, 3.0, 2.0, 1.0, 0.5, 0.25]) + 10.0
        sep = "\t" if i == 0 else ("  " if i % 3 == 0 else "\t")
        toks = ["%.6f" % v if i % 5 else "%.6e" % v for v in vals]
        lines.append(f"row_{i}" + "\t" + sep.join(toks) + "\n")
    out.append(("fractions_n41", "".join(lines), 3))
    out.append(("k2_n3", O.kmer_tsv(O.kmer_table(reads(3, 30, 60), 2)).decode(), 16))
    out.append(("k1_n1", O.kmer_tsv(O.kmer_table(reads(1, 30, 60), 1)).decode(), 2))
    return out


def kmer2pca_golden():
    """Eigenvalue and projection files and stdout of the reference's own
    kmer2pca.c (built into oracle/_ref and linked, through oracle/lapack_shim.c,
    to the LAPACK dsyev inside scipy's OpenBLAS) on kmer2pca_tables()."""
    cases = []
    with tempfile.TemporaryDirectory() as td:
        d = Path(td)
        for name, text, dims in kmer2pca_tables():
            (d / "in.tsv").write_text(text)
            r = O.run_ref_tool("kmer2pca", ["in.tsv", "proj.txt", "ev.txt", str(dims), "4"], d)
            assert r.returncode == 0, r.stdout[-400:]
            cases.append({"name": name, "table": text, "dims": dims, "stdout": r.stdout.decode(),
                          "ev": (d / "ev.txt").read_text(), "proj": (d / "proj.txt").read_text()})
    (OUT / "kmer2pca.json").write_text(json.dumps({"cases": cases}))


if __name__ == "__main__":
    if not O.ref_available():
        O.build()
    which = sys.argv[1:] or ["score", "fasta", "dbscan", "adaptive", "cluster", "closest", "config1", "subsets",
                             "kmer", "callers", "fasta2kmer", "points", "trees", "kmer2pca"]
    if "score" in which:
        score_pairs()
    if "fasta" in which:
        fasta_cases()
    if "dbscan" in which:
        dbscan_small()
    if "adaptive" in which:
        adaptive_small()
    if "cluster" in which:
        cluster_tool_small()
    if "closest" in which:
        find_closest_small()
    if "config1" in which:
        config1_golden()
    if "subsets" in which:
        subset_goldens()
    if "kmer" in which:
        kmer_golden()
    if "callers" in which:
        score_callers_golden()
    if "fasta2kmer" in which:
        fasta2kmer_golden()
    if "points" in which:
        points_golden()
    if "trees" in which:
        tree_golden()
    if "kmer2pca" in which:
        kmer2pca_golden()
