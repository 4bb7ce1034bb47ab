"""Benchmark of the all-pairs Smith-Waterman neighbourhood engine on B200.

Default workload (config 3): 100,000 satellite-like reads (50 tandem-repeat
monomer families of 171 bp, reads of 150-342 bp, 2-15% substitution, half
reverse-complemented).  One step = one all-pairs score pass (5e9 unique
pairs, 3.0e14 DP cells) followed by the DBSCAN it serves (eps 400, minpts 10),
labels produced exactly as the reference's cluster_dbscan_SW would.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl swgpu|reference]
                    [--config 2|3|4|5]

Under torchrun each rank drives its own GPU on its own independently seeded
dataset of the same configuration (independent objects, no data-path
collective: weak scaling); the step time is the max over ranks.

Printed value: exact SW GCUPS = unique-pair DP cells (sum over i<j of
len_i*len_j) / seconds of the whole step (score pass + clustering), inputs
already resident on the device.  `e2e` is the same metric through the C ABI
with host buffers (upload, score pass, clustering, results back on the host),
repeated --e2e-reps times (default 2).

On one GPU the config-3 line carries the other workloads as side legs, each
with --leg-warmup / --leg-steps steps: `sweep_config2` (20,000 reads, one
score pass + the 8-eps adaptive sweep), `config5` (500 split sets in one
score launch + every set's sweep, against the sets one by one) and `config4`
(the learned prefilter against the exact step: speed-up, eps-neighbour
recall, adjusted Rand, the same recipe without the network);
`prefilter_speedup` is config 4's headline speed-up.

`--impl reference` times the reference's own CPU score() (compiled from its
sources into oracle/_ref) on all host cores on a bounded row sample of the
same workload and prints the same metric from it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "mnhn-tree-tools_b200"))

METRIC = "exact SW GCUPS + DBSCAN sec; prefilter speedup at ≥99.9% eps-nbr recall"
# config 2: eps 200 gives 156 clusters and eps 1800 the first single cluster on
# this workload, so the sweep evaluates exactly 8 eps values (400 .. 1800)
WORKLOADS = {
    "2": {"gen": "config2", "mode": "adaptive", "eps_start": 200.0, "eps_inc": 200.0, "minpts": 5,
          "text": "config2: 20,000 DNA reads, lognormal lengths 100-600 bp (median 220), 200 families, "
                  "2-15% substitution, 1-3% indel, 2% N runs; one all-pairs score pass + adaptive DBSCAN "
                  "sweep over 8 eps values (eps_start 200, eps_inc 200, minpts 5)"},
    "4": {"gen": "config2", "mode": "prefilter", "eps_list": [300.0, 200.0], "minpts": 5,
          "text": "config4: learned prefilter on the config-2 distribution (20,000 reads); 5-mer features, MLP "
                  "1024-512-256-128 GELU, bf16 weights / fp32 accumulation, trained (Adam, weight decay 0.01) on 2M "
                  "exact-scored pairs of 60 datasets of 6,000 reads (36,000 families), three seeds, the network "
                  "with the fewest DP cells on the held-out calibration dataset kept (the projection baseline "
                  "chosen the same way), margins calibrated on 200k held-out pairs of that dataset; prefiltered "
                  "score pass + DBSCAN (minpts 5) against the exact pass + DBSCAN"},
    "5": {"gen": "config5", "mode": "multi", "eps_start": 300.0, "eps_inc": 100.0, "minpts": 5, "max_steps": 12,
          "text": "config5: 500 independent split sets of 50-5,000 reads (log-uniform sizes, 521,216 reads), "
                  "config-1 generator with 2-20 families per set; one score pass over all sets + every set's "
                  "adaptive DBSCAN sweep (eps_start 300, eps_inc 100, minpts 5, at most 12 steps)"},
    "3": {"gen": "config3", "mode": "dbscan", "eps": 400.0, "minpts": 10,
          "text": "config3: 100,000 satellite reads, 50 tandem-repeat monomer families of 171 bp, 150-342 bp, "
                  "2-15% substitution, half reverse-complemented; one all-pairs score pass + DBSCAN "
                  "(eps 400, minpts 10)"},
}


def dataset_seed(config: str, rank: int) -> int:
    """Seed of the dataset a rank works on: rank r of an N-GPU run scores its
    own independently seeded dataset of the same configuration (weak scaling,
    no data-path collective); rank 0 has the single-GPU dataset."""
    return {"2": 2, "3": 3, "4": 2, "5": 5}[config] + rank


def max_over_ranks(x: float, dist, device) -> float:
    """The largest x over all ranks (one all-reduce; x itself without a group)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0")), \
        int(os.environ.get("WORLD_SIZE", "1"))


# ---------------------------------------------------------------------------
# reference CPU arm / baseline
# ---------------------------------------------------------------------------
_REF_PROBE = {}


def reference_sample(seqs, target_s: float = 12.0, threads: int = 0):
    """Times the reference score() (or, without oracle/_ref, the oracle's C
    restatement) on all host cores over a bounded sample of query rows x all
    sequences.  Returns (GCUPS, info dict).  The first call on a data set
    times a probe of one row per thread to size the sample; later calls on
    the same data set reuse that rate (the sample is the same seeded row
    choice every time)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np

    import oracle as O
    threads = threads or os.cpu_count() or 1
    kind = "reference" if (O.REF_DIR / "libref_harness.so").exists() else "port"
    fn = O.ref_score_rows if kind == "reference" else O.score_rows
    L = np.array([len(s) for s in seqs], dtype=np.float64)
    rng = np.random.default_rng(0)
    key = (id(seqs), len(seqs), threads)
    if key not in _REF_PROBE:
        rows = [int(r) for r in rng.choice(len(seqs), size=max(threads, 8), replace=False)]
        t0 = time.perf_counter()
        fn(seqs, rows, threads)
        dt = time.perf_counter() - t0
        _REF_PROBE[key] = (len(rows), dt)
    probe_rows, probe_dt = _REF_PROBE[key]
    # grow the sample to about target_s seconds of CPU work
    n_rows = int(min(len(seqs), max(threads, probe_rows * target_s / max(probe_dt, 1e-3))))
    rows = [int(r) for r in rng.choice(len(seqs), size=n_rows, replace=False)]
    t0 = time.perf_counter()
    fn(seqs, rows, threads)
    dt = time.perf_counter() - t0
    cells = float(L[rows].sum() * L.sum())
    rate = cells / dt
    info = {"kind": kind, "cores": threads, "seconds": round(dt, 3), "rows": n_rows,
            "sample": f"{n_rows} query rows x all {len(seqs)} sequences of the same workload, "
                      f"region_query order (every ordered pair), {cells:.3e} cells"}
    return rate / 1e9, info


def fasta2kmer_leg(seqs, k: int = 5, cpu: bool = True, reps: int = 3):
    """fasta2kmer's two calls (kmers.c:292-385) on the same reads through the
    drop-in C ABI: frequencies_from_dataset (host sequences in, malloc'd host
    rows out) and write_kmer_base (text to /dev/null, so the file system is
    not timed), median of `reps` after one warm-up.  With cpu, the reference's
    own two functions (oracle/_ref/libref.so) on all host cores, timed the
    same way (one repetition)."""
    import ctypes as C

    import swgpu
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    buf = swgpu.SeqBuffer(seqs)
    ds = buf.dataset()

    def timed(lib_, threads):
        t0 = time.perf_counter()
        f = lib_.frequencies_from_dataset(ds, k, threads, 0)
        t1 = time.perf_counter()
        fp = libc.fopen(b"/dev/null", b"w")
        lib_.write_kmer_base(fp, f)
        libc.fclose(fp)
        t2 = time.perf_counter()
        ok = bool(f.frequencies) and f.n_seq == len(seqs)
        lib_.free_kmer_frequencies(f)
        if not ok:
            raise RuntimeError("frequencies_from_dataset failed")
        return 1e3 * (t1 - t0), 1e3 * (t2 - t1)

    L = swgpu.lib()
    timed(L, 1)
    runs = [timed(L, 1) for _ in range(reps)]
    counts_ms = statistics.median(r[0] for r in runs)
    text_ms = statistics.median(r[1] for r in runs)
    out = {"workload": f"fasta2kmer k={k} DNA over the same {len(seqs)} reads ({4 ** k} columns): "
                       "frequencies_from_dataset + write_kmer_base to /dev/null, host buffers",
           "counts_ms": round(counts_ms, 2), "text_ms": round(text_ms, 2),
           "e2e_ms": round(counts_ms + text_ms, 2), "cpu_baseline": None}
    if cpu:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O
        if (O.REF_DIR / "libref.so").exists():
            R = O.ref_lib()
            R.frequencies_from_dataset.restype = swgpu.KmerFrequencies
            R.frequencies_from_dataset.argtypes = [swgpu.Dataset, C.c_size_t, C.c_int, C.c_int]
            R.write_kmer_base.restype = None
            R.write_kmer_base.argtypes = [C.c_void_p, swgpu.KmerFrequencies]
            R.free_kmer_frequencies.restype = None
            R.free_kmer_frequencies.argtypes = [swgpu.KmerFrequencies]
            threads = os.cpu_count() or 1
            rc, rt = timed(R, threads)
            out["cpu_baseline"] = {"kind": "reference", "cores": threads, "counts_ms": round(rc, 1),
                                   "text_ms": round(rt, 1), "e2e_ms": round(rc + rt, 1),
                                   "sample": "the whole workload, one repetition (write_kmer_base is "
                                             "single-threaded in the reference)"}
            out["speedup_e2e"] = round((rc + rt) / (counts_ms + text_ms), 1)
    return out


def kmer_dbscan_leg(eng, seqs, dev, k: int = 5, cpu: bool = True, reps: int = 3):
    """dbscan_L2 over the k-mer tables of the same reads (the k-mer / PCA
    DBSCAN path, dbscan.c:563-779): the table from the GPU, then through the C
    ABI with host buffers the point upload (every L2 distance on the GPU) and
    one DBSCAN, median of `reps`.  The distance kernel's CUDA-event time gives
    its roofline: 2 FP32 instructions (subtract, fused multiply-add) per pair
    and dimension against 148 SMs x 128 FP32 lanes at the sampled clock.  With
    cpu, the reference's own dbscan_L2 (oracle/_ref/libref_l2.so, single
    threaded as the reference is) on the first m points, m sized for about
    10 s."""
    import ctypes as C

    import numpy as np
    import torch

    import swgpu
    table = eng.kmer_counts(seqs, k)
    V = np.ascontiguousarray(table.T, dtype=np.float32)  # values[dim][point]
    dims, n = V.shape
    rng = np.random.default_rng(0)
    sample = rng.choice(n, size=(64, 2))
    d = np.sqrt(((V[:, sample[:, 0]] - V[:, sample[:, 1]]) ** 2).sum(0))
    eps = float(np.quantile(d, 0.02))
    up, db, kern = [], [], []
    clusters = None
    for r in range(reps + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        eng.upload_points(V, 2)  # SWE_METRIC_L2
        t1 = time.perf_counter()
        clusters = eng.dbscan(eps, 5)
        t2 = time.perf_counter()
        if r:
            up.append(1e3 * (t1 - t0))
            db.append(1e3 * (t2 - t1))
            kern.append(eng.stats()["ms_score_pass"])
    kms = statistics.median(kern)
    pair_dims = n * (n - 1) / 2 * dims
    props = torch.cuda.get_device_properties(dev)
    peak = props.multi_processor_count * 128 * 1.965e9  # FP32 lanes x clocks.max.sm
    out = {"workload": f"dbscan_L2 (eps {eps:.3f}, minpts 5) over the {k}-mer tables of the same {n} reads "
                       f"({dims} dimensions), host values in, clusters out",
           "upload_ms": round(statistics.median(up), 2), "dbscan_ms": round(statistics.median(db), 2),
           "e2e_ms": round(statistics.median(up) + statistics.median(db), 2), "clusters": len(clusters),
           "kernel": {"name": "point_dist_kernel", "ms": round(kms, 3),
                      "unique_pair_dims_per_s": round(pair_dims / (kms * 1e-3), 1),
                      "bound": "fp32", "achieved": round(2 * pair_dims / (kms * 1e-3) / 1e12, 3),
                      "peak": round(peak / 1e12, 3), "unit": "T FP32 lane-instructions/s",
                      "frac": round(2 * pair_dims / (kms * 1e-3) / peak, 4),
                      "peak_source": "SMs x 128 FP32 lanes x 1,965 MHz (clocks.max.sm)"},
           "cpu_baseline": None}
    if cpu:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O
        lib_path = O.REF_DIR / "libref_l2.so"
        if lib_path.exists():
            R = C.CDLL(str(lib_path))
            R.dbscan_L2.restype = swgpu.SplitSet
            R.dbscan_L2.argtypes = [swgpu.Dataset, C.c_float, C.c_int]
            R.free_split_set_and_associated_clusters.argtypes = [swgpu.SplitSet]

            def aligned_row(x):
                # the reference's AVX loads need 32-byte aligned rows, readable in whole 8-float vectors
                buf = np.zeros(len(x) + 16, dtype=np.float32)
                off = (-buf.ctypes.data % 32) // 4
                row = buf[off:off + len(x) + 8]
                row[:len(x)] = x
                return row

            def ref_run(m):
                rows = [aligned_row(V[j, :m]) for j in range(dims)]
                ptrs = (C.c_void_p * dims)(*[r.ctypes.data for r in rows])
                ds = swgpu.Dataset(None, None, None, m, C.cast(ptrs, C.c_void_p), dims, 0)
                t0 = time.perf_counter()
                s = R.dbscan_L2(ds, C.c_float(eps), 5)
                dt = time.perf_counter() - t0
                R.free_split_set_and_associated_clusters(s)
                return dt

            m = min(n, 1000)
            dt = ref_run(m)
            m = int(min(n, m * (10.0 / max(dt, 1e-3)) ** 0.5))
            dt = ref_run(m)
            rate = m * m * dims / dt
            out["cpu_baseline"] = {"kind": "reference", "cores": 1, "seconds": round(dt, 3),
                                   "pair_dims_per_s": round(rate, 1),
                                   "sample": f"the reference's dbscan_L2 on the first {m} points (every region "
                                             f"query scans all {m} points: {m}^2 x {dims} pair-dimensions)"}
            # the reference evaluates every ordered pair in its region queries: n^2 x dims per pass
            out["dbscan_vs_cpu"] = round((n * n * dims / rate) / (out["e2e_ms"] * 1e-3), 1)
    return out


def kmer2pca_leg(eng, seqs, dev, k: int = 5, dims: int = 7, cpu: bool = True, reps: int = 3):
    """kmer2pca (kmer2pca.c) on the k-mer table of the same reads: through the
    C ABI with host buffers (kmer2pca's float64 table in; every eigenvalue and
    the projections onto the `dims` leading eigenvectors out), median of
    `reps` after one warm-up, and the drop-in tool on the table's text file.
    The Gram kernel's CUDA-event time gives its roofline: n4 nf (nf + 1) / 2
    multiply-adds (the lower triangle of X4^T X4, n4 = n - n % 4 samples)
    against 148 SMs x 64 FP64 FMA per clock x 2 at 1,965 MHz.  With cpu, the
    reference's own kmer2pca (oracle/_ref, LAPACK from scipy's OpenBLAS) on
    the same file with all host threads, on the first m rows when the whole
    table would take more than about 20 s."""
    import subprocess
    import tempfile

    import numpy as np
    import torch

    import swgpu
    table = eng.kmer_counts(seqs, k)
    X = table.astype(np.float64)
    n, nf = X.shape
    n4 = n - n % 4
    e2e, gram, cov_ms, eig, proj, up = [], [], [], [], [], []
    for r in range(reps + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        w, P, info = eng.pca(X, dims)
        t1 = time.perf_counter()
        if r:
            e2e.append(1e3 * (t1 - t0))
            gram.append(info["ms_gram"])
            cov_ms.append(info["ms_covariance"])
            eig.append(info["ms_eigen"])
            proj.append(info["ms_project"])
            up.append(info["ms_upload"])
    gms = statistics.median(gram)
    fmas = n4 * nf * (nf + 1) / 2
    props = torch.cuda.get_device_properties(dev)
    peak = props.multi_processor_count * 64 * 2 * 1.965e9
    achieved = 2 * fmas / (gms * 1e-3)
    out = {"workload": f"kmer2pca ({dims} dimensions) of the {k}-mer table of the same {n} reads ({nf} features), "
                       f"host float64 table in, eigenvalues and projections out",
           "e2e_ms": round(statistics.median(e2e), 2), "upload_ms": round(statistics.median(up), 2),
           "covariance_ms": round(statistics.median(cov_ms), 3), "eigen_ms": round(statistics.median(eig), 1),
           "project_ms": round(statistics.median(proj), 3), "exact_route": bool(info["exact"]),
           "top_eigenvalue": round(float(w[-1]), 6),
           "kernel": {"name": "pca_gram_kernel", "ms": round(gms, 3), "bound": "fp64",
                      "achieved": round(achieved / 1e12, 3), "peak": round(peak / 1e12, 2), "unit": "TFLOP/s",
                      "frac": round(achieved / peak, 4),
                      "peak_source": "SMs x 64 FP64 FMA/clock x 2 x 1,965 MHz (clocks.max.sm); nominal, not "
                                     "measured"},
           "tool_ms": None, "cpu_baseline": None}
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "table.tsv")
        with open(path, "wb") as f:
            eng_text = eng.kmer_tsv(table)
            f.write(eng_text)
        t0 = time.perf_counter()
        r = subprocess.run([str(swgpu.BIN_DIR / "kmer2pca"), path, os.path.join(td, "p"), os.path.join(td, "e"),
                            str(dims), "1"], capture_output=True, timeout=600)
        if r.returncode == 0:
            out["tool_ms"] = round(1e3 * (time.perf_counter() - t0), 1)
        if cpu:
            sys.path.insert(0, str(ROOT / "oracle"))
            import oracle as O
            ref = O.REF_DIR / "kmer2pca"
            if ref.exists():
                threads = os.cpu_count() or 1

                def ref_run(rows):
                    src = path
                    if rows < n:
                        src = os.path.join(td, f"head{rows}.tsv")
                        with open(src, "wb") as f:
                            f.write(b"".join(eng_text.splitlines(keepends=True)[:rows]))
                    t0 = time.perf_counter()
                    rr = subprocess.run([str(ref), src, os.path.join(td, "rp"), os.path.join(td, "re"), str(dims),
                                         str(threads)], capture_output=True, timeout=900)
                    return time.perf_counter() - t0, rr.returncode

                m = min(n, 1000)
                dt, rc = ref_run(m)
                if rc == 0:
                    if m < n and dt * n / m <= 20.0:
                        m = n
                    elif m < n:
                        m = int(min(n, max(m, m * 20.0 / max(dt, 1e-3))))
                    dt, rc = ref_run(m)
                if rc == 0:
                    out["cpu_baseline"] = {
                        "kind": "reference", "cores": threads, "seconds": round(dt, 3),
                        "rows_per_s": round(m / dt, 1),
                        "sample": f"the reference's kmer2pca tool (file in, files out; LAPACK dsyev from scipy's "
                                  f"OpenBLAS) on the first {m} of the {n} rows, {threads} threads"}
                    if out["tool_ms"]:
                        out["tool_vs_cpu"] = round((n * dt / m) / (out["tool_ms"] * 1e-3), 1)
    return out


def side_leg(fn, *args, **kw):
    """A side leg's object; a leg that fails reports its error in place of its
    numbers instead of taking the main line down with it."""
    try:
        return fn(*args, **kw)
    except Exception as e:  # noqa: BLE001 - any failure of a side measurement
        return {"error": f"{type(e).__name__}: {e}"}


def run_leg(args):
    """One side leg alone (profiling a small case of its kernels)."""
    import swgpu
    from swgpu import workloads as W
    seqs, _ = W.config2(seed=dataset_seed("2", 0))
    if args.n:
        seqs = seqs[:args.n]
    if args.leg == "fasta2kmer":
        out = fasta2kmer_leg(seqs, cpu=not args.no_cpu_baseline)
    else:
        eng = swgpu.Engine(device=0)
        leg = kmer2pca_leg if args.leg == "kmer2pca" else kmer_dbscan_leg
        out = leg(eng, seqs, 0, cpu=not args.no_cpu_baseline)
        eng.close()
    print(json.dumps({"leg": args.leg, **out}), flush=True)
    return 0


def run_reference(args):
    rank, _, world = env_rank()
    if rank != 0:
        return 0
    from swgpu import workloads as W
    wl = WORKLOADS[args.config]
    seqs, _ = getattr(W, wl["gen"])()
    cells = W.cells(seqs) if wl["mode"] != "multi" else sum(W.cells(st) for st in seqs)
    # the workload keys of the GPU arm's config, with the same values
    cfg = {"workload": wl["text"]}
    if wl["mode"] == "multi":  # the per-cell rate does not depend on the set boundaries
        cfg["n_sets"] = len(seqs)
        seqs = [q for st in seqs for q in st]
        cfg.update(n_sequences=len(seqs), cells_per_gpu=cells)
    else:
        cfg.update(n_sequences=len(seqs), cells_per_gpu=cells, pairs_per_gpu=len(seqs) * (len(seqs) - 1) // 2)
    times, rates = [], []
    info = None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        g, info = reference_sample(seqs, target_s=args.ref_seconds if i >= args.warmup else 1.0)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            rates.append(g)
            times.append(dt)
    value = statistics.median(rates)
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GCUPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * statistics.median(times), 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": cfg,
            "cpu_baseline": dict(info, value=round(value, 3), unit="GCUPS"),
            "e2e": {"value": round(value, 3), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference scores every ordered pair once per DBSCAN pass and re-scores per eps step"}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_traffic(kernel: str, workload: str):
    """DRAM bytes (read + write) of one launch of `kernel` on `workload`, from
    the committed ncu summary profiles/<kernel>_traffic.txt (lines
    `<workload> <read bytes> <write bytes>`), or None."""
    p = ROOT / "profiles" / f"{kernel}_traffic.txt"
    if not p.exists():
        return None
    for ln in p.read_text().splitlines():
        parts = ln.split()
        if len(parts) == 3 and parts[0] == workload:
            return int(float(parts[1]) + float(parts[2]))
    return None


def hbm_peak_gbs():
    """(GB/s, source) of the measured HBM copy bandwidth of this GPU pool."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "of measured (copy bandwidth)"
        except Exception:
            pass
    return 6650.0, "of fallback"


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
class Run:
    """One bench process: its rank and GPU, the process group (N > 1), the
    L2-flush buffer, the barrier and the max over ranks.  Every rank takes the
    same collective steps in the same order."""

    def __init__(self):
        import torch
        self.torch = torch
        self.rank, self.local, self.world = env_rank()
        self.dist = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
            self.dist = dist
        self.dev = self.local
        torch.cuda.set_device(self.dev)
        self.flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{self.dev}")

    def barrier(self):
        if self.dist:
            self.dist.barrier()
        self.torch.cuda.synchronize(self.dev)

    def flush_l2(self):
        """Writes 256 MB (more than the 126 MB L2) between timed steps."""
        self.flush.fill_(1)
        self.torch.cuda.synchronize(self.dev)

    def max(self, x: float) -> float:
        return max_over_ranks(x, self.dist, f"cuda:{self.dev}")

    def close(self):
        del self.flush
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()


def fast_roofline(eng_cells: float, kernel_ms: float, dev: int, traffic=None) -> dict:
    """The hot kernel against the integer roofline R = 2*P_int/K (P_int measured
    on this GPU by the instruction-mix probe)."""
    import swgpu
    fast_gcups = eng_cells / (kernel_ms * 1e-3) / 1e9
    _, peak_instr = swgpu.measure_mix_peak(dev)
    # R = 2 * P_int / K: P_int = lane instructions/s of the per-cell mix at full
    # issue on this GPU, K = 4.5 instructions per packed cell pair in that mix
    roof_peak = 2.0 * peak_instr / 4.5 / 1e9
    return {"bound": "int", "kernel": "fast_all_pairs_kernel", "achieved": round(fast_gcups, 1),
            "peak": round(roof_peak, 1), "unit": "Gcell/s", "frac": round(fast_gcups / roof_peak, 4),
            "peak_source": "measured on this GPU: issue rate of the kernel's per-cell 16x2 "
                           "instruction mix on independent chains, R = 2*P_int/4.5",
            "peak_k4": round(roof_peak * 4.5 / 4.0, 1),
            "frac_k4": round(fast_gcups / (roof_peak * 4.5 / 4.0), 4),
            "k4_note": "R = 2*P_int/4: the recurrence's minimum of 4 packed instructions per cell pair",
            "ms_per_launch": round(kernel_ms, 2),
            "traffic": traffic,
            "traffic_source": ("DRAM read+write bytes per launch from one ncu capture, stored in "
                               "profiles/fast_all_pairs_kernel_traffic.txt" if traffic else None)}


def measure_single(run: Run, config: str, args, steps: int, warmup: int, e2e_reps: int, cpu: bool,
                   kmer_legs: bool = False):
    """One data set: `warmup` untimed and `steps` timed steps of one all-pairs
    score pass + the DBSCAN (config 3) or adaptive sweep (config 2) it serves,
    then `e2e_reps` host-to-host repetitions through the C ABI.  Returns the
    line (rank 0) or None."""
    import swgpu
    from swgpu import workloads as W

    torch = run.torch
    rank, world, dev = run.rank, run.world, run.dev
    wl = WORKLOADS[config]
    gen = getattr(W, wl["gen"])
    split = bool(args.split)  # one data set over all ranks (strong scaling) instead of one per rank
    seqs, _ = gen(seed=dataset_seed(config, 0 if split else rank))
    if args.n:
        seqs = seqs[:args.n]
    cells = W.cells(seqs)
    eng = swgpu.Engine(device=dev)
    if split:
        from swgpu import split_pass
        eng.set_partition(rank, world)
    # tile plan of the 16x2 kernel from the autotuner (every rank of a split
    # pass must lay out the same tiles, so that mode keeps the default plan)
    tune = None if (split or args.no_autotune) else eng.autotune(seqs)
    eng.upload(seqs)

    exch = []

    def score():
        eng.score_all_pairs()
        if split and world > 1:  # the one exchange: bytewise minimum of the ranks' matrices
            exch.append(split_pass.exchange_tiles(eng, run.dist, f"cuda:{dev}"))

    def cluster():
        # the number of kept layers / clusters; the split sets stay in the library
        if wl["mode"] == "adaptive":
            return eng.adaptive(wl["eps_start"], wl["eps_inc"], wl["minpts"], prefix=None,
                                log_path="/dev/null", layers=False)[1]
        return eng.dbscan(wl["eps"], wl["minpts"], lists=False)

    def step():
        eng.timer_start()
        score()
        kept = cluster()
        return eng.timer_stop(), kept

    for _ in range(warmup):
        run.flush_l2()
        step()

    st0 = eng.stats()
    run.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    step_ms, kernel_ms, score_ms = [], [], []
    kept = None
    for _ in range(steps):
        run.flush_l2()  # L2 flush between timed steps (256 MB > 126 MB L2)
        ms, kept = step()
        s = eng.stats()
        step_ms.append(ms)
        kernel_ms.append(s["ms_fast_kernel"])
        score_ms.append(s["ms_score_pass"])
    run.barrier()
    clk = clocks.stop()
    st1 = eng.stats()
    total_ms = run.max(sum(step_ms))
    ms_per_step = total_ms / steps
    value = cells * (1 if split else world) / (ms_per_step * 1e-3) / 1e9
    launches = (st1["kernel_launches"] - st0["kernel_launches"]) // steps

    # the eps threshold kernel alone (HBM-bound): one launch per distinct
    # threshold, timed by the engine's CUDA events around the launch
    thr_ms = []
    for k in range(3):
        eng.dbscan((wl.get("eps") or wl["eps_start"]) + k, wl["minpts"], lists=False)
        thr_ms.append(eng.stats()["ms_last_neighbors"])
    thr_ms = statistics.median(thr_ms)

    # e2e through the C ABI with host buffers: upload + score + clustering + results on the host
    e2e_ms = []
    for _ in range(max(1, e2e_reps)):
        run.barrier()
        t0 = time.perf_counter()
        eng.upload(seqs)
        score()
        cluster()
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    b1 = eng.stats()
    e2e_total = run.max(sum(e2e_ms))
    e2e_value = cells * (1 if split else world) / (e2e_total / len(e2e_ms) * 1e-3) / 1e9
    # upload() resets the counters, so the last repetition's totals are the per-step figures
    h2d = b1["h2d_bytes"]
    d2h = b1["d2h_bytes"]

    line = None
    if rank == 0:
        kms = statistics.median(kernel_ms)
        traffic = measured_traffic("fast_all_pairs_kernel", f"config{config}") if not args.n else None
        roof = fast_roofline(st1["cells"] / (world if split else 1), kms, dev, traffic)
        n = len(seqs)
        dist_bytes = st1["dist_bytes"]
        thr_bytes = n * n * dist_bytes + n * ((n + 63) // 64) * 8 + n * 4
        hbm_peak = hbm_peak_gbs()
        cpu_line = None
        if world == 1 and cpu:
            g, info = reference_sample(seqs, target_s=args.ref_seconds)
            cpu_line = dict(info, value=round(g, 3), unit="GCUPS")
        sweep_s = (statistics.median(step_ms) - statistics.median(score_ms)) * 1e-3
        mat_gb = n * n * dist_bytes / 1e9
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GCUPS", "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": round(ms_per_step, 2), "higher_is_better": True,
            "scaling": "strong" if split else "weak", "vs_baseline": None, "dtype": "s16x2", "data": "synthetic",
            "config": {"workload": wl["text"], "n_sequences": n, "cells_per_gpu": cells,
                       "pairs_per_gpu": n * (n - 1) // 2,
                       "kept_layers" if wl["mode"] == "adaptive" else "clusters": kept,
                       "parallelism": (f"one dataset split over {world} GPUs (cost-balanced tile groups; each "
                                       f"rank all-gathers the others' tile rectangles)" if split
                                       else f"{world} independent datasets (one per GPU)"),
                       "l2": f"256 MB buffer written between timed steps (L2 flush); distance matrix "
                             f"{mat_gb:.1f} GB"},
            "dbscan_sec": round(ms_per_step * 1e-3, 4),
            "rerun_pairs": int(st1["reruns"]),
            "rerun_fraction": st1["reruns"] / max(n * (n - 1) // 2, 1),
            "score_pass_ms": round(statistics.median(score_ms), 2),
            ("sweep_ms" if wl["mode"] == "adaptive" else "dbscan_ms"): round(sweep_s * 1e3, 2),
            "roofline": roof,
            "threshold_roofline": {"bound": "hbm", "kernel": "thr_pack_kernel + thr_unpack_kernel", "achieved": round(
                thr_bytes / (thr_ms * 1e-3) / 1e9, 1), "peak": hbm_peak[0], "unit": "GB/s",
                "frac": round(thr_bytes / (thr_ms * 1e-3) / 1e9 / hbm_peak[0], 4), "peak_source": hbm_peak[1],
                "bytes_per_launch": thr_bytes, "ms_per_launch": round(thr_ms, 4)},
            "cpu_baseline": cpu_line,
            "e2e": {"value": round(e2e_value, 2), "unit": "GCUPS", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "reps": len(e2e_ms),
                    "note": "upload from host buffers + score pass + clustering + results on the host, "
                            "wall clock per repetition"},
            "gpu_launches": int(launches),
            "clocks": clk,
            "prefilter_speedup": None,
            "tile_plan": _plan(tune),
        }
        if exch:
            line["split_exchange"] = dict(exch[-1], matrix_bytes=int(eng.distance_bytes()))
        if world == 1 and kmer_legs:
            cpu_leg = not args.no_cpu_baseline
            line["fasta2kmer"] = side_leg(fasta2kmer_leg, seqs, cpu=cpu_leg)
            line["kmer_dbscan"] = side_leg(kmer_dbscan_leg, eng, seqs, dev, cpu=cpu_leg)
            line["kmer2pca"] = side_leg(kmer2pca_leg, eng, seqs, dev, cpu=cpu_leg)
    eng.close()
    return line


def _plan(tune):
    """The autotuner's choice as reported in the line (None: default plan)."""
    if not tune:
        return None
    return {"packs_per_block": tune["packs_per_block"], "threads": tune["threads"], "max_w": tune["max_w"],
            "from_cache": bool(tune["from_cache"]), "candidates": tune["candidates"],
            "sample_sequences": tune["sample"], "sample_ms_default": round(tune["ms_default"], 3),
            "sample_ms_best": round(tune["ms_best"], 3), "key": tune["key"],
            "note": "16x2 kernel tile plan timed on a length-stratified sample (untimed, before the warm-up); "
                    "default plan: 32 packs, 256 threads, max_w 24"}


# keys of a side leg's line that repeat the main line's
_LEG_DROP = ("metric", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "data", "prefilter_speedup")


def as_leg(line):
    if not isinstance(line, dict):
        return line
    return {k: v for k, v in line.items() if k not in _LEG_DROP}


def run_gpu(args):
    run = Run()
    line = measure_single(run, args.config, args, args.steps, args.warmup,
                          e2e_reps=min(max(args.steps, 1), args.e2e_reps), cpu=not args.no_cpu_baseline,
                          kmer_legs=(args.config == "2" and not args.no_kmer and not args.n))
    # the other workloads as side legs of the default line (one GPU; rank 0 alone,
    # so no rank waits in a collective meanwhile)
    if run.world == 1 and args.config == "3" and not args.no_legs and not args.n and line is not None:
        ls, lw = args.leg_steps, args.leg_warmup
        line["sweep_config2"] = side_leg(lambda: as_leg(measure_single(run, "2", args, ls, lw, e2e_reps=1,
                                                                       cpu=False)))
        line["config5"] = side_leg(lambda: as_leg(measure_multi(run, "5", args, ls, lw, e2e_reps=1)))
        c4 = side_leg(lambda: as_leg(measure_prefilter(run, "4", args, ls, lw, e2e_reps=1)))
        line["config4"] = c4
        if isinstance(c4, dict) and "value" in c4:
            line["prefilter_speedup"] = c4["value"]
    if line is not None:
        print(json.dumps(line), flush=True)
    run.close()
    return 0


def _pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
    return round(xs[k], 2)


def measure_multi(run: Run, config: str, args, steps: int, warmup: int, e2e_reps: int):
    """Many independent split sets: one score pass over every set, then all
    sets' sweeps advanced together (one threshold launch per round), against
    the same sets run one by one through the same engine.  Returns the line
    (rank 0) or None."""
    import swgpu
    from swgpu import workloads as W

    rank, world, dev = run.rank, run.world, run.dev
    wl = WORKLOADS[config]
    sets, _ = W.config5(seed=dataset_seed(config, rank))
    if args.n:
        sets = sets[:args.n]
    cells = sum(W.cells(st) for st in sets)
    nseq = sum(len(st) for st in sets)
    eng = swgpu.Engine(device=dev, dbscan_replay=args.dbscan_replay)
    tune = None if args.no_autotune else eng.autotune([q for st in sets for q in st])
    eng.upload_sets(sets)

    def sweeps():
        # layer counts only: the split sets stay in the library (freed there)
        return eng.adaptive_sets(wl["eps_start"], wl["eps_inc"], wl["minpts"], max_steps=wl["max_steps"],
                                 layers=False)

    def step():
        eng.timer_start()
        eng.score_all_pairs()
        score_ms = eng.stats()["ms_score_pass"]
        res = sweeps()
        return eng.timer_stop(), score_ms, res

    for _ in range(warmup):
        run.flush_l2()
        step()
    st0 = eng.stats()
    run.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    step_ms, score_ms, kernel_ms, lat = [], [], [], []
    res = None
    for _ in range(steps):
        run.flush_l2()
        ms, sms, res = step()
        step_ms.append(ms)
        score_ms.append(sms)
        kernel_ms.append(eng.stats()["ms_fast_kernel"])
        lat = [sms + r["done_ms"] for r in res]
    run.barrier()
    clk = clocks.stop()
    st1 = eng.stats()
    total_ms = run.max(sum(step_ms))
    ms_per_step = total_ms / steps
    value = cells * world / (ms_per_step * 1e-3) / 1e9
    launches = (st1["kernel_launches"] - st0["kernel_launches"]) // steps
    bad = [k for k, r in enumerate(res) if r["status"] != 0]

    # e2e: host sequences in, every set's layers back on the host
    e2e_ms = []
    for _ in range(max(1, e2e_reps)):
        run.barrier()
        t0 = time.perf_counter()
        eng.upload_sets(sets)
        eng.score_all_pairs()
        sweeps()
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    b1 = eng.stats()
    e2e_total = run.max(sum(e2e_ms))
    e2e_value = cells * world / (e2e_total / len(e2e_ms) * 1e-3) / 1e9

    # the same sets one by one (upload, score pass, sweep per set), rank 0 only
    one = None
    if rank == 0 and not args.no_one_by_one:
        solo = swgpu.Engine(device=dev, dbscan_replay=args.dbscan_replay)
        per = []
        t0 = time.perf_counter()
        for st in sets:
            t1 = time.perf_counter()
            solo.upload_sets([st])
            solo.score_all_pairs()
            solo.adaptive_sets(wl["eps_start"], wl["eps_inc"], wl["minpts"], max_steps=wl["max_steps"],
                               layers=False)
            per.append(1e3 * (time.perf_counter() - t1))
        total = time.perf_counter() - t0
        solo.close()
        done = []
        acc = 0.0
        for x in per:
            acc += x
            done.append(acc)
        one = {"total_s": round(total, 3), "sets_per_s": round(len(sets) / total, 2),
               "gcups": round(cells / total / 1e9, 2),
               "set_ms": {"p50": _pct(per, 50), "p90": _pct(per, 90), "p99": _pct(per, 99)},
               "latency_ms": {"p50": _pct(done, 50), "p90": _pct(done, 90), "p99": _pct(done, 99)}}

    line = None
    if rank == 0:
        kms = statistics.median(kernel_ms)
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": "GCUPS", "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": round(ms_per_step, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "s16x2", "data": "synthetic",
            "config": {"workload": wl["text"], "n_sets": len(sets), "n_sequences": nseq, "cells_per_gpu": cells,
                       "parallelism": f"{world} independent set collections (one per GPU)",
                       "l2": "256 MB buffer written between timed steps (L2 flush)"},
            "score_pass_ms": round(statistics.median(score_ms), 2),
            "sweeps_ms": round(statistics.median(step_ms) - statistics.median(score_ms), 2),
            "multi_instance": {
                "sets_per_s": round(len(sets) / (ms_per_step * 1e-3), 2),
                "latency_ms": {"p50": _pct(lat, 50), "p90": _pct(lat, 90), "p99": _pct(lat, 99)},
                "threshold_launches": st1["last_neighbor_launches"],
                "dbscan_replays": "host threads" if args.dbscan_replay == 1 else
                                  "device: one launch per round, one warp per (set, eps)",
                "failed_sets": bad[:10], "truncated_sets": sum(r["truncated"] for r in res),
                "one_by_one": one,
                "speedup_vs_one_by_one": round(one["total_s"] / (ms_per_step * 1e-3), 2) if one else None},
            "roofline": fast_roofline(st1["cells"], kms, dev),
            "cpu_baseline": None,
            "e2e": {"value": round(e2e_value, 2), "unit": "GCUPS", "h2d_bytes_per_step": int(b1["h2d_bytes"]),
                    "d2h_bytes_per_step": int(b1["d2h_bytes"]), "reps": len(e2e_ms)},
            "gpu_launches": int(launches),
            "clocks": clk,
            "prefilter_speedup": None,
            "tile_plan": _plan(tune),
        }
    eng.close()
    return line


def run_gpu_multi(args):
    run = Run()
    line = measure_multi(run, args.config, args, args.steps, args.warmup,
                         e2e_reps=min(max(args.steps, 1), args.e2e_reps))
    if line is not None:
        print(json.dumps(line), flush=True)
    run.close()
    return 0


def measure_prefilter(run: Run, config: str, args, steps: int, warmup: int, e2e_reps: int):
    """Learned prefilter (config 4): train on exact-scored pairs of other
    datasets of the distribution, calibrate on a held-out one, then time the
    prefiltered pass + DBSCAN against the exact pass + DBSCAN on the same GPU
    and report eps-neighbour recall and adjusted Rand of the clusters.
    Returns the line (rank 0) or None."""
    import numpy as np

    import swgpu
    from swgpu import prefilter as PF
    from swgpu import workloads as W

    rank, world, dev = run.rank, run.world, run.dev
    wl = WORKLOADS[config]
    t0 = time.perf_counter()
    # 60 datasets of 6,000 reads of the target distribution, 600 families of 10 reads each:
    # many families per pair sampled generalise to families the network never saw
    train_sets = [W.config2(seed=3000 + k, n=6000, n_fam=600)[0] for k in range(60)]
    cal_seqs, _ = W.config2(seed=101)
    test, _ = W.config2(seed=dataset_seed(config, rank))
    if args.n:
        test = test[:args.n]
    gen_s = time.perf_counter() - t0
    eng = swgpu.Engine(device=dev)
    eps_list = wl["eps_list"]
    # one network per seed, the one with the fewest DP cells on the held-out
    # calibration dataset at the headline eps kept (the test dataset plays no part)
    seeds = tuple(range(max(1, args.train_seeds)))
    trep = PF.train_select(eng, train_sets, cal_seqs, max(eps_list), seeds=seeds, weight_decay=args.weight_decay)
    cal = {eps: PF.calibrate(eng, cal_seqs, eps, seed=0) for eps in eps_list}
    n = len(test)
    cells = W.cells(test)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            run.flush_l2()
            fn()
        out, ms = None, []
        run.barrier()
        for _ in range(steps):
            run.flush_l2()
            eng.timer_start()
            out = fn()
            ms.append(eng.timer_stop())
        run.barrier()
        return out, statistics.median(ms)

    eng.upload(test)
    clocks = ClockSampler(dev)
    clocks.start()
    per_eps = {}
    launches_pf = None
    for eps in eps_list:
        margins, crep = cal[eps]

        def exact_step():
            eng.score_all_pairs()
            return eng.dbscan(eps, wl["minpts"])

        def pf_step():
            st = eng.score_prefiltered(eps, margins)
            return eng.dbscan(eps, wl["minpts"]), st

        lab_ex, ms_ex = timed(exact_step, steps, warmup)
        rp, _ = eng.neighbors(eps)
        exact_nbrs = int(rp[-1]) - n
        s0 = eng.stats()["kernel_launches"]
        (lab_pf, st), ms_pf = timed(pf_step, steps, warmup)
        launches_pf = (eng.stats()["kernel_launches"] - s0) // max(steps + warmup, 1)
        rp, _ = eng.neighbors(eps)
        recall = (int(rp[-1]) - n) / exact_nbrs if exact_nbrs else 1.0
        ari = PF.adjusted_rand(PF.labels_from_split(lab_ex, n), PF.labels_from_split(lab_pf, n))
        per_eps[str(int(eps))] = {
            "recall": round(recall, 6), "ari": round(ari, 6), "speedup": round(ms_ex / ms_pf, 3),
            "ms_exact_step": round(ms_ex, 2), "ms_prefilter_step": round(ms_pf, 2),
            "exact_neighbour_pairs": exact_nbrs // 2, "clusters_exact": len(lab_ex), "clusters_prefilter": len(lab_pf),
            "candidates": int(st["candidates"]), "tiles_kept": int(st["tiles_kept"]), "tiles_all": int(st["tiles_all"]),
            "tile_cells": st["tile_cells"], "ms_embed": round(st["ms_embed"], 2),
            "ms_candidates": round(st["ms_candidates"], 2), "ms_layout": round(st["ms_layout"], 2),
            "ms_layout_parts": {"groups": round(st["ms_groups"], 2), "tile_marks": round(st["ms_marks"], 2),
                                "upload": round(st["ms_upload"], 2)},
            "ms_score": round(st["ms_score"], 2), "margins": [[u, round(m, 5)] for u, m in margins],
            "scale": crep.get("scale"), "cal_recall_trials": crep.get("scale_trials")}
    clk = clocks.stop()
    head = str(int(eps_list[0]))

    # e2e through the C ABI with host buffers: upload, prefiltered pass, DBSCAN, clusters on the host
    margins0 = cal[eps_list[0]][0]
    e2e_ms = []
    b0 = eng.stats()
    e2e_parts = []
    for _ in range(max(1, e2e_reps)):
        run.barrier()
        t1 = time.perf_counter()
        eng.upload(test)
        t2 = time.perf_counter()
        eng.score_prefiltered(eps_list[0], margins0)
        t3 = time.perf_counter()
        eng.dbscan(eps_list[0], wl["minpts"])
        t4 = time.perf_counter()
        e2e_ms.append(1e3 * (t4 - t1))
        e2e_parts.append({"upload_ms": round(1e3 * (t2 - t1), 2), "prefiltered_pass_ms": round(1e3 * (t3 - t2), 2),
                          "dbscan_ms": round(1e3 * (t4 - t3), 2)})
    b1 = eng.stats()

    # the same recipe without the network: a fixed random projection of the k-mer features
    ablation = {}
    if not args.no_ablation:
        sub = train_sets[:5]
        eng.upload_sets(sub)
        Fsub = eng.kmer_features(5)
        ta, tb, td, tl = trep["train_pairs"]
        nsub = sum(len(x) for x in sub)
        keep = (ta < nsub) & (tb < nsub)
        # the same selection over projection seeds
        proj, prep = PF.projection_select(eng, Fsub, ta[keep], tb[keep], td[keep], tl, cal_seqs, max(eps_list),
                                          seeds=seeds)
        ablation["selection"] = prep
        for eps in eps_list:
            m2, r2 = PF.calibrate(eng, cal_seqs, eps, seed=0, embeddings=proj)
            eng.upload(test)
            eng.prefilter_set_embeddings(proj(eng))
            eng.score_all_pairs()
            rp, _ = eng.neighbors(eps)
            exact_nbrs = int(rp[-1]) - n

            def proj_step(eps=eps, m2=m2):
                st = eng.score_prefiltered(eps, m2)
                eng.dbscan(eps, wl["minpts"])
                return st

            # timed like the network's arm: warm-up steps, L2 flush, median of `steps`
            st2, ms2 = timed(proj_step, steps, warmup)
            rp, _ = eng.neighbors(eps)
            ablation[str(int(eps))] = {
                "recall": round((int(rp[-1]) - n) / exact_nbrs if exact_nbrs else 1.0, 6),
                "speedup": round(per_eps[str(int(eps))]["ms_exact_step"] / ms2, 3),
                "candidates": int(st2["candidates"]), "tiles_kept": int(st2["tiles_kept"]),
                "tile_cells": st2["tile_cells"], "ms_prefilter_step": round(ms2, 2),
                "fallback_full": int(st2["fallback_full"]), "scale": r2.get("scale"),
                "margins": [[u, round(m, 5)] for u, m in m2]}

    line = None
    if rank == 0:
        sp = per_eps[head]["speedup"]
        line = {
            "metric": METRIC, "value": sp, "unit": "x (prefiltered vs exact step, same GPU)", "n_gpus": world,
            "steps": steps, "warmup": warmup, "ms_per_step": per_eps[head]["ms_prefilter_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "s16x2 + bf16",
            "data": "synthetic",
            "config": {"workload": wl["text"], "n_sequences": n, "cells_per_gpu": cells, "eps": eps_list,
                       "headline_eps": eps_list[0], "minpts": wl["minpts"],
                       "parallelism": f"{world} independent datasets (one per GPU)",
                       "l2": "256 MB buffer written between timed steps (L2 flush)"},
            "prefilter": per_eps,
            "training": {"generation_s": round(gen_s, 2), "train_exact_pass_s": trep["train_exact_pass_s"],
                         "train_pair_scoring_s": trep["train_pair_scoring_s"], "train_s": trep["train_s"],
                         "epoch_loss": trep["epoch_loss"], "n_train": trep["n_train"],
                         "seed": trep["seed"], "selection": trep["selection"],
                         "n_cal": cal[eps_list[0]][1]["n_cal"], "train_pools": trep["train_pools"],
                         "weight_decay": args.weight_decay},
            "ablation_without_network": ablation,
            "e2e": {"value": round(per_eps[head]["ms_exact_step"] / statistics.median(e2e_ms), 3),
                    "unit": "x (exact device step / prefiltered host-to-host step)",
                    "h2d_bytes_per_step": int(b1["h2d_bytes"]), "d2h_bytes_per_step": int(b1["d2h_bytes"]),
                    "reps": len(e2e_ms), "parts": e2e_parts[-1]},
            "gpu_launches": int(launches_pf) if launches_pf is not None else None,
            "clocks": clk,
            "prefilter_speedup": sp,
        }
    eng.close()
    return line


def run_gpu_prefilter(args):
    run = Run()
    line = measure_prefilter(run, args.config, args, args.steps, args.warmup,
                             e2e_reps=min(max(args.steps, 1), args.e2e_reps))
    if line is not None:
        print(json.dumps(line), flush=True)
    run.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="swgpu", choices=["swgpu", "reference"])
    ap.add_argument("--ref-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", default="3", choices=sorted(WORKLOADS))
    ap.add_argument("--n", type=int, default=0, help="profile a smaller case: the first n reads of the workload "
                                                      "(config 5: the first n sets)")
    ap.add_argument("--no-one-by-one", action="store_true", help="config 5: skip the one-by-one comparison")
    ap.add_argument("--no-ablation", action="store_true", help="config 4: skip the run without the network")
    ap.add_argument("--train-seeds", type=int, default=3,
                    help="config 4: networks (and projections) tried; the one with the fewest DP cells on the "
                         "held-out calibration dataset is kept")
    ap.add_argument("--dbscan-replay", type=int, default=0, choices=(0, 1, 2),
                    help="config 5: DBSCAN replays of the sweeps on the device (0, 2) or on host threads (1)")
    ap.add_argument("--split", action="store_true",
                    help="config 2/3: one data set split over all ranks (strong scaling: tile groups, then an "
                         "all-gather of each rank's tile rectangles) instead of one data set per rank")
    ap.add_argument("--no-kmer", action="store_true", help="config 2: skip the fasta2kmer, k-mer DBSCAN and kmer2pca legs")
    ap.add_argument("--leg", choices=["fasta2kmer", "kmer_dbscan", "kmer2pca"],
                    help="run one side leg alone on the config-2 reads (the first --n) and print its object")
    ap.add_argument("--weight-decay", type=float, default=0.01, help="config 4: decoupled weight decay of Adam")
    ap.add_argument("--e2e-reps", type=int, default=2,
                    help="host-to-host repetitions of the step for `e2e` (at most --steps)")
    ap.add_argument("--no-legs", action="store_true",
                    help="config 3: skip the side legs (config-2 sweep, config 5, config 4)")
    ap.add_argument("--leg-steps", type=int, default=3, help="timed steps of each side leg")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default tile plan of the 16x2 kernel")
    ap.add_argument("--leg-warmup", type=int, default=3, help="warm-up steps of each side leg")
    args = ap.parse_args()
    if args.leg:
        return run_leg(args)
    if args.impl == "reference":
        return run_reference(args)
    if WORKLOADS[args.config]["mode"] == "multi":
        return run_gpu_multi(args)
    if WORKLOADS[args.config]["mode"] == "prefilter":
        return run_gpu_prefilter(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
