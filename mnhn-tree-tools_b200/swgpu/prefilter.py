"""Training and calibration recipe of the learned prefilter (host side).

Every computation runs in libswgpu: the exact kernel scores the training and
calibration pairs, the network trains on the tensor-core GEMMs, and the
calibrated margin feeds ``Engine.score_prefiltered``.  This module only picks
pairs and reads quantiles.

Recipe (datasets of the target distribution, none of them the data the
prefilter is used on):
  1. one exact score pass over the training datasets gives three pools:
     neighbours (d <= eps), near pairs (eps < d <= band) and all pairs;
  2. n_train training pairs drawn from the pools; their distances come from
     the exact kernel (``Engine.score_pairs``);
  3. Adam on the training pairs;
  4. n_cal held-out pairs drawn the same way from another dataset (families
     the network never saw), and per bucket of the longer length the margin =
     the q-quantile, over those with d <= eps, of
     emb_dist - floor(eps) / (4 max(len_a, len_b)), so that a fraction q of
     them pass the candidate test (q above the recall target);
  5. the prefiltered pass scores whole tiles around the candidates, so it
     finds more neighbours than the candidate test: on the held-out dataset
     the margins are scaled down (bisection) while the pass's own
     eps-neighbour recall stays >= q_pass (0.9998, above the 0.999 target).
"""
from __future__ import annotations

import math
import time

import numpy as np


def _pool(eng, eps: float, set: int | None = None):
    """Unordered pairs (i < j) with d <= eps of the scored dataset on ``eng``
    (one set of a several-set upload: indices of the whole upload)."""
    rp, cols = eng.neighbors(eps, set=set)
    off = 0 if set is None else eng.set_first[set]
    n = len(rp) - 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    keep = rows < cols
    return (rows[keep] + off).astype(np.int32), (cols[keep] + off).astype(np.int32)


def sample_pairs(eng, eps: float, band: float, counts, rng: np.random.Generator):
    """Disjoint pair samples from three pools of the scored upload on ``eng``
    (pairs inside one set): neighbours (d <= eps), near pairs
    (eps < d <= band) and uniform pairs.  counts = [(n_nbr, n_near,
    n_uniform), ...], one tuple per sample, drawn in that order (a pool that
    runs short is made up from uniform pairs); returns a list of (a, b)
    arrays and the pool sizes."""
    sets = range(eng.set_count())
    parts = [(_pool(eng, eps, k), _pool(eng, band, k)) for k in sets]
    na = np.concatenate([p[0][0] for p in parts])
    nb = np.concatenate([p[0][1] for p in parts])
    ba = np.concatenate([p[1][0] for p in parts])
    bb = np.concatenate([p[1][1] for p in parts])
    code = lambda x, y: x.astype(np.int64) * eng.n + y
    far = ~np.isin(code(ba, bb), code(na, nb))
    ba, bb = ba[far], bb[far]
    first = np.asarray(eng.set_first, dtype=np.int64)
    sizes = np.diff(first)
    wset = sizes * (sizes - 1) / 2.0
    wset = wset / wset.sum()
    p1 = rng.permutation(len(na))
    p2 = rng.permutation(len(ba))
    o1 = o2 = 0
    out = []
    for c1, c2, c3 in counts:
        want = c1 + c2 + c3
        c1 = min(c1, len(na) - o1)
        c2 = min(c2, len(ba) - o2)
        c3 = want - c1 - c2
        i1, i2 = p1[o1:o1 + c1], p2[o2:o2 + c2]
        o1 += c1
        o2 += c2
        ks = rng.choice(len(sizes), size=c3, p=wset)
        ua = rng.integers(0, sizes[ks])
        ub = (ua + 1 + rng.integers(0, np.maximum(sizes[ks] - 1, 1))) % sizes[ks]
        a = np.concatenate([na[i1], ba[i2], (first[ks] + ua).astype(np.int32)])
        b = np.concatenate([nb[i1], bb[i2], (first[ks] + ub).astype(np.int32)])
        perm = rng.permutation(len(a))
        out.append((a[perm], b[perm]))
    return out, (len(na), len(ba))


def calibrate_buckets(emb_dist, d, lens_a, lens_b, eps: float, q: float, buckets: int = 4, min_pairs: int = 4000):
    """Margins by the pair's longer length: bucket bounds at quantiles of the
    longer length over the held-out neighbours (each bucket with at least
    min_pairs of them), and in each bucket the q-quantile margin.  Returns
    [(upper, margin), ...] for ``Engine.score_prefiltered``."""
    T = math.floor(eps)
    d = np.asarray(d)
    nb = d <= T
    mx_all = np.maximum(np.asarray(lens_a), np.asarray(lens_b))
    mx = mx_all[nb]
    k = int(max(1, min(buckets, nb.sum() // max(min_pairs, 1))))
    edges = [int(np.quantile(mx, i / k, method="higher")) for i in range(1, k)] if k > 1 else []
    edges = sorted(set(e for e in edges if e > mx.min()))
    out = []
    lo = -1
    for up in edges + [10 ** 9]:
        sel = (mx_all >= (lo if lo >= 0 else 0)) & (mx_all < up)
        m = calibrate_margin(np.asarray(emb_dist)[sel], d[sel], np.asarray(lens_a)[sel], np.asarray(lens_b)[sel],
                             eps, q)
        out.append((up if up < 10 ** 9 else 0, m))
        lo = up
    return out


def pass_recall(eng, eps: float, margins, exact_count: int):
    """eps-neighbour recall of one prefiltered pass on the uploaded dataset
    (scored pairs are exact, so the prefiltered neighbour lists are subsets
    of the exact ones) and the pass statistics."""
    st = eng.score_prefiltered(eps, margins)
    rp, _ = eng.neighbors(eps)
    got = int(rp[-1]) - eng.n
    return (got / exact_count if exact_count else 1.0), st


def calibrate_scale(eng, eps: float, margins, q: float, trials: int = 7):
    """Smallest factor s in [0, 1] (bisection) such that the prefiltered pass
    with margins scaled by s keeps eps-neighbour recall >= q on the dataset
    uploaded and scored on ``eng``.  Returns (scaled margins, s, trials, DP
    cells of the pass with the scaled margins)."""
    eng.score_all_pairs()
    rp, _ = eng.neighbors(eps)
    exact = int(rp[-1]) - eng.n
    scaled = lambda f: [(u, f * m) for u, m in margins]
    lo, hi = 0.0, 1.0
    log = []
    cells = None  # DP cells of the pass at the chosen factor
    for _ in range(trials):
        mid = 0.5 * (lo + hi)
        r, st = pass_recall(eng, eps, scaled(mid), exact)
        log.append((round(mid, 4), r, int(st["candidates"]), int(st["tiles_kept"])))
        if r >= q:
            hi = mid
            cells = st["tile_cells"]
        else:
            lo = mid
    if cells is None:
        cells = eng.score_prefiltered(eps, scaled(hi))["tile_cells"]
    eng.score_all_pairs()
    return scaled(hi), hi, log, cells


def calibrate_margin(emb_dist, d, lens_a, lens_b, eps: float, q: float) -> float:
    """Smallest margin m with a fraction >= q of the pairs with d <= eps
    passing emb_dist <= floor(eps) / (4 max(len)) + m."""
    T = math.floor(eps)
    nb = np.asarray(d) <= T
    if not nb.any():
        return 0.0
    mx = np.maximum(np.asarray(lens_a)[nb], np.asarray(lens_b)[nb]).astype(np.float64)
    r = np.asarray(emb_dist, dtype=np.float64)[nb] - T / (4.0 * np.maximum(mx, 1))
    return float(np.quantile(r, q, method="higher"))


def train(eng, train_sets, eps: float, n_train: int = 2_000_000, epochs: int = 8, batch_pairs: int = 4096,
          lr: float = 1e-3, band_factor: float = 2.0, seed: int = 0, weight_decay: float = 0.0,
          mix=(0.25, 0.35), over_weight: float = 1.0):
    """Trains the prefilter on pairs of ``train_sets`` (independent datasets
    of the target distribution, scored in one exact pass): a fraction mix[0]
    of neighbours (d <= eps), mix[1] of near pairs (eps < d <= band_factor *
    eps), the rest uniform (default 25 / 35 / 40 %).  A neighbour's squared
    error counts over_weight times when its embedding distance over-estimates
    the target (the margins are set by such over-estimates).  The weights
    stay in ``eng``.  Returns a report."""
    rng = np.random.default_rng(seed)
    rep = {}
    t0 = time.perf_counter()
    eng.upload_sets(train_sets)
    eng.score_all_pairs()
    rep["train_exact_pass_s"] = round(time.perf_counter() - t0, 3)
    n_nb, n_near = int(n_train * mix[0]), int(n_train * mix[1])
    (tr,), pools = sample_pairs(eng, eps, band_factor * eps, [(n_nb, n_near, n_train - n_nb - n_near)], rng)
    rep["train_pools"] = [int(x) for x in pools]
    t1 = time.perf_counter()
    ta, tb = tr
    td = eng.score_pairs(ta, tb)
    rep["train_pair_scoring_s"] = round(time.perf_counter() - t1, 3)
    eng.prefilter_init(seed=seed + 1)
    t2 = time.perf_counter()
    losses = eng.prefilter_train(ta, tb, td, epochs=epochs, batch_pairs=batch_pairs, lr=lr, seed=seed + 2,
                                 weight_decay=weight_decay, over_eps=eps, over_weight=over_weight)
    rep["train_s"] = round(time.perf_counter() - t2, 3)
    rep["epoch_loss"] = [round(float(x), 6) for x in losses]
    rep["n_train"] = int(len(ta))
    rep["train_pairs"] = (ta, tb, td, np.array([len(x) for st in train_sets for x in st]))
    return rep


def calibrate(eng, cal_seqs, eps: float, n_cal: int = 200_000, q: float = 0.9995, band_factor: float = 2.0,
              tune_scale: bool = True, seed: int = 0, embeddings=None, q_pass: float = 0.9998, buckets: int = 4):
    """Margins for ``eps`` from held-out pairs of ``cal_seqs`` (a dataset of
    the distribution with families the network never saw): 60% neighbours,
    20% near pairs, 20% uniform; per bucket of the longer length the
    q-quantile margin, then (tune_scale) scaled down while the prefiltered
    pass itself keeps recall >= q_pass on this dataset.  q_pass sits above
    the 0.999 recall target because the recall of one pass varies from
    dataset to dataset by a few parts in 10^4 (families differ).
    ``embeddings``: a function of the uploaded engine returning embeddings
    to use instead of the network's (the method without the network).
    Returns (margins, report)."""
    rng = np.random.default_rng(seed + 7)
    rep = {}
    eng.upload(cal_seqs)
    eng.score_all_pairs()
    (cal,), cpools = sample_pairs(eng, eps, band_factor * eps,
                                  [(n_cal * 6 // 10, n_cal // 5, n_cal - n_cal * 6 // 10 - n_cal // 5)], rng)
    ca, cb = cal
    cd = eng.score_pairs(ca, cb)
    lens = np.array([len(x) for x in cal_seqs])
    if embeddings is not None:
        emb = embeddings(eng)
        eng.prefilter_set_embeddings(emb)
        ed = np.linalg.norm(emb[ca].astype(np.float64) - emb[cb], axis=1)
    else:
        ed = eng.prefilter_pair_dist(ca, cb)
    margins = calibrate_buckets(ed, cd, lens[ca], lens[cb], eps, q, buckets=buckets)
    rep["margins_pairs"] = margins
    rep["cal_pools"] = [int(x) for x in cpools]
    rep["cal_neighbours"] = int((cd <= math.floor(eps)).sum())
    rep["n_cal"] = int(len(ca))
    rep["cal_pairs"] = (ca, cb, cd, lens)
    if tune_scale:
        # the prefiltered pass scores whole tiles, so it finds more neighbours
        # than the candidate test alone: shrink the margins while the pass
        # itself keeps the recall on this held-out dataset
        margins, rep["scale"], rep["scale_trials"], rep["cal_cells"] = calibrate_scale(eng, eps, margins, q_pass)
    rep["margins"] = margins
    return margins, rep


def train_select(eng, train_sets, cal_seqs, eps: float, seeds=(0, 1, 2), **train_kw):
    """Model selection on held-out data: trains one network per seed (``train``
    with ``train_kw``), calibrates each for ``eps`` on ``cal_seqs`` and keeps
    the one whose calibrated prefiltered pass scores the fewest DP cells on
    that dataset.  The weights of the kept network stay in ``eng``; returns
    its training report with ``selection`` (seed, cells, final loss of
    every run).  Only the calibration dataset is used to choose, never the
    data the pass is later measured on."""
    best, runs = None, []
    for sd in seeds:
        rep = train(eng, train_sets, eps, seed=sd, **train_kw)
        _, crep = calibrate(eng, cal_seqs, eps, seed=0)
        runs.append({"seed": int(sd), "cal_cells": crep.get("cal_cells"), "loss": rep["epoch_loss"][-1]})
        if crep.get("cal_cells") is not None and (best is None or crep["cal_cells"] < best[0]):
            best = (crep["cal_cells"], sd, eng.prefilter_params(), rep)
    eng.prefilter_params(set_to=best[2])
    rep = best[3]
    rep["seed"] = int(best[1])
    rep["selection"] = runs
    return rep


def projection_select(eng, features, a, b, d, lens, cal_seqs, eps: float, seeds=(0, 1, 2)):
    """The same selection for the method without the network: one random
    projection per seed, each scaled by least squares on the exact-scored
    pairs (a, b, d) of the rows of ``features`` and calibrated on
    ``cal_seqs``; keeps the one with the fewest DP cells on that dataset.
    Returns (embedding function of an uploaded engine, report)."""
    best, runs = None, []
    for sd in seeds:
        scale = projection_scale(features, a, b, d, lens, seed=sd)
        fn = (lambda sc, s2: lambda en: (sc * projection_embeddings(en.kmer_features(5), seed=s2))
              .astype(np.float32))(scale, sd)
        _, crep = calibrate(eng, cal_seqs, eps, seed=0, embeddings=fn)
        runs.append({"seed": int(sd), "cal_cells": crep.get("cal_cells"), "scale": scale})
        if crep.get("cal_cells") is not None and (best is None or crep["cal_cells"] < best[0]):
            best = (crep["cal_cells"], sd, fn)
    return best[2], {"seed": int(best[1]), "selection": runs}


def fit(eng, train_sets, cal_seqs, eps: float, n_train: int = 2_000_000, n_cal: int = 200_000,
        epochs: int = 8, batch_pairs: int = 4096, lr: float = 1e-3, band_factor: float = 2.0, q: float = 0.9995,
        seed: int = 0, tune_scale: bool = True):
    """``train`` then ``calibrate`` for one eps; returns (margins, report)."""
    rep = train(eng, train_sets, eps, n_train, epochs, batch_pairs, lr, band_factor, seed)
    margins, crep = calibrate(eng, cal_seqs, eps, n_cal, q, band_factor, tune_scale, seed)
    rep.update(crep)
    return margins, rep


def projection_embeddings(features: np.ndarray, seed: int = 0, dim: int = 128) -> np.ndarray:
    """The method without the network: a fixed Gaussian random projection of
    the k-mer features (distances preserved up to scale, Johnson-Lindenstrauss)."""
    rng = np.random.default_rng(seed)
    R = rng.normal(0.0, 1.0 / math.sqrt(dim), size=(features.shape[1], dim))
    return (features.astype(np.float64) @ R).astype(np.float32)


def projection_scale(features: np.ndarray, a, b, d, lens, seed: int = 0) -> float:
    """Scale s of the projection fit by least squares on exact-scored pairs:
    s * ||P x_a - P x_b|| ~ d / (4 max(len_a, len_b)).  With it, the method
    without the network runs the same recipe (``calibrate`` with
    ``embeddings``) as the learned embedding."""
    P = projection_embeddings(features, seed)
    a, b = np.asarray(a), np.asarray(b)
    lens = np.asarray(lens)
    e = np.linalg.norm(P[a] - P[b], axis=1).astype(np.float64)
    t = np.asarray(d, dtype=np.float64) / (4.0 * np.maximum(np.maximum(lens[a], lens[b]), 1))
    return float((e * t).sum() / max((e * e).sum(), 1e-30))


def labels_from_split(split, n: int) -> np.ndarray:
    """Cluster label per point; points in no cluster (noise) get their own label."""
    lab = np.full(n, -1, dtype=np.int64)
    for c, members in enumerate(split):
        lab[np.asarray(members, dtype=np.int64)] = c
    noise = np.nonzero(lab < 0)[0]
    lab[noise] = len(split) + np.arange(len(noise))
    return lab


def adjusted_rand(x: np.ndarray, y: np.ndarray) -> float:
    """Adjusted Rand index of two labelings (Hubert & Arabie, 1985)."""
    x = np.asarray(x)
    y = np.asarray(y)
    n = len(x)
    if n < 2:
        return 1.0
    _, xi = np.unique(x, return_inverse=True)
    _, yi = np.unique(y, return_inverse=True)
    pairs = xi.astype(np.int64) * (yi.max() + 1) + yi
    _, nij = np.unique(pairs, return_counts=True)
    a = np.bincount(xi)
    b = np.bincount(yi)
    comb = lambda v: (v.astype(np.float64) * (v - 1) / 2.0).sum()
    sij, sa, sb = comb(nij), comb(a), comb(b)
    total = n * (n - 1) / 2.0
    expected = sa * sb / total
    mx = 0.5 * (sa + sb)
    if mx == expected:
        return 1.0
    return float((sij - expected) / (mx - expected))
