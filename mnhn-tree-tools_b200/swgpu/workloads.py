"""Seeded synthetic DNA workloads for the all-pairs Smith-Waterman engine.

There is no public benchmark for this path; each generator below produces a
dataset with the shapes and value distributions of one benchmark
configuration, from a fixed numpy PRNG seed so every run sees the same bytes.

* ``config1`` - 2,000 reads: 20 random ACGT roots of 250 bp, 100 descendants
  each, per-descendant substitution rate U(1%, 10%), indels at 1% per position
  with geometric lengths of mean 2.
* ``config2`` - 20,000 reads: 200 families from random roots, lognormal
  lengths (median 220) clipped to 100-600 bp, substitutions U(2%, 15%), indels
  U(1%, 3%), about 2% of positions in 'N' masking runs.
* ``config3`` - 100,000 satellite-like reads: 50 tandem-repeat monomer
  families of 171 bp; a read is a window of 150-342 bp from two monomer copies,
  substituted at U(2%, 15%), half of them reverse-complemented.
* ``config5`` - 500 independent sets, sizes log-uniform in [50, 5000], each
  drawn with the config-1 generator and 2-20 families.
"""
from __future__ import annotations

import numpy as np

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)
COMP = np.zeros(256, dtype=np.uint8)
for _a, _b in zip(b"ACGTN", b"TGCAN"):
    COMP[_a] = _b


def _random_seq(rng, n):
    return BASES[rng.integers(0, 4, size=n)]


def _mutate(rng, root, sub_rate, indel_rate, indel_mean=2.0):
    """Substitute each position with prob sub_rate (to a different base), then
    apply indels at indel_rate per position (insert or delete, 50/50), with
    geometric lengths of the given mean."""
    s = root.copy()
    n = len(s)
    m = rng.random(n) < sub_rate
    if m.any():
        shift = rng.integers(1, 4, size=int(m.sum()))
        idx = np.searchsorted(BASES, s[m])
        s[m] = BASES[(idx + shift) % 4]
    if indel_rate <= 0:
        return s
    ev = np.nonzero(rng.random(n) < indel_rate)[0]
    if len(ev) == 0:
        return s
    out = []
    pos = 0
    p = 1.0 / indel_mean
    for e in ev:
        if e < pos:
            continue
        out.append(s[pos:e])
        ln = int(rng.geometric(p))
        if rng.random() < 0.5:  # insertion before position e
            out.append(_random_seq(rng, ln))
            pos = e
        else:  # deletion of ln bases starting at e
            pos = min(n, e + ln)
    out.append(s[pos:])
    return np.concatenate(out) if out else s


def _to_bytes(arrs):
    return [a.tobytes() for a in arrs]


def config1(seed: int = 1, n_roots: int = 20, per_root: int = 100, root_len: int = 250):
    rng = np.random.default_rng(seed)
    roots = [_random_seq(rng, root_len) for _ in range(n_roots)]
    seqs, fam = [], []
    for f, r in enumerate(roots):
        for _ in range(per_root):
            seqs.append(_mutate(rng, r, rng.uniform(0.01, 0.10), 0.01))
            fam.append(f)
    return _to_bytes(seqs), np.asarray(fam)


def config2(seed: int = 2, n: int = 20000, n_fam: int = 200, n_frac: float = 0.02,
            min_len: int = 100, max_len: int = 600, median: float = 220.0, sigma: float = 0.45):
    rng = np.random.default_rng(seed)
    root_len = np.clip(np.round(np.exp(rng.normal(np.log(median), sigma, size=n_fam))),
                       min_len, max_len).astype(int)
    roots = [_random_seq(rng, L) for L in root_len]
    fam = rng.integers(0, n_fam, size=n)
    seqs = []
    for f in fam:
        s = _mutate(rng, roots[f], rng.uniform(0.02, 0.15), rng.uniform(0.01, 0.03))
        if len(s) > max_len:
            s = s[:max_len]
        if len(s) < min_len:
            s = np.concatenate([s, _random_seq(rng, min_len - len(s))])
        # 'N' masking runs covering about n_frac of the positions (mean run 10)
        L = len(s)
        n_runs = rng.poisson(n_frac * L / 10.0)
        for _ in range(n_runs):
            ln = int(rng.geometric(0.1))
            st = int(rng.integers(0, L))
            s[st:st + ln] = ord("N")
        seqs.append(s)
    return _to_bytes(seqs), fam


def config3(seed: int = 3, n: int = 100000, n_fam: int = 50, mono: int = 171,
            min_len: int = 150, max_len: int = 342, with_rc: bool = False):
    """Returns (reads, family of each read), plus with_rc a boolean array
    marking the reverse-complemented reads."""
    rng = np.random.default_rng(seed)
    monos = [_random_seq(rng, mono) for _ in range(n_fam)]
    fam = rng.integers(0, n_fam, size=n)
    seqs = []
    rc = np.zeros(n, dtype=bool)
    for k, f in enumerate(fam):
        arr = np.concatenate([monos[f], monos[f]])
        L = int(rng.integers(min_len, max_len + 1))
        st = int(rng.integers(0, 2 * mono - L + 1))
        s = arr[st:st + L].copy()
        s = _mutate(rng, s, rng.uniform(0.02, 0.15), 0.0)
        if rng.random() < 0.5:
            s = COMP[s[::-1]]
            rc[k] = True
        seqs.append(s)
    if with_rc:
        return _to_bytes(seqs), fam, rc
    return _to_bytes(seqs), fam


def config5(seed: int = 5, n_sets: int = 500, lo: int = 50, hi: int = 5000, root_len: int = 250):
    """Returns (list of per-set sequence lists, list of per-set family labels)."""
    rng = np.random.default_rng(seed)
    sizes = np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), size=n_sets))).astype(int)
    sets, fams = [], []
    for sz in sizes:
        nf = int(rng.integers(2, 21))
        roots = [_random_seq(rng, root_len) for _ in range(nf)]
        fam = rng.integers(0, nf, size=sz)
        sets.append(_to_bytes([_mutate(rng, roots[f], rng.uniform(0.01, 0.10), 0.01) for f in fam]))
        fams.append(fam)
    return sets, fams


def cells(seqs) -> int:
    """Unique-pair DP cells: sum over i<j of len_i * len_j."""
    L = np.array([len(s) for s in seqs], dtype=np.float64)
    tot = L.sum()
    return int(round((tot * tot - (L * L).sum()) / 2))


def write_fasta(path, seqs, width: int = 60) -> None:
    with open(path, "w") as f:
        for i, s in enumerate(seqs):
            f.write(">seq_%d\n" % i)
            t = s.decode("latin-1")
            for k in range(0, len(t), width):
                f.write(t[k:k + width] + "\n")
