"""The tile-plan autotuner (swe_autotune): the plan it picks gives the same
distance matrix as the default plan, bit for bit, and is no slower than it
on the full data set; a second engine reads the plan from the cache file
without timing anything."""
from __future__ import annotations

import numpy as np
import pytest

import swgpu
from swgpu import workloads as W

pytestmark = pytest.mark.gpu


def _kernel_ms(eng, reps=3):
    ms = []
    for _ in range(reps):
        eng.score_all_pairs()
        ms.append(eng.stats()["ms_fast_kernel"])
    return min(ms)


def test_autotuned_plan_is_exact_no_slower_and_cached(tmp_path):
    seqs, _ = W.config2(n=6000, n_fam=60)
    cache = str(tmp_path / "plans.txt")
    e0 = swgpu.Engine()
    e0.upload(seqs)
    t0 = _kernel_ms(e0)
    D0 = e0.distances()
    e0.close()

    e1 = swgpu.Engine()
    res = e1.autotune(seqs, cache_path=cache)
    assert res["from_cache"] == 0 and res["candidates"] >= 12 and res["sample"] == 4096
    assert res["ms_best"] <= res["ms_default"]
    e1.upload(seqs)
    t1 = _kernel_ms(e1)
    assert np.array_equal(e1.distances(), D0)
    assert t1 <= 1.05 * t0, (res, t0, t1)
    e1.close()

    e2 = swgpu.Engine()
    e2.upload(seqs)  # a held upload is laid out again with the cached plan
    r2 = e2.autotune(seqs, cache_path=cache)
    assert r2["from_cache"] == 1 and r2["candidates"] == 0 and r2["key"] == res["key"]
    assert (r2["packs_per_block"], r2["threads"], r2["max_w"]) == (res["packs_per_block"], res["threads"],
                                                                   res["max_w"])
    e2.score_all_pairs()
    assert np.array_equal(e2.distances(), D0)
    e2.close()


def test_every_candidate_plan_gives_the_same_matrix_on_mixed_lengths():
    """Each knob of the search space on sequences of 1 .. 768 symbols (every
    lane split), against the default plan."""
    rng = np.random.default_rng(4)
    seqs = [W.BASES[rng.integers(0, 4, size=int(L))].tobytes() for L in rng.integers(1, 769, size=700)]
    e = swgpu.Engine()
    e.upload(seqs)
    e.score_all_pairs()
    D = e.distances()
    e.close()
    for pb, th, w in [(16, 128, 16), (64, 256, 20), (16, 256, 24), (64, 128, 16)]:
        e = swgpu.Engine(packs_per_block=pb, threads=th, max_w=w)
        e.upload(seqs)
        e.score_all_pairs()
        assert np.array_equal(e.distances(), D), (pb, th, w)
        e.close()
