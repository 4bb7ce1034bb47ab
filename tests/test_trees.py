"""The split-set tree consumers (split_sets_to_newick.c, tree_pureness.c,
filter_split_sets_by_min.c, split_set_to_fasta.c over cluster_io.c and
volumes.c): the reference mains relinked on libswgpu, and this package's CLIs
of the same names, against the reference tools' outputs.  Host code only."""
from __future__ import annotations

import base64
import struct
import subprocess

import numpy as np
import pytest

import oracle as O
import swgpu
from conftest import load_golden
from swgpu import workloads as W


def _split_set_without_ids(raw: bytes) -> bytes:
    """A split-set file with every cluster id zeroed (store_split_set layout)."""
    n = struct.unpack_from("<i", raw, 9)[0]
    out = bytearray(raw)
    pos = 13
    for _ in range(n):
        m = struct.unpack_from("<i", raw, pos)[0]
        out[pos + 4:pos + 8] = b"\0\0\0\0"
        pos += 8 + 4 * m
    return bytes(out)


@pytest.mark.parametrize("build", ["reference_main", "cli"])
def test_tree_tools_match_reference(tmp_path, build):
    doc = load_golden("trees.json")
    src = load_golden(doc["source"])
    tools = sorted({r["tool"] for r in doc["runs"]})
    exe = {t: (O.REF_DIR / (t + "_on_swgpu") if build == "reference_main" else swgpu.BIN_DIR / t) for t in tools}
    if not all(p.exists() for p in exe.values()):
        pytest.skip("drop-in builds not present")
    W.write_fasta(tmp_path / "in.fa", [s.encode() for s in src["seqs"]])
    for ri in {r["source_run"] for r in doc["runs"]}:
        run = src["runs"][ri]
        for nm, b in run["files"].items():
            (tmp_path / f"r{ri}_{nm}").write_bytes(base64.b64decode(b))
        (tmp_path / f"r{ri}.log").write_text(run["stdout"])
    for run in doc["runs"]:
        for old in tmp_path.glob("out_*"):
            old.unlink()
        r = subprocess.run([str(exe[run["tool"]])] + run["args"], cwd=tmp_path, capture_output=True, timeout=120)
        assert r.returncode == 0, (run["tool"], r.stderr[-300:])
        assert r.stdout.decode("latin-1") == run["stdout"], (run["tool"], run["args"][:3])
        got = {p.name: p.read_bytes() for p in sorted(tmp_path.glob("out_*"))}
        want = {k: base64.b64decode(v) for k, v in run["files"].items()}
        if run["tool"] == "filter_split_sets_by_min":  # ids the reference leaves unset
            got = {k: _split_set_without_ids(v) for k, v in got.items()}
            want = {k: _split_set_without_ids(v) for k, v in want.items()}
        assert got == want, (run["tool"], run["args"][:3])


def _nested_layers(rng, n_points=400, n_layers=5):
    """Random layers of a sweep: layer 0 partitions most points into small
    clusters (the rest is noise), each next layer merges groups of the
    previous layer's clusters and absorbs some noise."""
    pts = rng.permutation(n_points)
    noise = set(pts[: n_points // 8].tolist())
    clusters = [list(c) for c in np.array_split(pts[n_points // 8:], 40)]
    layers = [clusters]
    for _ in range(n_layers - 1):
        prev = layers[-1]
        order = rng.permutation(len(prev))
        groups = np.array_split(order, max(1, len(prev) // int(rng.integers(2, 4))))
        nxt = []
        for g in groups:
            members = [m for k in g for m in prev[k]]
            take = [p for p in list(noise)[: int(rng.integers(0, 4))]]
            noise -= set(take)
            members += take
            rng.shuffle(members)
            nxt.append([int(m) for m in members])
        layers.append(nxt)
    return layers


@pytest.mark.parametrize("seed", [3, 4])
def test_tree_tools_on_random_nested_layers(tmp_path, seed):
    """split_sets_to_newick and tree_pureness on random nested layers (a
    target that splits clusters, and one whose clusters overlap and repeat
    members): the reference tools, the reference mains relinked on
    libswgpu.so and this package's CLIs print the same text."""
    names = ["split_sets_to_newick", "tree_pureness"]
    exe = {}
    for t in names:
        exe[("ref", t)] = O.REF_DIR / t
        exe[("dropin", t)] = O.REF_DIR / (t + "_on_swgpu")
        exe[("cli", t)] = swgpu.BIN_DIR / t
    if not all(p.exists() for p in exe.values()):
        pytest.skip("reference tree tools or drop-in builds not present")
    import numpy as np
    rng = np.random.default_rng(seed)
    layers = _nested_layers(rng)
    files = []
    for i, layer in enumerate(layers):
        (tmp_path / f"lay{i:04d}").write_bytes(O.split_set_bytes(layer))
        files.append(f"lay{i:04d}")
    near = [list(c) for c in layers[2]]  # layer 2 with a tenth of its points moved to another cluster
    for c in near:
        for _ in range(len(c) // 10):
            dst = near[int(rng.integers(0, len(near)))]
            if dst is not c and c:
                dst.append(c.pop(int(rng.integers(0, len(c)))))
    targets = {
        "t_near": near,
        "t_split": [list(c) for c in np.array_split(rng.permutation(400), 23)],
        "t_overlap": [list(rng.choice(400, size=30, replace=True)) for _ in range(15)],
    }
    for nm, t in targets.items():
        (tmp_path / nm).write_bytes(O.split_set_bytes([[int(x) for x in c] for c in t]))
    W.write_fasta(tmp_path / "in.fa", [b"ACGT" * 5] * 400)
    runs = [("split_sets_to_newick", ["0", "0"] + files), ("split_sets_to_newick", ["3", "0"] + files)]
    runs += [("tree_pureness", ["in.fa", nm] + files) for nm in targets]
    for tool, args in runs:
        outs = {}
        for kind in ("ref", "dropin", "cli"):
            r = subprocess.run([str(exe[(kind, tool)])] + args, cwd=tmp_path, capture_output=True, timeout=120)
            assert r.returncode == 0, (kind, tool, r.stderr[-300:])
            outs[kind] = r.stdout
        assert outs["ref"] and outs["dropin"] == outs["ref"] and outs["cli"] == outs["ref"], (tool, args[:2])
