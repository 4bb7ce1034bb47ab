"""Shared test setup.

* ``-m "not gpu"`` tests run on any machine: the oracle against the golden
  vectors produced by the reference itself, the host logic of libswgpu.so
  (loader, split-set formats, DBSCAN replay, adaptive driver) and the C ABI's
  exports.  They never launch a kernel.
* ``-m gpu`` tests need a CUDA device and compare the GPU engine with the
  golden vectors and the oracle.
"""
from __future__ import annotations

import gzip
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "mnhn-tree-tools_b200"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: long-running check")


def _ensure_built():
    import oracle as O
    import swgpu
    if not (ROOT / "oracle" / "liboracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    if os.path.isdir(O.reference_dir()) and not O.ref_available():
        O.build()
    swgpu.build()


@pytest.fixture(scope="session", autouse=True)
def built():
    _ensure_built()


def load_golden(name: str):
    p = GOLDEN / name
    if name.endswith(".gz"):
        with gzip.open(p, "rt") as f:
            return json.load(f)
    return json.loads(p.read_text())


@pytest.fixture(scope="session")
def golden():
    return load_golden


def fasta2kmer_input(doc, name: str) -> list[bytes]:
    """Sequences of one input of tests/golden/fasta2kmer.json: literal
    strings, or {"unit": u, "length": n} for u repeated to n symbols (the rule
    of make_golden.kmer_inputs)."""
    out = []
    for x in doc["inputs"][name]:
        if isinstance(x, str):
            out.append(x.encode("latin-1"))
        else:
            u = x["unit"]
            out.append((u * (x["length"] // len(u) + 1))[:x["length"]].encode("latin-1"))
    return out


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
