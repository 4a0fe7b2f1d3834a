"""Shared test setup: import paths, the `gpu` marker, golden-fixture loading and tolerances."""
import glob
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")

# Parity bars.  emp4/emp5 totals: 1e-11 relative (the FP64 target of the plain and fused GPU forms).
# Per-triple records are compared normwise per column: the reference itself (threaded OpenBLAS, OpenMP
# reduction order) only fixes them to ~1e-14 relative.
TOTAL_RTOL = 1e-11
RECORD_RTOL = 1e-11


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


def golden_cases():
    return sorted(os.path.basename(p)[:-5] for p in glob.glob(os.path.join(GOLDEN, "g_*.json")))


def load_golden(name):
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        return json.load(f)


def system_from_golden(g):
    import trpdrv_b200 as T
    s = T.synth_system(g["nocc"], g["nvir"], seed=g["seed"], ncor=g["ncor"], dist=g["dist"], a=g["a"])
    for n, (s1, s2) in g["checksums"].items():
        a = s.arrays[n]
        assert float(np.sum(a)) == s1 and float(np.sum(a * a)) == s2, f"generator drift in {n}"
    return s


def assert_records_close(got, want, rtol=RECORD_RTOL):
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    assert got.shape == want.shape
    for c in range(want.shape[1]):
        scale = np.max(np.abs(want[:, c])) + 1e-300
        err = np.max(np.abs(got[:, c] - want[:, c]))
        assert err <= rtol * scale, f"column {c}: max abs err {err:.3e} > {rtol:.0e} * {scale:.3e}"


def assert_total_close(got, want, rtol=TOTAL_RTOL, what="total"):
    err = abs(got - want)
    assert err <= rtol * abs(want), f"{what}: {got!r} vs {want!r} (rel {err / abs(want):.3e} > {rtol:.0e})"


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def T():
    import trpdrv_b200
    return trpdrv_b200


@pytest.fixture(scope="session")
def O():
    import oracle
    return oracle
