"""GPU tests of the FP32 parity form (libtrpdrv_b200_fp32.so), the single-precision variant of the
reference (gpu-omp/).

  * the reference's UNMODIFIED single-precision driver gpu-omp/test.c, linked against the library,
    prints the known answers of the reference variant built on the host (oracle/_ref/test_fp32) to
    within FP32 rounding: |difference| <= 2e-5 (the prints are around 0.1..6, six decimals);
  * per triple, the library's float energies agree with the reference's float body
    (oracle/_ref/libtrpdrv_ref_fp32.so, OpenBLAS sgemm) within 2e-4 of the largest |emp| of the
    sample, and with the FP64 oracle within the same bar, on inputs rounded to float;
  * the float tengy entry point against the reference's float ccsd_tengy_omp.
"""
import ctypes as C
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

LIB_FP32 = os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200", "lib", "libtrpdrv_b200_fp32.so")
REF_FP32 = os.path.join(ROOT, "oracle", "_ref", "libtrpdrv_ref_fp32.so")
KAT_TOL = 2e-5
TRIPLE_TOL = 2e-4

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


def _body(lib):
    fn = lib.ccsd_trpdrv_omp_cbody_
    fn.argtypes = [_fp] * 9 + [_ip] * 3 + [_fp] * 2 + [_ip] * 5 + [_fp] * 20
    fn.restype = None
    return fn


def _call(fn, T, s32, i, j, k, klo):
    """One float body call on the float32 copy of a system; returns the (emp4, emp5) increments."""
    sl = T.triple_slices(s32, i, j, k, klo)
    V = s32.nvir
    f = np.zeros((8, V * V), dtype=np.float32)
    fp = [f[q].ctypes.data_as(_fp) for q in range(8)]
    ints = [C.c_int(v) for v in (s32.ncor, s32.nocc, s32.nvir)]
    idx = [C.c_int(v) for v in (s32.a, i, j, k, klo)]
    e4, e5 = C.c_float(0.0), C.c_float(0.0)
    fn(*fp, sl["eorb"].ctypes.data_as(_fp), *[C.byref(v) for v in ints], C.byref(e4), C.byref(e5),
       *[C.byref(v) for v in idx], *[sl[n].ctypes.data_as(_fp) for n in T.BODY_ORDER])
    return e4.value, e5.value


def _float_system(T, nocc, nvir, seed):
    s = T.synth_system(nocc, nvir, seed=seed)
    s32 = T.System(s.ncor, s.nocc, s.nvir, s.a, {n: a.astype(np.float32) for n, a in s.arrays.items()})
    s64 = T.System(s.ncor, s.nocc, s.nvir, s.a, {n: a.astype(np.float64) for n, a in s32.arrays.items()})
    return s32, s64


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "test_fp32_b200")),
                    reason="single-precision driver not linked")
def test_unmodified_fp32_reference_driver_on_the_library():
    with open(os.path.join(GOLDEN, "kat_test_fp32_10_60.json")) as f:
        runs = json.load(f)["runs"]
    exe = os.path.join(ROOT, "oracle", "_ref", "test_fp32_b200")
    for run in runs:
        out = subprocess.run([exe, *run["argv"]], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        got = re.search(r"emp4=(\S+) emp5=(\S+)", out.stdout)
        want = re.search(r"emp4=(\S+) emp5=(\S+)", run["line"])
        for g, w in zip(got.groups(), want.groups()):
            assert abs(float(g) - float(w)) <= KAT_TOL, (run["argv"], out.stdout[-200:], run["line"])


@pytest.mark.skipif(not os.path.exists(REF_FP32), reason="reference single-precision body not built")
@pytest.mark.parametrize("shape", [(6, 48, 5), (5, 37, 6), (8, 96, 7)])
def test_fp32_body_against_the_reference_fp32_body_and_the_fp64_oracle(T, O, shape):
    nocc, nvir, seed = shape
    s32, s64 = _float_system(T, nocc, nvir, seed)
    ours, theirs = _body(C.CDLL(LIB_FP32)), _body(C.CDLL(REF_FP32))
    fn64 = O.port_body_fn()
    ijkl = T.enumerate_triples(nocc, 2)
    got, ref, exact = [], [], []
    for t in range(0, len(ijkl), 7):
        i, j, k, klo = (int(v) for v in ijkl[t])
        got.append(_call(ours, T, s32, i, j, k, klo))
        ref.append(_call(theirs, T, s32, i, j, k, klo))
        exact.append(T.body_call(fn64, s64, i, j, k, klo))
    got, ref, exact = np.array(got), np.array(ref), np.array(exact)
    for c in range(2):
        scale = np.max(np.abs(exact[:, c]))
        assert np.max(np.abs(got[:, c] - ref[:, c])) <= TRIPLE_TOL * scale
        assert np.max(np.abs(got[:, c] - exact[:, c])) <= TRIPLE_TOL * scale


@pytest.mark.skipif(not os.path.exists(REF_FP32), reason="reference single-precision body not built")
def test_fp32_tengy_against_the_reference_fp32_tengy():
    rng = np.random.default_rng(43)
    ncor, nocc, nvir = 1, 4, 70
    f8 = rng.uniform(-0.5, 0.5, (8, nvir * nvir)).astype(np.float32)
    vecs = [rng.uniform(-0.1, 0.1, nvir).astype(np.float32) for _ in range(6)]
    eorb = np.concatenate([np.sort(rng.uniform(-20, -5, ncor)), np.sort(rng.uniform(-2, -0.5, nocc)),
                           np.sort(rng.uniform(0.2, 3.0, nvir))]).astype(np.float32)
    outs = []
    for path in (LIB_FP32, REF_FP32):
        fn = C.CDLL(path).ccsd_tengy_omp
        fn.argtypes = [_fp] * 15 + [C.c_float] + [_fp] * 4 + [C.c_int] * 3
        fn.restype = None
        o = [C.c_float() for _ in range(4)]
        fn(*[f8[q].ctypes.data_as(_fp) for q in range(8)], *[v.ctypes.data_as(_fp) for v in vecs],
           eorb.ctypes.data_as(_fp), 1.7, *[C.byref(x) for x in o], ncor, nocc, nvir)
        outs.append([x.value for x in o])
    got, want = np.array(outs[0]), np.array(outs[1])
    assert np.all(np.abs(got - want) <= TRIPLE_TOL * np.max(np.abs(want)))
