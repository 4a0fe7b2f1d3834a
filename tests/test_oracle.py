"""The oracle (CPU restatement) pinned against the reference itself: golden vectors produced by the
reference's own body/tengy compiled unmodified (tests/golden/make_golden.py) and the reference
driver's known-answer print.  CPU only."""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, assert_records_close, assert_total_close, golden_cases, load_golden, system_from_golden
from kat import run_make_array_loop


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_port_matches_reference_golden(name, O):
    g = load_golden(name)
    s = system_from_golden(g)
    rec, tot, mism = O.run_system(s, "port", nkpass=g["nkpass"], nthreads=2)
    assert mism == 0
    assert rec.shape == (len(g["records"]), 4)
    ijk = O.enumerate_triples(g["nocc"], g["nkpass"])[:, :3]
    assert np.array_equal(ijk, np.array(g["triples"], dtype=np.int32))
    assert_records_close(rec, g["records"], rtol=1e-12)
    assert_total_close(tot[0], g["emp4"], rtol=1e-12, what="emp4")
    assert_total_close(tot[1], g["emp5"], rtol=1e-12, what="emp5")


def test_oracle_port_make_array_kat(O):
    with open(os.path.join(GOLDEN, "kat_test_c99_10_60.json")) as f:
        kat = json.load(f)
    line, calls = run_make_array_loop(O.port_body_fn(), 10, 60)
    assert calls == 550
    assert line == kat["line"] == "emp4=2.647247 emp5=-1.560018"


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "test_c99")),
                    reason="reference driver not built")
def test_reference_driver_kat(O):
    out = subprocess.run([O.REF_TEST, "10", "60", "100000"], capture_output=True, text=True, check=True,
                         env=dict(os.environ, OMP_NUM_THREADS="2", OPENBLAS_NUM_THREADS="1"))
    assert "emp4=2.647247 emp5=-1.560018" in out.stdout
    assert "SUCCESS" in out.stdout


@pytest.mark.parametrize("nkpass", [1, 3])
def test_oracle_nkpass_order_invariance(O, T, nkpass):
    s = T.synth_system(7, 20, seed=3)
    _, t1, _ = O.run_system(s, "port", nkpass=1)
    _, tn, _ = O.run_system(s, "port", nkpass=nkpass)
    assert_total_close(tn[0], t1[0], rtol=1e-13)
    assert_total_close(tn[1], t1[1], rtol=1e-13)


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T")])
def test_oracle_dgemm_against_numpy(O, ta, tb):
    rng = np.random.default_rng(5)
    m, n, k = 13, 17, 11
    A = np.asfortranarray(rng.standard_normal((m, k) if ta == "N" else (k, m)))
    B = np.asfortranarray(rng.standard_normal((k, n) if tb == "N" else (n, k)))
    Cm = np.asfortranarray(rng.standard_normal((m, n)))
    want = -1.0 * ((A if ta == "N" else A.T) @ (B if tb == "N" else B.T)) + 1.0 * Cm
    O.dgemm(ta, tb, -1.0, A, B, 1.0, Cm)
    np.testing.assert_allclose(Cm, want, rtol=1e-13, atol=1e-13)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref",
                                                    "libtrpdrv_ref.so")), reason="reference not built")
def test_oracle_tengy_matches_reference_tengy(O):
    rng = np.random.default_rng(9)
    ncor, nocc, nvir = 1, 3, 45
    f8 = rng.uniform(-1, 1, (8, nvir * nvir))
    vecs = [rng.uniform(-0.1, 0.1, nvir) for _ in range(6)]
    eorb = np.sort(rng.uniform(-2, 3, ncor + nocc + nvir))
    eorb[ncor + nocc:] = np.sort(rng.uniform(0.2, 3, nvir))
    got = O.tengy(f8, vecs, eorb, 2.5, ncor, nocc, nvir, which="port")
    want = O.tengy(f8, vecs, eorb, 2.5, ncor, nocc, nvir, which="reference")
    np.testing.assert_allclose(got, want, rtol=1e-13)


@pytest.mark.parametrize("shape", [(5, 33, 13, 2, 0, 0), (4, 30, 14, 0, 1, 0), (6, 40, 3, 0, 0, 2), (7, 21, 99, 1, 1, 3)])
def test_oracle_generator_restatement_equals_the_product_generator(O, T, shape):
    """oracle.synth_system (used by the benchmark's reference arm and the full-size fixtures) gives
    bit-identical tensors to the product's trpdrv_synth_fill, for every tensor and distribution."""
    nocc, nvir, seed, ncor, dist, a_block = shape
    so = O.synth_system(nocc, nvir, seed=seed, ncor=ncor, dist=dist, a_block=a_block)
    sp = T.synth_system(nocc, nvir, seed=seed, ncor=ncor, dist=dist, a_block=a_block)
    assert so.a == sp.a
    for name in O.TENSOR_NAMES:
        assert np.array_equal(so.arrays[name], sp.arrays[name]), name


def test_oracle_generator_matches_the_full_size_fixture_checksums(O):
    """The full-size fixtures record input checksums; the restated generator reproduces them (C2 is
    checked tensor by tensor on its 1.5 GB of inputs)."""
    path = os.path.join(GOLDEN, "big_c2_o40_v300.json")
    if not os.path.exists(path):
        pytest.skip("full-size fixture not generated")
    with open(path) as f:
        g = json.load(f)["systems"][0]
    s = O.synth_system(g["nocc"], g["nvir"], seed=g["seed"], dist=g["dist"], a=g["a"])
    for n, (s1, s2) in g["checksums"].items():
        a = s.arrays[n]
        assert float(np.sum(a)) == s1 and float(np.sum(a * a)) == s2, n


@pytest.mark.parametrize("which", ["port", "reference"])
def test_oracle_timed_loop_accumulates_like_the_driver(O, which):
    """oracle.time_body (the CPU baseline's loop: body calls only, the body accumulating emp4/emp5)
    gives the totals of the recorded run, split over two calls."""
    if which == "reference" and not O.have_reference():
        pytest.skip("reference not built")
    s = O.synth_system(5, 26, seed=21)
    n = O.count_triples(5)
    _, tot, _ = O.run_system(s, "port", nthreads=2)
    e4, e5 = O.time_body(s, which, t_begin=0, t_end=n // 3)
    e4, e5 = O.time_body(s, which, t_begin=n // 3, t_end=n, emp4=e4, emp5=e5)
    assert abs(e4 - tot[0]) <= 1e-12 * abs(tot[0]) and abs(e5 - tot[1]) <= 1e-12 * abs(tot[1])


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref", "test_fp32")),
                    reason="reference single-precision driver not built")
def test_reference_fp32_driver_kat(O):
    """The reference's single-precision variant (gpu-omp/test.c + gpu-omp/ccsd_trpdrv_omp_cbody.c, host
    build) reproduces its recorded known answers (one OpenMP/OpenBLAS thread: its float sums run in a
    fixed order)."""
    with open(os.path.join(GOLDEN, "kat_test_fp32_10_60.json")) as f:
        runs = json.load(f)["runs"]
    exe = os.path.join(os.path.dirname(O.REF_TEST), "test_fp32")
    for run in runs:
        out = subprocess.run([exe, *run["argv"]], capture_output=True, text=True, check=True,
                             env=dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1"))
        assert run["line"] in out.stdout and "SUCCESS" in out.stdout
