"""GPU parity at the full benchmark sizes, against fixtures the reference itself produced
(tests/golden/make_golden_large.py: every triple of one `a` through the reference body compiled
unmodified).

  big_c2_o40_v300      nocc=40, nvir=300, 32,800 triples (the headline workload)
  big_c3_o30_v400_log  nocc=30, nvir=400, log-uniform integral magnitudes in [1e-6, 1], 13,950 triples
  big_c4_six           six systems (8,80) .. (40,450) in one plan, 60,296 triples

Bars: totals within 1e-11 relative (TOTAL_RTOL), records (every 13th triple, or every triple of the
small systems) within 1e-11 normwise per column (RECORD_RTOL), for the fused FP64 kernel, the plain
per-triple path and the emulated form at its default 7 digit slices (and 8).  The emulated form's
error against the reference is printed per slice count (pytest -s shows it).
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, RECORD_RTOL, TOTAL_RTOL, assert_records_close, assert_total_close

pytestmark = pytest.mark.gpu


def _load(name):
    path = os.path.join(GOLDEN, name + ".json")
    if not os.path.exists(path):
        pytest.skip(f"{name}.json not generated")
    with open(path) as f:
        return json.load(f)


def _system(T, g):
    s = T.synth_system(g["nocc"], g["nvir"], seed=g["seed"], ncor=g["ncor"], dist=g["dist"], a=g["a"])
    for n, (s1, s2) in g["checksums"].items():
        a = s.arrays[n]
        assert float(np.sum(a)) == s1 and float(np.sum(a * a)) == s2, f"generator drift in {n}"
    return s


def _run(T, systems, **opt):
    with T.Plan(systems, device=0, **opt) as p:
        p.upload()
        p.execute()
        e4, e5 = p.energies()
        recs = [p.triple_energies(q) for q in range(len(systems))]
        staging = p.staging()
    return e4, e5, recs, staging


def _check(g, e4, e5, rec, rtol_tot=TOTAL_RTOL, rtol_rec=RECORD_RTOL, what=""):
    assert len(rec) == g["triples_total"]
    assert_total_close(e4, g["emp4"], rtol=rtol_tot, what=f"{what} emp4")
    assert_total_close(e5, g["emp5"], rtol=rtol_tot, what=f"{what} emp5")
    assert_records_close(np.asarray(rec)[g["record_index"]], g["records"], rtol=rtol_rec)


def _rel(e, want):
    return abs(e - want) / abs(want)


@pytest.mark.parametrize("mode", ["fused", "plain"])
def test_c2_fp64_matches_the_reference_on_every_triple(T, mode):
    g = _load("big_c2_o40_v300")["systems"][0]
    s = _system(T, g)
    e4, e5, recs, staging = _run(T, [s], mode=T.MODE_FUSED if mode == "fused" else T.MODE_PLAIN)
    if mode == "fused":
        assert staging == 2  # the TMA kernel the benchmark times
    _check(g, e4[0], e5[0], recs[0], what=f"c2 {mode}")


@pytest.mark.parametrize("slices", [7, 8])
def test_c2_emulated_matches_the_reference(T, slices):
    g = _load("big_c2_o40_v300")["systems"][0]
    s = _system(T, g)
    e4, e5, recs, _ = _run(T, [s], mode=T.MODE_EMULATED, slices=slices)
    print(f"c2 emulated {slices} slices vs reference: emp4 {_rel(e4[0], g['emp4']):.2e} "
          f"emp5 {_rel(e5[0], g['emp5']):.2e}")
    _check(g, e4[0], e5[0], recs[0], what=f"c2 emulated {slices}")


def test_c2_emulated_with_fused_energies_equals_the_separate_launch(T, monkeypatch):
    """The energies inside the contraction launch (the default) agree with the separate launch's
    (TRPDRV_OZ_FUSED_ENERGY=0) to 1e-13 (the kernels may contract multiplies and adds differently) and
    with the reference at the usual bars."""
    g = _load("big_c2_o40_v300")["systems"][0]
    s = _system(T, g)
    monkeypatch.setenv("TRPDRV_OZ_FUSED_ENERGY", "0")
    e4, e5, recs, _ = _run(T, [s], mode=T.MODE_EMULATED, slices=7)
    monkeypatch.delenv("TRPDRV_OZ_FUSED_ENERGY")
    e4f, e5f, recf, _ = _run(T, [s], mode=T.MODE_EMULATED, slices=7)
    assert_records_close(np.asarray(recf[0]), np.asarray(recs[0]), rtol=1e-13)
    assert_total_close(e4f[0], e4[0], rtol=1e-13, what="emp4 vs separate launch")
    assert_total_close(e5f[0], e5[0], rtol=1e-13, what="emp5 vs separate launch")
    _check(g, e4f[0], e5f[0], recf[0], what="c2 emulated fused energies")


@pytest.mark.parametrize("mode", ["fused", "plain"])
def test_c3_fp64_matches_the_reference_on_every_triple(T, mode):
    g = _load("big_c3_o30_v400_log")["systems"][0]
    s = _system(T, g)
    e4, e5, recs, _ = _run(T, [s], mode=T.MODE_FUSED if mode == "fused" else T.MODE_PLAIN)
    _check(g, e4[0], e5[0], recs[0], what=f"c3 {mode}")


def test_c3_emulated_error_against_the_reference_per_slice_count(T):
    """Log-uniform integrals (the splitting stress case): 7 and 8 slices meet the 1e-11 bar against the
    reference; the error falls with every added slice from 5 to 8."""
    g = _load("big_c3_o30_v400_log")["systems"][0]
    s = _system(T, g)
    errs = {}
    for sl in (5, 6, 7, 8):
        e4, e5, recs, _ = _run(T, [s], mode=T.MODE_EMULATED, slices=sl)
        errs[sl] = max(_rel(e4[0], g["emp4"]), _rel(e5[0], g["emp5"]))
        print(f"c3 emulated {sl} slices vs reference: emp4 {_rel(e4[0], g['emp4']):.2e} "
              f"emp5 {_rel(e5[0], g['emp5']):.2e}")
        if sl >= 7:
            _check(g, e4[0], e5[0], recs[0], what=f"c3 emulated {sl}")
    assert errs[5] > errs[6] > errs[7] >= 0.0
    assert errs[8] <= TOTAL_RTOL


def test_c3_emulated_accuracy_target_picks_slices_that_meet_it(T):
    g = _load("big_c3_o30_v400_log")["systems"][0]
    s = _system(T, g)
    with T.Plan([s], device=0, mode=T.MODE_EMULATED, target_digits=11) as p:
        p.upload()
        tune = p.autotune()
        p.execute()
        e4, e5 = p.energies()
        rec = p.triple_energies(0)
    assert 4 <= tune["slices"] <= 8
    _check(g, e4[0], e5[0], rec, what=f"c3 target 1e-11 ({tune['slices']} slices)")


@pytest.mark.parametrize("mode", ["fused", "plain", "emulated"])
def test_c4_six_systems_in_one_plan_match_the_reference(T, mode):
    doc = _load("big_c4_six")
    gs = doc["systems"]
    systems = [_system(T, g) for g in gs]
    opt = {"fused": dict(mode=T.MODE_FUSED), "plain": dict(mode=T.MODE_PLAIN),
           "emulated": dict(mode=T.MODE_EMULATED, slices=7)}[mode]
    e4, e5, recs, _ = _run(T, systems, **opt)
    for q, g in enumerate(gs):
        _check(g, e4[q], e5[q], recs[q], what=f"c4 {mode} system ({g['nocc']},{g['nvir']})")
