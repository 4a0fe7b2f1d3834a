"""GPU parity of the emulated-FP64 form (TRPDRV_MODE_EMULATED: Ozaki int8 digit slices on the
tcgen05 tensor cores, exact int32 sums, FP64 recombination and FP64 energies) against the reference's
golden vectors and the native FP64 paths.

Bars: with 7 or 8 slices the emulated form meets the native bars (emp4/emp5 totals within 1e-11
relative, per-triple records within 1e-11 normwise per column); fewer slices give errors that fall
by about 2^-7 per slice, which the sweep checks and reports.
"""
import numpy as np
import pytest

from conftest import (RECORD_RTOL, TOTAL_RTOL, assert_records_close, assert_total_close, golden_cases, load_golden,
                      system_from_golden)

pytestmark = pytest.mark.gpu


def _run(T, systems, mode=None, **opt):
    with T.Plan(systems, mode=T.MODE_EMULATED if mode is None else mode, **opt) as p:
        p.upload()
        p.execute()
        e4, e5 = p.energies()
        recs = [p.triple_energies(q) for q in range(len(systems))]
        launches = p.last_launches()
    return e4, e5, recs, launches


@pytest.mark.parametrize("slices", [7, 8])
@pytest.mark.parametrize("name", golden_cases())
def test_emulated_matches_reference_golden(T, name, slices):
    g = load_golden(name)
    s = system_from_golden(g)
    e4, e5, recs, launches = _run(T, [s], nkpass=g["nkpass"], slices=slices)
    assert launches > 0
    assert_records_close(recs[0], g["records"])
    assert_total_close(e4[0], g["emp4"], what="emp4")
    assert_total_close(e5[0], g["emp5"], what="emp5")


@pytest.mark.parametrize("name", ["g_o10_v60", "g_o4_v30_log"])
def test_emulated_error_falls_with_slices(T, name):
    g = load_golden(name)
    s = system_from_golden(g)
    ref = np.asarray(g["records"], dtype=np.float64)
    errs = []
    for sl in range(4, 9):
        _, _, recs, _ = _run(T, [s], nkpass=g["nkpass"], slices=sl)
        errs.append(float(np.max(np.abs(recs[0] - ref)) / np.max(np.abs(ref))))
    print(name, ["%.2e" % e for e in errs])
    floor = 1e-14
    for a, b in zip(errs, errs[1:]):
        assert b <= max(a / 16.0, floor), errs
    assert errs[0] < 1e-6  # four digits: 28 bits of every operand


@pytest.mark.parametrize("nocc,nvir,seed,ncor", [(8, 100, 41, 0), (5, 129, 42, 1), (6, 200, 43, 0), (3, 8, 44, 0)])
def test_emulated_matches_fused_on_other_shapes(T, nocc, nvir, seed, ncor):
    s = T.synth_system(nocc, nvir, seed=seed, ncor=ncor)
    e4f, e5f, recf, _ = _run(T, [s], mode=T.MODE_FUSED)
    e4, e5, rec, _ = _run(T, [s], slices=8)
    assert_records_close(rec[0], recf[0])
    assert_total_close(e4[0], e4f[0], what="emp4")
    assert_total_close(e5[0], e5f[0], what="emp5")


def test_emulated_batches_and_shards_recombine(T):
    s = T.synth_system(7, 64, seed=45)
    e4, e5, rec, _ = _run(T, [s], slices=7, batch=5)
    e4b, e5b, recb, _ = _run(T, [s], slices=7, batch=64)
    assert np.array_equal(rec[0], recb[0])  # the batch size changes no arithmetic
    parts = [_run(T, [s], slices=7, rank=r, world=3)[2][0] for r in range(3)]
    assert np.array_equal(np.concatenate(parts), rec[0])


def test_emulated_uneven_systems_equal_single_runs(T):
    systems = [T.synth_system(4, 40, seed=46), T.synth_system(6, 90, seed=47, ncor=2), T.synth_system(3, 17, seed=48)]
    e4b, e5b, recb, _ = _run(T, systems, slices=7)
    for q, s in enumerate(systems):
        e4, e5, rec, _ = _run(T, [s], slices=7)
        assert np.array_equal(recb[q], rec[0])
        assert e4b[q] == e4[0] and e5b[q] == e5[0]


def test_emulated_rejects_bad_slice_counts(T):
    s = T.synth_system(2, 8, seed=1)
    for bad in (3, 9):
        with pytest.raises(T.TrpdrvError) as ei:
            T.Plan([s], mode=T.MODE_EMULATED, slices=bad)
        assert ei.value.status == 1


@pytest.mark.parametrize("name,digits", [("g_o10_v60", 12), ("g_o4_v30_log", 11), ("g_o4_v30_log", 13)])
def test_target_digits_picks_the_fewest_slices_that_meet_it(T, name, digits):
    g = load_golden(name)
    s = system_from_golden(g)
    with T.Plan([s], mode=T.MODE_EMULATED, nkpass=g["nkpass"], target_digits=digits) as p:
        p.upload()
        r = p.autotune()
        assert 4 <= r["slices"] <= 8 and r["est_rel_err"] <= 10.0 ** -(digits + 1)
        p.execute()
        e4, e5 = p.energies()
        rec = p.triple_energies(0)
    assert_records_close(rec, g["records"], rtol=10.0 ** -digits)
    assert_total_close(e4[0], g["emp4"], rtol=10.0 ** -digits, what="emp4")
    # fewer slices than chosen would miss the target on the same records
    if r["slices"] > 4:
        _, _, recs, _ = _run(T, [s], nkpass=g["nkpass"], slices=r["slices"] - 1)
        ref = np.asarray(g["records"])
        dev = np.max(np.abs(recs[0] - ref)) / np.max(np.abs(ref))
        assert dev > 10.0 ** -(digits + 2)


# ------------------------------------------------------------------------------------------------
# Energies inside the contraction launch (the default for even nvir): the kernel's energy warps compute
# the previous batch's tile pairs.  TRPDRV_OZ_FUSED_ENERGY=0 selects the separate energy launch; both
# walk the same 128-thread diagonals and sum the warps in the same order, but the two kernels may
# contract multiplies and adds into FMAs differently, so the records agree to a few units in the last
# place (SAME_PATH_RTOL), not bitwise.
# ------------------------------------------------------------------------------------------------
SAME_PATH_RTOL = 1e-13


def _even_goldens():
    return [n for n in golden_cases() if load_golden(n)["nvir"] % 2 == 0]


@pytest.fixture
def fused_energy(monkeypatch):
    monkeypatch.delenv("TRPDRV_OZ_FUSED_ENERGY", raising=False)  # the default
    yield


@pytest.mark.parametrize("name", _even_goldens())
def test_fused_energies_match_reference_golden_and_separate_launch(T, monkeypatch, name):
    g = load_golden(name)
    s = system_from_golden(g)
    monkeypatch.delenv("TRPDRV_OZ_FUSED_ENERGY", raising=False)
    e4f, e5f, recf, launches_f = _run(T, [s], nkpass=g["nkpass"], slices=7)
    monkeypatch.setenv("TRPDRV_OZ_FUSED_ENERGY", "0")
    e4, e5, recs, launches = _run(T, [s], nkpass=g["nkpass"], slices=7)
    monkeypatch.delenv("TRPDRV_OZ_FUSED_ENERGY")
    assert launches_f <= launches  # the energies ride in the contraction launches (plus one per system)
    assert_records_close(recf[0], recs[0], rtol=SAME_PATH_RTOL)
    assert_total_close(e4f[0], e4[0], rtol=SAME_PATH_RTOL, what="emp4 vs separate launch")
    assert_total_close(e5f[0], e5[0], rtol=SAME_PATH_RTOL, what="emp5 vs separate launch")
    assert_records_close(recf[0], g["records"])
    assert_total_close(e4f[0], g["emp4"], what="emp4")
    assert_total_close(e5f[0], g["emp5"], what="emp5")
    assert_records_close(recs[0], g["records"])  # the separate launch meets the bars too


def test_fused_energies_batches_and_shards_recombine(T, fused_energy):
    s = T.synth_system(7, 64, seed=45)
    rec = _run(T, [s], slices=7, batch=5)[2][0]
    assert np.array_equal(_run(T, [s], slices=7, batch=64)[2][0], rec)
    parts = [_run(T, [s], slices=7, rank=r, world=3)[2][0] for r in range(3)]
    assert np.array_equal(np.concatenate(parts), rec)


def test_fused_energies_leave_odd_nvir_on_the_separate_launch(T, monkeypatch):
    """Odd nvir (the f rows are not 16-byte multiples for TMA): the default runs the separate energy
    launch, exactly as TRPDRV_OZ_FUSED_ENERGY=0 does."""
    s = T.synth_system(5, 37, seed=49, ncor=1)
    monkeypatch.delenv("TRPDRV_OZ_FUSED_ENERGY", raising=False)
    base = _run(T, [s], slices=7)
    monkeypatch.setenv("TRPDRV_OZ_FUSED_ENERGY", "0")
    sep = _run(T, [s], slices=7)
    monkeypatch.delenv("TRPDRV_OZ_FUSED_ENERGY")
    assert sep[3] == base[3]
    assert np.array_equal(sep[2][0], base[2][0])
