"""GPU tests of the autotuner (trpdrv_plan_autotune): it times only compiled variants that the plan
can run, keeps the fastest, caches the choice per device and shapes, and changes no result beyond the
tolerance the variants share (bitwise where the arithmetic is the same)."""
import numpy as np
import pytest

from conftest import assert_records_close, assert_total_close, load_golden, system_from_golden

pytestmark = pytest.mark.gpu


def _energies(p):
    p.execute()
    e4, e5 = p.energies()
    return e4, e5, [p.triple_energies(q) for q in range(len(p.systems))]


def test_fused_autotune_picks_a_valid_variant_and_keeps_parity(T):
    g = load_golden("g_o10_v60")  # even sizes: TMA and cp.async candidates
    s = system_from_golden(g)
    with T.Plan([s], mode=T.MODE_FUSED) as p:
        p.upload()
        r = p.autotune()
        assert not r["from_cache"]
        cands = r["candidates"]
        assert len(cands) >= 3 and {c["staging"] for c in cands} == {1, 2}
        best = cands[r["chosen"]]
        assert best["ms_estimate"] == min(c["ms_estimate"] for c in cands) > 0
        assert p.staging() == best["staging"]
        e4, e5, recs = _energies(p)
    assert_records_close(recs[0], g["records"])
    assert_total_close(e4[0], g["emp4"], what="emp4")
    assert_total_close(e5[0], g["emp5"], what="emp5")
    # a second plan with the same shapes takes the cached choice without timing
    with T.Plan([s], mode=T.MODE_FUSED) as p2:
        p2.upload()
        r2 = p2.autotune()
        assert r2["from_cache"] and r2["candidates"][0] == best
        assert p2.staging() == best["staging"]
        e4b, e5b, recs2 = _energies(p2)
    assert np.array_equal(recs2[0], recs[0])


def test_forced_cpasync_plan_times_only_cpasync_variants(T):
    s = T.synth_system(6, 48, seed=61)
    with T.Plan([s], mode=T.MODE_FUSED, staging=T.STAGING_CPASYNC) as p:
        p.upload()
        r = p.autotune()
        assert r["candidates"] and all(c["staging"] == 1 for c in r["candidates"])
        assert {c["mma_k"] for c in r["candidates"]} >= {4, 8}
        assert p.staging() == 1
        e4, e5, recs = _energies(p)
    with T.Plan([s], mode=T.MODE_FUSED, staging=T.STAGING_CPASYNC) as ref:
        ref.upload()
        r4, r5, rrec = _energies(ref)
    assert_records_close(recs[0], rrec[0])


def test_emulated_autotune_picks_a_batch_and_results_do_not_change(T):
    s = T.synth_system(7, 64, seed=62)
    with T.Plan([s], mode=T.MODE_EMULATED, slices=7) as ref:
        ref.upload()
        r4, r5, rrec = _energies(ref)
    with T.Plan([s], mode=T.MODE_EMULATED, slices=7) as p:
        p.upload()
        r = p.autotune()
        assert [c["batch"] for c in r["candidates"]] == [4, 8, 16, 32]
        e4, e5, recs = _energies(p)
    assert np.array_equal(recs[0], rrec[0])  # the batch size changes no arithmetic


def test_autotune_needs_bound_inputs(T):
    s = T.synth_system(3, 16, seed=63)
    with T.Plan([s], mode=T.MODE_FUSED) as p:
        with pytest.raises(T.TrpdrvError) as ei:
            p.autotune()
        assert ei.value.status == 5  # TRPDRV_ERR_STATE
