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
        assert r["from_cache"] == 0
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
        assert [c["batch"] for c in r["candidates"]] == [8, 16, 32, 64]
        e4, e5, recs = _energies(p)
    assert np.array_equal(recs[0], rrec[0])  # the batch size changes no arithmetic


def test_autotune_needs_bound_inputs(T):
    s = T.synth_system(3, 16, seed=63)
    with T.Plan([s], mode=T.MODE_FUSED) as p:
        with pytest.raises(T.TrpdrvError) as ei:
            p.autotune()
        assert ei.value.status == 5  # TRPDRV_ERR_STATE


def test_tuning_cache_file_is_read_by_a_second_process(T, tmp_path):
    """TRPDRV_TUNE_CACHE: the first process times the candidates and appends its choice to the file; a
    second process with the same shapes takes the choice from the file without timing."""
    import json
    import os
    import subprocess
    import sys
    cache = tmp_path / "tune.txt"
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import json, sys\n"
        f"sys.path.insert(0, {os.path.join(root, 'nwchem-ccsd-trpdrv_b200')!r})\n"
        "import trpdrv_b200 as T\n"
        "s = T.synth_system(8, 64, seed=64)\n"
        "with T.Plan([s], mode=T.MODE_FUSED, device=0) as p:\n"
        "    p.upload()\n"
        "    r = p.autotune()\n"
        "    p.execute()\n"
        "    e4, e5 = p.energies()\n"
        "print('RESULT', json.dumps({'from_cache': r['from_cache'], 'best': r['candidates'][r['chosen']],\n"
        "                            'e4': e4[0], 'e5': e5[0]}))\n")
    env = dict(os.environ, TRPDRV_TUNE_CACHE=str(cache))
    runs = []
    for _ in range(2):
        out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, env=env,
                             check=True).stdout
        runs.append(json.loads([ln for ln in out.splitlines() if ln.startswith("RESULT")][0][7:]))
    assert runs[0]["from_cache"] == 0 and runs[1]["from_cache"] == 2
    assert runs[1]["best"]["staging"] == runs[0]["best"]["staging"]
    assert runs[1]["best"]["mma_k"] == runs[0]["best"]["mma_k"]
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and "trpdrv-tune" in lines[0] and "shapes=8,64,1" in lines[0]
    assert abs(runs[1]["e4"] - runs[0]["e4"]) <= 1e-12 * abs(runs[0]["e4"])


def test_edge_tile_shape_is_a_tuning_choice_and_keeps_parity(T, O):
    """nvir = 134: the last tile holds 6 indices, so the TMA candidates come with packed (two 32x16 pairs
    per item) and ordinary edge items; whichever is chosen matches the oracle."""
    s = T.synth_system(6, 134, seed=65)
    rec_o, tot_o, mism = O.run_system(s, "port", nthreads=4)
    assert mism == 0
    with T.Plan([s], mode=T.MODE_FUSED) as p:
        p.upload()
        r = p.autotune()
        tma = [c for c in r["candidates"] if c["staging"] == 2]
        assert {c["edge_pack"] for c in tma} == {0, 1} and {c["mma_k"] for c in tma} == {8, 16}
        e4, e5, recs = _energies(p)
    assert_records_close(recs[0], rec_o)
    assert_total_close(e4[0], tot_o[0], what="emp4")
    assert_total_close(e5[0], tot_o[1], what="emp5")
