"""GPU parity of the library against the oracle and the reference's golden vectors (B200 only).

Every call goes through the C ABI (libtrpdrv_b200.so).  Bars: emp4/emp5 totals within 1e-11
relative (TOTAL_RTOL); per-triple records within 1e-11 normwise per column (RECORD_RTOL); f arrays
within 1e-12 normwise; shards, batches and repeated runs bit-identical where the arithmetic is.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import (GOLDEN, RECORD_RTOL, TOTAL_RTOL, assert_records_close, assert_total_close, golden_cases,
                      load_golden, system_from_golden)
from kat import run_make_array_loop

pytestmark = pytest.mark.gpu

MODES = {"fused": dict(mode=1), "fused_cpasync": dict(mode=1, staging=1, mma_k=8),
         "fused_cpasync_k4": dict(mode=1, staging=1, mma_k=4), "plain": dict(mode=0)}


def _plan_run(T, systems, **opt):
    with T.Plan(systems, **opt) as p:
        p.upload()
        p.execute()
        e4, e5 = p.energies()
        recs = [p.triple_energies(q) for q in range(len(systems))]
        launches = p.last_launches()
        staging = p.staging()
    if opt.get("mode", 1) == 1:  # TMA wherever the shapes allow it, cp.async otherwise
        even = all(s.nvir % 2 == 0 and s.nocc % 2 == 0 for s in systems)
        want = {0: 2 if even else 1, 1: 1, 2: 2}[opt.get("staging", 0)]
        assert staging == want, (staging, want)
    return e4, e5, recs, launches


@pytest.mark.parametrize("mode", list(MODES))
@pytest.mark.parametrize("name", golden_cases())
def test_plan_matches_reference_golden(T, name, mode):
    g = load_golden(name)
    s = system_from_golden(g)
    e4, e5, recs, launches = _plan_run(T, [s], nkpass=g["nkpass"], **MODES[mode])
    assert launches > 0
    assert_records_close(recs[0], g["records"])
    assert_total_close(e4[0], g["emp4"], what="emp4")
    assert_total_close(e5[0], g["emp5"], what="emp5")


def test_fused_uneven_batch_equals_single_runs(T):
    names = golden_cases()
    systems = [system_from_golden(load_golden(n)) for n in names]
    nk = [load_golden(n)["nkpass"] for n in names]
    # one plan needs one nkpass; use 1 for all and compare against single-system plans with nkpass 1.
    # The batch holds odd sizes, so it runs with cp.async staging; compare with the same staging.
    e4b, e5b, recb, _ = _plan_run(T, systems, mode=1, staging=1)
    for q, s in enumerate(systems):
        e4, e5, rec, _ = _plan_run(T, [s], mode=1, staging=1)
        assert np.array_equal(recb[q], rec[0]), names[q]
        assert e4b[q] == e4[0] and e5b[q] == e5[0], names[q]
    assert len(nk) == len(systems)


def test_tma_uneven_batch_equals_single_runs(T):
    shapes = [(4, 24, 51), (8, 80, 52), (6, 130, 53)]
    systems = [T.synth_system(o, v, seed=sd) for o, v, sd in shapes]
    e4b, e5b, recb, _ = _plan_run(T, systems, mode=1, staging=2)
    for q, s in enumerate(systems):
        e4, e5, rec, _ = _plan_run(T, [s], mode=1, staging=2)
        assert np.array_equal(recb[q], rec[0]) and e4b[q] == e4[0] and e5b[q] == e5[0], shapes[q]


def test_sharded_plans_cover_the_system(T):
    g = load_golden("g_o10_v60")
    s = system_from_golden(g)
    whole4, whole5, wrec, _ = _plan_run(T, [s], mode=1)
    world = 3
    tri_all, rec_all, s4, s5 = [], [], 0.0, 0.0
    for r in range(world):
        with T.Plan([s], mode=1, rank=r, world=world) as p:
            p.upload()
            p.execute()
            e4, e5 = p.energies()
            tri_all.append(p.triples(0))
            rec_all.append(p.triple_energies(0))
            assert np.array_equal(p.triples(0), T.shard_triples(s.nocc, 1, r, world))
        s4 += e4[0]
        s5 += e5[0]
    assert np.array_equal(np.concatenate(tri_all), T.enumerate_triples(s.nocc, 1)[:, :3])
    assert np.array_equal(np.concatenate(rec_all), wrec[0])
    assert_total_close(s4, whole4[0], rtol=1e-13)
    assert_total_close(s5, whole5[0], rtol=1e-13)


def test_repeat_execute_is_bitwise_deterministic(T):
    s = T.synth_system(6, 64, seed=21)
    with T.Plan([s], mode=1) as p:
        p.upload()
        out = []
        for _ in range(3):
            p.execute()
            out.append(p.energies())
            out.append(p.triple_energies(0))
    assert out[0][0][0] == out[2][0][0] and out[0][1][0] == out[2][1][0]
    assert np.array_equal(out[1], out[3]) and np.array_equal(out[1], out[5])


def test_bind_device_matches_upload(T):
    import torch
    s = T.synth_system(5, 48, seed=22)
    e4u, e5u, recu, _ = _plan_run(T, [s], mode=1)
    dev = {n: torch.from_numpy(a).cuda() for n, a in s.arrays.items()}
    torch.cuda.synchronize()
    with T.Plan([s], mode=1) as p:
        p.bind_device([{n: t.data_ptr() for n, t in dev.items()}])
        p.execute()
        e4, e5 = p.energies()
        rec = p.triple_energies(0)
    assert np.array_equal(rec, recu[0]) and e4[0] == e4u[0] and e5[0] == e5u[0]


def test_fused_without_graph_matches_graph(T):
    s = T.synth_system(5, 40, seed=23)
    a = _plan_run(T, [s], mode=1, use_graph=1)
    b = _plan_run(T, [s], mode=1, use_graph=0)
    assert np.array_equal(a[2][0], b[2][0])


@pytest.mark.parametrize("nocc,nvir,seed,ncor", [(8, 100, 31, 0), (5, 129, 32, 1), (4, 31, 33, 0), (3, 8, 34, 0),
                                                 (2, 1, 35, 0), (1, 33, 36, 0)])
def test_fused_and_plain_match_reference_odd_shapes(T, O, nocc, nvir, seed, ncor):
    """Ragged tails (nvir not a multiple of 32, odd sizes -> 8-byte staging), tiny systems."""
    if not O.have_reference():
        pytest.skip("oracle/_ref not built")
    s = T.synth_system(nocc, nvir, seed=seed, ncor=ncor)
    rec_ref, tot_ref, mism = O.run_system(s, "reference", nthreads=8)
    assert mism == 0
    for opt in MODES.values():
        e4, e5, recs, _ = _plan_run(T, [s], **opt)
        assert_records_close(recs[0], rec_ref)
        assert_total_close(e4[0], tot_ref[0], what="emp4")
        assert_total_close(e5[0], tot_ref[1], what="emp5")


def test_tengy_dropin_matches_oracle(T, O):
    rng = np.random.default_rng(41)
    ncor, nocc, nvir = 2, 5, 77
    f8 = rng.uniform(-0.5, 0.5, (8, nvir * nvir))
    vecs = [rng.uniform(-0.1, 0.1, nvir) for _ in range(6)]
    eorb = np.concatenate([np.sort(rng.uniform(-20, -5, ncor)), np.sort(rng.uniform(-2, -0.5, nocc)),
                           np.sort(rng.uniform(0.2, 3.0, nvir))])
    want = np.array(O.tengy(f8, vecs, eorb, 1.7, ncor, nocc, nvir))
    for entry in ("ccsd_tengy_omp", "ccsd_tengy", "ccsd_tengy_omp_"):
        got = np.array(T.tengy(f8, vecs, eorb, 1.7, ncor, nocc, nvir, entry=entry))
        np.testing.assert_allclose(got, want, rtol=1e-12, err_msg=entry)


def test_cbody_dropin_writes_f_and_accumulates(T, O, monkeypatch):
    monkeypatch.setenv("TRPDRV_WRITE_F", "1")
    g = load_golden("g_c2_o5_v33")
    s = system_from_golden(g)
    V = s.nvir
    fn_port = O.port_body_fn()
    ijkl = T.enumerate_triples(s.nocc, 1)
    for t in (0, 7, 31, len(ijkl) - 1):
        i, j, k, klo = (int(v) for v in ijkl[t])
        f_gpu = np.zeros((8, V * V))
        f_cpu = np.zeros((8, V * V))
        e4, e5 = T.cbody(s, i, j, k, klo, emp4=1.25, emp5=-0.5, f=f_gpu)
        T.body_call(fn_port, s, i, j, k, klo, 1.25, -0.5, f=f_cpu)
        scale = np.max(np.abs(f_cpu))
        assert np.max(np.abs(f_gpu - f_cpu)) <= 1e-12 * scale
        r = g["records"][t]
        want4 = 1.25 + r[0] + (r[2] if i != k else 0.0)
        want5 = -0.5 + r[1] + (r[3] if i != k else 0.0)
        assert abs(e4 - want4) <= 1e-12 * (abs(want4) + 1.0)
        assert abs(e5 - want5) <= 1e-12 * (abs(want5) + 1.0)


@pytest.mark.parametrize("entry", ["ccsd_trpdrv_omp_cbody_", "ccsd_trpdrv_omp_fbody_", "ccsd_trpdrv_cbody_",
                                   "ccsd_trpdrv_opencl_"])
def test_body_aliases_agree(T, entry):
    g = load_golden("g_o4_v24")
    s = system_from_golden(g)
    e = [T.cbody(s, 3, 2, 2, 1, entry=entry) for _ in range(2)]
    ref = T.cbody(s, 3, 2, 2, 1)
    assert e[0] == e[1] == ref


def test_dropin_make_array_kat(T):
    """The reference driver's loop and fixture (omp/test.c) through our ccsd_trpdrv_omp_cbody_."""
    line, calls = run_make_array_loop(T.lib.ccsd_trpdrv_omp_cbody_, 10, 60)
    assert calls == 550
    assert line == "emp4=2.647247 emp5=-1.560018"


@pytest.mark.parametrize("binary", ["test_c99_b200", "test_f77_b200"])
def test_unmodified_reference_driver_links_and_passes_kat(O, binary):
    path = os.path.join(os.path.dirname(O.ORACLE_LIB), "_ref", binary)
    if not os.path.exists(path):
        pytest.skip(f"{binary} not built")
    with open(os.path.join(GOLDEN, "kat_test_c99_10_60.json")) as f:
        runs = json.load(f)["runs"]
    assert runs[0]["line"] == "emp4=2.647247 emp5=-1.560018"
    for run in runs:  # (10, 60), (10, 60, nkpass 3), (12, 50, nkpass 2): the reference driver's own prints
        out = subprocess.run([path, *run["argv"]], capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr
        assert run["line"] in out.stdout, (run, out.stdout[-300:])


def test_dropin_errors_are_reported_not_computed(T, monkeypatch):
    monkeypatch.setenv("TRPDRV_ON_ERROR", "return")
    s = T.synth_system(3, 16, seed=1)
    T.clear_error()
    e4, e5 = T.cbody(s, 4, 1, 1, 1, emp4=0.5, emp5=0.25)  # i = 4 > nocc = 3
    assert (e4, e5) == (0.5, 0.25)
    code, msg = T.last_error()
    assert code == 1 and "i=4" in msg
    T.clear_error()
    e4, e5 = T.cbody(s, 2, 1, 2, 3, emp4=0.5, emp5=0.25)  # klo > k
    assert (e4, e5) == (0.5, 0.25) and T.last_error()[0] == 1


def test_plan_rejects_bad_arguments(T):
    s = T.synth_system(3, 16, seed=1)
    bad = T.System(0, 3, 16, 0, s.arrays)  # a = 0
    with pytest.raises(T.TrpdrvError) as ei:
        T.Plan([bad])
    assert ei.value.status == 1
    with pytest.raises(T.TrpdrvError):
        T.Plan([s], rank=2, world=2)
    with T.Plan([s]) as p:
        with pytest.raises(T.TrpdrvError) as ei:
            p.execute()
        assert ei.value.status == 5


def test_full_size_fused_vs_plain_and_reference_sample(T, O):
    """(nocc, nvir) = (40, 300): fused and plain totals agree; sampled triples match the reference."""
    s = T.synth_system(40, 300, seed=2024)
    e4f, e5f, recf, _ = _plan_run(T, [s], mode=1)
    e4p, e5p, recp, _ = _plan_run(T, [s], mode=0)
    assert_total_close(e4f[0], e4p[0], rtol=1e-12, what="emp4 fused vs plain")
    assert_total_close(e5f[0], e5p[0], rtol=1e-12, what="emp5 fused vs plain")
    assert_records_close(recf[0], recp[0], rtol=1e-12)
    if O.have_reference():
        for lo in (0, 777, 16400, 32790):
            rec, _, mism = O.run_system(s, "reference", t_begin=lo, t_end=lo + 8, nthreads=8)
            assert mism == 0
            assert_records_close(recf[0][lo:lo + 8], rec)


def test_config1_plain_and_fused_match_the_reference_on_every_triple(T, O):
    """nocc=20, nvir=200, all 4,200 triples of the driver, plain per-triple path and
    fused kernel against the reference body compiled unmodified (run on every host thread)."""
    if not O.have_reference():
        pytest.skip("reference build missing")
    import os
    s = T.synth_system(20, 200, seed=2025)
    ref, tot, mism = O.run_system(s, "reference", nthreads=os.cpu_count() or 1)
    assert mism == 0 and len(ref) == 4200
    for mode in (0, 1):
        e4, e5, rec, _ = _plan_run(T, [s], mode=mode)
        assert_records_close(rec[0], ref)
        assert_total_close(e4[0], tot[0], what=f"emp4 mode {mode}")
        assert_total_close(e5[0], tot[1], what=f"emp5 mode {mode}")


def test_tma_staging_is_refused_for_odd_sizes(T):
    s = T.synth_system(5, 33, seed=3)
    with T.Plan([s], mode=1, staging=2) as p:
        with pytest.raises(T.TrpdrvError) as ei:
            p.upload()
        assert ei.value.status == 6


def test_tma_and_cpasync_stagings_agree(T):
    """Both stagings feed identical operands to identical MMA sequences; only the scalar epilogue may
    round differently (FMA contraction), so the records agree to a few ulps."""
    s = T.synth_system(6, 96, seed=44)
    a = _plan_run(T, [s], mode=1, staging=2)
    b = _plan_run(T, [s], mode=1, staging=1, mma_k=8)
    assert_records_close(a[2][0], b[2][0], rtol=1e-13)


@pytest.mark.parametrize("mode,extra", [(1, {}), (0, {}), (2, {"slices": 8})])
def test_one_call_run_equals_the_plan(T, mode, extra):
    systems = [T.synth_system(4, 30, seed=91), T.synth_system(5, 22, seed=92, ncor=1)]
    e4, e5 = T.run(systems, mode=mode, **extra)
    p4, p5, _, _ = _plan_run(T, systems, mode=mode, **extra)
    assert np.array_equal(e4, p4) and np.array_equal(e5, p5)


def test_more_systems_than_tma_maps_fall_back_to_cpasync(T):
    # even sizes: each alone could use TMA; nine exceed the 8 tensor-map sets a TMA launch carries
    systems = [T.synth_system(2 + 2 * (q % 2), 16 + 2 * q, seed=100 + q) for q in range(9)]
    with T.Plan(systems, mode=1) as p:
        p.upload()
        p.execute()
        e4, e5 = p.energies()
        recs = [p.triple_energies(q) for q in range(9)]
        assert p.staging() == 1
    for q, s in enumerate(systems):
        a4, a5, arec, _ = _plan_run(T, [s], mode=1, staging=1)
        assert np.array_equal(recs[q], arec[0]) and e4[q] == a4[0] and e5[q] == a5[0]


def test_c_caller_of_the_plan_interface_gives_the_python_plan_energies(T, tmp_path):
    """tests/c_plan_caller.c (synthetic inputs, fused plan, autotune, execute) prints the energies the
    Python binding's plan gives on the same seeded system."""
    from test_abi import _build_c_caller
    exe = _build_c_caller(tmp_path)
    out = subprocess.run([exe, "6", "50", "77"], check=True, capture_output=True, text=True).stdout.split()
    s = T.synth_system(6, 50, seed=77)
    with T.Plan([s], mode=1) as p:
        p.upload()
        p.autotune()
        p.execute()
        e4, e5 = p.energies()
    # each process autotunes for itself and may keep another variant: compare at the parity bar
    assert_total_close(float(out[0]), e4[0], what="emp4")
    assert_total_close(float(out[1]), e5[0], what="emp5")


@pytest.mark.parametrize("shape", [(6, 70, 31), (4, 104, 32), (6, 134, 33), (2, 48, 34)])
@pytest.mark.parametrize("mma_k", [8, 16])
def test_tma_packed_edge_items_match_the_oracle_and_the_unpacked_kernel(T, O, monkeypatch, shape, mma_k):
    """Where the last tile holds at most 16 virtual indices the TMA kernel runs the edge pairs two to a
    work item (the last one alone when their count is odd); with TRPDRV_TMA_PACK_EDGE=0 it runs them as
    ordinary items.  Both match the oracle; the f values are the same products, so the two agree to
    rounding of the per-warp sums."""
    nocc, nvir, seed = shape
    s = T.synth_system(nocc, nvir, seed=seed)
    rec_o, tot_o, mism = O.run_system(s, "port", nthreads=4)
    assert mism == 0
    got = {}
    for pack in ("1", "0"):
        monkeypatch.setenv("TRPDRV_TMA_PACK_EDGE", pack)
        e4, e5, recs, _ = _plan_run(T, [s], mode=1, staging=2, mma_k=mma_k)
        assert_records_close(recs[0], rec_o)
        assert_total_close(e4[0], tot_o[0], what="emp4")
        assert_total_close(e5[0], tot_o[1], what="emp5")
        got[pack] = recs[0]
    assert_records_close(got["1"], got["0"], rtol=1e-13)
