"""Host-side logic of the library (no GPU): triple enumeration, partitioning, shards, the synthetic
generator, argument validation of the drop-in entry points and plan creation without a device."""
import os

import numpy as np
import pytest

from conftest import has_gpu


@pytest.mark.parametrize("nocc", [1, 2, 5, 8, 13])
@pytest.mark.parametrize("nkpass", [1, 2, 3, 7])
def test_enumeration_matches_reference_driver_order(T, O, nocc, nkpass):
    got = T.enumerate_triples(nocc, nkpass)
    want = O.enumerate_triples(nocc, nkpass)
    assert np.array_equal(got, want)
    assert len(got) == T.count_triples(nocc) == nocc * nocc * (nocc + 1) // 2
    # every (i, j, k <= i) exactly once, whatever the k-chunking
    assert len({tuple(r[:3]) for r in got}) == len(got)
    assert np.all(got[:, 2] <= got[:, 0]) and np.all(got[:, 3] <= got[:, 2])


def test_partition_is_contiguous_and_balanced(T):
    rng = np.random.default_rng(0)
    cost = rng.uniform(0.5, 2.0, 1000)
    for world in (1, 2, 3, 7, 16):
        b = T.partition(cost, len(cost), world)
        assert b[0] == 0 and b[-1] == len(cost) and np.all(np.diff(b) >= 0)
        shares = np.array([cost[b[r]:b[r + 1]].sum() for r in range(world)])
        assert shares.max() - shares.min() <= 2 * cost.max()
    b = T.partition(None, 10, 3)
    assert list(b) == [0, 3, 7, 10]
    b = T.partition(None, 2, 4)  # more ranks than items
    assert b[0] == 0 and b[-1] == 2 and np.all(np.diff(b) >= 0)


@pytest.mark.parametrize("nocc,world", [(5, 2), (6, 3), (3, 8), (10, 7)])
def test_shards_cover_the_driver_order(T, nocc, world):
    parts = [T.shard_triples(nocc, 1, r, world) for r in range(world)]
    assert np.array_equal(np.concatenate(parts), T.enumerate_triples(nocc, 1)[:, :3])
    sizes = [len(p) for p in parts]
    assert max(sizes) - min(sizes) <= 1
    with pytest.raises(T.TrpdrvError):
        T.shard_triples(nocc, 1, world, world)


def test_synthetic_generator_is_deterministic_and_in_range(T):
    a = T.synth_system(4, 20, seed=5, ncor=2)
    b = T.synth_system(4, 20, seed=5, ncor=2)
    c = T.synth_system(4, 20, seed=6, ncor=2)
    for n in T.TENSOR_NAMES:
        assert np.array_equal(a.arrays[n], b.arrays[n])
        assert not np.array_equal(a.arrays[n], c.arrays[n])
        assert a.arrays[n].size == T.tensor_elems(T.TENSOR_NAMES.index(n), 2, 4, 20)
    e = a.arrays["eorb"]
    core, occ, vir = e[:2], e[2:6], e[6:]
    assert np.all(np.diff(core) >= 0) and np.all(np.diff(occ) >= 0) and np.all(np.diff(vir) >= 0)
    assert core.min() >= -20 and core.max() <= -5 and occ.min() >= -2 and occ.max() <= -0.5
    assert vir.min() >= 0.2 and vir.max() <= 3.0
    assert np.abs(a.arrays["t2"]).max() <= 0.05 and np.abs(a.arrays["tov"]).max() <= 0.02
    assert np.abs(a.arrays["jvv"]).max() <= 0.1 and np.abs(a.arrays["t1v"]).max() <= 0.02
    assert a.a == 2 + 4 + 1  # first virtual: every denominator e_b + e_c + eaijk >= 2.1
    lg = T.synth_system(3, 16, seed=1, dist=T.DIST_LOGUNIFORM)
    mag = np.abs(lg.arrays["kvv"])
    assert mag.min() >= 1e-6 * (1 - 1e-12) and mag.max() <= 1.0
    assert (lg.arrays["kvv"] < 0).mean() > 0.3 and (lg.arrays["kvv"] > 0).mean() > 0.3
    assert np.abs(lg.arrays["t2"]).max() <= 0.05  # amplitudes keep the uniform distribution


def test_dropin_rejects_bad_arguments_before_touching_a_device(T, monkeypatch):
    monkeypatch.setenv("TRPDRV_ON_ERROR", "return")
    s = T.synth_system(3, 12, seed=2)
    T.clear_error()
    assert T.cbody(s, 4, 1, 1, 1, emp4=1.5, emp5=2.5) == (1.5, 2.5)  # i > nocc
    code, msg = T.last_error()
    assert code == 1 and "outside" in msg
    T.clear_error()
    assert T.cbody(s, 2, 1, 2, 3, emp4=1.5, emp5=2.5) == (1.5, 2.5)  # klo > k
    assert T.last_error()[0] == 1


@pytest.mark.skipif(has_gpu(), reason="checks the behaviour without a device")
def test_plan_without_a_device_reports_nodev(T):
    s = T.synth_system(2, 8, seed=1)
    with pytest.raises(T.TrpdrvError) as ei:
        T.Plan([s])
    assert ei.value.status in (4, 2)


def test_plan_argument_checks_precede_device_use(T):
    s = T.synth_system(2, 8, seed=1)
    with pytest.raises(T.TrpdrvError) as ei:
        T.Plan([T.System(0, 2, 8, 0, s.arrays)])
    assert ei.value.status == 1
    with pytest.raises(T.TrpdrvError) as ei:
        T.Plan([s], rank=3, world=2)
    assert ei.value.status == 1
    with pytest.raises(T.TrpdrvError) as ei:
        T.Plan([s], staging=5)
    assert ei.value.status == 1


def _lru_misses(ijk, order, cap_slices):
    """Slices (T2[j][x] per (j, x); J[x] and K[x] per x) that an LRU cache of cap_slices slices misses."""
    from collections import OrderedDict
    lru, miss = OrderedDict(), 0
    for t in order:
        i, j, k = (int(v) for v in ijk[t])
        for key in (("t2", j, i), ("t2", j, k), ("jk", i), ("jk", k)):
            if key in lru:
                lru.move_to_end(key)
            else:
                miss += 1
                lru[key] = 1
                if len(lru) > cap_slices:
                    lru.popitem(last=False)
    return miss


@pytest.mark.parametrize("nocc,nkpass,world", [(1, 1, 1), (7, 1, 1), (12, 3, 1), (20, 1, 3), (40, 1, 1)])
def test_processing_order_is_a_permutation_that_keeps_slices_resident(T, nocc, nkpass, world):
    for rank in range(world):
        ijk = T.shard_triples(nocc, nkpass, rank, world)
        order = T.processing_order(ijk)
        assert np.array_equal(np.sort(order), np.arange(len(ijk)))
        # the runs of equal j stay whole: one j's T2 slices at a time
        js = ijk[order, 1]
        assert np.count_nonzero(np.diff(js)) == np.count_nonzero(np.diff(ijk[:, 1]))
    if nocc == 40:
        # with room for 24 slices the driver order re-reads most of them; the blocked order does not
        ident = np.arange(len(ijk))
        assert _lru_misses(ijk, order, 24) * 4 < _lru_misses(ijk, ident, 24)


def test_processing_order_rejects_bad_arguments(T):
    assert T.lib.trpdrv_processing_order(None, 3, 0, None) == -1
    assert T.lib.trpdrv_processing_order(None, -1, 0, None) == -1
    assert len(T.processing_order(np.zeros((0, 3), np.int32))) == 0


@pytest.mark.parametrize("nocc,nkpass,world,chunks", [(40, 1, 1, 16), (40, 1, 1, 1), (40, 1, 1, 100),
                                                       (13, 3, 1, 5), (17, 1, 3, 4), (2, 1, 1, 16)])
def test_upload_spans_cover_the_order_and_never_split_a_j_run(T, nocc, nkpass, world, chunks):
    """The spans trpdrv_plan_upload_execute launches one by one: contiguous, covering every position,
    at most `chunks`, each ending where j changes, and (one k pass) each reading a j range of its own."""
    for rank in range(world):
        ijk = T.shard_triples(nocc, nkpass, rank, world)
        order = T.processing_order(ijk)
        b = T.upload_spans(ijk, order, chunks)
        n = len(ijk)
        assert b[0] == 0 and b[-1] == n and np.all(np.diff(b) > 0) and len(b) - 1 <= chunks
        js = ijk[order, 1]
        for e in b[1:-1]:
            assert js[e] != js[e - 1]
        if nkpass == 1:  # j rises along the order: the spans' j ranges are disjoint and ascending
            ranges = [(js[lo], js[hi - 1]) for lo, hi in zip(b[:-1], b[1:])]
            assert all(r0[1] < r1[0] for r0, r1 in zip(ranges[:-1], ranges[1:]))
        if chunks >= len(np.unique(js)) and nkpass == 1:
            assert len(b) - 1 == len(np.unique(js))  # one span per j when chunks allow
    # list order (no permutation) and the empty list
    ijk = T.shard_triples(6, 1, 0, 1)
    assert np.array_equal(T.upload_spans(ijk, None, 6), np.concatenate([[0], np.cumsum(np.arange(1, 7) * 0 + 21)]))
    assert list(T.upload_spans(np.zeros((0, 3), np.int32), None, 4)) == [0]


def test_upload_spans_reject_bad_arguments(T):
    ijk = T.shard_triples(5, 1, 0, 1)
    with pytest.raises(T.TrpdrvError):
        T.upload_spans(ijk, None, 0)
    bad = T.processing_order(ijk)
    bad[3] = len(ijk)  # not a position of the list
    with pytest.raises(T.TrpdrvError):
        T.upload_spans(ijk, bad, 4)
    assert T.lib.trpdrv_plan_upload_execute(None, None, 0, None) == 1


def test_autotune_rejects_a_null_plan(T):
    import ctypes as C
    r = T.TuneResult()
    assert T.lib.trpdrv_plan_autotune(None, C.byref(r)) == 1
    assert r.ncand == 0


def test_a_block_generates_one_block_of_the_sweep(T):
    sweep = T.synth_system(4, 20, seed=9, a_count=3)
    for m in range(3):
        one = T.synth_system(4, 20, seed=9, a_block=m)
        v = sweep.a_view(m)
        assert one.a == v.a == sweep.a + m and one.a_count == 1
        for name in T.TENSOR_NAMES:
            assert np.array_equal(one.arrays[name], v.arrays[name])
    tail = T.synth_system(4, 20, seed=9, a_count=2, a_block=1)  # blocks 1 and 2 of the same sweep
    assert np.array_equal(tail.a_view(1).arrays["jvv"], sweep.a_view(2).arrays["jvv"])
    with pytest.raises(T.TrpdrvError):
        T.synth_system(4, 20, seed=9, a_block=-1)


def test_a_sweep_synthetic_blocks_and_views(T):
    one = T.synth_system(4, 20, seed=9)
    three = T.synth_system(4, 20, seed=9, a_count=3)
    for t, name in enumerate(T.TENSOR_NAMES):
        n = T.tensor_elems(t, 0, 4, 20)
        dep = T.tensor_a_dependent(t)
        assert three.arrays[name].size == n * (3 if dep else 1)
        assert np.array_equal(three.arrays[name][:n], one.arrays[name])  # block 0 is the single-a system
        v = three.a_view(2)
        assert v.a == three.a + 2 and v.arrays[name].size == n
        if dep:
            assert not np.array_equal(v.arrays[name], one.arrays[name])
    assert [T.TENSOR_NAMES[t] for t in range(len(T.TENSOR_NAMES)) if T.tensor_a_dependent(t)] == \
        ["jvv", "kvv", "dintc", "dintx", "t1v"]


def test_a_sweep_range_is_checked_before_device_use(T):
    s = T.synth_system(2, 8, seed=1, a_count=4)  # a = 3 (first virtual), basis 10: a + 3 <= 10 is fine
    bad = T.synth_system(2, 8, seed=1, a=8, a_count=4)  # 8 + 3 > 10
    with pytest.raises(T.TrpdrvError) as ei:
        T.Plan([bad])
    assert ei.value.status == 1 and "a_count" in str(ei.value)
    with pytest.raises(T.TrpdrvError) as ei:
        T.Plan([s, T.synth_system(2, 8, seed=2)])  # mixed a_count
    assert ei.value.status == 1


def test_register_host_checks_arguments_first(T):
    assert T.lib.trpdrv_register_host(None, 8) == 1
    assert T.lib.trpdrv_refresh_host(None) == 1
    assert T.lib.trpdrv_unregister_host(None) == 1


def test_size_limits_are_checked_before_device_use(T):
    s = T.synth_system(2, 8, seed=1)
    for nocc, nvir in ((1024, 8), (2, 16385), (0, 8), (2, 0)):
        with pytest.raises(T.TrpdrvError) as ei:
            T.Plan([T.System(0, nocc, nvir, 1, s.arrays)])
        assert ei.value.status == 1
    with pytest.raises(T.TrpdrvError) as ei:
        T.Plan([s], mode=T.MODE_EMULATED, target_digits=16)
    assert ei.value.status == 1


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                    "oracle", "_ref", "libtrpdrv_ref.so")),
                    reason="reference not built")
def test_bench_reference_arm_prints_one_contract_line():
    """`bench.py --impl reference` (the reference's CPU body on this host, no GPU needed) prints one JSON
    line with the keys the benchmark contract asks of the reference arm."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], check=True, capture_output=True, text=True, timeout=600).stdout
    lines = [l for l in out.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "triples/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["n_gpus"] == 1
    assert d["config"]["triples_per_step"] == 32800 and d["config"]["nocc"] == 40 and d["config"]["nvir"] == 300
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "triples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                    "oracle", "_ref", "libtrpdrv_ref.so")),
                    reason="reference not built")
def test_bench_reference_arm_maps_no_product_library():
    """The reference arm runs the reference's CPU body on inputs from the oracle's generator: the
    product library is never mapped into that process, and libgomp sees the passive wait policy."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import os, sys\n"
        f"sys.path.insert(0, {root!r})\n"
        "os.environ.pop('OMP_WAIT_POLICY', None)\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', '--workload', 'c1']\n"
        "import bench\n"
        "bench.main()\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('MAPS', 'libtrpdrv_b200' in maps, 'libtrpdrv_ref' in maps, os.environ.get('OMP_WAIT_POLICY'))\n")
    env = dict(os.environ)
    env.pop("OMP_WAIT_POLICY", None)
    out = subprocess.run([sys.executable, "-c", code], check=True, capture_output=True, text=True, timeout=600,
                         env=env).stdout
    tail = [ln for ln in out.splitlines() if ln.startswith("MAPS")][0]
    assert tail == "MAPS False True passive", tail


def test_bench_config_is_shared_by_both_arms():
    """Both arms print the same `config` object for the same arguments (the lines then compare)."""
    import importlib
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    bench = importlib.import_module("bench")
    for wl in ("c1", "c2", "c3", "c4"):
        sys_argv = sys.argv
        sys.argv = ["bench.py", "--workload", wl]
        try:
            args = bench.parse()
        finally:
            sys.argv = sys_argv
        cfg = bench.config_for(args)
        assert cfg["triples_per_step"] == sum(o * o * (o + 1) // 2 for o, _, _, _ in
                                              bench.workload_shapes(wl, args.nocc, args.nvir))
        assert "parallelism" in cfg and "workload" in cfg
