"""trpdrv_plan_upload_execute (B200 only): the upload overlapped with the fused kernel, span by span of
the processing order, gives the records and totals of trpdrv_plan_upload + trpdrv_plan_execute bit
for bit (the same kernels write every record's own energy slots; only the launch boundaries move).
"""
import numpy as np
import pytest

from conftest import assert_total_close, golden_cases, load_golden, system_from_golden

pytestmark = pytest.mark.gpu


def _serial(T, systems, **opt):
    with T.Plan(systems, **opt) as p:
        p.upload()
        p.execute()
        e4, e5 = p.energies()
        return e4, e5, [p.triple_energies(q) for q in range(len(systems))]


def _streamed(T, systems, chunks=0, stream=0, **opt):
    with T.Plan(systems, **opt) as p:
        p.upload_execute(chunks=chunks, stream=stream)
        e4, e5 = p.energies()
        recs = [p.triple_energies(q) for q in range(len(systems))]
        launches = p.last_launches()
    return e4, e5, recs, launches


def _same(a, b):
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for ra, rb in zip(a[2], b[2]):
        assert np.array_equal(ra, rb)


@pytest.mark.parametrize("chunks", [0, 1, 3, 16, 1000])
@pytest.mark.parametrize("staging", [0, 1])
def test_streamed_equals_upload_then_execute(T, chunks, staging):
    s = T.synth_system(8, 96, seed=61)
    ref = _serial(T, [s], mode=1, staging=staging)
    got = _streamed(T, [s], chunks=chunks, mode=1, staging=staging)
    _same(got, ref)
    spans = len(T.upload_spans(T.shard_triples(8, 1, 0, 1), T.processing_order(T.shard_triples(8, 1, 0, 1)),
                               chunks or 16)) - 1
    assert got[3] == spans + 2  # one fused launch per span + the two reductions


@pytest.mark.parametrize("name", golden_cases())
def test_streamed_matches_the_golden_totals(T, name):
    g = load_golden(name)
    s = system_from_golden(g)
    e4, e5, _, _ = _streamed(T, [s], chunks=3, mode=1, nkpass=g["nkpass"])
    assert_total_close(e4[0], g["emp4"], what="emp4")
    assert_total_close(e5[0], g["emp5"], what="emp5")


def test_streamed_uneven_systems_a_sweep_and_shards(T):
    systems = [T.synth_system(6, 50, seed=62), T.synth_system(3, 30, seed=63, ncor=2), T.synth_system(7, 64, seed=64)]
    _same(_streamed(T, systems, chunks=4, mode=1), _serial(T, systems, mode=1))
    odd = [T.synth_system(5, 41, seed=65), T.synth_system(4, 30, seed=66)]  # cp.async staging (odd sizes)
    _same(_streamed(T, odd, chunks=3, mode=1), _serial(T, odd, mode=1))
    sweep = [T.synth_system(5, 40, seed=67, a_count=3)]
    _same(_streamed(T, sweep, chunks=5, mode=1), _serial(T, sweep, mode=1))
    for rank in range(3):
        _same(_streamed(T, [systems[0]], chunks=2, mode=1, rank=rank, world=3),
              _serial(T, [systems[0]], mode=1, rank=rank, world=3))
    k_passes = [T.synth_system(7, 40, seed=68)]
    _same(_streamed(T, k_passes, chunks=6, mode=1, nkpass=3), _serial(T, k_passes, mode=1, nkpass=3))


def test_streamed_reupload_replaces_the_data(T):
    s1, s2 = T.synth_system(6, 48, seed=69), T.synth_system(6, 48, seed=70)
    want1, want2 = _serial(T, [s1], mode=1), _serial(T, [s2], mode=1)
    with T.Plan([s1], mode=1) as p:
        p.upload_execute([s1], chunks=3)
        got1 = p.energies()
        p.upload_execute([s2], chunks=5)
        got2 = p.energies()
        p.execute()  # the streamed upload leaves the plan bound: a plain execute reruns s2
        again = p.energies()
        rec = p.triple_energies(0)
    assert np.array_equal(got1[0], want1[0]) and np.array_equal(got1[1], want1[1])
    assert np.array_equal(got2[0], want2[0]) and np.array_equal(got2[1], want2[1])
    assert np.array_equal(again[0], want2[0]) and np.array_equal(rec, want2[2][0])


def test_streamed_on_a_caller_stream(T):
    import torch
    s = T.synth_system(6, 64, seed=71)
    ref = _serial(T, [s], mode=1)
    st = torch.cuda.Stream()
    got = _streamed(T, [s], chunks=4, stream=st.cuda_stream, mode=1)
    _same(got, ref)


@pytest.mark.parametrize("mode,extra", [(0, {}), (2, {"slices": 8})])
def test_streamed_falls_back_to_upload_then_execute(T, mode, extra):
    s = T.synth_system(4, 40, seed=72)
    _same(_streamed(T, [s], chunks=4, mode=mode, **extra), _serial(T, [s], mode=mode, **extra))


def test_streamed_rejects_bad_chunks(T):
    s = T.synth_system(3, 16, seed=73)
    with T.Plan([s], mode=1) as p:
        for bad in (-1, 4097):
            with pytest.raises(T.TrpdrvError):
                p.upload_execute(chunks=bad)
