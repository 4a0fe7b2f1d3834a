"""GPU parity of the full (T) sweep over the virtual index a (options a_count): every plan mode runs
the (a, i, j, k) work of a_count consecutive virtual indices in one execution; per-(a, triple) records
and the summed energies are checked against the oracle run on each single-a view (the reference
driver's fixed-a body, omp/test.c:160-165, with a = system.a + m)."""
import numpy as np
import pytest

from conftest import RECORD_RTOL, TOTAL_RTOL, assert_records_close, assert_total_close

pytestmark = pytest.mark.gpu

MODES = {"fused_tma": dict(mode=1), "fused_cpasync": dict(mode=1, staging=1), "plain": dict(mode=0),
         "emulated8": dict(mode=2, slices=8)}


def _run(T, systems, **opt):
    with T.Plan(systems, **opt) as p:
        p.upload()
        p.execute()
        e4, e5 = p.energies()
        recs = [p.triple_energies(q) for q in range(len(systems))]
    return e4, e5, recs


def _oracle(O, s):
    recs, tots = [], np.zeros(2)
    for m in range(s.a_count):
        r, t, mism = O.run_system(s.a_view(m), "port")
        assert mism == 0
        recs.append(r)
        tots += t
    return np.concatenate(recs), tots


@pytest.mark.parametrize("mode", list(MODES))
def test_a_sweep_matches_the_oracle_per_a(T, O, mode):
    s = T.synth_system(4, 34, seed=71, a_count=3)  # a = 5, 6, 7: all virtual
    want_rec, want_tot = _oracle(O, s)
    e4, e5, recs = _run(T, [s], **MODES[mode])
    assert recs[0].shape == want_rec.shape
    assert_records_close(recs[0], want_rec)
    assert_total_close(e4[0], want_tot[0], what="emp4")
    assert_total_close(e5[0], want_tot[1], what="emp5")


def test_a_sweep_first_block_is_the_single_a_run(T):
    s3 = T.synth_system(6, 40, seed=72, a_count=3)
    s1 = T.synth_system(6, 40, seed=72)
    _, _, r3 = _run(T, [s3], mode=1)
    _, _, r1 = _run(T, [s1], mode=1)
    n = len(r1[0])
    assert np.array_equal(r3[0][:n], r1[0])  # same kernel, same bits
    # the other blocks equal single-a runs of their views
    _, _, r2 = _run(T, [s3.a_view(2)], mode=1)
    assert np.array_equal(r3[0][2 * n:], r2[0])


def test_a_sweep_shards_and_uneven_systems(T):
    a = T.synth_system(5, 32, seed=73, a_count=2)
    b = T.synth_system(3, 18, seed=74, ncor=1, a_count=2)
    e4, e5, recs = _run(T, [a, b], mode=1, staging=1)
    for q, s in enumerate((a, b)):
        _, _, r1 = _run(T, [s], mode=1, staging=1)
        assert np.array_equal(recs[q], r1[0])
    # shards: each rank's records are its triples of every a
    parts = [_run(T, [a], mode=1, rank=r, world=3)[2][0] for r in range(3)]
    full = _run(T, [a], mode=1)[2][0]
    nt = T.count_triples(5)
    got = np.concatenate([np.concatenate([p.reshape(2, -1, 4)[m] for p in parts]) for m in range(2)])
    assert np.array_equal(got, full.reshape(2 * nt, 4))
