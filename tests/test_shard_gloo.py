"""The multi-rank paths on CPU, as world-2 `gloo` ranks evaluated through the oracle (the CPU checker),
each ending in one all-reduce of the energies -- the only exchange step of a multi-GPU run:
* strong split: each rank takes its share of one a's triples exactly as a plan with rank/world does
  (trpdrv_shard_triples); the reduced totals equal the single-process total and the shards cover
  every triple once;
* split over a (the default of bench.py at N > 1): rank r takes the virtual index a + r, the block r of
  an a-sweep system (the a loop of the full (T)); the reduced totals equal the serial sum over a."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, nocc, nvir, seed, out):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist
    import oracle as O
    import trpdrv_b200 as T

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        s = T.synth_system(nocc, nvir, seed=seed)
        mine = T.shard_triples(nocc, 1, rank, world)
        counts = [len(T.shard_triples(nocc, 1, r, world)) for r in range(world)]
        lo = sum(counts[:rank])
        # the shard is the contiguous range [lo, lo + n) of the driver order
        assert np.array_equal(mine, T.enumerate_triples(nocc, 1)[lo:lo + len(mine), :3])
        _, tot, mism = O.run_system(s, "port", t_begin=lo, t_end=lo + len(mine), nthreads=1)
        assert mism == 0
        t = torch.tensor([tot[0], tot[1], float(len(mine))], dtype=torch.float64)
        dist.all_reduce(t)
        out[rank] = t.tolist()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gloo_sharded_energies_equal_single_rank(O, T, world):
    nocc, nvir, seed = 6, 28, 19
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, nocc, nvir, seed, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    s = T.synth_system(nocc, nvir, seed=seed)
    _, whole, _ = O.run_system(s, "port")
    for r in range(world):
        e4, e5, n = out[r]
        assert n == T.count_triples(nocc)
        assert abs(e4 - whole[0]) <= 1e-13 * abs(whole[0])
        assert abs(e5 - whole[1]) <= 1e-13 * abs(whole[1])


def _rank_main_a(rank, world, port, nocc, nvir, seed, out):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "nwchem-ccsd-trpdrv_b200"))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist
    import oracle as O
    import trpdrv_b200 as T

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        mine = T.synth_system(nocc, nvir, seed=seed, a_block=rank)  # this rank's a, as bench.py makes it
        _, tot, mism = O.run_system(mine, "port", nthreads=1)
        assert mism == 0
        t = torch.tensor([tot[0], tot[1], float(T.count_triples(nocc))], dtype=torch.float64)
        dist.all_reduce(t)
        out[rank] = t.tolist()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_gloo_split_over_a_sums_the_full_t(O, T, world):
    nocc, nvir, seed = 5, 24, 23
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main_a, args=(r, world, port, nocc, nvir, seed, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    sweep = T.synth_system(nocc, nvir, seed=seed, a_count=world)
    per_a = [O.run_system(sweep.a_view(r), "port")[1] for r in range(world)]
    want4, want5 = sum(t[0] for t in per_a), sum(t[1] for t in per_a)
    assert per_a[0][0] != per_a[1][0]  # the ranks really evaluate different a
    for r in range(world):
        e4, e5, n = out[r]
        assert n == world * T.count_triples(nocc)
        assert abs(e4 - want4) <= 1e-13 * abs(want4)
        assert abs(e5 - want5) <= 1e-13 * abs(want5)
