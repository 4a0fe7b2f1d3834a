"""The multi-rank path on CPU: world-2 `gloo` ranks each take their share of the triples exactly as a
plan with rank/world does (trpdrv_shard_triples), evaluate it (through the oracle, the CPU checker),
and all-reduce the two energies -- the only exchange step of the sharded GPU run.  The reduced totals
must equal the single-process total, and the shards must cover every triple once."""
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
