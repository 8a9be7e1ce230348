"""The N > 1 host path on CPU: world_size-2 gloo ranks shard the batched
soils (no collective on the data path), and the only collectives — the
barrier and the max-over-ranks step time — behave as the benchmark uses them.
The per-rank compute is the oracle here (no GPU in this test)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import sys
    from datetime import timedelta
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import __graft_entry__
    import bench
    import oracle as O
    gfk = __graft_entry__.load_package()
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    soils, ranges, nk, kmax = gfk.workloads.batched_soils(count=5, seed=3)
    soils = [(st, fr[::200]) for st, fr in soils]
    mine = gfk.workloads.shard(soils, rank, world)
    rows = {}
    for st, fr in mine:
        key = tuple(round(l.vs, 6) for l in st)
        tup = [(l.thickness, l.vp, l.vs, l.density, l.qs, l.qp) for l in st]
        g, status = O.bank_spectra(tup, ranges[::32], fr, samples=256, kmax=kmax, formulation=O.DUNKIN, threads=1)
        assert (status == 0).all()
        rows[key] = g
    gathered = [None] * world
    dist.all_gather_object(gathered, rows)
    bench.barrier(world)
    t = bench.allmax(float(rank + 1), world)
    if rank == 0:
        union = {}
        for part in gathered:
            assert not (set(part) & set(union)), "a soil was built twice"
            union.update(part)
        np.save(os.path.join(out_dir, "union.npy"), np.array([union[k] for k in sorted(union)], dtype=object),
                allow_pickle=True)
        with open(os.path.join(out_dir, "max.txt"), "w") as fh:
            fh.write(repr(t))
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce(tmp_path, gfk, oracle):
    world, port = 2, _free_port()
    mp.spawn(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    assert float((tmp_path / "max.txt").read_text()) == 2.0
    union = np.load(tmp_path / "union.npy", allow_pickle=True)
    soils, ranges, nk, kmax = gfk.workloads.batched_soils(count=5, seed=3)
    soils = [(st, fr[::200]) for st, fr in soils]
    single = {}
    for st, fr in soils:
        tup = [(l.thickness, l.vp, l.vs, l.density, l.qs, l.qp) for l in st]
        single[tuple(round(l.vs, 6) for l in st)] = oracle.bank_spectra(
            tup, ranges[::32], fr, samples=256, kmax=kmax, formulation=oracle.DUNKIN, threads=1)[0]
    want = [single[k] for k in sorted(single)]
    assert len(union) == len(want)
    for a, b in zip(union, want):
        assert np.array_equal(a, b)


def test_shard_covers_every_unit_once(gfk):
    soils, *_ = gfk.workloads.batched_soils(count=64, seed=5)
    for world in (1, 2, 3, 8):
        parts = [gfk.workloads.shard(soils, r, world) for r in range(world)]
        ids = sorted(id(u) for p in parts for u in p)
        assert ids == sorted(id(u) for u in soils)
        cost = [sum(len(fr) * len(st) for st, fr in p) for p in parts]
        assert max(cost) - min(cost) <= max(len(fr) * len(st) for st, fr in soils)
