"""Sharding of an ensemble over ranks (sph_ensemble.shard / gather_by_box): every box runs
on exactly one rank, loads are balanced by particle-steps, and the per-box results come
back in box order on every rank.  Two gloo ranks on the CPU; the per-box "run" is the
engine's host set-up (no GPU needed), whose particle count is the result."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import sph_b200
import sph_ensemble

NBOX = 24


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def rank_main(rank, world, port, workdir, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pts = sph_ensemble.draw_points(NBOX, seed=11)
        specs = [sph_ensemble.box_spec(pt, nsteps=100) for pt in pts]
        parts = sph_ensemble.shard([sph_ensemble.box_cost(s) for s in specs], world)
        mine = parts[rank]
        paths, _ = sph_ensemble.write_inputs([pts[b] for b in mine],
                                             os.path.join(workdir, "r%d" % rank), nsteps=100)
        rows = []
        for b, p in zip(mine, paths):
            st = sph_b200.host_setup(p)
            info = [x for x in st if isinstance(x, dict) and "N" in x][0]
            rows.append((b, info["N"], rank))
        res = sph_ensemble.gather_by_box(dist, parts, rank, rows, NBOX)
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_cover_every_box_once(tmp_path):
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(rank_main, args=(world, free_port(), str(tmp_path), out), nprocs=world, join=True)
    res0, res1 = out[0], out[1]
    assert res0 == res1
    assert [r[0] for r in res0] == list(range(NBOX))
    owners = [r[2] for r in res0]
    assert set(owners) == {0, 1}
    # balance: particle-step loads within the largest single box of each other
    pts = sph_ensemble.draw_points(NBOX, seed=11)
    costs = [sph_ensemble.box_cost(sph_ensemble.box_spec(p, nsteps=100)) for p in pts]
    loads = [sum(c for c, o in zip(costs, owners) if o == r) for r in range(world)]
    assert abs(loads[0] - loads[1]) <= max(costs)
    # the particle counts are those of the host set-up, i.e. the boxes really ran
    assert all(r[1] > 0 for r in res0)


def test_shard_single_rank_and_more_ranks_than_boxes():
    costs = [5, 1, 3]
    assert sph_ensemble.shard(costs, 1) == [[0, 1, 2]]
    parts = sph_ensemble.shard(costs, 4)
    assert sorted(b for p in parts for b in p) == [0, 1, 2]
    assert [len(p) for p in parts].count(0) == 1
    with pytest.raises(AssertionError):
        sph_ensemble.gather_by_box(None, [[0, 1]], 0, [1, 2], 3)
