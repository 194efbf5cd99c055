"""Batched sweep (C2) on the host: the spec generator, the balanced sharding
of discharges over ranks, and the multi-rank plumbing on world_size 2 with
the gloo backend (no GPU)."""
import os
import socket

import numpy as np
import pytest


def test_c2_specs_are_seeded_and_in_range(cudapic):
    from cudapic_b200.batch import c2_specs
    a, b = c2_specs(), c2_specs()
    assert a == b and len(a) == 256
    assert all(100 <= s.voltage <= 500 and 5 <= s.pressure <= 50 and 0.015 <= s.gap <= 0.040 for s in a)
    assert {s.n_g for s in a} == {200, 400, 800}
    p = np.array([s.particles for s in a])
    assert p.min() >= 1e4 and p.max() <= 1e6 and 5e4 < np.median(p) < 2e5   # log-uniform: median 1e5
    assert len({s.seed for s in a}) == 256 and c2_specs(seed=1) != a


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_is_a_balanced_partition(cudapic, world):
    from cudapic_b200.batch import c2_specs, shard
    specs = c2_specs()
    parts = shard(specs, world)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(specs)))
    loads = [sum(specs[k].particles for k in p) for p in parts]
    assert max(loads) - min(loads) <= max(s.particles for s in specs)   # greedy bound


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    from cudapic_b200.batch import c2_specs, gather, reduce_max_sum, shard
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        specs = c2_specs(n=40)
        mine = shard(specs, world)[rank]
        work = sum(specs[k].particles for k in mine)
        everyone = gather({"rank": rank, "discharges": mine, "work": work}, world)
        t, w = reduce_max_sum(world, 1.0 + rank, work)
        np.save(os.path.join(out_dir, "r%d.npy" % rank),
                np.array([t, w, sum(len(e["discharges"]) for e in everyone)] +
                         sorted(k for e in everyone for k in e["discharges"]), np.float64))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_gather_and_reduce(cudapic, tmp_path):
    import torch.multiprocessing as mp
    from cudapic_b200.batch import c2_specs
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    total = sum(s.particles for s in c2_specs(n=40))
    for r in range(2):
        v = np.load(tmp_path / ("r%d.npy" % r))
        assert v[0] == 2.0 and v[1] == total and v[2] == 40     # max time, summed work, all discharges
        assert list(v[3:].astype(int)) == list(range(40))      # every rank sees the whole partition
