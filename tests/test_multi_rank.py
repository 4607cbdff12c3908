"""The multi-GPU path on CPU: world-size-2 process groups over gloo.

Each rank computes the same cost partition of a mixed tile batch without
communicating, interpolates its share (the CPU oracle stands in for the
device here), and the shares are gathered on rank 0, where they must cover
every tile exactly once and equal the single-process results; the timing
collective is the max over ranks.  Also: a rank that fails between steps is
seen by the other on its next collective as an error, not a hang."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _small_specs():
    from terranni_b200 import synth
    specs = synth.mixed_tiles(count=10, seed=4242, max_points=6000)
    for s in specs:
        s["side"] = min(s["side"], 96)
        s["n"] = min(s["n"], 6000)
    return specs


def _tile_result(s):
    from oracle import oracle
    from terranni_b200 import synth
    xyz = synth.tile_points(s)
    r = oracle.interpolate(oracle.make_wp(s["side"], s["side"], s["cell"]), xyz)
    return r["h"]


def _worker(rank, world, port, outdir, mode):
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    import torch.distributed as dist
    from terranni_b200 import shard
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        if mode == "fail":
            if rank == 1:
                raise SystemExit(3)          # leaves before its next collective
            try:
                dist.barrier()
                np.save(os.path.join(outdir, "fail.npy"), np.array([0]))
            except Exception:
                np.save(os.path.join(outdir, "fail.npy"), np.array([1]))
            return
        specs = _small_specs()
        costs = [shard.tile_cost(s["side"], s["side"], s["n"]) for s in specs]
        parts = shard.partition_by_cost(costs, world)
        mine = {k: _tile_result(specs[k]) for k in parts[rank]}
        slowest = shard.max_over_ranks(float(rank + 1))
        got = shard.gather_to_root(mine)
        if rank == 0:
            merged = {}
            for d in got:
                for k, h in d.items():
                    assert k not in merged
                    merged[k] = h
            np.savez(os.path.join(outdir, "merged.npz"), keys=np.array(sorted(merged)),
                     slowest=np.array([slowest]), **{f"h{k}": merged[k] for k in merged})
    finally:
        if dist.is_initialized():
            dist.destroy_process_group()


def test_partition_by_cost_is_balanced_and_complete():
    from terranni_b200 import shard
    rng = np.random.default_rng(3)
    costs = rng.integers(1, 10**6, 300)
    for world in (1, 2, 3, 8):
        parts = shard.partition_by_cost(costs, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(300))
        loads = [int(costs[p].sum()) for p in parts]
        assert max(loads) - min(loads) <= costs.max()        # LPT bound
    assert shard.partition_by_cost([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]


def test_route_least_loaded():
    from terranni_b200 import shard
    loads = [0, 0, 0]
    ranks = [shard.route_least_loaded(loads, c) for c in (10, 5, 5, 1, 20)]
    assert ranks == [0, 1, 2, 1, 2] and loads == [10, 6, 25]


def test_two_ranks_shard_and_gather_equal_one_process(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), "run"), nprocs=2, join=True)
    d = np.load(tmp_path / "merged.npz")
    specs = _small_specs()
    assert list(d["keys"]) == list(range(len(specs)))
    assert float(d["slowest"][0]) == 2.0
    for k, s in enumerate(specs):
        assert np.array_equal(d[f"h{k}"].view(np.uint32), _tile_result(s).view(np.uint32))


def test_a_rank_that_leaves_is_an_error_on_the_other(tmp_path):
    import torch.multiprocessing as mp
    with pytest.raises(Exception):
        mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), "fail"), nprocs=2, join=True)
    assert int(np.load(tmp_path / "fail.npy")[0]) == 1
