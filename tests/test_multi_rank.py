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


SEG_NCOLS, SEG_NROWS, SEG_TILE = 300, 240, 64


def _segment_cloud():
    from terranni_b200 import synth
    xyz, _ = synth.generate(77, 40_000, SEG_NCOLS * 1.0, SEG_NROWS * 1.0, kind="terrain", nclusters=4,
                            cluster_sigma=6.0, nlakes=3, lake_rmin=10.0, lake_rmax=35.0, nthreads=1)
    return xyz


def _segment_tiles():
    """The segment driver's tile grid (row-major) with each tile's cost
    (cells + points in its core)."""
    xyz = _segment_cloud()
    tiles, costs = [], []
    for y in range(0, SEG_NROWS, SEG_TILE):
        for x in range(0, SEG_NCOLS, SEG_TILE):
            x1, y1 = min(x + SEG_TILE, SEG_NCOLS), min(y + SEG_TILE, SEG_NROWS)
            inside = ((xyz[:, 0] >= x * 100) & (xyz[:, 0] < x1 * 100) & (xyz[:, 1] >= y * 100) &
                      (xyz[:, 1] < y1 * 100))
            tiles.append((x, y, x1, y1))
            costs.append((x1 - x) * (y1 - y) + int(inside.sum()))
    return xyz, tiles, costs


def _segment_tile_heights(xyz, tile, halo):
    """One tile as its own work package: its cells, a raster `halo` cells
    wider (clipped to the grid, as the segment driver clips it) and the
    points within twice the halo; exact for halos above the largest disc
    radius (the oracle stands in for the device)."""
    from oracle import oracle
    x0, y0, x1, y1 = tile
    rx0, ry0 = max(0, x0 - halo) - x0, max(0, y0 - halo) - y0
    rx1, ry1 = min(SEG_NCOLS, x1 + halo) - x0, min(SEG_NROWS, y1 + halo) - y0
    sel = ((xyz[:, 0] >= (x0 - 2 * halo) * 100) & (xyz[:, 0] < (x1 + 2 * halo) * 100) &
           (xyz[:, 1] >= (y0 - 2 * halo) * 100) & (xyz[:, 1] < (y1 + 2 * halo) * 100))
    wp = oracle.make_wp(x1 - x0, y1 - y0, 100, x0 * 100, y0 * 100, raster=(rx0, ry0, rx1, ry1))
    return oracle.interpolate(wp, xyz[sel])["h"]


def _segment_halo(xyz):
    from oracle import oracle
    _, _, r2 = oracle.nearest(oracle.make_wp(SEG_NCOLS, SEG_NROWS, 100), xyz)
    return int(np.ceil(np.sqrt(r2.max() + 1.0))) + 3


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
        if mode == "segment":
            # one grid split across the ranks as dnni_segment_run's parts do:
            # a contiguous cost-balanced range of the row-major tiles each
            from terranni_b200 import engine
            xyz, tiles, costs = _segment_tiles()
            first = engine.partition_contiguous(costs, world)
            halo = _segment_halo(xyz)
            mine = {k: _segment_tile_heights(xyz, tiles[k], halo) for k in range(first[rank], first[rank + 1])}
            got = shard.gather_to_root(mine)
            if rank == 0:
                grid = np.full((SEG_NROWS, SEG_NCOLS), np.nan, np.float32)
                seen = []
                for d in got:
                    for k, h in d.items():
                        x0, y0, x1, y1 = tiles[k]
                        grid[y0:y1, x0:x1] = h
                        seen.append(k)
                np.savez(os.path.join(outdir, "segment.npz"), grid=grid, seen=np.array(sorted(seen)),
                         first=first)
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


def test_partition_contiguous_is_balanced_and_complete():
    from terranni_b200 import engine
    rng = np.random.default_rng(5)
    costs = rng.integers(0, 10**6, 256)
    for parts in (1, 2, 3, 8, 300):
        first = engine.partition_contiguous(costs, parts)
        assert first[0] == 0 and first[-1] == 256 and np.all(np.diff(first) >= 0)
        if parts <= 8:
            loads = [int(costs[first[p]:first[p + 1]].sum()) for p in range(parts)]
            assert max(loads) - min(loads) <= 2 * costs.max()
    assert list(engine.partition_contiguous([1, 1, 1, 1], 2)) == [0, 2, 4]
    assert list(engine.partition_contiguous([], 3)) == [0, 0, 0, 0]


def test_two_ranks_split_one_segment_grid_and_stitch_it(tmp_path):
    import torch.multiprocessing as mp
    from oracle import oracle
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), "segment"), nprocs=2, join=True)
    d = np.load(tmp_path / "segment.npz")
    _, tiles, _ = _segment_tiles()
    assert list(d["seen"]) == list(range(len(tiles)))           # every tile once
    assert 0 < d["first"][1] < len(tiles)                       # both ranks had work
    ref = oracle.interpolate(oracle.make_wp(SEG_NCOLS, SEG_NROWS, 100), _segment_cloud())["h"]
    assert np.array_equal(d["grid"].view(np.uint32), ref.view(np.uint32))


def test_a_rank_that_leaves_is_an_error_on_the_other(tmp_path):
    import torch.multiprocessing as mp
    with pytest.raises(Exception):
        mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), "fail"), nprocs=2, join=True)
    assert int(np.load(tmp_path / "fail.npy")[0]) == 1
