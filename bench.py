#!/usr/bin/env python
"""Benchmark of the discrete natural-neighbour interpolation hot path.

Workloads (one step = one pass of the hot path over one batch):
  "mixed" (default): 4096 independent tiles, side log-uniform in 64-1024
  cells, cells of 0.5/1/2 m, 1e3-1e6 points per tile (density log-uniform in
  0.05-8 points/cell), per-tile fBm terrain with 0-4 lakes, each tile at its
  own origin.  The batched form runs all tiles in one graph-captured launch
  sequence (dnni_batch_run_device); the plain form beside it makes one
  blocking dnni_interpolate_segment_device call per tile.
  "tile4096": one 4096 x 4096 work package at 1 m cells, 20M points
  (70 % uniform + 30 % in 64 Gaussian clusters, 16 empty lakes of radius
  50-400 m, fBm z 0-300 m + N(0, 0.1 m)), plain per-call form.
Seeded synthetic data, int32 LAS coordinates at 0.01 m; each rank
interpolates its own tiles (weak scaling, no collective on the data path).

value   cells/s with the points already in HBM, timed with CUDA events on
        the launch stream, max over ranks.
e2e     the same metric through the host-buffer C-ABI call (dnni_batch_run
        or dnni_interpolate_segment) from pinned host memory: the point
        upload and the height download are inside the timed region.

``--impl reference`` times the CPU rendition of the reference's algorithm
(the oracle port; the reference itself cannot be built) with all host threads
on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DEM cells/s batched vs plain GPU NNI at ≤1e-4 m err vs FP64; p50/p99 tile latency"
UNIT = "cells/s"
KERNELS_PER_CALL = 16      # own kernel launches per single-work-package call with points
KERNELS_PER_BATCH = 15     # per batch run (the bounding boxes come with the bin counts)
FALLBACK_HBM_GBS = 6650.0
BASE_SEED = 20261203


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--workload", choices=["mixed", "tile4096", "segment", "served", "spacetime", "compat"], default="mixed")
    ap.add_argument("--cp-side", type=int, default=2000, help="compat: work-package side in cells (2 m)")
    ap.add_argument("--cp-points", type=int, default=16_000_000, help="compat: points")
    ap.add_argument("--st-side", type=int, default=4096, help="spacetime: grid side in cells (1 m)")
    ap.add_argument("--st-points", type=int, default=36_000_000, help="spacetime: points over all time values")
    ap.add_argument("--st-radius", type=int, default=2, help="spacetime: time radius (slices 2r+1)")
    ap.add_argument("--srv-points", type=int, default=2_000_000_000, help="served: cloud points")
    ap.add_argument("--srv-side", type=float, default=64000.0, help="served: cloud side, metres")
    ap.add_argument("--srv-requests", type=int, default=200, help="served: requests per arrival rate")
    ap.add_argument("--srv-rates", default="20,100,1000,20000", help="served: Poisson arrival rates, 1/s")
    ap.add_argument("--srv-block-side", type=float, default=16000.0,
                    help="mixed: side (m) of the cloud of the served block in the default line (0: none)")
    ap.add_argument("--srv-block-requests", type=int, default=48, help="mixed: requests per rate of the served block")
    ap.add_argument("--srv-block-rates", default="100,2000", help="mixed: arrival rates of the served block")
    ap.add_argument("--seg-side", type=int, default=32768, help="segment: grid side in cells (1 m)")
    ap.add_argument("--seg-points", type=int, default=1_500_000_000, help="segment: points")
    ap.add_argument("--seg-tile", type=int, default=2048)
    ap.add_argument("--seg-halo", type=int, default=0,
                    help="segment: first raster halo tried (cells); 0 = bound from block occupancy")
    ap.add_argument("--seg-batch", type=int, default=64, help="segment: tiles per batch")
    ap.add_argument("--tiles", type=int, default=4096, help="tiles of the mixed workload")
    ap.add_argument("--plain-steps", type=int, default=2,
                    help="timed passes of the plain per-tile form (0: skip the plain form)")
    ap.add_argument("--side", type=int, default=4096)
    ap.add_argument("--points", type=int, default=20_000_000)
    ap.add_argument("--cpu-window", type=int, default=2048, help="side of the CPU baseline sample window")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--small-radius", type=int, default=0)
    ap.add_argument("--bin-target", type=int, default=0)
    ap.add_argument("--span-window", type=int, default=0,
                    help="64-bit words of shared memory per raster tile for the span window (0 = default)")
    ap.add_argument("--no-autotune", action="store_true", help="mixed: skip the autotuner (context defaults)")
    ap.add_argument("--tune-sample", type=int, default=256, help="mixed: tiles the autotuner times")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, which):
        """Record the start or end of the timed region (host clock)."""
        setattr(self, which, time.time())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        """Samples that arrived inside the timed region (the nearest one when
        the region is shorter than the 200 ms sampling period)."""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = getattr(self, "t_start", 0.0), getattr(self, "t_end", float("inf"))
        inside = [ln for ts, ln in self.lines if t0 <= ts <= t1 + 0.2]
        if not inside and self.lines:
            inside = [min(self.lines, key=lambda x: abs(x[0] - t1))[1]]
        for ln in inside:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def host_cpu():
    """The host's CPU model and logical core count, for the CPU baselines."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count()}


def dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def workload(side, npts, seed):
    from terranni_b200 import synth
    w = synth.config2(seed=seed, n=npts, side=side)
    return w["xyz"]


def cpu_baseline(xyz, side, window, seed_note):
    """Oracle port, one thread, on a window of the same tile (its own work
    package: the window's cells, the points inside it)."""
    from oracle import oracle
    lo, hi = 0, window * 100
    m = (xyz[:, 0] >= lo) & (xyz[:, 0] < hi) & (xyz[:, 1] >= lo) & (xyz[:, 1] < hi)
    sub = xyz[m]
    wp = oracle.make_wp(window, window, 100, origin_x=lo, origin_y=lo)
    t0 = time.perf_counter()
    oracle.interpolate(wp, sub)
    dt = time.perf_counter() - t0
    return {"value": window * window / dt, "unit": UNIT, "cores": 1, "kind": "port", "host": host_cpu(),
            "sample": f"{window}x{window}-cell lower-left window ({sub.shape[0]} points) of the {seed_note}; "
                      f"single-thread C oracle (k-d tree nearest site + row-span scatter), {dt:.2f} s"}


OPS_PER_EVAL = 5   # a candidate evaluation: 2 subtractions, 1 multiply, 1 multiply-add, 1 compare


def ops_roofline(peaks, evals_dense, evals_far, spans, ms_dense, ms_far, ms_spans):
    """Op-count rooflines of the three kernels that dominate a step, against
    the device's measured throughput of the operation bounding each
    (dnni_measure_peaks): integer ops of the distance evaluations for the
    nearest-site kernels, shared-memory atomics of the span window (two per
    marker, two markers per span row; rows clipped by the grid included)."""
    def one(work, ms, peak, unit, note):
        ach = work / (ms / 1000.0) if ms > 0 else 0.0
        return {"work": int(work), "ms": round(ms, 3), "achieved": ach, "peak": peak, "unit": unit,
                "frac_ops": ach / peak if peak else None, "work_def": note}
    return {
        "peaks_measured": peaks,
        "k_near_dense": one(OPS_PER_EVAL * evals_dense, ms_dense, peaks["int_ops_per_s"], "int32 ops/s",
                            f"{OPS_PER_EVAL} integer ops per candidate distance evaluation"),
        "k_near_far": one(OPS_PER_EVAL * evals_far, ms_far, peaks["int_ops_per_s"], "int32 ops/s",
                          f"{OPS_PER_EVAL} integer ops per candidate distance evaluation (seeds and disc search)"),
        "k_scatter_window": one(4 * spans, ms_spans, peaks["smem_atomics_per_s"], "smem atomics/s",
                                "4 shared-memory atomic adds per span row (z and count at both ends)"),
    }


def fp64_errors(oracle, ref, h, z_scale=0.01, z_offset=0.0):
    """Max and RMS |h - h_FP64| over the cells with data, h_FP64 from the
    oracle's exact integer sums (the FP64 checker)."""
    import numpy as np
    ok = ref["C"] > 0
    truth = oracle.exact_height_f64(ref["Z"][ok], ref["C"][ok], z_scale, z_offset)
    e = np.abs(np.asarray(h)[ok].astype(np.float64) - truth)
    return float(e.max(initial=0.0)), float(np.sqrt(np.mean(e * e))) if e.size else 0.0


def window_accuracy(oracle, h_grid, xyz, x0, y0, win, halo, cell=100, origin=(0, 0)):
    """Checks the cells [x0, x0+win) x [y0, y0+win) of a grid that one work
    package over the whole grid defines (raster = grid) against the oracle's
    work package over those cells alone, with a raster `halo` cells wider on
    each side (every pixel whose disc can reach them, for halos above the
    largest disc radius) and the points within twice the halo (every pixel's
    nearest site): heights bit for bit and their FP64 error."""
    import numpy as np
    ox, oy = origin[0] + x0 * cell, origin[1] + y0 * cell
    lo_x, hi_x = ox - 2 * halo * cell, ox + (win + 2 * halo) * cell
    lo_y, hi_y = oy - 2 * halo * cell, oy + (win + 2 * halo) * cell
    sel = (xyz[:, 0] >= lo_x) & (xyz[:, 0] < hi_x) & (xyz[:, 1] >= lo_y) & (xyz[:, 1] < hi_y)
    wp = oracle.make_wp(win, win, cell, ox, oy, raster=(-halo, -halo, win + halo, win + halo))
    ref = oracle.interpolate(wp, xyz[sel])
    g = np.ascontiguousarray(h_grid[y0:y0 + win, x0:x0 + win])
    mx, rms = fp64_errors(oracle, ref, g)
    return {"window": [int(x0), int(y0), int(win)], "halo_cells": int(halo), "points": int(sel.sum()),
            "bit_exact_vs_oracle": bool(np.array_equal(g.view(np.uint32), ref["h"].view(np.uint32))),
            "max_abs_err_m": mx, "rms_err_m": rms}


def depth_disagreement(oracle, cases, budget_s, max_pixels=2_000_000, max_side=384):
    """The reference's site choice by float32 lifted-plane depth in a 32-bit
    depth buffer (GL_DEPTH_COMPONENT32, nni.cpp:420-424; emulated by the
    oracle, LEQUAL with the later-drawn site winning) against the exact
    nearest site, over (wp, xyz) cases of at most max_side cells a side until
    the budget or the pixel count is spent: fractions of raster pixels.  The
    emulation considers the sites whose exact squared distance lies within
    2^-15 * halfwidth^2 of the nearest one; float32 depths (values up to 8,
    a few ulp of error) cannot order sites much closer than that."""
    pix = site = zd = 0
    used = 0
    sides = []
    t0 = time.perf_counter()
    for wp, xyz in cases:
        if time.perf_counter() - t0 >= budget_s or pix >= max_pixels:
            break
        if max(wp.ncols, wp.nrows) > max_side:
            continue
        hw = (wp.nrows - 1) * wp.cell_size / 2.0
        slack = int(max(2.0 ** -15 * hw * hw, 4.0 * wp.cell_size * wp.cell_size))
        r = oracle.gl_disagreement(wp, xyz, depth_bits=32, slack_units2=slack)
        pix += r["pixels"]
        site += r["site_differs"]
        zd += r["z_differs"]
        used += 1
        sides.append(int(wp.ncols))
    n = max(pix, 1)
    return {"cases": used, "pixels": pix, "site_frac": site / n, "z_frac": zd / n, "depth_bits": 32,
            "tile_sides": sides, "seconds": round(time.perf_counter() - t0, 1)}


def run_reference_tile4096(args, world, rank):
    """CPU rendition of the reference's algorithm with all host threads."""
    if rank != 0:
        return
    import concurrent.futures as cf
    import numpy as np
    from oracle import oracle
    nthreads = os.cpu_count() or 1
    xyz = workload(args.side, args.points, 20261203 + 2)
    win = min(args.cpu_window, 1024, args.side)
    nwx = args.side // win
    windows = [(i % nwx, (i // nwx) % nwx) for i in range(nthreads)]
    # partition the points once, outside the timed region
    wid = (xyz[:, 1] // (win * 100)) * nwx + xyz[:, 0] // (win * 100)
    parts = {}
    for (i, j) in set(windows):
        parts[(i, j)] = np.ascontiguousarray(xyz[wid == j * nwx + i])

    def job(wij):
        i, j = wij
        wp = oracle.make_wp(win, win, 100, origin_x=i * win * 100, origin_y=j * win * 100)
        oracle.interpolate(wp, parts[(i, j)])
        return win * win

    times = []
    with cf.ThreadPoolExecutor(nthreads) as ex:
        for step in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            cells = sum(ex.map(job, windows))
            dt = time.perf_counter() - t0
            if step >= args.warmup:
                times.append((cells, dt))
    cells = sum(c for c, _ in times)
    tot = sum(d for _, d in times)
    v = cells / tot
    sample = (f"{nthreads} concurrent {win}x{win}-cell windows of the {args.side}x{args.side} tile per step "
              f"(one work package each), C oracle on {nthreads} host threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * tot / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": "tile4096", "side": args.side, "points": args.points, "cell_m": 1.0},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "host": host_cpu(),
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_engine_tile4096(args, world, rank, local):
    import numpy as np
    import torch
    from terranni_b200 import engine

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            import torch.distributed as tdist
            tdist.barrier()

    side, npts = args.side, args.points
    seed = 20261203 + 2 + rank
    xyz = workload(side, npts, seed)
    cells = side * side
    wp = engine.make_wp(side, side, 100)
    eng = engine.Engine(device=local, flags=engine.F_TIMING)
    d_xyz = torch.from_numpy(xyz).cuda()
    d_h = torch.empty((side, side), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()           # the engine launches on exactly this stream
    sp = stream.cuda_stream

    phases = []
    with ClockSampler(local) as clk:
        for _ in range(args.warmup):
            eng.interpolate_device(wp, d_xyz, npts, d_h, stream=sp, stats=True)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clk.mark("t_start")
        ev0.record(stream)
        for _ in range(args.steps):
            eng.interpolate_device(wp, d_xyz, npts, d_h, stream=sp, stats=False)
        ev1.record(stream)
        torch.cuda.synchronize()
        clk.mark("t_end")
    barrier()
    # per-phase device times and counts from untimed calls with statistics
    for _ in range(2):
        phases.append(eng.interpolate_device(wp, d_xyz, npts, d_h, stream=sp, stats=True))
    ms = ev0.elapsed_time(ev1)
    ms_t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        import torch.distributed as tdist
        tdist.all_reduce(ms_t, op=tdist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = cells * args.steps * world / (ms_max / 1000.0)

    # end to end through the host-buffer call, pinned host memory
    h_xyz = torch.from_numpy(xyz).pin_memory()
    h_out = torch.empty((side, side), dtype=torch.float32).pin_memory()
    xyz_p, out_p = h_xyz.numpy(), h_out.numpy()
    for _ in range(max(1, args.warmup)):
        eng.interpolate(wp, xyz_p, out_h=out_p)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.interpolate(wp, xyz_p, out_h=out_p)
    e2e_s = time.perf_counter() - t0
    e_t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if world > 1:
        import torch.distributed as tdist
        tdist.all_reduce(e_t, op=tdist.ReduceOp.MAX)
        barrier()
    e2e_value = cells * args.steps * world / float(e_t.item())
    nod = int(np.count_nonzero(out_p == np.float32(-9999.0)))

    if rank == 0:
        peak, peak_kind = peaks()
        ms_step = ms_max / args.steps
        ph = {k: sum(getattr(p, k) for p in phases) / len(phases)
              for k in ("ms_bin", "ms_nearest", "ms_dense", "ms_far", "ms_scatter", "ms_finalize", "ms_total")}
        last = phases[-1]
        ops = ops_roofline(engine.measure_peaks(local), last.evals_dense, last.evals_far, last.spans, ph["ms_dense"],
                           ph["ms_far"], ph["ms_scatter"])
        alg_bytes = 12 * npts + 4 * cells
        achieved = alg_bytes / (ms_step / 1000.0) / 1e9
        dom = max(("ms_bin", "ms_nearest", "ms_scatter", "ms_finalize"), key=lambda k: ph[k])
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic_tile4096.json")
        if os.path.exists(tp):
            traffic = json.load(open(tp)).get("dram_bytes_per_step")
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32/int64", "data": "synthetic (seeded fBm terrain, clusters, lakes)",
            "config": {"workload": "tile4096", "side": side, "cell_m": 1.0, "points": npts, "cells": cells,
                       "form": "plain per-tile (one work package per call)",
                       "l2": "inputs larger than L2 (240 MB points, ~1 GB scratch per step)",
                       "parallelism": f"dp{world} (independent tiles)"},
            "roofline": {"bound": "hbm", "kernel": f"whole hot path per tile ({KERNELS_PER_CALL} launches)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic,
                         "algorithmic_bytes": alg_bytes, "dominant_phase": dom,
                         "phase_ms": {k: round(v, 4) for k, v in ph.items()}, "ops": ops},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(xyz.nbytes),
                    "d2h_bytes_per_step": int(cells * 4)},
            "gpu_launches": KERNELS_PER_CALL * args.steps,
            "clocks": clk.summary(),
            "work": {"span_pixels": phases[-1].big_pixels, "spans": phases[-1].spans,
                     "max_r2": phases[-1].max_r2, "packed": phases[-1].packed, "bin_size": phases[-1].bin_size,
                     "nodata_cells": nod},
        }
        if not args.no_cpu_baseline:
            from oracle import oracle
            out["cpu_baseline"] = cpu_baseline(xyz, side, min(args.cpu_window, side), "same tile")
            # the whole tile against the oracle (one work package, as run)
            ref = oracle.interpolate(oracle.make_wp(side, side, 100), xyz)
            mx, rms = fp64_errors(oracle, ref, out_p)
            out["accuracy"] = {"cells_checked": cells, "bit_exact_vs_oracle":
                               bool(np.array_equal(out_p.view(np.uint32), ref["h"].view(np.uint32))),
                               "max_abs_err_m": mx, "rms_err_m": rms}
            del ref
            win = 256
            sub = xyz[(xyz[:, 0] < win * 100) & (xyz[:, 1] < win * 100)]
            out["ref_depth_disagreement"] = depth_disagreement(
                oracle, [(oracle.make_wp(win, win, 100), sub)], 30.0)
        print(json.dumps(out), flush=True)
    eng.close()
    if world > 1:
        import torch.distributed as tdist
        tdist.destroy_process_group()


# ---------------------------------------------------------------------------
# mixed-tile batch
# ---------------------------------------------------------------------------

def mixed_workload(count, rank, pinned, world=1):
    """Specs, layout, points (absolute LAS xyz rows, pinned when asked) and
    per-tile point extents of this rank's share of the mixed batch: world x
    count tiles are drawn and split over the ranks by estimated cost
    (terranni_b200.shard), so each rank gets about `count` tiles."""
    import numpy as np
    from terranni_b200 import shard, synth
    specs = synth.mixed_tiles(count=count * world, seed=BASE_SEED + 4)
    if world > 1:
        parts = shard.partition_by_cost([shard.tile_cost(s["side"], s["side"], s["n"]) for s in specs], world)
        specs = [specs[k] for k in parts[rank]]
    lay, npt, nout = synth.mixed_layout(specs)
    if pinned:
        import torch
        h = torch.empty((max(npt, 1), 3), dtype=torch.int32, pin_memory=True)
        xyz = h.numpy()[:npt]
    else:
        h = None
        xyz = np.empty((npt, 3), np.int32)
    ext = synth.fill_mixed(specs, lay, xyz)
    return {"specs": specs, "lay": lay, "npt": npt, "nout": nout, "xyz": xyz, "ext": ext, "host": h}


def mixed_tiles_abi(w):
    from terranni_b200 import engine
    return [engine.make_tile(engine.make_wp(L["side"], L["side"], L["cell"], *L["origin"]), L["pt"], L["n"],
                             L["out"], -1, extent=w["ext"][k]) for k, L in enumerate(w["lay"])]


def sample_order(n):
    """Fixed visiting order of tiles for bounded CPU samples (a stride
    through the list, so the sample spans the size distribution)."""
    step = 97 if n > 97 else 1
    return [(k * step) % n for k in range(n)]


def cpu_baseline_mixed(w, h_gpu, budget_s):
    """Oracle port, one thread, on tiles of the same batch until the budget
    is spent; the same tiles' GPU heights are checked against it (bit-exact
    float32, and the error against the FP64 height)."""
    import numpy as np
    from oracle import oracle
    cells = 0
    spent = 0.0
    ntile = 0
    exact = True
    errs = []
    for k in sample_order(len(w["lay"])):
        if spent >= budget_s:
            break
        L = w["lay"][k]
        wp = oracle.make_wp(L["side"], L["side"], L["cell"], *L["origin"])
        pts = w["xyz"][L["pt"]:L["pt"] + L["n"]]
        t0 = time.perf_counter()
        r = oracle.interpolate(wp, pts)
        spent += time.perf_counter() - t0
        cells += L["side"] * L["side"]
        ntile += 1
        g = h_gpu[L["out"]:L["out"] + L["side"] * L["side"]].reshape(L["side"], L["side"])
        exact &= bool(np.array_equal(g.view(np.uint32), r["h"].view(np.uint32)))
        ok = r["C"] > 0
        truth = oracle.exact_height_f64(r["Z"][ok], r["C"][ok], wp.z_scale, wp.z_offset)
        errs.append(np.abs(g[ok].astype(np.float64) - truth))
    e = np.concatenate(errs) if errs else np.zeros(1)
    acc = {"tiles_checked": ntile, "cells_checked": cells, "bit_exact_vs_oracle": exact,
           "max_abs_err_m": float(e.max(initial=0.0)), "rms_err_m": float(np.sqrt(np.mean(e * e)))}
    base = {"value": cells / spent, "unit": UNIT, "cores": 1, "kind": "port", "host": host_cpu(),
            "sample": f"{ntile} tiles ({cells} cells) of the same batch in a fixed stride order, "
                      f"single-thread C oracle (k-d tree nearest site + row-span scatter), {spent:.1f} s"}
    return base, acc


def run_reference_mixed(args, world, rank):
    """CPU rendition of the reference's algorithm, all host threads, one tile
    per thread at a time, on a fixed sample of the batch per step."""
    if rank != 0:
        return
    import concurrent.futures as cf
    from oracle import oracle
    nthreads = os.cpu_count() or 1
    w = mixed_workload(args.tiles, 0, pinned=False)
    order = sample_order(len(w["lay"]))
    # about 1.5 s of work per step on this many threads (oracle ~0.6 M cells/s
    # per thread on these tiles)
    target = int(1.5 * 0.6e6 * nthreads)
    sample, cells = [], 0
    for k in order:
        if cells >= target:
            break
        sample.append(k)
        cells += w["lay"][k]["side"] ** 2

    def job(k):
        L = w["lay"][k]
        wp = oracle.make_wp(L["side"], L["side"], L["cell"], *L["origin"])
        oracle.interpolate(wp, w["xyz"][L["pt"]:L["pt"] + L["n"]])
        return L["side"] ** 2

    times = []
    with cf.ThreadPoolExecutor(nthreads) as ex:
        for step in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            c = sum(ex.map(job, sample))
            dt = time.perf_counter() - t0
            if step >= args.warmup:
                times.append((c, dt))
    tot = sum(d for _, d in times)
    v = sum(c for c, _ in times) / tot
    desc = (f"{len(sample)} tiles ({cells} cells) of the {args.tiles}-tile batch per step, fixed stride order, "
            f"C oracle on {nthreads} host threads (one tile per thread at a time)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * tot / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": {"workload": f"mixed{args.tiles}", "tiles": args.tiles, "sample_tiles": len(sample)},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "host": host_cpu(),
                         "sample": desc},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def _pct(v, q):
    import numpy as np
    return float(np.percentile(np.asarray(v, dtype=np.float64), q)) if len(v) else None


def run_engine_mixed(args, world, rank, local):
    import numpy as np
    import torch
    from terranni_b200 import engine

    torch.cuda.set_device(local)
    tdist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if tdist is not None:
            tdist.barrier()

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        if tdist is not None:
            tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        return float(t.item())

    w = mixed_workload(args.tiles, rank, pinned=True, world=world)
    npt, nout, xyz = w["npt"], w["nout"], w["xyz"]
    tiles = mixed_tiles_abi(w)
    eng = engine.Engine(device=local)
    d_xyz = torch.from_numpy(xyz).cuda()
    d_h = torch.empty(max(nout, 1), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()           # the engine launches on exactly this stream
    sp = stream.cuda_stream
    opts = dict(small_radius=args.small_radius, bin_target=args.bin_target, span_window=args.span_window)
    tune = None
    if not args.no_autotune:              # outside the timed region
        t0 = time.perf_counter()
        opts, rep = eng.autotune(tiles, d_xyz, sample_tiles=args.tune_sample, **opts)
        tune = {"sample_tiles": rep["sample_tiles"], "ms_default": rep["ms_default"], "best": rep["best"],
                "trials": len(rep["trials"]), "seconds": time.perf_counter() - t0}

    # batched form: one graph-captured launch sequence per step
    b = eng.batch(tiles, use_graph=True, order_by_cost=True, **opts)
    st0 = b.run_device(d_xyz, d_h, stream=sp, stats=True)       # first warm-up: checks extents, captures
    for _ in range(max(args.warmup - 1, 0)):
        b.run_device(d_xyz, d_h, stream=sp)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        clk.mark("t_start")
        evs[0].record(stream)
        for k in range(args.steps):
            b.run_device(d_xyz, d_h, stream=sp)
            evs[k + 1].record(stream)
        torch.cuda.synchronize()
        clk.mark("t_end")
    barrier()
    step_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    ms_max = max_over_ranks(evs[0].elapsed_time(evs[-1]))
    value = nout * args.steps * world / (ms_max / 1000.0)
    b.close()

    # per-phase device times from one run without the graph, and the
    # measured peaks of the operations that bound the largest kernels
    with eng.batch(tiles, use_graph=False, order_by_cost=True, **opts) as bp:
        bp.run_device(d_xyz, d_h, stream=sp)
        ph = bp.run_device(d_xyz, d_h, stream=sp, stats=True)
    phases = {k: round(getattr(ph, k), 4) for k in ("ms_bin", "ms_nearest", "ms_dense", "ms_far", "ms_scatter",
                                                     "ms_finalize", "ms_total")}
    ops = ops_roofline(engine.measure_peaks(local), ph.evals_dense, ph.evals_far, ph.spans, ph.ms_dense, ph.ms_far,
                       ph.ms_scatter)

    # plain form: one dnni_interpolate_segment_device call per tile, same
    # tiles, same stream, no statistics (the call's only wait is the one it
    # needs, for the bounding box that sizes its bins); one event pair around
    # each pass over the tiles
    d_hp = torch.empty(max(nout, 1), dtype=torch.float32, device="cuda")
    wps = [engine.make_wp(L["side"], L["side"], L["cell"], *L["origin"]) for L in w["lay"]]
    base_xyz, base_h = d_xyz.data_ptr(), d_hp.data_ptr()
    tile_ms, plain_ms = [], []
    pa, pb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for rnd in range(1 + args.plain_steps if args.plain_steps > 0 else 0):
        torch.cuda.synchronize()
        barrier()
        pa.record(stream)
        for L, wp in zip(w["lay"], wps):
            eng.interpolate_device(wp, base_xyz + 12 * L["pt"], L["n"], base_h + 4 * L["out"], stream=sp,
                                   stats=False)
        pb.record(stream)
        torch.cuda.synchronize()
        if rnd:
            plain_ms.append(pa.elapsed_time(pb))
    # per-tile latency of the plain form, in a separate untimed pass: from the
    # call to the tile's completion on the device
    if args.plain_steps > 0:
        for L, wp in zip(w["lay"], wps):
            t0 = time.perf_counter()
            eng.interpolate_device(wp, base_xyz + 12 * L["pt"], L["n"], base_h + 4 * L["out"], stream=sp,
                                   stats=False)
            stream.synchronize()
            tile_ms.append(1e3 * (time.perf_counter() - t0))
    plain_max = max_over_ranks(sum(plain_ms))
    plain_value = nout * len(plain_ms) * world / (plain_max / 1000.0) if plain_ms else None
    same = bool(torch.equal(d_h.view(torch.int32), d_hp.view(torch.int32))) if plain_ms else None
    del d_hp

    # end to end: host-buffer batch call from pinned memory, graph replay
    h_out = torch.empty(max(nout, 1), dtype=torch.float32, pin_memory=True).numpy()
    with eng.batch(tiles, use_graph=True, order_by_cost=True, **opts) as be:
        for _ in range(max(1, args.warmup)):
            be.run(xyz, h_out, stats=False)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            be.run(xyz, h_out, stats=False)
        e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = nout * args.steps * world / e2e_s
    h_gpu = h_out[:nout].copy()
    nod = int(np.count_nonzero(h_gpu == np.float32(-9999.0)))
    served = None
    if world == 1 and args.srv_block_side > 0:
        # a bounded serving run beside the batch (outside its timed region)
        del d_xyz, d_h
        torch.cuda.empty_cache()
        eng.clear()
        served = served_block(eng, args, local)

    if rank == 0:
        peak, peak_kind = peaks()
        ms_step = ms_max / args.steps
        alg_bytes = 12 * npt + 4 * nout
        achieved = alg_bytes / (ms_step / 1000.0) / 1e9
        dom = max(("ms_bin", "ms_nearest", "ms_scatter", "ms_finalize"), key=lambda k: phases[k])
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic_mixed4096.json")
        if os.path.exists(tp):
            traffic = json.load(open(tp)).get("dram_bytes_per_step")
        sides = np.array([L["side"] for L in w["lay"]])
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32/int64", "data": "synthetic (seeded fBm terrain, clusters, lakes)",
            "config": {"workload": f"mixed{args.tiles}", "tiles": args.tiles, "cells": nout, "points": npt,
                       "side_min": int(sides.min()), "side_median": int(np.median(sides)),
                       "side_max": int(sides.max()),
                       "form": "batched: all tiles in one CUDA-graph launch sequence per step",
                       "small_radius": opts["small_radius"] or 3, "bin_target": opts["bin_target"] or 4,
                       "span_window": opts["span_window"] or 4096, "far_group": opts.get("far_group") or 2,
                       "dense_band": opts.get("dense_band") or 64,
                       "order_by_cost": True, "autotune": tune,
                       "l2": f"inputs larger than L2 ({xyz.nbytes / 1e9:.1f} GB points per step)",
                       "parallelism": f"dp{world} (independent tiles)"},
            "plain": {"value": plain_value, "unit": UNIT,
                      "ms_per_step": plain_max / len(plain_ms) if plain_ms else None,
                      "form": "one dnni_interpolate_segment_device call per tile (no statistics)",
                      "tile_ms_p50": _pct(tile_ms, 50), "tile_ms_p99": _pct(tile_ms, 99),
                      "batched_over_plain": value / plain_value if plain_value else None,
                      "heights_identical_to_batched": same},
            "latency": {"batch_ms_p50": _pct(step_ms, 50), "batch_ms_p99": _pct(step_ms, 99),
                        "note": "batched: every tile of a step completes with its batch"},
            "roofline": {"bound": "hbm", "kernel": f"whole hot path per batch ({KERNELS_PER_BATCH} launches)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic, "algorithmic_bytes": alg_bytes,
                         "dominant_phase": dom, "phase_ms": phases, "ops": ops},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(xyz.nbytes),
                    "d2h_bytes_per_step": int(nout * 4)},
            "gpu_launches": KERNELS_PER_BATCH * args.steps,
            "clocks": clk.summary(),
            "served": served,
            "work": {"span_pixels": st0.big_pixels, "spans": st0.spans, "max_r2": st0.max_r2,
                     "nodata_cells": nod, "evals_dense": ph.evals_dense, "evals_far": ph.evals_far,
                     "span_radius_hist": {"bucket_lo": [0] + [1 << (k - 1) for k in range(1, 16)],
                                          "spans": list(ph.span_hist)}},
        }
        if not args.no_cpu_baseline:
            from oracle import oracle
            out["cpu_baseline"], out["accuracy"] = cpu_baseline_mixed(w, h_gpu, args.cpu_seconds)
            cases = []
            for k in sample_order(len(w["lay"]))[:out["accuracy"]["tiles_checked"]]:
                L = w["lay"][k]
                cases.append((oracle.make_wp(L["side"], L["side"], L["cell"], *L["origin"]),
                              w["xyz"][L["pt"]:L["pt"] + L["n"]]))
            out["ref_depth_disagreement"] = depth_disagreement(oracle, cases, 0.5 * args.cpu_seconds)
        print(json.dumps(out), flush=True)
    eng.close()
    if tdist is not None:
        tdist.destroy_process_group()


# ---------------------------------------------------------------------------
# segment-streamed grid
# ---------------------------------------------------------------------------

def run_engine_segment(args, world, rank, local):
    """One side x side grid at 1 m from points in pinned host memory, through
    dnni_segment_run (upload, device bucketing, tiles with self-checked halos,
    download into the host grid).  Each step is one whole call, host to host.
    With N ranks the one grid is split: every rank holds the same cloud and
    runs its part of the tiles (a contiguous cost-balanced range, no
    collective on the data path); value = the grid's cells / the slowest
    rank's time (strong scaling)."""
    import numpy as np
    import torch
    from terranni_b200 import engine, synth

    torch.cuda.set_device(local)
    tdist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        if tdist is not None:
            tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        return float(t.item())

    side, n = args.seg_side, args.seg_points
    t0 = time.perf_counter()
    h_xyz = torch.empty((n, 3), dtype=torch.int32, pin_memory=True)
    xyz = h_xyz.numpy()
    synth.config3(seed=BASE_SEED + 3, n=n, side=side, out=xyz)
    h_out = torch.empty((side, side), dtype=torch.float32, pin_memory=True).numpy()
    gen_s = time.perf_counter() - t0
    eng = engine.Engine(device=local)
    kw = dict(tile=args.seg_tile, halo=args.seg_halo, tiles_per_batch=args.seg_batch, out_h=h_out,
              part=rank if world > 1 else 0, parts=world if world > 1 else 0)
    for _ in range(args.warmup):
        eng.segment_run(xyz, side, side, 100, **kw)
    stats = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if tdist is not None:
            tdist.barrier()
        clk.mark("t_start")
        t1 = time.perf_counter()
        for _ in range(args.steps):
            _, _, st = eng.segment_run(xyz, side, side, 100, **kw)
            stats.append(st)
        dt = time.perf_counter() - t1
        clk.mark("t_end")
    dt_max = max_over_ranks(dt)
    cells = side * side
    value = cells * args.steps / dt_max
    nod = int(np.count_nonzero(h_out == np.float32(-9999.0)))
    acc = None
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        # a window in the middle of the mosaic, across tile seams, against the
        # oracle's work package over it with a halo above the largest disc
        from oracle import oracle
        win = 256
        x0 = y0 = max(0, side // 2 - win // 2 - args.seg_tile // 2 + 7)
        acc = window_accuracy(oracle, h_out, xyz, x0, y0, min(win, side), halo=min(600, side // 2))
    if rank == 0:
        peak, peak_kind = peaks()
        ms_step = 1000 * dt_max / args.steps
        alg = 12 * n + 4 * cells
        achieved = alg / (ms_step / 1000) / 1e9
        st = stats[-1]
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "int32/int64", "data": "synthetic (seeded fBm terrain, clusters, lakes)",
            "config": {"workload": f"segment{side}", "side": side, "cell_m": 1.0, "points": n, "cells": cells,
                       "tile": args.seg_tile, "first_halo": args.seg_halo, "tiles_per_batch": args.seg_batch,
                       "form": "dnni_segment_run: pinned host points -> host grid, timed host to host",
                       "l2": f"inputs larger than L2 ({12 * n / 1e9:.1f} GB points per step)",
                       "parallelism": (f"{world} parts of one grid (tiles split by cost, each rank writes "
                                       f"its tiles; no collective on the data path)" if world > 1 else "1 GPU"),
                       "generate_s": round(gen_s, 1)},
            "segment": {k: (round(v, 3) if isinstance(v, float) else v) for k, v in st.as_dict().items()},
            "roofline": {"bound": "hbm", "kernel": "whole segment call, host to host", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": None, "algorithmic_bytes": alg},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": int(st.h2d_bytes),
                    "d2h_bytes_per_step": int(st.d2h_bytes),
                    "note": "the segment call is host to host: its value is already end to end"},
            # per call: bucket counts, two partition passes, bucket boxes and the
            # occupancy map; per batch: the gather, the batch's sequence and the
            # halo check
            "gpu_launches": int(sum(5 + x.batches * (KERNELS_PER_BATCH + 2) for x in stats)),
            "clocks": clk.summary(), "nodata_cells": nod, "accuracy": acc,
        }), flush=True)
    eng.close()
    if tdist is not None:
        tdist.destroy_process_group()


# ---------------------------------------------------------------------------
# spacetime: one grid at time cur from points of 4r+1 time values
# ---------------------------------------------------------------------------

def run_engine_spacetime(args, world, rank, local):
    """One side x side grid at 1 m, time radius r (2r+1 slices, one time step
    = 1 m), points spread evenly over the 4r+1 time values that reach it,
    through dnni_interpolate_spacetime from host buffers.  cpu_baseline: the
    oracle's space-time restatement on one thread over a window of the same
    cloud, checked bit-exact against the engine on that window."""
    import numpy as np
    import torch
    from oracle import oracle
    from terranni_b200 import engine, synth

    torch.cuda.set_device(local)
    side, n, rt = args.st_side, args.st_points, args.st_radius
    cur, tau = 100, 100
    t0 = time.perf_counter()
    xyz = torch.empty((n, 3), dtype=torch.int32, pin_memory=True).numpy()      # pinned host buffers
    tt = torch.empty(n, dtype=torch.int32, pin_memory=True).numpy()
    h = torch.empty((side, side), dtype=torch.float32, pin_memory=True).numpy()
    synth.config3(seed=BASE_SEED + 7 + 1000 * rank, n=n, side=side, out=xyz)
    tt[:] = np.random.default_rng(BASE_SEED + 8 + rank).integers(cur - 2 * rt, cur + 2 * rt + 1, n)
    gen_s = time.perf_counter() - t0
    eng = engine.Engine(device=local)
    wp = engine.make_wp(side, side, 100, raster=(-2, -2, side + 2, side + 2))
    for _ in range(args.warmup):
        eng.interpolate_spacetime(wp, xyz, tt, cur, rt, tau, out_h=h)
    stats = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        clk.mark("t_start")
        t1 = time.perf_counter()
        for _ in range(args.steps):
            _, st = eng.interpolate_spacetime(wp, xyz, tt, cur, rt, tau, out_h=h)
            stats.append(st)
        dt = time.perf_counter() - t1
        clk.mark("t_end")
    cells = side * side
    dev_ms = float(np.mean([x.ms_total for x in stats]))
    # CPU baseline and parity on a window of the same cloud (the oracle is
    # test infrastructure: here it only times and checks)
    cpu = acc = None
    if rank == 0 and not args.no_cpu_baseline:
        win = 512
        sel = (xyz[:, 0] < (win + 8) * 100) & (xyz[:, 1] < (win + 8) * 100)
        wwp_o = oracle.make_wp(win, win, 100, raster=(-2, -2, win + 2, win + 2))
        wwp_e = engine.make_wp(win, win, 100, raster=(-2, -2, win + 2, win + 2))
        tc = time.perf_counter()
        ref = oracle.interpolate_spacetime(wwp_o, xyz[sel], tt[sel], cur, rt, tau)
        cpu_s = time.perf_counter() - tc
        got, _ = eng.interpolate_spacetime(wwp_e, xyz[sel], tt[sel], cur, rt, tau)
        cpu = {"value": win * win / cpu_s, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"oracle space-time k-d restatement, one {win}x{win} window of the same cloud "
                         f"({int(sel.sum())} points), {cpu_s:.1f} s",
               "bit_exact_vs_engine": bool(np.array_equal(got.view(np.uint32), ref["h"].view(np.uint32)))}
        mx, rms = fp64_errors(oracle, ref, got)
        acc = {"cells_checked": win * win, "bit_exact_vs_oracle": cpu["bit_exact_vs_engine"],
               "max_abs_err_m": mx, "rms_err_m": rms,
               "note": "the engine on a window of the same cloud as its own work package"}
    if rank == 0:
        peak, peak_kind = peaks()
        ms_step = 1000 * dt / args.steps
        st = stats[-1]
        alg = 16 * n + 4 * cells
        print(json.dumps({
            "metric": METRIC, "value": cells * 1000.0 / dev_ms, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32/int64", "data": "synthetic (seeded fBm terrain, clusters, lakes)",
            "config": {"workload": f"spacetime{side}", "side": side, "cell_m": 1.0, "points": n, "time_radius": rt,
                       "slices": 2 * rt + 1, "time_values": 4 * rt + 1, "time_scale_las": tau,
                       "form": "dnni_interpolate_spacetime from pinned host buffers; value from its device events",
                       "l2": f"inputs larger than L2 ({16 * n / 1e9:.2f} GB points per step)",
                       "generate_s": round(gen_s, 1)},
            "stats": {"ms_values_batch": round(st.ms_bin, 3), "ms_lift": round(st.ms_nearest, 3),
                      "ms_spans": round(st.ms_scatter, 3), "ms_final": round(st.ms_finalize, 3),
                      "slice_pixels": int(st.n_pixels), "nodata_cells": int(st.nodata_cells)},
            "roofline": {"bound": "hbm", "kernel": "whole space-time call on the device", "achieved":
                         alg / (dev_ms / 1000) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (dev_ms / 1000) / 1e9 / peak, "peak_kind": peak_kind, "traffic": None,
                         "algorithmic_bytes": alg},
            "e2e": {"value": cells * args.steps / dt, "unit": UNIT, "h2d_bytes_per_step": int(st.h2d_bytes),
                    "d2h_bytes_per_step": int(st.d2h_bytes), "ms_per_step": ms_step,
                    "note": "host to host from pinned buffers (upload, grouping by time on the device, download)"},
            # per call: grouping (3), the per-value nearest-site batch (12), the
            # lift and packing decision (3), one span pass per slice, the row scan
            # and the gather-and-divide
            "gpu_launches": args.steps * (20 + 2 * rt + 1),
            "cpu_baseline": cpu, "accuracy": acc, "clocks": clk.summary(),
        }), flush=True)
    eng.close()


# ---------------------------------------------------------------------------
# compat: one work package in the reference's default semantics
# ---------------------------------------------------------------------------

def run_engine_compat(args, world, rank, local):
    """terranni's defaults (scaling 5, 2 m cells, site radius 5 m, query
    radius 4.99 m, pointMin 0, zMultiplier from the z range) on one side x side
    work package, through dnni_interpolate_compat from pinned host buffers.
    cpu_baseline: the oracle's compat restatement on one thread over a window
    of the same cloud, checked bit-exact against the engine there."""
    import numpy as np
    import torch
    from oracle import oracle
    from terranni_b200 import engine, synth

    torch.cuda.set_device(local)
    side, n = args.cp_side, args.cp_points
    cell, scale, sr, qr = 2.0, 5, 5.0, 5 * 2.0 / 2.0 - 0.01
    t0 = time.perf_counter()
    raw = synth.config3(seed=BASE_SEED + 9 + 1000 * rank, n=n, side=int(side * cell))["xyz"]
    pts = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    pts[:] = raw * 0.01
    h = torch.empty((side, side), dtype=torch.float32, pin_memory=True).numpy()
    gen_s = time.perf_counter() - t0
    mult = oracle.compat_multiplier(sr, scale, cell, float(pts[:, 2].max()), 0)
    kw = dict(scale=scale, cell_size=cell, site_radius=sr, query_radius=qr, point_min=0, multiplier=mult)
    se = engine.CompatSettings(total_ncols=side, total_nrows=side, **kw)
    we = engine.CompatWP(nrows=side, ncols=side)
    eng = engine.Engine(device=local)
    for _ in range(args.warmup):
        eng.interpolate_compat(se, we, pts)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        clk.mark("t_start")
        t1 = time.perf_counter()
        for _ in range(args.steps):
            h[:], _ = eng.interpolate_compat(se, we, pts)
        dt = time.perf_counter() - t1
        clk.mark("t_end")
    cpu = acc = None
    if rank == 0 and not args.no_cpu_baseline:
        win = 250
        sel = (pts[:, 0] < (win + 8) * cell) & (pts[:, 1] < (win + 8) * cell)
        so = oracle.CompatSettings(total_ncols=win, total_nrows=win, **kw)
        wo = oracle.CompatWP(origin_x=0.0, origin_y=0.0, grid_origin_x=0.0, grid_origin_y=0.0, nrows=win, ncols=win)
        tc = time.perf_counter()
        ref, _ = oracle.compat(so, wo, pts[sel])
        cpu_s = time.perf_counter() - tc
        got, _ = eng.interpolate_compat(engine.CompatSettings(total_ncols=win, total_nrows=win, **kw),
                                        engine.CompatWP(nrows=win, ncols=win), pts[sel])
        cpu = {"value": win * win / cpu_s, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"oracle compat restatement, one {win}x{win} window of the same cloud "
                         f"({int(sel.sum())} points), {cpu_s:.1f} s",
               "bit_exact_vs_engine": bool(np.array_equal(got.view(np.uint32), ref.view(np.uint32)))}
        acc = {"cells_checked": win * win, "bit_exact_vs_oracle": cpu["bit_exact_vs_engine"],
               "note": "reference-default semantics: heights carry the reference's own zMultiplier "
                       "quantisation and truncating divide, so no FP64 error is stated"}
    if rank == 0:
        peak, peak_kind = peaks()
        cells = side * side
        ms_step = 1000 * dt / args.steps
        po = int(np.ceil((qr - 2 * cell / scale) / (cell / scale))) + 1
        pix = (side * scale + 2 * po) ** 2
        alg = 24 * n + 8 * pix + 4 * cells
        print(json.dumps({
            "metric": METRIC, "value": cells * 1000.0 / ms_step, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32/f64/int32", "data": "synthetic (seeded fBm terrain, clusters, lakes)",
            "config": {"workload": f"compat{side}", "side": side, "cell_m": cell, "scale": scale, "points": n,
                       "site_radius_m": sr, "query_radius_m": qr, "multiplier": mult, "raster_pixels": pix,
                       "form": "dnni_interpolate_compat from pinned host buffers, timed host to host",
                       "generate_s": round(gen_s, 1)},
            "roofline": {"bound": "hbm", "kernel": "whole compat call, host to host", "achieved":
                         alg / (ms_step / 1000) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (ms_step / 1000) / 1e9 / peak, "peak_kind": peak_kind, "traffic": None,
                         "algorithmic_bytes": alg},
            "e2e": {"value": cells * 1000.0 / ms_step, "unit": UNIT, "h2d_bytes_per_step": 24 * n,
                    "d2h_bytes_per_step": 4 * cells, "note": "the call is host to host"},
            "gpu_launches": 5 * args.steps, "cpu_baseline": cpu, "accuracy": acc, "clocks": clk.summary(),
        }), flush=True)
    eng.close()


# ---------------------------------------------------------------------------
# served: DEM requests against a resident cloud
# ---------------------------------------------------------------------------

def serve_rates(srv, reqs, outs, rates, rng, max_over_ranks=lambda x: x, world=1, barrier=None):
    """For each arrival rate, a Poisson stream of the requests submitted by a
    client thread at their arrival times and collected in order; latency =
    submit -> heights in host memory.  Per rate: cells/s over the stream's
    span, p50/p99/max latency, mean batch size, the median queueing delay,
    and the device time line of the server's slots over the stream (time
    busy, time with two or more slots' batches running at once)."""
    import numpy as np
    sizes = [r["ncols"] * r["nrows"] for r in reqs]
    results = []
    for rate in rates:
        if barrier is not None:
            barrier()
        st0 = srv.stats()
        gaps = rng.exponential(1.0 / rate, len(reqs))
        arrive = np.cumsum(gaps) - gaps[0]
        tickets = [None] * len(reqs)
        lat = [None] * len(reqs)
        ready = threading.Semaphore(0)

        def client():
            base = time.perf_counter()
            for k, r in enumerate(reqs):
                d = base + arrive[k] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets[k] = srv.submit(**r, out_h=outs[k])
                ready.release()

        c = threading.Thread(target=client)
        t_first = time.perf_counter()
        c.start()
        for k in range(len(reqs)):
            ready.acquire()
            _, _, res = srv.wait(tickets[k], timeout=600)
            lat[k] = res
        t_last = time.perf_counter()
        c.join()
        st1 = srv.stats()
        span = max_over_ranks(t_last - t_first)
        cells = sum(sizes)
        ms = np.array([x["ms_latency"] for x in lat])
        busy = st1["ms_device_busy"] - st0["ms_device_busy"]
        overlap = st1["ms_device_overlap"] - st0["ms_device_overlap"]
        results.append({"rate_per_s": rate, "requests": len(reqs), "cells": cells,
                        "cells_per_s": cells * world / span, "p50_ms": float(np.percentile(ms, 50)),
                        "p99_ms": float(np.percentile(ms, 99)), "max_ms": float(ms.max()),
                        "mean_batch": float(np.mean([x["batch_size"] for x in lat])),
                        "queue_p50_ms": float(np.percentile([x["ms_queue"] for x in lat], 50)),
                        "device_busy_frac": busy / (1000.0 * span) if span > 0 else None,
                        "slot_overlap_frac": overlap / busy if busy > 0 else 0.0})
    return results


def served_block(eng, args, local):
    """A bounded serving run for the default bench line: a cloud at the
    served configuration's density (0.49 points/m^2, fBm terrain, clusters,
    lakes of 50-400 m) over a smaller area, requests drawn as there (side
    log-uniform 128 m - 8 km, capped by the area; 0.5/1/2 m cells) at two
    Poisson rates, and two served windows checked against the oracle."""
    import numpy as np
    import torch
    from terranni_b200 import synth
    side_m, n = args.srv_block_side, int(round(0.4883 * args.srv_block_side ** 2))
    t0 = time.perf_counter()
    xyz = torch.empty((n, 3), dtype=torch.int32, pin_memory=True).numpy()
    synth.config5(seed=BASE_SEED + 15, n=n, side_m=side_m, out=xyz)
    gen_s = time.perf_counter() - t0
    reqs = synth.served_requests(args.srv_block_requests, seed=BASE_SEED + 16, side_m=side_m)
    sizes = [r["ncols"] * r["nrows"] for r in reqs]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    pool = torch.empty(int(offs[-1]), dtype=torch.float32, pin_memory=True).numpy()
    outs = [pool[offs[k]:offs[k + 1]].reshape(reqs[k]["nrows"], reqs[k]["ncols"]) for k in range(len(reqs))]
    rates = [float(x) for x in args.srv_block_rates.split(",") if x]
    with eng.server(xyz) as srv:
        for k in range(min(3, len(reqs))):                     # warm-up
            srv.wait(srv.submit(**reqs[k], out_h=outs[k]), timeout=600)
        results = serve_rates(srv, reqs, outs, rates, np.random.default_rng(BASE_SEED + 17))
        st = srv.stats()
    acc = None if args.no_cpu_baseline else served_accuracy(reqs, outs, xyz, 2)
    return {"cloud_points": n, "cloud_side_m": side_m, "requests_per_rate": len(reqs),
            "mean_request_cells": float(np.mean(sizes)), "generate_s": round(gen_s, 1),
            "form": "continuous batching over 2 slots, footprint admission; latency = submit to heights in host memory",
            "rates": results, "server": st, "accuracy": acc}


def served_accuracy(reqs, outs, xyz, count, reach_m=450.0, win=128):
    """The lower-left win x win cells of the `count` smallest requests whose
    window, with a raster halo of reach_m (above the largest nearest-site
    distance of the cloud's lakes) on every side, lies inside the cloud's box,
    checked against the oracle (window_accuracy); a request's result is the
    window of the interpolation over the whole cloud on its lattice."""
    from oracle import oracle
    wx0, wx1 = int(xyz[:, 0].min()), int(xyz[:, 0].max())
    wy0, wy1 = int(xyz[:, 1].min()), int(xyz[:, 1].max())
    checks = []
    for k in sorted(range(len(reqs)), key=lambda k: reqs[k]["ncols"] * reqs[k]["nrows"]):
        r = reqs[k]
        cs = r["cell_size"]
        halo = int(-(-reach_m * 100 // cs))
        w = min(win, r["ncols"], r["nrows"])
        if (r["x0"] - halo * cs < wx0 or r["y0"] - halo * cs < wy0 or r["x0"] + (w + halo) * cs > wx1 or
                r["y0"] + (w + halo) * cs > wy1):
            continue
        c = window_accuracy(oracle, outs[k], xyz, 0, 0, w, halo, cell=cs, origin=(r["x0"], r["y0"]))
        c["request"] = k
        checks.append(c)
        if len(checks) == count:
            break
    if not checks:
        return None
    return {"windows": checks, "bit_exact_vs_oracle": all(c["bit_exact_vs_oracle"] for c in checks),
            "max_abs_err_m": max(c["max_abs_err_m"] for c in checks),
            "rms_err_m": max(c["rms_err_m"] for c in checks)}


def run_engine_served(args, world, rank, local):
    """A resident cloud on each GPU (per-rank seed) and a Poisson stream of
    box requests per arrival rate, submitted by a client thread at their
    arrival times and collected by another; latency = submit -> heights in
    (pinned) host memory.  Each rank serves its own stream."""
    import numpy as np
    import torch
    from terranni_b200 import engine, synth

    torch.cuda.set_device(local)
    tdist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))

    def max_over_ranks(x):
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        if tdist is not None:
            tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        return float(t.item())

    n = args.srv_points
    t0 = time.perf_counter()
    h_xyz = torch.empty((n, 3), dtype=torch.int32, pin_memory=True)
    xyz = h_xyz.numpy()
    synth.config5(seed=BASE_SEED + 5 + 1000 * rank, n=n, side_m=args.srv_side, out=xyz)
    gen_s = time.perf_counter() - t0
    reqs = synth.served_requests(args.srv_requests, seed=BASE_SEED + 6 + 1000 * rank, side_m=args.srv_side)
    sizes = [r["ncols"] * r["nrows"] for r in reqs]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    pool = torch.empty(int(offs[-1]), dtype=torch.float32, pin_memory=True).numpy()
    outs = [pool[offs[k]:offs[k + 1]].reshape(reqs[k]["nrows"], reqs[k]["ncols"]) for k in range(len(reqs))]
    eng = engine.Engine(device=local)
    srv = eng.server(xyz)
    rates = [float(x) for x in args.srv_rates.split(",") if x]
    rng = np.random.default_rng(BASE_SEED + 7 + rank)
    with ClockSampler(local) as clk:
        # warm-up: a few requests alone
        for k in range(min(args.warmup, len(reqs))):
            srv.wait(srv.submit(**reqs[k], out_h=outs[k]), timeout=600)
        clk.mark("t_start")
        results = serve_rates(srv, reqs, outs, rates, rng, max_over_ranks, world,
                              barrier=(tdist.barrier if tdist is not None else None))
        clk.mark("t_end")
    st = srv.stats()
    srv.close()
    acc = None
    if rank == 0 and not args.no_cpu_baseline:
        acc = served_accuracy(reqs, outs, xyz, 2)
    if rank == 0:
        best = max(results, key=lambda r: r["cells_per_s"])
        top = results[-1]
        peak, peak_kind = peaks()
        print(json.dumps({
            "metric": METRIC, "value": top["cells_per_s"], "unit": UNIT, "n_gpus": world,
            "steps": len(rates), "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32/int64",
            "data": "synthetic (seeded fBm terrain, clusters, lakes)",
            "config": {"workload": "served", "cloud_points": n, "cloud_side_m": args.srv_side,
                       "requests_per_rate": len(reqs), "request_side_m": "log-U[128, 8192]",
                       "cell_m": [0.5, 1, 2], "rates": rates, "generate_s": round(gen_s, 1),
                       "form": "continuous batching over 2 slots of 16 GiB, footprint admission",
                       "parallelism": f"dp{world} (independent servers)"},
            "served": results, "best_cells_per_s": best["cells_per_s"],
            "latency": {"p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"], "at_rate": top["rate_per_s"]},
            "server": st,
            "e2e": {"value": top["cells_per_s"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(4 * sum(sizes)),
                    "note": "requests return heights in host memory: the value is already end to end"},
            "roofline": {"bound": "hbm", "kernel": "whole request path", "peak": peak, "peak_kind": peak_kind,
                         "unit": "GB/s", "achieved": None, "frac": None, "traffic": None},
            "gpu_launches": int(st["batches"] * (KERNELS_PER_BATCH + 1)), "clocks": clk.summary(),
            "accuracy": acc,
        }), flush=True)
    eng.close()
    if tdist is not None:
        tdist.destroy_process_group()


def main():
    args = parse()
    world, rank, local = dist()
    if args.workload == "served":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "metric": METRIC, "unit": UNIT, "workload": "served",
                              "note": "the CPU reference arm is measured on the mixed workload"}))
            return
        run_engine_served(args, world, rank, local)
        return
    if args.workload == "compat":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "metric": METRIC, "unit": UNIT, "workload": "compat",
                              "note": "the CPU reference arm is measured on the mixed workload"}))
            return
        if world > 1:
            raise SystemExit("the compat workload runs on one GPU")
        run_engine_compat(args, world, rank, local)
        return
    if args.workload == "spacetime":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "metric": METRIC, "unit": UNIT, "workload": "spacetime",
                              "note": "the CPU reference arm is measured on the mixed workload"}))
            return
        if world > 1:
            raise SystemExit("the spacetime workload runs on one GPU")
        run_engine_spacetime(args, world, rank, local)
        return
    if args.workload == "segment":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "metric": METRIC, "unit": UNIT, "workload": "segment",
                              "note": "the CPU reference arm is measured on the mixed workload"}))
            return
        run_engine_segment(args, world, rank, local)
        return
    if args.workload == "mixed":
        if args.impl == "reference":
            run_reference_mixed(args, world, rank)
        else:
            run_engine_mixed(args, world, rank, local)
        return
    if args.impl == "reference":
        run_reference_tile4096(args, world, rank)
        return
    run_engine_tile4096(args, world, rank, local)


if __name__ == "__main__":
    main()
