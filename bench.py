#!/usr/bin/env python
"""Total-viewshed benchmark: LOS samples/s and seconds per 180-sector TVS.

One step = one full total viewshed (all 180 sectors: the shape stage and the
sweep) of the 3601 x 3601 precision-form DEM (seeded ridged multifractal,
10 % flat sea, 30 m cells, 36 km line of sight, observer 1.65 m), with the
DEM resident in HBM.  A LOS sample is one (band, step) iteration of the
reference kernel loop (kernel.rs:153): samples per TVS = 180 * total_bands *
band_deltas_size.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun every rank computes the total viewshed of its own DEM tile
(seed + rank): independent objects, no collective on the data path (weak
scaling); with --shard rows the ranks split one DEM's computable rows instead
(strong scaling; each point's summation order is unchanged, the rows are
gathered outside the timed region).  Times are the max over ranks.
"""

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time
from datetime import timedelta
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
METRIC = "LOS samples/s & s per 180-sector TVS, 3601² DEM: mixed vs FP32 on 1 B200"
UNIT = "LOS samples/s"
SECTORS = 180
FLUSH_BYTES = 256 << 20  # > 126 MB L2
WORKLOADS = {
    "precision": "precision form (ridged multifractal, 10% flat 0 m)",
    "plain_gpu": "plain FP32 GPU form (fBm Hurst 0.75, 15% flat 0 m)",
    "plain_cpu": "plain CPU-runnable form (fBm Hurst 0.8)",
    "large": "large single region (2x2 stitched fBm)",
    "medium": "profiling stand-in (ridged multifractal, 10% flat 0 m)",
}


def load_package():
    import importlib.util
    if "total_viewsheds_b200" in sys.modules:
        return sys.modules["total_viewsheds_b200"]
    pkg = ROOT / "total-viewsheds_b200"
    spec = importlib.util.spec_from_file_location("total_viewsheds_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["total_viewsheds_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(name, rank):
    tvs = load_package()
    import total_viewsheds_b200.dem_synth as ds
    cfg = ds.CONFIGS[name]
    if rank == 0:
        z = ds.config_dem(name)
    else:  # weak scaling: another tile of the same family per rank
        saved = ds.BASE_SEED
        ds.BASE_SEED = saved + 1000 * rank
        try:
            z = ds.config_dem(name)
        finally:
            ds.BASE_SEED = saved
    return tvs, cfg, z


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=10)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        rows = [[c.strip() for c in l.split(",")] for l in getattr(self, "lines", [])]
        rows = [r for r in rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in rows if num(r[1])]
        power = [num(r[3]) for r in rows if num(r[3])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        loaded = [s for s in sm if s >= 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": num(rows[0][2]), "reasons": reasons,
                "power_w_max": max(power) if power else None, "samples": len(rows)}


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus and world > 1:
        print(f"warning: WORLD_SIZE={world} but --gpus {args.gpus}", file=sys.stderr)
    return rank, world, local


# The CPU legs time these sectors: 0 and 90 degrees follow the grid axes, 1
# and 46 degrees do not, and 45 is the diagonal (the reference notes that 0 is
# much faster than 1, README.md:110); a TVS is extrapolated from their mean.
CPU_SECTORS = (0, 1, 45, 46, 90)


def oracle_sector(oracle, g, z, observer_height, angle, threads, rows=None):
    """One sector on the host: the shape stage (two full projections and
    stable sorts) and the sweep of every band (of `rows`, when given)."""
    d, x, _ = oracle.compile_band_data(g, float(angle))
    oracle.sweep_sector(g, z, observer_height, d, x, rows=rows, threads=threads)


def run_reference(args, rank, world):
    """The reference arm: the oracle (the reference's CPU path restated in C;
    the Rust reference cannot be built here) on all host cores, one of the
    sectors 0, 1, 45, 46, 90 of the same DEM per step."""
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    tvs, cfg, z = workload(args.config, 0)
    g = oracle.geometry(cfg["width"], cfg["scale"], cfg["max_line_of_sight"], cfg["rings_per_km"])
    threads = len(os.sched_getaffinity(0))
    samples = g.total_bands * g.band_deltas_size
    for w in range(args.warmup):
        oracle_sector(oracle, g, z, cfg["observer_height"], CPU_SECTORS[w % 5], threads)
    t = 0.0
    for k in range(args.steps):
        t0 = time.perf_counter()
        oracle_sector(oracle, g, z, cfg["observer_height"], CPU_SECTORS[k % 5], threads)
        t += time.perf_counter() - t0
    value = samples * args.steps / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOADS.get(args.config, args.config) +
                               f": {cfg['width']}x{cfg['width']} DEM, LOS {g.max_los_as_points} "
                               "cells; one sector (shape + sweep) per step, cycling through "
                               f"sectors {list(CPU_SECTORS)}",
                   "s_per_tvs_extrapolated": SECTORS * t / args.steps},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"sectors {list(CPU_SECTORS)} of the same DEM, one per step: "
                                   "two full FP64 projections + stable radix sorts, the band "
                                   f"shape, and all {g.total_bands} bands swept in exact f32; a "
                                   "TVS is 180 x the mean sector time (an extrapolation)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(cfg, z, tvs_geom):
    """The oracle on the host cores: sectors 0, 1, 45, 46, 90 of the same
    workload on every core, and one thread (as the reference runs,
    compute.rs:228-240) over a row sample of sector 1; a TVS is extrapolated
    from the mean sector time."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    g = oracle.geometry(cfg["width"], cfg["scale"], cfg["max_line_of_sight"], cfg["rings_per_km"])
    threads = len(os.sched_getaffinity(0))
    samples = g.total_bands * g.band_deltas_size
    per_sector = {}
    for a in CPU_SECTORS:
        t0 = time.perf_counter()
        oracle_sector(oracle, g, z, cfg["observer_height"], a, threads)
        per_sector[a] = time.perf_counter() - t0
    t_all = statistics.mean(per_sector.values())
    # one thread: the whole shape stage plus the bands of 1/16 of the rows
    rows = (0, max(1, g.tvs_height // 16))
    frac = (rows[1] - rows[0]) / g.tvs_height
    t0 = time.perf_counter()
    d, x, _ = oracle.compile_band_data(g, 1.0)
    t_shape = time.perf_counter() - t0
    t0 = time.perf_counter()
    oracle.sweep_sector(g, z, cfg["observer_height"], d, x, rows=rows, threads=1)
    t_sweep = (time.perf_counter() - t0) / frac
    t_one = t_shape + t_sweep
    return {"value": samples / t_all, "unit": UNIT, "cores": threads, "kind": "port",
            "s_per_tvs_extrapolated": SECTORS * t_all,
            "threads_1": {"value": samples / t_one, "s_per_tvs_extrapolated": SECTORS * t_one,
                          "sample": f"sector 1: the shape stage, and the sweep of rows {rows[0]}-"
                                    f"{rows[1]} of {g.tvs_height} scaled to all rows"},
            "threads_all": {"value": samples / t_all, "threads": threads,
                            "s_per_sector": {str(k): round(v, 3) for k, v in per_sector.items()}},
            "sample": f"sectors {list(CPU_SECTORS)} of the same DEM on {threads} threads (shape: "
                      f"2 full sorts of {g.size} points; sweep: {g.total_bands} bands x "
                      f"{g.band_deltas_size} steps each); a TVS is 180 x their mean (an "
                      "extrapolation); the oracle restates the reference CPU path"}


def run_batching(args, rank, world, local, torch):
    """The batching form: 48 seeded DEM tiles of uneven, partly rectangular size
    (sides U[257, 1601]), all 180 sectors of all tiles per step: one shape launch
    and one persistent sweep, replayed from a CUDA graph; the sweep
    configuration comes from the autotuner."""
    tvs = load_package()
    import total_viewsheds_b200.dem_synth as ds
    tiles = ds.batching_tiles(48, seed=ds.BASE_SEED + 3 + 1000 * rank)
    dev = torch.device("cuda", local)
    b = tvs.Batch(tiles, observer_height=1.65, precision=args.precision, device=local)
    ref_samples = sum(180 * g.total_bands * g.band_deltas_size for g in b.geometry)
    eval_samples = sum(180 * g.total_bands * (g.band_steps_filled +
                                              min(g.band_deltas_size - g.band_steps_filled, 2))
                       for g in b.geometry)
    t0 = time.perf_counter()
    cfg = b.autotune(sample_sectors=4)
    tune_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        b.run()
        b.finish()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(k & 0xFF)
                ev[k][0].record(stream)
                b.run()
                ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
    b.finish()
    total_ms = sum(e[0].elapsed_time(e[1]) for e in ev)
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    if rank == 0:
        sides = [(g.width, g.height) for g in b.geometry]
        line = {
            "metric": METRIC, "value": world * args.steps * ref_samples / (total_ms * 1e-3),
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": {"exact32": "f32", "fp64": "f64", "mixed64": "f32+f64"}[args.precision],
            "data": "synthetic",
            "config": {
                "workload": "batching form: 48 seeded fBm DEM tiles, sides U[257,1601] per axis "
                            f"({sum(1 for w, h in sides if w != h)} rectangular), LOS = 1/3 of the "
                            "shorter side, all 180 sectors of every tile per step",
                "precision": args.precision,
                "autotuned_sweep": repr(cfg), "autotune_s": tune_s,
                "los_samples_per_step": ref_samples, "evaluated_samples_per_step": eval_samples,
                "hbm_bytes_batch": b.device_bytes(),
                "launches_per_step": "1 graph replay: surface resets, 1 shape launch, 1 sweep",
                "l2": "flushed between steps (256 MiB write)",
            },
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    b.close()


def traffic_from_profiles(kernel_name):
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        return json.loads(p.read_text()).get(kernel_name)
    except (ValueError, OSError):
        return None


def targets(value, legs, precision):
    """Which engine meets which half of the target: the reference CPU ring
    records bit for bit, per-point surface error <= 1e-5 against FP64, and the
    headline against the plain FP32 GPU sweeps."""
    exact = legs["exact32_engine"]["surfaces_vs_fp64"]
    return {
        "reference_cpu_ring_records_bit_for_bit":
            "exact32 engine (its surfaces equal the plain port's: "
            f"{legs['exact32_engine'].get('identical_to_plain_port')}); MIXED64 records are the "
            "FP64 ones, which differ from the reference's f32 records at ties",
        "surface_rel_error_le_1e-5_vs_fp64": {
            "headline": precision in ("mixed64", "fp64"),
            "fp32_form": legs["plain_fp32_sweep"]["surfaces_vs_fp64"]["rel_max"] <= 1e-5
            if legs["plain_fp32_sweep"]["surfaces_vs_fp64"] else None,
            "exact32": exact["rel_max"] <= 1e-5 if exact else None},
        "headline_over_plain_port": value / legs["plain_port"]["value"],
        "headline_over_fp32_form": value / legs["plain_fp32_sweep"]["value"],
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--config", default="precision")
    ap.add_argument("--precision", default="mixed64",
                    help="mixed64 (headline), exact32 (the reference's f32 arithmetic) or fp64")
    ap.add_argument("--kernel", default="engine")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-rings", action="store_true")
    ap.add_argument("--shard", default="dems", choices=["dems", "rows"],
                    help="N>1: every rank its own DEM (weak scaling, default) or one DEM's "
                         "rows split over the ranks (strong scaling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_setup(args)

    import torch
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if world > 1:
            torch.distributed.destroy_process_group()
        return

    if args.config == "batching":
        torch.cuda.set_device(local)
        run_batching(args, rank, world, local, torch)
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    # weak scaling gives every rank its own DEM; a row split shares one
    tvs, cfg, z = workload(args.config, 0 if args.shard == "rows" else rank)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    rows = None
    if args.shard == "rows" and world > 1:
        import total_viewsheds_b200.sharding as sh
        g_full = tvs.compute_geometry(tvs.make_params(cfg["width"], cfg["scale"],
                                                      cfg["max_line_of_sight"]))
        rows = sh.shard_rows(g_full.tvs_height, rank, world)
    eng = tvs.Engine(z, cfg["width"], cfg["scale"], cfg["max_line_of_sight"],
                     observer_height=cfg["observer_height"], rings_per_km=cfg["rings_per_km"],
                     precision=args.precision, sweep_kernel=args.kernel, device=local, rows=rows)
    g = eng.geometry
    ref_samples = SECTORS * g.total_bands * g.band_deltas_size
    steps_eval = g.band_steps_filled + min(g.band_deltas_size - g.band_steps_filled, 2)
    eval_samples = SECTORS * g.total_bands * steps_eval
    # this rank's share of the samples (a row shard sweeps its rows only)
    my_rows = g.tvs_height if rows is None else rows[1] - rows[0]
    my_eval = eval_samples * my_rows // g.tvs_height
    stream = torch.cuda.ExternalStream(eng.stream(), device=dev)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    fp32_peak = tvs.measure_fp32_issue(local)
    l1_peak = tvs.measure_l1_load(local)

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            torch.distributed.barrier()

    for _ in range(args.warmup):
        eng.device_run_tvs()     # the first call captures the graph
        eng.device_finish()
    if args.precision in ("mixed64", "exact32"):
        eng.read_rechecks(reset=True)

    # Timed: one graph replay per step (reset, 180 shape stages, one persistent
    # sweep); L2 flushed before each step outside the events; the graph's own
    # events give the shape and sweep stages of every step.
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    shape_ms, sweep_ms = [], []
    barrier()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(k & 0xFF)
                ev[k][0].record(stream)
                eng.device_run_tvs()
                ev[k][1].record(stream)
            sh_ms, sw_ms = eng.last_run_times()   # waits for this step
            shape_ms.append(sh_ms)
            sweep_ms.append(sw_ms)
        torch.cuda.synchronize(dev)
    eng.device_finish()
    barrier()
    launches_per_step = eng.last_launch_count()
    gpu_launches = args.steps * launches_per_step
    rechecks = eng.read_rechecks(reset=True) if args.precision in ("mixed64", "exact32") else None
    step_ms = [ev[k][0].elapsed_time(ev[k][1]) for k in range(args.steps)]
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    # the whole job: every rank's samples (a full DEM per rank, or one DEM's rows)
    job_samples = ref_samples * (world if rows is None else 1)
    value = args.steps * job_samples / (total_ms * 1e-3)

    # Untimed: the sweep counters of one more TVS (swept / skipped / filtered steps)
    counters = None
    if args.kernel == "engine" and eng.sweep_config().layout:
        eng.sweep_counters(enable=True)
        eng.device_reset()
        eng.device_run_sectors(0, SECTORS)
        eng.device_finish()
        counters = eng.sweep_counters()
        eng.sweep_counters(enable=False)

    # e2e: through the public C ABI with host buffers (pinned), H2D + D2H per step
    e2e = None
    if not args.no_e2e:
        host_z = torch.from_numpy(np.ascontiguousarray(z, np.float32).ravel()).pin_memory()
        cum = torch.empty(eng.count, dtype=torch.float32).pin_memory()
        tot = torch.empty(eng.count, dtype=torch.float32).pin_memory()
        L = tvs.lib()
        nullcb = tvs.SECTOR_CALLBACK()

        def e2e_step():
            rc = L.tvs_set_elevations(eng.ctx, ctypes.c_void_p(host_z.data_ptr()), host_z.numel())
            rc = rc or L.tvs_run(eng.ctx, ctypes.c_void_p(cum.data_ptr()),
                                 ctypes.c_void_p(tot.data_ptr()), 0, nullcb, None)
            if rc:
                raise tvs.TvsError(rc, L.tvs_last_error(eng.ctx).decode())

        e2e_step()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e2e_ms = 0.0
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(k & 0xFF)
                e0.record(stream)
                e2e_step()
                e1.record(stream)
            e1.synchronize()
            e2e_ms += e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_ms = float(t.item())
        e2e = {"value": args.steps * job_samples / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(host_z.numel() * 4),
               "d2h_bytes_per_step": int(2 * eng.count * 4),
               "ms_per_step": e2e_ms / args.steps,
               "path": "tvs_set_elevations (H2D) + tvs_run (graph replay, D2H of the "
                       "cumulative and heatmap surfaces)"}

    # a row split: the ranks' rows are gathered into the whole grid (outside
    # the timed region; the only exchange of the path)
    gathered = None
    if rows is not None:
        import total_viewsheds_b200.sharding as sh
        c_mine, _ = eng.read_surfaces()
        mine = torch.from_numpy(
            np.ascontiguousarray(c_mine.reshape(-1, g.tvs_width)[rows[0]:rows[1]]).ravel()).to(dev)
        full = sh.gather_rows(mine, g.tvs_width, g.tvs_height, world)
        gathered = {"rows_of_rank0": list(rows), "grid_points_gathered": int(full.size),
                    "nonzero_points": int(np.count_nonzero(full))}

    def time_one_tvs(engine):
        """Device time of one full TVS on `engine` (after one untimed TVS)."""
        engine.device_run_tvs()
        engine.device_finish()
        es = torch.cuda.ExternalStream(engine.stream(), device=dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(es):
            flush.fill_(1)
            e0.record(es)
            engine.device_run_tvs()
            e1.record(es)
        e1.synchronize()
        engine.device_finish()
        return e0.elapsed_time(e1) * 1e-3

    # The legs of "mixed vs FP32" on the same GPU and DEM: the reciprocal-table
    # FP32 form in the same engine (same layouts, segment skipping), the
    # exact-f32 engine (the reference's arithmetic) and the plain port of the
    # reference shader (one thread per band).  Each reports how its surfaces
    # differ from the FP64-exact result.
    legs = {}
    if not args.no_plain and args.kernel == "engine" and rows is None:
        kw = dict(observer_height=cfg["observer_height"], rings_per_km=cfg["rings_per_km"],
                  device=local)
        c_head, _ = eng.read_surfaces()
        ref64 = c_head.astype(np.float64) if args.precision in ("mixed64", "fp64") else None

        def surface_error(c):
            if ref64 is None:
                return None
            rel = np.abs(c.astype(np.float64) - ref64) / np.maximum(np.abs(ref64), 1e-30)
            return {"points_differing": int(np.count_nonzero(c != c_head)),
                    "rel_p50": float(np.percentile(rel, 50)),
                    "rel_p99": float(np.percentile(rel, 99)), "rel_max": float(rel.max())}

        outs = {}
        for name, kwargs, what in [
                ("plain_fp32_sweep", dict(precision="fp32"),
                 "k_sweep_split<fp32>: angle = fma(h - h_pov, RN(1/d), -RN(d/R)) in f32, f32 "
                 "comparisons and surfaces; same layouts and segment skipping as the headline"),
                ("exact32_engine", dict(precision="exact32"),
                 "k_sweep_split<exact32>: the reference's f32 arithmetic, guard band + exact "
                 "re-decision"),
                ("plain_port", dict(sweep_kernel="plain"),
                 "k_sweep_plain: one thread per band, IEEE divisions, every delta-table step")]:
            with tvs.Engine(z, cfg["width"], cfg["scale"], cfg["max_line_of_sight"], **kwargs,
                            **kw) as e:
                t = time_one_tvs(e)
                outs[name], _ = e.read_surfaces()
            legs[name] = {"value": ref_samples / t, "s_per_tvs": t, "kernel": what,
                          "surfaces_vs_fp64": surface_error(outs[name])}
        legs["exact32_engine"]["identical_to_plain_port"] = bool(np.array_equal(
            outs["exact32_engine"].view(np.uint32), outs["plain_port"].view(np.uint32)))

    # Ring records of a whole TVS through the compact stream: sectors in groups
    # of RING_SECTORS per tvs_compute_sectors_rings call (one sweep launch per
    # group; the surfaces and the records of every band kept on the device);
    # host-timed, every call synchronises.
    rings_leg = None
    if not args.no_rings and args.kernel == "engine" and rows is None:
        RING_SECTORS = 6
        cum_r = torch.zeros(eng.count, dtype=torch.float32).pin_memory().numpy()
        total_ids = ctypes.c_uint64()
        st = tvs.SectorStats()
        L = tvs.lib()

        def ring_call(first):
            rc = L.tvs_compute_sectors_rings(eng.ctx, first, RING_SECTORS, tvs._ptr(cum_r),
                                             ctypes.byref(total_ids), ctypes.byref(st))
            if rc:
                raise tvs.TvsError(rc, L.tvs_last_error(eng.ctx).decode())

        ring_call(0)  # allocates the record buffers
        cum_r[:] = 0
        ids_all, most = 0, 0
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for first in range(0, SECTORS, RING_SECTORS):
            ring_call(first)
            ids_all += total_ids.value
            most = max(most, st.max_ring_ids)
        t_rings = time.perf_counter() - t0
        rings_leg = {"s_per_tvs": t_rings, "ids_per_tvs": ids_all,
                     "record_bytes_per_tvs": 4 * ids_all + 8 * (g.total_bands + 1) * SECTORS,
                     "most_ids_in_a_band": most,
                     "vs_surfaces_only": t_rings / (total_ms / args.steps * 1e-3),
                     "sectors_per_call": RING_SECTORS,
                     "path": f"tvs_compute_sectors_rings, {RING_SECTORS} sectors per call: H2D + D2H "
                             "of the surfaces (pinned), one split-sweep launch writing ring slots, "
                             "scan + gather into the compact stream (host-timed)"}

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(cfg, z, g)

    if rank == 0:
        clk = clocks.summary()
        sweep_avg_s = statistics.mean(sweep_ms) * 1e-3
        achieved = my_eval * 5 / sweep_avg_s           # FP32 lane-instructions / s
        roof = {
            "bound": "fp32_issue", "achieved": achieved / 1e12,
            "peak": fp32_peak / 1e12, "unit": "Tinstr/s", "frac": achieved / fp32_peak,
            "traffic": (traffic_from_profiles(f"k_sweep_split<{args.precision}>")
                        if args.kernel == "engine" else None),
            "kernel": f"k_sweep_split<{args.precision}> (one persistent launch: 180 sectors)"
                      if args.kernel == "engine" else "k_sweep_plain (one launch per sector)",
            "algorithmic_work": "5 FP32 instructions per evaluated sample (sub, fma, setp, max, "
                                "predicated add); the 2 zero-distance tail steps are the last "
                                "evaluated ones",
            "peak_source": "measured: FFMA issue microbenchmark on this GPU "
                           "(tvs_measure_fp32_issue), run before the timed region",
            "sweep_ms_source": "the graph's own events around the sweep, every timed step",
        }
        if counters and counters[2]:
            executed = counters[0] / counters[2]
            ach_exec = achieved * executed
            l1_bytes = my_eval * executed * 4 / sweep_avg_s   # one f32 load per executed sample
            roof.update({
                "executed_fraction": executed,
                "filter_pass_fraction": counters[1] / counters[0] if counters[0] else None,
                "frac_executed": ach_exec / fp32_peak,
                "l1": {"achieved": l1_bytes / 1e12, "peak": l1_peak / 1e12, "unit": "TB/s",
                       "frac": l1_bytes / l1_peak,
                       "algorithmic": "4 B (one f32 elevation) per executed sample",
                       "peak_source": "measured: L1 load microbenchmark (tvs_measure_l1_load)"},
            })
            if l1_bytes / l1_peak > ach_exec / fp32_peak:
                roof["bound"] = "l1_load"
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "strong" if rows is not None else "weak",
            "vs_baseline": None,
            "dtype": {"exact32": "f32", "fp64": "f64", "mixed64": "f32+f64", "fp32": "f32"}[
                args.precision],
            "data": "synthetic",
            "config": {
                "workload": WORKLOADS.get(args.config, args.config) +
                            f": {cfg['width']}x{cfg['width']} DEM, {cfg['scale']:g} m cells, "
                            f"LOS {g.max_los_as_points} cells, 180 sectors, observer "
                            f"{cfg['observer_height']} m" +
                            (f"; rows split over {world} ranks" if rows is not None else ""),
                "precision": args.precision, "sweep_kernel": args.kernel,
                "sweep_layout": repr(eng.sweep_config()),
                "l2": "flushed between steps (256 MiB write); DEM 52 MB is L2-resident within a step",
                "s_per_tvs": total_ms / args.steps * 1e-3,
                "shape_ms_per_tvs": statistics.mean(shape_ms),
                "sweep_ms_per_tvs": statistics.mean(sweep_ms),
                "launches_per_step": f"1 graph replay ({launches_per_step} kernels: shape, sweep; "
                                     "surface resets and queue counters are memset nodes)",
                "los_samples_per_tvs": ref_samples,
                "evaluated_samples_per_tvs": eval_samples,
                "hbm_bytes_context": eng.device_bytes(),
                "ring_buffer_bytes_per_sector": int(g.ring_slots_per_sector * 4),
                "rechecks_per_evaluated_sample":
                    None if rechecks is None else rechecks / (args.steps * my_eval),
                "note": "delta-table entries the reference leaves at 0 after the first two are "
                        "provably no-ops and are not evaluated; samples counted as the reference "
                        "loop counts them. The split sweep also skips 32-step segments whose "
                        "DEM block maxima prove that no chain can change state; roofline.frac "
                        "counts those samples as evaluated, roofline.frac_executed does not",
            },
            "roofline": roof,
            "cpu_baseline": base, "e2e": e2e, "gpu_launches": gpu_launches,
            **({"row_split": gathered} if gathered else {}),
            **({"rings_compact": rings_leg} if rings_leg else {}),
            **legs,
            **({"targets": targets(value, legs, args.precision)} if legs else {}),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
