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
scaling); times are the max over ranks.
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


def run_reference(args, rank, world):
    """The reference arm: the oracle (the reference's CPU path restated in C;
    the Rust reference cannot be built here) on the host cores, one sector of
    the same 3601^2 DEM per step."""
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    tvs, cfg, z = workload(args.config, 0)
    g = oracle.geometry(cfg["width"], cfg["scale"], cfg["max_line_of_sight"], cfg["rings_per_km"])
    threads = len(os.sched_getaffinity(0))
    samples = g.total_bands * g.band_deltas_size
    cum = np.zeros(g.computable_points_count, np.float32)

    def one(angle):
        d, x, _ = oracle.compile_band_data(g, float(angle))
        oracle.compute_sector(g, z, cfg["observer_height"], d, x, cum, None, threads=threads)

    for w in range(args.warmup):
        one(1 + w % 179)
    t = 0.0
    for k in range(args.steps):
        t0 = time.perf_counter()
        one(1 + (args.warmup + k) % 179)
        t += time.perf_counter() - t0
    value = samples * args.steps / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{cfg['width']}x{cfg['width']} DEM, LOS {g.max_los_as_points} cells, "
                               "one sector (shape + sweep) per step",
                   "s_per_tvs_extrapolated": SECTORS * t / args.steps},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": "one sector per step of the 3601^2 DEM: two full FP64 "
                                   "projections + stable radix sorts, the band shape, and all "
                                   f"{g.total_bands} bands swept in exact f32"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(cfg, z, tvs_geom):
    """The oracle on the host cores over one sector of the same workload."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    g = oracle.geometry(cfg["width"], cfg["scale"], cfg["max_line_of_sight"], cfg["rings_per_km"])
    threads = len(os.sched_getaffinity(0))
    cum = np.zeros(g.computable_points_count, np.float32)
    t0 = time.perf_counter()
    d, x, _ = oracle.compile_band_data(g, 1.0)
    oracle.compute_sector(g, z, cfg["observer_height"], d, x, cum, None, threads=threads)
    t = time.perf_counter() - t0
    samples = g.total_bands * g.band_deltas_size
    return {"value": samples / t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"sector 1 of the same DEM (shape: 2 full sorts of {g.size} points; "
                      f"sweep: {g.total_bands} bands x {g.band_deltas_size} steps), "
                      f"{t:.1f} s on {threads} threads; the oracle restates the reference CPU path"}


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
    tvs, cfg, z = workload(args.config, rank)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    eng = tvs.Engine(z, cfg["width"], cfg["scale"], cfg["max_line_of_sight"],
                     observer_height=cfg["observer_height"], rings_per_km=cfg["rings_per_km"],
                     precision=args.precision, sweep_kernel=args.kernel, device=local)
    g = eng.geometry
    ref_samples = SECTORS * g.total_bands * g.band_deltas_size
    steps_eval = g.band_steps_filled + min(g.band_deltas_size - g.band_steps_filled, 2)
    eval_samples = SECTORS * g.total_bands * steps_eval
    stream = torch.cuda.ExternalStream(eng.stream(), device=dev)
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    fp32_peak = tvs.measure_fp32_issue(local)

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            torch.distributed.barrier()

    def full_tvs():
        eng.device_reset()
        eng.device_shape_sectors(0, SECTORS)
        eng.device_sweep_sectors(0, SECTORS)

    for _ in range(args.warmup):
        full_tvs()
        eng.device_finish()
    if args.precision == "mixed64":
        eng.read_rechecks(reset=True)

    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    launches0 = eng.last_launch_count()
    barrier()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(k & 0xFF)                 # L2 flush, outside the timed events
                ev[k][0].record(stream)
                eng.device_reset()
                eng.device_shape_sectors(0, SECTORS)
                ev[k][1].record(stream)
                eng.device_sweep_sectors(0, SECTORS)
                ev[k][2].record(stream)
        torch.cuda.synchronize(dev)
    eng.device_finish()
    barrier()
    gpu_launches = eng.last_launch_count() - launches0
    rechecks = eng.read_rechecks(reset=True) if args.precision == "mixed64" else None
    step_ms = [ev[k][0].elapsed_time(ev[k][2]) for k in range(args.steps)]
    shape_ms = [ev[k][0].elapsed_time(ev[k][1]) for k in range(args.steps)]
    sweep_ms = [ev[k][1].elapsed_time(ev[k][2]) for k in range(args.steps)]
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps * ref_samples / (total_ms * 1e-3)

    # e2e: through the public C ABI with host buffers (pinned), H2D + D2H per step
    e2e = None
    if not args.no_e2e:
        host_z = torch.from_numpy(np.ascontiguousarray(z, np.float32).ravel()).pin_memory()
        cum = torch.empty(g.computable_points_count, dtype=torch.float32).pin_memory()
        tot = torch.empty(g.computable_points_count, dtype=torch.float32).pin_memory()
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
        e2e = {"value": world * args.steps * ref_samples / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(host_z.numel() * 4),
               "d2h_bytes_per_step": int(2 * g.computable_points_count * 4),
               "ms_per_step": e2e_ms / args.steps}

    def time_one_tvs(engine):
        """Device time of one full TVS on `engine` (after one untimed TVS)."""
        engine.device_reset()
        engine.device_run_sectors(0, SECTORS)
        engine.device_finish()
        es = torch.cuda.ExternalStream(engine.stream(), device=dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(es):
            flush.fill_(1)
            e0.record(es)
            engine.device_reset()
            engine.device_run_sectors(0, SECTORS)
            e1.record(es)
        e1.synchronize()
        engine.device_finish()
        return e0.elapsed_time(e1) * 1e-3

    # the FP32 legs of "mixed vs FP32" on the same GPU: the exact-f32 engine
    # (the reference's arithmetic, bit for bit) and the plain one-thread-per-
    # band port of the reference shader
    fp32_engine = plain = None
    if not args.no_plain and args.kernel == "engine":
        kw = dict(observer_height=cfg["observer_height"], rings_per_km=cfg["rings_per_km"],
                  device=local)
        with tvs.Engine(z, cfg["width"], cfg["scale"], cfg["max_line_of_sight"],
                        precision="exact32", **kw) as e32:
            t32 = time_one_tvs(e32)
            c32, _ = e32.read_surfaces()
        with tvs.Engine(z, cfg["width"], cfg["scale"], cfg["max_line_of_sight"],
                        sweep_kernel="plain", **kw) as pe:
            tpl = time_one_tvs(pe)
            c_plain, _ = pe.read_surfaces()
        c_head, _ = eng.read_surfaces()
        fp32_engine = {"value": ref_samples / t32, "s_per_tvs": t32,
                       "kernel": "k_sweep_queue<exact32>: the reference's f32 arithmetic",
                       "identical_to_plain_port": bool(np.array_equal(c32.view(np.uint32),
                                                                      c_plain.view(np.uint32)))}
        plain = {"value": ref_samples / tpl, "s_per_tvs": tpl,
                 "kernel": "one thread per band, IEEE divisions, every delta-table step"}
        if args.precision == "exact32":
            fp32_engine["identical_to_headline"] = bool(np.array_equal(c32.view(np.uint32),
                                                                       c_head.view(np.uint32)))

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(cfg, z, g)

    if rank == 0:
        clk = clocks.summary()
        sweep_avg_s = statistics.mean(sweep_ms) * 1e-3
        achieved = eval_samples * 5 / sweep_avg_s           # FP32 lane-instructions / s
        traffic = (traffic_from_profiles(f"k_sweep_queue<{args.precision}>")
                   if args.kernel == "engine" else None)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"exact32": "f32", "fp64": "f64", "mixed64": "f32+f64"}[args.precision],
            "data": "synthetic",
            "config": {
                "workload": WORKLOADS.get(args.config, args.config) +
                            f": {cfg['width']}x{cfg['width']} DEM, {cfg['scale']:g} m cells, "
                            f"LOS {g.max_los_as_points} cells, 180 sectors, observer "
                            f"{cfg['observer_height']} m",
                "precision": args.precision, "sweep_kernel": args.kernel,
                "l2": "flushed between steps (256 MiB write); DEM 52 MB is L2-resident within a step",
                "s_per_tvs": total_ms / args.steps * 1e-3 / 1.0,
                "shape_ms_per_tvs": statistics.mean(shape_ms),
                "sweep_ms_per_tvs": statistics.mean(sweep_ms),
                "los_samples_per_tvs": ref_samples,
                "evaluated_samples_per_tvs": eval_samples,
                "evaluated_samples_per_s": world * args.steps * eval_samples / (total_ms * 1e-3),
                "hbm_bytes_context": eng.device_bytes(),
                "ring_buffer_bytes_per_sector": int(g.ring_slots_per_sector * 4),
                "fp64_rechecks_per_evaluated_sample":
                    None if rechecks is None else rechecks / (args.steps * eval_samples),
                "note": "delta-table entries the reference leaves at 0 after the first two are "
                        "provably no-ops and are not evaluated; samples counted as the reference "
                        "loop counts them. The split sweeps also skip 32-step segments whose "
                        "DEM block maxima prove that no chain's filter can pass (about half "
                        "at 3601^2); those samples count as evaluated, so roofline.achieved "
                        "is algorithmic work per second, above the instructions issued",
            },
            "roofline": {
                "bound": "fp32_issue", "achieved": achieved / 1e12,
                "peak": fp32_peak / 1e12, "unit": "Tinstr/s",
                "frac": achieved / fp32_peak, "traffic": traffic,
                "kernel": f"k_sweep_queue<{args.precision}> (one persistent launch: 180 sectors)"
                          if args.kernel == "engine" else "k_sweep_plain (one launch per sector)",
                "algorithmic_work": "5 FP32 instructions per evaluated sample (sub, fma, "
                                    "setp, max, predicated add)",
                "peak_source": "measured: FFMA issue microbenchmark on this GPU "
                               "(tvs_measure_fp32_issue), run before the timed region",
            },
            "cpu_baseline": base, "e2e": e2e, "gpu_launches": gpu_launches,
            "fp32_exact_engine": fp32_engine, "plain_fp32_sweep": plain,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
