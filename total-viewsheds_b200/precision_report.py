"""Precision report of the precision form (3601^2 DEM, 1200-cell line of sight,
180 sectors): how far the exact-f32 engine (bit-identical to the reference's
f32 CPU path), the MIXED64 engine and the reciprocal-table FP32 form are from
the all-FP64 sweep.

    python total-viewsheds_b200/precision_report.py [--sectors 0,1,45,46,90]

Per point of view: the relative error of the cumulative surface after 180
sectors, |x - x64| / |x64|, as p50 / p99 / max (points with x64 == 0 excluded).
Per sector (the listed ones): ring records compared band by band; a band
whose open/close ids differ is a ring-boundary disagreement.  MIXED64 decides
every comparison as the FP64 sweep does, so its rings are the FP64 rings; they
are compared too, as are the FP32 form's.
Prints one JSON object.
"""

import argparse
import importlib.util
import json
import sys
import time
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent


def _package():
    if "total_viewsheds_b200" in sys.modules:
        return sys.modules["total_viewsheds_b200"]
    spec = importlib.util.spec_from_file_location("total_viewsheds_b200", PKG / "__init__.py",
                                                  submodule_search_locations=[str(PKG)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["total_viewsheds_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def rel_error_stats(x, ref):
    x = x.astype(np.float64)
    ref = ref.astype(np.float64)
    keep = ref != 0
    r = np.abs(x[keep] - ref[keep]) / np.abs(ref[keep])
    return {"p50": float(np.percentile(r, 50)), "p99": float(np.percentile(r, 99)),
            "max": float(r.max()), "points": int(keep.sum()),
            "identical_points": int((x[keep] == ref[keep]).sum())}


def ring_disagreements(ra, rb, reserved):
    """Bands whose ring records differ (ids or count); and the number of ring
    ids that differ position by position."""
    a = ra.reshape(-1, reserved)
    b = rb.reshape(-1, reserved)
    differ = np.any(a != b, axis=1)
    return int(differ.sum()), int((a != b).sum())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="precision")
    ap.add_argument("--sectors", default="0,1,45,46,90")
    ap.add_argument("--rings-per-km", type=float, default=5.0)
    args = ap.parse_args()
    tvs = _package()
    import total_viewsheds_b200.dem_synth as ds
    cfg = ds.CONFIGS[args.config]
    z = ds.config_dem(args.config)
    w, s, los = cfg["width"], cfg["scale"], cfg["max_line_of_sight"]
    out = {"workload": f"{args.config}: {w}x{w} DEM, LOS {los} m, 180 sectors, observer "
                       f"{cfg['observer_height']} m"}
    cum, timing = {}, {}
    for p in ("fp64", "mixed64", "exact32", "fp32"):
        with tvs.Engine(z, w, s, los, observer_height=cfg["observer_height"],
                        rings_per_km=args.rings_per_km, precision=p) as eng:
            t0 = time.perf_counter()
            cum[p], _, _ = eng.run()
            timing[p] = time.perf_counter() - t0
            if p == "mixed64":
                out["mixed64_fp64_rechecks"] = eng.read_rechecks(reset=True)
    out["seconds_per_tvs_host_timed"] = timing
    out["surface_rel_error_vs_fp64"] = {
        "exact32 (= reference f32 CPU path)": rel_error_stats(cum["exact32"], cum["fp64"]),
        "mixed64": rel_error_stats(cum["mixed64"], cum["fp64"]),
        "fp32 (reciprocal-table form)": rel_error_stats(cum["fp32"], cum["fp64"]),
    }
    out["surface_rel_error_vs_cpu_f32_path"] = {
        "mixed64": rel_error_stats(cum["mixed64"], cum["exact32"]),
        "fp64": rel_error_stats(cum["fp64"], cum["exact32"]),
    }
    sectors = [int(x) for x in args.sectors.split(",") if x]
    engines = {p: tvs.Engine(z, w, s, los, observer_height=cfg["observer_height"],
                             rings_per_km=args.rings_per_km, precision=p)
               for p in ("fp64", "exact32", "mixed64", "fp32")}
    try:
        reserved = engines["fp64"].geometry.reserved_rings_per_band
        n = engines["fp64"].geometry.ring_slots_per_sector
        rings = {k: {} for k in ("exact32", "mixed64", "fp32")}
        for a in sectors:
            recs, stats = {}, {}
            try:
                for p, e in engines.items():
                    recs[p] = np.zeros(n, np.uint32)
                    stats[p] = e.compute_sector(a, np.zeros(e.count, np.float32), recs[p])
            except tvs.TvsError as err:  # e.g. ring records past the buffer end
                for k in rings:
                    rings[k][str(a)] = {"error": str(err)}
                continue
            for k in rings:
                bands, ids = ring_disagreements(recs[k], recs["fp64"], reserved)
                rings[k][str(a)] = {"bands": int(engines[k].geometry.total_bands),
                                    "disagreeing_bands": bands, "disagreeing_ring_slots": ids,
                                    "max_ring_ids": int(stats[k].max_ring_ids),
                                    "overflow_bands": int(stats[k].overflow_bands)}
    finally:
        for e in engines.values():
            e.close()
    out["ring_boundary_disagreements_vs_fp64"] = rings
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
