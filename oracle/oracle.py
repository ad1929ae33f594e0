"""ctypes binding of the CPU oracle (libtvs_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine.  Only tests/,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use it.
The engine never imports this module.

Also holds ``ascii_viewshed``, a restatement of the reference's test-only ring
decoder (crates/total-viewsheds/src/output/ascii.rs:24-104).
"""

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libtvs_oracle.so"

ERRORS = {
    -1: "invalid arguments",
    -2: "line of sight longer than the DEM allows (dem.rs:56-62)",
    -3: "band-of-sight shape index out of bounds (band_of_sight.rs panic)",
    -4: "elevation index out of bounds (kernel.rs:164 panic)",
    -5: "ring index out of bounds (kernel.rs:307 panic)",
    -6: "out of memory",
}


class OracleError(RuntimeError):
    def __init__(self, code):
        super().__init__(f"oracle error {code}: {ERRORS.get(code, 'unknown')}")
        self.code = code


MODES = {"exact32": 0, "fp64": 1, "fp32": 2}


class SweepOpts(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int),
        ("row_begin", ctypes.c_uint32),
        ("row_end", ctypes.c_uint32),
        ("cum32", ctypes.c_void_p),
        ("cum64", ctypes.c_void_p),
        ("rings", ctypes.c_void_p),
        ("rings_len", ctypes.c_uint64),
        ("counts", ctypes.c_void_p),
        ("ids", ctypes.c_void_p),
        ("ids_cap", ctypes.c_uint64),
        ("ids_total", ctypes.c_void_p),
        ("threads", ctypes.c_int),
    ]


class Geometry(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("scale", ctypes.c_float),
        ("max_line_of_sight", ctypes.c_uint32),
        ("max_los_as_points", ctypes.c_uint32),
        ("band_size", ctypes.c_uint32),
        ("band_deltas_size", ctypes.c_uint32),
        ("tvs_width", ctypes.c_uint32),
        ("tvs_height", ctypes.c_uint32),
        ("reserved_rings_per_band", ctypes.c_uint32),
        ("size", ctypes.c_uint64),
        ("computable_points_count", ctypes.c_uint64),
        ("total_bands", ctypes.c_uint64),
    ]


def build():
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.POINTER
        L.tvso_geometry_new.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                                        ctypes.c_uint32, ctypes.c_float, P(Geometry)]
        L.tvso_calculate_distances.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                                               ctypes.c_void_p]
        L.tvso_calculate_distances.restype = None
        L.tvso_order_by_distance.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
        L.tvso_axes.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, ctypes.c_void_p,
                                ctypes.c_void_p, ctypes.c_void_p]
        L.tvso_compile_band_data.argtypes = [P(Geometry), ctypes.c_float, ctypes.c_void_p,
                                             ctypes.c_void_p, P(ctypes.c_uint32)]
        L.tvso_compute_sector.argtypes = [P(Geometry), ctypes.c_void_p, ctypes.c_float,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int]
        L.tvso_compute_sector_f64.argtypes = L.tvso_compute_sector.argtypes
        L.tvso_run.argtypes = [P(Geometry), ctypes.c_void_p, ctypes.c_float, ctypes.c_uint32,
                               ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.c_int]
        L.tvso_run_f64.argtypes = [P(Geometry), ctypes.c_void_p, ctypes.c_float, ctypes.c_uint32,
                                   ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_int]
        L.tvso_sweep_sector.argtypes = [P(Geometry), ctypes.c_void_p, ctypes.c_float,
                                        ctypes.c_void_p, ctypes.c_void_p, P(SweepOpts)]
        L.tvso_run_ex.argtypes = [P(Geometry), ctypes.c_void_p, ctypes.c_float, ctypes.c_uint32,
                                  ctypes.c_uint32, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32,
                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise OracleError(rc)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def default_threads():
    return len(os.sched_getaffinity(0))


def geometry(width, scale, max_line_of_sight, rings_per_km=5.0, height=None):
    g = Geometry()
    _check(lib().tvso_geometry_new(width, width if height is None else height, scale,
                                   max_line_of_sight, rings_per_km, ctypes.byref(g)))
    return g


def calculate_distances(width, angle, height=None):
    h = width if height is None else height
    out = np.empty(width * h, np.float64)
    lib().tvso_calculate_distances(width, h, angle, _ptr(out))
    return out


def order_by_distance(distances):
    d = np.ascontiguousarray(distances, np.float64)
    out = np.empty(d.size, np.uint32)
    _check(lib().tvso_order_by_distance(_ptr(d), d.size, _ptr(out)))
    return out


def axes(width, angle, height=None):
    """(f32 sight distances, ids in sight order, ids in sector order)."""
    h = width if height is None else height
    n = width * h
    d = np.empty(n, np.float32)
    sight = np.empty(n, np.uint32)
    sector = np.empty(n, np.uint32)
    _check(lib().tvso_axes(width, h, angle, _ptr(d), _ptr(sight), _ptr(sector)))
    return d, sight, sector


def compile_band_data(g, angle):
    """(deltas i32[band_deltas_size], distances f32[band_deltas_size], n_filled)."""
    n = max(g.band_deltas_size, 1)
    deltas = np.zeros(n, np.int32)
    dists = np.zeros(n, np.float32)
    filled = ctypes.c_uint32(0)
    _check(lib().tvso_compile_band_data(ctypes.byref(g), angle, _ptr(deltas), _ptr(dists),
                                        ctypes.byref(filled)))
    return deltas[:g.band_deltas_size], dists[:g.band_deltas_size], filled.value


def ring_len(g):
    return g.total_bands * g.reserved_rings_per_band


def compute_sector(g, elevations, observer_height, deltas, dists, cumulative, rings=None,
                   threads=None, f64=False):
    """In place on cumulative (f32, or f64 when f64=True) and rings (zeroed u32)."""
    e = np.ascontiguousarray(elevations, np.float32)
    fn = lib().tvso_compute_sector_f64 if f64 else lib().tvso_compute_sector
    _check(fn(ctypes.byref(g), _ptr(e), observer_height,
              _ptr(np.ascontiguousarray(deltas, np.int32)),
              _ptr(np.ascontiguousarray(dists, np.float32)), _ptr(cumulative), _ptr(rings),
              0 if rings is None else rings.size, threads or default_threads()))


def run(g, elevations, observer_height, first_angle=0, n_angles=180, rings=False, threads=None):
    """compute.rs:101-115 over a range of sectors.

    Returns (cumulative f32, heatmap total f32, rings u32[n_angles, ring_len] or None)."""
    e = np.ascontiguousarray(elevations, np.float32)
    cum = np.empty(g.computable_points_count, np.float32)
    total = np.empty(g.computable_points_count, np.float32)
    r = np.empty((n_angles, ring_len(g)), np.uint32) if rings else None
    _check(lib().tvso_run(ctypes.byref(g), _ptr(e), observer_height, first_angle, n_angles,
                          _ptr(cum), _ptr(total), _ptr(r), threads or default_threads()))
    return cum, total, r


def run_f64(g, elevations, observer_height, first_angle=0, n_angles=180, rings=False,
            threads=None):
    e = np.ascontiguousarray(elevations, np.float32)
    cum = np.empty(g.computable_points_count, np.float64)
    r = np.empty((n_angles, ring_len(g)), np.uint32) if rings else None
    _check(lib().tvso_run_f64(ctypes.byref(g), _ptr(e), observer_height, first_angle,
                              n_angles, _ptr(cum), _ptr(r), threads or default_threads()))
    return cum, r


def sweep_sector(g, elevations, observer_height, deltas, dists, mode="exact32", rows=None,
                 cumulative=None, compact=False, rings=None, threads=None):
    """One sector in any mode over a row range (None = every row).

    cumulative (f32, or f64 for mode "fp64"; [rows * tvs_width]) is advanced in
    place (zeros when None).  Returns (cumulative, counts, ids): with
    compact=True, counts (u32 [total_bands], 0 outside the rows) and the ids of
    every band's ring record back to back in kernel-id order (the engine's
    compact stream); otherwise (cumulative, None, None).  rings (zeroed u32
    [total_bands * reserved], nullable) receives the reference's layout."""
    rb, re = (0, g.tvs_height) if rows is None else rows
    n = (re - rb) * g.tvs_width
    f64 = mode == "fp64"
    if cumulative is None:
        cumulative = np.zeros(n, np.float64 if f64 else np.float32)
    assert cumulative.dtype == (np.float64 if f64 else np.float32) and cumulative.size == n
    e = np.ascontiguousarray(elevations, np.float32)
    o = SweepOpts()
    o.mode = MODES[mode]
    o.row_begin, o.row_end = rb, re
    if f64:
        o.cum64 = cumulative.ctypes.data
    else:
        o.cum32 = cumulative.ctypes.data
    o.threads = threads or default_threads()
    if rings is not None:
        assert rings.dtype == np.uint32 and not compact
        o.rings, o.rings_len = rings.ctypes.data, rings.size
    counts = ids = None
    args = (ctypes.byref(g), _ptr(e), observer_height,
            _ptr(np.ascontiguousarray(deltas, np.int32)),
            _ptr(np.ascontiguousarray(dists, np.float32)))
    if compact:
        counts = np.zeros(g.total_bands, np.uint32)
        total = ctypes.c_uint64(0)
        saved = cumulative.copy()
        cap = 24 * max(n, 1) * 2
        ids = np.empty(cap, np.uint32)
        o.counts, o.ids, o.ids_cap = counts.ctypes.data, ids.ctypes.data, cap
        o.ids_total = ctypes.addressof(total)
        _check(lib().tvso_sweep_sector(*args, ctypes.byref(o)))
        if total.value > cap:  # the stream did not fit: once more with the exact size
            cumulative[:] = saved
            cap = total.value
            ids = np.empty(cap, np.uint32)
            o.ids, o.ids_cap = ids.ctypes.data, cap
            _check(lib().tvso_sweep_sector(*args, ctypes.byref(o)))
        ids = ids[:total.value]
    else:
        _check(lib().tvso_sweep_sector(*args, ctypes.byref(o)))
    return cumulative, counts, ids


def run_ex(g, elevations, observer_height, first_angle=0, n_angles=180, mode="exact32",
           rows=None, threads=None):
    """tvso_run over a row range in any mode: (cumulative, total or None)."""
    rb, re = (0, 0) if rows is None else rows
    nrows = (g.tvs_height if rows is None else re - rb)
    n = nrows * g.tvs_width
    e = np.ascontiguousarray(elevations, np.float32)
    if mode == "fp64":
        cum = np.empty(n, np.float64)
        _check(lib().tvso_run_ex(ctypes.byref(g), _ptr(e), observer_height, first_angle,
                                 n_angles, MODES[mode], rb, re, None, None, _ptr(cum),
                                 threads or default_threads()))
        return cum, None
    cum = np.empty(n, np.float32)
    total = np.empty(n, np.float32)
    _check(lib().tvso_run_ex(ctypes.byref(g), _ptr(e), observer_height, first_angle, n_angles,
                             MODES[mode], rb, re, _ptr(cum), _ptr(total), None,
                             threads or default_threads()))
    return cum, total


def ascii_viewshed(g, pov_id, all_ring_data, reserved):
    """output/ascii.rs:24-104: decode one PoV's viewshed from every sector's rings."""
    cells = ["."] * (g.width * g.height)

    def populate(opening, closing):
        cells[opening] = "+" if cells[opening] == "." else "±"
        cells[closing] = "-" if cells[closing] == "." else "±"
        if opening == closing:
            cells[opening] = "±"

    for sector in all_ring_data:
        it = iter(int(v) for v in sector)
        for _ in range(g.computable_points_count * 2):
            pairs = next(it) // 2
            band_pov = next(it)
            for index in range(pairs):
                opening = band_pov if index == 0 else next(it)
                closing = next(it)
                if band_pov == pov_id:
                    populate(opening, closing)
            skip = reserved - pairs * 2 - 2
            for _ in range(skip + 1):  # Iterator::nth(skip) consumes skip + 1 items
                next(it, None)
    cells[pov_id] = "o"
    return [" ".join(cells[r * g.width:(r + 1) * g.width]) for r in range(g.height)]
