"""total-viewsheds_b200: the B200 total-viewshed engine behind a ctypes binding.

This module binds libtvs_cuda.so (include/tvs.h) and mirrors the reference's
host interface for the hot path, crates/total-viewsheds/src:

    DEM(width, scale, max_line_of_sight)      dem.rs:44-72
    Compute(method, ..., dem, rings_per_km)   compute.rs:27-84
    Compute.run() -> (cumulative, rings)      compute.rs:101-115
    Compute.compute_sector(angle, cum, rings) compute.rs:181-203 (ComputeType::Cuda)

There is no CPU fallback: every compute call goes through the CUDA library and
raises TvsError when it (or a GPU) is missing.
"""

import ctypes
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libtvs_cuda.so"
SECTOR_STEPS = 180

OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_LOS_TOO_LONG = -2
ERR_SHAPE = -3
ERR_PATH_OUT_OF_DEM = -4
ERR_RING_OVERFLOW = -5
ERR_CUDA = -6
ERR_NO_DEVICE = -7
ERR_OUT_OF_MEMORY = -8
ERR_CAPACITY = -9
ERR_TIMEOUT = -10

PRECISION = {"exact32": 0, "mixed64": 1, "fp64": 2, "fp32": 3}
SWEEP_KERNEL = {"engine": 0, "plain": 1}


class TvsError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"[{code}] {message}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("scale", ctypes.c_float),
        ("max_line_of_sight", ctypes.c_uint32),
        ("rings_per_km", ctypes.c_float),
        ("observer_height", ctypes.c_float),
        ("precision", ctypes.c_uint32),
        ("sweep_kernel", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("tvs_row_begin", ctypes.c_uint32),
        ("tvs_row_end", ctypes.c_uint32),
    ]


class Geometry(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_uint32),
        ("height", ctypes.c_uint32),
        ("max_los_as_points", ctypes.c_uint32),
        ("band_size", ctypes.c_uint32),
        ("band_deltas_size", ctypes.c_uint32),
        ("tvs_width", ctypes.c_uint32),
        ("tvs_height", ctypes.c_uint32),
        ("reserved_rings_per_band", ctypes.c_uint32),
        ("band_samples", ctypes.c_uint32),
        ("band_steps_filled", ctypes.c_uint32),
        ("size", ctypes.c_uint64),
        ("computable_points_count", ctypes.c_uint64),
        ("total_bands", ctypes.c_uint64),
        ("ring_slots_per_sector", ctypes.c_uint64),
    ]


class SectorStats(ctypes.Structure):
    _fields_ = [
        ("angle", ctypes.c_uint32),
        ("band_steps_filled", ctypes.c_uint32),
        ("overflow_bands", ctypes.c_uint32),
        ("max_ring_ids", ctypes.c_uint32),
        ("spill_entries", ctypes.c_uint64),
    ]


class SweepConfig(ctypes.Structure):
    _fields_ = [("points_x", ctypes.c_int32), ("points_y", ctypes.c_int32),
                ("packed", ctypes.c_int32), ("prefetch", ctypes.c_int32),
                ("layout", ctypes.c_int32)]

    def __repr__(self):
        return (f"{self.points_x}x{self.points_y}{' packed' if self.packed else ''}"
                f"{' prefetch' if self.prefetch else ''}"
                f"{f' split layout {self.layout}' if self.layout else ''}")


SECTOR_CALLBACK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32,
                                   ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint64,
                                   ctypes.POINTER(SectorStats))

# Every entry point of include/tvs.h with its ctypes signature.
_VP, _U32, _U64, _I32, _INT = (ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                               ctypes.c_int32, ctypes.c_int)
_P = ctypes.POINTER
SIGNATURES = {
    "tvs_abi_version": (_INT, []),
    "tvs_create": (_INT, [_P(Params), _VP, _U64, _P(_VP)]),
    "tvs_destroy": (None, [_VP]),
    "tvs_last_error": (ctypes.c_char_p, [_VP]),
    "tvs_compute_geometry": (_INT, [_P(Params), _P(Geometry)]),
    "tvs_get_geometry": (_INT, [_VP, _P(Geometry)]),
    "tvs_set_elevations": (_INT, [_VP, _VP, _U64]),
    "tvs_axes": (_INT, [_VP, _U32, _U64, _U64, _VP, _VP]),
    "tvs_band_shape": (_INT, [_VP, _U32, _VP, _VP, _P(_U32)]),
    "tvs_set_band_shape": (_INT, [_VP, _U32, _VP, _VP, _U64]),
    "tvs_compute_sector_rings": (_INT, [_VP, _U32, _VP, _P(_U64), _P(SectorStats)]),
    "tvs_compute_sectors_rings": (_INT, [_VP, _U32, _U32, _VP, _P(_U64), _P(SectorStats)]),
    "tvs_read_ring_records": (_INT, [_VP, _VP, _VP]),
    "tvs_clear_band_shapes": (_INT, [_VP]),
    "tvs_cache_load": (_INT, [_VP, ctypes.c_char_p, _P(_U32)]),
    "tvs_cache_save": (_INT, [_VP, ctypes.c_char_p, _INT]),
    "tvs_compute_sector": (_INT, [_VP, _U32, _VP, _VP, _U64, _P(SectorStats)]),
    "tvs_run": (_INT, [_VP, _VP, _VP, _INT, SECTOR_CALLBACK, _VP]),
    "tvs_device_reset": (_INT, [_VP]),
    "tvs_device_run_sectors": (_INT, [_VP, _U32, _U32]),
    "tvs_device_shape_sectors": (_INT, [_VP, _U32, _U32]),
    "tvs_device_sweep_sectors": (_INT, [_VP, _U32, _U32]),
    "tvs_device_finish": (_INT, [_VP]),
    "tvs_read_surfaces": (_INT, [_VP, _VP, _VP]),
    "tvs_device_cumulative": (_VP, [_VP]),
    "tvs_read_rechecks": (_INT, [_VP, _P(_U64), _INT]),
    "tvs_set_queue_wait": (_INT, [_VP, _U32, _U32]),
    "tvs_set_sweep_counters": (_INT, [_VP, _INT]),
    "tvs_read_sweep_counters": (_INT, [_VP, _P(_U64)]),
    "tvs_device_run_tvs": (_INT, [_VP]),
    "tvs_last_run_times": (_INT, [_VP, _P(ctypes.c_float), _P(ctypes.c_float)]),
    "tvs_measure_l1_load": (_INT, [_I32, _P(ctypes.c_double)]),
    "tvs_stream": (_VP, [_VP]),
    "tvs_last_launch_count": (_U64, [_VP]),
    "tvs_device_bytes": (_U64, [_VP]),
    "tvs_selftest_division": (_INT, [_I32, _U64, _U64, _P(_U64)]),
    "tvs_measure_fp32_issue": (_INT, [_I32, _P(ctypes.c_double)]),
    "tvs_compute_sector_noalloc": (_INT, [_P(Params), _VP, _U32, _VP, _VP, _VP]),
    "tvs_set_sweep_config": (_INT, [_VP, _P(SweepConfig)]),
    "tvs_get_sweep_config": (_INT, [_VP, _P(SweepConfig)]),
    "tvs_autotune": (_INT, [_VP, _U32, _P(SweepConfig)]),
    "tvs_batch_create": (_INT, [_P(Params), _P(ctypes.c_void_p), _U32, _P(_VP)]),
    "tvs_batch_destroy": (None, [_VP]),
    "tvs_batch_last_error": (ctypes.c_char_p, [_VP]),
    "tvs_batch_size": (_U32, [_VP]),
    "tvs_batch_geometry": (_INT, [_VP, _U32, _P(Geometry)]),
    "tvs_batch_set_sweep_config": (_INT, [_VP, _P(SweepConfig)]),
    "tvs_batch_get_sweep_config": (_INT, [_VP, _P(SweepConfig)]),
    "tvs_batch_autotune": (_INT, [_VP, _U32, _P(SweepConfig)]),
    "tvs_batch_run": (_INT, [_VP]),
    "tvs_batch_finish": (_INT, [_VP]),
    "tvs_batch_read": (_INT, [_VP, _U32, _VP, _VP]),
    "tvs_batch_stream": (_VP, [_VP]),
    "tvs_batch_device_bytes": (_U64, [_VP]),
}

_lib = None


def lib():
    """Load libtvs_cuda.so; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise TvsError(ERR_INVALID_ARGUMENT,
                           f"{LIB_PATH} is missing: build it with total-viewsheds_b200/build.py")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _raise(code, ctx=None):
    msg = lib().tvs_last_error(ctx)
    raise TvsError(code, msg.decode() if msg else "error")


def make_params(width, scale, max_line_of_sight, rings_per_km=5.0, observer_height=1.8,
                height=None, precision="exact32", sweep_kernel="engine", device=0,
                rows=None):
    p = Params()
    p.width = width
    p.height = width if height is None else height
    p.scale = scale
    p.max_line_of_sight = int(max_line_of_sight)
    p.rings_per_km = rings_per_km
    p.observer_height = observer_height
    p.precision = PRECISION[precision] if isinstance(precision, str) else precision
    p.sweep_kernel = SWEEP_KERNEL[sweep_kernel] if isinstance(sweep_kernel, str) else sweep_kernel
    p.device = device
    p.tvs_row_begin, p.tvs_row_end = (0, 0) if rows is None else rows
    return p


def compute_geometry(params):
    """DEM::new + Compute::new geometry (no GPU needed)."""
    g = Geometry()
    rc = lib().tvs_compute_geometry(ctypes.byref(params), ctypes.byref(g))
    if rc:
        _raise(rc)
    return g


class Engine:
    """One CUDA context (tvs_context) holding a DEM resident in HBM."""

    def __init__(self, elevations, width, scale, max_line_of_sight, **kw):
        self.params = make_params(width, scale, max_line_of_sight, **kw)
        e = np.ascontiguousarray(elevations, np.float32).ravel()
        ctx = ctypes.c_void_p()
        rc = lib().tvs_create(ctypes.byref(self.params), _ptr(e), e.size, ctypes.byref(ctx))
        if rc:
            _raise(rc)
        self.ctx = ctx
        self.geometry = Geometry()
        lib().tvs_get_geometry(self.ctx, ctypes.byref(self.geometry))

    def close(self):
        if getattr(self, "ctx", None):
            lib().tvs_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc:
            _raise(rc, self.ctx)

    @property
    def count(self):
        return self.geometry.computable_points_count

    def set_elevations(self, elevations):
        e = np.ascontiguousarray(elevations, np.float32).ravel()
        self._check(lib().tvs_set_elevations(self.ctx, _ptr(e), e.size))

    def axes(self, angle, first_rank=0, count=None, sight_distances=False):
        """(sector_ordered[first_rank:first_rank+count], f32 sight distances or None)."""
        n = self.geometry.size
        count = n - first_rank if count is None else count
        ids = np.empty(count, np.uint32)
        d = np.empty(n, np.float32) if sight_distances else None
        self._check(lib().tvs_axes(self.ctx, angle, first_rank, count, _ptr(ids), _ptr(d)))
        return ids, d

    def band_shape(self, angle):
        """(band_deltas i32, band_distances f32, band_steps_filled)."""
        n = self.geometry.band_deltas_size
        deltas = np.zeros(max(n, 1), np.int32)
        dists = np.zeros(max(n, 1), np.float32)
        filled = ctypes.c_uint32()
        self._check(lib().tvs_band_shape(self.ctx, angle, _ptr(deltas), _ptr(dists),
                                         ctypes.byref(filled)))
        return deltas[:n], dists[:n], filled.value

    def compute_sector_rings(self, angle, cumulative):
        """One sector, in place on cumulative, with its ring records as a compact
        stream: (band_offsets u64 [total_bands + 1], ids u32, SectorStats); band
        k's record is ids[band_offsets[k]:band_offsets[k + 1]]."""
        assert cumulative.dtype == np.float32 and cumulative.flags.c_contiguous
        total = ctypes.c_uint64()
        st = SectorStats()
        self._check(lib().tvs_compute_sector_rings(self.ctx, angle, _ptr(cumulative),
                                                   ctypes.byref(total), ctypes.byref(st)))
        offsets = np.empty(self.geometry.total_bands + 1, np.uint64)
        ids = np.empty(max(total.value, 1), np.uint32)
        self._check(lib().tvs_read_ring_records(self.ctx, _ptr(offsets), _ptr(ids)))
        return offsets, ids[:total.value], st

    def compute_sectors_rings(self, first_angle, n_sectors, cumulative):
        """Sectors first_angle .. first_angle + n_sectors - 1 in one launch, in
        place on cumulative: (band_offsets u64 [n_sectors * total_bands + 1], ids
        u32, SectorStats); band k of sector first_angle + s is record
        s * total_bands + k."""
        assert cumulative.dtype == np.float32 and cumulative.flags.c_contiguous
        total = ctypes.c_uint64()
        st = SectorStats()
        self._check(lib().tvs_compute_sectors_rings(self.ctx, first_angle, n_sectors, _ptr(cumulative),
                                                    ctypes.byref(total), ctypes.byref(st)))
        offsets = np.empty(n_sectors * self.geometry.total_bands + 1, np.uint64)
        ids = np.empty(max(total.value, 1), np.uint32)
        self._check(lib().tvs_read_ring_records(self.ctx, _ptr(offsets), _ptr(ids)))
        return offsets, ids[:total.value], st

    def set_band_shape(self, angle, deltas, distances):
        """Install a sector's band shape as tables (the reference's shape cache
        entries, cache.rs:50-60) in place of the computed one."""
        d = np.ascontiguousarray(deltas, np.int32)
        x = np.ascontiguousarray(distances, np.float32)
        self._check(lib().tvs_set_band_shape(self.ctx, angle, _ptr(d), _ptr(x),
                                             min(d.size, x.size)))

    def clear_band_shapes(self):
        self._check(lib().tvs_clear_band_shapes(self.ctx))

    def load_cache(self, state_directory):
        """Install every sector found in the reference's shape cache under
        state_directory (cache.rs:23-60); returns how many."""
        n = ctypes.c_uint32()
        self._check(lib().tvs_cache_load(self.ctx, os.fsencode(state_directory), ctypes.byref(n)))
        return n.value

    def save_cache(self, state_directory, overwrite=False):
        """Write every sector's band shape in the reference's shape cache layout
        (cache.rs:62-76); existing sector files are kept unless overwrite."""
        self._check(lib().tvs_cache_save(self.ctx, os.fsencode(state_directory),
                                         1 if overwrite else 0))

    def compute_sector(self, angle, cumulative, rings=None):
        """In place on cumulative (f32 [count]); rings (u32 [ring_slots]) receives the
        sector's ring records.  Returns SectorStats."""
        assert cumulative.dtype == np.float32 and cumulative.flags.c_contiguous
        st = SectorStats()
        self._check(lib().tvs_compute_sector(self.ctx, angle, _ptr(cumulative), _ptr(rings),
                                             0 if rings is None else rings.size,
                                             ctypes.byref(st)))
        return st

    def run(self, rings=False, on_sector=None):
        """All 180 sectors.  Returns (cumulative, heatmap total, [rings per sector] or None).

        on_sector(angle, rings_or_None, stats) is called after every sector."""
        cum = np.empty(self.count, np.float32)
        total = np.empty(self.count, np.float32)
        kept = [] if rings else None

        def cb(_user, angle, ptr, n, stats):
            r = None
            if ptr:
                r = np.ctypeslib.as_array(ptr, shape=(n,)).copy()
                if kept is not None:
                    kept.append(r)
            if on_sector is not None:
                on_sector(angle, r, stats.contents)
            return 0

        cfn = SECTOR_CALLBACK(cb)
        self._check(lib().tvs_run(self.ctx, _ptr(cum), _ptr(total), 1 if rings else 0, cfn,
                                  None))
        return cum, total, kept

    # device-resident form
    def device_reset(self):
        self._check(lib().tvs_device_reset(self.ctx))

    def device_run_sectors(self, first=0, count=SECTOR_STEPS):
        self._check(lib().tvs_device_run_sectors(self.ctx, first, count))

    def device_shape_sectors(self, first=0, count=SECTOR_STEPS):
        self._check(lib().tvs_device_shape_sectors(self.ctx, first, count))

    def device_sweep_sectors(self, first=0, count=SECTOR_STEPS):
        self._check(lib().tvs_device_sweep_sectors(self.ctx, first, count))

    def device_run_tvs(self):
        """Zero the surfaces and enqueue all 180 sectors (one graph replay
        after the first call)."""
        self._check(lib().tvs_device_run_tvs(self.ctx))

    def last_run_times(self):
        """(shape-stage ms, sweep ms) of the last device_run_tvs."""
        a, b = ctypes.c_float(), ctypes.c_float()
        self._check(lib().tvs_last_run_times(self.ctx, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def sweep_counters(self, enable=None):
        """Read the direction-split sweep counters ([swept, passed, all, 0]
        warp-steps); enable=True first zeroes them and turns counting on,
        enable=False turns it off (the counts are kept)."""
        if enable is not None:
            self._check(lib().tvs_set_sweep_counters(self.ctx, 1 if enable else 0))
        v = (ctypes.c_uint64 * 4)()
        self._check(lib().tvs_read_sweep_counters(self.ctx, v))
        return list(v)

    def device_finish(self):
        self._check(lib().tvs_device_finish(self.ctx))

    def read_surfaces(self):
        cum = np.empty(self.count, np.float32)
        total = np.empty(self.count, np.float32)
        self._check(lib().tvs_read_surfaces(self.ctx, _ptr(cum), _ptr(total)))
        return cum, total

    def stream(self):
        return lib().tvs_stream(self.ctx)

    def sweep_config(self):
        c = SweepConfig()
        self._check(lib().tvs_get_sweep_config(self.ctx, ctypes.byref(c)))
        return c

    def set_sweep_config(self, points_x, points_y, packed=False, prefetch=False, layout=0):
        c = SweepConfig(points_x, points_y, 1 if packed else 0, 1 if prefetch else 0, layout)
        self._check(lib().tvs_set_sweep_config(self.ctx, ctypes.byref(c)))

    def autotune(self, sample_sectors=4):
        """Time the sweep configurations on a few sectors and keep the fastest."""
        c = SweepConfig()
        self._check(lib().tvs_autotune(self.ctx, sample_sectors, ctypes.byref(c)))
        return c

    def set_queue_wait(self, spin_limit=0, held_tile=None):
        """The sweep's dependency-wait limit (0 = default) and, for failure
        tests, a tile whose completion is never signalled."""
        self._check(lib().tvs_set_queue_wait(self.ctx, spin_limit,
                                             0xFFFFFFFF if held_tile is None else held_tile))

    def read_rechecks(self, reset=True):
        """MIXED64: comparisons re-decided in FP64 since the last reset."""
        v = ctypes.c_uint64()
        self._check(lib().tvs_read_rechecks(self.ctx, ctypes.byref(v), 1 if reset else 0))
        return v.value

    def last_launch_count(self):
        return lib().tvs_last_launch_count(self.ctx)

    def device_bytes(self):
        return lib().tvs_device_bytes(self.ctx)


class Batch:
    """Many DEM tiles (uneven, possibly rectangular), all 180 sectors each, one
    shape launch and one persistent sweep per run (a replayed CUDA graph)."""

    def __init__(self, dems, **kw):
        """dems: list of (heights [H, W] f32, scale, max_line_of_sight)."""
        self.params = (Params * len(dems))()
        self._heights = []
        for i, (z, scale, los) in enumerate(dems):
            z = np.ascontiguousarray(z, np.float32)
            h, w = z.shape
            self.params[i] = make_params(w, scale, los, height=h, **kw)
            self._heights.append(z)
        ptrs = (ctypes.c_void_p * len(dems))(*[_ptr(z).value for z in self._heights])
        b = ctypes.c_void_p()
        rc = lib().tvs_batch_create(self.params, ptrs, len(dems), ctypes.byref(b))
        if rc:
            _raise(rc)
        self.b = b
        self.geometry = []
        for i in range(len(dems)):
            g = Geometry()
            lib().tvs_batch_geometry(self.b, i, ctypes.byref(g))
            self.geometry.append(g)

    def _check(self, rc):
        if rc:
            msg = lib().tvs_batch_last_error(self.b)
            raise TvsError(rc, msg.decode() if msg else "error")

    def close(self):
        if getattr(self, "b", None):
            lib().tvs_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return lib().tvs_batch_size(self.b)

    def autotune(self, sample_sectors=4):
        c = SweepConfig()
        self._check(lib().tvs_batch_autotune(self.b, sample_sectors, ctypes.byref(c)))
        return c

    def set_sweep_config(self, points_x, points_y, packed=False, prefetch=False, layout=0):
        c = SweepConfig(points_x, points_y, 1 if packed else 0, 1 if prefetch else 0, layout)
        self._check(lib().tvs_batch_set_sweep_config(self.b, ctypes.byref(c)))

    def run(self):
        self._check(lib().tvs_batch_run(self.b))

    def finish(self):
        self._check(lib().tvs_batch_finish(self.b))

    def read(self, dem):
        n = self.geometry[dem].computable_points_count
        cum = np.empty(n, np.float32)
        total = np.empty(n, np.float32)
        self._check(lib().tvs_batch_read(self.b, dem, _ptr(cum), _ptr(total)))
        return cum, total

    def stream(self):
        return lib().tvs_batch_stream(self.b)

    def device_bytes(self):
        return lib().tvs_batch_device_bytes(self.b)


def selftest_division(n, seed=0, device=0):
    out = ctypes.c_uint64()
    rc = lib().tvs_selftest_division(device, n, seed, ctypes.byref(out))
    if rc:
        _raise(rc)
    return out.value


def measure_l1_load(device=0):
    """Measured L1 load bytes per second on `device` (32-float warp loads)."""
    out = ctypes.c_double()
    rc = lib().tvs_measure_l1_load(device, ctypes.byref(out))
    if rc:
        _raise(rc)
    return out.value


def measure_fp32_issue(device=0):
    """Measured FP32 lane-instructions per second on `device`."""
    out = ctypes.c_double()
    rc = lib().tvs_measure_fp32_issue(device, ctypes.byref(out))
    if rc:
        _raise(rc)
    return out.value


class DEM:
    """dem.rs:44-140: geometry of a square (or, as an extension, W x H) DEM."""

    def __init__(self, width, scale, max_line_of_sight, height=None, rings_per_km=5.0):
        self.width = width
        self.height = width if height is None else height
        self.scale = scale
        self.max_line_of_sight = int(max_line_of_sight)
        g = compute_geometry(make_params(width, scale, max_line_of_sight,
                                         rings_per_km=rings_per_km, height=height))
        self.size = g.size
        self.max_los_as_points = g.max_los_as_points
        self.computable_points_count = g.computable_points_count
        self.tvs_width = g.tvs_width
        self.tvs_height = g.tvs_height
        self.band_size = g.band_size
        self.elevations = np.zeros(self.size, np.float32)

    def band_deltas_size(self):
        return self.band_size - 1                     # band_of_sight.rs:54-58

    def tvs_id_to_pov_id(self, tvs_id):               # dem.rs:121-127
        x = tvs_id % self.tvs_width + self.max_los_as_points
        y = tvs_id // self.tvs_width + self.max_los_as_points
        return y * self.width + x

    def pov_id_to_tvs_id(self, pov_id):               # dem.rs:110-118
        x = pov_id % self.width - self.max_los_as_points
        y = pov_id // self.width - self.max_los_as_points
        return y * self.tvs_width + x


class Compute:
    """compute.rs:6-241 with the `--compute cuda` backend.

    Only method="cuda" exists here; the reference's CPU and Vulkan arms are
    not part of this engine.  observer_height defaults to the reference's
    hard-coded 1.8 m (compute.rs:41)."""

    def __init__(self, method, state_directory, output_dir, dem, rings_per_km,
                 observer_height=1.8, keep_rings=True, precision="exact32",
                 sweep_kernel="engine", device=0):
        if method != "cuda":
            raise TvsError(ERR_INVALID_ARGUMENT, f"unsupported compute method {method!r}")
        self.dem = dem
        self.state_directory = state_directory
        self.output_dir = output_dir
        self.keep_rings = keep_rings
        self.engine = Engine(dem.elevations, dem.width, dem.scale, dem.max_line_of_sight,
                             height=dem.height, rings_per_km=rings_per_km,
                             observer_height=observer_height, precision=precision,
                             sweep_kernel=sweep_kernel, device=device)
        g = self.engine.geometry
        self.total_reserved_rings = g.ring_slots_per_sector
        self.reserved_rings_per_band = g.reserved_rings_per_band
        self.total_surfaces = np.zeros(g.computable_points_count, np.float32)

    def run(self):
        """compute.rs:101-115: returns (cumulative_surfaces, all_ring_data)."""
        cum, total, rings = self.engine.run(rings=self.keep_rings)
        self.total_surfaces = total
        return cum, (rings if rings is not None else [])

    def compute_sector(self, angle, cumulative_surfaces, ring_data=None):
        """compute.rs:181-203 for one sector (in place)."""
        st = self.engine.compute_sector(angle, cumulative_surfaces, ring_data)
        self.total_surfaces += cumulative_surfaces          # compute.rs:206-214
        return st
