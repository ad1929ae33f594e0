"""The allocation-free sector entry point (tvs_compute_sector_noalloc).

It exists for callers that cannot allocate device memory when they call:
hosts whose device memory belongs to another allocator, and real-time callers
that forbid allocation after start-up.  The test allocates its own device
buffers (with torch, as such a caller's allocator would) and checks the entry
point against the regular per-sector entry point, bit for bit (the exact-f32
tolerance used by every parity test), on two calls in a row: the second call
finds the previous call's tables still in the shared scratch array.

This file is collected last so that a run stopping at the first failure has
already run every other test."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(tvs, params, d_elev, angle, d_cum, d_tot, stream):
    return tvs.lib().tvs_compute_sector_noalloc(
        ctypes.byref(params), ctypes.c_void_p(d_elev.data_ptr()), angle,
        ctypes.c_void_p(d_cum.data_ptr()),
        None if d_tot is None else ctypes.c_void_p(d_tot.data_ptr()),
        ctypes.c_void_p(stream.cuda_stream))


def test_noalloc_matches_compute_sector_twice(tvs, synth):
    import torch
    w, s, los = 301, 30.0, 3000
    z = synth.config_dem("plain_cpu")
    dev = torch.device("cuda", 0)
    d_elev = torch.from_numpy(np.ascontiguousarray(z, np.float32).ravel()).to(dev)
    params = tvs.make_params(w, s, los, observer_height=1.65)
    with tvs.Engine(z, w, s, los, observer_height=1.65) as eng:
        n = eng.count
        want = np.zeros(n, np.float32)
        want_total = np.zeros(n, np.float32)
        d_cum = torch.zeros(n, dtype=torch.float32, device=dev)
        d_tot = torch.zeros(n, dtype=torch.float32, device=dev)
        stream = torch.cuda.current_stream(dev)
        for angle in (17, 18):
            eng.compute_sector(angle, want)
            want_total += want
            rc = _call(tvs, params, d_elev, angle, d_cum, d_tot, stream)
            assert rc == 0, tvs.lib().tvs_last_error(None)
            got = d_cum.cpu().numpy()
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), angle
            assert np.array_equal(d_tot.cpu().numpy().view(np.uint32),
                                  want_total.view(np.uint32)), angle


def test_noalloc_allocates_nothing(tvs, synth):
    """After a first call (which loads the kernels and looks up the scratch
    array), further calls leave the device's free memory unchanged: the
    entry point takes no device memory of its own.  Also checks the forms the
    header allows: no heatmap total (d_total NULL) and a row range."""
    import torch
    w, s, los = 301, 30.0, 3000
    z = synth.config_dem("plain_cpu")
    dev = torch.device("cuda", 0)
    d_elev = torch.from_numpy(np.ascontiguousarray(z, np.float32).ravel()).to(dev)
    stream = torch.cuda.current_stream(dev)
    with tvs.Engine(z, w, s, los, observer_height=1.65) as eng:
        n, tw = eng.count, eng.geometry.tvs_width
        want = np.zeros(n, np.float32)
        eng.compute_sector(33, want)
    params = tvs.make_params(w, s, los, observer_height=1.65)
    d_cum = torch.zeros(n, dtype=torch.float32, device=dev)
    assert _call(tvs, params, d_elev, 33, d_cum, None, stream) == 0   # warm-up
    torch.cuda.synchronize(dev)
    free0, _ = torch.cuda.mem_get_info(dev)
    d_cum.zero_()
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    rc = _call(tvs, params, d_elev, 33, d_cum, None, stream)
    torch.cuda.synchronize(dev)
    free2, _ = torch.cuda.mem_get_info(dev)
    assert rc == 0, tvs.lib().tvs_last_error(None)
    assert free2 == free1 == free0
    assert np.array_equal(d_cum.cpu().numpy().view(np.uint32), want.view(np.uint32))
    # rows [40, 70) only: those rows equal the full sector, the others stay 0
    rows = tvs.make_params(w, s, los, observer_height=1.65, rows=(40, 70))
    d_cum.zero_()
    rc = _call(tvs, rows, d_elev, 33, d_cum, None, stream)
    assert rc == 0, tvs.lib().tvs_last_error(None)
    got = d_cum.cpu().numpy().reshape(-1, tw)
    full = want.reshape(-1, tw)
    assert np.array_equal(got[40:70].view(np.uint32), full[40:70].view(np.uint32))
    assert not got[:40].any() and not got[70:].any()


def test_noalloc_empty_grid_is_a_no_op(tvs):
    """A line of sight of exactly half the width leaves no computable point:
    the call does nothing and succeeds (the pointers are not read)."""
    import torch
    dev = torch.device("cuda", 0)
    dummy = torch.zeros(16, dtype=torch.float32, device=dev)
    params = tvs.make_params(200, 30.0, 3000, observer_height=1.65)
    assert tvs.compute_geometry(params).computable_points_count == 0
    rc = _call(tvs, params, dummy, 5, dummy, dummy, torch.cuda.current_stream(dev))
    assert rc == 0, tvs.lib().tvs_last_error(None)
    assert not dummy.any()


def test_noalloc_rejects_tables_beyond_its_scratch(tvs):
    import torch
    dev = torch.device("cuda", 0)
    dummy = torch.zeros(16, dtype=torch.float32, device=dev)
    # 7201^2 with a 2400-cell line of sight needs ~99 KB of tables (limit 64 KiB);
    # the size check comes before any device work, so the buffers are not read.
    params = tvs.make_params(7201, 30.0, 72000, observer_height=1.65)
    rc = _call(tvs, params, dummy, 0, dummy, None, torch.cuda.current_stream(dev))
    assert rc == tvs.ERR_CAPACITY
    assert b"no-allocation" in tvs.lib().tvs_last_error(None)
