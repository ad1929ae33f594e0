"""The C ABI without a GPU: the library loads, exports exactly what
include/tvs.h declares, and derives the reference's geometry (and its error
cases) identically to the oracle."""

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT


def header_functions():
    text = (ROOT / "include" / "tvs.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tvs_[a-z_0-9]+)\s*\(", text)) - {"tvs_sector_callback"})


def test_header_declares_every_binding(tvs):
    assert header_functions() == sorted(tvs.SIGNATURES)


def test_library_exports_every_declared_symbol(tvs):
    lib = tvs.lib()
    for name in header_functions():
        assert hasattr(lib, name), name
    assert lib.tvs_abi_version() == 5


def test_struct_layouts(tvs):
    assert ctypes.sizeof(tvs.Params) == 44
    assert ctypes.sizeof(tvs.Geometry) == 72
    assert ctypes.sizeof(tvs.SectorStats) == 24


CASES = [(301, 30.0, 3000, 5.0), (1201, 90.0, 36000, 5.0), (3601, 30.0, 36000, 5.0),
         (7201, 30.0, 72000, 5.0), (9, 1.0, 3, 5000.0), (100, 7.5, 333, 12.5),
         (257, 90.0, 7710, 5.0), (1000, 33.3, 10000, 3.0)]


@pytest.mark.parametrize("w,s,los,rpk", CASES)
def test_geometry_matches_oracle(tvs, oracle, w, s, los, rpk):
    g = tvs.compute_geometry(tvs.make_params(w, s, los, rings_per_km=rpk))
    o = oracle.geometry(w, s, los, rpk)
    for f in ("max_los_as_points", "band_size", "band_deltas_size", "tvs_width", "tvs_height",
              "reserved_rings_per_band", "size", "computable_points_count", "total_bands"):
        assert getattr(g, f) == getattr(o, f), f
    assert g.ring_slots_per_sector == o.total_bands * o.reserved_rings_per_band
    _, _, filled = oracle.compile_band_data(o, 3.0)
    assert g.band_steps_filled == filled


def test_rectangular_geometry(tvs, oracle):
    g = tvs.compute_geometry(tvs.make_params(400, 30.0, 3000, height=300))
    o = oracle.geometry(400, 30.0, 3000, 5.0, height=300)
    assert (g.tvs_width, g.tvs_height) == (o.tvs_width, o.tvs_height) == (200, 100)


@pytest.mark.parametrize("w,s,los,code", [
    (101, 1.0, 51, -2),      # dem.rs:56-62
    (101, 1.0, 1, -3),       # band_of_sight.rs index panic (band_size 2)
    (101, 1.0, 0, -3),
    (0, 1.0, 3, -1),
    (101, 0.0, 3, -1),
    (50000, 1.0, 3, -1),     # ids no longer fit i32
])
def test_geometry_errors(tvs, w, s, los, code):
    with pytest.raises(tvs.TvsError) as e:
        tvs.compute_geometry(tvs.make_params(w, s, los))
    assert e.value.code == code
    assert tvs.lib().tvs_last_error(None)


def test_create_validates_before_touching_a_device(tvs):
    z = np.zeros(10, np.float32)
    with pytest.raises(tvs.TvsError) as e:
        tvs.Engine(z, 301, 30.0, 3000)           # wrong elevation count
    assert e.value.code == tvs.ERR_INVALID_ARGUMENT


def test_no_device_is_reported(tvs):
    z = np.zeros(301 * 301, np.float32)
    try:
        eng = tvs.Engine(z, 301, 30.0, 3000)
    except tvs.TvsError as e:
        assert e.code == tvs.ERR_NO_DEVICE
        return
    eng.close()
    pytest.skip("a CUDA device is present")


def test_dem_mirror(tvs):
    dem = tvs.DEM(9, 1.0, 3)
    assert dem.computable_points_count == 9 and dem.band_deltas_size() == 3
    assert [dem.tvs_id_to_pov_id(t) for t in (0, 4, 8)] == [30, 40, 50]
    assert dem.pov_id_to_tvs_id(40) == 4
    with pytest.raises(tvs.TvsError):
        tvs.Compute("cpu", None, None, dem, 5.0)
