"""The reference's own unit-test vectors, run through the CUDA engine's C ABI
(the same vectors that pin the oracle in test_oracle_golden.py).  Both sweep
kernels (the tiled engine and the plain one-thread-per-band port) must
reproduce them bit for bit."""

import numpy as np
import pytest

from conftest import f32

pytestmark = pytest.mark.gpu

KERNELS = ["engine", "plain"]


@pytest.mark.parametrize("angle", ["0", "135"])
def test_axes(tvs, golden, angle):
    """axes.rs:216-333: f32 sight distances and the full sector order of a 5x5 DEM."""
    want = golden["axes"][angle]
    with tvs.Engine(np.zeros(25, np.float32), 5, 1.0, 2) as eng:
        ids, d = eng.axes(int(angle), 0, 25, sight_distances=True)
    assert np.array_equal(d.view(np.uint32), f32(want["distances"]).view(np.uint32))
    assert ids.tolist() == want["sector_ordered"]


@pytest.mark.parametrize("angle", ["0", "15", "90", "135"])
def test_band_of_sight(tvs, golden, angle):
    """band_of_sight.rs:198-315: bands rebuilt from the GPU delta table."""
    want = golden["band_of_sight"][angle]
    with tvs.Engine(np.zeros(81, np.float32), 9, 1.0, 3) as eng:
        deltas, dists, filled = eng.band_shape(int(angle))
        g = eng.geometry
    assert filled == 3
    dem = tvs.DEM(9, 1.0, 3)
    bands = []
    for point in range(dem.computable_points_count):
        pov = dem.tvs_id_to_pov_id(point)
        front, back = [pov], [pov]
        for d in deltas:
            front.append(front[-1] + int(d))
            back.append(back[-1] - int(d))
        bands += [back[::-1], front]
    assert g.band_deltas_size == 3
    assert bands == want["bands"]
    assert np.array_equal(dists.view(np.uint32), f32(want["distances"]).view(np.uint32))


def test_cache_shape_at_35(tvs, golden):
    want = golden["cache"]
    with tvs.Engine(np.zeros(81, np.float32), 9, 1.0, 3) as eng:
        deltas, _, _ = eng.band_shape(35)
        _, d = eng.axes(35, 0, 1, sight_distances=True)
    assert deltas.tolist() == want["band_deltas"]
    assert d.size == want["distances_len"]
    assert d[40] == np.float32(want["distance_40"]) and d[-1] == np.float32(want["distance_last"])


def _compute(tvs, golden, dem_name, kernel):
    c = golden["compute"]
    dem = tvs.DEM(c["width"], c["scale"], c["max_line_of_sight"])
    dem.elevations = f32(c["dems"][dem_name])
    comp = tvs.Compute("cuda", None, None, dem, c["rings_per_km"],
                       observer_height=c["observer_height"], sweep_kernel=kernel)
    return comp, comp.run()


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("name", ["single_peak", "double_peak"])
def test_totals(tvs, golden, name, kernel):
    """compute.rs:306-333."""
    _, (cum, _) = _compute(tvs, golden, name, kernel)
    want = f32(golden["compute"]["totals"][name])
    assert np.array_equal(cum.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("name", ["summit", "off_summit", "double_peak"])
def test_viewsheds(tvs, oracle, golden, name, kernel):
    """compute.rs:358-416 through the reference's ASCII ring decoder."""
    v = golden["compute"]["viewsheds"][name]
    comp, (_, rings) = _compute(tvs, golden, v["dem"], kernel)
    assert len(rings) == 180
    g = oracle.geometry(9, 1.0, 3, 5000.0)
    assert oracle.ascii_viewshed(g, v["pov_id"], rings, comp.reserved_rings_per_band) == v["rows"]
