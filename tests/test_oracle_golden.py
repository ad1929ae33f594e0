"""Pin the CPU oracle to the reference's own unit-test vectors (transcribed into
tests/golden/reference_vectors.json by extract_reference_vectors.py).

Each test mirrors one reference test:
  axes.rs:216-333            at_0_degrees, at_135_degrees
  band_of_sight.rs:230-315   sector_at_{0,15,90,135}_degrees
  cache.rs:87-105           saves_and_loads (shape at 35 degrees)
  compute.rs:306-333         single_peak_totals, double_peak_totals
  compute.rs:358-416         viewsheds::{summit, off_summit, double_peak}
Float vectors are compared bit for bit: Rust prints the shortest decimal that
round-trips to the same f32."""

import numpy as np
import pytest

from conftest import f32


def reconstruct_bands(oracle, angle):
    """band_of_sight.rs:198-228."""
    g = oracle.geometry(9, 1.0, 3)
    assert g.computable_points_count == 9
    deltas, dists, _ = oracle.compile_band_data(g, float(angle))
    bands = []
    for point in range(g.computable_points_count):
        pov = ((point // g.tvs_width + g.max_los_as_points) * g.width
               + point % g.tvs_width + g.max_los_as_points)
        front, back = [pov], [pov]
        for d in deltas:
            front.append(front[-1] + int(d))
            back.append(back[-1] - int(d))
        bands.append(back[::-1])
        bands.append(front)
    return bands, dists


@pytest.mark.parametrize("angle", ["0", "135"])
def test_axes(oracle, golden, angle):
    want = golden["axes"][angle]
    d, sight, sector = oracle.axes(want["width"], float(angle))
    assert np.array_equal(d.view(np.uint32), f32(want["distances"]).view(np.uint32))
    assert sight.tolist() == want["sight_order"]
    assert sector.tolist() == want["sector_ordered"]


@pytest.mark.parametrize("angle", ["0", "15", "90", "135"])
def test_band_of_sight(oracle, golden, angle):
    want = golden["band_of_sight"][angle]
    bands, dists = reconstruct_bands(oracle, int(angle))
    assert bands == want["bands"]
    assert np.array_equal(dists.view(np.uint32), f32(want["distances"]).view(np.uint32))


def test_cache_shape_at_35(oracle, golden):
    want = golden["cache"]
    g = oracle.geometry(9, 1.0, 3)
    deltas, _, _ = oracle.compile_band_data(g, 35.0)
    assert deltas.tolist() == want["band_deltas"]
    d, _, _ = oracle.axes(9, 35.0)
    assert d.size == want["distances_len"]
    assert d[40] == np.float32(want["distance_40"])
    assert d[-1] == np.float32(want["distance_last"])


@pytest.mark.parametrize("name", ["single_peak", "double_peak"])
@pytest.mark.parametrize("threads", [1, 4])
def test_totals(oracle, golden, name, threads):
    c = golden["compute"]
    g = oracle.geometry(c["width"], c["scale"], c["max_line_of_sight"], c["rings_per_km"])
    cum, _, _ = oracle.run(g, f32(c["dems"][name]), c["observer_height"], threads=threads)
    assert np.array_equal(cum.view(np.uint32), f32(c["totals"][name]).view(np.uint32))


@pytest.mark.parametrize("name", ["summit", "off_summit", "double_peak"])
def test_viewsheds(oracle, golden, name):
    c = golden["compute"]
    v = c["viewsheds"][name]
    g = oracle.geometry(c["width"], c["scale"], c["max_line_of_sight"], c["rings_per_km"])
    _, _, rings = oracle.run(g, f32(c["dems"][v["dem"]]), c["observer_height"], rings=True)
    assert oracle.ascii_viewshed(g, v["pov_id"], rings, g.reserved_rings_per_band) == v["rows"]
