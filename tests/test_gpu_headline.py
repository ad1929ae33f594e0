"""The benchmark configurations themselves against the oracle.

The 3601^2 precision form (ridged multifractal with a flat 0 m sea, 1200-cell
line of sight) at the sectors where the reference's cost and tie behaviour
differ most (0, 1, 45, 46 and 90 degrees: the reference's README.md:110 notes that 0 degrees
is far faster than 1), the 7201^2 large region, and the 48-tile batching set.
Integer data (ring records) and the exact-f32 surfaces must match the oracle
bit for bit; MIXED64 and FP64 must match the oracle's all-FP64 restatement bit
for bit (surfaces rounded once to f32, ring records exactly)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRECISION = (3601, 30.0, 36000)
LARGE = (7201, 30.0, 72000)
SECTORS = (0, 1, 45, 46, 90)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def records(offsets, ids):
    """(counts per band, ids) of an engine compact stream."""
    return np.diff(offsets).astype(np.uint32), ids


@pytest.fixture(scope="module")
def dem3601(synth):
    return synth.config_dem("precision")


@pytest.fixture(scope="module")
def geom3601(oracle):
    w, s, los = PRECISION
    return oracle.geometry(w, s, los)


@pytest.fixture(scope="module")
def oracle3601(oracle, dem3601, geom3601):
    """Per sector: (f32 surfaces of that sector alone, counts, ids) in exact f32."""
    out = {}
    for a in SECTORS:
        d, x, _ = oracle.compile_band_data(geom3601, float(a))
        out[a] = oracle.sweep_sector(geom3601, dem3601, 1.65, d, x, compact=True)
    return out


def test_precision_form_device_path_and_heatmap(tvs, oracle, dem3601, geom3601):
    """The default (fastest) sweep over sectors 0, 1, 45, 46, 90 in that order:
    cumulative surfaces and the heatmap running total (compute.rs:206-214)."""
    w, s, los = PRECISION
    run_cum = np.zeros(geom3601.computable_points_count, np.float32)
    run_total = np.zeros_like(run_cum)
    for a in SECTORS:
        d, x, _ = oracle.compile_band_data(geom3601, float(a))
        oracle.sweep_sector(geom3601, dem3601, 1.65, d, x, cumulative=run_cum)
        run_total += run_cum
    with tvs.Engine(dem3601, w, s, los, observer_height=1.65) as eng:
        eng.device_reset()
        for a in SECTORS:
            eng.device_run_sectors(a, 1)
        eng.device_finish()
        c1, t1 = eng.read_surfaces()
    assert np.array_equal(bits(c1), bits(run_cum))
    assert np.array_equal(bits(t1), bits(run_total))


@pytest.mark.parametrize("angle", SECTORS)
def test_precision_form_sector_rings(tvs, dem3601, geom3601, oracle3601, angle):
    """One sector through the compact ring stream: surfaces and every band's
    ring record (kernel.rs:141-145,220-243) bit for bit."""
    w, s, los = PRECISION
    c0, n0, ids0 = oracle3601[angle]
    with tvs.Engine(dem3601, w, s, los, observer_height=1.65) as eng:
        cum = np.zeros(eng.count, np.float32)
        offsets, ids, st = eng.compute_sector_rings(angle, cum)
    n1, ids1 = records(offsets, ids)
    assert np.array_equal(bits(cum), bits(c0))
    assert np.array_equal(n1, n0)
    assert np.array_equal(ids1, ids0)
    assert st.max_ring_ids == int(n0.max())


@pytest.mark.parametrize("precision", ["mixed64", "fp64"])
@pytest.mark.parametrize("angle", [0, 46])
def test_precision_form_fp64_decisions(tvs, oracle, dem3601, geom3601, precision, angle):
    """MIXED64 (FP32 estimates, FP64 re-decisions) and the all-FP64 sweep equal
    the oracle's FP64 restatement: surfaces and ring records."""
    w, s, los = PRECISION
    d, x, _ = oracle.compile_band_data(geom3601, float(angle))
    c0, n0, ids0 = oracle.sweep_sector(geom3601, dem3601, 1.65, d, x, mode="fp64", compact=True)
    with tvs.Engine(dem3601, w, s, los, observer_height=1.65, precision=precision) as eng:
        cum = np.zeros(eng.count, np.float32)
        offsets, ids, _ = eng.compute_sector_rings(angle, cum)
        cum_dev = np.zeros(eng.count, np.float32)
        eng.device_reset()
        eng.device_run_sectors(angle, 1)
        eng.device_finish()
        cum_dev, _ = eng.read_surfaces()
    n1, ids1 = records(offsets, ids)
    assert np.array_equal(bits(cum), bits(c0.astype(np.float32)))
    assert np.array_equal(bits(cum_dev), bits(c0.astype(np.float32)))
    assert np.array_equal(n1, n0) and np.array_equal(ids1, ids0)


def test_large_region_sector(tvs, oracle, synth):
    """7201^2 with a 2400-cell line of sight (2x2 stitched fBm), sector 46:
    surfaces through the default sweep and ring records, against the oracle."""
    w, s, los = LARGE
    z = synth.config_dem("large")
    g = oracle.geometry(w, s, los)
    d, x, _ = oracle.compile_band_data(g, 46.0)
    c0, n0, ids0 = oracle.sweep_sector(g, z, 1.65, d, x, compact=True)
    with tvs.Engine(z, w, s, los, observer_height=1.65) as eng:
        eng.device_reset()
        eng.device_run_sectors(46, 1)
        eng.device_finish()
        c1, _ = eng.read_surfaces()
        cum = np.zeros(eng.count, np.float32)
        offsets, ids, _ = eng.compute_sector_rings(46, cum)
    assert np.array_equal(bits(c1), bits(c0))
    assert np.array_equal(bits(cum), bits(c0))
    n1, ids1 = records(offsets, ids)
    assert np.array_equal(n1, n0) and np.array_equal(ids1, ids0)


@pytest.fixture(scope="module")
def batch49(synth):
    """The benchmark's 48-tile batching set plus one square tile."""
    tiles = synth.batching_tiles(48, seed=synth.BASE_SEED + 3)
    tiles.append((synth.fbm(385, 385, 0.75, 4242, 0.0, 3000.0), 30.0, 3850))
    return tiles


@pytest.mark.parametrize("precision", ["exact32", "mixed64"])
def test_batching_set_equals_single_dems(tvs, batch49, precision):
    with tvs.Batch(batch49, observer_height=1.65, precision=precision) as b:
        b.run()
        b.finish()
        got = [b.read(i) for i in range(len(batch49))]
    for i, (z, scale, los) in enumerate(batch49):
        h, w = z.shape
        with tvs.Engine(z, w, scale, los, height=h, observer_height=1.65,
                        precision=precision) as eng:
            c, t, _ = eng.run()
        assert np.array_equal(bits(got[i][0]), bits(c)), i
        assert np.array_equal(bits(got[i][1]), bits(t)), i


def test_batching_set_square_and_smallest_tiles_match_oracle(tvs, oracle, batch49):
    with tvs.Batch(batch49, observer_height=1.65) as b:
        b.run()
        b.finish()
        sizes = [z.size for z, _, _ in batch49[:48]]
        for i in (48, int(np.argmin(sizes))):
            z, scale, los = batch49[i]
            h, w = z.shape
            g = oracle.geometry(w, scale, los, height=h)
            c0, t0, _ = oracle.run(g, z, 1.65)
            c1, t1 = b.read(i)
            assert np.array_equal(bits(c1), bits(c0)), i
            assert np.array_equal(bits(t1), bits(t0)), i
