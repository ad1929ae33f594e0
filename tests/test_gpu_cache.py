"""Band shapes given as tables and the reference's shape cache on disk
(cache.rs:23-78, compute.rs:118-162): the files the engine writes hold the
oracle's compile_band_data tables bit for bit, a context that loads them gives
the results of one that computes them, and an installed shape (any tables) is
swept exactly as the oracle sweeps those tables."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, SCALE, LOS, OBS = 301, 30.0, 3000, 1.65


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.fixture(scope="module")
def dem(synth):
    return synth.config_dem("plain_cpu")


@pytest.fixture(scope="module")
def state(tmp_path_factory, tvs, dem):
    d = tmp_path_factory.mktemp("state")
    with tvs.Engine(dem, W, SCALE, LOS, observer_height=OBS) as eng:
        eng.save_cache(d)
    return d


def test_saved_files_are_the_reference_tables(oracle, state):
    g = oracle.geometry(W, SCALE, LOS)
    base = state / "total-viewsheds" / str(W)
    for angle in range(180):
        d, x, _ = oracle.compile_band_data(g, float(angle))
        got_d = np.fromfile(base / "band_deltas" / f"{angle}.bin", np.int32)
        got_x = np.fromfile(base / "distances" / f"{angle}.bin", np.float32)
        assert np.array_equal(got_d, d), angle
        assert np.array_equal(bits(got_x), bits(x)), angle


@pytest.mark.parametrize("precision", ["exact32", "mixed64"])
def test_loaded_cache_gives_the_computed_results(tvs, dem, state, precision):
    with tvs.Engine(dem, W, SCALE, LOS, observer_height=OBS, precision=precision) as eng:
        want, wt, _ = eng.run()
    with tvs.Engine(dem, W, SCALE, LOS, observer_height=OBS, precision=precision) as eng:
        assert eng.load_cache(state) == 180
        got, gt, _ = eng.run()
    assert np.array_equal(bits(want), bits(got)) and np.array_equal(bits(wt), bits(gt))


def test_installed_foreign_shape_is_swept_like_the_oracle(tvs, oracle, dem):
    """Sector 10 given the tables of 37 degrees: surfaces and ring records are
    the oracle's sweep of those tables; tvs_band_shape returns them."""
    g = oracle.geometry(W, SCALE, LOS)
    d37, x37, f37 = oracle.compile_band_data(g, 37.0)
    want = np.zeros(g.computable_points_count, np.float32)
    want_r = np.zeros(oracle.ring_len(g), np.uint32)
    oracle.compute_sector(g, dem, OBS, d37, x37, want, want_r)
    with tvs.Engine(dem, W, SCALE, LOS, observer_height=OBS) as eng:
        eng.set_band_shape(10, d37, x37)
        d, x, filled = eng.band_shape(10)
        assert np.array_equal(d, d37) and np.array_equal(bits(x), bits(x37))
        assert filled == f37
        cum = np.zeros(eng.count, np.float32)
        rings = np.zeros(eng.geometry.ring_slots_per_sector, np.uint32)
        eng.compute_sector(10, cum, rings)
        assert np.array_equal(bits(cum), bits(want))
        assert np.array_equal(rings, want_r)
        # back to the computed shape
        eng.clear_band_shapes()
        d, _, _ = eng.band_shape(10)
        assert np.array_equal(d, oracle.compile_band_data(g, 10.0)[0])


def test_table_length_rules(tvs, oracle, dem):
    g = oracle.geometry(W, SCALE, LOS)
    d, x, filled = oracle.compile_band_data(g, 20.0)
    with tvs.Engine(dem, W, SCALE, LOS, observer_height=OBS) as eng:
        want, _, _ = eng.run()
        with pytest.raises(tvs.TvsError) as e:          # shorter than the kernel reads
            eng.set_band_shape(20, d[:-1], x[:-1])
        assert e.value.code == -3
        over_d, over_x = d.copy(), x.copy()
        over_d[filled + 1] = 7                          # fills past this geometry's band
        with pytest.raises(tvs.TvsError) as e:
            eng.set_band_shape(20, over_d, over_x)
        assert e.value.code == -3
        # longer tables: the first band_deltas_size entries count
        eng.set_band_shape(20, np.concatenate([d, [5, 6, 7]]), np.concatenate([x, [1.0, 2.0, 3.0]]))
        got, _, _ = eng.run()
    assert np.array_equal(bits(want), bits(got))


def test_partial_cache_and_rectangles(tvs, synth, tmp_path):
    """A sector missing one of its two files is computed (cache.rs:31); a
    rectangular DEM keeps its files under <width>x<height>."""
    z = synth.fbm(311, 197, 0.8, 3, 0.0, 900.0)
    los = int(197 / 3 * 30.0)
    with tvs.Engine(z, 311, 30.0, los, height=197, observer_height=OBS) as eng:
        want, _, _ = eng.run()
        eng.save_cache(tmp_path)
    base = tmp_path / "total-viewsheds" / "311x197"
    (base / "distances" / "5.bin").unlink()
    with tvs.Engine(z, 311, 30.0, los, height=197, observer_height=OBS) as eng:
        assert eng.load_cache(tmp_path) == 179
        got, _, _ = eng.run()
        eng.save_cache(tmp_path)                        # writes the missing sector only
    assert (base / "distances" / "5.bin").exists()
    assert np.array_equal(bits(want), bits(got))
