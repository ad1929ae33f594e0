"""Batches of uneven, partly rectangular DEM tiles (one shape launch and one
persistent sweep per graph replay), the sweep configurations and the
autotuner: every configuration and every batch gives the single-DEM results
bit for bit, and rectangular tiles match the oracle's W x H restatement."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.fixture(scope="module")
def tiles(synth):
    rng = np.random.default_rng(7)
    out = []
    for i, (w, h) in enumerate([(257, 257), (311, 197), (180, 260), (403, 331), (220, 220)]):
        z = synth.fbm(w, h, float(rng.uniform(0.6, 0.9)), 100 + i, 0.0, 3000.0)
        scale = 30.0 if i % 2 == 0 else 90.0
        out.append((z, scale, int(min(w, h) / 3 * scale)))
    return out


def test_rectangular_engine_matches_oracle(tvs, oracle, tiles):
    z, scale, los = tiles[1]
    h, w = z.shape
    g = oracle.geometry(w, scale, los, height=h)
    c0, t0, _ = oracle.run(g, z, 1.65, 0, 180)
    with tvs.Engine(z, w, scale, los, height=h, observer_height=1.65) as eng:
        c1, t1, _ = eng.run()
    assert (eng.geometry.tvs_width, eng.geometry.tvs_height) == (g.tvs_width, g.tvs_height)
    assert np.array_equal(bits(c0), bits(c1)) and np.array_equal(bits(t0), bits(t1))


@pytest.mark.parametrize("precision", ["exact32", "mixed64"])
def test_batch_equals_single_dems(tvs, tiles, precision):
    singles = []
    for z, scale, los in tiles:
        h, w = z.shape
        with tvs.Engine(z, w, scale, los, height=h, observer_height=1.65,
                        precision=precision) as eng:
            singles.append(eng.run()[:2])
    with tvs.Batch(tiles, observer_height=1.65, precision=precision) as b:
        for _ in range(2):  # capture, then replay
            b.run()
            b.finish()
            for i, (c, t) in enumerate(singles):
                bc, bt = b.read(i)
                assert np.array_equal(bits(bc), bits(c)), i
                assert np.array_equal(bits(bt), bits(t)), i


def test_batch_autotune_keeps_results(tvs, tiles):
    with tvs.Batch(tiles, observer_height=1.65) as b:
        b.run()
        b.finish()
        before = [b.read(i) for i in range(len(tiles))]
        cfg = b.autotune(sample_sectors=3)
        assert (cfg.points_x, cfg.points_y) in [(1, 1), (2, 1), (4, 1), (2, 2)]
        b.run()
        b.finish()
        for i, (c, t) in enumerate(before):
            bc, bt = b.read(i)
            assert np.array_equal(bits(bc), bits(c)) and np.array_equal(bits(bt), bits(t))


@pytest.mark.parametrize("shape", [(1, 1, 0), (4, 1, 0), (2, 2, 0), (8, 1, 0), (2, 1, 1), (4, 1, 1),
                                   (1, 1, 0, 1), (2, 1, 0, 1), (4, 1, 0, 1), (2, 2, 0, 1),
                                   (8, 1, 0, 1)])
def test_sweep_configurations_agree(tvs, synth, shape):
    z = synth.config_dem("plain_cpu")
    with tvs.Engine(z, 301, 30.0, 3000, observer_height=1.65) as eng:
        want, wt, _ = eng.run()
        eng.set_sweep_config(*shape)
        got, gt, _ = eng.run()
    assert np.array_equal(bits(want), bits(got)) and np.array_equal(bits(wt), bits(gt))


@pytest.mark.parametrize("w,h,rows", [(301, 301, None), (311, 197, None), (301, 301, (37, 90)),
                                      (301, 301, (40, 41))])
@pytest.mark.parametrize("layout", [0, 1, 2, 3, 4, 5, 6, 7, 8, 9])
@pytest.mark.parametrize("precision,reference", [("mixed64", "fp64"), ("exact32", "exact32")])
def test_split_layouts_agree(tvs, synth, w, h, layout, rows, precision, reference):
    """Every sweep layout (rows of lanes over both directions, and one direction
    at a time over 8 x 4, 16 x 2 and 32 x 1 lanes, with each lane's four points of
    view in one row or in 2 x 2) gives the reference sweep bit
    for bit (MIXED64: the FP64 sweep; exact f32: the row layout, itself checked
    against the oracle elsewhere), on square and rectangular DEMs and on a row
    shard."""
    z = synth.fbm(w, h, 0.8, 11, 0.0, 1200.0)
    los = int(min(w, h) / 3 * 30.0)
    kw = dict(observer_height=1.65, height=h, rows=rows)
    with tvs.Engine(z, w, 30.0, los, precision=reference, **kw) as e64:
        if reference == "exact32":
            e64.set_sweep_config(2, 1)
        want, wt, _ = e64.run()
    with tvs.Engine(z, w, 30.0, los, precision=precision, **kw) as eng:
        eng.set_sweep_config(4, 1, layout=layout) if layout else eng.set_sweep_config(2, 1)
        assert eng.sweep_config().layout == layout
        got, gt, _ = eng.run()
    assert np.array_equal(bits(want), bits(got)) and np.array_equal(bits(wt), bits(gt))


def test_split_layout_is_not_for_fp64(tvs, synth):
    z = synth.config_dem("plain_cpu")
    with tvs.Engine(z, 301, 30.0, 3000, precision="fp64") as eng:
        with pytest.raises(tvs.TvsError):
            eng.set_sweep_config(4, 1, layout=1)


@pytest.mark.parametrize("precision", ["mixed64", "fp64"])
@pytest.mark.parametrize("shape", [(1, 1), (2, 1), (4, 1), (2, 2)])
def test_prefetch_configurations_agree_wide(tvs, synth, precision, shape):
    """The prefetching sweep gives the default sweep's FP64 and MIXED64
    results bit for bit."""
    z = synth.config_dem("plain_cpu")
    with tvs.Engine(z, 301, 30.0, 3000, observer_height=1.65, precision=precision) as eng:
        want, wt, _ = eng.run()
        eng.set_sweep_config(*shape, prefetch=True)
        assert eng.sweep_config().prefetch == 1
        got, gt, _ = eng.run()
    assert np.array_equal(bits(want), bits(got)) and np.array_equal(bits(wt), bits(gt))


def test_engine_autotune(tvs, synth):
    z = synth.config_dem("plain_gpu")
    with tvs.Engine(z, 1201, 90.0, 36000, observer_height=1.65) as eng:
        want, _, _ = eng.run()
        cfg = eng.autotune(sample_sectors=2)
        assert cfg.points_x in (1, 2, 4) and cfg.points_y in (1, 2)
        assert eng.sweep_config().points_x == cfg.points_x
        got, _, _ = eng.run()
    assert np.array_equal(bits(want), bits(got))


@pytest.mark.parametrize("kind", ["terraces", "steep"])
@pytest.mark.parametrize("layout", [1, 2, 3, 4, 5, 6, 7, 8, 9])
@pytest.mark.parametrize("precision,reference", [("mixed64", "fp64"), ("exact32", "exact32")])
def test_split_layouts_on_hard_terrain(tvs, synth, kind, layout, precision, reference):
    """The filtered layouts on terrain that stresses the filter: terraces (many
    equal elevations, so equal and near-equal angles) and 1 m cells with 6 km of
    relief (angles in the thousands, near the initial maximum of -2000)."""
    w = 161
    z = synth.fbm(w, w, 0.7, 5, 0.0, 1500.0)
    scale, los = 30.0, 1500
    if kind == "terraces":
        z = (np.round(z / 50.0) * 50.0).astype(np.float32)
    else:
        z = synth.fbm(w, w, 0.5, 6, 0.0, 6000.0)
        scale, los = 1.0, 50
    with tvs.Engine(z, w, scale, los, precision=reference, observer_height=1.65) as ref:
        if reference == "exact32":
            ref.set_sweep_config(2, 1)
        want, wt, _ = ref.run()
    with tvs.Engine(z, w, scale, los, precision=precision, observer_height=1.65) as eng:
        eng.set_sweep_config(4, 1, layout=layout)
        got, gt, _ = eng.run()
    assert np.array_equal(bits(want), bits(got)) and np.array_equal(bits(wt), bits(gt))
