"""The direction-split sweep (layouts 1-8) in every precision it runs, with
and without ring records, against the oracle.

EXACT32 must equal the reference f32 restatement, MIXED64 the all-FP64
restatement, and the reciprocal-table FP32 form the oracle's FP32 form, bit
for bit: surfaces, heatmap totals and every band's ring record (the compact
stream and the reference's reserved layout with its overflow semantics)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PLAIN_CPU = (301, 30.0, 3000)
ORACLE_MODE = {"exact32": "exact32", "mixed64": "fp64", "fp32": "fp32"}


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def f32(c):
    return c.astype(np.float32) if c.dtype == np.float64 else c


@pytest.fixture(scope="module")
def dem301(synth):
    return synth.config_dem("plain_cpu")


@pytest.fixture(scope="module")
def dem1201(synth):
    return synth.config_dem("plain_gpu")


@pytest.mark.parametrize("layout", [1, 2, 3, 4, 5, 6, 7, 8, 9])
def test_fp32_form_all_sectors(tvs, oracle, dem301, layout):
    w, s, los = PLAIN_CPU
    g = oracle.geometry(w, s, los)
    c0, t0 = oracle.run_ex(g, dem301, 1.65, mode="fp32")
    with tvs.Engine(dem301, w, s, los, observer_height=1.65, precision="fp32") as eng:
        eng.set_sweep_config(4, 1, layout=layout)
        c1, t1, _ = eng.run()
    assert np.array_equal(bits(c0), bits(c1)) and np.array_equal(bits(t0), bits(t1))


@pytest.mark.parametrize("angle", [0, 1, 45, 90])
def test_fp32_form_flat_sea_sector(tvs, oracle, dem1201, angle):
    """1201^2 with a flat 0 m sea (exact ties): surfaces and ring records."""
    w, s, los = 1201, 90.0, 36000
    g = oracle.geometry(w, s, los)
    d, x, _ = oracle.compile_band_data(g, float(angle))
    c0, n0, ids0 = oracle.sweep_sector(g, dem1201, 1.65, d, x, mode="fp32", compact=True)
    with tvs.Engine(dem1201, w, s, los, observer_height=1.65, precision="fp32") as eng:
        cum = np.zeros(eng.count, np.float32)
        offsets, ids, _ = eng.compute_sector_rings(angle, cum)
    assert np.array_equal(bits(cum), bits(c0))
    assert np.array_equal(np.diff(offsets).astype(np.uint32), n0)
    assert np.array_equal(ids, ids0)


@pytest.mark.parametrize("precision", ["exact32", "mixed64", "fp32"])
@pytest.mark.parametrize("layout", [1, 2, 3, 4, 5, 6, 7, 8, 9])
@pytest.mark.parametrize("rows", [None, (37, 90)])
def test_ring_records_every_layout(tvs, oracle, dem301, precision, layout, rows):
    """The compact stream straight from the split sweep, for a whole grid and a
    row shard (the other bands' records are empty)."""
    w, s, los = PLAIN_CPU
    g = oracle.geometry(w, s, los, 20.0)
    with tvs.Engine(dem301, w, s, los, rings_per_km=20.0, observer_height=1.65,
                    precision=precision, rows=rows) as eng:
        eng.set_sweep_config(4, 1, layout=layout)
        for angle in (0, 1, 46, 90, 133):
            d, x, _ = oracle.compile_band_data(g, float(angle))
            c0, n0, ids0 = oracle.sweep_sector(g, dem301, 1.65, d, x, mode=ORACLE_MODE[precision],
                                               rows=rows, compact=True)
            cum = np.zeros(eng.count, np.float32)
            offsets, ids, _ = eng.compute_sector_rings(angle, cum)
            assert np.array_equal(np.diff(offsets).astype(np.uint32), n0), angle
            assert np.array_equal(ids, ids0), angle
            rb, re = (0, g.tvs_height) if rows is None else rows
            mine = cum.reshape(g.tvs_height, -1)[rb:re].ravel()
            assert np.array_equal(bits(mine), bits(f32(c0))), angle


@pytest.mark.parametrize("precision", ["exact32", "mixed64", "fp32"])
@pytest.mark.parametrize("rpk", [5.0, 10.0, 20.0])
def test_reference_layout_every_precision(tvs, oracle, dem301, precision, rpk):
    """tvs_compute_sector's reserved-slot layout (kernel.rs:141-145,302-309),
    including the reference's overflow into later records at few slots."""
    w, s, los = PLAIN_CPU
    g = oracle.geometry(w, s, los, rpk)
    with tvs.Engine(dem301, w, s, los, rings_per_km=rpk, observer_height=1.65,
                    precision=precision) as eng:
        cum = np.zeros(eng.count, np.float32)
        rings = np.zeros(eng.geometry.ring_slots_per_sector, np.uint32)
        for angle in (2, 47):
            d, x, _ = oracle.compile_band_data(g, float(angle))
            r0 = np.zeros(oracle.ring_len(g), np.uint32)
            try:
                c0, _, _ = oracle.sweep_sector(g, dem301, 1.65, d, x, mode=ORACLE_MODE[precision],
                                               rings=r0)
                err0 = None
            except oracle.OracleError as e:
                err0 = e.code
            cum[:] = 0
            try:
                eng.compute_sector(angle, cum, rings)
                err1 = None
            except tvs.TvsError as e:
                err1 = e.code
            if err0 is not None:
                assert err0 == -5 and err1 == tvs.ERR_RING_OVERFLOW
                continue
            assert err1 is None
            assert np.array_equal(bits(cum), bits(f32(c0))), angle
            assert np.array_equal(rings, r0), angle


@pytest.mark.parametrize("precision", ["exact32", "mixed64", "fp32"])
def test_graph_replay_equals_the_oracle(tvs, oracle, dem301, precision):
    """tvs_device_run_tvs: plain launches on the first call, graph replays
    after; a new configuration or an installed shape recaptures it."""
    w, s, los = PLAIN_CPU
    g = oracle.geometry(w, s, los)
    if precision == "mixed64":
        c0 = oracle.run_f64(g, dem301, 1.65)[0].astype(np.float32)
        t0 = None
    else:
        c0, t0 = oracle.run_ex(g, dem301, 1.65, mode=ORACLE_MODE[precision])
    with tvs.Engine(dem301, w, s, los, observer_height=1.65, precision=precision) as eng:
        for layout in (None, 2):
            if layout:
                eng.set_sweep_config(4, 1, layout=layout)
            for _ in range(3):
                eng.device_run_tvs()
                eng.device_finish()
                c1, t1 = eng.read_surfaces()
                assert np.array_equal(bits(c1), bits(c0))
                if t0 is not None:
                    assert np.array_equal(bits(t1), bits(t0))
        shape_ms, sweep_ms = eng.last_run_times()
        assert shape_ms > 0 and sweep_ms > 0
        assert eng.last_launch_count() == 2          # the shape stage and the sweep
        d, x, _ = eng.band_shape(7)
        eng.set_band_shape(7, d, x)                   # one more launch: recaptured
        eng.device_run_tvs()
        eng.device_finish()
        assert eng.last_launch_count() == 3
        assert np.array_equal(bits(eng.read_surfaces()[0]), bits(c0))


@pytest.mark.parametrize("precision", ["exact32", "mixed64", "fp32"])
def test_sweep_counters(tvs, synth, precision):
    z = synth.config_dem("plain_gpu")
    with tvs.Engine(z, 1201, 90.0, 36000, observer_height=1.65, precision=precision) as eng:
        assert eng.sweep_counters(enable=True) == [0, 0, 0, 0]
        eng.device_reset()
        eng.device_run_sectors(0, 180)
        eng.device_finish()
        swept, passed, total, spare = eng.sweep_counters(enable=False)
    assert 0 < swept <= total and spare == 0
    assert passed <= swept if precision != "fp32" else passed == 0


def test_peak_probes(tvs):
    assert tvs.measure_fp32_issue(0) > 1e13      # FFMA lane-instructions / s
    assert tvs.measure_l1_load(0) > 1e12         # bytes / s


@pytest.mark.parametrize("precision", ["exact32", "mixed64", "fp32"])
def test_quad_layout_wide_steps(tvs, oracle, synth, precision):
    """A short line of sight on a wide DEM: at many angles a step moves a point
    of view more than the line of sight sideways, so the reference's linear
    sample ids wrap rows (kernel.rs:259-292).  The quad layout reads the plain
    DEM for those sectors; surfaces and ring records equal the oracle's at
    every angle whose bands stay on the DEM."""
    z = synth.fbm(101, 101, 0.8, 4, 0.0, 100.0)
    w, s, los = 101, 1.0, 10
    g = oracle.geometry(w, s, los)
    swept = 0
    with tvs.Engine(z, w, s, los, observer_height=1.65, precision=precision) as eng:
        eng.set_sweep_config(4, 1, layout=9)
        for angle in range(0, 180, 5):
            try:
                d, x, _ = oracle.compile_band_data(g, float(angle))
                c0, n0, ids0 = oracle.sweep_sector(g, z, 1.65, d, x, mode=ORACLE_MODE[precision],
                                                   compact=True)
            except oracle.OracleError as e:
                assert e.code == -4
                with pytest.raises(tvs.TvsError) as err:
                    eng.compute_sector(angle, np.zeros(eng.count, np.float32))
                assert err.value.code == tvs.ERR_PATH_OUT_OF_DEM
                continue
            cum = np.zeros(eng.count, np.float32)
            offsets, ids, _ = eng.compute_sector_rings(angle, cum)
            assert np.array_equal(bits(cum), bits(f32(c0))), angle
            assert np.array_equal(np.diff(offsets).astype(np.uint32), n0), angle
            assert np.array_equal(ids, ids0), angle
            swept += 1
    assert swept > 0


def test_mixed64_lean_form_long_line_of_sight(tvs, oracle, synth):
    """A 1900-cell line of sight: MIXED64's per-step tables would hold fewer
    CTAs per SM than the register limit, so its surfaces run the lean form (the
    maximum's step in registers, the FP64 addend recomputed from d).  Bit for
    bit the FP64 oracle, on several layouts."""
    w, s, los = 3900, 30.0, 57000
    z = synth.fbm(w, w, 0.8, 21, 0.0, 3000.0)
    g = oracle.geometry(w, s, los)
    assert g.max_los_as_points == 1900 and g.tvs_width == 100
    want = {}
    for angle in (0, 46, 90):
        d, x, _ = oracle.compile_band_data(g, float(angle))
        want[angle] = oracle.sweep_sector(g, z, 1.65, d, x, mode="fp64")[0]
    with tvs.Engine(z, w, s, los, observer_height=1.65, precision="mixed64") as eng:
        for layout in (1, 5, 9):
            eng.set_sweep_config(4, 1, layout=layout)
            for angle, c0 in want.items():
                cum = np.zeros(eng.count, np.float32)
                eng.compute_sector(angle, cum)
                assert np.array_equal(bits(cum), bits(f32(c0))), (layout, angle)
