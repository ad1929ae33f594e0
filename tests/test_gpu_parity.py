"""CUDA engine against the CPU oracle on seeded synthetic DEMs.

Integer and index data (delta tables, ring records) and the exact-f32
surfaces must match bit for bit; the FP64 sweep must match the oracle's FP64
restatement bit for bit too.  Sizes are the benchmark configurations (or
stated subsets of their sectors) so the oracle finishes in seconds."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PLAIN_CPU = (301, 30.0, 3000)
PLAIN_GPU = (1201, 90.0, 36000)
PRECISION = (3601, 30.0, 36000)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.fixture(scope="module")
def dem301(synth):
    return synth.config_dem("plain_cpu")


@pytest.fixture(scope="module")
def dem1201(synth):
    return synth.config_dem("plain_gpu")


def test_division_identity(tvs):
    """The table division equals CUDA's IEEE division on 2^28 random pairs."""
    assert tvs.selftest_division(1 << 28, seed=12345) == 0


@pytest.mark.parametrize("cfg", [PLAIN_CPU, PLAIN_GPU, (257, 90.0, 7710), (640, 30.0, 9000)])
def test_shapes_every_sector(tvs, oracle, cfg):
    w, s, los = cfg
    g = oracle.geometry(w, s, los)
    with tvs.Engine(np.zeros(w * w, np.float32), w, s, los) as eng:
        for angle in range(180):
            d0, x0, f0 = oracle.compile_band_data(g, float(angle))
            d1, x1, f1 = eng.band_shape(angle)
            assert f0 == f1, angle
            assert np.array_equal(d0, d1), angle
            assert np.array_equal(bits(x0), bits(x1)), angle


@pytest.mark.parametrize("angle", [0, 1, 45, 46, 90, 135, 179])
def test_shapes_3601(tvs, oracle, angle):
    w, s, los = PRECISION
    g = oracle.geometry(w, s, los)
    d0, x0, f0 = oracle.compile_band_data(g, float(angle))
    with tvs.Engine(np.zeros(w * w, np.float32), w, s, los) as eng:
        d1, x1, f1 = eng.band_shape(angle)
    assert f0 == f1 and np.array_equal(d0, d1) and np.array_equal(bits(x0), bits(x1))


@pytest.mark.parametrize("angle", [0, 45, 91, 150])
def test_sector_order_window(tvs, oracle, angle):
    """tvs_axes against the full reference sort, on a window and at the ends."""
    w = 211
    _, _, sector = oracle.axes(w, float(angle))
    with tvs.Engine(np.zeros(w * w, np.float32), w, 10.0, 600) as eng:
        for first, count in [(w * w // 2 - 500, 1000), (0, 700), (w * w - 300, 300)]:
            ids, _ = eng.axes(angle, first, count)
            assert np.array_equal(ids, sector[first:first + count]), (first, count)


@pytest.mark.parametrize("kernel", ["engine", "plain"])
def test_surfaces_301_all_sectors(tvs, oracle, dem301, kernel):
    w, s, los = PLAIN_CPU
    g = oracle.geometry(w, s, los)
    c0, t0, _ = oracle.run(g, dem301, 1.65)
    with tvs.Engine(dem301, w, s, los, observer_height=1.65, sweep_kernel=kernel) as eng:
        c1, t1, _ = eng.run()
    assert np.array_equal(bits(c0), bits(c1))
    assert np.array_equal(bits(t0), bits(t1))


@pytest.mark.parametrize("kernel", ["engine", "plain"])
def test_rings_301_all_sectors(tvs, oracle, dem301, kernel):
    w, s, los = PLAIN_CPU
    rpk = 20.0
    g = oracle.geometry(w, s, los, rpk)
    c0, _, r0 = oracle.run(g, dem301, 1.65, rings=True)
    with tvs.Engine(dem301, w, s, los, rings_per_km=rpk, observer_height=1.65,
                    sweep_kernel=kernel) as eng:
        c1, _, r1 = eng.run(rings=True)
    assert np.array_equal(bits(c0), bits(c1))
    assert len(r1) == 180
    for a in range(180):
        assert np.array_equal(r0[a], r1[a]), a


@pytest.mark.parametrize("rpk", [5.0, 8.0, 10.0, 11.0, 12.0])
def test_ring_overflow_matches_reference_semantics(tvs, oracle, dem301, rpk):
    """Too few slots: ids spill into the next records exactly as the reference's
    sequential writes do, or both report the reference's out-of-bounds panic."""
    w, s, los = PLAIN_CPU
    g = oracle.geometry(w, s, los, rpk)
    try:
        _, _, r0 = oracle.run(g, dem301, 1.65, 0, 30, rings=True)
        err0 = None
    except oracle.OracleError as e:
        err0 = e.code
    with tvs.Engine(dem301, w, s, los, rings_per_km=rpk, observer_height=1.65) as eng:
        cum = np.zeros(eng.count, np.float32)
        rings = np.zeros(eng.geometry.ring_slots_per_sector, np.uint32)
        err1 = None
        got = []
        overflowed = 0
        for a in range(30):
            try:
                st = eng.compute_sector(a, cum, rings)
            except tvs.TvsError as e:
                err1 = e.code
                break
            overflowed += st.overflow_bands
            got.append(rings.copy())
    if err0 is not None:
        assert err0 == -5 and err1 == tvs.ERR_RING_OVERFLOW
        return
    assert err1 is None and overflowed > 0
    for a in range(30):
        assert np.array_equal(r0[a], got[a]), a


@pytest.mark.parametrize("angle", [0, 1, 45, 46, 90, 179])
def test_sector_1201_with_flat_sea(tvs, oracle, dem1201, angle):
    w, s, los = PLAIN_GPU
    g = oracle.geometry(w, s, los)
    deltas, dists, _ = oracle.compile_band_data(g, float(angle))
    c0 = np.zeros(g.computable_points_count, np.float32)
    r0 = np.zeros(oracle.ring_len(g), np.uint32)
    oracle.compute_sector(g, dem1201, 1.65, deltas, dists, c0, r0)
    with tvs.Engine(dem1201, w, s, los, observer_height=1.65) as eng:
        c1 = np.zeros(eng.count, np.float32)
        r1 = np.zeros(eng.geometry.ring_slots_per_sector, np.uint32)
        eng.compute_sector(angle, c1, r1)
    assert np.array_equal(bits(c0), bits(c1))
    assert np.array_equal(r0, r1)


def test_fp64_sweep_matches_fp64_oracle(tvs, oracle, dem301):
    w, s, los = PLAIN_CPU
    rpk = 20.0
    g = oracle.geometry(w, s, los, rpk)
    c0, r0 = oracle.run_f64(g, dem301, 1.65, rings=True)
    with tvs.Engine(dem301, w, s, los, rings_per_km=rpk, observer_height=1.65,
                    precision="fp64") as eng:
        c1, _, r1 = eng.run(rings=True)
    assert np.array_equal(bits(c0.astype(np.float32)), bits(c1))
    for a in range(180):
        assert np.array_equal(r0[a], r1[a]), a


def test_row_shards_reassemble(tvs, dem301):
    w, s, los = PLAIN_CPU
    with tvs.Engine(dem301, w, s, los, observer_height=1.65) as eng:
        full, total, _ = eng.run()
        tw = eng.geometry.tvs_width
    parts = []
    for rows in [(0, 40), (40, 41), (41, tw)]:
        with tvs.Engine(dem301, w, s, los, observer_height=1.65, rows=rows) as eng:
            c, _, _ = eng.run()
        parts.append(c.reshape(tw, tw)[rows[0]:rows[1]])
    assert np.array_equal(bits(np.concatenate(parts).ravel()), bits(full))


def test_path_off_the_dem_is_an_error(tvs, oracle, synth):
    """A short line of sight on a wide DEM makes the strip's steps long enough
    to leave the DEM at most angles: the reference panics (kernel.rs:164).
    The engine reports the same sectors as errors and computes the others."""
    z = synth.fbm(101, 101, 0.8, 4, 0.0, 100.0)
    g = oracle.geometry(101, 1.0, 10)
    outcomes = []
    with tvs.Engine(z, 101, 1.0, 10, observer_height=1.65) as eng:
        for angle in range(0, 180, 15):
            try:
                c0, _, _ = oracle.run(g, z, 1.65, angle, 1)
                e0 = 0
            except oracle.OracleError as e:
                e0 = e.code
            c1 = np.zeros(eng.count, np.float32)
            try:
                eng.compute_sector(angle, c1)
                e1 = 0
            except tvs.TvsError as e:
                e1 = e.code
            outcomes.append((e0, e1))
            if e0 == 0:
                assert e1 == 0 and np.array_equal(bits(c0), bits(c1)), angle
            else:
                assert e0 == -4 and e1 == tvs.ERR_PATH_OUT_OF_DEM, angle
        with pytest.raises(tvs.TvsError) as e:
            eng.run()
        assert e.value.code == tvs.ERR_PATH_OUT_OF_DEM
    assert {o[0] for o in outcomes} == {0, -4}


def test_set_elevations_and_device_path(tvs, oracle, synth):
    w, s, los = 257, 90.0, 7710
    z1 = synth.fbm(w, w, 0.7, 11, 0.0, 3000.0)
    z2 = synth.fbm(w, w, 0.9, 12, 0.0, 3000.0)
    g = oracle.geometry(w, s, los)
    c2, t2, _ = oracle.run(g, z2, 1.65)
    with tvs.Engine(z1, w, s, los, observer_height=1.65) as eng:
        eng.run()
        eng.set_elevations(z2)
        eng.device_reset()
        eng.device_run_sectors(0, 90)
        eng.device_run_sectors(90, 90)
        eng.device_finish()
        c, t = eng.read_surfaces()
    assert np.array_equal(bits(c), bits(c2)) and np.array_equal(bits(t), bits(t2))


def test_mixed64_matches_fp64_oracle(tvs, oracle, dem301):
    """MIXED64 decides every comparison as the all-FP64 sweep does and sums the
    surfaces in FP64 in step order, so it equals the FP64 oracle bit for bit."""
    w, s, los = PLAIN_CPU
    rpk = 20.0
    g = oracle.geometry(w, s, los, rpk)
    c0, r0 = oracle.run_f64(g, dem301, 1.65, rings=True)
    with tvs.Engine(dem301, w, s, los, rings_per_km=rpk, observer_height=1.65,
                    precision="mixed64") as eng:
        c1, _, _ = eng.run()
        c2, _, r2 = eng.run(rings=True)
    assert np.array_equal(bits(c0.astype(np.float32)), bits(c1))
    assert np.array_equal(bits(c1), bits(c2))
    for a in range(180):
        assert np.array_equal(r0[a], r2[a]), a


@pytest.mark.parametrize("cfg,name", [(PLAIN_GPU, "plain_gpu"), ((2401, 30.0, 24000), "medium")])
def test_mixed64_equals_fp64_sweep(tvs, synth, cfg, name):
    """Flat 0 m sea and ridges at 1201^2 and 2401^2: MIXED64 == FP64, all sectors."""
    w, s, los = cfg
    z = synth.config_dem(name)
    with tvs.Engine(z, w, s, los, observer_height=1.65, precision="fp64") as eng:
        c64, t64, _ = eng.run()
    with tvs.Engine(z, w, s, los, observer_height=1.65, precision="mixed64") as eng:
        cm, tm, _ = eng.run()
    assert np.array_equal(bits(c64), bits(cm)) and np.array_equal(bits(t64), bits(tm))


@pytest.mark.parametrize("angle", [0, 46])
def test_shapes_7201(tvs, oracle, angle):
    """The large-region geometry (7201^2, 2400-cell line of sight): 6791-point
    windows of a 51.9 M-point sector order."""
    w, s, los = 7201, 30.0, 72000
    g = oracle.geometry(w, s, los)
    d0, x0, f0 = oracle.compile_band_data(g, float(angle))
    with tvs.Engine(np.zeros(w * w, np.float32), w, s, los) as eng:
        d1, x1, f1 = eng.band_shape(angle)
    assert f0 == f1 and np.array_equal(d0, d1) and np.array_equal(bits(x0), bits(x1))


@pytest.mark.parametrize("w,h,s", [(311, 197, 90.0), (180, 260, 30.0), (640, 301, 30.0)])
def test_rectangular_shapes_every_sector(tvs, oracle, w, h, s):
    """Rectangular DEMs build each sector's shape on the central min(W, H) square."""
    los = int(min(w, h) / 3 * s)
    g = oracle.geometry(w, s, los, height=h)
    with tvs.Engine(np.zeros(w * h, np.float32), w, s, los, height=h) as eng:
        for angle in range(180):
            d0, x0, f0 = oracle.compile_band_data(g, float(angle))
            d1, x1, f1 = eng.band_shape(angle)
            assert f0 == f1 and np.array_equal(d0, d1), angle
            assert np.array_equal(bits(x0), bits(x1)), angle


@pytest.mark.parametrize("precision", ["fp64", "mixed64"])
def test_fp64_compute_sector_matches_oracle(tvs, oracle, dem1201, precision):
    """One sector in double from the caller's f32 surfaces, with ring records."""
    w, s, los = PLAIN_GPU
    angle = 45
    g = oracle.geometry(w, s, los)
    deltas, dists, _ = oracle.compile_band_data(g, float(angle))
    c0 = np.zeros(g.computable_points_count, np.float64)
    r0 = np.zeros(oracle.ring_len(g), np.uint32)
    oracle.compute_sector(g, dem1201, 1.65, deltas, dists, c0, r0, f64=True)
    with tvs.Engine(dem1201, w, s, los, observer_height=1.65, precision=precision) as eng:
        c1 = np.zeros(eng.count, np.float32)
        r1 = np.zeros(eng.geometry.ring_slots_per_sector, np.uint32)
        eng.compute_sector(angle, c1, r1)
    assert np.array_equal(bits(c0.astype(np.float32)), bits(c1))
    assert np.array_equal(r0, r1)
