"""Properties of the CPU oracle beyond the reference's vectors: the stable radix
order against a second, independent sort; thread-count invariance; the
reference's panic cases as error codes; the unfilled delta-table tail."""

import numpy as np
import pytest

from conftest import f32


def radix_key(values32):
    bits = values32.view(np.uint32)
    mask = (-(bits >> 31).astype(np.int64)).astype(np.uint32) | np.uint32(0x80000000)
    return bits ^ mask


@pytest.mark.parametrize("width,angle", [(64, 0.0), (64, 33.0), (97, 90.0), (301, 135.0),
                                         (301, 179.0)])
def test_order_matches_lexsort(oracle, width, angle):
    """radsort's stable LSD order == a sort on (f32 key, index)."""
    d = oracle.calculate_distances(width, angle + 0.001)
    order = oracle.order_by_distance(d)
    keys = radix_key(d.astype(np.float32))
    ref = np.lexsort((np.arange(d.size), keys))
    assert np.array_equal(order, ref.astype(np.uint32))


def test_negative_zero_sorts_before_positive_zero(oracle):
    d = np.array([0.0, -0.0, 1e-50, -1e-50, 0.0], np.float64)
    # f32 casts: 0, -0, +0 (underflow), -0 (underflow), 0
    order = oracle.order_by_distance(d)
    assert order.tolist() == [1, 3, 0, 2, 4]


def test_threads_do_not_change_results(oracle, synth):
    z = synth.fbm(81, 81, 0.7, 7, 0.0, 300.0)
    g = oracle.geometry(81, 10.0, 300, 50.0)
    a = oracle.run(g, z, 1.65, 0, 30, rings=True, threads=1)
    b = oracle.run(g, z, 1.65, 0, 30, rings=True, threads=6)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_unfilled_delta_tail(oracle):
    """band_of_sight.rs:158 fills 2*band_size - band_samples/2 entries of the
    band_size - 1 table; the rest keep delta 0 and distance 0."""
    g = oracle.geometry(301, 30.0, 3000)
    deltas, dists, filled = oracle.compile_band_data(g, 17.0)
    assert g.band_deltas_size == 100 and filled == 60
    assert not deltas[filled:].any() and not dists[filled:].any()
    assert (dists[:filled] > 0).all()


def test_los_too_long(oracle):
    with pytest.raises(oracle.OracleError) as e:
        oracle.geometry(101, 1.0, 51)
    assert e.value.code == -2


def test_los_too_short_for_shape(oracle):
    g = oracle.geometry(101, 1.0, 1)  # band_size 2: band_of_sight.rs indexes past the table
    with pytest.raises(oracle.OracleError) as e:
        oracle.compile_band_data(g, 0.0)
    assert e.value.code == -3


def test_ring_overflow_past_buffer_end_is_an_error(oracle, synth):
    z = synth.fbm(301, 301, 0.8, 20261203, 0.0, 1500.0)
    g = oracle.geometry(301, 30.0, 3000, 5.0)  # 15 slots: the reference panics
    with pytest.raises(oracle.OracleError) as e:
        oracle.run(g, z, 1.65, 0, 180, rings=True)
    assert e.value.code == -5


def test_f64_close_to_f32(oracle, synth):
    z = synth.fbm(61, 61, 0.8, 3, 0.0, 200.0)
    g = oracle.geometry(61, 5.0, 100)
    c32, _, _ = oracle.run(g, z, 1.65, 0, 180)
    c64, _ = oracle.run_f64(g, z, 1.65, 0, 180)
    rel = np.abs(c32 - c64) / np.maximum(np.abs(c64), 1e-9)
    assert rel.max() < 5e-3
    assert np.median(rel) < 1e-5


def test_geometry_matches_dem_rs(oracle):
    """dem.rs:44-82 for the benchmark configurations."""
    for w, s, los, lp, tvs in [(301, 30.0, 3000, 100, 101), (1201, 90.0, 36000, 400, 401),
                               (3601, 30.0, 36000, 1200, 1201), (7201, 30.0, 72000, 2400, 2401)]:
        g = oracle.geometry(w, s, los)
        assert (g.max_los_as_points, g.tvs_width, g.computable_points_count) == (lp, tvs, tvs * tvs)
        assert g.band_size == lp + 1 and g.total_bands == 2 * tvs * tvs


def test_zero_total_bands_is_fine(oracle):
    g = oracle.geometry(9, 1.0, 4)
    z = f32(np.arange(81) % 5)
    cum, total, _ = oracle.run(g, z, 1.8, 0, 3)
    assert cum.size == g.computable_points_count


@pytest.mark.parametrize("w,h", [(311, 197), (180, 260), (97, 61)])
def test_rectangular_shapes_stay_on_the_dem(oracle, synth, w, h):
    """With the line of sight at a third of the shorter side, bands built on the
    central square never leave a rectangular DEM (every sector runs)."""
    s = 30.0
    g = oracle.geometry(w, s, int(min(w, h) / 3 * s), height=h)
    z = synth.fbm(w, h, 0.8, 3, 0.0, 500.0)
    cum, _, _ = oracle.run(g, z, 1.65, 0, 180)
    assert np.isfinite(cum).all() and cum.size == g.tvs_width * g.tvs_height


def test_square_window_is_the_whole_dem(oracle):
    """For a square DEM the window construction is the reference's: rebuild
    band_of_sight.rs:95-170 from the full sorts of tvso_axes and compare."""
    g = oracle.geometry(61, 5.0, 100)
    size = 61 * 61
    bs = int((2 * g.band_size) * 1.4142135623730951)
    for angle in (0.0, 37.0, 135.0, 179.0):
        dist, sight, sector = oracle.axes(61, angle)
        rank = np.empty(size, np.int64)
        rank[sight] = np.arange(size)
        window = sector[size // 2 - bs // 2: size // 2 - bs // 2 + bs]
        strip = window[np.argsort(rank[window], kind="stable")]
        m = bs // 2
        n = 2 * g.band_size - m
        want_d = np.zeros(g.band_deltas_size, np.int32)
        want_x = np.zeros(g.band_deltas_size, np.float32)
        want_d[:n] = strip[m:m + n].astype(np.int64) - strip[m + 1:m + n + 1].astype(np.int64)
        want_x[:n] = np.abs(dist[size // 2] - dist[strip[m + 1:m + n + 1]])
        d, x, filled = oracle.compile_band_data(g, angle)
        assert filled == n
        assert np.array_equal(d, want_d) and np.array_equal(x.view(np.uint32), want_x.view(np.uint32))


def test_compact_records_equal_the_reference_layout(oracle, synth):
    """The compact stream (counts + ids back to back) holds exactly the ids each
    band writes into its reserved slots (kernel.rs:141-145,220-243)."""
    z = synth.fbm(121, 121, 0.75, 21, 0.0, 900.0)
    g = oracle.geometry(121, 30.0, 1200, 60.0)
    for angle in (0.0, 37.0, 90.0):
        d, x, _ = oracle.compile_band_data(g, angle)
        c0 = np.zeros(g.computable_points_count, np.float32)
        r0 = np.zeros(oracle.ring_len(g), np.uint32)
        oracle.compute_sector(g, z, 1.65, d, x, c0, r0)
        c1, counts, ids = oracle.sweep_sector(g, z, 1.65, d, x, compact=True)
        R = g.reserved_rings_per_band
        rec = r0.reshape(-1, R)
        assert np.array_equal(rec[:, 0], counts) and counts.max() < R
        mask = np.arange(R - 1)[None, :] < counts[:, None]
        assert np.array_equal(rec[:, 1:][mask], ids)
        assert np.array_equal(c0.view(np.uint32), c1.view(np.uint32))


@pytest.mark.parametrize("mode", ["exact32", "fp64", "fp32"])
def test_row_ranges_are_slices_of_the_full_sweep(oracle, synth, mode):
    z = synth.fbm(101, 101, 0.8, 23, 0.0, 600.0)
    g = oracle.geometry(101, 10.0, 300)
    full, full_total = oracle.run_ex(g, z, 1.65, 0, 20, mode)
    for rows in [(0, 17), (17, 18), (18, g.tvs_height)]:
        part, part_total = oracle.run_ex(g, z, 1.65, 0, 20, mode, rows=rows)
        want = full.reshape(g.tvs_height, -1)[rows[0]:rows[1]].ravel()
        assert np.array_equal(part, want), rows
        if mode != "fp64":
            want_t = full_total.reshape(g.tvs_height, -1)[rows[0]:rows[1]].ravel()
            assert np.array_equal(part_total, want_t), rows


def test_fp32_form_is_the_reciprocal_table_expression(oracle, synth):
    """The FP32 comparison form evaluates fmaf(h - h_pov, RN(1/d), -RN(d/R)):
    checked here on one band against a direct numpy restatement."""
    z = synth.fbm(61, 61, 0.8, 29, 0.0, 400.0)
    g = oracle.geometry(61, 10.0, 200)
    d, x, n = oracle.compile_band_data(g, 23.0)
    c, counts, ids = oracle.sweep_sector(g, z, 1.65, d, x, mode="fp32", rows=(0, 1),
                                         compact=True)
    # band 0 (forward), computed with numpy in f32 with one rounding for the fma
    zf = z.astype(np.float32).ravel()
    los = g.max_los_as_points
    pov = los * 61 + los
    hp = np.float32(zf[pov] + np.float32(1.65))
    m, s, vis_prev, out = np.float32(-2000.0), np.float32(0.0), True, [pov]
    dem = pov
    for i in range(g.band_deltas_size):
        dem += int(d[i])
        e = np.float32(zf[dem] - hp)
        dist = np.float32(x[i])
        with np.errstate(divide="ignore", invalid="ignore"):
            y = np.float32(np.float32(1.0) / dist)
            cc = np.float32(dist / np.float32(12742000.0))
            a = np.float32(np.float64(e) * np.float64(y) - np.float64(cc))  # exact product
        vis = bool(a > m)
        if vis:
            s = np.float32(s + np.float32(dist * np.float32(0.0174533)))
        if vis != vis_prev:
            out.append(dem)
        vis_prev = vis
        m = a if np.isnan(m) else (m if np.isnan(a) else max(a, m))
    if vis_prev:
        out.append(dem)
    assert counts[0] == len(out) and list(ids[:counts[0]]) == out
