"""Ring records as a compact stream (tvs_compute_sector_rings): every band's
record is the reference's per-band record (kernel.rs:141-145,220-243) whatever
the reserved slots, so a context with few slots per band gives, untruncated,
the records the oracle writes into generously sized slots."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, SCALE, LOS, OBS = 301, 30.0, 3000, 1.65


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.fixture(scope="module")
def dem(synth):
    return synth.config_dem("plain_cpu")


def oracle_records(oracle, dem, angles, f64=False, rpk=60.0):
    """Per-sector compact records from the oracle's reference layout with enough
    slots that no band overflows."""
    g = oracle.geometry(W, SCALE, LOS, rpk)
    R = g.reserved_rings_per_band
    out = []
    for a in angles:
        d, x, _ = oracle.compile_band_data(g, float(a))
        if f64:
            cum = np.zeros(g.computable_points_count, np.float64)
        else:
            cum = np.zeros(g.computable_points_count, np.float32)
        rings = np.zeros(oracle.ring_len(g), np.uint32)
        oracle.compute_sector(g, dem, OBS, d, x, cum, rings, f64=f64)
        rec = rings.reshape(-1, R)
        n = rec[:, 0].astype(np.int64)
        assert (n + 1 <= R).all(), "the oracle needs more slots"
        offsets = np.concatenate([[0], np.cumsum(n)]).astype(np.uint64)
        ids = np.concatenate([rec[k, 1:1 + n[k]] for k in range(rec.shape[0])]) if n.sum() else \
            np.zeros(0, np.uint32)
        out.append((offsets, ids.astype(np.uint32)))
    return out


@pytest.mark.parametrize("rpk", [5.0, 20.0])
def test_compact_records_match_the_oracle(tvs, oracle, dem, rpk):
    """5 rings/km reserves 15 slots, fewer than some bands need: the compact
    records are still complete."""
    angles = [0, 1, 45, 90, 133]
    want = oracle_records(oracle, dem, angles)
    with tvs.Engine(dem, W, SCALE, LOS, rings_per_km=rpk, observer_height=OBS) as eng:
        cum = np.zeros(eng.count, np.float32)
        overflowed = 0
        for a, (wo, wi) in zip(angles, want):
            off, ids, st = eng.compute_sector_rings(a, cum)
            overflowed += st.overflow_bands
            assert np.array_equal(off, wo), a
            assert np.array_equal(ids, wi), a
    if rpk == 5.0:
        assert overflowed > 0  # the case the reserved layout cannot hold


def test_compact_records_equal_the_reserved_layout(tvs, dem):
    """With slots to spare the compact stream is the reserved layout without
    its empty slots, and the surfaces advance the same."""
    with tvs.Engine(dem, W, SCALE, LOS, rings_per_km=60.0, observer_height=OBS) as eng:
        R = eng.geometry.reserved_rings_per_band
        c1 = np.zeros(eng.count, np.float32)
        c2 = np.zeros(eng.count, np.float32)
        rings = np.zeros(eng.geometry.ring_slots_per_sector, np.uint32)
        for a in (7, 100):
            eng.compute_sector(a, c1, rings)
            off, ids, _ = eng.compute_sector_rings(a, c2)
            rec = rings.reshape(-1, R)
            n = rec[:, 0].astype(np.int64)
            assert np.array_equal(np.diff(off.astype(np.int64)), n)
            for k in range(0, rec.shape[0], 997):
                assert np.array_equal(ids[off[k]:off[k + 1]], rec[k, 1:1 + n[k]])
        assert np.array_equal(bits(c1), bits(c2))


def test_compact_records_mixed64_are_the_fp64_records(tvs, oracle, dem):
    angles = [3, 46]
    want = oracle_records(oracle, dem, angles, f64=True)
    with tvs.Engine(dem, W, SCALE, LOS, rings_per_km=5.0, observer_height=OBS,
                    precision="mixed64") as eng:
        cum = np.zeros(eng.count, np.float32)
        for a, (wo, wi) in zip(angles, want):
            off, ids, _ = eng.compute_sector_rings(a, cum)
            assert np.array_equal(off, wo) and np.array_equal(ids, wi), a


def test_compact_records_of_a_row_shard(tvs, oracle, dem):
    """Bands outside the shard's rows have empty records."""
    (wo, wi), = oracle_records(oracle, dem, [30])
    rows = (20, 61)
    with tvs.Engine(dem, W, SCALE, LOS, rings_per_km=5.0, observer_height=OBS, rows=rows) as eng:
        cum = np.zeros(eng.count, np.float32)
        off, ids, _ = eng.compute_sector_rings(30, cum)
        tw = eng.geometry.tvs_width
        half = eng.geometry.total_bands // 2
        for k in range(0, eng.geometry.total_bands, 131):
            row = (k % half) // tw
            got = ids[off[k]:off[k + 1]]
            if rows[0] <= row < rows[1]:
                assert np.array_equal(got, wi[wo[k]:wo[k + 1]]), k
            else:
                assert got.size == 0, k


def test_read_before_compute_is_an_error(tvs, dem):
    with tvs.Engine(dem, W, SCALE, LOS, observer_height=OBS) as eng:
        assert tvs.lib().tvs_read_ring_records(eng.ctx, None, None) == tvs.ERR_INVALID_ARGUMENT


def split_records(off, ids, bands, n_sectors):
    """Per-sector (offsets, ids) of a several-sector stream."""
    out = []
    for s in range(n_sectors):
        o = off[s * bands:(s + 1) * bands + 1].astype(np.int64)
        out.append(((o - o[0]).astype(np.uint64), ids[o[0]:o[-1]]))
    return out


@pytest.mark.parametrize("precision,rpk", [("exact32", 5.0), ("mixed64", 20.0), ("fp32", 5.0)])
def test_several_sectors_equal_one_at_a_time(tvs, dem, precision, rpk):
    """tvs_compute_sectors_rings gives every sector the records and surfaces of
    the one-sector calls, also where bands overflow the reserved slots."""
    first, n = 40, 7
    with tvs.Engine(dem, W, SCALE, LOS, rings_per_km=rpk, observer_height=OBS,
                    precision=precision) as eng:
        bands = eng.geometry.total_bands
        c1 = np.zeros(eng.count, np.float32)
        want = [eng.compute_sector_rings(a, c1)[:2] for a in range(first, first + n)]
        c2 = np.zeros(eng.count, np.float32)
        off, ids, st = eng.compute_sectors_rings(first, n, c2)
        assert off.size == n * bands + 1 and int(off[-1]) == ids.size
        for s, (got, w) in enumerate(zip(split_records(off, ids, bands, n), want)):
            assert np.array_equal(got[0], w[0]) and np.array_equal(got[1], w[1]), first + s
        if precision == "mixed64":
            # double across the call's sectors, as the device path keeps it
            eng.device_reset()
            eng.device_run_sectors(first, n)
            eng.device_finish()
            c1, _ = eng.read_surfaces()
        assert np.array_equal(bits(c1), bits(c2))
        # the last call's records are what tvs_read_ring_records returns
        off1, ids1, _ = eng.compute_sector_rings(first, np.zeros(eng.count, np.float32))
        assert off1.size == bands + 1 and np.array_equal(ids1, want[0][1])


def test_several_sectors_match_the_oracle(tvs, oracle, dem):
    angles = list(range(88, 93))
    want = oracle_records(oracle, dem, angles, f64=True)
    with tvs.Engine(dem, W, SCALE, LOS, rings_per_km=5.0, observer_height=OBS,
                    precision="mixed64") as eng:
        bands = eng.geometry.total_bands
        off, ids, _ = eng.compute_sectors_rings(angles[0], len(angles), np.zeros(eng.count, np.float32))
        for a, got, (wo, wi) in zip(angles, split_records(off, ids, bands, len(angles)), want):
            assert np.array_equal(got[0], wo) and np.array_equal(got[1], wi), a


def test_several_sectors_of_a_row_shard(tvs, dem):
    rows = (20, 61)
    with tvs.Engine(dem, W, SCALE, LOS, rings_per_km=5.0, observer_height=OBS, rows=rows) as eng:
        bands = eng.geometry.total_bands
        c1 = np.zeros(eng.count, np.float32)
        want = [eng.compute_sector_rings(a, c1)[:2] for a in (170, 171, 172)]
        c2 = np.zeros(eng.count, np.float32)
        off, ids, _ = eng.compute_sectors_rings(170, 3, c2)
        for got, w in zip(split_records(off, ids, bands, 3), want):
            assert np.array_equal(got[0], w[0]) and np.array_equal(got[1], w[1])
        assert np.array_equal(bits(c1), bits(c2))


def test_several_sectors_argument_errors(tvs, dem):
    import ctypes
    L = tvs.lib()
    cum = np.zeros(1, np.float32)
    total = ctypes.c_uint64()
    with tvs.Engine(dem, W, SCALE, LOS, observer_height=OBS) as eng:
        cum = np.zeros(eng.count, np.float32)
        for first, n in ((179, 2), (0, 0), (180, 1)):
            assert L.tvs_compute_sectors_rings(eng.ctx, first, n, tvs._ptr(cum), ctypes.byref(total),
                                               None) == tvs.ERR_INVALID_ARGUMENT, (first, n)
    with tvs.Engine(dem, W, SCALE, LOS, observer_height=OBS, precision="fp64") as eng:
        cum = np.zeros(eng.count, np.float32)
        assert L.tvs_compute_sectors_rings(eng.ctx, 0, 2, tvs._ptr(cum), ctypes.byref(total),
                                           None) == tvs.ERR_INVALID_ARGUMENT
        assert b"split sweep" in L.tvs_last_error(eng.ctx)
