"""Synthetic DEM generators and the .bt reader (input.rs:86-185)."""

import numpy as np
import pytest


def test_fbm_is_seeded_and_scaled(synth):
    a = synth.fbm(301, 301, 0.8, 1, 0.0, 1500.0)
    b = synth.fbm(301, 301, 0.8, 1, 0.0, 1500.0)
    c = synth.fbm(301, 301, 0.8, 2, 0.0, 1500.0)
    assert a.dtype == np.float32 and a.shape == (301, 301)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert a.min() == 0.0 and a.max() == 1500.0


def test_flat_region_fraction(synth):
    z = synth.config_dem("plain_gpu")
    assert z.shape == (1201, 1201)
    assert abs((z == 0.0).mean() - 0.15) < 0.005


def test_ridged_multifractal(synth):
    z = synth.ridged_multifractal(257, 193, 10, 5, 0.0, 4500.0)
    assert z.shape == (193, 257) and z.min() == 0.0 and z.max() == 4500.0
    assert np.isfinite(z).all()


def test_stitched_tiles_are_continuous(synth):
    z = synth.stitched_fbm(129, 129, 0.8, 9, 0.0, 6000.0)
    assert z.shape == (129, 129)
    # the seams (row/column 64) are shared edges, not discontinuities
    jump = np.abs(np.diff(z, axis=0)).max()
    seam = np.abs(z[64] - z[63]).max()
    assert seam <= jump


def test_batching_tiles(synth):
    tiles = synth.batching_tiles(4)
    for z, scale, los in tiles:
        h, w = z.shape
        assert 257 <= w <= 1601 and 257 <= h <= 1601
        assert scale in (30.0, 90.0) and los == int(min(w, h) / 3 * scale)


@pytest.mark.parametrize("as_float", [True, False])
def test_bt_round_trip(bt, tmp_path, as_float):
    z = (np.arange(35 * 21).reshape(21, 35) % 700).astype(np.float32)
    p = tmp_path / "t.bt"
    bt.write_bt(p, z, as_float=as_float)
    header, back = bt.read_bt(p)
    assert header["width"] == 35 and header["height"] == 21
    assert header["is_float"] == as_float
    assert np.array_equal(back, z)


def test_bt_rejects_bad_magic(bt, tmp_path):
    p = tmp_path / "bad.bt"
    p.write_bytes(b"binterr1.2" + b"\0" * 300)
    with pytest.raises(bt.BtError, match="Not a Binary Terrain"):
        bt.read_bt(p)


def test_bt_rejects_truncated_data(bt, tmp_path):
    p = tmp_path / "short.bt"
    bt.write_bt(p, np.zeros((10, 10), np.float32))
    p.write_bytes(p.read_bytes()[:-4])
    with pytest.raises(bt.BtError, match="truncated"):
        bt.read_bt(p)


def test_bt_scale_haversine(bt):
    # 1 degree of "latitude" spacing across 1201 columns at the reference's
    # argument order is ~92.6 m per cell.
    h = dict(width=1201, left=0.0, right=1.0, top=0.0, bottom=-1.0)
    assert abs(bt.scale(h) - 111195.08 / 1201) < 0.01
