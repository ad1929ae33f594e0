"""The C++ front end (total-viewsheds_b200/tvs) as the reference's CLI is used:
a .bt DEM in (input.rs:86-175), `--compute cuda`, heatmap.png out
(png.rs:5-37, compute.rs:165-178), checked against the oracle."""

import os
import struct
import subprocess
import tempfile
import zlib

import numpy as np
import pytest

from conftest import PKG_DIR

pytestmark = pytest.mark.gpu
CLI = PKG_DIR / "tvs"


def read_png_gray(path):
    data = path.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w = 8, b"", None
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if kind == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
            assert body[8:10] == b"\x08\x00"
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    rows = [raw[r * (w + 1) + 1:(r + 1) * (w + 1)] for r in range(h)]
    assert all(raw[r * (w + 1)] == 0 for r in range(h))
    return np.frombuffer(b"".join(rows), np.uint8).reshape(h, w)


def expected_png(total):
    """png.rs:5-37 in f32."""
    t = total.astype(np.float32)
    mn, mx = t.min(), t.max()
    rng = np.float32(1.0) if mx - mn == 0 else np.float32(mx - mn)
    v = np.clip((t - mn) / rng * np.float32(255.0), 0, 255).astype(np.float32)
    return v.astype(np.uint8)


# the CLI keeps the reference's shape cache in the OS state directory
# ($XDG_STATE_HOME); the tests point it at a directory of their own
STATE = tempfile.mkdtemp(prefix="tvs-state-")


def run_cli(*args, state=STATE):
    env = dict(os.environ, XDG_STATE_HOME=str(state))
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True, env=env)


@pytest.fixture(scope="module")
def dem(synth):
    return synth.config_dem("plain_cpu")


@pytest.mark.parametrize("heatmap", ["final", "every-sector"])
def test_cli_f32_bt(bt, oracle, dem, tmp_path, heatmap):
    p = tmp_path / "dem.bt"
    bt.write_bt(p, dem)
    out = tmp_path / "out"
    out.mkdir()
    r = run_cli("--input", p, "--scale", 30, "--max-line-of-sight", 3000, "--observer-height",
                1.65, "--compute", "cuda", "--output-dir", out, "--heatmap", heatmap,
                "--surfaces-out", tmp_path / "s.bin")
    assert r.returncode == 0, r.stderr
    g = oracle.geometry(301, 30.0, 3000)
    cum, total, _ = oracle.run(g, dem, 1.65)
    got = np.fromfile(tmp_path / "s.bin", np.float32)
    assert np.array_equal(got.view(np.uint32), cum.view(np.uint32))
    png = read_png_gray(out / "heatmap.png")
    assert png.shape == (g.tvs_height, g.tvs_width)
    assert np.array_equal(png, expected_png(total).reshape(png.shape))


def test_cli_i16_bt_and_default_line_of_sight(bt, oracle, dem, tmp_path):
    """i16 heights are widened to f32 (main.rs:51-56); without --max-line-of-sight
    the line of sight is width/3 * scale (main.rs:36-38), here 3000 m."""
    z16 = np.round(dem).astype(np.int16)
    p = tmp_path / "dem16.bt"
    bt.write_bt(p, z16, as_float=False)
    r = run_cli("--input", p, "--scale", 30, "--reference-observer-height", "--output-dir",
                tmp_path, "--heatmap", "final", "--surfaces-out", tmp_path / "s.bin")
    assert r.returncode == 0, r.stderr
    g = oracle.geometry(301, 30.0, 3000)
    cum, _, _ = oracle.run(g, z16.astype(np.float32), 1.8)
    got = np.fromfile(tmp_path / "s.bin", np.float32)
    assert np.array_equal(got.view(np.uint32), cum.view(np.uint32))


def test_cli_rejects_other_backends_and_bad_input(bt, tmp_path):
    r = run_cli("--input", tmp_path / "missing.bt", "--compute", "vulkan")
    assert r.returncode == 1 and "cuda" in r.stderr
    bad = tmp_path / "bad.bt"
    bad.write_bytes(b"binterr1.2" + b"\0" * 300)
    r = run_cli("--input", bad, "--scale", 30)
    assert r.returncode == 1 and "Not a Binary Terrain" in r.stderr
    p = tmp_path / "small.bt"
    bt.write_bt(p, np.zeros((101, 101), np.float32))
    r = run_cli("--input", p, "--scale", 1, "--max-line-of-sight", 51)
    assert r.returncode == 1 and "longer than the maximum distance" in r.stderr


def test_cli_shape_cache(bt, oracle, dem, tmp_path):
    """compute.rs:118-162: the first run computes and saves every sector's shape
    under <state>/total-viewsheds/<width>/, the second loads all 180 and gives
    the same surfaces; another line of sight on the same width (the reference's
    cache key is the width alone) is refused instead of misread; --no-cache
    touches nothing."""
    p = tmp_path / "dem.bt"
    bt.write_bt(p, dem)
    state = tmp_path / "state"
    args = ("--input", p, "--scale", 30, "--observer-height", 1.65, "--heatmap", "final",
            "--output-dir", tmp_path)
    r1 = run_cli(*args, "--max-line-of-sight", 3000, "--surfaces-out", tmp_path / "a.bin",
                 state=state)
    assert r1.returncode == 0, r1.stderr
    assert "0 of 180 sectors loaded" in r1.stderr
    base = state / "total-viewsheds" / "301"
    assert len(list((base / "band_deltas").glob("*.bin"))) == 180
    assert len(list((base / "distances").glob("*.bin"))) == 180
    g = oracle.geometry(301, 30.0, 3000)
    d, x, _ = oracle.compile_band_data(g, 90.0)
    assert np.array_equal(np.fromfile(base / "band_deltas" / "90.bin", np.int32), d)
    assert np.array_equal(np.fromfile(base / "distances" / "90.bin", np.float32).view(np.uint32),
                          x.view(np.uint32))
    r2 = run_cli(*args, "--max-line-of-sight", 3000, "--surfaces-out", tmp_path / "b.bin",
                 state=state)
    assert r2.returncode == 0, r2.stderr
    assert "180 of 180 sectors loaded" in r2.stderr
    assert (tmp_path / "a.bin").read_bytes() == (tmp_path / "b.bin").read_bytes()
    r3 = run_cli(*args, "--max-line-of-sight", 2400, state=state)
    assert r3.returncode == 1 and "line of sight" in r3.stderr
    fresh = tmp_path / "fresh"
    r4 = run_cli(*args, "--max-line-of-sight", 3000, "--no-cache", state=fresh)
    assert r4.returncode == 0, r4.stderr
    assert not fresh.exists()
