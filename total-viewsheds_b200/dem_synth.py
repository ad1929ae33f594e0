"""Seeded synthetic DEMs standing in for real terrain.

The reference ships no DEM (its .gitignore drops /dems) and the real SRTM /
viewfinderpanoramas tiles are not available offline, so every workload here
uses seeded synthetic heights with the shapes, sizes and value ranges of the
benchmark configurations:

  plain_cpu   301 x 301    fBm diamond-square, Hurst 0.8, 0-1500 m, 30 m, LOS 3 km
  plain_gpu   1201 x 1201  fBm, Hurst 0.75, 0-2500 m, 15 % contiguous 0 m, 90 m, LOS 36 km
  precision   3601 x 3601  ridged multifractal (10 octaves), 0-4500 m, 10 % flat 0 m,
                           30 m, LOS 36 km
  batching    48 tiles, sides U[257, 1601], fBm Hurst U[0.6, 0.9], 0-3000 m,
                           30 or 90 m, LOS = 1/3 of the shorter side
  large       7201 x 7201  2 x 2 stitched fBm tiles with continuous edges, 0-6000 m,
                           30 m, LOS 72 km

Seeds are 20261203 + the configuration's index.
"""

import numpy as np

BASE_SEED = 20261203


def _rescale(z, lo, hi):
    z = z.astype(np.float64)
    zmin, zmax = z.min(), z.max()
    if zmax == zmin:
        return np.full(z.shape, lo, np.float32)
    return (lo + (z - zmin) * ((hi - lo) / (zmax - zmin))).astype(np.float32)


def diamond_square(n_levels, hurst, rng, corners=None):
    """Fractional-Brownian surface on a (2^n + 1)^2 grid (Fournier-Fussell-Carpenter
    midpoint displacement): the displacement scale halves by 2^-hurst per level."""
    n = (1 << n_levels) + 1
    z = np.zeros((n, n), np.float32)
    if corners is None:
        corners = rng.standard_normal(4)
    z[0, 0], z[0, -1], z[-1, 0], z[-1, -1] = corners
    step = n - 1
    scale = 1.0
    while step > 1:
        h = step // 2
        # diamond step: centres of squares
        c = (z[0:-1:step, 0:-1:step] + z[0:-1:step, step::step] + z[step::step, 0:-1:step]
             + z[step::step, step::step]) * 0.25
        z[h::step, h::step] = c + scale * rng.standard_normal(c.shape).astype(np.float32)
        # square step: edge midpoints (average of the in-grid neighbours)
        for (r0, c0) in ((0, h), (h, 0)):
            rows = np.arange(r0, n, step)
            cols = np.arange(c0, n, step)
            rr, cc = np.meshgrid(rows, cols, indexing="ij")
            acc = np.zeros(rr.shape, np.float32)
            cnt = np.zeros(rr.shape, np.float32)
            for dr, dc in ((-h, 0), (h, 0), (0, -h), (0, h)):
                r2, c2 = rr + dr, cc + dc
                ok = (r2 >= 0) & (r2 < n) & (c2 >= 0) & (c2 < n)
                acc[ok] += z[r2[ok], c2[ok]]
                cnt[ok] += 1
            z[rr, cc] = acc / cnt + scale * rng.standard_normal(rr.shape).astype(np.float32)
        scale *= 0.5 ** hurst
        step = h
    return z


def fbm(width, height, hurst, seed, lo, hi):
    """Seeded fBm heights (metres, f32, row-major [height, width])."""
    rng = np.random.default_rng(seed)
    levels = max(1, int(np.ceil(np.log2(max(width, height) - 1))))
    z = diamond_square(levels, hurst, rng)
    return _rescale(z[:height, :width], lo, hi)


def _value_noise(width, height, period, rng):
    """Smooth lattice noise in [-1, 1] with lattice spacing `period` cells
    (random lattice values, smoothstep-interpolated)."""
    gy = int(np.ceil(height / period)) + 2
    gx = int(np.ceil(width / period)) + 2
    lattice = rng.uniform(-1.0, 1.0, (gy, gx)).astype(np.float32)
    oy, ox = rng.uniform(0, period, 2)
    y = (np.arange(height) + oy) / period
    x = (np.arange(width) + ox) / period
    y0 = np.floor(y).astype(np.int64)
    x0 = np.floor(x).astype(np.int64)
    ty = (y - y0).astype(np.float32)
    tx = (x - x0).astype(np.float32)
    ty = ty * ty * (3 - 2 * ty)
    tx = tx * tx * (3 - 2 * tx)
    a = lattice[y0][:, x0]
    b = lattice[y0][:, x0 + 1]
    c = lattice[y0 + 1][:, x0]
    d = lattice[y0 + 1][:, x0 + 1]
    top = a + (b - a) * tx[None, :]
    bot = c + (d - c) * tx[None, :]
    return top + (bot - top) * ty[:, None]


def ridged_multifractal(width, height, octaves, seed, lo, hi, lacunarity=2.0, gain=2.0,
                        offset=1.0, h=1.0):
    """Musgrave's ridged multifractal over value noise: each octave's ridge
    signal (offset - |n|)^2 is weighted by the previous octave's signal."""
    rng = np.random.default_rng(seed)
    period = max(width, height) / 4.0
    total = np.zeros((height, width), np.float32)
    weight = np.ones((height, width), np.float32)
    freq = 1.0
    for _ in range(octaves):
        n = _value_noise(width, height, max(period / freq, 1.5), rng)
        signal = (offset - np.abs(n)) ** 2 * weight
        weight = np.clip(signal * gain, 0.0, 1.0)
        total += signal * np.float32(freq ** -h)
        freq *= lacunarity
    return _rescale(total, lo, hi)


def flatten(z, fraction, seed):
    """Set one contiguous block covering `fraction` of the area to exactly 0 m
    (sea): a full-width band along a seed-chosen edge."""
    rng = np.random.default_rng(seed)
    h, w = z.shape
    z = z.copy()
    side = int(rng.integers(4))
    if side in (0, 1):
        k = int(round(fraction * h))
        if side == 0:
            z[:k, :] = 0.0
        else:
            z[h - k:, :] = 0.0
    else:
        k = int(round(fraction * w))
        if side == 2:
            z[:, :k] = 0.0
        else:
            z[:, w - k:] = 0.0
    return z


def stitched_fbm(width, height, hurst, seed, lo, hi):
    """2 x 2 tiles of fBm sharing their edge values (one midpoint-displacement
    parent grid split into quadrants, each refined with its own seed), so
    heights are continuous across the seams."""
    rng = np.random.default_rng(seed)
    levels = max(2, int(np.ceil(np.log2(max(width, height) - 1))))
    parent = diamond_square(levels - 1, hurst, rng)          # one shared coarse tile
    n = parent.shape[0]
    tile = np.zeros((2 * n - 1, 2 * n - 1), np.float32)
    # quadrants use the parent's corner values, so shared edges coincide
    for qi in range(2):
        for qj in range(2):
            trng = np.random.default_rng(seed * 7 + qi * 2 + qj + 1)
            c = [parent[0, 0], parent[0, -1], parent[-1, 0], parent[-1, -1]]
            q = diamond_square(levels - 1, hurst, trng, corners=c)
            tile[qi * (n - 1):qi * (n - 1) + n, qj * (n - 1):qj * (n - 1) + n] = q
    return _rescale(tile[:height, :width], lo, hi)


CONFIGS = {
    "plain_cpu": dict(index=0, width=301, scale=30.0, max_line_of_sight=3000,
                      observer_height=1.65, rings_per_km=5.0),
    "plain_gpu": dict(index=1, width=1201, scale=90.0, max_line_of_sight=36000,
                      observer_height=1.65, rings_per_km=5.0),
    "precision": dict(index=2, width=3601, scale=30.0, max_line_of_sight=36000,
                      observer_height=1.65, rings_per_km=5.0),
    "large": dict(index=4, width=7201, scale=30.0, max_line_of_sight=72000,
                  observer_height=1.65, rings_per_km=5.0),
    # not a benchmark configuration: a 2401^2 stand-in with the precision
    # form's terrain, sized for multi-pass profiler captures
    "medium": dict(index=5, width=2401, scale=30.0, max_line_of_sight=24000,
                   observer_height=1.65, rings_per_km=5.0),
}


def config_dem(name):
    """Heights (f32 [W, W]) of a named benchmark configuration."""
    cfg = CONFIGS[name]
    seed = BASE_SEED + cfg["index"]
    w = cfg["width"]
    if name == "plain_cpu":
        return fbm(w, w, 0.8, seed, 0.0, 1500.0)
    if name == "plain_gpu":
        return flatten(fbm(w, w, 0.75, seed, 0.0, 2500.0), 0.15, seed + 100)
    if name == "precision":
        return flatten(ridged_multifractal(w, w, 10, seed, 0.0, 4500.0), 0.10, seed + 100)
    if name == "large":
        return stitched_fbm(w, w, 0.8, seed, 0.0, 6000.0)
    if name == "medium":
        return flatten(ridged_multifractal(w, w, 10, seed, 0.0, 4500.0), 0.10, seed + 100)
    raise KeyError(name)


def batching_tiles(n_tiles=48, seed=BASE_SEED + 3):
    """The batching workload: (heights, scale, max_line_of_sight) per tile."""
    rng = np.random.default_rng(seed)
    tiles = []
    for t in range(n_tiles):
        w = int(rng.integers(257, 1602))
        h = int(rng.integers(257, 1602))
        hurst = float(rng.uniform(0.6, 0.9))
        scale = float(rng.choice([30.0, 90.0]))
        z = fbm(w, h, hurst, seed * 1000 + t, 0.0, 3000.0)
        los = int(min(w, h) / 3 * scale)
        tiles.append((z, scale, los))
    return tiles
