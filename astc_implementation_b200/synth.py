"""Seeded synthetic RGBA8 textures for tests and benchmarks.

The generator stands in for the reference's (git-ignored, absent) test images.
For a texture of width W and height H from seed s (numpy PCG64 via
``np.random.default_rng(s)``):

* RGB and alpha start as per-channel 4-octave value noise: octave o in 0..3 is a
  grid of (2**(o+2) + 1)**2 uniform values, bilinearly upsampled to H x W and
  weighted 0.5**o; the weighted sum is normalised to [0, 1] and scaled to [0, 255].
* 32 hard-edged rectangles (uniform corners) are filled with uniform random RGB.
* 16 diagonal half-plane splits: each picks a random box and a line through the
  box centre at 45 or 135 degrees (plus up to 15 degrees of jitter); texels of
  the box on the positive side of the line get a uniform random RGB.
* Alpha is 255 where x < W // 2 and the alpha noise channel elsewhere.
"""
import numpy as np


def _value_noise(rng, h, w):
    out = np.zeros((h, w), np.float64)
    total = 0.0
    ys = np.linspace(0.0, 1.0, h)
    xs = np.linspace(0.0, 1.0, w)
    for o in range(4):
        g = 2 ** (o + 2) + 1
        grid = rng.random((g, g))
        gy = ys * (g - 1)
        gx = xs * (g - 1)
        y0 = np.minimum(np.floor(gy).astype(int), g - 2)
        x0 = np.minimum(np.floor(gx).astype(int), g - 2)
        fy = (gy - y0)[:, None]
        fx = (gx - x0)[None, :]
        a = grid[y0][:, x0]
        b = grid[y0][:, x0 + 1]
        c = grid[y0 + 1][:, x0]
        d = grid[y0 + 1][:, x0 + 1]
        layer = (a * (1 - fx) + b * fx) * (1 - fy) + (c * (1 - fx) + d * fx) * fy
        wgt = 0.5 ** o
        out += wgt * layer
        total += wgt
    return out / total


def make_texture(width, height, seed):
    """Returns an (height, width, 4) uint8 array."""
    rng = np.random.default_rng(seed)
    img = np.zeros((height, width, 4), np.float64)
    for c in range(4):
        img[:, :, c] = _value_noise(rng, height, width) * 255.0
    for _ in range(32):
        x0, x1 = np.sort(rng.integers(0, width + 1, 2))
        y0, y1 = np.sort(rng.integers(0, height + 1, 2))
        img[y0:y1, x0:x1, :3] = rng.integers(0, 256, 3)
    yy, xx = np.mgrid[0:height, 0:width]
    for _ in range(16):
        x0, x1 = np.sort(rng.integers(0, width + 1, 2))
        y0, y1 = np.sort(rng.integers(0, height + 1, 2))
        ang = np.deg2rad(rng.choice([45.0, 135.0]) + rng.uniform(-15.0, 15.0))
        cx, cy = (x0 + x1) / 2.0, (y0 + y1) / 2.0
        side = (xx - cx) * np.sin(ang) - (yy - cy) * np.cos(ang) > 0
        box = (xx >= x0) & (xx < x1) & (yy >= y0) & (yy < y1)
        img[side & box, :3] = rng.integers(0, 256, 3)
    img[:, : width // 2, 3] = 255.0
    return np.clip(np.rint(img), 0, 255).astype(np.uint8)


def texel_blocks(img, bx, by):
    """Splits an RGBA8 image into blocks the way the reference does
    (code/compression_pipeline.cpp:7-86): raster block order, texels in raster
    order inside a block, edge texels clamped, values (v / 255) * 65536 in f32.
    Returns (nblocks, bx*by, 4) float32."""
    h, w, _ = img.shape
    nbx, nby = (w + bx - 1) // bx, (h + by - 1) // by
    ys = np.minimum(np.arange(nby * by), h - 1).reshape(nby, by)
    xs = np.minimum(np.arange(nbx * bx), w - 1).reshape(nbx, bx)
    blk = img[ys[:, None, :, None], xs[None, :, None, :]]  # nby, nbx, by, bx, 4
    f = (blk.astype(np.float32) / np.float32(255.0)) * np.float32(65536.0)
    return f.reshape(nby * nbx, by * bx, 4).astype(np.float32)
