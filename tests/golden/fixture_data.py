"""Bit-reproducible inputs for the golden cases.

Golden pick lists are produced on one machine and checked on others, so their
inputs must be identical to the last bit everywhere.  Everything here uses only
integer hashing and IEEE +, -, * on float64 values that are exact or
deterministically rounded (no FFTs, transcendental functions or BLAS, whose last
bits can depend on the CPU):
  * noise: Irwin-Hall sum of 12 uniforms from a splitmix64 hash, minus 6;
  * templates: sums of polynomial bumps a (1 - r^2/R^2)^2 with dyadic centres, radii
    and amplitudes;
  * particles: templates planted at integer positions, rotated by multiples of 90 deg.
"""
from __future__ import annotations

import numpy as np

_M1, _M2, _M3 = np.uint64(0x9E3779B97F4A7C15), np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB)


def _hash(seed: int, n: int) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (np.arange(n, dtype=np.uint64) + np.uint64(seed) * np.uint64(1 << 32)) * _M1
        z = (z ^ (z >> np.uint64(30))) * _M2
        z = (z ^ (z >> np.uint64(27))) * _M3
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, n: int) -> np.ndarray:
    """Exact multiples of 2^-53 in [0, 1)."""
    return (_hash(seed, n) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def noise(seed: int, shape) -> np.ndarray:
    n = int(np.prod(shape))
    acc = np.zeros(n, dtype=np.float64)
    for k in range(12):
        acc += uniform(seed * 16 + k, n)
    return (acc - 6.0).reshape(shape)


def bump_image(size: int, centres, radii, amps) -> np.ndarray:
    yy, xx = np.mgrid[0:size, 0:size].astype(np.float64)
    img = np.zeros((size, size), dtype=np.float64)
    for (cx, cy), r, a in zip(centres, radii, amps):
        q = ((xx - cx) * (xx - cx) + (yy - cy) * (yy - cy)) / (r * r)
        img += a * np.where(q < 1.0, (1.0 - q) * (1.0 - q), 0.0)
    return img


def make_inputs(shape, n_templates: int, tsize: int, n_blobs: int, n_particles: int, amp: float, seed: int,
                margin: int):
    """Returns (image float32 [ny, nx], templates float32 [n, t, t], particles int [m, 4]: x, y, template, quarter)."""
    ny, nx = shape
    u = uniform(seed * 7919 + 1, n_templates * n_blobs * 4).reshape(n_templates, n_blobs, 4)
    templates = np.zeros((n_templates, tsize, tsize), dtype=np.float64)
    for j in range(n_templates):
        # dyadic centres within the central 60 % of the box, radii 2..8 px, amplitudes 0.5..1
        c = np.floor((0.2 + 0.6 * u[j, :, :2]) * tsize * 8) / 8
        r = 2.0 + np.floor(u[j, :, 2] * 48) / 8
        a = 0.5 + np.floor(u[j, :, 3] * 32) / 64
        templates[j] = bump_image(tsize, c, r, a)
    p = uniform(seed * 7919 + 2, n_particles * 4).reshape(n_particles, 4)
    image = noise(seed, shape)
    parts = np.zeros((n_particles, 4), dtype=np.int64)
    for k in range(n_particles):
        x = margin + int(p[k, 0] * (nx - 2 * margin - tsize))
        y = margin + int(p[k, 1] * (ny - 2 * margin - tsize))
        j = int(p[k, 2] * n_templates)
        q = int(p[k, 3] * 4)
        image[y:y + tsize, x:x + tsize] += amp * np.rot90(templates[j], q)
        parts[k] = (x + tsize // 2, y + tsize // 2, j, q)
    return image.astype(np.float32), templates.astype(np.float32), parts


def bump_volume(size: int, n_blobs: int, seed: int) -> np.ndarray:
    """float32 [size]^3 (z, y, x) sum of polynomial bumps a (1 - r^2/R^2)^2 with dyadic
    centres (central 60 % of the box), radii 2..6 px and amplitudes 0.5..1."""
    u = uniform(seed * 104729 + 3, n_blobs * 5).reshape(n_blobs, 5)
    c = np.floor((0.2 + 0.6 * u[:, :3]) * size * 8) / 8
    r = 2.0 + np.floor(u[:, 3] * 32) / 8
    a = 0.5 + np.floor(u[:, 4] * 64) / 128
    zz, yy, xx = np.mgrid[0:size, 0:size, 0:size].astype(np.float64)
    vol = np.zeros((size, size, size), dtype=np.float64)
    for (cx, cy, cz), rr, aa in zip(c, r, a):
        q = ((xx - cx) * (xx - cx) + (yy - cy) * (yy - cy) + (zz - cz) * (zz - cz)) / (rr * rr)
        vol += aa * np.where(q < 1.0, (1.0 - q) * (1.0 - q), 0.0)
    return vol.astype(np.float32)


# Projection cases: (volume size, blobs, seed, mask radius ri, angles (alt, az, phi) in radians,
# dyadic so that they print and parse exactly).
PROJECTION_CASES = {
    "vol40": (40, 24, 5, 0, [(0.0, 0.0, 0.0), (0.5, 0.25, 1.0), (1.25, 2.5, 0.75), (2.0, 4.0, 5.5),
                              (0.875, 3.125, 2.25), (3.0, 0.125, 6.0)]),
    "vol33_ri12": (33, 16, 6, 12, [(0.375, 1.5, 0.5), (1.75, 5.25, 3.0), (2.625, 0.75, 4.5)]),
}
