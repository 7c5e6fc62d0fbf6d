"""Seeded synthetic micrographs and template stacks.

The reference ships no data (its test script expects PSII_data, which is not
public), so every workload here is generated: a 3D volume of Gaussian blobs is
projected analytically (a 3D Gaussian projects to a 2D Gaussian), particles are
planted at seeded positions and in-plane angles, modulated by the micrograph's
CTF, scaled to the requested SNR and added to N(0, 1) noise.  Rendering uses
separable Gaussians (one small matrix product per image), so the 8192^2 /
1000-template case builds in seconds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

try:
    import scipy.fft as sfft
except Exception:  # pragma: no cover
    sfft = None


@dataclass
class Case:
    image: np.ndarray          # (ny, nx) float32
    templates: np.ndarray      # (n, t, t) float32
    euler: np.ndarray          # (n, 3) float32: alt, az, phi
    particles: np.ndarray      # (m, 4): x, y, template, psi
    defocus: float = 1.5
    dfdiff: float = 0.0
    dfang: float = 0.0
    meta: dict = field(default_factory=dict)


def blob_volume(rng: np.random.Generator, size: int, n_blobs: int, sigma=(2.0, 6.0)):
    """Blob centres (relative to the volume centre), widths and amplitudes."""
    r = 0.28 * size
    pts = []
    while len(pts) < n_blobs:
        p = rng.uniform(-r, r, size=3)
        if p @ p <= r * r:
            pts.append(p)
    centres = np.array(pts)
    sig = rng.uniform(sigma[0], sigma[1], size=n_blobs)
    amp = rng.uniform(0.5, 1.0, size=n_blobs)
    return centres, sig, amp


def rotation(alt: float, az: float, phi: float = 0.0) -> np.ndarray:
    """EMAN-style rotation (az about z, alt about x, phi about z), degrees."""
    a, b, c = np.radians([az, alt, phi])
    rz1 = np.array([[math.cos(a), -math.sin(a), 0], [math.sin(a), math.cos(a), 0], [0, 0, 1]])
    rx = np.array([[1, 0, 0], [0, math.cos(b), -math.sin(b)], [0, math.sin(b), math.cos(b)]])
    rz2 = np.array([[math.cos(c), -math.sin(c), 0], [math.sin(c), math.cos(c), 0], [0, 0, 1]])
    return rz2 @ rx @ rz1


def render(px: np.ndarray, py: np.ndarray, sig: np.ndarray, amp: np.ndarray, w: int, h: int, ox: float = 0.0,
           oy: float = 0.0) -> np.ndarray:
    """Sum of 2D Gaussians amp*exp(-r^2/2sig^2) at (px+ox, py+oy) on an h x w grid (separable product)."""
    xs = np.arange(w, dtype=np.float64)
    ys = np.arange(h, dtype=np.float64)
    gx = np.exp(-((xs[None, :] - (px + ox)[:, None]) ** 2) / (2 * sig[:, None] ** 2))
    gy = np.exp(-((ys[None, :] - (py + oy)[:, None]) ** 2) / (2 * sig[:, None] ** 2))
    return (gy * amp[:, None]).T @ gx


def project(centres, sig, amp, alt, az, tsize):
    """Analytic projection of the blob volume along the rotated z axis into a tsize^2 template."""
    R = rotation(alt, az)
    c2 = centres @ R.T
    a2 = amp * sig * math.sqrt(2 * math.pi)
    return c2[:, 0] + tsize / 2, c2[:, 1] + tsize / 2, a2


def ctf_2d(ny: int, nx: int, apix: float, defocus: float, dfdiff: float, dfang: float, kv: float = 300.0,
           cs: float = 2.7, ampc: float = 0.07) -> np.ndarray:
    """Signed astigmatic CTF on the rfft grid (defocus in um, cs in mm), physical convention."""
    lam = 12.2639 / math.sqrt(kv * 1000.0 + 0.97845 * kv * kv)
    fy = np.fft.fftfreq(ny)[:, None] / apix
    fx = np.fft.rfftfreq(nx)[None, :] / apix
    s2 = fx * fx + fy * fy
    ang = np.arctan2(fy, fx)
    df = (defocus + dfdiff * np.cos(2 * (np.radians(dfang) - ang))) * 1e4
    gamma = math.pi * lam * df * s2 - 0.5 * math.pi * cs * 1e7 * lam ** 3 * s2 * s2
    return math.sqrt(1 - ampc * ampc) * np.sin(gamma) + ampc * np.cos(gamma)


def make_case(shape=(1024, 1024), n_particles=50, snr=0.1, n_templates=8, tsize=128, n_blobs=200, seed=0,
              defocus=1.5, dfdiff=0.0, dfang=0.0, apix=1.0, margin=None) -> Case:
    rng = np.random.default_rng(seed)
    ny, nx = shape
    centres, sig, amp = blob_volume(rng, tsize, n_blobs)
    alts = np.degrees(np.arccos(rng.uniform(-1, 1, size=n_templates)))
    azs = rng.uniform(0, 360, size=n_templates)
    templates = np.zeros((n_templates, tsize, tsize), np.float32)
    proj = []
    for j in range(n_templates):
        px, py, a2 = project(centres, sig, amp, alts[j], azs[j], tsize)
        proj.append((px, py, a2))
        templates[j] = render(px, py, sig, a2, tsize, tsize)
    margin = tsize // 2 if margin is None else margin
    clean = np.zeros((ny, nx), np.float64)
    parts = np.zeros((n_particles, 4))
    for k in range(n_particles):
        j = int(rng.integers(n_templates))
        psi = float(rng.uniform(0, 360))
        x = float(rng.uniform(margin, nx - margin))
        y = float(rng.uniform(margin, ny - margin))
        px, py, a2 = proj[j]
        c, s = math.cos(math.radians(psi)), math.sin(math.radians(psi))
        dx, dy = px - tsize / 2, py - tsize / 2
        rx, ry = c * dx - s * dy, s * dx + c * dy
        x0, y0 = int(x) - tsize, int(y) - tsize
        x0c, y0c = max(x0, 0), max(y0, 0)
        x1c, y1c = min(x0 + 2 * tsize, nx), min(y0 + 2 * tsize, ny)
        patch = render(rx, ry, sig, a2, x1c - x0c, y1c - y0c, ox=x - x0c, oy=y - y0c)
        clean[y0c:y1c, x0c:x1c] += patch
        parts[k] = (x, y, j, psi)
    if n_particles:
        if sfft is not None:
            F = sfft.rfft2(clean.astype(np.float32), workers=-1)
            F *= ctf_2d(ny, nx, apix, defocus, dfdiff, dfang).astype(np.float32)
            clean = sfft.irfft2(F, s=(ny, nx), workers=-1)
        else:  # pragma: no cover
            F = np.fft.rfft2(clean) * ctf_2d(ny, nx, apix, defocus, dfdiff, dfang)
            clean = np.fft.irfft2(F, s=(ny, nx))
        # scale so the signal variance over the particle footprints equals snr (noise variance 1)
        foot = np.abs(clean) > 1e-3 * np.abs(clean).max()
        pv = float(np.mean(clean[foot] ** 2)) if foot.any() else 1.0
        clean *= math.sqrt(snr / pv)
    noise = rng.standard_normal((ny, nx), dtype=np.float32)
    image = (noise + clean.astype(np.float32)).astype(np.float32)
    euler = np.stack([alts, azs, np.zeros(n_templates)], axis=1).astype(np.float32)
    return Case(image=image, templates=templates, euler=euler, particles=parts, defocus=defocus, dfdiff=dfdiff,
                dfang=dfang, meta=dict(seed=seed, snr=snr, shape=shape))


# Workloads named by what they are (sizes from the project's benchmark table).
WORKLOADS = {
    # 1024^2, 8 templates of 128^2, 10 deg, norm_type=0 in 720^2 tiles, 512 windows overlap 128
    "tiled_1024_t8": dict(shape=(1024, 1024), n_particles=50, snr=0.1, n_templates=8, tsize=128, seed=1,
                          defocus=1.5, dfdiff=0.0, dfang=0.0),
    # 4096^2, 200 templates of 180^2, 5 deg, norm_type=1, 512 windows overlap 192
    "whole_4096_t200": dict(shape=(4096, 4096), n_particles=300, snr=0.05, n_templates=200, tsize=180, seed=2,
                            defocus=1.7, dfdiff=0.1, dfang=30.0),
    # 8192^2, 1000 templates of 256^2, 5 deg, norm_type=1, 1024 windows overlap 256
    "whole_8192_t1000": dict(shape=(8192, 8192), n_particles=1000, snr=0.05, n_templates=1000, tsize=256, seed=5,
                             defocus=1.7, dfdiff=0.1, dfang=30.0),
    # the 4096^2 workload at the reference's default window size 320 (overlap 120): window sizes
    # without hand-tuned kernels
    "whole_4096_t200_w320": dict(shape=(4096, 4096), n_particles=300, snr=0.05, n_templates=200, tsize=180, seed=2,
                                 defocus=1.7, dfdiff=0.1, dfang=30.0),
    # profiling case: the 4096^2 workload's kernel shapes (512 windows, 180^2 templates) at 2048^2,
    # 24 templates, 4 angles
    "whole_2048_t24": dict(shape=(2048, 2048), n_particles=40, snr=0.05, n_templates=24, tsize=180, seed=3,
                           defocus=1.7, dfdiff=0.1, dfang=30.0),
    # the reference's default window 320 on the 4096^2 micrograph with 400 templates: the
    # reference reads past its template stack when windows (400 here) outnumber the templates
    # (norm.cu:141-147), so its CUDA build is timed on this variant
    "whole_4096_t400_w320": dict(shape=(4096, 4096), n_particles=300, snr=0.05, n_templates=400, tsize=180, seed=2,
                                 defocus=1.7, dfdiff=0.1, dfang=30.0),
    # profiling case at the reference's default window size 320 (overlap 120)
    "whole_2048_t24_w320": dict(shape=(2048, 2048), n_particles=40, snr=0.05, n_templates=24, tsize=180, seed=3,
                                defocus=1.7, dfdiff=0.1, dfang=30.0),
}

SEARCH_PARAMS = {
    "tiled_1024_t8": dict(angpix=1.0, phistep=10.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                          diameter=100.0, threshold=7.0, window_size=512, overlap=128, norm_type=0),
    "whole_4096_t200": dict(angpix=1.0, phistep=5.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                            diameter=140.0, threshold=7.0, window_size=512, overlap=192, norm_type=1),
    "whole_4096_t200_w320": dict(angpix=1.0, phistep=5.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                                 diameter=140.0, threshold=7.0, window_size=320, overlap=120, norm_type=1),
    "whole_8192_t1000": dict(angpix=1.0, phistep=5.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                             diameter=200.0, threshold=7.0, window_size=1024, overlap=256, norm_type=1),
    # batching: uneven micrographs (batch_cases), 500 templates of 200^2, 3 degree step
    "batch_c3": dict(angpix=1.0, phistep=3.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                     diameter=150.0, threshold=7.0, window_size=512, overlap=200, norm_type=1),
    "whole_2048_t24": dict(angpix=1.0, phistep=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                           diameter=140.0, threshold=7.0, window_size=512, overlap=192, norm_type=1),
    "whole_4096_t400_w320": dict(angpix=1.0, phistep=5.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                                 diameter=140.0, threshold=7.0, window_size=320, overlap=120, norm_type=1),
    "whole_2048_t24_w320": dict(angpix=1.0, phistep=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                                diameter=140.0, threshold=7.0, window_size=320, overlap=120, norm_type=1),
}


def batch_cases(n=32, seed=3, n_templates=500, tsize=200):
    """Uneven micrograph batch: sizes cycle through 2048^2, 3710x3838, 4096^2, 4092x5760."""
    rng = np.random.default_rng(seed)
    shapes = [(2048, 2048), (3838, 3710), (4096, 4096), (5760, 4092)]
    out = []
    for i in range(n):
        shp = shapes[i % len(shapes)]
        df = float(rng.uniform(0.8, 3.0))
        out.append(dict(shape=shp, n_particles=int(rng.integers(100, 401)), snr=0.05, n_templates=n_templates,
                        tsize=tsize, seed=seed * 1000 + i, defocus=df, dfdiff=float(rng.uniform(0, 0.2)),
                        dfang=float(rng.uniform(0, 180))))
    return out
