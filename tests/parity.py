"""Shared helpers of the parity tests: small seeded cases and pick-list comparison."""
from __future__ import annotations

import numpy as np

import gisspa
import synth

SCORE_RTOL = 1e-4   # plain FP32 form vs the FP64 oracle (relative)
SCORE_ATOL = 2e-5   # absolute slack for scores near zero


def config_from(cfg_dict: dict, **over) -> gisspa.Config:
    d = dict(cfg_dict)
    if "Highres" in d:
        d["highres"] = d.pop("Highres")
    if "Lowres" in d:
        d["lowres"] = d.pop("Lowres")
    d.update(over)
    return gisspa.Config.default(**d)


# Small cases (oracle runs in seconds); the reference's preconditions hold except where noted.
SMALL = {
    # whole-image norm_type=1, 3x3 windows, more windows than templates (padded templates count in N)
    "norm_l256_w9": (dict(shape=(512, 512), n_particles=5, snr=0.6, n_templates=4, tsize=64, seed=21, defocus=1.5,
                          dfdiff=0.08, dfang=35.0, margin=40),
                     dict(angpix=1.0, phistep=45.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                          diameter=48.0, threshold=3.0, window_size=256, overlap=64, norm_type=1)),
    # l = 512 windows on a 1024^2 micrograph
    "norm_l512_w4": (dict(shape=(1024, 1024), n_particles=8, snr=0.5, n_templates=4, tsize=128, seed=22,
                          defocus=1.8, dfdiff=0.1, dfang=30.0),
                     dict(angpix=1.0, phistep=30.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                          diameter=100.0, threshold=3.0, window_size=512, overlap=0, norm_type=1)),
    # l = 1024 windows (the 8192^2 workload's window size) on a 1536^2 micrograph, 2x2 windows
    "norm_l1024_w4": (dict(shape=(1536, 1536), n_particles=6, snr=0.5, n_templates=3, tsize=160, seed=24,
                           defocus=1.7, dfdiff=0.1, dfang=30.0),
                      dict(angpix=1.0, phistep=90.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                           diameter=120.0, threshold=3.0, window_size=1024, overlap=512, norm_type=1)),
    # the reference's default window size 320 (no hand-tuned kernels: the generic path), 2x2 windows
    "norm_l320_w4": (dict(shape=(640, 640), n_particles=5, snr=0.6, n_templates=3, tsize=96, seed=25,
                          defocus=1.6, dfdiff=0.05, dfang=20.0),
                     dict(angpix=1.0, phistep=45.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                          diameter=70.0, threshold=3.0, window_size=320, overlap=0, norm_type=1)),
    # 336 = 2^4 3 7 (mixed-radix stages with radix 3 and 7, 16-row blocks for the chunk scans)
    "norm_l336_w4": (dict(shape=(672, 672), n_particles=5, snr=0.6, n_templates=3, tsize=96, seed=27,
                          defocus=1.6, dfdiff=0.05, dfang=20.0),
                     dict(angpix=1.0, phistep=45.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                          diameter=70.0, threshold=3.0, window_size=336, overlap=0, norm_type=1)),
    # 176 = 16 11: a prime factor above 7 (Bluestein transforms, the unfused generic form)
    "norm_l176_w4": (dict(shape=(352, 352), n_particles=4, snr=0.6, n_templates=3, tsize=64, seed=28,
                          defocus=1.6, dfdiff=0.05, dfang=20.0),
                     dict(angpix=1.0, phistep=45.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                          diameter=50.0, threshold=3.0, window_size=176, overlap=0, norm_type=1)),
    "nonorm_l176": (dict(shape=(800, 800), n_particles=6, snr=0.5, n_templates=3, tsize=64, seed=29,
                         defocus=1.5, dfdiff=0.0, dfang=0.0),
                    dict(angpix=1.0, phistep=60.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                         diameter=50.0, threshold=8.0, window_size=176, overlap=60, norm_type=0)),
    "nonorm_l320": (dict(shape=(800, 800), n_particles=6, snr=0.5, n_templates=3, tsize=96, seed=26,
                         defocus=1.5, dfdiff=0.0, dfang=0.0),
                    dict(angpix=1.0, phistep=60.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                         diameter=70.0, threshold=8.0, window_size=320, overlap=100, norm_type=0)),
    # norm_type=0 on 720^2 tiles of a 1024^2 micrograph with 512 windows (the tiled workload's geometry)
    "nonorm_l512": (dict(shape=(1024, 1024), n_particles=10, snr=0.5, n_templates=4, tsize=128, seed=23,
                         defocus=1.5, dfdiff=0.0, dfang=0.0),
                    dict(angpix=1.0, phistep=45.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                         diameter=100.0, threshold=8.0, window_size=512, overlap=128, norm_type=0)),
}


def planted_copies_case():
    """Known-answer input: three distinct band-limited random textures (64^2, inside a disk),
    each planted once as an exact copy rotated by a multiple of 90 degrees (exact on the pixel
    grid) at an integer offset, CTF-modulated, in unit noise.  Returns (image, templates, ctf,
    config, truth) with truth rows (template, centre x, centre y, rotation in degrees); a
    64-pixel template's centre lies between pixels (offset + 31.5)."""
    rng = np.random.default_rng(7)
    t, nt = 64, 3
    yy, xx = np.mgrid[0:t, 0:t] - (t - 1) / 2
    disk = (np.hypot(xx, yy) < 26).astype(np.float64)
    ky = np.fft.fftfreq(t)[:, None]
    kx = np.fft.fftfreq(t)[None, :]
    lowpass = np.exp(-(kx ** 2 + ky ** 2) * (2 * np.pi * 1.5) ** 2 / 2)  # Gaussian blur, sigma 1.5 px
    tmpl = np.stack([np.fft.ifft2(np.fft.fft2(rng.standard_normal((t, t))) * lowpass).real * disk
                     for _ in range(nt)])
    tmpl = (tmpl / tmpl.std(axis=(1, 2), keepdims=True)).astype(np.float32)
    ny, nx = 512, 640
    placed = [(1, 150, 170, 1), (0, 400, 130, 2), (2, 300, 380, 3)]  # template, x0, y0, quarter turns
    clean = np.zeros((ny, nx))
    for j, x0, y0, k in placed:
        clean[y0:y0 + t, x0:x0 + t] += np.rot90(tmpl[j], k)
    F = np.fft.rfft2(clean) * synth.ctf_2d(ny, nx, 1.0, 1.5, 0.0, 0.0)
    img = (np.fft.irfft2(F, s=(ny, nx)) * 3.0 + rng.standard_normal((ny, nx))).astype(np.float32)
    cfg = gisspa.Config.default(angpix=1.0, phistep=10.0, kk=3.0, energy=300.0, cs=2.7, highres=4.0, lowres=200.0,
                                diameter=64.0, threshold=1.0, window_size=256, overlap=64, norm_type=1,
                                pick_mode=gisspa.PICK_TOPK, topk=3, exclusion_radius=40.0)
    truth = np.array([(j, x0 + (t - 1) / 2, y0 + (t - 1) / 2, 90.0 * k) for j, x0, y0, k in placed])
    return img, tmpl, gisspa.Ctf(1.5, 0.0, 0.0), cfg, truth


def assert_planted_copies_found(picks: np.ndarray, truth: np.ndarray):
    """Each planted copy is one of the top picks: its template, its rotation (the reported
    angle of a norm_type=1 pick is 360 - the search angle, norm.cu:654) and its centre within a
    pixel."""
    assert len(picks) == len(truth)
    for j, cx, cy, ang in truth:
        hit = [p for p in picks if p["template_id"] == int(j)]
        assert len(hit) == 1, (j, picks)
        p = hit[0]
        assert abs(p["x"] - cx) <= 1.0 and abs(p["y"] - cy) <= 1.0, (j, p, cx, cy)
        assert abs(((p["angle"] - ang) + 180.0) % 360.0 - 180.0) < 1e-3, (j, p, ang)


def small_case(name: str):
    data, cfg = SMALL[name]
    c = synth.make_case(**data)
    return c.image, c.templates, gisspa.Ctf(c.defocus, c.dfdiff, c.dfang), gisspa.Config.default(**cfg)


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def half_spectrum(full: np.ndarray) -> np.ndarray:
    """[n][ky][kx] full complex spectra -> [n][kx in 0..L/2][ky] (the library's kx-major layout)."""
    L = full.shape[-1]
    return np.ascontiguousarray(np.swapaxes(full[..., : L // 2 + 1], -1, -2))


# ---------------------------------------------------------------- margin-based pick identity
# The rule: a pick must come out identically -- same (x, y, template, angle), score within the
# tolerance tol(z) = rtol |z| + atol -- unless its decision margin (oracle.search(...,
# want_margins=True): how far in z its outcome stands from the nearest alternative outcome) is
# at most 2 tol(z), in which case FP32 rounding may legitimately choose the alternative.  Picks
# whose score lies within tol of the threshold may appear on one side only.  Every other
# difference is a failure.

def _tol(z, rtol, atol):
    return rtol * abs(float(z)) + atol


def check_chunk_picks(gpu, ref, margins, near, near_margins, thresh, rtol=SCORE_RTOL, atol=SCORE_ATOL):
    """Reference chunk picks (norm.cu:583-597): keyed by (angle, window, template, chunk)."""
    key = lambda p: (int(p["angle_index"]), int(p["window"]), int(p["template_id"]), int(p["chunk"]))
    G = {key(p): p for p in gpu}
    R = {key(p): (p, float(m)) for p, m in zip(ref, margins)}
    N = {key(p): (p, float(m)) for p, m in zip(near, near_margins)}
    band = _tol(thresh, rtol, atol)
    fail, exempt = [], 0
    max_rel = 0.0
    for k, (r, m) in R.items():
        z = float(r["score"])
        t = _tol(z, rtol, atol)
        g = G.get(k)
        if g is None:
            if z < thresh + band or m <= 2 * t:
                exempt += 1
            else:
                fail.append(("missing", k, z, m))
            continue
        same_pos = (float(g["x"]), float(g["y"])) == (float(r["x"]), float(r["y"]))
        if not same_pos:
            if m <= 2 * t:
                exempt += 1
            else:
                fail.append(("position", k, z, m, (float(g["x"]), float(g["y"])), (float(r["x"]), float(r["y"]))))
        d = abs(float(g["score"]) - z)
        max_rel = max(max_rel, d / max(abs(z), 1e-9))
        if d > t + (0.0 if same_pos else m):
            fail.append(("score", k, float(g["score"]), z))
    for k, g in G.items():
        if k in R:
            continue
        z = float(g["score"])
        t = _tol(z, rtol, atol)
        if z < thresh + band:
            exempt += 1
            continue
        nr = N.get(k)
        if nr is not None and nr[1] <= 2 * t and abs(float(nr[0]["score"]) - z) <= t:
            exempt += 1
            continue
        fail.append(("extra", k, z))
    return dict(n_gpu=len(G), n_ref=len(R), failures=fail, exempt=exempt, max_rel=max_rel)


def check_template_picks(gpu, ref, margins, thresh, rtol=SCORE_RTOL, atol=SCORE_ATOL):
    """norm_type=0 picks: one per (tile, angle, template) (nonorm.cu:488-557)."""
    key = lambda p: (int(p["tile"]), int(p["angle_index"]), int(p["template_id"]))
    G = {key(p): p for p in gpu}
    R = {key(p): (p, float(m)) for p, m in zip(ref, margins)}
    band = _tol(thresh, rtol, atol)
    fail, exempt = [], 0
    max_rel = 0.0
    for k, (r, m) in R.items():
        z = float(r["score"])
        t = _tol(z, rtol, atol)
        g = G.get(k)
        if g is None:
            if z < thresh + band:
                exempt += 1
            else:
                fail.append(("missing", k, z, m))
            continue
        same_pos = abs(float(g["x"]) - float(r["x"])) <= 1e-3 and abs(float(g["y"]) - float(r["y"])) <= 1e-3
        if not same_pos:
            if m <= 2 * t:
                exempt += 1
            else:
                fail.append(("position", k, z, m))
        d = abs(float(g["score"]) - z)
        max_rel = max(max_rel, d / max(abs(z), 1e-9))
        if d > t + (0.0 if same_pos else m):
            fail.append(("score", k, float(g["score"]), z))
    for k, g in G.items():
        if k not in R:
            if float(g["score"]) < thresh + band:
                exempt += 1
            else:
                fail.append(("extra", k, float(g["score"])))
    return dict(n_gpu=len(G), n_ref=len(R), failures=fail, exempt=exempt, max_rel=max_rel)


def check_topk_picks(gpu, ref, margins, rtol=SCORE_RTOL, atol=SCORE_ATOL):
    """Top-K picks with an exclusion radius: compared as sets of (x, y, template, angle)."""
    key = lambda p: (float(p["x"]), float(p["y"]), int(p["template_id"]), int(p["angle_index"]))
    fail, exempt = [], 0
    if len(gpu) != len(ref):
        fail.append(("count", len(gpu), len(ref)))
    G = {key(p): p for p in gpu}
    R = {key(p) for p in ref}
    loose = []  # ambiguous oracle picks the GPU did not reproduce
    max_rel = 0.0
    for r, m in zip(ref, margins):
        z = float(r["score"])
        t = _tol(z, rtol, atol)
        g = G.get(key(r))
        if g is None:
            if m <= 2 * t:
                loose.append(z)
            else:
                fail.append(("missing", key(r), z, float(m)))
            continue
        d = abs(float(g["score"]) - z)
        max_rel = max(max_rel, d / max(abs(z), 1e-9))
        if d > t:
            fail.append(("score", key(r), float(g["score"]), z))
    for g in gpu:
        if key(g) in R:
            continue
        z = float(g["score"])
        t = _tol(z, rtol, atol)
        hit = [i for i, zr in enumerate(loose) if abs(zr - z) <= 3 * t]
        if hit:
            loose.pop(hit[0])
            exempt += 1
        else:
            fail.append(("extra", key(g), z))
    return dict(n_gpu=len(gpu), n_ref=len(ref), failures=fail, exempt=exempt, max_rel=max_rel)
