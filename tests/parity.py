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


def compare_chunk_picks(gpu: np.ndarray, ref: np.ndarray, thresh: float, rtol=SCORE_RTOL, atol=SCORE_ATOL):
    """Chunk picks must match by (angle, window, template, chunk) with scores within tolerance and
    identical centres, except picks whose score lies within the tolerance of the threshold."""
    key = lambda p: (int(p["angle_index"]), int(p["window"]), int(p["template_id"]), int(p["chunk"]))
    G = {key(p): p for p in gpu}
    R = {key(p): p for p in ref}
    band = rtol * abs(thresh) + atol
    report = dict(n_gpu=len(G), n_ref=len(R), missing=0, extra=0, score_bad=0, pos_bad=0, max_rel=0.0)
    for k, r in R.items():
        if k not in G:
            if r["score"] >= thresh + band:
                report["missing"] += 1
            continue
        g = G[k]
        d = abs(float(g["score"]) - float(r["score"]))
        report["max_rel"] = max(report["max_rel"], d / max(abs(float(r["score"])), 1e-9))
        if d > rtol * abs(float(r["score"])) + atol:
            report["score_bad"] += 1
        if (g["x"], g["y"]) != (r["x"], r["y"]):
            report["pos_bad"] += 1
    for k, g in G.items():
        if k not in R and g["score"] >= thresh + band:
            report["extra"] += 1
    return report


def compare_template_picks(gpu: np.ndarray, ref: np.ndarray, thresh: float, rtol=SCORE_RTOL, atol=SCORE_ATOL,
                           key_fields=("tile", "angle_index", "template_id")):
    """norm_type=0 picks: one per (tile, angle, template); centre and score compared."""
    key = lambda p: tuple(int(p[f]) for f in key_fields)
    G = {key(p): p for p in gpu}
    R = {key(p): p for p in ref}
    band = rtol * abs(thresh) + atol
    report = dict(n_gpu=len(G), n_ref=len(R), missing=0, extra=0, score_bad=0, pos_bad=0, max_rel=0.0)
    for k, r in R.items():
        if k not in G:
            if r["score"] >= thresh + band:
                report["missing"] += 1
            continue
        g = G[k]
        d = abs(float(g["score"]) - float(r["score"]))
        report["max_rel"] = max(report["max_rel"], d / max(abs(float(r["score"])), 1e-9))
        if d > rtol * abs(float(r["score"])) + atol:
            report["score_bad"] += 1
        if abs(float(g["x"]) - float(r["x"])) > 1e-3 or abs(float(g["y"]) - float(r["y"])) > 1e-3:
            report["pos_bad"] += 1
    for k, g in G.items():
        if k not in R and g["score"] >= thresh + band:
            report["extra"] += 1
    return report
