"""ctypes wrapper of the FP64 oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "gisspa_v2.0_b200"))
import gisspa  # noqa: E402  (struct definitions shared with the product binding)

LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lib = None
_P = C.c_void_p


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle not built: {LIB_PATH}")
        lib = C.CDLL(LIB_PATH)
        lib.orc_fft2d.argtypes = [_P, C.c_int, C.c_int, C.c_int]
        lib.orc_prep_templates.argtypes = [C.POINTER(gisspa.Config), C.POINTER(gisspa.Ctf), _P, C.c_int, C.c_int,
                                           C.c_int, _P]
        lib.orc_prep_image.argtypes = [C.POINTER(gisspa.Config), C.POINTER(gisspa.Ctf), _P, C.c_int, C.c_int, _P]
        lib.orc_window_offsets.argtypes = [C.c_int, C.c_int, C.c_int, _P, C.c_int]
        lib.orc_window_spectra.argtypes = [C.POINTER(gisspa.Config), _P, C.c_int, C.c_int, _P]
        lib.orc_rotated_spectrum.argtypes = [C.POINTER(gisspa.Config), C.POINTER(gisspa.Ctf), _P, C.c_float, _P]
        lib.orc_search_norm.argtypes = [C.POINTER(gisspa.Config), C.POINTER(gisspa.Ctf), _P, C.c_int, C.c_int, _P,
                                        C.c_int, C.c_int, C.c_int, _P, C.c_size_t, C.POINTER(C.c_size_t), _P,
                                        C.c_int, C.c_int, _P, _P, _P, C.c_size_t, C.POINTER(C.c_size_t)]
        lib.orc_search_nonorm.argtypes = [C.POINTER(gisspa.Config), C.POINTER(gisspa.Ctf), _P, C.c_int, C.c_int,
                                          _P, C.c_int, C.c_int, C.c_int, _P, C.c_size_t, C.POINTER(C.c_size_t),
                                          C.c_int, _P]
        lib.orc_tiles.argtypes = [C.c_int, C.c_int, C.c_int, _P, _P, C.c_int]
        lib.orc_num_threads.restype = C.c_int
        lib.orc_project3d.argtypes = [_P, C.c_int, C.c_int, C.c_int, _P, C.c_int, C.c_int, _P]
        _lib = lib
    return _lib


def fft2(a: np.ndarray, sign: int) -> np.ndarray:
    """Unnormalised 2D transform (sign -1 forward, +1 inverse) of a complex array."""
    d = np.ascontiguousarray(a, dtype=np.complex128).copy()
    load().orc_fft2d(d.ctypes.data, d.shape[0], d.shape[1], sign)
    return d


def prep_templates(cfg, ctf, stack: np.ndarray) -> np.ndarray:
    stack = np.ascontiguousarray(stack, dtype=np.float32)
    n, th, tw = stack.shape
    l = cfg.window_size
    out = np.zeros((n, l, l), dtype=np.complex128)
    st = load().orc_prep_templates(C.byref(cfg), C.byref(ctf), stack.ctypes.data, n, tw, th, out.ctypes.data)
    assert st == 0, st
    return out


def prep_image(cfg, ctf, img: np.ndarray) -> np.ndarray:
    img = np.ascontiguousarray(img, dtype=np.float32)
    out = np.zeros(img.shape, dtype=np.float64)
    load().orc_prep_image(C.byref(cfg), C.byref(ctf), img.ctypes.data, img.shape[1], img.shape[0], out.ctypes.data)
    return out


def window_offsets(length: int, l: int, ov: int) -> list:
    buf = np.zeros(4096, dtype=np.int32)
    n = load().orc_window_offsets(length, l, ov, buf.ctypes.data, 4096)
    return buf[:n].tolist()


def window_spectra(cfg, img_pre: np.ndarray) -> np.ndarray:
    img_pre = np.ascontiguousarray(img_pre, dtype=np.float64)
    ny, nx = img_pre.shape
    l = cfg.window_size
    W = len(window_offsets(nx, l, cfg.overlap)) * len(window_offsets(ny, l, cfg.overlap))
    out = np.zeros((W, l, l), dtype=np.complex128)
    load().orc_window_spectra(C.byref(cfg), img_pre.ctypes.data, nx, ny, out.ctypes.data)
    return out


def rotated_spectrum(cfg, ctf, prep: np.ndarray, theta: float) -> np.ndarray:
    prep = np.ascontiguousarray(prep, dtype=np.complex128)
    out = np.zeros_like(prep)
    load().orc_rotated_spectrum(C.byref(cfg), C.byref(ctf), prep.ctypes.data, theta, out.ctypes.data)
    return out


def search(cfg, ctf, image: np.ndarray, stack: np.ndarray, cap: int = 1 << 20, want_stats: bool = False,
           max_templates: int = 0, max_angles: int = 0, want_margins: bool = False):
    """Full search; returns picks (PICK_DTYPE) and, for norm_type=1 with want_stats, (mu, sigma) maps.
    want_margins: also returns each pick's decision margin in z (see orc_search_norm /
    orc_search_nonorm) and, for chunk picks, the near misses (picks, margins) that FP32 rounding
    could turn into picks: the result is then (picks, margins, near, near_margins[, stats])."""
    image = np.ascontiguousarray(image, dtype=np.float32)
    stack = np.ascontiguousarray(stack, dtype=np.float32)
    ny, nx = image.shape
    n, th, tw = stack.shape
    out = np.zeros(cap, dtype=gisspa.PICK_DTYPE)
    nout = C.c_size_t(0)
    margins = np.zeros(cap, dtype=np.float64) if want_margins else None
    near_cap = 1 << 16
    near = np.zeros(near_cap, dtype=gisspa.PICK_DTYPE) if want_margins else None
    near_m = np.zeros(near_cap, dtype=np.float64) if want_margins else None
    n_near = C.c_size_t(0)
    lib = load()
    ptr = lambda a: a.ctypes.data if a is not None else None
    if cfg.norm_type:
        l = cfg.window_size
        W = len(window_offsets(nx, l, cfg.overlap)) * len(window_offsets(ny, l, cfg.overlap))
        stats = np.zeros((W, l, l, 2), dtype=np.float64) if want_stats else None
        st = lib.orc_search_norm(C.byref(cfg), C.byref(ctf), image.ctypes.data, nx, ny, stack.ctypes.data, n, tw, th,
                                 out.ctypes.data, cap, C.byref(nout), ptr(stats), max_templates, max_angles,
                                 ptr(margins), ptr(near), ptr(near_m), near_cap, C.byref(n_near))
    else:
        stats = None
        st = lib.orc_search_nonorm(C.byref(cfg), C.byref(ctf), image.ctypes.data, nx, ny, stack.ctypes.data, n, tw,
                                   th, out.ctypes.data, cap, C.byref(nout), max_angles, ptr(margins))
    if st == gisspa.ERR_CAPACITY:
        return search(cfg, ctf, image, stack, cap=int(nout.value), want_stats=want_stats,
                      max_templates=max_templates, max_angles=max_angles, want_margins=want_margins)
    if st != 0:
        raise RuntimeError(f"oracle status {st}")
    assert n_near.value <= near_cap, "more near misses than the buffer holds"
    picks = out[: nout.value].copy()
    if want_margins:
        res = (picks, margins[: nout.value].copy(), near[: n_near.value].copy(), near_m[: n_near.value].copy())
        return res + (stats,) if want_stats else res
    return (picks, stats) if want_stats else picks


def tiles(width: int, height: int, tile: int = 720):
    ulx = np.zeros(4096, np.int32)
    uly = np.zeros(4096, np.int32)
    n = load().orc_tiles(width, height, tile, ulx.ctypes.data, uly.ctypes.data, 4096)
    return list(zip(ulx[:n].tolist(), uly[:n].tolist()))


def project3d(volume: np.ndarray, angles, ri: int = 0) -> np.ndarray:
    """Projections [n][ny][nx] of a float32 volume [nz][ny][nx] at (alt, az, phi) radians
    (emdata::project3d semantics; see orc_project3d)."""
    vol = np.ascontiguousarray(volume, dtype=np.float32)
    nz, ny, nx = vol.shape
    ang = np.ascontiguousarray(np.asarray(angles, dtype=np.float32).reshape(-1, 3))
    out = np.zeros((len(ang), ny, nx), dtype=np.float32)
    st = load().orc_project3d(vol.ctypes.data, nx, ny, nz, ang.ctypes.data, len(ang), ri, out.ctypes.data)
    assert st == 0, st
    return out


def num_threads() -> int:
    return load().orc_num_threads()


# ---------------------------------------------------------------- adjoint checker (FP64)
REF_PI = 3.1415926535  # utils/constants.h:3


def _shell_index(a, b):
    n = a.astype(np.int64) ** 2 + b.astype(np.int64) ** 2
    k = np.floor(np.sqrt(n.astype(np.float64)) + 0.5).astype(np.int64)
    k = np.where((k > 0) & (k * k - k >= n), k - 1, k)
    k = np.where(k * k + k < n, k + 1, k)
    return k - 1


def window_rms_factor(win: np.ndarray) -> float:
    """Radial RMS factor m of one real window (norm.cu:431-466): F = FFT/L^2,
    m = sqrt(sum |F|^2 / count^2) over x <= L/2 and valid shells."""
    L = win.shape[0]
    F = np.fft.fft2(win) / (L * L)
    y, x = np.mgrid[0:L, 0:L]
    r = _shell_index(np.minimum(y, L - y), np.minimum(x, L - x))
    sel = (x <= L // 2) & (r >= 0) & (r < L // 2)
    return float(np.sqrt(np.sum(np.abs(F[sel]) ** 2) / sel.sum() ** 2))


def pick_score(cfg, prep_t: np.ndarray, img_pre: np.ndarray, off: tuple, px: int, py: int, dx: float, dy: float,
               theta: float, mu: float, sigma: float) -> float:
    """FP64 restatement of the score the adjoint differentiates (z of one pick at a continuous
    shift (dx, dy) and search angle theta), from a prepared real-space template prep_t
    [L, L] (the CTF enters through it) and the preprocessed micrograph.

    c = (1/L^2) sum_y W(y + p + L/2) n(y - d), W = window / (L^2 m), n = the rotated (bilinear,
    reference boundary rules), masked, mean/variance-normalised template; z = (c - mu)/sigma."""
    L = cfg.window_size
    ox, oy = off
    ny, nx = img_pre.shape
    win = np.zeros((L, L))
    h_, w_ = min(L, ny - oy), min(L, nx - ox)
    win[:h_, :w_] = img_pre[oy:oy + h_, ox:ox + w_]
    W = win / (L * L * window_rms_factor(win))
    Y, X = np.mgrid[0:L, 0:L].astype(np.float64)
    ux, uy = X - (L // 2 + dx), Y - (L // 2 + dy)
    r = np.hypot(ux, uy)
    dm = 1.5 * cfg.diameter
    r_in, r_out = dm / 2, dm / 2 + 2 * cfg.edge_half_width
    m = np.where(r > r_out, 0.0, np.where(r >= r_in, 0.5 * np.cos(REF_PI * (r - r_in) / (2 * cfg.edge_half_width)) + 0.5,
                                          1.0))
    th = theta * REF_PI / 180
    cs, sn = np.cos(th), np.sin(th)
    x2 = cs * ux + sn * uy + L // 2
    y2 = -sn * ux + cs * uy + L // 2
    inside = ~((x2 < 0) | (x2 > L - 1.0) | (y2 < 0) | (y2 > L - 1.0))
    x2c, y2c = np.where(inside, x2, 0.0), np.where(inside, y2, 0.0)
    ii, jj = np.floor(x2c).astype(int), np.floor(y2c).astype(int)
    i1 = np.where(ii == L - 1, ii, ii + 1)
    j1 = np.where(jj == L - 1, jj, jj + 1)
    t, u = x2c - ii, y2c - jj
    P = prep_t
    R = (P[jj, ii] * (1 - t) * (1 - u) + P[jj, i1] * t * (1 - u) + P[j1, i1] * t * u + P[j1, ii] * (1 - t) * u)
    a = np.where(inside, m * R, 0.0)
    mean = a.sum() / (L * L)
    sd = np.sqrt((a * a).sum() / (L * L) - mean * mean)
    n = (a - mean) / sd
    Ws = np.roll(W, shift=(-(py + L // 2), -(px + L // 2)), axis=(0, 1))  # W(y + p + L/2)
    c = float((Ws * n).sum()) / (L * L)
    return (c - mu) / sigma
