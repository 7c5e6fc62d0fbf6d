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
                                        C.c_int, C.c_int]
        lib.orc_search_nonorm.argtypes = [C.POINTER(gisspa.Config), C.POINTER(gisspa.Ctf), _P, C.c_int, C.c_int,
                                          _P, C.c_int, C.c_int, C.c_int, _P, C.c_size_t, C.POINTER(C.c_size_t),
                                          C.c_int]
        lib.orc_tiles.argtypes = [C.c_int, C.c_int, C.c_int, _P, _P, C.c_int]
        lib.orc_num_threads.restype = C.c_int
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
           max_templates: int = 0, max_angles: int = 0):
    """Full search; returns picks (PICK_DTYPE) and, for norm_type=1 with want_stats, (mu, sigma) maps."""
    image = np.ascontiguousarray(image, dtype=np.float32)
    stack = np.ascontiguousarray(stack, dtype=np.float32)
    ny, nx = image.shape
    n, th, tw = stack.shape
    out = np.zeros(cap, dtype=gisspa.PICK_DTYPE)
    nout = C.c_size_t(0)
    lib = load()
    if cfg.norm_type:
        l = cfg.window_size
        W = len(window_offsets(nx, l, cfg.overlap)) * len(window_offsets(ny, l, cfg.overlap))
        stats = np.zeros((W, l, l, 2), dtype=np.float64) if want_stats else None
        st = lib.orc_search_norm(C.byref(cfg), C.byref(ctf), image.ctypes.data, nx, ny, stack.ctypes.data, n, tw, th,
                                 out.ctypes.data, cap, C.byref(nout),
                                 stats.ctypes.data if stats is not None else None, max_templates, max_angles)
    else:
        stats = None
        st = lib.orc_search_nonorm(C.byref(cfg), C.byref(ctf), image.ctypes.data, nx, ny, stack.ctypes.data, n, tw,
                                   th, out.ctypes.data, cap, C.byref(nout), max_angles)
    if st == gisspa.ERR_CAPACITY:
        return search(cfg, ctf, image, stack, cap=int(nout.value), want_stats=want_stats,
                      max_templates=max_templates, max_angles=max_angles)
    if st != 0:
        raise RuntimeError(f"oracle status {st}")
    picks = out[: nout.value].copy()
    return (picks, stats) if want_stats else picks


def tiles(width: int, height: int, tile: int = 720):
    ulx = np.zeros(4096, np.int32)
    uly = np.zeros(4096, np.int32)
    n = load().orc_tiles(width, height, tile, ulx.ctypes.data, uly.ctypes.data, 4096)
    return list(zip(ulx[:n].tolist(), uly[:n].tolist()))


def num_threads() -> int:
    return load().orc_num_threads()
