"""Python binding of libgisspa.so (ctypes over the C-ABI in include/gisspa.h).

The classes at the bottom mirror the reference's host interface for the search
path: ``SearchNorm`` / ``SearchNoNorm`` (GisSPA_v2.0 include/norm.cuh:37-54,
include/nonorm.cuh:44-48) with ``work(templates, image, output)`` writing the
reference pick-list lines (norm.cu:602-618, nonorm.cu:539-557).  All compute
runs in the CUDA library; this module only marshals arguments.  Loading fails
loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "_build", "libgisspa.so")

OK = 0
ERR_ARG, ERR_SHAPE, ERR_UNSUPPORTED, ERR_CUDA, ERR_NOMEM, ERR_CAPACITY, ERR_STATE, ERR_TIMEOUT, ERR_IO = range(1, 10)
PICK_CHUNK, PICK_TOPK = 0, 1
SPEC_FP32, SPEC_FP16, SPEC_BF16 = 0, 1, 2
QUIRK_OUTLIER_FP32_SERIAL = 0x1
QUIRK_COUNT_PADDED_TEMPLATES = 0x2
QUIRK_NEULER_TRUNC = 0x4
QUIRKS_REFERENCE = 0x7


class Config(C.Structure):
    """gisspa_config (include/gisspa.h); first block = reference Config keys."""

    _fields_ = [(n, C.c_float) for n in ("angpix", "phistep", "kk", "energy", "cs", "highres", "lowres",
                                         "diameter", "threshold")] + \
               [(n, C.c_int) for n in ("window_size", "overlap", "norm_type", "invert", "phase_flip")] + \
               [(n, C.c_float) for n in ("edge_half_width", "ampconst", "a", "b", "b2", "bfactor", "bfactor2",
                                         "bfactor3")] + \
               [("pick_mode", C.c_int), ("topk", C.c_int), ("exclusion_radius", C.c_float),
                ("spectrum_precision", C.c_int), ("template_batch", C.c_int), ("window_batch", C.c_int),
                ("quirks", C.c_int), ("tile_size", C.c_int), ("cuda_graphs", C.c_int), ("pass_b_shape", C.c_int),
                ("tensor_cores", C.c_int), ("pass_a_shape", C.c_int),
                ("prune_sweep2", C.c_int)]

    @classmethod
    def default(cls, **kw) -> "Config":
        """Reference defaults (EMReader/DataReader2.h:19-44, 73-77) plus the additions."""
        c = cls()
        c.angpix, c.phistep, c.kk, c.energy, c.cs = -1.0, -1.0, -1.0, -1.0, -1.0
        c.highres, c.lowres, c.diameter, c.threshold = -1.0, 0.0, -1.0, 7.0
        c.window_size, c.overlap, c.norm_type, c.invert, c.phase_flip = 320, 0, 0, 0, 0
        c.edge_half_width, c.ampconst = 4.0, 0.07
        c.a, c.b, c.b2, c.bfactor, c.bfactor2, c.bfactor3 = -10.81, 1.0, 0.32, -18.17, -15.22, 1.72
        c.pick_mode, c.topk, c.exclusion_radius = PICK_CHUNK, 1000, 64.0
        c.spectrum_precision, c.template_batch, c.window_batch = SPEC_FP32, 0, 0
        c.quirks, c.tile_size, c.cuda_graphs, c.pass_b_shape = QUIRKS_REFERENCE, 720, 1, -1
        c.tensor_cores = 0
        c.pass_a_shape = -1
        c.prune_sweep2 = 1
        for k, v in kw.items():
            if not hasattr(c, k):
                raise KeyError(k)
            setattr(c, k, v)
        return c

    def copy(self, **kw) -> "Config":
        c = Config()
        C.pointer(c)[0] = self
        for k, v in kw.items():
            setattr(c, k, v)
        return c


class Ctf(C.Structure):
    _fields_ = [("defocus", C.c_double), ("dfdiff", C.c_double), ("dfang", C.c_double)]


class Pick(C.Structure):
    _fields_ = [("score", C.c_float), ("x", C.c_float), ("y", C.c_float), ("angle", C.c_float),
                ("template_id", C.c_int), ("window", C.c_int), ("tile", C.c_int), ("angle_index", C.c_int),
                ("chunk", C.c_int), ("theta", C.c_float)]


PICK_DTYPE = np.dtype([("score", "<f4"), ("x", "<f4"), ("y", "<f4"), ("angle", "<f4"), ("template_id", "<i4"),
                       ("window", "<i4"), ("tile", "<i4"), ("angle_index", "<i4"), ("chunk", "<i4"),
                       ("theta", "<f4")])
assert PICK_DTYPE.itemsize == C.sizeof(Pick)


class Grad(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("score", "d_dx", "d_dy", "d_theta", "d_dfu", "d_dfv", "d_dfang")]


GRAD_DTYPE = np.dtype([(n, "<f4") for n in ("score", "d_dx", "d_dy", "d_theta", "d_dfu", "d_dfv", "d_dfang")])


class RunPaths(C.Structure):
    _fields_ = [("input", C.c_char * 1024), ("template_path", C.c_char * 1024), ("eulerfile", C.c_char * 1024),
                ("output", C.c_char * 1024), ("first", C.c_int), ("last", C.c_int), ("gpu_id", C.c_int),
                ("template_volume", C.c_char * 1024)]


class Stats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_prep", C.c_double), ("ms_sweep1", C.c_double),
                ("ms_sweep2", C.c_double), ("ms_pick", C.c_double), ("pairs", C.c_longlong),
                ("kernel_launches", C.c_longlong), ("candidates", C.c_longlong), ("pass_a_us", C.c_double),
                ("pass_b_us", C.c_double), ("pairs_per_launch", C.c_double), ("templates_per_launch", C.c_double),
                ("pass_samples", C.c_int), ("window_size", C.c_int), ("pass_b_variant", C.c_int),
                ("tuned_us_per_pair", C.c_double), ("graph_replays", C.c_longlong), ("corr_pair_us", C.c_double),
                ("corr_timed_launches", C.c_longlong), ("pass_a_variant", C.c_int),
                ("rows_alive", C.c_double), ("pairs_alive", C.c_double)]


class ShardInfo(C.Structure):
    _fields_ = [("n_pixels", C.c_size_t), ("n_windows", C.c_int), ("n_angles", C.c_int), ("pick_mode", C.c_int)]


# Exported symbols and their ctypes signatures (kept in sync with include/gisspa.h).
_P = C.c_void_p
SIGNATURES = {
    "gisspa_config_default": (None, [C.POINTER(Config)]),
    "gisspa_config_load": (C.c_int, [C.c_char_p, C.POINTER(Config), C.POINTER(RunPaths)]),
    "gisspa_create": (C.c_int, [C.POINTER(Config), C.c_int, C.POINTER(_P)]),
    "gisspa_set_templates": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int]),
    "gisspa_search": (C.c_int, [_P, _P, C.c_int, C.c_int, C.POINTER(Ctf), _P, C.c_size_t,
                                C.POINTER(C.c_size_t)]),
    "gisspa_search_device": (C.c_int, [_P, _P, C.c_int, C.c_int, C.POINTER(Ctf), _P, C.c_size_t,
                                       C.POINTER(C.c_size_t)]),
    "gisspa_search_batch": (C.c_int, [_P, C.c_int, _P, _P, _P, _P, _P, C.c_size_t, _P]),
    "gisspa_format_pick": (C.c_int, [C.POINTER(Pick), C.c_int, C.c_char_p, C.POINTER(Ctf), C.c_float, C.c_float,
                                     C.c_char_p, C.c_size_t]),
    "gisspa_get_stats": (C.c_int, [_P, C.POINTER(Stats)]),
    "gisspa_last_error": (C.c_char_p, [_P]),
    "gisspa_destroy": (None, [_P]),
    "gisspa_version": (C.c_char_p, []),
    "gisspa_score_grad": (C.c_int, [_P, _P, C.c_size_t, _P, C.POINTER(Ctf), _P]),
    "gisspa_refine": (C.c_int, [_P, _P, C.c_size_t, C.c_int, C.POINTER(Ctf), _P]),
    "gisspa_cc_maps": (C.c_int, [_P, _P, C.c_int, _P, C.c_int, C.c_int, _P]),
    "gisspa_cc_maps_noalloc": (C.c_int, [_P, C.c_int, _P, C.c_int, C.c_int, C.c_int, _P, _P]),
    "gisspa_debug_stage": (C.c_int, [_P, C.c_int, _P, C.c_int, C.c_int, C.POINTER(Ctf), C.c_float, _P,
                                     C.c_size_t]),
    "gisspa_shard_begin": (C.c_int, [_P, _P, C.c_int, C.c_int, C.POINTER(Ctf), C.POINTER(ShardInfo)]),
    "gisspa_shard_sweep": (C.c_int, [_P, C.c_int, C.c_int, C.c_int]),
    "gisspa_shard_export": (C.c_int, [_P, _P, _P, _P]),
    "gisspa_shard_import": (C.c_int, [_P, _P, _P, _P]),
    "gisspa_shard_picks": (C.c_int, [_P, _P, C.c_size_t, C.POINTER(C.c_size_t)]),
    "gisspa_debug_wait_probe": (C.c_int, [_P, C.c_double]),
    "gisspa_debug_fft": (C.c_int, [_P, _P, C.c_longlong, C.c_int, C.c_int]),
    "gisspa_project": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, _P, C.c_int, C.c_int, _P]),
    "gisspa_set_templates_from_volume": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, _P, C.c_int, C.c_int]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libgisspa.so; raises if it is missing (there is no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(f"libgisspa.so not built: {path} (run __graft_entry__.build())")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class GisspaError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"gisspa status {status}: {msg}")
        self.status = status


def _check(h, st: int):
    if st != OK:
        msg = load().gisspa_last_error(h)
        raise GisspaError(st, msg.decode() if msg else "")


def load_config(path: str) -> tuple[Config, RunPaths]:
    c, p = Config(), RunPaths()
    st = load().gisspa_config_load(path.encode(), C.byref(c), C.byref(p))
    _check(None, st)
    return c, p


class Searcher:
    """One handle on one device (gisspa_create ... gisspa_destroy)."""

    def __init__(self, cfg: Config, device: int = 0):
        self.lib = load()
        self.cfg = cfg
        h = _P()
        _check(None, self.lib.gisspa_create(C.byref(cfg), device, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.lib.gisspa_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_templates(self, stack: np.ndarray):
        stack = np.ascontiguousarray(stack, dtype=np.float32)
        n, h, w = stack.shape
        _check(self.h, self.lib.gisspa_set_templates(self.h, stack.ctypes.data, n, w, h))
        self._tmpl_keep = stack

    def search(self, image: np.ndarray, ctf: Ctf, cap: int = 1 << 20) -> np.ndarray:
        image = np.ascontiguousarray(image, dtype=np.float32)
        ny, nx = image.shape
        out = np.zeros(cap, dtype=PICK_DTYPE)
        n = C.c_size_t(0)
        st = self.lib.gisspa_search(self.h, image.ctypes.data, nx, ny, C.byref(ctf), out.ctypes.data, cap,
                                    C.byref(n))
        if st == ERR_CAPACITY:
            return self.search(image, ctf, cap=int(n.value))
        _check(self.h, st)
        return out[: n.value].copy()

    def search_device(self, d_image_ptr: int, nx: int, ny: int, ctf: Ctf, out: np.ndarray) -> int:
        n = C.c_size_t(0)
        st = self.lib.gisspa_search_device(self.h, C.c_void_p(d_image_ptr), nx, ny, C.byref(ctf),
                                           out.ctypes.data, out.shape[0], C.byref(n))
        _check(self.h, st)
        return int(n.value)

    def search_batch(self, images: list, ctfs: list, cap: int = 1 << 22):
        imgs = [np.ascontiguousarray(i, dtype=np.float32) for i in images]
        n = len(imgs)
        ptrs = (C.c_void_p * n)(*[i.ctypes.data for i in imgs])
        nxs = (C.c_int * n)(*[i.shape[1] for i in imgs])
        nys = (C.c_int * n)(*[i.shape[0] for i in imgs])
        cs = (Ctf * n)(*ctfs)
        out = np.zeros(cap, dtype=PICK_DTYPE)
        offs = (C.c_size_t * (n + 1))()
        st = self.lib.gisspa_search_batch(self.h, n, ptrs, nxs, nys, cs, out.ctypes.data, cap, offs)
        _check(self.h, st)
        o = list(offs)
        return [out[o[i]:o[i + 1]].copy() for i in range(n)]

    def score_grad(self, picks: np.ndarray, params: np.ndarray | None = None, ctf: Ctf | None = None) -> np.ndarray:
        """Scores and gradients of picks from the last norm_type=1 search (gisspa_score_grad)."""
        picks = np.ascontiguousarray(picks, dtype=PICK_DTYPE)
        out = np.zeros(len(picks), dtype=GRAD_DTYPE)
        pp = None
        if params is not None:
            params = np.ascontiguousarray(params, dtype=np.float32).reshape(len(picks), 3)
            pp = params.ctypes.data
        _check(self.h, self.lib.gisspa_score_grad(self.h, picks.ctypes.data, len(picks), pp,
                                                  C.byref(ctf) if ctf is not None else None, out.ctypes.data))
        return out

    def refine(self, picks: np.ndarray, steps: int = 20, ctf: Ctf | None = None):
        """Refined copies of picks and the refined CTF (gisspa_refine)."""
        picks = np.ascontiguousarray(picks, dtype=PICK_DTYPE).copy()
        c = Ctf(ctf.defocus, ctf.dfdiff, ctf.dfang) if ctf is not None else None
        params = np.zeros((len(picks), 3), np.float32)
        _check(self.h, self.lib.gisspa_refine(self.h, picks.ctypes.data, len(picks), steps,
                                              C.byref(c) if c is not None else None, params.ctypes.data))
        return picks, c, params

    # ---- template generation (projections of a 3D map, emdata::project3d semantics)
    def project(self, volume: np.ndarray, angles, ri: int = 0) -> np.ndarray:
        vol = np.ascontiguousarray(volume, dtype=np.float32)
        nz, ny, nx = vol.shape
        ang = np.ascontiguousarray(np.asarray(angles, dtype=np.float32).reshape(-1, 3))
        out = np.zeros((len(ang), ny, nx), dtype=np.float32)
        _check(self.h, self.lib.gisspa_project(self.h, vol.ctypes.data, nx, ny, nz, ang.ctypes.data, len(ang), ri,
                                               out.ctypes.data))
        return out

    def set_templates_from_volume(self, volume: np.ndarray, angles, ri: int = 0):
        vol = np.ascontiguousarray(volume, dtype=np.float32)
        nz, ny, nx = vol.shape
        ang = np.ascontiguousarray(np.asarray(angles, dtype=np.float32).reshape(-1, 3))
        _check(self.h, self.lib.gisspa_set_templates_from_volume(self.h, vol.ctypes.data, nx, ny, nz,
                                                                 ang.ctypes.data, len(ang), ri))

    # ---- one micrograph across ranks (gisspa_shard_*); device pointers are ints
    def shard_begin(self, image: np.ndarray, ctf: Ctf) -> ShardInfo:
        image = np.ascontiguousarray(image, dtype=np.float32)
        ny, nx = image.shape
        info = ShardInfo()
        _check(self.h, self.lib.gisspa_shard_begin(self.h, image.ctypes.data, nx, ny, C.byref(ctf), C.byref(info)))
        return info

    def shard_sweep(self, sweep: int, angle_begin: int, angle_end: int):
        _check(self.h, self.lib.gisspa_shard_sweep(self.h, sweep, angle_begin, angle_end))

    def shard_export(self, d_sum: int, d_sum_sq: int, d_key: int | None):
        _check(self.h, self.lib.gisspa_shard_export(self.h, C.c_void_p(d_sum), C.c_void_p(d_sum_sq),
                                                    C.c_void_p(d_key) if d_key else None))

    def shard_import(self, d_sum: int, d_sum_sq: int, d_key: int | None):
        _check(self.h, self.lib.gisspa_shard_import(self.h, C.c_void_p(d_sum), C.c_void_p(d_sum_sq),
                                                    C.c_void_p(d_key) if d_key else None))

    def shard_picks(self, cap: int = 1 << 20) -> np.ndarray:
        out = np.zeros(cap, dtype=PICK_DTYPE)
        n = C.c_size_t(0)
        st = self.lib.gisspa_shard_picks(self.h, out.ctypes.data, cap, C.byref(n))
        if st == ERR_CAPACITY:
            return self.shard_picks(cap=int(n.value))
        _check(self.h, st)
        return out[: n.value].copy()

    def stats(self) -> Stats:
        s = Stats()
        _check(self.h, self.lib.gisspa_get_stats(self.h, C.byref(s)))
        return s


def format_pick(p, lst_index: int, path: str, ctf: Ctf, euler1: float, euler2: float) -> str:
    rec = Pick()
    for k in PICK_DTYPE.names:
        setattr(rec, k, p[k].item() if hasattr(p[k], "item") else p[k])
    buf = C.create_string_buffer(2048)
    n = load().gisspa_format_pick(C.byref(rec), lst_index, path.encode(), C.byref(ctf), euler1, euler2, buf, 2048)
    if n < 0:
        raise GisspaError(ERR_ARG, "format buffer too small")
    return buf.value.decode()


# ---------------------------------------------------------------- reference-shaped interface
@dataclass
class EulerData:
    """EulerData (EMReader/DataReader2.h:85-91): one (euler1, euler2, euler3) per template."""
    euler1: list
    euler2: list
    euler3: list

    def size(self) -> int:
        return len(self.euler1)


@dataclass
class Templates:
    """Templates (utils/templates.hpp): a contiguous float stack of count x height x width."""
    data: np.ndarray

    @property
    def width(self):
        return self.data.shape[2]

    @property
    def height(self):
        return self.data.shape[1]


@dataclass
class Image:
    """Image (utils/image.hpp): one micrograph plus its LST entry fields."""
    data: np.ndarray
    rpath: str = ""
    unused: int = 0
    defocus: float = 0.0
    dfdiff: float = 0.0
    dfang: float = 0.0


class _SearchBase:
    def __init__(self, config: Config, euler: EulerData, size, device: int = 0):
        self.para = config
        self.euler = euler
        self.size = size
        self.searcher = Searcher(config, device)
        self.line_count = 0

    def work(self, temp: Templates, image: Image, output) -> np.ndarray:
        self.searcher.set_templates(temp.data)
        ctf = Ctf(image.defocus, image.dfdiff, image.dfang)
        picks = self.searcher.search(image.data, ctf)
        for p in picks:
            j = int(p["template_id"])
            output.write(format_pick(p, image.unused, image.rpath, ctf, self.euler.euler1[j], self.euler.euler2[j]))
            self.line_count += 1
        return picks


class SearchNorm(_SearchBase):
    """norm_type=1 search (SearchNorm, include/norm.cuh:37-54)."""

    def __init__(self, config: Config, euler: EulerData, size, device: int = 0):
        super().__init__(config.copy(norm_type=1), euler, size, device)


class SearchNoNorm(_SearchBase):
    """norm_type=0 tiled search (SearchNoNorm, include/nonorm.cuh:44-48)."""

    def __init__(self, config: Config, euler: EulerData, size, device: int = 0):
        super().__init__(config.copy(norm_type=0), euler, size, device)
