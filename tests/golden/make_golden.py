"""Generate golden pick lists by running the reference build (oracle/_ref/gisspa_ref).

Run on a machine with a GPU after oracle/ref_build.sh has compiled the reference
search sources:

    python tests/golden/make_golden.py --out tests/golden

For each case below it writes the seeded synthetic inputs as MRC files plus the
reference's config / LST / Euler files into a scratch directory, runs the
reference binary exactly as its test script does (``main <config>``), parses the
pick list it prints and stores ``<case>.json``: the case parameters, a checksum of
the generated inputs and the reference's pick lines.  The Euler file gives
template j the angles (j, 0, 0), so euler1 in each line identifies the template.
norm_type=1 cases also store the pick lines of oracle/_ref/gisspa_ref_sync, the same
sources with kernels.cu compiled for device debug (its warp-synchronous reduction tails
then read what their neighbours wrote), as ``picks_sync``.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
import fixture_data  # noqa: E402

# Pick thresholds of the later cases, set from the oracle's score distribution so that each
# case prints tens to hundreds of picks.
THRESH = {"norm_1024_l512": 4.37, "norm_840_l320": 4.29, "nonorm_1024_l512_t8": 7.45, "nonorm_1024_l320": 12.9}

# Cases satisfy the reference's preconditions: window_size % 16 == 0, windows <= templates
# (norm.cu:141-147 reads past the stack otherwise) and images >= 720 for norm_type=0.
CASES = {
    "norm_512_l256": dict(
        data=dict(shape=(512, 512), n_templates=4, tsize=64, n_blobs=12, n_particles=5, amp=0.6, seed=11, margin=40),
        ctf=dict(defocus=1.4, dfdiff=0.05, dfang=20.0),
        outliers=[(30, 40, 25.0), (100, 300, -20.0), (400, 200, 12.0)],
        cfg=dict(angpix=1.0, phistep=30.0, kk=3.0, energy=300.0, cs=2.7, Highres=8.0, Lowres=200.0, diameter=48.0,
                 threshold=3.7, window_size=256, overlap=0, norm_type=1, invert=0, phase_flip=0)),
    "norm_1024x768_l256": dict(
        data=dict(shape=(768, 1024), n_templates=20, tsize=48, n_blobs=10, n_particles=8, amp=0.6, seed=12,
                  margin=40),
        ctf=dict(defocus=2.1, dfdiff=0.15, dfang=70.0),
        outliers=[(5, 5, 30.0), (700, 500, -30.0)],
        cfg=dict(angpix=1.2, phistep=30.0, kk=2.0, energy=300.0, cs=2.7, Highres=9.0, Lowres=150.0, diameter=40.0,
                 threshold=4.3, window_size=256, overlap=32, norm_type=1, invert=0, phase_flip=0)),
    "nonorm_768_l256": dict(
        data=dict(shape=(768, 768), n_templates=16, tsize=64, n_blobs=12, n_particles=6, amp=0.6, seed=13, margin=40),
        ctf=dict(defocus=1.6, dfdiff=0.0, dfang=0.0),
        outliers=[],
        cfg=dict(angpix=1.0, phistep=30.0, kk=3.0, energy=300.0, cs=2.7, Highres=8.0, Lowres=200.0, diameter=64.0,
                 threshold=7.3, window_size=256, overlap=64, norm_type=0, invert=0, phase_flip=0)),
    "nonorm_768_l256_flip": dict(
        data=dict(shape=(768, 768), n_templates=16, tsize=64, n_blobs=12, n_particles=6, amp=0.6, seed=14, margin=40),
        ctf=dict(defocus=1.6, dfdiff=0.1, dfang=45.0),
        outliers=[],
        cfg=dict(angpix=1.0, phistep=30.0, kk=3.0, energy=300.0, cs=2.7, Highres=8.0, Lowres=200.0, diameter=64.0,
                 threshold=7.6, window_size=256, overlap=64, norm_type=0, invert=1, phase_flip=1)),
    # the bench geometry's window (512, overlap 192: 3 x 3 windows on 1024^2)
    "norm_1024_l512": dict(
        data=dict(shape=(1024, 1024), n_templates=10, tsize=96, n_blobs=12, n_particles=8, amp=0.6, seed=15,
                  margin=60),
        ctf=dict(defocus=1.7, dfdiff=0.1, dfang=30.0),
        outliers=[(900, 40, 22.0)],
        cfg=dict(angpix=1.0, phistep=30.0, kk=3.0, energy=300.0, cs=2.7, Highres=8.0, Lowres=200.0, diameter=80.0,
                 threshold=THRESH["norm_1024_l512"], window_size=512, overlap=192, norm_type=1, invert=0,
                 phase_flip=0)),
    # the reference's default window 320 with overlap 120 (4 x 4 windows on 840^2)
    "norm_840_l320": dict(
        data=dict(shape=(840, 840), n_templates=16, tsize=48, n_blobs=10, n_particles=8, amp=0.6, seed=16,
                  margin=40),
        ctf=dict(defocus=1.5, dfdiff=0.05, dfang=60.0),
        outliers=[],
        cfg=dict(angpix=1.0, phistep=30.0, kk=3.0, energy=300.0, cs=2.7, Highres=8.0, Lowres=200.0, diameter=40.0,
                 threshold=THRESH["norm_840_l320"], window_size=320, overlap=120, norm_type=1, invert=0,
                 phase_flip=0)),
    # the tiled workload's geometry: 1024^2, 8 templates of 128^2, 10 degree steps, norm_type=0 in
    # 720^2 tiles, 512 windows with 128 px overlap
    "nonorm_1024_l512_t8": dict(
        data=dict(shape=(1024, 1024), n_templates=8, tsize=128, n_blobs=16, n_particles=12, amp=0.5, seed=17,
                  margin=60),
        ctf=dict(defocus=1.5, dfdiff=0.0, dfang=0.0),
        outliers=[],
        cfg=dict(angpix=1.0, phistep=10.0, kk=3.0, energy=300.0, cs=2.7, Highres=8.0, Lowres=200.0, diameter=100.0,
                 threshold=THRESH["nonorm_1024_l512_t8"], window_size=512, overlap=128, norm_type=0, invert=0,
                 phase_flip=0)),
    # the reference's defaults: norm_type=0, window 320, no overlap
    "nonorm_1024_l320": dict(
        data=dict(shape=(1024, 1024), n_templates=6, tsize=96, n_blobs=12, n_particles=10, amp=0.6, seed=18,
                  margin=60),
        ctf=dict(defocus=1.9, dfdiff=0.0, dfang=0.0),
        outliers=[],
        cfg=dict(angpix=1.0, phistep=30.0, kk=3.0, energy=300.0, cs=2.7, Highres=8.0, Lowres=200.0, diameter=70.0,
                 threshold=THRESH["nonorm_1024_l320"], window_size=320, overlap=0, norm_type=0, invert=0,
                 phase_flip=0)),
}


class _Ctf:
    def __init__(self, defocus, dfdiff, dfang):
        self.defocus, self.dfdiff, self.dfang = defocus, dfdiff, dfang


def case_inputs(name: str):
    """Bit-reproducible inputs of a case: (image float32 [ny, nx], templates float32 [n, t, t], CTF)."""
    spec = CASES[name]
    img, tmpl, _ = fixture_data.make_inputs(**spec["data"])
    for (x, y, v) in spec["outliers"]:
        img[y, x] = v
    return img, tmpl, _Ctf(**spec["ctf"])


def checksum(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def write_mrc(path: str, data: np.ndarray):
    data = np.ascontiguousarray(data, dtype="<f4")
    if data.ndim == 2:
        data = data[None]
    nz, ny, nx = data.shape
    hdr = np.zeros(256, dtype="<i4")
    hdr[0:4] = (nx, ny, nz, 2)
    hdr[7:10] = (nx, ny, nz)
    f = hdr.view("<f4")
    f[10:13] = (nx, ny, nz)
    f[13:16] = (90.0, 90.0, 90.0)
    hdr[16:19] = (1, 2, 3)
    f[19], f[20], f[21] = float(data.min()), float(data.max()), float(data.mean())
    hdr[52] = int.from_bytes(b"MAP ", "little")
    hdr[53] = 0x00004444
    with open(path, "wb") as fh:
        fh.write(hdr.tobytes())
        fh.write(data.tobytes())


def parse_line(line: str) -> dict:
    parts = line.rstrip("\n").split("\t")
    kv = {}
    for p in parts[2:]:
        k, v = p.split("=", 1)
        kv[k] = v
    e = [float(x) for x in kv["euler"].split(",")]
    cx, cy = (float(x) for x in kv["center"].split(","))
    return dict(index=int(parts[0]), path=parts[1], defocus=float(kv["defocus"]), dfdiff=float(kv["dfdiff"]),
                dfang=float(kv["dfang"]), euler1=e[0], euler2=e[1], angle=e[2], x=cx, y=cy, score=float(kv["score"]))


def run_case(name: str, ref_bin: str, workdir: str) -> dict:
    spec = CASES[name]
    img, tmpl, c = case_inputs(name)
    d = os.path.join(workdir, name)
    os.makedirs(d, exist_ok=True)
    write_mrc(os.path.join(d, "mic.mrc"), img)
    write_mrc(os.path.join(d, "tmpl.mrc"), tmpl)
    with open(os.path.join(d, "euler.txt"), "w") as fh:
        for j in range(tmpl.shape[0]):
            fh.write(f"{j}.0 0.0 0.0\n")
    with open(os.path.join(d, "mics.lst"), "w") as fh:
        fh.write("#LST\n")
        fh.write(f"0 {os.path.join(d, 'mic.mrc')} defocus={c.defocus} dfdiff={c.dfdiff} dfang={c.dfang}\n")
    cfg = dict(spec["cfg"])
    cfg.update(input=os.path.join(d, "mics.lst"), template=os.path.join(d, "tmpl.mrc"),
               eulerfile=os.path.join(d, "euler.txt"), output=os.path.join(d, "picks.txt"), first=0, last=1,
               GPU_ID=0)
    with open(os.path.join(d, "config"), "w") as fh:
        for k, v in cfg.items():
            fh.write(f"{k} = {v}\n")
    r = subprocess.run([ref_bin, os.path.join(d, "config")], cwd=d, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"{name}: reference exited {r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    with open(os.path.join(d, "picks.txt")) as fh:
        lines = [ln for ln in fh if ln.strip()]
    return dict(case=name, params=spec, checksum=checksum(img, tmpl), n_picks=len(lines),
                picks=[parse_line(ln) for ln in lines])


def main_sync_only(a, wd):
    """Adds to existing fixtures the pick list of the warp-safe test build (gisspa_ref_sync:
    kernels.cu compiled with -G by oracle/ref_build.sh), keeping their reference picks."""
    for name in a.cases:
        path = os.path.join(a.out, f"{name}.json")
        with open(path) as fh:
            g = json.load(fh)
        r = run_case(name, a.ref_sync, wd)
        assert r["checksum"] == g["checksum"]
        g["picks_sync"] = r["picks"]
        with open(path, "w") as fh:
            json.dump(g, fh, indent=0)
        print(f"{name}: {len(r['picks'])} picks from the warp-safe build")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--ref", default=os.path.join(REPO, "oracle", "_ref", "gisspa_ref"))
    ap.add_argument("--ref-sync", default=os.path.join(REPO, "oracle", "_ref", "gisspa_ref_sync"))
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    ap.add_argument("--sync-only", action="store_true",
                    help="only add the warp-safe build's picks to existing fixtures")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    with tempfile.TemporaryDirectory() as wd:
        if a.sync_only:
            return main_sync_only(a, wd)
        for name in a.cases:
            res = run_case(name, a.ref, wd)
            if CASES[name]["cfg"]["norm_type"] != 0 and os.path.exists(a.ref_sync):
                res["picks_sync"] = run_case(name, a.ref_sync, wd)["picks"]
            with open(os.path.join(a.out, f"{name}.json"), "w") as fh:
                json.dump(res, fh, indent=0)
            print(f"{name}: {res['n_picks']} reference picks")


if __name__ == "__main__":
    main()
