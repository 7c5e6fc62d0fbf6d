"""Times the reference's own CUDA build and this library's drop-in driver on the same files.

MEASUREMENT INFRASTRUCTURE, run on a GPU machine.  ``oracle/_ref/gisspa_ref`` is the
reference's search compiled from its unmodified sources by ``oracle/ref_build.sh`` (cuFFT,
its own kernels and host scans); ``gisspa_v2.0_b200/_build/gisspa_main`` is this library's
command-line driver with the reference's interface (``main <config>``, main.cu:14-97).

For a bench workload this script writes its seeded synthetic inputs (the same generator and
seed as ``bench.py``) as MRC files with the reference's config / LST / Euler files, then runs
each binary twice: on a list holding the micrograph once and twice.  The difference of the
two wall times is the steady per-micrograph cost (process start, file reads, plans and
template loading cancel); the remainder is reported as set-up.  It prints one JSON line
with both figures per binary and the pick counts of the one-micrograph runs.

    python oracle/ref_time.py --workload whole_4096_t200
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "gisspa_v2.0_b200"))
sys.path.insert(0, os.path.join(REPO, "tests", "golden"))
import synth  # noqa: E402
from make_golden import write_mrc  # noqa: E402

# reference config keys for the bench parameter names (DataReader2.h:20-43)
KEYS = {"highres": "Highres", "lowres": "Lowres"}


def write_inputs(d: str, wl: str) -> tuple[str, str]:
    case = synth.make_case(**synth.WORKLOADS[wl])
    write_mrc(os.path.join(d, "mic.mrc"), case.image)
    write_mrc(os.path.join(d, "tmpl.mrc"), case.templates)
    with open(os.path.join(d, "euler.txt"), "w") as fh:
        for e in case.euler:
            fh.write(f"{float(e[0])} {float(e[1])} {float(e[2])}\n")
    lsts = []
    for n in (1, 2):
        p = os.path.join(d, f"mics{n}.lst")
        with open(p, "w") as fh:
            fh.write("#LST\n")
            for i in range(n):
                fh.write(f"{i} {os.path.join(d, 'mic.mrc')} defocus={case.defocus} dfdiff={case.dfdiff} "
                         f"dfang={case.dfang}\n")
        lsts.append(p)
    return lsts[0], lsts[1]


def write_config(path: str, wl: str, d: str, lst: str, n: int, out: str):
    cfg = {KEYS.get(k, k): v for k, v in synth.SEARCH_PARAMS[wl].items()}
    cfg.update(input=lst, template=os.path.join(d, "tmpl.mrc"), eulerfile=os.path.join(d, "euler.txt"),
               output=out, first=0, last=n, GPU_ID=0, invert=0, phase_flip=0)
    with open(path, "w") as fh:
        for k, v in cfg.items():
            fh.write(f"{k} = {v}\n")


def run(binary: str, config: str, cwd: str, timeout: float) -> float:
    t0 = time.perf_counter()
    r = subprocess.run([binary, config], cwd=cwd, capture_output=True, text=True, timeout=timeout)
    el = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"{binary} exited {r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    return el


def time_binaries(wl: str, binaries: dict, timeout: float = 900.0, single: bool = False, repeat: int = 1) -> dict:
    """Per-micrograph and set-up wall time of each binary ({name: path}) on the workload's files
    (single: one run on a one-micrograph list, whose time includes the set-up)."""
    res = {"workload": wl, "params": synth.SEARCH_PARAMS[wl], "repeat": repeat,
           "timing": ("wall clock of the whole process on one micrograph (set-up included)" if single else
                      "wall clock of the whole process; per_micrograph = t(2 micrographs) - t(1)")}
    with tempfile.TemporaryDirectory() as d:
        lst1, lst2 = write_inputs(d, wl)
        for name, binary in binaries.items():
            t = {}
            for n, lst in ((1, lst1),) + (() if single else ((2, lst2),)):
                cfg = os.path.join(d, f"config_{name}_{n}")
                out = os.path.join(d, f"picks_{name}_{n}.txt")
                write_config(cfg, wl, d, lst, n, out)
                t[n] = min(run(binary, cfg, d, timeout) for _ in range(max(1, repeat)))
                if n == 1:
                    with open(out) as fh:
                        res[f"{name}_picks"] = sum(1 for ln in fh if ln.strip())
            res[name] = ({"s_1_micrograph": t[1]} if single else
                         {"s_1_micrograph": t[1], "s_2_micrographs": t[2], "s_per_micrograph": t[2] - t[1],
                          "s_setup": 2 * t[1] - t[2]})
            print(json.dumps({name: res[name]}), file=sys.stderr, flush=True)
    if "reference" in res and "ours" in res:
        k = "s_1_micrograph" if single else "s_per_micrograph"
        res["speedup_per_micrograph"] = res["reference"][k] / res["ours"][k]
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="whole_4096_t200", choices=list(synth.WORKLOADS))
    ap.add_argument("--ref", default=os.path.join(HERE, "_ref", "gisspa_ref"))
    ap.add_argument("--ours", default=os.path.join(REPO, "gisspa_v2.0_b200", "_build", "gisspa_main"))
    ap.add_argument("--timeout", type=float, default=900.0)
    ap.add_argument("--single", action="store_true", help="one run on one micrograph (set-up included)")
    ap.add_argument("--repeat", type=int, default=1, help="runs of each list; the fastest counts")
    a = ap.parse_args()
    print(json.dumps(time_binaries(a.workload, {"reference": a.ref, "ours": a.ours}, a.timeout, a.single, a.repeat)))


if __name__ == "__main__":
    main()
