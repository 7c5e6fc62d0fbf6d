#!/usr/bin/env python
"""Throughput of the template-matching search on one node.

One step = the full search of one synthetic micrograph (default: 4096^2, 200
templates of 180^2, 72 in-plane angles, norm_type=1, 512 windows with 192 px
overlap) with the inputs resident in device memory.  Every rank searches its own
micrograph (micrographs are independent: replicas, no collective), so scaling is
weak and `value` is the whole-job micrographs/s.  `e2e` repeats the measurement
through gisspa_search with the micrograph in pinned host memory (host->device
copy and the pick read-back inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--form plain|fp16|topk|fp16_topk]

`--impl reference` times the reference algorithm's CPU restatement (the FP64
oracle; the reference itself has no CPU path) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "gisspa_v2.0_b200"))
import gisspa  # noqa: E402
import synth  # noqa: E402

METRIC = "micrographs/s and template-rotations/s vs plain FP32 path at ≤1e-3 score err"

FORMS = {
    "plain": dict(spectrum_precision=gisspa.SPEC_FP32, pick_mode=gisspa.PICK_CHUNK),
    "fp16": dict(spectrum_precision=gisspa.SPEC_FP16, pick_mode=gisspa.PICK_CHUNK),
    "topk": dict(spectrum_precision=gisspa.SPEC_FP32, pick_mode=gisspa.PICK_TOPK),
    "fp16_topk": dict(spectrum_precision=gisspa.SPEC_FP16, pick_mode=gisspa.PICK_TOPK),
}


def args_parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="whole_4096_t200",
                    choices=list(synth.WORKLOADS) + ["batch_c3", "project_c5", "adjoint_c4"])
    ap.add_argument("--batch-n", type=int, default=8,
                    help="batch_c3: micrographs per gisspa_search_batch call (the first n of the 32-micrograph batch)")
    ap.add_argument("--form", default="plain", choices=list(FORMS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-full-sweeps", action="store_true",
                    help="skip timing the plain form with every row of sweep 2 transformed (prune_sweep2=0)")
    ap.add_argument("--no-precision-check", action="store_true",
                    help="skip the untimed FP32 / BF16 top-K searches that measure the chosen form's score error")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="--impl reference: skip timing the reference's own CUDA build beside the oracle")
    ap.add_argument("--tensor-cores", type=int, default=0, choices=[0, 1],
                    help="1: run the FP16 forms' transforms on the tensor cores (tcgen05) instead of the CUDA cores")
    ap.add_argument("--eager", action="store_true",
                    help="launch every kernel from the host (cuda_graphs = 0), e.g. for per-launch profiling")
    ap.add_argument("--shape", type=int, default=-1,
                    help="with --batch: row-transform kernel shape (pass_b_shape) instead of the first")
    ap.add_argument("--a-shape", type=int, default=-1,
                    help="with --batch: column-transform kernel shape (pass_a_shape) instead of the first")
    ap.add_argument("--batch", default=None,
                    help="D,E: fix templates x windows per correlation launch instead of autotuning (profiling)")
    ap.add_argument("--chosen", default="fp16_topk", choices=list(FORMS) + ["none"],
                    help="with --form plain: also time this form on the same micrograph (reported as chosen_form)")
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of this rank's GPU during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ roofline
def measured_peak_hbm():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_bytes(L: int, spec: int, D: float):
    """Per (window, template-rotation) pair, split per kernel:
    B = H b_t + 2 H b_m + (H b_i + L^2 b_s) / D, H = L (L/2 + 1)."""
    H = L * (L // 2 + 1)
    b_t = 8 if spec == gisspa.SPEC_FP32 else 4
    b_m, b_i, b_s = 8, 8, 48
    pass_a = H * b_t + H * b_m + H * b_i / D
    pass_b = H * b_m + L * L * b_s / D
    return pass_a, pass_b


def traffic_from_profiles(kernel: str, spec: int, pairs_per_launch: float):
    """DRAM bytes per launch: the per-pair dram__bytes_read.sum + dram__bytes_write.sum of the
    committed ncu capture (profiles/ncu_traffic.json, warm caches, the bench workload with a
    fixed launch shape) times this run's pairs per launch; None when absent."""
    p = os.path.join(REPO, "profiles", "ncu_traffic.json")
    try:
        with open(p) as fh:
            t = json.load(fh)
    except Exception:
        return None
    key = f"{kernel}/{'fp32' if spec == gisspa.SPEC_FP32 else 'fp16'}"
    e = t.get(key) or t.get(kernel)
    return None if e is None else float(e["bytes_per_pair"]) * pairs_per_launch


# ------------------------------------------------------------------ CPU leg (the FP64 oracle)
def oracle_rate(case, cfg, n_angles: int):
    """Micrograph time of the FP64 oracle on the host cores, from two bounded samples of the
    same workload (4 and 10 templates at one angle, ~20 s of CPU work): slope = cost of one
    template-rotation over all windows (both sweeps), intercept = per-micrograph preparation.
    The oracle keeps the rotated template spectra of an angle (4 MB each at 512^2) and reads
    them for every window: a sample of only 1-3 templates stays in the CPU caches and would
    understate the cost of the full 200 (800 MB); at 4-10 templates the slope is measured
    mostly outside them (any remaining bias makes the CPU look faster)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle

    ctf = gisspa.Ctf(case.defocus, case.dfdiff, case.dfang)
    t = []
    lo, hi = 4, 10
    for nts in (lo, hi):
        t0 = time.perf_counter()
        oracle.search(cfg, ctf, case.image, case.templates, max_templates=nts, max_angles=1)
        t.append(time.perf_counter() - t0)
    per_rot = max((t[1] - t[0]) / (hi - lo), 1e-9)
    prep = max(t[0] - lo * per_rot, 0.0)
    nt = case.templates.shape[0]
    mic_s = prep + per_rot * nt * n_angles
    return 1.0 / mic_s, oracle.num_threads(), sum(t), per_rot, prep


def precision_check(case, ctf, d_img, nx, ny, wl, chosen_name, chosen_picks, local, out) -> dict:
    """Peak-score error of the reduced-precision template forms against the FP32 form of the
    same one-sweep top-K search on the same micrograph (untimed): the picks of the timed chosen
    form and of one BF16 search, each matched to the FP32 picks by (x, y, template, angle)."""
    def run(spec):
        p = dict(synth.SEARCH_PARAMS[wl])
        p.update(spectrum_precision=spec, pick_mode=gisspa.PICK_TOPK)
        s = gisspa.Searcher(gisspa.Config.default(**p), local)
        s.set_templates(case.templates)
        n = s.search_device(d_img.data_ptr(), nx, ny, ctf, out)
        s.close()
        return out[:n].copy()

    ref = run(gisspa.SPEC_FP32)
    key = lambda q: (float(q["x"]), float(q["y"]), int(q["template_id"]), int(q["angle_index"]))
    R = {key(q): float(q["score"]) for q in ref}
    res = {"picks_fp32": len(ref)}
    for name, picks in ((chosen_name, chosen_picks), ("bf16_topk", run(gisspa.SPEC_BF16))):
        rel = [abs(float(q["score"]) - R[key(q)]) / abs(R[key(q)]) for q in picks if key(q) in R]
        res[name] = {"picks": len(picks), "same_picks": len(rel),
                     "max_rel": float(max(rel)) if rel else None,
                     "p99_rel": float(np.quantile(rel, 0.99)) if rel else None,
                     "median_rel": float(np.median(rel)) if rel else None}
    return res


def reference_cuda_timing(wl: str) -> dict:
    """The reference's own CUDA build (its unmodified search sources, cuFFT, compiled for sm_100a
    by oracle/ref_build.sh into oracle/_ref/gisspa_ref) beside this library's drop-in driver
    gisspa_main on the same MRC / config / LST / Euler files of the workload, on this GPU: whole
    process wall times for one and two micrographs, whose difference is the steady cost of one
    micrograph (reference: norm.cu / nonorm.cu with cuFFT; ours: the C-ABI search)."""
    ref_bin = os.path.join(REPO, "oracle", "_ref", "gisspa_ref")
    ours_bin = os.path.join(REPO, "gisspa_v2.0_b200", "_build", "gisspa_main")
    if not os.path.exists(ref_bin):
        return {"unavailable": "oracle/_ref/gisspa_ref not built (the reference sources were absent at build time)"}
    try:
        import torch

        if not torch.cuda.is_available():
            return {"unavailable": "no GPU visible"}
    except Exception as e:  # noqa: BLE001
        return {"unavailable": f"torch: {e}"}
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ref_time

    # the reference once (about 30 s per micrograph); the driver, whose seconds make the
    # difference of two process wall times noisy, as the fastest of three runs of each list
    r = ref_time.time_binaries(wl, {"reference": ref_bin})
    r.update(ref_time.time_binaries(wl, {"ours": ours_bin}, repeat=3))
    ref_s = r["reference"]["s_per_micrograph"]
    ours_s = r["ours"]["s_per_micrograph"]
    return {"value": 1.0 / ref_s, "unit": "micrographs/s", "s_per_micrograph": ref_s,
            "s_setup": r["reference"]["s_setup"], "picks": r.get("reference_picks"),
            "ours_gisspa_main": {"value": 1.0 / ours_s, "s_per_micrograph": ours_s, "s_setup": r["ours"]["s_setup"],
                                 "picks": r.get("ours_picks")},
            "speedup_per_micrograph": ref_s / ours_s,
            "timing": "same B200, same files and config: t(2 micrographs) - t(1 micrograph), whole process "
                      "(the driver's as the fastest of three runs of each)"}


# ------------------------------------------------------------------ batching workload
def bench_batch(a, rank: int, world: int, local: int):
    """One step = one gisspa_search_batch call over n uneven micrographs (2048^2, 3710x3838,
    4096^2, 4092x5760 in turn, each with its own CTF) from host memory, 500 templates of 200^2,
    120 angles: the batching form (uneven sizes, per-micrograph CTF, graph-replayed angles)."""
    import torch

    if world > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    cases = [synth.make_case(**c) for c in synth.batch_cases(n=a.batch_n, seed=3 + 100 * rank)]
    forms = [a.form] + ([a.chosen] if a.form == "plain" and a.chosen not in ("none", "plain") else [])
    res_forms = {}
    for form in forms:
        params = dict(synth.SEARCH_PARAMS["batch_c3"])
        params.update(FORMS[form])
        cfg = gisspa.Config.default(**params)
        s = gisspa.Searcher(cfg, local)
        s.set_templates(cases[0].templates)
        imgs = [c.image for c in cases]
        ctfs = [gisspa.Ctf(c.defocus, c.dfdiff, c.dfang) for c in cases]
        for _ in range(a.warmup):
            s.search_batch(imgs, ctfs)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(a.steps):
            picks = s.search_batch(imgs, ctfs)
        ev1.record()
        torch.cuda.synchronize()
        t = torch.tensor([ev0.elapsed_time(ev1)], device=dev)
        if world > 1:
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
        st = s.stats()
        n_rot = cases[0].templates.shape[0] * int(math.ceil(360.0 / cfg.phistep - 1e-9))
        res_forms[form] = {"value": world * a.steps * len(cases) / (ms / 1000.0), "ms_per_step": ms / a.steps,
                           "template_rotations_per_s": world * a.steps * len(cases) * n_rot / (ms / 1000.0),
                           "pairs_per_step": int(st.pairs), "picks_per_step": int(sum(len(p) for p in picks)),
                           "gpu_launches": int(st.kernel_launches)}
        s.close()
    if rank == 0:
        main_form = res_forms[a.form]
        res = {"metric": METRIC, "value": main_form["value"], "unit": "micrographs/s", "n_gpus": world,
               "steps": a.steps, "warmup": a.warmup, "ms_per_step": main_form["ms_per_step"],
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded Gaussian-blob projections planted in N(0,1) noise)",
               "config": {"workload": "batch_c3", "form": a.form, "micrographs_per_step": len(cases),
                          "sizes": [list(c.image.shape) for c in cases], "templates": 500, "template_size": 200,
                          "angles": 120, "window_size": 512, "overlap": 200, "norm_type": 1,
                          "parallelism": f"replicas{world}", "entry": "gisspa_search_batch (host images)"},
               "forms": res_forms}
        if len(forms) > 1:
            res["chosen_form"] = {"form": forms[1], **res_forms[forms[1]],
                                  "vs_plain": res_forms[forms[1]]["value"] / main_form["value"]}
        print(json.dumps(res))
    if world > 1:
        torch.distributed.destroy_process_group()


# ------------------------------------------------------------------ differentiation workload
def bench_adjoint(a, rank: int, local: int):
    """Picks of the 4096^2 workload (200 templates of 180^2, 72 angles) with one top-K sweep
    (K = 10,000, exclusion radius 16 px) in the FP32 and the BF16 template form; then per step,
    for each form: the batched adjoint of all 10,000 picks (score and gradient in dx, dy, theta,
    dfu, dfv, dfang; one call) and 20 steps of batched gradient-ascent refinement of the picks
    and the micrograph CTF (one call).  The search itself is set-up, outside the timed region.
    A sample of 32 picks is checked against central differences (h = 1e-3 px / degree) of the
    library's own scores."""
    import torch

    torch.cuda.set_device(local)
    wl = "whole_4096_t200"
    case = synth.make_case(**synth.WORKLOADS[wl])
    ctf = gisspa.Ctf(case.defocus, case.dfdiff, case.dfang)
    res_forms = {}
    for form, spec in (("fp32", gisspa.SPEC_FP32), ("bf16", gisspa.SPEC_BF16)):
        params = dict(synth.SEARCH_PARAMS[wl])
        params.update(spectrum_precision=spec, pick_mode=gisspa.PICK_TOPK, topk=10000, exclusion_radius=16.0,
                      threshold=0.0)
        s = gisspa.Searcher(gisspa.Config.default(**params), local)
        s.set_templates(case.templates)
        picks = s.search(case.image, ctf)
        n = len(picks)
        for _ in range(a.warmup):
            s.score_grad(picks)
        torch.cuda.synchronize()
        tg, tr = [], []
        for _ in range(a.steps):
            t0 = time.perf_counter()
            g = s.score_grad(picks)
            tg.append(time.perf_counter() - t0)
            t0 = time.perf_counter()
            refined, c2, _ = s.refine(picks, steps=20, ctf=gisspa.Ctf(ctf.defocus, ctf.dfdiff, ctf.dfang))
            tr.append(time.perf_counter() - t0)
        # central differences of the library's scores on a sample of the picks
        smp = picks[:: max(1, n // 32)][:32]
        base = np.stack([np.full(len(smp), 0.21), np.full(len(smp), -0.17), smp["theta"] + 0.9], 1).astype(np.float32)
        gb = s.score_grad(smp, base)
        adj = np.stack([gb["d_dx"], gb["d_dy"], gb["d_theta"]], 1).astype(np.float64)
        fd = np.zeros_like(adj)
        for k in range(3):
            d = np.zeros_like(base)
            d[:, k] = 1e-3
            hi, lo = base + d, base - d
            step = hi[:, k].astype(np.float64) - lo[:, k].astype(np.float64)
            fd[:, k] = (s.score_grad(smp, hi)["score"].astype(np.float64) -
                        s.score_grad(smp, lo)["score"].astype(np.float64)) / step
        rel = np.linalg.norm(adj - fd, axis=1) / np.maximum(np.linalg.norm(fd, axis=1), 1e-6)
        res_forms[form] = {"picks": n, "grad_ms": 1000 * float(np.median(tg)), "refine20_ms": 1000 * float(np.median(tr)),
                           "grad_picks_per_s": n / float(np.median(tg)),
                           "refine_us_per_pick_step": 1e6 * float(np.median(tr)) / (20 * n),
                           "mean_score_before": float(picks["score"].mean()),
                           "mean_score_after": float(refined["score"].mean()),
                           "ctf_after": [c2.defocus, c2.dfdiff, c2.dfang],
                           "fd_check": {"picks": len(smp), "h": 1e-3, "median_rel": float(np.median(rel)),
                                        "p90_rel": float(np.quantile(rel, 0.9)), "max_rel": float(rel.max())}}
        s.close()
    main = res_forms["fp32"]
    res = {"metric": "picks/s of the batched adjoint (score + 6 gradients) on 10,000 picks", "value":
           main["grad_picks_per_s"], "unit": "picks/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": main["grad_ms"] + main["refine20_ms"], "higher_is_better": True, "dtype": "f32 (f64 sums)",
           "data": "synthetic (seeded Gaussian-blob projections planted in N(0,1) noise)",
           "config": {"workload": "adjoint_c4", "picks_from": wl, "topk": 10000, "exclusion_radius": 16,
                      "refine_steps": 20, "timing": "host wall clock around each synchronous C-ABI call"},
           "forms": res_forms}
    if rank == 0:
        print(json.dumps(res))


# ------------------------------------------------------------------ template generation workload
def bench_project(a, rank: int, local: int):
    """One step = the 1000 projections of 256^2 that the 8192^2 workload searches, made from a
    256^3 map (seeded Gaussian blobs) through gisspa_project: host volume in, host stack out."""
    import torch

    torch.cuda.set_device(local)
    rng = np.random.default_rng(9 + rank)
    size, n = 256, 1000
    zz, yy, xx = np.mgrid[0:size, 0:size, 0:size].astype(np.float32)
    vol = np.zeros((size, size, size), np.float32)
    for c, sg in zip(rng.uniform(0.3 * size, 0.7 * size, (40, 3)), rng.uniform(3.0, 8.0, 40)):
        vol += np.exp(-((xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2) / (2 * sg * sg)).astype(np.float32)
    angles = rng.uniform(0.0, 2 * np.pi, (n, 3)).astype(np.float32)
    params = dict(synth.SEARCH_PARAMS["whole_8192_t1000"])
    s = gisspa.Searcher(gisspa.Config.default(**params), local)
    for _ in range(a.warmup):
        s.project(vol, angles)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        s.project(vol, angles)
    el = time.perf_counter() - t0
    value = a.steps * n / el
    res = {"metric": "projections/s (template generation, emdata::project3d semantics)", "value": value,
           "unit": "projections/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
           "ms_per_step": 1000.0 * el / a.steps, "higher_is_better": True, "dtype": "f32 (f64 z-interpolation)",
           "data": "synthetic 256^3 Gaussian-blob map, uniform random Euler angles",
           "config": {"workload": "project_c5", "volume": [size] * 3, "projections": n,
                      "timing": "host wall clock around gisspa_project (volume H2D, projections D2H inside)"}}
    if not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle

        k = 16
        t0 = time.perf_counter()
        oracle.project3d(vol, angles[:k])
        cpu = k / (time.perf_counter() - t0)
        res["cpu_baseline"] = {"value": cpu, "unit": "projections/s", "cores": oracle.num_threads(), "kind": "port",
                               "sample": f"oracle restatement (bit-identical to the reference's project3d), {k} projections"}
    s.close()
    if rank == 0:
        print(json.dumps(res))


# ------------------------------------------------------------------ main
def same_picks(a: np.ndarray, b: np.ndarray) -> dict:
    """Two pick lists of one micrograph: whether they hold the same (x, y, template, angle) picks,
    and the largest relative score difference between matching picks (two searches may tune
    different launch shapes, whose rounding differs in the last bits)."""
    key = lambda p: (float(p["x"]), float(p["y"]), int(p["template_id"]), int(p["angle_index"]))
    da = {key(p): float(p["score"]) for p in a}
    db = {key(p): float(p["score"]) for p in b}
    common = set(da) & set(db)
    rel = max((abs(da[k] - db[k]) / max(abs(db[k]), 1e-30) for k in common), default=0.0)
    return {"n": [len(a), len(b)], "same": len(a) == len(b) and set(da) == set(db), "max_rel_score_diff": rel}


def main():
    a = args_parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    wl = a.workload
    if wl in ("batch_c3", "project_c5", "adjoint_c4") and a.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": f"{wl}: the reference arm (the FP64 oracle on the "
                              "host cores) is timed on the single-micrograph workloads only"}))
        return
    if wl == "batch_c3":
        return bench_batch(a, rank, world, local)
    if wl == "project_c5":
        return bench_project(a, rank, local)
    if wl == "adjoint_c4":
        return bench_adjoint(a, rank, local)
    params = dict(synth.SEARCH_PARAMS[wl])
    params.update(FORMS[a.form])
    if a.batch:
        params["template_batch"], params["window_batch"] = (int(x) for x in a.batch.split(","))
        params["pass_b_shape"] = a.shape
        params["pass_a_shape"] = a.a_shape
    if a.eager:
        params["cuda_graphs"] = 0
    params["tensor_cores"] = a.tensor_cores
    cfg = gisspa.Config.default(**params)
    angles = int(math.ceil(360.0 / cfg.phistep - 1e-9))
    data = dict(synth.WORKLOADS[wl])
    config_desc = {"workload": wl, "form": a.form, "image": list(data["shape"]), "templates": data["n_templates"],
                   "template_size": data["tsize"], "angles": angles, "window_size": cfg.window_size,
                   "overlap": cfg.overlap, "norm_type": cfg.norm_type, "parallelism": f"replicas{world}",
                   "l2": "working set > 1 GB per step (larger than L2)"}

    if a.impl == "reference":
        if rank != 0:
            return
        case = synth.make_case(**data)
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle

        ctf0 = gisspa.Ctf(case.defocus, case.dfdiff, case.dfang)
        for _ in range(a.warmup):  # warm-up: threads and caches (one template at one angle)
            oracle.search(cfg, ctf0, case.image, case.templates, max_templates=1, max_angles=1)
        steps, step_s = [], []
        for i in range(a.steps):
            t0 = time.perf_counter()
            steps.append(oracle_rate(case, cfg, angles))
            step_s.append(time.perf_counter() - t0)
        rate = float(np.mean([s[0] for s in steps]))
        cores = steps[0][1]
        sample = (f"FP64 oracle, {wl}: 4 and 10 templates x 1 angle over all windows (both sweeps), "
                  f"extrapolated linearly to {data['n_templates']} templates x {angles} angles")
        line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "micrographs/s",
                "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "higher_is_better": True,
                "template_rotations_per_s": rate * data["n_templates"] * angles,
                "ms_per_step": 1000.0 * float(np.mean(step_s)),
                "ms_per_step_is": "host wall time of one step's bounded sample (value is extrapolated from it)",
                "extrapolated": True, "extrapolated_ms_per_micrograph": 1000.0 / rate,
                "dtype": "f64", "data": "synthetic", "config": config_desc,
                "cpu_baseline": {"value": rate, "unit": "micrographs/s", "cores": cores, "kind": "port",
                                 "sample": sample, "extrapolated": True, "sample_s": float(np.mean(step_s))},
                "e2e": {"value": rate, "unit": "micrographs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        if not a.no_reference_cuda:
            line["reference_cuda"] = reference_cuda_timing(wl)
        print(json.dumps(line))
        return

    import torch

    if world > 1:
        import datetime

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    case = synth.make_case(**{**data, "seed": data["seed"] + 1000 * rank})
    s = gisspa.Searcher(cfg, local)
    s.set_templates(case.templates)
    ny, nx = case.image.shape
    d_img = torch.from_numpy(case.image).to(dev)
    out = np.zeros(1 << 22, dtype=gisspa.PICK_DTYPE)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(a.warmup):
        s.search_device(d_img.data_ptr(), nx, ny, gisspa.Ctf(case.defocus, case.dfdiff, case.dfang), out)
    torch.cuda.synchronize()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    smi_index = int(vis.split(",")[local]) if vis and vis.split(",")[local].strip().isdigit() else local
    clocks = ClockSampler(smi_index)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    launches, npicks, stats = 0, 0, []
    ctf = gisspa.Ctf(case.defocus, case.dfdiff, case.dfang)
    for _ in range(a.steps):
        npicks = s.search_device(d_img.data_ptr(), nx, ny, ctf, out)
        st = s.stats()
        launches += st.kernel_launches
        stats.append(st)
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    t = torch.tensor([ms], device=dev)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * a.steps / (ms_max / 1000.0)

    e2e = None
    if not a.no_e2e:
        host = torch.from_numpy(case.image).pin_memory()
        himg = host.numpy()
        s.search(himg, ctf)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n_e2e = 0
        for _ in range(a.steps):
            picks = s.search(himg, ctf)
            n_e2e = len(picks)
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        te = torch.tensor([el], device=dev)
        if world > 1:
            torch.distributed.all_reduce(te, op=torch.distributed.ReduceOp.MAX)
        e2e = {"value": world * a.steps / float(te.item()), "unit": "micrographs/s",
               "h2d_bytes_per_step": int(nx * ny * 4), "d2h_bytes_per_step": int(n_e2e * gisspa.PICK_DTYPE.itemsize),
               "timing": "host wall clock around the synchronous C-ABI call, max over ranks"}

    # roofline of the dominant kernel: the correlation launch pair (pass A + pass B, which run
    # back to back with programmatic dependent launch), timed by CUDA events around whole runs
    # of launch pairs inside the timed steps (nothing recorded between the two passes)
    t_pair = float(np.mean([x.corr_pair_us for x in stats]))
    ppl = float(np.mean([x.pairs_per_launch for x in stats]))
    dpl = float(np.mean([x.templates_per_launch for x in stats]))
    ba, bb = algorithmic_bytes(cfg.window_size, cfg.spectrum_precision, max(dpl, 1.0))
    peak, peak_kind = measured_peak_hbm()
    alg = (ba + bb) * ppl
    achieved = alg / (t_pair * 1e-6) / 1e9 if t_pair > 0 else 0.0
    tuned = cfg.window_size in (256, 320, 512, 1024)
    # the committed per-pair DRAM bytes describe the hand-tuned kernels; window sizes without
    # them run the generic column / row kernels
    tr = None
    if cfg.window_size == 512:  # the committed DRAM bytes were captured at window 512
        ta_ = traffic_from_profiles("pass_a", cfg.spectrum_precision, ppl)
        tb_ = traffic_from_profiles("pass_b", cfg.spectrum_precision, ppl)
        tr = ta_ + tb_ if ta_ is not None and tb_ is not None else None
    kern = "pass_a+pass_b" if tuned else "generic_cols+generic_rows"
    timed_pairs = int(sum(x.corr_timed_launches for x in stats))
    roofline = {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": tr,
                "bytes_per_launch": alg, "bytes_per_pair": ba + bb, "launch_us": t_pair,
                "pairs_per_launch": ppl, "templates_per_launch": dpl, "timed_launch_pairs": timed_pairs,
                "launch_pairs_per_step": int(round(stats[-1].pairs / max(ppl, 1e-9))),
                "pass_b_variant": int(stats[-1].pass_b_variant), "pass_a_variant": int(stats[-1].pass_a_variant),
                "timing": "CUDA events around each host-launched angle's run of launch pairs (first angle of "
                          "each sweep; a pruned second sweep, which skips rows, is left out), on the "
                          "launching stream, inside the timed steps"}

    # the plain form again with every row of sweep 2 transformed (prune_sweep2 = 0): the same
    # picks, the work of two full sweeps
    full = None
    if a.form == "plain" and cfg.norm_type == 1 and cfg.pick_mode == gisspa.PICK_CHUNK and not a.no_full_sweeps:
        pruned_picks = out[:npicks].copy()
        s3 = gisspa.Searcher(cfg.copy(prune_sweep2=0), local)
        s3.set_templates(case.templates)
        for _ in range(a.warmup):
            s3.search_device(d_img.data_ptr(), nx, ny, ctf, out)
        barrier()
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(a.steps):
            n3 = s3.search_device(d_img.data_ptr(), nx, ny, ctf, out)
        ev1.record()
        torch.cuda.synchronize()
        barrier()
        t3 = torch.tensor([ev0.elapsed_time(ev1)], device=dev)
        if world > 1:
            torch.distributed.all_reduce(t3, op=torch.distributed.ReduceOp.MAX)
        full = {"value": world * a.steps / (float(t3.item()) / 1000.0), "unit": "micrographs/s",
                "ms_per_step": float(t3.item()) / a.steps, "picks_per_step": int(n3),
                "same_picks_as_pruned": same_picks(out[:n3], pruned_picks),
                "stage_ms": {"sweep1": s3.stats().ms_sweep1, "sweep2": s3.stats().ms_sweep2}}
        s3.close()

    # the chosen form on the same micrograph: FP16 spectra, one top-K sweep (the numerator of
    # the target ratio against the plain FP32 two-sweep form timed above)
    chosen = None
    if a.form == "plain" and a.chosen not in ("none", "plain"):
        p2 = dict(synth.SEARCH_PARAMS[wl])
        p2.update(FORMS[a.chosen])
        p2["tensor_cores"] = a.tensor_cores
        s2 = gisspa.Searcher(gisspa.Config.default(**p2), local)
        s2.set_templates(case.templates)
        for _ in range(a.warmup):
            s2.search_device(d_img.data_ptr(), nx, ny, ctf, out)
        barrier()
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(a.steps):
            n2 = s2.search_device(d_img.data_ptr(), nx, ny, ctf, out)
        ev1.record()
        torch.cuda.synchronize()
        barrier()
        t2 = torch.tensor([ev0.elapsed_time(ev1)], device=dev)
        if world > 1:
            torch.distributed.all_reduce(t2, op=torch.distributed.ReduceOp.MAX)
        v2 = world * a.steps / (float(t2.item()) / 1000.0)
        st2 = s2.stats()
        chosen_picks = out[:n2].copy()
        chosen = {"form": a.chosen, "value": v2, "unit": "micrographs/s", "ms_per_step": float(t2.item()) / a.steps,
                  "vs_plain": v2 / value, "vs_plain_full_sweeps": v2 / full["value"] if full else None,
                  "picks_per_step": int(n2), "launch_pair_us": st2.corr_pair_us,
                  "pairs_per_launch": st2.pairs_per_launch}
        s2.close()
        if not a.no_precision_check:
            chosen["score_err_vs_fp32"] = precision_check(case, ctf, d_img, nx, ny, wl, a.chosen, chosen_picks, local,
                                                          out)

    res = None
    if rank == 0:
        res = {"metric": METRIC, "value": value, "unit": "micrographs/s", "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32" if cfg.spectrum_precision == 0 else "f16-spectra/f32",
               "data": "synthetic (seeded Gaussian-blob projections planted in N(0,1) noise)",
               "config": config_desc,
               "template_rotations_per_s": value * data["n_templates"] * angles,
               "pairs_per_step": int(stats[-1].pairs), "picks_per_step": int(npicks),
               "stage_ms": {"prep": stats[-1].ms_prep, "sweep1": stats[-1].ms_sweep1,
                            "sweep2": stats[-1].ms_sweep2, "pick": stats[-1].ms_pick},
               "gpu_launches": int(launches), "graph_replays": int(stats[-1].graph_replays), "clocks": clk,
               "roofline": roofline, "e2e": e2e, "rows_alive": float(stats[-1].rows_alive),
               "pairs_alive": float(stats[-1].pairs_alive),
               "plain_full_sweeps": full}
        if chosen is not None:
            res["chosen_form"] = chosen
        if world == 1 and not a.no_cpu_baseline:
            rate, cores, secs, per_rot, prep = oracle_rate(case, cfg, angles)
            res["cpu_baseline"] = {"value": rate, "unit": "micrographs/s", "cores": cores, "kind": "port",
                                   "sample": f"FP64 oracle, 4 and 10 templates x 1 angle over all windows "
                                             f"({secs:.1f} s), extrapolated to the full workload",
                                   "extrapolated": True, "sample_s": secs}
        print(json.dumps(res))
    s.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
