"""Pin the oracle (CPU) and the CUDA path (GPU) to pick lists printed by the reference
build itself (tests/golden/*.json, made by tests/golden/make_golden.py)."""
import glob
import json
import os

import numpy as np
import pytest

import gisspa
import make_golden
import oracle
from parity import config_from

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.json")))
# Tolerances against the reference's printed scores (six decimals, FP32 arithmetic):
#  * norm_type=0 without phase flip: every stage is well defined and the FP64 oracle agrees
#    with the reference to 2e-6 relative; pinned at 2e-5.
#  * norm_type=1: the reference normalises every rotated template by a mean and variance from
#    compute_sum_sqr (kernels.cu:384-443), whose warp-synchronous tail has no volatile or
#    __syncwarp (kernels.cu:423-436), so on Volta and later its sums are undefined.  The mean
#    leaves a DC residue and the variance a per-template scale inside the per-pixel mean and
#    sigma, so the printed z-scores carry that error (measured up to 3e-3 relative here; the
#    oracle uses exact sums, as does the CUDA path).  Picks within the tolerance band of the
#    threshold may appear on one side only.
#  * norm_type=0 with phase flip: 2e-4 measured, 1e-3 allowed.
REF_RTOL = {"nonorm_768_l256": 2e-5, "nonorm_768_l256_flip": 1e-3}
REF_RTOL_DEFAULT = 5e-3
REF_ATOL = 2e-6


def load(path):
    with open(path) as fh:
        return json.load(fh)


def case_setup(g):
    img, tmpl, c = make_golden.case_inputs(g["case"])
    assert make_golden.checksum(img, tmpl) == g["checksum"], "regenerated inputs differ from the golden inputs"
    cfg = config_from(g["params"]["cfg"])
    ctf = gisspa.Ctf(c.defocus, c.dfdiff, c.dfang)
    return img, tmpl, ctf, cfg


def ref_rows(g):
    """(template, printed angle, x, y) -> score for the reference picks."""
    rows = {}
    for p in g["picks"]:
        rows.setdefault((int(round(p["euler1"])), round(p["angle"], 3), round(p["x"], 3), round(p["y"], 3)), []).append(
            p["score"])
    return rows


def our_rows(picks):
    rows = {}
    for p in picks:
        rows.setdefault((int(p["template_id"]), round(float(p["angle"]), 3), round(float(p["x"]), 3),
                         round(float(p["y"]), 3)), []).append(float(p["score"]))
    return rows


def check_against_reference(g, picks, thresh):
    rtol = REF_RTOL.get(g["case"], REF_RTOL_DEFAULT)
    R, O = ref_rows(g), our_rows(picks)
    band = rtol * abs(thresh) + REF_ATOL
    missing = [k for k, v in R.items() if k not in O and max(v) >= thresh + band]
    extra = [k for k, v in O.items() if k not in R and max(v) >= thresh + band]
    bad = []
    for k in set(R) & set(O):
        a, b = sorted(R[k]), sorted(O[k])
        if len(a) == len(b) and not np.allclose(a, b, rtol=rtol, atol=REF_ATOL + 5e-7):
            bad.append((k, a, b))
    return missing, extra, bad


@pytest.mark.skipif(not GOLDEN, reason="no golden fixtures")
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-5] for p in GOLDEN])
def test_oracle_matches_reference_picks(path):
    g = load(path)
    img, tmpl, ctf, cfg = case_setup(g)
    picks = oracle.search(cfg, ctf, img, tmpl)
    missing, extra, bad = check_against_reference(g, picks, cfg.threshold)
    assert not missing and not extra and not bad, (missing[:5], extra[:5], bad[:5])
    assert g["n_picks"] > 0


@pytest.mark.gpu
@pytest.mark.skipif(not GOLDEN, reason="no golden fixtures")
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-5] for p in GOLDEN])
def test_gpu_matches_reference_picks(path):
    g = load(path)
    img, tmpl, ctf, cfg = case_setup(g)
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    picks = s.search(img, ctf)
    missing, extra, bad = check_against_reference(g, picks, cfg.threshold)
    assert not missing and not extra and not bad, (missing[:5], extra[:5], bad[:5])
