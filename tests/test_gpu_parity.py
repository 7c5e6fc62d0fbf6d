"""GPU parity: the CUDA path (through the C-ABI) against the FP64 oracle, stage by stage
and end to end, on small seeded cases."""
import ctypes as C

import numpy as np
import pytest

import gisspa
import oracle
from parity import (check_chunk_picks, check_template_picks, check_topk_picks, half_spectrum, rel_err,
                    small_case)

pytestmark = pytest.mark.gpu


def stage(s: gisspa.Searcher, what: int, image, ctf, theta: float, shape, dtype):
    out = np.zeros(shape, dtype=dtype)
    img_ptr, nx, ny = (None, 0, 0)
    if image is not None:
        image = np.ascontiguousarray(image, dtype=np.float32)
        img_ptr, (ny, nx) = image.ctypes.data, image.shape
    lib = gisspa.load()
    st = lib.gisspa_debug_stage(s.h, what, img_ptr, nx, ny, C.byref(ctf), theta, out.ctypes.data, out.nbytes)
    assert st == 0, lib.gisspa_last_error(s.h)
    return out


@pytest.fixture(scope="module")
def norm_case():
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    return img, tmpl, ctf, cfg, s


def test_stage_templates_norm(norm_case):
    img, tmpl, ctf, cfg, s = norm_case
    L = cfg.window_size
    g = stage(s, 1, None, ctf, 0.0, (tmpl.shape[0], L, L), np.float32)
    o = oracle.prep_templates(cfg, ctf, tmpl).real
    assert rel_err(g, o) < 1e-4


def test_stage_image_norm(norm_case):
    img, tmpl, ctf, cfg, s = norm_case
    g = stage(s, 2, img, ctf, 0.0, img.shape, np.float32)
    o = oracle.prep_image(cfg, ctf, img)
    assert rel_err(g, o) < 1e-4


def test_stage_window_spectra(norm_case):
    img, tmpl, ctf, cfg, s = norm_case
    L = cfg.window_size
    o = oracle.window_spectra(cfg, oracle.prep_image(cfg, ctf, img))
    g = stage(s, 3, img, ctf, 0.0, (o.shape[0], L // 2 + 1, L), np.complex64)
    assert rel_err(g, half_spectrum(o)) < 1e-4


@pytest.mark.parametrize("theta", [0.0, 45.0, 135.0])
def test_stage_template_spectra(norm_case, theta):
    img, tmpl, ctf, cfg, s = norm_case
    L = cfg.window_size
    prep = oracle.prep_templates(cfg, ctf, tmpl)
    o = np.stack([oracle.rotated_spectrum(cfg, ctf, prep[n], theta) for n in range(tmpl.shape[0])])
    g = stage(s, 4, None, ctf, theta, (tmpl.shape[0], L // 2 + 1, L), np.complex64)
    assert rel_err(g, half_spectrum(o)) < 1e-4


def test_cc_maps_against_oracle(norm_case):
    """CC maps through gisspa_cc_maps: the hot correlation kernels on oracle spectra."""
    torch = pytest.importorskip("torch")
    img, tmpl, ctf, cfg, s = norm_case
    L = cfg.window_size
    win = oracle.window_spectra(cfg, oracle.prep_image(cfg, ctf, img))[:3]
    prep = oracle.prep_templates(cfg, ctf, tmpl)
    T = np.stack([oracle.rotated_spectrum(cfg, ctf, prep[n], 45.0) for n in range(2)])
    dW = torch.from_numpy(half_spectrum(win).astype(np.complex64)).cuda()
    dT = torch.from_numpy(half_spectrum(T).astype(np.complex64)).cuda()
    out = torch.zeros((3, 2, L, L), dtype=torch.float32, device="cuda")
    lib = gisspa.load()
    st = lib.gisspa_cc_maps(s.h, dW.data_ptr(), 3, dT.data_ptr(), 2, gisspa.SPEC_FP32, out.data_ptr())
    assert st == 0, lib.gisspa_last_error(s.h)
    g = out.cpu().numpy()
    yy, xx = np.mgrid[0:L, 0:L]
    chk = np.where((xx + yy) % 2 == 1, -1.0, 1.0)
    for b in range(3):
        for n in range(2):
            ref = np.fft.ifft2(win[b] * np.conj(T[n]) * chk).real  # = IFFT_unnormalised / L^2
            assert rel_err(g[b, n], ref) < 1e-4, (b, n)


@pytest.mark.parametrize("name", ["norm_l320_w4", "norm_l336_w4", "norm_l176_w4"])
def test_cc_maps_generic_window(name):
    """Correlation maps at window sizes without hand-tuned kernels (the reference's default 320,
    a mixed-radix 336 and a Bluestein 176) against numpy."""
    torch = pytest.importorskip("torch")
    img, tmpl, ctf, cfg = small_case(name)
    s = gisspa.Searcher(cfg)
    L = cfg.window_size
    win = oracle.window_spectra(cfg, oracle.prep_image(cfg, ctf, img))[:2]
    prep = oracle.prep_templates(cfg, ctf, tmpl)
    T = np.stack([oracle.rotated_spectrum(cfg, ctf, prep[n], 30.0) for n in range(3)])
    dW = torch.from_numpy(half_spectrum(win).astype(np.complex64)).cuda()
    dT = torch.from_numpy(half_spectrum(T).astype(np.complex64)).cuda()
    out = torch.zeros((2, 3, L, L), dtype=torch.float32, device="cuda")
    lib = gisspa.load()
    st = lib.gisspa_cc_maps(s.h, dW.data_ptr(), 2, dT.data_ptr(), 3, gisspa.SPEC_FP32, out.data_ptr())
    assert st == 0, lib.gisspa_last_error(s.h)
    g = out.cpu().numpy()
    yy, xx = np.mgrid[0:L, 0:L]
    chk = np.where((xx + yy) % 2 == 1, -1.0, 1.0)
    for b in range(2):
        for n in range(3):
            ref = np.fft.ifft2(win[b] * np.conj(T[n]) * chk).real
            assert rel_err(g[b, n], ref) < 1e-4, (b, n)


def run_both(name, **over):
    """GPU search and oracle search (with decision margins) of a small case."""
    img, tmpl, ctf, cfg = small_case(name)
    cfg = cfg.copy(**over)
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    g = s.search(img, ctf)
    o, m, near, nm = oracle.search(cfg, ctf, img, tmpl, want_margins=True)
    return g, (o, m, near, nm), cfg, s


@pytest.mark.parametrize("name", ["norm_l256_w9", "norm_l512_w4", "norm_l1024_w4", "norm_l320_w4", "norm_l336_w4",
                                  "norm_l176_w4"])
def test_search_norm_chunk_picks(name):
    g, (o, m, near, nm), cfg, s = run_both(name)
    rep = check_chunk_picks(g, o, m, near, nm, cfg.threshold)
    assert len(o) > 0
    assert not rep["failures"], rep


def test_search_norm_stats_maps():
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    s.search(img, ctf)
    picks, st = oracle.search(cfg, ctf, img, tmpl, want_stats=True)
    W, L = st.shape[0], cfg.window_size
    ms = stage(s, 5, None, ctf, 0.0, (W, L, L, 2), np.float32)
    mu_o, sd_o = st[..., 0], st[..., 1]
    assert np.abs(ms[..., 0] - mu_o).max() <= 1e-4 * np.abs(sd_o).max()
    sd_g = np.where(ms[..., 1] > 0, 1.0 / np.maximum(ms[..., 1], 1e-30), 0.0)
    assert rel_err(sd_g, sd_o) < 1e-4


@pytest.mark.parametrize("name", ["norm_l256_w9", "norm_l1024_w4", "norm_l320_w4", "norm_l336_w4", "norm_l176_w4"])
def test_search_norm_topk(name):
    g, (o, m, _, _), cfg, s = run_both(name, pick_mode=gisspa.PICK_TOPK, topk=20, exclusion_radius=30.0,
                                       threshold=2.0)
    assert len(o) > 0
    rep = check_topk_picks(g, o, m)
    assert not rep["failures"], rep


@pytest.mark.parametrize("name", ["nonorm_l512", "nonorm_l320", "nonorm_l176"])
def test_search_nonorm(name):
    g, (o, m, _, _), cfg, s = run_both(name)
    rep = check_template_picks(g, o, m, cfg.threshold)
    assert len(o) > 0
    assert not rep["failures"], rep


@pytest.mark.parametrize("spec", [gisspa.SPEC_FP16, gisspa.SPEC_BF16])
def test_half_precision_spectra_close(spec):
    """FP16/BF16 template spectra against the FP64 oracle: top-K picks by the margin rule at the
    precision form's tolerance (FP16 1e-3 relative, the chosen form's bar; BF16, with 8 bits of
    mantissa, 1e-2)."""
    tol = 1e-3 if spec == gisspa.SPEC_FP16 else 1e-2
    g, (o, m, _, _), cfg, s = run_both("norm_l256_w9", spectrum_precision=spec, pick_mode=gisspa.PICK_TOPK, topk=20,
                                       exclusion_radius=30.0, threshold=2.0)
    rep = check_topk_picks(g, o, m, rtol=tol, atol=0.0)
    assert not rep["failures"], rep


def test_search_host_and_device_paths_agree():
    torch = pytest.importorskip("torch")
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    a = s.search(img, ctf)
    d = torch.from_numpy(img).cuda()
    out = np.zeros(1 << 16, dtype=gisspa.PICK_DTYPE)
    n = s.search_device(d.data_ptr(), img.shape[1], img.shape[0], ctf, out)
    assert n == len(a) and np.array_equal(out[:n], a)


def test_batch_matches_single_searches():
    """A batch (each micrograph's upload and statistics overlapped with the previous one's
    sweep, in two alternating buffers) gives the single searches' picks bit for bit, across
    uneven sizes and CTFs."""
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    img2 = np.ascontiguousarray(img[:, ::-1])
    img3 = np.ascontiguousarray(np.concatenate([img, img[:200]], axis=0)[:, :448])
    ctf3 = gisspa.Ctf(ctf.defocus + 0.3, ctf.dfdiff, ctf.dfang + 10.0)
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    imgs, ctfs = [img, img2, img3, img], [ctf, ctf, ctf3, ctf]
    one = [s.search(i, c) for i, c in zip(imgs, ctfs)]
    batch = s.search_batch(imgs, ctfs)
    assert len(batch) == len(one)
    for x, y in zip(one, batch):
        assert len(x) > 0 and np.array_equal(x, y)


@pytest.mark.parametrize("tensor_cores", [1, 0])
@pytest.mark.parametrize("name", ["norm_l256_w9", "norm_l512_w4"])
def test_chosen_form_picks_and_scores(name, tensor_cores):
    """The chosen form (FP16 template spectra, one top-K sweep) against the FP64 oracle: picks by
    the margin rule, peak scores within 1e-3 (relative).  At window 512 the column transforms run
    on the tensor cores (tcgen05, FP16 operands) or, with tensor_cores = 0, on the CUDA cores."""
    g, (o, m, _, _), cfg, s = run_both(name, spectrum_precision=gisspa.SPEC_FP16, pick_mode=gisspa.PICK_TOPK,
                                       topk=30, exclusion_radius=30.0, threshold=2.5, tensor_cores=tensor_cores)
    assert len(o) >= 5
    rep = check_topk_picks(g, o, m, rtol=1e-3, atol=0.0)
    assert not rep["failures"], rep


@pytest.mark.parametrize("name,shapes,a_shapes", [("norm_l256_w9", 2, 1), ("norm_l512_w4", 5, 2),
                                                  ("norm_l1024_w4", 5, 1)])
@pytest.mark.parametrize("mode", ["chunk", "topk"])
def test_every_row_kernel_shape(name, shapes, a_shapes, mode):
    """Each compiled row-transform shape, and at window 512 each column-transform shape (forced
    with fixed launch batches), against the oracle."""
    img, tmpl, ctf, cfg = small_case(name)
    over = dict(template_batch=2, window_batch=2)
    if mode == "topk":
        over.update(pick_mode=gisspa.PICK_TOPK, topk=20, exclusion_radius=30.0, threshold=2.0)
    cfg = cfg.copy(**over)
    o, m, near, nm = oracle.search(cfg, ctf, img, tmpl, want_margins=True)
    assert len(o) > 0
    for v, av in [(v, 0) for v in range(shapes)] + [(0, av) for av in range(1, a_shapes)]:
        s = gisspa.Searcher(cfg.copy(pass_b_shape=v, pass_a_shape=av))
        s.set_templates(tmpl)
        g = s.search(img, ctf)
        if mode == "chunk":
            rep = check_chunk_picks(g, o, m, near, nm, cfg.threshold)
        else:
            rep = check_topk_picks(g, o, m)
        assert not rep["failures"], (v, av, rep)


def test_tensor_core_column_pass_chunk_picks():
    """FP16 spectra with the reference's chunk picks (two sweeps) at window 512: the tensor-core
    column pass against the oracle by the margin rule at the FP16 form's 1e-3."""
    g, (o, m, near, nm), cfg, s = run_both("norm_l512_w4", spectrum_precision=gisspa.SPEC_FP16, tensor_cores=1)
    assert len(o) > 0
    rep = check_chunk_picks(g, o, m, near, nm, cfg.threshold, rtol=1e-3, atol=0.0)
    assert not rep["failures"], rep


@pytest.mark.parametrize("graphs", [1, 0])
@pytest.mark.parametrize("mode", ["chunk", "topk", "fp16_topk"])
def test_pair_engine_bit_identical_to_per_pass_kernels(mode, graphs):
    """The pair engine (row shape 4 at window 512: pass A of one batch and pass B of the batch
    before it in one launch, Q in two alternating slots) computes every value with the per-pass
    kernels' device code and folds each batch into the per-pixel state in the same order: its
    picks (and, for chunk picks, the mean / sigma maps) equal those of shape 0 bit for bit.  Uneven batches (4
    templates in batches of 3, 4 windows in batches of 3), with and without CUDA graphs."""
    img, tmpl, ctf, cfg = small_case("norm_l512_w4")
    over = dict(template_batch=3, window_batch=3, cuda_graphs=graphs)
    if mode != "chunk":
        over.update(pick_mode=gisspa.PICK_TOPK, topk=20, exclusion_radius=30.0, threshold=2.0)
    if mode == "fp16_topk":
        over.update(spectrum_precision=gisspa.SPEC_FP16)
    cfg = cfg.copy(**over)
    res = []
    for v in (0, 4):
        s = gisspa.Searcher(cfg.copy(pass_b_shape=v))
        s.set_templates(tmpl)
        g = s.search(img, ctf)
        W, L = 4, cfg.window_size
        ms = stage(s, 5, None, ctf, 0.0, (W, L, L, 2), np.float32) if mode == "chunk" else None
        res.append((g, ms, s.stats().pairs))
        s.close()
    (g0, ms0, p0), (g4, ms4, p4) = res
    assert len(g0) > 0 and p0 == p4
    assert np.array_equal(g0, g4)
    if mode == "chunk":
        assert np.array_equal(ms0, ms4)


@pytest.mark.parametrize("raise_threshold", [0.0, 2.0])
@pytest.mark.parametrize("name", ["norm_l256_w9", "norm_l512_w4", "norm_l1024_w4", "norm_l320_w4"])
def test_pruned_second_sweep_gives_the_same_picks(name, raise_threshold):
    """Sweep 2 with the rows that cannot hold a pick skipped (prune_sweep2 = 1, the default)
    against sweep 2 over every row: the same chunk picks bit for bit (none, for some cases, at
    the raised threshold, where rows are skipped).  (Fixed launch shapes: the autotuner may pick another column-transform shape
    for either search, whose rounding differs in the last bits.)"""
    img, tmpl, ctf, cfg = small_case(name)
    cfg = cfg.copy(threshold=cfg.threshold + raise_threshold, template_batch=2, window_batch=2, pass_a_shape=0,
                   pass_b_shape=0)
    res = []
    for prune in (0, 1):
        s = gisspa.Searcher(cfg.copy(prune_sweep2=prune))
        s.set_templates(tmpl)
        g = s.search(img, ctf)
        res.append((g, s.stats().rows_alive))
        s.close()
    (g0, r0), (g1, r1) = res
    assert (len(g0) > 0 or raise_threshold) and np.array_equal(g0, g1)
    assert r0 == 1.0 and 0.0 <= r1 <= 1.0
    if raise_threshold:
        assert r1 < 1.0


def test_pruned_second_sweep_with_a_large_template_batch():
    """A fixed template batch above the 256 templates that pass B lists: the pruned sweep rebuilds
    every template's spectra at each angle, and the picks equal those without pruning."""
    img, tmpl, ctf, cfg = small_case("norm_l512_w4")
    cfg = cfg.copy(threshold=cfg.threshold + 2.0, template_batch=300, window_batch=2, pass_a_shape=0,
                   pass_b_shape=0)
    res = []
    for prune in (0, 1):
        s = gisspa.Searcher(cfg.copy(prune_sweep2=prune))
        s.set_templates(tmpl)
        res.append(s.search(img, ctf))
        s.close()
    assert np.array_equal(res[0], res[1])
