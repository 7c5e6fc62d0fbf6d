"""CPU tests of the FP64 oracle: its FFT against numpy, and the reference's geometry rules."""
import math

import numpy as np
import pytest

import gisspa
import oracle
import synth
from parity import assert_planted_copies_found, planted_copies_case, small_case


@pytest.mark.parametrize("shape", [(8, 16), (64, 64), (30, 42), (7, 5), (1, 12), (256, 96)])
def test_fft_matches_numpy(shape):
    rng = np.random.default_rng(0)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    f = oracle.fft2(a, -1)
    assert np.abs(f - np.fft.fft2(a)).max() <= 1e-12 * np.abs(f).max()
    i = oracle.fft2(a, +1)
    assert np.abs(i - np.fft.ifft2(a) * a.size).max() <= 1e-12 * np.abs(i).max()


def test_fft_impulse_and_dc():
    a = np.zeros((16, 16), complex)
    a[0, 0] = 1
    assert np.allclose(oracle.fft2(a, -1), 1)
    b = np.ones((12, 20), complex)
    f = oracle.fft2(b, -1)
    assert abs(f[0, 0] - 240) < 1e-9 and np.abs(f.ravel()[1:]).max() < 1e-9


def test_window_offsets_match_reference_rule():
    # blocks_one_axis (norm.cu:68-81): step l - ov, last clamped to len - l
    assert oracle.window_offsets(4096, 512, 192) == [0, 320, 640, 960, 1280, 1600, 1920, 2240, 2560, 2880, 3200,
                                                     3520, 3584]
    assert len(oracle.window_offsets(4096, 512, 192)) ** 2 == 169
    assert oracle.window_offsets(512, 256, 0) == [0, 256]
    assert oracle.window_offsets(200, 256, 0) == [0]
    assert len(oracle.window_offsets(8192, 1024, 256)) ** 2 == 121


def test_tiles_match_reference_rule():
    # TileImages (tileimages.cpp:18-70): 1024^2 -> 2x2 tiles, column-major, last centred at width - 360
    assert oracle.tiles(1024, 1024) == [(0, 0), (0, 304), (304, 0), (304, 304)]
    assert oracle.tiles(720, 720) == [(0, 0)]
    t = oracle.tiles(3000, 2000)
    assert len(t) == 5 * 3 and t[0] == (0, 0) and t[-1] == (3000 - 720, 2000 - 720)


def test_shell_index_is_exact():
    # floor(hypot + 0.5) - 1 on integer grids, against an exact rational test
    for a in range(0, 300, 7):
        for b in range(0, 300, 5):
            n = a * a + b * b
            if n == 0:
                continue
            k = int(math.floor(math.sqrt(n) + 0.5))
            # integer form used by the oracle and the kernels: k^2 - k < n <= k^2 + k
            assert k * k - k < n <= k * k + k


def test_planted_particle_peak_position():
    """Known answer: a noise-free planted particle correlates best at its own centre."""
    c = synth.make_case(shape=(512, 512), n_particles=1, snr=100.0, n_templates=2, tsize=64, seed=5, margin=150)
    cfg = gisspa.Config.default(angpix=1.0, phistep=10.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                                diameter=48.0, threshold=-100.0, window_size=256, overlap=0, norm_type=1)
    ctf = gisspa.Ctf(c.defocus, c.dfdiff, c.dfang)
    prep = oracle.prep_templates(cfg, ctf, c.templates)
    win = oracle.window_spectra(cfg, oracle.prep_image(cfg, ctf, c.image))
    offs = oracle.window_offsets(512, 256, 0)
    j = int(c.particles[0, 2])
    L = 256
    yy, xx = np.mgrid[0:L, 0:L]
    chk = np.where((xx + yy) % 2, -1.0, 1.0)
    best = None
    for th in range(0, 360, 10):
        T = oracle.rotated_spectrum(cfg, ctf, prep[j], float(th))
        for b in range(4):
            cc = np.fft.ifft2(win[b] * np.conj(T) * chk).real
            k = int(np.argmax(cc))
            cand = (cc.flat[k], offs[b % 2] + k % L, offs[b // 2] + k // L)
            best = max(best, cand) if best else cand
    px, py = c.particles[0, :2]
    assert abs(best[1] - px) <= 6 and abs(best[2] - py) <= 6


def test_oracle_search_runs_small():
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    picks, st = oracle.search(cfg, ctf, img, tmpl, want_stats=True)
    assert len(picks) > 0
    assert np.all(picks["score"] >= cfg.threshold)
    assert st.shape == (9, 256, 256, 2) and np.all(st[..., 1] > 0)
    order = np.lexsort((picks["chunk"], picks["template_id"], picks["window"], picks["angle_index"]))
    assert np.array_equal(order, np.arange(len(picks)))


def test_oracle_finds_planted_copies():
    """Known answer: rotated exact copies of three templates at their centres and rotations."""
    img, tmpl, ctf, cfg, truth = planted_copies_case()
    assert_planted_copies_found(oracle.search(cfg, ctf, img, tmpl), truth)
