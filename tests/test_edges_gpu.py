"""Edge cases at the C-ABI: call order, pick-buffer capacity, empty results, and micrographs
that do not tile evenly into windows.

The reference exits on bad input (utils.h:24-28) and its window split (split_IMG via
norm.cu:404-477) reads past the micrograph when a window extends beyond it (an image axis
shorter than window_size: blocks_one_axis, norm.cu:68-81, then yields the single offset 0).
The library returns status codes instead, and zero-pads such windows; the oracle pads the same
way, so those searches are compared pick for pick."""
import ctypes as C

import numpy as np
import pytest

import gisspa
import oracle
from parity import check_chunk_picks, small_case

pytestmark = pytest.mark.gpu


def test_search_before_set_templates_is_a_state_error():
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    s = gisspa.Searcher(cfg)
    with pytest.raises(gisspa.GisspaError) as e:
        s.search(img, ctf)
    assert e.value.status == gisspa.ERR_STATE


def test_template_larger_than_window_is_a_shape_error():
    _, _, _, cfg = small_case("norm_l256_w9")
    s = gisspa.Searcher(cfg)
    big = np.zeros((2, 300, 300), np.float32)
    st = s.lib.gisspa_set_templates(s.h, big.ctypes.data, 2, 300, 300)
    assert st == gisspa.ERR_SHAPE


def test_nonorm_image_smaller_than_a_tile_is_a_shape_error():
    img, tmpl, ctf, cfg = small_case("nonorm_l512")
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    with pytest.raises(gisspa.GisspaError) as e:
        s.search(np.ascontiguousarray(img[:600, :600]), ctf)
    assert e.value.status == gisspa.ERR_SHAPE


def test_capacity_error_reports_the_count_needed():
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    full = s.search(img, ctf)
    assert len(full) > 2
    im = np.ascontiguousarray(img, dtype=np.float32)
    out = np.zeros(1, dtype=gisspa.PICK_DTYPE)
    n = C.c_size_t(0)
    st = s.lib.gisspa_search(s.h, im.ctypes.data, im.shape[1], im.shape[0], C.byref(ctf), out.ctypes.data, 1,
                             C.byref(n))
    assert st == gisspa.ERR_CAPACITY and n.value == len(full)
    again = s.search(img, ctf)  # the handle stays usable
    assert len(again) == len(full)


def test_threshold_above_every_score_gives_no_picks():
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    s = gisspa.Searcher(cfg.copy(threshold=1e6))
    s.set_templates(tmpl)
    assert len(s.search(img, ctf)) == 0


@pytest.mark.parametrize("shape,threshold", [((200, 300), 3.0), ((777, 1000), 5.0)])
def test_small_and_ragged_micrographs_match_the_oracle(shape, threshold):
    """200x300: the height is shorter than the 256 window (every window zero-padded below the
    image; the two columns of windows at offsets 0 and 44).  777x1000: the last window of each
    axis clamped to the edge, a non-square image with odd height."""
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    cfg = cfg.copy(threshold=threshold)
    rng = np.random.default_rng(31)
    ny, nx = shape
    canvas = rng.standard_normal(shape).astype(np.float32)
    h, w = min(ny, img.shape[0]), min(nx, img.shape[1])
    canvas[:h, :w] = img[:h, :w]
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    g = s.search(canvas, ctf)
    o, m, near, nm = oracle.search(cfg, ctf, canvas, tmpl, want_margins=True)
    rep = check_chunk_picks(g, o, m, near, nm, cfg.threshold)
    assert len(o) > 0
    assert not rep["failures"], rep
