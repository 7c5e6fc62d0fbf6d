"""Known answer through the C-ABI: exact copies of three distinct templates, rotated by
multiples of 90 degrees (exact on the pixel grid), CTF-modulated and planted in noise at
integer offsets, are the top-K picks of the search, each with its own template, its rotation
and its centre within a pixel, with FP32 and with FP16 template spectra (the chosen form)."""
import pytest

import gisspa
from parity import assert_planted_copies_found, planted_copies_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("spec", [gisspa.SPEC_FP32, gisspa.SPEC_FP16])
def test_search_finds_planted_copies(spec):
    img, tmpl, ctf, cfg, truth = planted_copies_case()
    s = gisspa.Searcher(cfg.copy(spectrum_precision=spec))
    s.set_templates(tmpl)
    assert_planted_copies_found(s.search(img, ctf), truth)
