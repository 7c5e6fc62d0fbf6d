"""Failure path of the device waits, without a GPU fault: a bounded mbarrier wait is made to
run out on an arrival that never comes (gisspa_debug_wait_probe).  The C-ABI must return
GISSPA_ERR_TIMEOUT with its reason, and the handle and context must stay usable."""
import ctypes as C

import numpy as np
import pytest

import gisspa
from parity import small_case

pytestmark = pytest.mark.gpu


def test_wait_probe_times_out_and_handle_recovers():
    img, tmpl, ctf, cfg = small_case("norm_l256_w9")
    s = gisspa.Searcher(cfg)
    s.set_templates(tmpl)
    before = s.search(img, ctf)
    st = s.lib.gisspa_debug_wait_probe(s.h, 0.05)
    assert st == gisspa.ERR_TIMEOUT
    assert b"wait probe" in s.lib.gisspa_last_error(s.h)
    assert s.lib.gisspa_debug_wait_probe(s.h, 0.0) == gisspa.ERR_ARG
    after = s.search(img, ctf)  # the same handle still searches, with the same result
    assert after.tobytes() == before.tobytes()
    assert s.lib.gisspa_debug_wait_probe(s.h, 0.02) == gisspa.ERR_TIMEOUT
