"""gisspa_cc_maps_noalloc: the allocation-free correlation-map entry point.

It is for callers that cannot allocate device memory (a framework that owns the
device memory pool or budget, a locked-down allocator).  It must give the same maps
as the allocating gisspa_cc_maps on two calls in a row (the second reuses the shared
fixed scratch), whether it runs alone in a fresh process or after every other test;
this file is collected last.
"""
import numpy as np
import pytest

import gisspa
from parity import rel_err

pytestmark = pytest.mark.gpu


def test_noalloc_maps_match_allocating_entry_point():
    torch = pytest.importorskip("torch")
    L, nw, nt = 512, 3, 4  # 12 pairs: within the 16-pair limit at window_size 512
    cfg = gisspa.Config.default(angpix=1.0, phistep=5.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                                diameter=100.0, window_size=L, norm_type=1)
    s = gisspa.Searcher(cfg)
    lib = gisspa.load()
    gen = torch.Generator(device="cpu").manual_seed(1234)
    for call in range(2):
        W = torch.randn((nw, L // 2 + 1, L, 2), generator=gen).cuda()
        T = torch.randn((nt, L // 2 + 1, L, 2), generator=gen).cuda()
        ref = torch.zeros((nw, nt, L, L), device="cuda")
        out = torch.full((nw, nt, L, L), float("nan"), device="cuda")
        st = lib.gisspa_cc_maps(s.h, W.data_ptr(), nw, T.data_ptr(), nt, gisspa.SPEC_FP32, ref.data_ptr())
        assert st == 0, lib.gisspa_last_error(s.h)
        st = lib.gisspa_cc_maps_noalloc(W.data_ptr(), nw, T.data_ptr(), nt, L, gisspa.SPEC_FP32, out.data_ptr(),
                                        None)
        assert st == 0, lib.gisspa_last_error(None)
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.isfinite(a).all(), call
        assert rel_err(a, b) < 1e-4, call


def test_noalloc_rejects_calls_beyond_the_fixed_scratch():
    torch = pytest.importorskip("torch")
    L = 1024
    lib = gisspa.load()
    W = torch.zeros((5, L // 2 + 1, L, 2), device="cuda")
    out = torch.zeros((5, 1, L, L), device="cuda")
    st = lib.gisspa_cc_maps_noalloc(W.data_ptr(), 5, W.data_ptr(), 1, L, gisspa.SPEC_FP32, out.data_ptr(), None)
    assert st == gisspa.ERR_CAPACITY
    assert b"scratch" in lib.gisspa_last_error(None)
