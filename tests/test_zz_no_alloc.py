"""gisspa_cc_maps_noalloc: the allocation-free correlation-map entry point.

It is for callers that cannot allocate device memory (a framework that owns the
device memory pool or budget, a locked-down allocator).  It must give the same maps
as the allocating gisspa_cc_maps on two calls in a row (the second reuses the shared
fixed scratch and error flag), whether it runs alone in a fresh process or after
every other test; this file is collected last.  A GISSPA_OK return also says that the
call read its timeout flag back clear after the launches.
"""
import numpy as np
import pytest

import gisspa
from parity import rel_err

pytestmark = pytest.mark.gpu

# the fixed scratch holds 16 MiB / (L^2 * 4 B) pairs
CAPACITY = {256: 64, 512: 16, 1024: 4}


def _spectra(torch, gen, n, L, spec):
    x = torch.randn((n, L // 2 + 1, L, 2), generator=gen)
    if spec == gisspa.SPEC_FP16:
        x = x.half()
    elif spec == gisspa.SPEC_BF16:
        x = x.bfloat16()
    return x.cuda()


def _run_pair(torch, lib, s, L, nw, nt, spec, gen, stream=None):
    W = _spectra(torch, gen, nw, L, gisspa.SPEC_FP32)
    T = _spectra(torch, gen, nt, L, spec)
    ref = torch.zeros((nw, nt, L, L), device="cuda")
    out = torch.full((nw, nt, L, L), float("nan"), device="cuda")
    st = lib.gisspa_cc_maps(s.h, W.data_ptr(), nw, T.data_ptr(), nt, spec, ref.data_ptr())
    assert st == 0, lib.gisspa_last_error(s.h)
    torch.cuda.synchronize()
    sp = None if stream is None else stream.cuda_stream
    st = lib.gisspa_cc_maps_noalloc(W.data_ptr(), nw, T.data_ptr(), nt, L, spec, out.data_ptr(), sp)
    assert st == 0, lib.gisspa_last_error(None)
    torch.cuda.synchronize()
    a, b = out.cpu().numpy(), ref.cpu().numpy()
    assert np.isfinite(a).all()
    return rel_err(a, b)


def _searcher(L):
    cfg = gisspa.Config.default(angpix=1.0, phistep=5.0, kk=3.0, energy=300.0, cs=2.7, highres=8.0, lowres=200.0,
                                diameter=100.0, window_size=L, norm_type=1)
    return gisspa.Searcher(cfg)


@pytest.mark.parametrize("spec", [gisspa.SPEC_FP32, gisspa.SPEC_FP16, gisspa.SPEC_BF16])
@pytest.mark.parametrize("L", [256, 512, 1024])
def test_noalloc_maps_match_allocating_entry_point(L, spec):
    torch = pytest.importorskip("torch")
    s = _searcher(L)
    lib = gisspa.load()
    gen = torch.Generator(device="cpu").manual_seed(1234 + L + spec)
    nw, nt = (3, 4) if L < 1024 else (1, 3)
    for call in range(2):
        assert _run_pair(torch, lib, s, L, nw, nt, spec, gen) < 1e-4, call
    s.close()


@pytest.mark.parametrize("L", [256, 512, 1024])
def test_noalloc_at_exact_capacity_on_a_side_stream(L):
    """A call that fills the fixed scratch exactly, issued on a non-default stream; the device's
    free memory is the same before and after it (the call allocates nothing)."""
    torch = pytest.importorskip("torch")
    s = _searcher(L)
    lib = gisspa.load()
    gen = torch.Generator(device="cpu").manual_seed(99 + L)
    cap = CAPACITY[L]
    nw = {256: 8, 512: 4, 1024: 2}[L]
    nt = cap // nw
    stream = torch.cuda.Stream()
    W = _spectra(torch, gen, nw, L, gisspa.SPEC_FP32)
    T = _spectra(torch, gen, nt, L, gisspa.SPEC_FP32)
    ref = torch.zeros((nw, nt, L, L), device="cuda")
    out = torch.full((nw, nt, L, L), float("nan"), device="cuda")
    assert lib.gisspa_cc_maps(s.h, W.data_ptr(), nw, T.data_ptr(), nt, gisspa.SPEC_FP32, ref.data_ptr()) == 0
    torch.cuda.synchronize()
    # the first call on this device already ran (earlier tests or the call below): measure a later one
    lib.gisspa_cc_maps_noalloc(W.data_ptr(), nw, T.data_ptr(), nt, L, gisspa.SPEC_FP32, out.data_ptr(),
                               stream.cuda_stream)
    torch.cuda.synchronize()
    out.fill_(float("nan"))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st = lib.gisspa_cc_maps_noalloc(W.data_ptr(), nw, T.data_ptr(), nt, L, gisspa.SPEC_FP32, out.data_ptr(),
                                    stream.cuda_stream)
    free1 = torch.cuda.mem_get_info()[0]
    assert st == 0, lib.gisspa_last_error(None)
    assert free1 == free0
    torch.cuda.synchronize()
    a, b = out.cpu().numpy(), ref.cpu().numpy()
    assert np.isfinite(a).all()
    assert rel_err(a, b) < 1e-4
    s.close()


def test_noalloc_rejects_calls_beyond_the_fixed_scratch():
    torch = pytest.importorskip("torch")
    L = 1024
    lib = gisspa.load()
    W = torch.zeros((5, L // 2 + 1, L, 2), device="cuda")
    out = torch.zeros((5, 1, L, L), device="cuda")
    st = lib.gisspa_cc_maps_noalloc(W.data_ptr(), 5, W.data_ptr(), 1, L, gisspa.SPEC_FP32, out.data_ptr(), None)
    assert st == gisspa.ERR_CAPACITY
    assert b"scratch" in lib.gisspa_last_error(None)
