"""The generic FFT engine (register Stockham rows for 256, 512 and 1024, radix 2, mixed radix
2/3/4/5/7, Bluestein) against numpy's FFT.

These transforms prepare templates, micrographs and windows (the reference calls cuFFT at
norm.cu:106-120 and its uses) and, for window sizes without hand-tuned kernels, carry the
correlation itself."""
import numpy as np
import pytest

import gisspa
from parity import small_case

pytestmark = pytest.mark.gpu

# (length, rows): powers of two, 2/3/5/7-smooth lengths (mixed-radix kernel, incl. the
# reference's default window 320 and the 5760 edge of a 4092x5760 micrograph), lengths with a
# prime factor above 7 (Bluestein: 3838 = 2 19 101, 4092 = 4 3 11 31)
CASES = [(1, 3), (2, 5), (256, 16), (256, 13), (512, 21), (1024, 6), (2048, 3), (3, 7), (6, 9), (105, 4),
         (320, 41), (336, 8), (720, 6),
         (960, 5), (5760, 2), (7168, 1), (53, 6), (176, 5), (3838, 2), (4092, 2)]


@pytest.fixture(scope="module")
def searcher():
    _, _, _, cfg = small_case("norm_l256_w9")
    return gisspa.Searcher(cfg)


@pytest.mark.parametrize("n,rows", CASES)
@pytest.mark.parametrize("sign", [-1, 1])
def test_engine_rows_match_numpy(searcher, n, rows, sign):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(n * 7 + rows)
    x = (rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))).astype(np.complex64)
    d = torch.from_numpy(x.copy()).cuda()
    lib = gisspa.load()
    st = lib.gisspa_debug_fft(searcher.h, d.data_ptr(), rows, n, sign)
    assert st == 0, lib.gisspa_last_error(searcher.h)
    got = d.cpu().numpy().astype(np.complex128)
    x64 = x.astype(np.complex128)
    ref = np.fft.fft(x64, axis=1) if sign < 0 else np.fft.ifft(x64, axis=1) * n
    # FP32 transform: relative RMS error grows like eps * log(n); Bluestein adds two transforms
    err = np.linalg.norm(got - ref) / max(np.linalg.norm(ref), 1e-30)
    assert err < 3e-6 * max(1.0, np.log2(n)), (n, rows, sign, err)


def test_engine_rejects_bad_arguments(searcher):
    lib = gisspa.load()
    assert lib.gisspa_debug_fft(searcher.h, None, 1, 16, -1) == gisspa.ERR_ARG
    assert lib.gisspa_debug_fft(None, None, 1, 16, -1) == gisspa.ERR_ARG
