"""The fast path's reciprocal and square root (hardware seed + polynomial
correction, mpd_fast_math) against correctly rounded results: within 1 ulp
over random doubles of every exponent the solver meets, and the special
cases of the square root."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(pkg, x):
    import torch
    lib = pkg._native.load()
    dx = torch.from_numpy(x).cuda()
    rcp = torch.empty_like(dx)
    sqr = torch.empty_like(dx)
    stream = torch.cuda.current_stream().cuda_stream
    pkg._native.check(lib.mpd_fast_math(C.c_void_p(dx.data_ptr()), x.size,
                                        C.c_void_p(rcp.data_ptr()), C.c_void_p(sqr.data_ptr()),
                                        C.c_void_p(stream)), lib)
    torch.cuda.synchronize()
    return rcp.cpu().numpy(), sqr.cpu().numpy()


def _ulps(a, b):
    return np.abs(a - b) / np.spacing(np.abs(b))


def test_reciprocal_and_sqrt_within_one_ulp(pkg):
    rng = np.random.default_rng(7)
    n = 1 << 22
    x = rng.uniform(1.0, 2.0, n) * np.exp2(rng.integers(-60, 61, n).astype(np.float64))
    rcp, sqr = _run(pkg, x)
    assert _ulps(rcp, 1.0 / x).max() <= 1.0
    assert _ulps(sqr, np.sqrt(x)).max() <= 1.0
    xn = -x[:1000]
    rcp_n, _ = _run(pkg, xn)
    assert _ulps(rcp_n, 1.0 / xn).max() <= 1.0


def test_sqrt_special_cases(pkg):
    x = np.array([0.0, -1.0, 4.0, 1e-300, 1e300])
    _, sqr = _run(pkg, x)
    assert sqr[0] == 0.0
    assert np.isnan(sqr[1])
    assert sqr[2] == 2.0
    assert _ulps(sqr[3:], np.sqrt(x[3:])).max() <= 1.0
