"""fb_predict_draw_static, the predict call that allocates no device memory, checked through the C ABI.

Callers that cannot allocate device memory (another framework owns it, or a cudaFree would stall their other
streams) use fb_predict_draw_static in place of fb_predict_draw.  Its results must be the same bit for bit, call
after call, even though every call reuses one fixed device array.  This file is collected last so that a run that
stops at the first failure has already run every other test; it sets up everything it needs and also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

import fastbart_b200 as F
from fastbart_b200 import _lib
from fastbart_b200 import workloads as W

pytestmark = pytest.mark.gpu

SCRATCH_DOUBLES = 1 << 20   # the documented limit: n * (ncol + 1) doubles


def _call(name, ct, X, draw, mu):
    cols = [np.ascontiguousarray(X[:, j]) for j in range(X.shape[1])]
    ptrs = (C.c_void_p * max(1, len(cols)))(*[c.ctypes.data for c in cols])
    out = np.full(X.shape[0], np.nan)
    st = getattr(_lib.lib(), name)(ct.handle(), ptrs, len(cols), X.shape[0], draw, mu, out.ctypes.data)
    return st, out


@pytest.fixture(scope="module")
def compiled():
    x, y = W.hazard_data(2500, 5)
    ch = W.fpbart_chain(x, y, ntree=15, nskip=20, ndpost=6, seed=21)
    g = F.fit_batch([ch], 20, 6)[0]
    ct = F.CompiledTrees(F.trees_text(g["trees"], x.shape[1]), ch["xi"], mu=ch["offset"])
    return ct, x.shape[1], ch["offset"]


def test_two_calls_in_a_row_match_predict_draw(compiled):
    ct, p, mu = compiled
    # a call that fills the array, then a smaller one with another draw: nothing of the first may show in the second
    big, _ = W.hazard_data(SCRATCH_DOUBLES // (p + 1), 77)
    small, _ = W.hazard_data(1234, 78)
    for X, draw in ((big, 2), (small, 5)):
        s0, ref = _call("fb_predict_draw", ct, X, draw, mu)
        s1, got = _call("fb_predict_draw_static", ct, X, draw, mu)
        assert s0 == _lib.FB_OK and s1 == _lib.FB_OK, _lib.lib().fb_last_error().decode()
        assert np.array_equal(got, ref)   # bit-exact, as every predict test here


def test_calls_leave_free_device_memory_unchanged(compiled):
    """After a first (set-up) call, further calls take no device memory: the driver's free-memory figure stays put."""
    import torch
    ct, p, mu = compiled
    X, _ = W.hazard_data(SCRATCH_DOUBLES // (p + 1), 79)
    st, first = _call("fb_predict_draw_static", ct, X, 1, mu)
    assert st == _lib.FB_OK
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for draw in (2, 3, 4, 1):
        st, got = _call("fb_predict_draw_static", ct, X, draw, mu)
        assert st == _lib.FB_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert np.array_equal(got, first)


def test_limit_and_argument_errors(compiled):
    ct, p, mu = compiled
    too_big = np.zeros((SCRATCH_DOUBLES // (p + 1) + 1, p))
    st, _ = _call("fb_predict_draw_static", ct, too_big, 1, mu)
    assert st == _lib.FB_ERR_LIMIT
    assert "fixed device scratch" in _lib.lib().fb_last_error().decode()
    x, _ = W.hazard_data(100, 3)
    st, _ = _call("fb_predict_draw_static", ct, x, 99, mu)
    assert st == _lib.FB_ERR_RANGE
    st, _ = _call("fb_predict_draw_static", ct, x[:, :2], 1, mu)
    assert st == _lib.FB_ERR_SHAPE
    # a rejected call leaves the array usable
    s0, ref = _call("fb_predict_draw", ct, x, 3, mu)
    s1, got = _call("fb_predict_draw_static", ct, x, 3, mu)
    assert s0 == s1 == _lib.FB_OK and np.array_equal(got, ref)
