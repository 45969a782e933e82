"""fb_fbart, the one-for-one replacement of fbart_cpp (src/glue.cpp:10-62), called through the C ABI with R's memory
layouts: q an n x p integer matrix (column-major), yhat.train ndpost x n and varcount ndpost x p (column-major), the
tree text sized by a first call with trees_text = NULL.  Its outputs must equal, bit for bit, those of the batch
entry point (fb_fit_batch) plus the host writers fb_trees_text and fb_varcount on the same chain."""
import ctypes as C

import numpy as np
import pytest

import fastbart_b200 as F
from fastbart_b200 import _lib, workloads as W
from fastbart_b200.api import fit_batch

pytestmark = pytest.mark.gpu


def _fbart(ch, nskip, ndpost, text: bool):
    """One fb_fbart call; returns its outputs in R's shapes (numpy views of the column-major buffers)."""
    q = np.ascontiguousarray(ch["q"], dtype=np.int32)          # [p][n] row-major == n x p column-major
    p, n = q.shape
    probit = int(ch["probit"])
    y = None if probit else np.ascontiguousarray(ch["y"], np.float64)
    wt = None if probit else np.ascontiguousarray(ch["wt"], np.float64)
    ybin = np.ascontiguousarray(ch["ybin"], np.int32) if probit else None
    numcut = np.ascontiguousarray(ch["numcut"], np.int32)
    pg = np.ascontiguousarray(ch["pgtab"], np.float64)
    sigma = np.full(nskip + ndpost, np.nan)
    ymean = np.full(n, np.nan)
    yhat = np.full(ndpost * n, np.nan)      # column-major ndpost x n
    vc = np.full(ndpost * p, -1, np.int32)  # column-major ndpost x p
    moves = np.zeros(3, np.int32)
    ln = C.c_size_t(0)
    buf = C.create_string_buffer(text) if isinstance(text, int) and text > 1 else None
    cap = len(buf) if buf is not None else 0
    P = _lib.ptr
    st = _lib.lib().fb_fbart(P(q), n, p, P(y), P(wt), P(ybin), P(numcut), P(pg), int(ch["ntree"]), nskip, ndpost,
                             float(ch["tau"]), float(ch["lambda"]), float(ch["nu"]), float(ch["sigest"]),
                             int(ch["seed"]), probit, float(ch["offset"]), P(sigma), P(ymean), P(yhat), P(vc),
                             buf, cap, C.byref(ln), P(moves))
    _lib.check(st)
    return dict(sigma=sigma, yhat_mean=ymean, yhat=yhat.reshape(n, ndpost).T, varcount=vc.reshape(p, ndpost).T,
                text=None if buf is None else buf.raw[:ln.value].decode(), text_len=ln.value, moves=moves,
                raw_text_buffer=buf)


@pytest.mark.parametrize("kind", ["fwbart", "fpbart"])
def test_fbart_matches_batch_entry_point_in_r_layouts(kind):
    if kind == "fwbart":
        ch = W.fwbart_friedman(n=777, p=5, seed=8, ntree=25, nskip=30, ndpost=12)
    else:
        ch = W.fpbart_hazard(n=1501, seed=9, ntree=10, nskip=30, ndpost=12)
    nskip, ndpost = 30, 12
    p = np.asarray(ch["q"]).shape[0]
    ref = fit_batch([ch], nskip, ndpost)[0]
    text = F.trees_text(ref["trees"], p)
    # first call: sizes the text (trees_text = NULL); second call: fills a buffer of text_len + 1 bytes
    a = _fbart(ch, nskip, ndpost, text=False)
    assert a["text_len"] == len(text)
    b = _fbart(ch, nskip, ndpost, text=a["text_len"] + 1)
    assert b["text"] == text
    assert b["raw_text_buffer"].raw[a["text_len"]] == 0   # NUL-terminated
    for o in (a, b):
        assert np.array_equal(o["sigma"], ref["sigma"])
        assert np.array_equal(o["yhat_mean"], ref["yhat_mean"])
        assert np.array_equal(o["yhat"], ref["yhat"])                       # yhat.train[dr, i]
        assert np.array_equal(o["varcount"], F.varcount(ref["trees"], p))  # varcount[dr, v]
        assert np.array_equal(o["moves"], ref["moves"])
    assert a["moves"][0] > 0 and a["moves"][1] > 0


def test_fbart_small_text_buffer_is_truncated_and_terminated():
    ch = W.fwbart_friedman(n=300, p=3, seed=10, ntree=8, nskip=10, ndpost=4)
    full = _fbart(ch, 10, 4, text=False)
    cut = _fbart(ch, 10, 4, text=33)
    assert cut["text_len"] == full["text_len"]          # the full length is reported
    assert cut["raw_text_buffer"].raw[32] == 0          # at most cap bytes, NUL-terminated
    ref = F.trees_text(fit_batch([ch], 10, 4)[0]["trees"], 3)
    assert cut["raw_text_buffer"].raw[:32].decode() == ref[:32]


def test_fbart_rejects_codes_outside_a_byte():
    ch = W.fwbart_friedman(n=100, p=2, seed=11, ntree=4, nskip=2, ndpost=2)
    bad = dict(ch)
    q = np.asarray(ch["q"], np.int32).copy()
    q[1, 7] = 256
    bad["q"] = q
    with pytest.raises(F.FastbartError, match="outside 0..255") as e:
        _fbart(bad, 2, 2, text=False)
    assert e.value.status == _lib.FB_ERR_LIMIT
