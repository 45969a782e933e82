"""CPU tests of the C ABI: the library loads, exports every function include/fastbart_b200.h declares, validates
arguments before touching a device, and its host-only functions (tree text, varcount) match the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest
import torch

import fastbart_b200 as F
from fastbart_b200 import _lib, workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "fastbart_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fb_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 19
    for f in names:
        assert hasattr(L, f), f
    assert set(names) == set(_lib.EXPORTS)
    assert "sm_100a" in F.version()


def _chain(**over):
    ch = W.fwbart_friedman(n=100, p=3, seed=1, ntree=5, nskip=2, ndpost=2)
    ch.update(over)
    return ch


@pytest.mark.parametrize("over,status,msg", [
    (dict(ntree=201), _lib.FB_ERR_LIMIT, "ntree"),
    (dict(numcut=np.array([256, 10, 10], np.int32)), _lib.FB_ERR_LIMIT, "numcut"),
    (dict(numcut=np.zeros(3, np.int32)), _lib.FB_ERR_ARG, "cutpoint"),
    (dict(tau=0.0), _lib.FB_ERR_ARG, "tau"),
    (dict(y=np.full(100, np.nan)), _lib.FB_ERR_ARG, "not finite"),
])
def test_argument_errors_before_device(over, status, msg):
    with pytest.raises(F.FastbartError, match=msg) as e:
        F.fit_batch([_chain(**over)], 2, 2)
    assert e.value.status == status


def test_limits_on_shape():
    big = dict(q=np.zeros((33, 10), np.uint8), numcut=np.ones(33, np.int32))
    with pytest.raises(F.FastbartError, match="predictors") as e:
        F.fit_batch([_chain(**big)], 2, 2)
    assert e.value.status == _lib.FB_ERR_LIMIT


def test_sigma_estimate_argument_errors():
    with pytest.raises(F.FastbartError, match="n >= 2") as e:
        F.sigma_estimate(np.zeros((1, 2)), np.zeros(1))
    assert e.value.status == _lib.FB_ERR_ARG
    with pytest.raises(F.FastbartError, match="at most 32") as e:
        F.sigma_estimate(np.zeros((40, 33)), np.zeros(40))
    assert e.value.status == _lib.FB_ERR_LIMIT


def test_latent_redraw_argument_errors():
    with pytest.raises(F.FastbartError, match="sweep") as e:
        F.probit_latent_device(1, 1, 10, 0.0, 1, -2, 1)
    assert e.value.status == _lib.FB_ERR_ARG
    with pytest.raises(F.FastbartError, match="required"):
        F.probit_latent_device(0, 0, 10, 0.0, 1, 0, 0)
    F.probit_latent_device(0, 0, 0, 0.0, 1, 0, 0)   # nothing to draw


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    with pytest.raises(F.FastbartError) as e:
        F.fit_batch([_chain()], 2, 2)
    assert e.value.status == _lib.FB_ERR_CUDA
    with pytest.raises(F.FastbartError):
        F.CompiledTrees("1 1 1\n1\n1 0 0 0.5\n", [np.array([0.5])])
    with pytest.raises(F.FastbartError) as e:   # non-null stand-ins: the device check comes before any access
        F.probit_latent_device(1, 1, 10, 0.0, 1, 0, 1)
    assert e.value.status == _lib.FB_ERR_CUDA


def test_text_and_varcount_match_oracle(orc):
    ch = W.fwbart_friedman(n=200, p=4, seed=2, ntree=12, nskip=30, ndpost=6)
    o = orc.fit(ch, orc.MODE_REF)
    assert F.trees_text(o["trees"], 4) == orc.trees_text(o["trees"], 4)
    assert np.array_equal(F.varcount(o["trees"], 4), orc.varcount(o["trees"], 4))


def test_text_format_of_a_known_tree():
    """A draw with one split: v 1, c 7, leaves 0.25 and -1.5 (pre-order ids 1, 2, 3; 10 significant digits)."""
    t = np.zeros((1, 1, 64), np.uint64)
    t[0, 0, 0] = np.uint64(1 | (7 << 8) | (1 << 16) | (2 << 24))
    t[0, 0, 1] = np.uint64(np.float32(0.25).view(np.uint32)) << np.uint64(32)
    t[0, 0, 2] = np.uint64(np.float32(-1.5).view(np.uint32)) << np.uint64(32)
    assert F.trees_text(t, 3) == "1 1 3\n3\n1 1 7 0\n2 0 0 0.25\n3 0 0 -1.5\n"
    assert F.varcount(t, 3).tolist() == [[0, 1, 0]]
