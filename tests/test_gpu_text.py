"""Tree text assembled on the device (fb_trees_text_gpu, fb_batch_trees_text) against the host writer
fb_trees_text, whose "%.10g" is the C library's printf: the same bytes for fitted chains and for leaf values chosen
to reach every branch of the decimal conversion (ties, both output styles, subnormals, signed zero, inf, nan)."""
import numpy as np
import pytest

import fastbart_b200 as F
from fastbart_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _pack(v, c, l, r, th):
    th = np.asarray(th, np.float32).view(np.uint32).astype(np.uint64)
    return (np.uint64(v) | (np.uint64(c) << np.uint64(8)) | (np.uint64(l) << np.uint64(16))
            | (np.uint64(r) << np.uint64(24)) | (th << np.uint64(32)))


def _trees_with_leaves(values, ntree=10):
    """Trees of 5 nodes (root, an inner left child, three leaves) carrying the given leaf values, unused slots 255."""
    vals = np.asarray(values, np.float32)
    per = 3 * ntree
    nd = -(-len(vals) // per)
    vals = np.concatenate([vals, np.zeros(nd * per - len(vals), np.float32)]).reshape(nd, ntree, 3)
    T = np.full((nd, ntree, 64), 255, np.uint64)
    T[:, :, 0] = _pack(2, 17, 1, 2, 0.0)
    T[:, :, 1] = _pack(0, 3, 3, 4, 0.0)
    T[:, :, 2] = _pack(0, 0, 0, 0, vals[:, :, 0])
    T[:, :, 3] = _pack(0, 0, 0, 0, vals[:, :, 1])
    T[:, :, 4] = _pack(0, 0, 0, 0, vals[:, :, 2])
    return T


def test_fitted_chains_text_matches_host_writer():
    x, y = W.hazard_data(3000, 7)
    chains = [W.fwbart_friedman(n=800, p=9, seed=3, ntree=30, nskip=20, ndpost=12),
              W.fpbart_chain(x, y, ntree=20, nskip=20, ndpost=12, seed=5)]
    b = F.Batch(chains, 20, 12)
    b.run()
    b.sync()
    outs = b.download()
    for k, (ch, o) in enumerate(zip(chains, outs)):
        p = ch["q"].shape[0]
        host = F.trees_text(o["trees"], p)
        assert b.trees_text(k) == host
        assert F.trees_text_gpu(o["trees"], p) == host
    b.close()


def test_decimal_conversion_edge_values_match_printf():
    special = [0.0, -0.0, 1.0, -1.0, 0.1, 0.5, 1e-4, 1e-5, 0.0001, 0.00001, 9.9999997e-05, 1e10, 1e9, 9999999999.0,
               123456789.0, 1234567890.0, 12345678901.0, 1000000.0625, 1000000.1875, 1000000.3125, 524288.03125,
               3.4028235e38, -3.4028235e38, 1.1754944e-38, 1.4e-45, -1.4e-45, 2.5e-45, 9.8e-39, 1e-38, 3.0e-39,
               np.inf, -np.inf, 0.3, 2.0 / 3.0, 1.0 / 3.0, 65504.0, 16777216.0, 16777215.0, 99999.99, 0.099999994]
    vals = [np.float32(v) for v in special]
    vals += [np.uint32(u).view(np.float32) for u in (0x7fc00000, 0xffc00000, 0x00000001, 0x80000001, 0x007fffff,
                                                     0x00800000, 0x7f7fffff, 0x3f7fffff, 0x3dcccccd, 0x49742424)]
    rng = np.random.default_rng(11)
    bits = rng.integers(0, 2**32, 60000, dtype=np.uint64).astype(np.uint32)
    bits = bits[(bits & 0x7f800000) != 0x7f800000]          # finite bit patterns over the whole range
    vals += list(bits.view(np.float32))
    vals += list(rng.normal(0, 0.05, 20000).astype(np.float32))   # leaf-value-like magnitudes
    # values with exactly 11 significant digits ending in 5 (exact ties at the tenth digit): m / 16 near 1e6
    vals += [np.float32(m / 16.0) for m in range(16000000, 16000400)]
    T = _trees_with_leaves(vals)
    host = F.trees_text(T, 20)
    assert F.trees_text_gpu(T, 20) == host


def test_empty_and_root_only_trees():
    for nd, m in ((0, 5), (3, 0), (2, 4)):
        T = np.full((nd, m, 64), 255, np.uint64)
        if nd and m:
            T[:, :, 0] = _pack(255, 0, 0, 0, -0.25)
        assert F.trees_text_gpu(T, 4) == F.trees_text(T, 4)
