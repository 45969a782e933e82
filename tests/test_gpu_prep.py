"""fb_sigma_estimate, the least-squares sigest of the preprocessing (R/fwbart.R:22: summary(lm(yc ~ X))$sigma, or
sd(yc) when p >= n), from FP64 Gram sums on the device: equal to the residual standard error of numpy's least-squares
fit to 1e-9 relative, with aliased columns dropped as lm drops them, ragged row counts and the p >= n case."""
import numpy as np
import pytest

import fastbart_b200 as F
from fastbart_b200 import prep, workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,p,kind", [(5000, 10, "uniform"), (70001, 32, "uniform"), (4573, 19, "titer"),
                                      (3000, 8, "aliased"), (200, 3, "uniform"), (10, 12, "wide")])
def test_sigma_estimate_matches_least_squares(n, p, kind):
    rng = np.random.default_rng(n + p)
    if kind == "titer":
        x, y, _ = W.titer_like(n, p, seed=3)
    else:
        x = rng.random((n, p))
        if kind == "aliased":   # a repeated column and an affine copy: two columns lm drops
            x[:, 3] = x[:, 1]
            x[:, 5] = 2.0 * x[:, 0] + 1.0
        y = x @ rng.normal(0, 1, p) + rng.normal(0, 0.7, n)
    yc = y - y.mean()
    s, rank = F.sigma_estimate(x, yc)
    ref = prep.sigest_lm(x, yc)
    assert abs(s - ref) <= 1e-9 * ref, (s, ref)
    if kind == "wide":
        assert rank == 0
    else:
        assert rank == np.linalg.matrix_rank(np.column_stack([np.ones(n), x]))
