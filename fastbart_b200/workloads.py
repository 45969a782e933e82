"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference's own datasets (titer models, person-week hazard data) come from an external pipeline and are not
shipped, so these generators stand in for them with the same shapes, sizes and value distributions:

  fwbart_friedman   n 4,096, p 16, x ~ U(0,1), y = 10 sin(pi x1 x2) + 20 (x3 - .5)^2 + 10 x4 + 5 x5 + N(0,1),
                    w ~ Gamma(4, rate 4), numcut 100, ntree 200, nskip 1000, ndpost 100
  fpbart_hazard     n 24,576 person-weeks, p 3 (week 1..52, Bernoulli(.5), N(0,1)),
                    y ~ Bernoulli(Phi(-1.8 + .015 x1 + .5 x2 + .3 x3)), ntree 50, nskip 1000, ndpost 100
  titer_bootstrap   96 chains: 6 shapes (n, p) in {(3091,15), (3400,16), (3760,17), (4102,18), (4388,19), (4573,19)}
                    x 16 multinomial bootstrap resamples; half U(0,1) and half integer 0..9 columns;
                    y = linear term on 4 columns + sin(pi xa xb) + N(0, .5^2); w ~ Gamma(4, 4); ntree 200
  friedman_large    n 65,536, p 32, numcut 255, Friedman-5 on x1..x5 + N(0,1), 16 chains
  mixed_batch       256 chains in one batch: 128 fwbart chains of titer-like data (n uniform in 2,000..65,536, p in
                    8..32, ntree 200) and 128 fpbart chains of hazard data (n uniform in 4,096..24,576, ntree 50);
                    ten of the fwbart chains (p 32) share one cutpoint grid, so their kept draws pool into one
                    1,000-draw forest for bulk predict on fresh rows of the same distribution
  random_forest     posterior draws of trees grown from BART's tree prior (packed node format), for bulk predict
  posterior_forest  the same, shaped like consecutive draws of one chain (most tree structures kept from draw to draw)
"""
from __future__ import annotations

import numpy as np
from scipy import stats

from . import prep

TITER_SHAPES = [(3091, 15), (3400, 16), (3760, 17), (4102, 18), (4388, 19), (4573, 19)]


def friedman(x: np.ndarray) -> np.ndarray:
    """Friedman's function of the first five columns (columns beyond p count as 0.5)."""
    c = [x[:, k] if k < x.shape[1] else np.full(x.shape[0], 0.5) for k in range(5)]
    return 10 * np.sin(np.pi * c[0] * c[1]) + 20 * (c[2] - 0.5) ** 2 + 10 * c[3] + 5 * c[4]


def fwbart_chain(x, y, w=None, *, ntree=200, nskip=1000, ndpost=100, numcut=100, k=2.0, power=2.0, base=0.95,
                 sigdf=3.0, sigquant=0.9, seed=1, fmean=None, xinfo=None) -> dict:
    """Prepares one fwbart chain exactly as the R wrapper does (R/fwbart.R:8-27); returns the chain dict.  xinfo:
    fixed cutpoints per column (as R's xinfo argument), else the cutpoint rule of prep.cutpoints."""
    d = prep.model_matrix(x, numcut, True, xinfo)
    y = np.asarray(y, dtype=np.float64)
    n = y.size
    w = np.ones(n) if w is None else np.asarray(w, dtype=np.float64)
    fm = float(np.mean(y)) if fmean is None else float(fmean)
    yc = y - fm
    nu = float(sigdf)
    sig = prep.sigest_lm(d.X, yc)
    lam = sig * sig * stats.chi2.ppf(1.0 - sigquant, nu) / nu
    tau = (yc.max() - yc.min()) / (2 * k * np.sqrt(ntree))
    wt = 1.0 / (w * w)
    s, srss = prep.fx_shifts(n, wt, float(np.max(np.abs(yc))))
    return dict(q=d.q, y=yc, wt=wt, numcut=d.numcut, pgtab=prep.pg_table(base, power), tau=float(tau),
                **{"lambda": float(lam)}, nu=nu, sigest=float(sig), offset=0.0, seed=int(seed), probit=0,
                ntree=int(ntree), nskip=int(nskip), ndpost=int(ndpost), fx_shift=s, rss_shift=srss,
                fmean=fm, xi=d.xi, rm_const=d.rm_const)


def fpbart_chain(x, y, *, ntree=50, nskip=1000, ndpost=100, numcut=100, k=2.0, power=2.0, base=0.95,
                 binary_offset=None, seed=1, xinfo=None) -> dict:
    """Prepares one fpbart chain as R/fpbart.R:7-24 does."""
    d = prep.model_matrix(x, numcut, True, xinfo)
    y = np.asarray(y).astype(np.int32)
    n = y.size
    off = float(stats.norm.ppf(np.mean(y))) if binary_offset is None else float(binary_offset)
    tau = 3.0 / (k * np.sqrt(ntree))
    s, srss = prep.fx_shifts(n, np.ones(n), 10.0)
    return dict(q=d.q, y=np.zeros(n), wt=np.ones(n), ybin=y, numcut=d.numcut, pgtab=prep.pg_table(base, power),
                tau=float(tau), **{"lambda": 1.0}, nu=3.0, sigest=1.0, offset=off, seed=int(seed), probit=1,
                ntree=int(ntree), nskip=int(nskip), ndpost=int(ndpost), fx_shift=s, rss_shift=srss,
                binaryOffset=off, xi=d.xi, rm_const=d.rm_const)


def friedman_data(n=4096, p=16, seed=0, weights=True):
    rng = np.random.default_rng(seed)
    x = rng.random((n, p))
    y = friedman(x) + rng.standard_normal(n)
    w = rng.gamma(4.0, 1.0 / 4.0, n) if weights else np.ones(n)
    return x, y, w


def fwbart_friedman(n=4096, p=16, seed=0, **kw) -> dict:
    x, y, w = friedman_data(n, p, seed)
    kw.setdefault("seed", seed + 1)
    return fwbart_chain(x, y, w, **kw)


def hazard_data(n=24576, seed=0):
    rng = np.random.default_rng(seed)
    x1 = rng.integers(1, 53, n).astype(np.float64)
    x2 = rng.integers(0, 2, n).astype(np.float64)
    x3 = rng.standard_normal(n)
    eta = -1.8 + 0.015 * x1 + 0.5 * x2 + 0.3 * x3
    y = (rng.random(n) < stats.norm.cdf(eta)).astype(np.int32)
    return np.column_stack([x1, x2, x3]), y


def fpbart_hazard(n=24576, seed=0, **kw) -> dict:
    x, y = hazard_data(n, seed)
    kw.setdefault("seed", seed + 1)
    return fpbart_chain(x, y, **kw)


def titer_model(shape_idx: int, seed=0):
    """Base data of one titer-like model: half U(0,1), half integer 0..9 columns; y = a linear term on 4 columns
    (coefficients N(0,1)) + sin(pi xa xb) on two U(0,1) columns + N(0, 0.5^2); weights w ~ Gamma(4, rate 4)."""
    n, p = TITER_SHAPES[shape_idx]
    rng = np.random.default_rng(1000 + 17 * shape_idx + seed)
    x = np.empty((n, p))
    half = p // 2
    x[:, :half] = rng.random((n, half))
    x[:, half:] = rng.integers(0, 10, (n, p - half))
    lin = rng.choice(p, 4, replace=False)
    a, b = rng.choice(half, 2, replace=False)
    beta = rng.normal(0, 1, 4)
    y = x[:, lin] @ beta + np.sin(np.pi * x[:, a] * x[:, b]) + rng.normal(0, 0.5, n)
    w = rng.gamma(4.0, 1.0 / 4.0, n)
    return x, y, w


def titer_bootstrap(reps=16, shapes=range(6), seed=0, **kw) -> list:
    """The 96-chain batched workload: every shape x `reps` multinomial bootstrap resamples of its rows."""
    chains = []
    for si in shapes:
        x, y, w = titer_model(si, seed)
        n = y.size
        for r in range(reps):
            rng = np.random.default_rng(50_000 + 1000 * si + r + seed)
            idx = rng.integers(0, n, n)
            kw2 = dict(kw)
            kw2.setdefault("seed", 12345 + len(chains))
            chains.append(fwbart_chain(x[idx], y[idx], w[idx], **kw2))
    return chains


def titer_like(n: int, p: int, seed=0):
    """Titer-like data of any shape: the first p // 2 columns U(0,1), the rest integer 0..9; y = a linear term on 4
    columns (coefficients N(0,1)) + sin(pi xa xb) on two U(0,1) columns + N(0, 0.5^2); w ~ Gamma(4, rate 4)."""
    rng = np.random.default_rng(seed)
    half = p // 2
    x = np.empty((n, p))
    x[:, :half] = rng.random((n, half))
    x[:, half:] = rng.integers(0, 10, (n, p - half))
    lin = rng.choice(p, 4, replace=False)
    a, b = rng.choice(half, 2, replace=False)
    y = x[:, lin] @ rng.normal(0, 1, 4) + np.sin(np.pi * x[:, a] * x[:, b]) + rng.normal(0, 0.5, n)
    return x, y, rng.gamma(4.0, 1.0 / 4.0, n)


def titer_like_grid(p: int, numcut: int = 100) -> list:
    """The shared cutpoint grid of titer_like columns: numcut uniform interior points of (0, 1) for the U(0,1)
    columns, the midpoints 0.5 .. 8.5 for the integer columns."""
    half = p // 2
    u = np.arange(1, numcut + 1, dtype=np.float64) / (numcut + 1)
    return [u.copy() for _ in range(half)] + [np.arange(9, dtype=np.float64) + 0.5 for _ in range(p - half)]


MIXED_PREDICT_FITS = 10


def mixed_batch(seed=0, n_wbart=128, n_pbart=128, nskip=1000, ndpost=100, predict_fits=MIXED_PREDICT_FITS) -> list:
    """The mixed 256-chain workload (see the module docstring).  Chains 0 .. predict_fits-1 are the p = 32 fwbart
    fits on the shared grid of titer_like_grid(32)."""
    rng = np.random.default_rng(90_000 + seed)
    out = []
    for c in range(n_wbart):
        n = int(rng.integers(2000, 65537))
        p = 32 if c < predict_fits else int(rng.integers(8, 33))
        x, y, w = titer_like(n, p, seed=91_000 + 1000 * seed + c)
        xinfo = titer_like_grid(p) if c < predict_fits else None
        out.append(fwbart_chain(x, y, w, ntree=200, nskip=nskip, ndpost=ndpost, seed=500_000 + 1000 * seed + c,
                                xinfo=xinfo))
    for c in range(n_pbart):
        n = int(rng.integers(4096, 24577))
        x, y = hazard_data(n, seed=92_000 + 1000 * seed + c)
        out.append(fpbart_chain(x, y, ntree=50, nskip=nskip, ndpost=ndpost, seed=600_000 + 1000 * seed + c))
    return out


def friedman_large(nchains=16, n=65536, p=32, seed=0, **kw) -> list:
    x, y, w = friedman_data(n, p, seed, weights=False)
    out = []
    for c in range(nchains):
        kw2 = dict(kw)
        kw2.setdefault("seed", 777 + c)
        kw2.setdefault("numcut", 255)
        out.append(fwbart_chain(x, y, None, **kw2))
    return out


def _grow_tree(rng, p, nc, base, power, sd, max_depth) -> dict:
    """One tree from BART's tree prior as {slot: packed word}: a node at depth d splits with probability
    base / (1 + d)^power, on a uniform predictor and cut index; leaf values N(0, sd^2) as float."""
    words = {}
    free = list(range(1, 64))

    def grow(s, depth):
        if (depth < max_depth and len(free) >= 2 and p > 0
                and rng.random() < base / (1.0 + depth) ** power):
            l, r = free.pop(0), free.pop(0)
            v = int(rng.integers(p))
            c = int(rng.integers(max(int(nc[v]), 1)))
            words[s] = v | (c << 8) | (l << 16) | (r << 24)
            grow(l, depth + 1)
            grow(r, depth + 1)
        else:
            th = int(np.float32(rng.normal(0.0, sd)).view(np.uint32))
            words[s] = th << 32
    grow(0, 0)
    return words


def random_forest(ndpost: int, ntree: int, p: int, ncut, seed=0, base=0.95, power=2.0, sd=0.3,
                  max_depth=6) -> np.ndarray:
    """Packed trees [ndpost][ntree][64] (src/bart_kernel.cpp:559-571 format: v | c<<8 | l<<16 | r<<24 |
    float_bits(theta)<<32, v = 255 for unused slots), every tree grown independently from BART's tree prior.
    `ncut` is the cutpoint count of every predictor (an int, or one per predictor)."""
    rng = np.random.default_rng(seed)
    nc = np.broadcast_to(np.asarray(ncut, dtype=np.int64), (p,))
    out = np.full((ndpost, ntree, 64), 255, dtype=np.uint64)
    for d in range(ndpost):
        for t in range(ntree):
            for sl, wd in _grow_tree(rng, p, nc, base, power, sd, max_depth).items():
                out[d, t, sl] = np.uint64(wd)
    return out


def posterior_forest(ndpost: int, ntree: int, p: int, ncut, change=0.25, seed=0, base=0.95, power=2.0, sd=0.3,
                     max_depth=6) -> np.ndarray:
    """Packed trees [ndpost][ntree][64] shaped like consecutive posterior draws of one chain: draw 0 from BART's
    tree prior; each later draw keeps the previous draw's tree structures except a fraction `change` of the trees,
    which are grown again (BART accepts a move for a minority of its trees per sweep), and redraws every leaf value
    (as every sweep does)."""
    rng = np.random.default_rng(seed)
    nc = np.broadcast_to(np.asarray(ncut, dtype=np.int64), (p,))
    out = np.full((ndpost, ntree, 64), 255, dtype=np.uint64)
    for d in range(ndpost):
        regrow = np.ones(ntree, bool) if d == 0 else rng.random(ntree) < change
        if d > 0:
            kept = out[d - 1, ~regrow]
            leaf = ((kept & np.uint64(255)) != np.uint64(255)) & (((kept >> np.uint64(16)) & np.uint64(255)) == 0)
            th = rng.normal(0.0, sd, int(leaf.sum())).astype(np.float32).view(np.uint32).astype(np.uint64)
            kept = kept.copy()
            kept[leaf] = th << np.uint64(32)
            out[d, ~regrow] = kept
        for t in np.flatnonzero(regrow):
            for sl, wd in _grow_tree(rng, p, nc, base, power, sd, max_depth).items():
                out[d, t, sl] = np.uint64(wd)
    return out
