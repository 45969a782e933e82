"""Host-side preprocessing of fwbart()/fpbart(): model matrix, cutpoints, uint8 codes and priors.

Follows the steps of the reference R wrappers (R/fwbart.R:8-27, R/fpbart.R:7-20):
  * cutpoints per column, constant columns dropped (rm.const);
  * codes q[i, v] = findInterval(x[i, v], xi[v]), so that x < xi[v][c]  <=>  q <= c (0-based c);
  * fwbart: yc = y - fmean, sigest from a least-squares fit (residual standard error) or sd(yc) when p >= n,
    lambda = sigest^2 * qchisq(1 - sigquant, nu) / nu, tau = (max yc - min yc) / (2 k sqrt(ntree));
  * fpbart: binaryOffset = qnorm(mean(y)), tau = 3 / (k sqrt(ntree)), sigma fixed at 1;
  * tree prior table pgtab[d] = base / (1 + d)^power, d = 0..63.

The cutpoint rule is this project's: BART::bartModelMatrix is a third-party R function that is not available here.
A column with fewer than numcut + 1 distinct values gets the midpoints between consecutive distinct values; otherwise
numcut equally spaced interior points between its minimum and maximum.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from scipy import stats

NODES = 64
PMAX = 32
MMAX = 200
NMAX = 65536
NUMCUT_MAX = 255


@dataclass
class Design:
    X: np.ndarray                 # [n, p] numeric model matrix (constant columns removed)
    xi: list                      # per column: cutpoints (float64)
    numcut: np.ndarray            # [p] int32
    q: np.ndarray                 # [p, n] uint8 codes
    rm_const: np.ndarray          # 1-based indices of the kept columns (R's rm.const convention)
    colnames: list = field(default_factory=list)


def cutpoints(col: np.ndarray, numcut: int) -> np.ndarray:
    xs = np.unique(col)
    if xs.size <= 1:
        return np.zeros(0)
    if xs.size - 1 <= numcut:
        return (xs[:-1] + xs[1:]) / 2.0
    lo, hi = float(xs[0]), float(xs[-1])
    return lo + (hi - lo) * np.arange(1, numcut + 1, dtype=np.float64) / (numcut + 1)


def model_matrix(x, numcut: int = 100, rm_const: bool = True, xinfo=None) -> Design:
    X = np.asarray(x, dtype=np.float64)
    if X.ndim == 1:
        X = X[:, None]
    n, p0 = X.shape
    names = [f"x{j + 1}" for j in range(p0)]
    keep, xi = [], []
    for j in range(p0):
        cp = np.asarray(xinfo[j], dtype=np.float64) if xinfo is not None else cutpoints(X[:, j], numcut)
        if rm_const and np.unique(X[:, j]).size <= 1:
            continue
        keep.append(j)
        xi.append(cp)
    Xk = X[:, keep]
    q = np.zeros((len(keep), n), dtype=np.uint8)
    for v in range(len(keep)):
        if xi[v].size > NUMCUT_MAX:
            raise ValueError(f"column {keep[v] + 1} has {xi[v].size} cutpoints; at most {NUMCUT_MAX} are supported")
        q[v] = np.searchsorted(xi[v], Xk[:, v], side="right").astype(np.uint8)
    nc = np.array([c.size for c in xi], dtype=np.int32)
    return Design(Xk, xi, nc, q, np.array(keep, dtype=np.int64) + 1, [names[j] for j in keep])


def pg_table(base: float = 0.95, power: float = 2.0) -> np.ndarray:
    return base / (1.0 + np.arange(NODES, dtype=np.float64)) ** power


def sigest_lm(X: np.ndarray, yc: np.ndarray) -> float:
    """Residual standard error of the least-squares fit yc ~ 1 + X (summary(lm(...))$sigma), or sd(yc) if p >= n."""
    n, p = X.shape
    if p >= n:
        return float(np.std(yc, ddof=1))
    A = np.column_stack([np.ones(n), X])
    coef, _, rank, _ = np.linalg.lstsq(A, yc, rcond=None)
    res = yc - A @ coef
    return float(np.sqrt(res @ res / (n - rank)))


def fx_shifts(n: int, wt: np.ndarray, ymax: float) -> tuple[int, int]:
    """Fixed-point scales for the exact int64 row sums.

    Every per-row term fx(w*R) = llrint(w*R*2^S) and fx(w*e^2) = llrint(w*e^2*2^Srss) must stay far from int64
    overflow when summed over n rows.  The bound assumes |R|, |e| <= 64 (ymax + 1), well beyond any residual a chain
    reaches, and keeps 2 bits of headroom.
    """
    wmax = float(np.max(wt)) if wt.size else 1.0
    rb = 64.0 * (abs(ymax) + 1.0)
    s = 61 - int(np.ceil(np.log2(max(n, 1) * max(wmax, 1e-300) * rb + 1.0)))
    srss = 61 - int(np.ceil(np.log2(max(n, 1) * max(wmax, 1e-300) * rb * rb + 1.0)))
    return int(min(max(s, 8), 40)), int(min(max(srss, 0), 40))
