"""MCMC diagnostics: effective sample size by Geyer's initial monotone sequence estimator.

Geyer, C. J. (1992), "Practical Markov chain Monte Carlo", Statistical Science 7(4): sums of adjacent pairs of
autocovariances Gamma_k = gamma_{2k} + gamma_{2k+1} are truncated at the first non-positive pair and forced to be
non-increasing; ESS = n * gamma_0 / (-gamma_0 + 2 * sum_k Gamma_k).
"""
from __future__ import annotations

import numpy as np


def _autocov(x: np.ndarray) -> np.ndarray:
    """Autocovariances of each column of x ([n, k]) at lags 0..n-1 (biased, divisor n), by FFT."""
    n = x.shape[0]
    xc = x - x.mean(axis=0, keepdims=True)
    nfft = 1 << (2 * n - 1).bit_length()
    f = np.fft.rfft(xc, n=nfft, axis=0)
    ac = np.fft.irfft(f * np.conj(f), n=nfft, axis=0)[:n]
    return ac / n


def ess(x) -> np.ndarray:
    """ESS of each column of x (or of a single series).  Constant series get ESS = n."""
    a = np.asarray(x, dtype=np.float64)
    single = a.ndim == 1
    if single:
        a = a[:, None]
    n, k = a.shape
    g = _autocov(a)
    out = np.empty(k)
    for j in range(k):
        g0 = g[0, j]
        if not g0 > 0:
            out[j] = n
            continue
        m = (n - 1) // 2
        pairs = g[0:2 * m:2, j] + g[1:2 * m:2, j]
        s = 0.0
        prev = np.inf
        for P in pairs:
            if P <= 0:
                break
            P = min(P, prev)
            s += P
            prev = P
        tau = (-g0 + 2.0 * s) / g0
        out[j] = n / tau if tau > 0 else n
    out = np.minimum(out, n * np.log10(max(n, 10)))   # cap antithetic blow-ups (as common practice)
    return out[0] if single else out


def chain_ess(sigma_kept: np.ndarray, yhat: np.ndarray, rows: int = 256, seed: int = 0) -> dict:
    """ESS of the kept sigma draws and the median ESS of f over a fixed random sample of rows."""
    rng = np.random.default_rng(seed)
    n = yhat.shape[1]
    idx = rng.choice(n, size=min(rows, n), replace=False)
    ef = ess(yhat[:, idx])
    return dict(sigma=float(ess(sigma_kept)), f_median=float(np.median(ef)))
