"""GPU parity of the sampler: the fused per-tree pass and whole chains are bit-exact against the oracle's DEV
arithmetic on identical state.  Statistical agreement with the reference sampler at the benchmark shapes is in
test_gpu_parity_shapes.py."""
import ctypes as C

import numpy as np
import pytest

import fastbart_b200 as F
from fastbart_b200 import _lib, workloads as W
from fastbart_b200.api import fit_batch

pytestmark = pytest.mark.gpu


def _gpu_pass(n, lp, lc, r, w, qp, qc, upd, th, prop, apply, stats, leafmask, S, threads):
    st = _lib.PassState()
    st.n, st.apply, st.stats, st.fx_shift, st.threads = n, apply, stats, S, threads
    st.pmode, st.pnx, st.pc, st.pL, st.pR, st.pl, st.pr = (upd[k] for k in ("mode", "nx", "c", "L", "R", "l", "r"))
    st.cmode, st.cnx, st.cc = prop["mode"], prop["nx"], prop["c"]
    st.leafmask = int(leafmask)
    st.leaf_prev, st.leaf_cur, st.qprev, st.qcur = lp.ctypes.data, lc.ctypes.data, qp.ctypes.data, qc.ctypes.data
    st.r, st.w = r.ctypes.data, w.ctypes.data
    st.tho, st.thn, st.thc = th[0].ctypes.data, th[1].ctypes.data, th[2].ctypes.data
    out = np.zeros(70, dtype=np.int64)
    _lib.check(_lib.lib().fb_debug_tree_pass(C.byref(st), out.ctypes.data))
    return out


@pytest.mark.parametrize("n,nleaf,pmode,cmode,threads", [
    (1, 1, 0, 0, 64), (7, 2, 1, 1, 64), (1000, 1, 0, 1, 256), (1000, 3, 1, 1, 256), (4573, 5, 2, 1, 256),
    (4573, 8, 1, 2, 512), (3091, 9, 1, 1, 128), (20000, 17, 2, 1, 512), (65536, 32, 1, 1, 512),
    (24576, 2, 2, 0, 512)])
def test_tree_pass_bit_exact(orc, n, nleaf, pmode, cmode, threads):
    rng = np.random.default_rng(n * 7 + nleaf)
    slots = np.sort(rng.choice(np.arange(64), size=nleaf, replace=False)).astype(np.uint8)
    lc = rng.choice(slots, n).astype(np.uint8)
    lp = rng.choice(slots, n).astype(np.uint8)
    r = rng.normal(0, 3, n).astype(np.float32)
    w = rng.gamma(4, 0.25, n).astype(np.float32)
    qp = rng.integers(0, 100, n).astype(np.uint8)
    qc = rng.integers(0, 100, n).astype(np.uint8)
    th = [rng.normal(0, 1, 64).astype(np.float32) for _ in range(3)]
    upd = dict(mode=pmode, nx=int(lp[0]), v=0, c=40, L=int(rng.integers(1, 64)), R=int(rng.integers(1, 64)),
               l=int(lp[0]), r=int(lp[-1]))
    prop = dict(mode=cmode, nx=int(lc[0]), v=0, c=50)
    S = 30
    leafmask = sum(1 << int(s) for s in slots)
    lp_o, r_o = lp.copy(), r.copy()
    ref = orc.pass_dev(n, lp_o, lc, r_o, w, qp, qc, upd, th[0], th[1], 1, prop, th[2], S)
    lp_g, r_g = lp.copy(), r.copy()
    out = _gpu_pass(n, lp_g, lc, r_g, w, qp, qc, upd, th, prop, 1, 1, leafmask, S, threads)
    assert np.array_equal(lp_g, lp_o)
    assert np.array_equal(r_g.view(np.uint32), r_o.view(np.uint32))
    for s in slots:
        assert out[s] == ref["S1"][s], s
    if cmode == 1:
        assert np.array_equal(out[64:68], ref["split"])
        assert out[68] == ref["nL"] and out[69] == ref["nR"]


def _compare(a, b, keys=("sigma", "yhat_mean", "yhat", "trees", "moves")):
    m = {"yhat_mean": "fmean"}
    for k in keys:
        x, y = np.asarray(a[k]), np.asarray(b[k] if k in b else b[m[k]])
        assert x.shape == y.shape, k
        assert np.array_equal(x, y), f"{k}: first mismatch at {np.argwhere(x != y)[:3]}"


def test_chain_bit_exact_wbart(orc):
    ch = W.fwbart_friedman(n=300, p=5, seed=3, ntree=20, nskip=40, ndpost=20)
    g = fit_batch([ch], 40, 20)[0]
    o = orc.fit(ch, orc.MODE_DEV)
    _compare(g, o)


def test_chain_bit_exact_pbart(orc):
    ch = W.fpbart_hazard(n=1000, seed=2, ntree=10, nskip=30, ndpost=10)
    g = fit_batch([ch], 30, 10)[0]
    o = orc.fit(ch, orc.MODE_DEV)
    _compare(g, o)
    assert g["rtnorm_caps"] == o["rtnorm_caps"]


def test_batch_uneven_chains_bit_exact(orc):
    """Chains of uneven n, p and ntree, probit and weighted, in one launch; also ragged n (not a multiple of 4)."""
    chains = [W.fwbart_friedman(n=n, p=p, seed=s, ntree=m, nskip=15, ndpost=6)
              for n, p, m, s in [(37, 3, 7, 1), (513, 8, 30, 2), (1001, 4, 12, 3), (64, 2, 3, 4)]]
    chains.append(W.fpbart_hazard(n=777, seed=9, ntree=9, nskip=15, ndpost=6))
    outs = fit_batch(chains, 15, 6)
    for ch, g in zip(chains, outs):
        _compare(g, orc.fit(ch, orc.MODE_DEV))


def test_fit_batch_over_devices_equals_one_batch():
    """fit_batch(devices=...) partitions the chains (longest processing time first) and runs each share as its own
    batch from its own host thread; with the one GPU of this box listed twice, two batches run concurrently on it.
    Chains are independent, so every chain's outputs equal those of the single batch bit for bit, in chain order."""
    chains = [W.fwbart_friedman(n=n, p=4, seed=50 + n, ntree=15, nskip=10, ndpost=5) for n in (300, 1200, 700, 2000)]
    chains.append(W.fpbart_hazard(n=900, seed=57, ntree=8, nskip=10, ndpost=5))
    one = fit_batch(chains, 10, 5)
    two = fit_batch(chains, 10, 5, devices=[0, 0])
    assert len(two) == len(chains)
    for a, b in zip(one, two):
        _compare(b, a, keys=("sigma", "yhat_mean", "yhat", "trees", "moves"))


@pytest.mark.parametrize("threads,spl", [(64, 7), (512, 0)])
def test_launch_shape_does_not_change_results(orc, threads, spl):
    ch = W.fwbart_friedman(n=700, p=6, seed=21, ntree=25, nskip=20, ndpost=10)
    base = fit_batch([ch], 20, 10)[0]
    other = fit_batch([ch], 20, 10, threads=threads, sweeps_per_launch=spl)[0]
    _compare(other, base, keys=("sigma", "yhat_mean", "yhat", "trees", "moves"))


def test_staged_batch_repeats_identically():
    chains = W.titer_bootstrap(reps=2, shapes=[0, 5], nskip=10, ndpost=5, ntree=50)
    b = F.Batch(chains, 10, 5)
    b.run(); b.sync()
    a = b.download()
    b.run(); b.sync()
    c = b.download()
    for x, y in zip(a, c):
        _compare(x, y)
    b.close()


def test_probit_large_n_rows_in_global(orc):
    """n = 24,576 person-weeks (shared memory holds the rows) and n = 40,000 (rows stay in global memory)."""
    for n in (24576, 40000):
        ch = W.fpbart_hazard(n=n, seed=5, ntree=6, nskip=4, ndpost=3)
        g = fit_batch([ch], 4, 3, cluster=1)[0]
        _compare(g, orc.fit(ch, orc.MODE_DEV))


@pytest.mark.parametrize("cluster,spl", [(2, 0), (3, 0), (4, 7), (8, 0), (11, 0), (16, 5)])
def test_cluster_chains_bit_exact(orc, cluster, spl):
    """A chain split over a thread-block cluster (rows sliced across CTAs, totals through distributed shared memory)
    gives the one-CTA results bit for bit: weighted and probit chains, ragged n, slices with no rows (n 37 on 8 CTAs),
    resumed launches."""
    chains = [W.fwbart_friedman(n=5000, p=6, seed=41, ntree=20, nskip=12, ndpost=6),
              W.fpbart_hazard(n=3001, seed=42, ntree=8, nskip=12, ndpost=6),
              W.fwbart_friedman(n=37, p=3, seed=43, ntree=7, nskip=12, ndpost=6)]
    outs = fit_batch(chains, 12, 6, cluster=cluster, sweeps_per_launch=spl)
    for ch, g in zip(chains, outs):
        o = orc.fit(ch, orc.MODE_DEV)
        _compare(g, o)
        assert g["rtnorm_caps"] == o["rtnorm_caps"]


def test_cluster_rows_beyond_one_cta(orc):
    """n = 65,536 (one CTA keeps the rows in global memory; 8 CTAs hold 8,192 rows each in shared memory)."""
    ch = W.fwbart_friedman(n=65536, p=8, seed=44, ntree=10, nskip=3, ndpost=2)
    one = fit_batch([ch], 3, 2, cluster=1)[0]
    eight = fit_batch([ch], 3, 2, cluster=8)[0]
    _compare(eight, one)
    _compare(one, orc.fit(ch, orc.MODE_DEV))


def test_autotune_picks_a_shape_with_identical_results():
    chains = [W.fwbart_friedman(n=3000, p=6, seed=51 + k, ntree=20, nskip=8, ndpost=4) for k in range(3)]
    best = F.autotune(chains, 8, 4, trial_sweeps=2)
    assert best["threads"] in (256, 384, 416, 448, 512) and 1 <= best["cluster"] <= 16 and best["trial_ms"] > 0
    tuned = fit_batch(chains, 8, 4, threads=best["threads"], cluster=best["cluster"])
    plain = fit_batch(chains, 8, 4, cluster=1)
    for a, b in zip(tuned, plain):
        _compare(a, b)
