"""GPU parity of the learned cutpoint proposal (the cut head, drawn after the tree's fused pass from features that
include the node's residual mean and spread): whole chains with the cut head, alone or with the variable head, on
one CTA or a cluster, are bit-exact against the oracle's DEV arithmetic; the collected cut examples equal the
oracle's; the training kernels' gradients match the oracle's FP64 gradients; a trained head moves away from the
uniform cut, and chains with both learned heads target the same posterior as BART's proposal."""
import numpy as np
import pytest

import fastbart_b200 as F
from fastbart_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _bf16(a):
    a = np.asarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def random_cut(seed, scale=0.3, mix=0.5):
    rng = np.random.default_rng(seed)
    return dict(w1=_bf16(rng.normal(0, scale, (64, 40))), b1=rng.normal(0, 0.1, 64).astype(np.float32),
                w2=_bf16(rng.normal(0, scale, (64, 64))), b2=rng.normal(0, 0.1, 64).astype(np.float32),
                w3=_bf16(rng.normal(0, scale, (16, 64))), b3=rng.normal(0, 0.1, 16).astype(np.float32),
                emb=_bf16(rng.normal(0, 1.0, (255, 16))), be=rng.normal(0, 0.5, 255).astype(np.float32), mix=mix)


def random_model(seed, scale=0.3, mix=0.5):
    rng = np.random.default_rng(seed)
    return dict(w1=_bf16(rng.normal(0, scale, (64, 98))), b1=rng.normal(0, 0.1, 64).astype(np.float32),
                w2=_bf16(rng.normal(0, scale, (64, 64))), b2=rng.normal(0, 0.1, 64).astype(np.float32),
                w3=_bf16(rng.normal(0, scale, (32, 64))), b3=rng.normal(0, 0.5, 32).astype(np.float32), mix=mix)


def _run(ch, nskip, ndpost, cut=None, model=None, collect=0, cluster=0, threads=0):
    b = F.Batch([ch], nskip, ndpost, cluster=cluster, threads=threads)
    if model is not None:
        b.set_proposal(model)
    if cut is not None:
        b.set_cut_proposal(cut)
    if collect:
        b.collect(collect)
    b.run()
    b.sync()
    out = b.download()[0]
    data = (b.training_data(), b.cut_training_data()) if collect else None
    b.close()
    return out, data


def _same(out, ref):
    for k, r in (("sigma", "sigma"), ("yhat_mean", "fmean"), ("trees", "trees"), ("moves", "moves")):
        assert np.array_equal(np.asarray(out[k]), np.asarray(ref[r])), k


@pytest.mark.parametrize("kind,cluster,threads,vmodel", [
    ("wbart", 1, 0, False), ("wbart", 1, 0, True), ("wbart", 3, 0, True), ("wbart", 1, 256, False),
    ("pbart", 1, 0, False), ("pbart", 2, 0, True)])
def test_cut_chain_bit_exact(orc, kind, cluster, threads, vmodel):
    if kind == "wbart":
        ch = W.fwbart_friedman(n=1200, p=7, seed=12, ntree=20, nskip=30, ndpost=10)
    else:
        ch = W.fpbart_hazard(n=2000, seed=13, ntree=10, nskip=30, ndpost=10)
    cut = random_cut(7, mix=0.6)
    model = random_model(3, mix=0.5) if vmodel else None
    out, _ = _run(ch, 30, 10, cut=cut, model=model, cluster=cluster, threads=threads)
    ref = orc.fit(ch, orc.MODE_DEV, cut=cut, model=model)
    _same(out, ref)
    plain = orc.fit(ch, orc.MODE_DEV, model=model)
    assert not np.array_equal(plain["trees"], ref["trees"])   # the cut head does change the proposals


def test_cut_examples_bit_exact(orc):
    ch = W.fwbart_friedman(n=700, p=8, seed=14, ntree=25, nskip=40, ndpost=10)
    out, ((x, y, m, cnt), (cx, cc, lo, hi)) = _run(ch, 40, 10, collect=20000, cluster=1)
    ref = orc.fit(ch, orc.MODE_DEV, train_cap=20000)
    assert np.array_equal(out["sigma"], ref["sigma"])
    assert cnt == ref["moves"][0] == len(ref["train_c"])
    assert np.array_equal(cc, ref["train_c"]) and np.array_equal(lo, ref["train_lo"])
    assert np.array_equal(hi, ref["train_hi"])
    assert np.array_equal(cx.view(np.uint32), ref["train_cx"].view(np.uint32))
    assert np.all((cc >= lo) & (cc <= hi))


def test_cut_examples_of_a_learned_chain_bit_exact(orc):
    ch = W.fwbart_friedman(n=700, p=8, seed=15, ntree=25, nskip=30, ndpost=10)
    cut = random_cut(9)
    out, (_, (cx, cc, lo, hi)) = _run(ch, 30, 10, cut=cut, collect=20000, cluster=1)
    ref = orc.fit(ch, orc.MODE_DEV, cut=cut, train_cap=20000)
    _same(out, ref)
    assert np.array_equal(cc, ref["train_c"]) and np.array_equal(cx.view(np.uint32), ref["train_cx"].view(np.uint32))


def test_cut_gradients_match_oracle(orc):
    ch = W.fwbart_friedman(n=800, p=8, seed=16, ntree=25, nskip=40, ndpost=10)
    ref = orc.fit(ch, orc.MODE_DEV, train_cap=20000)
    x, c, lo, hi = (ref[k][:300] for k in ("train_cx", "train_c", "train_lo", "train_hi"))
    cut = random_cut(11, scale=0.2)
    loss, g = F.cut_loss_grad(cut, x, c, lo, hi)
    oloss, og = orc.cut_loss_grad(cut, x, c, lo, hi)
    assert abs(loss - oloss) <= 1e-4 * max(1.0, abs(oloss))
    for k in og:   # FP32 atomics and sums against FP64: relative to each gradient's scale
        tol = 2e-3 * max(np.abs(og[k]).max(), 1e-6)
        assert np.abs(g[k] - og[k]).max() <= tol, k


def test_cut_gradients_match_oracle_many_tiles(orc):
    # 6,000 examples: CTAs sum several 32-example tiles before their atomics
    rng = np.random.default_rng(22)
    n = 6000
    x = rng.random((n, 40), dtype=np.float32)
    lo = rng.integers(0, 200, n).astype(np.int32)
    hi = np.minimum(lo + rng.integers(0, 60, n), 254).astype(np.int32)
    c = (lo + (rng.random(n) * (hi - lo + 1)).astype(np.int32)).astype(np.int32)
    cut = random_cut(13, scale=0.2)
    loss, g = F.cut_loss_grad(cut, x, c, lo, hi)
    oloss, og = orc.cut_loss_grad(cut, x, c, lo, hi)
    assert abs(loss - oloss) <= 1e-4 * max(1.0, abs(oloss))
    for k in og:
        tol = 2e-3 * max(np.abs(og[k]).max(), 1e-6)
        assert np.abs(g[k] - og[k]).max() <= tol, k


def test_cut_training_and_posterior_unchanged(orc):
    # accepted births of plain chains teach both heads; chains with both learned heads agree with plain chains
    ch0 = W.fwbart_friedman(n=1500, p=16, seed=41, ntree=50, nskip=200, ndpost=100)
    b = F.Batch([ch0], 200, 100)
    b.collect(100000)
    b.run()
    b.sync()
    x, y, m, _ = b.training_data()
    cx, cc, lo, hi = b.cut_training_data()
    b.close()
    assert len(cc) == len(y) > 1000
    model, _ = F.train_proposal(x, y, m, epochs=10, batch=512, lr=3e-3, seed=2)
    cut, closs = F.train_cut_proposal(cx, cc, lo, hi, epochs=10, batch=512, lr=3e-3, seed=3)
    uniform = float(np.mean(np.log(hi - lo + 1.0)))
    assert closs[-1] < closs[0] and closs[-1] < uniform   # better than the uniform cut on its own examples
    fp, fl, sp, sl = [], [], [], []
    for k in range(4):
        ch = W.fwbart_friedman(n=1500, p=16, seed=41, ntree=50, nskip=600, ndpost=400)
        ch["seed"] = 700 + k
        a, _ = _run(ch, 600, 400)
        c, _ = _run(ch, 600, 400, model=model, cut=cut)
        fp.append(a["yhat_mean"]); fl.append(c["yhat_mean"])
        sp.append(a["sigma"][600:].mean()); sl.append(c["sigma"][600:].mean())
    assert np.corrcoef(np.mean(fp, axis=0), np.mean(fl, axis=0))[0, 1] > 0.995
    assert abs(np.mean(sl) / np.mean(sp) - 1) < 0.02


def test_cut_proposal_arguments():
    ch = W.fwbart_friedman(n=300, p=4, seed=17, ntree=5, nskip=2, ndpost=2)
    b = F.Batch([ch], 2, 2, threads=128, cluster=1)
    with pytest.raises(F.FastbartError, match="256 threads") as e:
        b.set_cut_proposal(random_cut(1))
    assert e.value.status == 2
    b.set_cut_proposal(None)   # restores BART's cut
    b.close()
    with pytest.raises(F.FastbartError, match="not in its range"):
        F.cut_loss_grad(random_cut(1), np.zeros((1, 40), np.float32), [9], [0], [5])
