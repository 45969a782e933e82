"""GPU parity of the learned split-variable proposal: collected training examples and whole chains with a model are
bit-exact against the oracle's DEV arithmetic; the training kernels' gradients match the oracle's FP64 gradients;
training on accepted births learns the signal predictors; and the learned chain targets the same posterior as BART's
proposal (the exact proposal probabilities enter the Metropolis-Hastings ratio)."""
import numpy as np
import pytest

import fastbart_b200 as F
from fastbart_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _bf16(a):
    a = np.asarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def random_model(seed, scale=0.3, mix=0.5):
    rng = np.random.default_rng(seed)
    return dict(w1=_bf16(rng.normal(0, scale, (64, 98))), b1=rng.normal(0, 0.1, 64).astype(np.float32),
                w2=_bf16(rng.normal(0, scale, (64, 64))), b2=rng.normal(0, 0.1, 64).astype(np.float32),
                w3=_bf16(rng.normal(0, scale, (32, 64))), b3=rng.normal(0, 0.5, 32).astype(np.float32), mix=mix)


def _run(ch, nskip, ndpost, model=None, collect=0, cluster=0, threads=0):
    b = F.Batch([ch], nskip, ndpost, cluster=cluster, threads=threads)
    if model is not None:
        b.set_proposal(model)
    if collect:
        b.collect(collect)
    b.run()
    b.sync()
    out = b.download()[0]
    data = b.training_data() if collect else None
    b.close()
    return out, data


@pytest.mark.parametrize("cluster", [1, 4])
def test_collected_examples_bit_exact(orc, cluster):
    ch = W.fwbart_friedman(n=500, p=9, seed=4, ntree=25, nskip=40, ndpost=10)
    out, (x, y, m, cnt) = _run(ch, 40, 10, collect=20000, cluster=cluster)
    ref = orc.fit(ch, orc.MODE_DEV, train_cap=20000)
    assert np.array_equal(out["sigma"], ref["sigma"])          # collecting changes nothing in the chain
    assert cnt == ref["moves"][0] == len(ref["train_y"])
    assert np.array_equal(y, ref["train_y"]) and np.array_equal(m, ref["train_mask"])
    assert np.array_equal(x.view(np.uint32), ref["train_x"].view(np.uint32))


# threads 512: the weights staged in the pass bins; 256: behind the shared layout; cluster 2: split over two CTAs
@pytest.mark.parametrize("mix,cluster,threads", [(0.5, 1, 0), (1.0, 1, 0), (0.5, 2, 0), (0.5, 1, 256)])
def test_model_chain_bit_exact(orc, mix, cluster, threads):
    ch = W.fwbart_friedman(n=400, p=12, seed=8, ntree=20, nskip=30, ndpost=10)
    model = random_model(3, mix=mix)
    out, _ = _run(ch, 30, 10, model=model, cluster=cluster, threads=threads)
    ref = orc.fit(ch, orc.MODE_DEV, model=model)
    for k, r in (("sigma", "sigma"), ("yhat_mean", "fmean"), ("trees", "trees"), ("moves", "moves")):
        assert np.array_equal(np.asarray(out[k]), np.asarray(ref[r])), k
    plain = orc.fit(ch, orc.MODE_DEV)
    assert not np.array_equal(plain["trees"], ref["trees"])   # the model does change the proposals


def test_model_chain_collecting_examples_bit_exact(orc):
    # a learned chain that also collects its accepted births (the collecting kernel variant runs the model too)
    ch = W.fwbart_friedman(n=400, p=12, seed=9, ntree=20, nskip=30, ndpost=10)
    model = random_model(5, mix=0.5)
    out, (x, y, m, cnt) = _run(ch, 30, 10, model=model, collect=20000)
    ref = orc.fit(ch, orc.MODE_DEV, model=model, train_cap=20000)
    assert np.array_equal(out["sigma"], ref["sigma"]) and np.array_equal(out["trees"], ref["trees"])
    assert cnt == len(ref["train_y"]) and np.array_equal(y, ref["train_y"]) and np.array_equal(m, ref["train_mask"])
    assert np.array_equal(x.view(np.uint32), ref["train_x"].view(np.uint32))


def test_training_gradients_match_oracle(orc):
    ch = W.fwbart_friedman(n=500, p=9, seed=4, ntree=25, nskip=40, ndpost=10)
    ref = orc.fit(ch, orc.MODE_DEV, train_cap=20000)
    x, y, m = ref["train_x"][:300], ref["train_y"][:300], ref["train_mask"][:300]
    model = random_model(11, scale=0.2)
    loss, g = F.mlp_loss_grad(model, x, y, m)
    oloss, og = orc.mlp_loss_grad(model, x, y, m)
    assert abs(loss - oloss) <= 1e-4 * max(1.0, abs(oloss))
    for k in og:   # FP32 atomics and sums against FP64: relative to each gradient's scale
        tol = 2e-3 * max(np.abs(og[k]).max(), 1e-6)
        assert np.abs(g[k] - og[k]).max() <= tol, k


def test_training_gradients_match_oracle_many_tiles(orc):
    # 6,000 examples: 188 tiles of 32 on at most one CTA per SM, so CTAs sum several tiles before their atomics
    rng = np.random.default_rng(21)
    n = 6000
    x = rng.random((n, 98), dtype=np.float32)
    m = rng.integers(1, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    y = np.array([rng.choice(np.flatnonzero((int(v) >> np.arange(32)) & 1)) for v in m], np.int32)
    model = random_model(12, scale=0.2)
    loss, g = F.mlp_loss_grad(model, x, y, m)
    oloss, og = orc.mlp_loss_grad(model, x, y, m)
    assert abs(loss - oloss) <= 1e-4 * max(1.0, abs(oloss))
    for k in og:
        tol = 2e-3 * max(np.abs(og[k]).max(), 1e-6)
        assert np.abs(g[k] - og[k]).max() <= tol, k


def test_training_learns_the_signal_predictors(orc):
    # Friedman signal on x1..x5 among 16 predictors: accepted births concentrate on the signal
    chains = [W.fwbart_friedman(n=2000, p=16, seed=20 + k, ntree=50, nskip=150, ndpost=50) for k in range(4)]
    b = F.Batch(chains, 150, 50)
    b.collect(100000)
    b.run()
    b.sync()
    x, y, m, cnt = b.training_data()
    b.close()
    assert cnt == len(y) and len(y) > 2000
    model, losses = F.train_proposal(x, y, m, epochs=12, batch=512, lr=3e-3, seed=1)
    assert losses[-1] < losses[0] < np.log(16) + 0.05
    # the trained model's probability mass on the signal predictors at root nodes of fresh trees
    xr = np.zeros(98, np.float32)
    xr[1] = 11 / 16.0
    xr[34:50] = 1.0
    z = orc.mlp_logits(model, xr)
    q = np.exp(z[:16] - z[:16].max())
    q /= q.sum()
    frac = np.mean(y < 5)          # accepted births on the signal predictors (uniform proposals give 5/16)
    assert frac > 5 / 16 + 0.03
    assert q[:5].sum() > (5 / 16 + frac) / 2   # the model moves from uniform toward the accepted moves


def test_learned_chain_targets_the_same_posterior(orc):
    ch0 = W.fwbart_friedman(n=1500, p=16, seed=31, ntree=50, nskip=200, ndpost=100)
    b = F.Batch([ch0], 200, 100)
    b.collect(100000)
    b.run()
    b.sync()
    x, y, m, _ = b.training_data()
    b.close()
    model, _ = F.train_proposal(x, y, m, epochs=10, batch=512, lr=3e-3, seed=2)
    fp, fl, sp, sl = [], [], [], []
    for k in range(4):
        ch = W.fwbart_friedman(n=1500, p=16, seed=31, ntree=50, nskip=600, ndpost=400)
        ch["seed"] = 500 + k
        a, _ = _run(ch, 600, 400)
        c, _ = _run(ch, 600, 400, model=model)
        fp.append(a["yhat_mean"]); fl.append(c["yhat_mean"])
        sp.append(a["sigma"][600:].mean()); sl.append(c["sigma"][600:].mean())
    mp, ml = np.mean(fp, axis=0), np.mean(fl, axis=0)
    assert np.corrcoef(mp, ml)[0, 1] > 0.995
    assert abs(np.mean(sl) / np.mean(sp) - 1) < 0.02


@pytest.mark.parametrize("cluster", [1, 3])
def test_mixed_batch_with_model_bit_exact(orc, cluster):
    """The mixed configuration at test size: fwbart and fpbart chains of uneven n, p and ntree in one launch, all with
    the learned proposal; every chain equals its own oracle run bit for bit."""
    chains = [W.fwbart_friedman(n=900, p=8, seed=61, ntree=25, nskip=15, ndpost=6),
              W.fpbart_hazard(n=1500, seed=62, ntree=10, nskip=15, ndpost=6),
              W.fwbart_friedman(n=2300, p=14, seed=63, ntree=18, nskip=15, ndpost=6),
              W.fpbart_hazard(n=700, seed=64, ntree=7, nskip=15, ndpost=6)]
    model = random_model(21, mix=0.7)
    b = F.Batch(chains, 15, 6, cluster=cluster)
    b.set_proposal(model)
    b.run()
    b.sync()
    outs = b.download()
    b.close()
    for ch, o in zip(chains, outs):
        ref = orc.fit(ch, orc.MODE_DEV, model=model)
        for k, r in (("sigma", "sigma"), ("yhat_mean", "fmean"), ("trees", "trees"), ("moves", "moves")):
            assert np.array_equal(np.asarray(o[k]), np.asarray(ref[r])), k


def test_clearing_the_model_restores_bart_proposals(orc):
    # one batch: a learned run, then the model cleared (the plain kernel variant again), then the model set again
    ch = W.fwbart_friedman(n=600, p=10, seed=71, ntree=15, nskip=20, ndpost=5)
    model = random_model(8, mix=0.6)
    b = F.Batch([ch], 20, 5)
    runs = []
    for mdl in (model, None, model):
        b.set_proposal(mdl)
        b.run()
        b.sync()
        runs.append(b.download()[0])
    b.close()
    learned, plain = orc.fit(ch, orc.MODE_DEV, model=model), orc.fit(ch, orc.MODE_DEV)
    assert np.array_equal(runs[0]["trees"], learned["trees"]) and np.array_equal(runs[2]["trees"], learned["trees"])
    assert np.array_equal(runs[1]["trees"], plain["trees"]) and np.array_equal(runs[1]["sigma"], plain["sigma"])
