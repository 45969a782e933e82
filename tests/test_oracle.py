"""CPU tests of the oracle: pinned to the reference's own outputs (golden fixtures made by oracle/_ref) and to the
published known-answer vector of Philox4x32-10; sanity of the DEV arithmetic and of the evaluator restatement."""
import math
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402

from fastbart_b200 import workloads as W  # noqa: E402


@pytest.mark.parametrize("name", sorted(make_golden.CASES))
def test_ref_mode_matches_reference_golden(orc, name):
    """The oracle's REF mode reproduces bart_fit_cpu's outputs bit for bit (golden made by the reference itself)."""
    ch, ref = make_golden.load(name)
    out = orc.fit(ch, orc.MODE_REF)
    assert np.array_equal(out["sigma"], ref["sigma"])
    assert np.array_equal(out["fmean"], ref["fmean"])
    assert np.array_equal(out["trees"], ref["trees"])
    assert np.array_equal(out["moves"], ref["moves"])


@pytest.mark.parametrize("seed", [11, 12])
@pytest.mark.parametrize("probit", [0, 1])
def test_ref_mode_matches_reference_library(orc, seed, probit):
    """Live comparison with oracle/_ref/libbartref.so when the reference was built here."""
    if not orc.ref_available():
        pytest.skip("reference library not built (needs the reference sources)")
    if probit:
        ch = W.fpbart_hazard(n=333, seed=seed, ntree=8, nskip=25, ndpost=6)
    else:
        ch = W.fwbart_friedman(n=257, p=6, seed=seed, ntree=15, nskip=25, ndpost=8)
    a, b = orc.fit(ch, orc.MODE_REF), orc.ref_fit(ch)
    for k in ("sigma", "fmean", "trees", "moves"):
        assert np.array_equal(a[k], b[k]), k


def test_philox_known_answer(orc):
    # Random123 known-answer vector of philox4x32-10: counter 0, key 0
    assert orc.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]


def test_log_exp_accuracy(orc):
    xs = np.exp(np.linspace(-740, 700, 4001))
    for x in xs:
        if x != 1.0:
            assert abs(orc.log(x) - math.log(x)) <= 4e-16 * abs(math.log(x)) + 1e-300
    assert orc.log(1.0) == 0.0
    assert orc.log(5e-324) == pytest.approx(math.log(5e-324), rel=1e-15)
    for x in np.linspace(-745, 709, 4001):
        assert abs(orc.exp(x) - math.exp(x)) <= 2e-15 * math.exp(x) + 1e-323
    assert orc.exp(-800.0) == 0.0 and math.isinf(orc.exp(710.0))


def test_normal_gamma_rtnorm_moments(orc):
    z = np.array([orc.normal(99, (s << 8), 7, 3, 3) for s in range(20000)])
    assert abs(z.mean()) < 0.03 and abs(z.std() - 1) < 0.03
    g = np.array([orc.gamma(5 + k, k, 30.0) for k in range(4000)])
    assert abs(g.mean() - 30.0) < 0.4 and abs(g.var() - 30.0) < 3.0
    t = np.array([orc.rtnorm(3, i, 0, 0.0, 1.5)[0] for i in range(4000)])
    assert t.min() > 1.5
    ref = 0.0 + math.exp(-1.5**2 / 2) / math.sqrt(2 * math.pi) / (0.5 * math.erfc(1.5 / math.sqrt(2)))
    assert abs(t.mean() - ref) < 0.03


def test_oracle_probit_latent_truncation_and_moments(orc):
    # the latent redraw the GPU kernel is checked against: z on the side of -offset that ybin gives, row by row the
    # rtnorm of the sampler's counters, and N(f, 1) truncated to that side in distribution
    rng = np.random.default_rng(8)
    n, off = 20000, 0.4
    f = rng.normal(0.0, 0.5, n)
    yb = (rng.random(n) < 0.5).astype(np.int32)
    z, caps = orc.probit_latent(77, 12, off, f, yb)
    assert caps == 0
    assert np.all(z[yb == 1] > -off) and np.all(z[yb == 0] < -off)
    for i in (0, 1, 2, 999):
        one = orc.rtnorm(77, i, 12, f[i], -off)[0] if yb[i] else -orc.rtnorm(77, i, 12, -f[i], off)[0]
        assert one == z[i]
    c = np.zeros(n)   # fit 0: E[z | z > -off] for ybin 1
    z0, _ = orc.probit_latent(5, 0, off, c, np.ones(n, np.int32))
    a = -off
    ref = math.exp(-a * a / 2) / math.sqrt(2 * math.pi) / (0.5 * math.erfc(a / math.sqrt(2)))
    assert abs(z0.mean() - ref) < 0.02


def test_posterior_forest_keeps_structures_and_redraws_leaves():
    from fastbart_b200 import workloads as W
    t = W.posterior_forest(40, 50, 6, 20, change=0.25, seed=3)
    low = np.uint64(0xFFFFFFFF)
    same = np.array([np.all((t[d] & low) == (t[d - 1] & low), axis=1) for d in range(1, 40)])
    assert 0.65 < same.mean() < 0.85                      # about 1 - change of the trees keep their structure
    leaf = ((t & np.uint64(255)) != np.uint64(255)) & (((t >> np.uint64(16)) & np.uint64(255)) == np.uint64(0))
    kept = same[:, :, None] & leaf[1:]
    assert np.mean((t[1:] >> np.uint64(32))[kept] != (t[:-1] >> np.uint64(32))[kept]) > 0.99   # new leaf values


def _random_pass_state(rng, n, nleaf, pmode):
    slots = np.sort(rng.choice(np.arange(64), size=nleaf, replace=False)).astype(np.uint8)
    lc = rng.choice(slots, n).astype(np.uint8)
    lp = rng.integers(0, 64, n).astype(np.uint8)
    r = rng.normal(0, 3, n).astype(np.float32)
    w = rng.gamma(4, 0.25, n).astype(np.float32)
    qp = rng.integers(0, 50, n).astype(np.uint8)
    qc = rng.integers(0, 50, n).astype(np.uint8)
    th = [rng.normal(0, 1, 64).astype(np.float32) for _ in range(3)]
    upd = dict(mode=pmode, nx=int(lp[0]), v=0, c=25, L=int(rng.integers(1, 64)), R=int(rng.integers(1, 64)),
               l=int(lp[1]), r=int(lp[2]))
    prop = dict(mode=1, nx=int(slots[0]), v=0, c=20)
    return slots, lc, lp, r, w, qp, qc, th, upd, prop


def test_pass_dev_sums_are_exact(orc):
    """DEV pass: int64 sums equal brute-force sums of the per-row fixed-point terms."""
    rng = np.random.default_rng(0)
    n, S = 1000, 30
    slots, lc, lp, r, w, qp, qc, th, upd, prop = _random_pass_state(rng, n, 5, 1)
    lp0, r0 = lp.copy(), r.copy()
    st = orc.pass_dev(n, lp, lc, r, w, qp, qc, upd, th[0], th[1], 1, prop, th[2], S)
    # recompute in numpy: r -= delta, delta = thn[dest] - tho[src] (FP32); fx terms of (w 2^S) * R
    lf = lp0.astype(int)
    lf2 = lf.copy()
    sel = lf == upd["nx"]
    left = qp[sel] <= upd["c"]
    lf2[sel] = np.where(left, upd["L"], upd["R"])
    D = (th[1] - th[0]).astype(np.float32)
    delta = D[lf]
    delta[sel] = np.where(left, np.float32(th[1][upd["L"]] - th[0][upd["nx"]]), np.float32(th[1][upd["R"]] - th[0][upd["nx"]]))
    rr = (r0 - delta).astype(np.float32)
    assert np.array_equal(lp, lf2.astype(np.uint8)) and np.array_equal(r, rr)
    R = (rr + th[2][lc]).astype(np.float32)
    ws = (w * np.float32(2.0**S)).astype(np.float32)
    fx = np.rint((ws * R).astype(np.float32).astype(np.float64)).astype(np.int64)
    for s in slots:
        assert st["S1"][s] == fx[lc == s].sum()
    inx = lc == prop["nx"]
    left = inx & (qc <= prop["c"])
    assert st["nL"] == left.sum() and st["nR"] == (inx & ~left).sum()
    assert st["split"][1] == fx[left].sum() and st["split"][3] == fx[inx & ~left].sum()


def test_dev_mode_is_deterministic_and_sane(orc):
    ch = W.fwbart_friedman(n=400, p=5, seed=4, ntree=20, nskip=60, ndpost=30)
    a = orc.fit(ch, orc.MODE_DEV)
    b = orc.fit(ch, orc.MODE_DEV)
    for k in ("sigma", "fmean", "yhat", "trees", "moves"):
        assert np.array_equal(a[k], b[k])
    # yhat from the FP64 refresh equals glue.cpp's re-traversal of the packed kept trees
    assert np.array_equal(a["yhat"], orc.yhat_from_trees(a["trees"], ch["q"]))
    assert np.allclose(a["fmean"], a["yhat"].mean(axis=0), atol=1e-12)
    x, y, w = W.friedman_data(400, 5, 4)
    assert np.corrcoef(a["fmean"] + ch["fmean"], W.friedman(x))[0, 1] > 0.95


def test_text_compile_predict_roundtrip(orc):
    """Tree text -> compile_trees -> predict_draw on the training x reproduces yhat.train to 1e-8 (10-digit text)."""
    x, y, w = W.friedman_data(300, 4, 8)
    ch = W.fwbart_chain(x, y, w, ntree=10, nskip=20, ndpost=5, numcut=30, seed=5)
    a = orc.fit(ch, orc.MODE_DEV)
    text = orc.trees_text(a["trees"], 4)
    assert text.startswith("5 10 4\n")
    ct = orc.compile_trees(text, ch["xi"])
    cols = [x[:, v] for v in range(4)]
    for d in range(1, 6):
        f = orc.predict_draw(ct, cols, d, 0.0)
        assert np.max(np.abs(f - a["yhat"][d - 1])) < 1e-8
    with pytest.raises(ValueError, match="out of range"):
        orc.predict_draw(ct, cols, 6, 0.0)
    with pytest.raises(ValueError, match="columns"):
        orc.predict_draw(ct, cols[:3], 1, 0.0)
    vc = orc.varcount(a["trees"], 4)
    internal = np.array([[((a["trees"][d, j] >> np.uint64(16)) & np.uint64(255)) != 0 for j in range(10)]
                         for d in range(5)]).reshape(5, -1).sum(axis=1)
    assert np.array_equal(vc.sum(axis=1), internal)


def _rand_model(seed, scale=0.3, mix=0.5):
    rng = np.random.default_rng(seed)
    bf = lambda a: ((np.asarray(a, np.float32).view(np.uint32).astype(np.uint64) + 0x7FFF
                     + ((np.asarray(a, np.float32).view(np.uint32).astype(np.uint64) >> 16) & 1)) >> 16).astype(np.uint16)
    return dict(w1=bf(rng.normal(0, scale, (64, 98))), b1=rng.normal(0, 0.1, 64).astype(np.float32),
                w2=bf(rng.normal(0, scale, (64, 64))), b2=rng.normal(0, 0.1, 64).astype(np.float32),
                w3=bf(rng.normal(0, scale, (32, 64))), b3=rng.normal(0, 0.5, 32).astype(np.float32), mix=mix)


def test_oracle_model_proposal_and_collection(orc):
    """mix 0 is BART's proposal bit for bit; collected examples are the accepted births with valid labels."""
    ch = W.fwbart_friedman(n=300, p=7, seed=5, ntree=15, nskip=20, ndpost=10)
    plain = orc.fit(ch, orc.MODE_DEV, train_cap=10000)
    m0 = orc.fit(ch, orc.MODE_DEV, model=_rand_model(1, mix=0.0))
    assert np.array_equal(plain["sigma"], m0["sigma"]) and np.array_equal(plain["trees"], m0["trees"])
    assert len(plain["train_y"]) == plain["moves"][0] > 0
    assert all((mk >> yy) & 1 for mk, yy in zip(plain["train_mask"], plain["train_y"]))
    m5 = orc.fit(ch, orc.MODE_DEV, model=_rand_model(1, mix=0.5))
    assert np.isfinite(m5["sigma"]).all() and m5["moves"][0] > 0


def test_oracle_mlp_gradient_finite_differences(orc):
    ch = W.fwbart_friedman(n=300, p=7, seed=5, ntree=15, nskip=20, ndpost=10)
    d = orc.fit(ch, orc.MODE_DEV, train_cap=10000)
    x, y, m = d["train_x"][:40], d["train_y"][:40], d["train_mask"][:40]
    model = _rand_model(2, scale=0.2)
    loss, g = orc.mlp_loss_grad(model, x, y, m)
    for key, idx in (("b3", 3), ("b2", 10), ("b1", 7), ("b3", 0)):
        h = 1e-3
        mp = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in model.items()}
        mm = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in model.items()}
        mp[key][idx] += h
        mm[key][idx] -= h
        fd = (orc.mlp_loss_grad(mp, x, y, m)[0] - orc.mlp_loss_grad(mm, x, y, m)[0]) / (
            float(mp[key][idx]) - float(mm[key][idx]))
        assert abs(fd - g[key][idx]) <= 2e-3 + 2e-2 * abs(g[key][idx]), (key, idx, fd, g[key][idx])


@pytest.mark.parametrize("name", make_golden.PREDICT_CASES)
def test_predict_oracle_matches_reference_golden(orc, name):
    """The oracle's restatement of compile_trees_cpp / predict_draw_cpp equals the reference's own src/predict.cpp
    (golden made by it): node arrays, and every draw on rows with values on cutpoints, NaN and infinities."""
    text, cps, x, mu, out, arrays = make_golden.load_predict(name)
    ct = orc.compile_trees(text, cps)
    for k, v in arrays.items():
        assert np.array_equal(getattr(ct, k), v), k
    cols = [np.ascontiguousarray(x[:, v]) for v in range(x.shape[1])]
    for d in range(out.shape[0]):
        assert np.array_equal(orc.predict_draw(ct, cols, d + 1, mu), out[d]), d


@pytest.mark.parametrize("seed", [3, 4])
def test_predict_oracle_matches_reference_library(orc, seed):
    """Live comparison with the reference evaluator built here (oracle/_ref/libpredref.so): arrays, predictions and
    the two error cases of src/predict.cpp:51-52."""
    if not orc.ref_predict_available():
        pytest.skip("reference evaluator not built (needs the reference sources)")
    rng = np.random.default_rng(seed)
    p, ncut = 4 + seed, 30
    cps = [np.sort(rng.normal(size=ncut)) for _ in range(p)]
    trees = W.random_forest(5, 17, p, ncut, seed=seed, base=0.9, power=0.8, max_depth=6)
    text = orc.trees_text(trees, p)
    ref = orc.RefCompiled(text, cps)
    ct = orc.compile_trees(text, cps)
    for k in ("var", "child", "cut", "theta", "root"):
        assert np.array_equal(getattr(ct, k), getattr(ref, k)), k
    x = rng.normal(size=(700, p))
    x[::11, 0] = cps[0][rng.integers(0, ncut, x[::11].shape[0])]
    cols = [x[:, v] for v in range(p)]
    for d in (1, 3, 5):
        assert np.array_equal(orc.predict_draw(ct, cols, d, 0.5), ref.predict_draw(cols, d, 0.5))
    with pytest.raises(ValueError, match="out of range"):
        ref.predict_draw(cols, 6, 0.0)
    with pytest.raises(ValueError, match="columns"):
        ref.predict_draw(cols[:-1], 1, 0.0)


def test_oracle_cut_head_forward_and_examples(orc):
    """The cut head's logits equal a float64 numpy forward of the same BF16 weights (to FP32 rounding); a collecting
    chain's cut examples lie in their ranges, carry the variable one-hot, and a chain with the cut head is
    deterministic and differs from BART's uniform cut."""
    rng = np.random.default_rng(3)

    def bf(a):
        return (np.asarray(a, np.float32).view(np.uint32) >> 16).astype(np.uint16)

    cut = dict(w1=bf(rng.normal(0, .3, (64, 40))), b1=rng.normal(0, .1, 64).astype(np.float32),
               w2=bf(rng.normal(0, .3, (64, 64))), b2=rng.normal(0, .1, 64).astype(np.float32),
               w3=bf(rng.normal(0, .3, (16, 64))), b3=rng.normal(0, .1, 16).astype(np.float32),
               emb=bf(rng.normal(0, 1, (255, 16))), be=rng.normal(0, .5, 255).astype(np.float32), mix=0.5)
    f = {k: (v.astype(np.uint32) << 16).view(np.float32).astype(np.float64) if v.dtype == np.uint16 else
         v.astype(np.float64) for k, v in cut.items() if k != "mix"}
    x = rng.random(40).astype(np.float32)
    h1 = np.maximum(f["w1"] @ x + f["b1"], 0)
    h2 = np.maximum(f["w2"] @ h1 + f["b2"], 0)
    e = f["w3"] @ h2 + f["b3"]
    z = f["emb"] @ e + f["be"]
    zo = orc.cut_logits(cut, x, 3, 200)
    assert np.allclose(zo[3:201], z[3:201], rtol=1e-4, atol=1e-4)
    ch = W.fwbart_friedman(n=600, p=6, seed=5, ntree=15, nskip=30, ndpost=10)
    o = orc.fit(ch, orc.MODE_DEV, train_cap=5000)
    assert len(o["train_c"]) == o["moves"][0] > 0
    assert np.all((o["train_lo"] <= o["train_c"]) & (o["train_c"] <= o["train_hi"]))
    assert np.array_equal(np.argmax(o["train_cx"][:, 8:], axis=1), o["train_y"])
    a, b = orc.fit(ch, orc.MODE_DEV, cut=cut), orc.fit(ch, orc.MODE_DEV, cut=cut)
    assert np.array_equal(a["trees"], b["trees"])
    assert not np.array_equal(a["trees"], orc.fit(ch, orc.MODE_DEV)["trees"])
