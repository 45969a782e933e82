"""GPU parity of compile_trees / predict_draw: bit-exact against the oracle's restatement of src/predict.cpp and
against golden vectors made by the reference's own src/predict.cpp (tests/golden/ref_predict_*.npz)."""
import numpy as np
import pytest

import fastbart_b200 as F
from fastbart_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_predict_draw_bit_exact_and_errors(orc):
    x, y = W.hazard_data(3000, 4)
    ch = W.fpbart_chain(x, y, ntree=12, nskip=20, ndpost=8, seed=3)
    g = F.fit_batch([ch], 20, 8)[0]
    text = F.trees_text(g["trees"], 3)
    assert text == orc.trees_text(g["trees"], 3)
    cps = ch["xi"]
    ct = F.CompiledTrees(text, cps, mu=ch["offset"])
    ref = orc.compile_trees(text, cps)
    arr = ct.arrays()
    for k in ("var", "child", "cut", "theta", "root"):
        assert np.array_equal(arr[k], getattr(ref, k)), k
    xn, _ = W.hazard_data(5000, 99)
    for d in (1, 4, 8):
        f = F.predict_draw(ct, xn, d)
        o = orc.predict_draw(ref, [xn[:, v] for v in range(3)], d, ch["offset"])
        assert np.array_equal(f, o)
    with pytest.raises(F.FastbartError, match="out of range"):
        F.predict_draw(ct, xn, 9)
    with pytest.raises(F.FastbartError, match="columns"):
        F.predict_draw(ct, xn[:, :2], 1)


def test_fwbart_object_and_predict_reproduces_yhat():
    x, y, w = W.friedman_data(800, 6, 12)
    fit = F.fwbart(x, y, w=w, ntree=30, nskip=50, ndpost=20, seed=5)
    assert fit.cls == "wbart"
    assert fit["yhat.train"].shape == (20, 800) and fit["sigma"].shape == (70,)
    assert fit["varcount"].shape == (20, 6)
    ct = F.compile_trees(fit)
    for d in (1, 20):
        f = F.predict_draw(ct, x, d)
        assert np.max(np.abs(f - fit["yhat.train"][d - 1])) < 1e-8
    assert np.corrcoef(fit["yhat.train.mean"], W.friedman(x))[0, 1] > 0.95


def test_fpbart_object():
    x, y = W.hazard_data(2000, 1)
    fit = F.fpbart(x, y, ntree=20, nskip=50, ndpost=20, seed=9)
    assert fit.cls == "pbart"
    assert fit["prob.train"].shape == (20, 2000)
    assert abs(fit["prob.train.mean"].mean() - y.mean()) < 0.05
    ct = F.compile_trees(fit)
    f = F.predict_draw(ct, x, 3)
    assert np.max(np.abs(f - fit["yhat.train"][2])) < 1e-8


@pytest.mark.parametrize("p, n, ndraws, dup", [(3, 1, 3, False), (5, 333, 7, False), (95, 300, 4, False),
                                                (120, 129, 2, False), (5, 333, 7, True), (95, 300, 4, True),
                                                (96, 300, 4, True)])
def test_bulk_predict_bit_exact_all_evaluators(orc, p, n, ndraws, dup):
    """Strictly increasing cutpoints run the code-compare evaluator; a repeated cutpoint (dup) forces the FP64
    comparisons: the tiled evaluator for p < 96, the streaming one beyond.  Ragged row tiles, several draws, x values
    that sit exactly on cutpoints."""
    import torch
    rng = np.random.default_rng(p * 1000 + n)
    ncut = 20
    cps = [np.sort(rng.random(ncut)) for _ in range(p)]
    if dup:
        cps[0][1] = cps[0][0]
    trees = W.random_forest(ndraws, 37, p, ncut, seed=p + n, base=0.9, power=0.8, max_depth=5)
    text = orc.trees_text(trees, p)
    ct = F.CompiledTrees(text, cps, mu=0.25)
    ref = orc.compile_trees(text, cps)
    x = rng.random((n, p))
    for v in range(p):   # some values exactly on a cutpoint (x >= cut goes right)
        hit = rng.random(n) < 0.2
        x[hit, v] = cps[v][rng.integers(0, ncut, hit.sum())]
    xd = torch.tensor(np.ascontiguousarray(x.T), device="cuda")
    out = torch.full((ndraws, n), float("nan"), dtype=torch.float64, device="cuda")
    F.predict_draws_device(ct, xd.data_ptr(), p, n, n, 1, ndraws, out.data_ptr(), n)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for d in range(ndraws):
        o = orc.predict_draw(ref, [x[:, v] for v in range(p)], d + 1, 0.25)
        assert np.array_equal(got[d], o), d
        assert np.array_equal(F.predict_draw(ct, x, d + 1), o)


@pytest.mark.parametrize("n,ndraws,ntree,change", [(1000, 40, 37, 0.25), (257, 9, 200, 0.0), (3001, 25, 50, 1.0)])
def test_carry_evaluator_bit_exact(orc, n, ndraws, ntree, change):
    """Draws shaped like consecutive posterior draws (most tree structures kept, every leaf value redrawn) run the
    evaluator that carries each row's leaves across draws; its results equal the oracle's for every draw, and the
    single-draw path's.  change 1.0 (independent draws) keeps the plain code-compare evaluator."""
    import torch
    p, ncut = 7, 20
    rng = np.random.default_rng(n + ndraws)
    cps = [np.sort(rng.random(ncut)) for _ in range(p)]
    trees = W.posterior_forest(ndraws, ntree, p, ncut, change=change, seed=n, base=0.95, power=1.0, max_depth=6)
    text = orc.trees_text(trees, p)
    ct = F.CompiledTrees(text, cps, mu=-0.5)
    ev, shared = ct.evaluator(n, ndraws)
    assert ev == ("codes_carry" if change < 0.5 else "codes"), (ev, shared)
    if change == 0.0:
        assert shared == (ndraws - 1) * ntree
    ref = orc.compile_trees(text, cps)
    x = rng.random((n, p))
    for v in range(p):
        hit = rng.random(n) < 0.2
        x[hit, v] = cps[v][rng.integers(0, ncut, hit.sum())]
    xd = torch.tensor(np.ascontiguousarray(x.T), device="cuda")
    out = torch.full((ndraws, n), float("nan"), dtype=torch.float64, device="cuda")
    F.predict_draws_device(ct, xd.data_ptr(), p, n, n, 1, ndraws, out.data_ptr(), n)
    # a range that starts inside the forest (its first draw walks every tree)
    out2 = torch.full((ndraws - 3, n), float("nan"), dtype=torch.float64, device="cuda")
    F.predict_draws_device(ct, xd.data_ptr(), p, n, n, 4, ndraws - 3, out2.data_ptr(), n)
    torch.cuda.synchronize()
    got, got2 = out.cpu().numpy(), out2.cpu().numpy()
    cols = [x[:, v] for v in range(p)]
    for d in range(ndraws):
        o = orc.predict_draw(ref, cols, d + 1, -0.5)
        assert np.array_equal(got[d], o), d
        if d >= 3:
            assert np.array_equal(got2[d - 3], o), d
    assert np.array_equal(F.predict_draw(ct, x, ndraws), got[-1])


def test_cut_codes_match_find_interval():
    """Device cut codes equal numpy searchsorted(side='right') (R's findInterval), ties and NaN included."""
    rng = np.random.default_rng(5)
    x, _ = W.hazard_data(10007, 8)
    d = F.prep.model_matrix(x, numcut=100)
    x[::97, 2] = np.nan
    x[::13, 0] = d.xi[0][rng.integers(0, d.xi[0].size, x[::13, 0].size)]   # values exactly on a cutpoint
    q = F.cut_codes(x[:, d.rm_const - 1], d.xi)
    for v in range(q.shape[0]):
        col = x[:, d.rm_const[v] - 1]
        ref = np.searchsorted(d.xi[v], col, side="right")
        ref[np.isnan(col)] = 0
        assert np.array_equal(q[v], ref.astype(np.uint8)), v


@pytest.mark.parametrize("name", ["ref_predict_fit", "ref_predict_dup"])
def test_predict_matches_reference_golden(name):
    """fb_compile_trees / fb_predict_draw / fb_predict_draws_device against golden vectors made by the reference's own
    src/predict.cpp: compiled arrays and every draw, bit for bit, on rows with values on cutpoints, NaN and
    infinities (the dup case has a repeated cutpoint, so it runs the FP64-compare evaluator)."""
    import os
    import sys
    import torch
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    text, cps, x, mu, out, arrays = make_golden.load_predict(name)
    ct = F.CompiledTrees(text, cps, mu=mu)
    got = ct.arrays()
    for k, v in arrays.items():
        assert np.array_equal(got[k], v), k
    for d in range(out.shape[0]):
        assert np.array_equal(F.predict_draw(ct, x, d + 1), out[d]), d
    n, p = x.shape
    xd = torch.tensor(np.ascontiguousarray(x.T), device="cuda")
    od = torch.full((out.shape[0], n), float("nan"), dtype=torch.float64, device="cuda")
    F.predict_draws_device(ct, xd.data_ptr(), p, n, n, 1, out.shape[0], od.data_ptr(), n)
    torch.cuda.synchronize()
    assert np.array_equal(od.cpu().numpy(), out)
