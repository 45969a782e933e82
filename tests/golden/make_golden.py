"""Generates the golden fixtures of tests/golden/ from the reference's own sampler and evaluator.

The reference sampler src/bart_kernel.cpp is built from its sources by oracle/Makefile into oracle/_ref/libbartref.so
(-DFAST_CPU, the internal xoshiro128** generator) and run on small seeded chains; its outputs (sigma draws, posterior
mean, packed kept trees, move counts) and inputs are stored as .npz.  The oracle's REF mode must reproduce them bit
for bit (tests/test_oracle.py), which pins the oracle to the reference without needing the reference at test time.

The reference evaluator src/predict.cpp (compile_trees_cpp, predict_draw_cpp) is built unmodified by oracle/Makefile
into oracle/_ref/libpredref.so against a stand-in for its few Rcpp types; ref_predict_*.npz hold its compiled node
arrays and its predictions of every draw on newdata with values on cutpoints, NaN and infinities.

Usage: python tests/golden/make_golden.py   (needs the reference checkout; writes tests/golden/*.npz)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fastbart_b200 import workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {
    # name: (builder, kwargs)
    "ref_wbart_a": (W.fwbart_friedman, dict(n=300, p=5, seed=3, ntree=20, nskip=40, ndpost=20)),
    "ref_wbart_ragged": (W.fwbart_friedman, dict(n=37, p=3, seed=5, ntree=7, nskip=30, ndpost=9, numcut=10)),
    "ref_wbart_p1": (W.fwbart_friedman, dict(n=200, p=1, seed=7, ntree=10, nskip=20, ndpost=10, numcut=255)),
    "ref_pbart_a": (W.fpbart_hazard, dict(n=500, seed=2, ntree=10, nskip=30, ndpost=10)),
}

SCALARS = ("tau", "lambda", "nu", "sigest", "offset", "seed", "probit", "ntree", "nskip", "ndpost")


def main():
    O.build()
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libbartref.so is missing: the reference sources are needed")
    for name, (fn, kw) in CASES.items():
        ch = fn(**kw)
        out = O.ref_fit(ch)
        arrays = {k: np.asarray(ch[k]) for k in ("q", "y", "wt", "numcut", "pgtab") if ch.get(k) is not None}
        if ch.get("ybin") is not None:
            arrays["ybin"] = np.asarray(ch["ybin"])
        arrays.update({f"s_{k}": np.asarray(ch[k]) for k in SCALARS})
        arrays.update({f"out_{k}": np.asarray(v) for k, v in out.items()})
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        print(name, "moves", out["moves"], "sigma[-1]", out["sigma"][-1])


PREDICT_CASES = ("ref_predict_fit", "ref_predict_dup")


def _predict_case(name):
    """(tree text, cutpoints, newdata [n][p], mu) of a predict fixture."""
    rng = np.random.default_rng(7 if name == "ref_predict_fit" else 8)
    if name == "ref_predict_fit":   # the kept draws of a small reference fit on its own cutpoints
        ch = W.fwbart_friedman(n=400, p=5, seed=13, ntree=15, nskip=60, ndpost=12)
        out = O.ref_fit(ch)
        text, cps, mu = O.trees_text(out["trees"], 5), [np.asarray(c) for c in ch["xi"]], 0.7
    else:                           # prior-grown forest on cutpoints with a repeated value (ties between cutpoints)
        p, ncut = 6, 25
        cps = [np.sort(rng.random(ncut)) for _ in range(p)]
        cps[0][3] = cps[0][2]
        cps[4][10] = cps[4][11]
        trees = W.random_forest(9, 21, p, ncut, seed=19, base=0.9, power=0.8, max_depth=5)
        text, mu = O.trees_text(trees, p), -0.25
    p = len(cps)
    n = 1500
    x = rng.random((n, p))
    for v in range(p):
        lo, hi = float(cps[v][0]) if len(cps[v]) else 0.0, float(cps[v][-1]) if len(cps[v]) else 1.0
        x[:, v] = lo + (hi - lo) * rng.random(n) * 1.2 - 0.1 * (hi - lo)
        hit = rng.random(n) < 0.25                  # exactly on a cutpoint: x >= cut goes right
        x[hit, v] = cps[v][rng.integers(0, len(cps[v]), hit.sum())]
    x[::53, 0] = np.nan
    x[5::61, 1] = np.inf
    x[7::67, 2] = -np.inf
    return text, cps, x, mu


def make_predict():
    if not O.ref_predict_available():
        raise SystemExit("oracle/_ref/libpredref.so is missing: the reference sources are needed")
    for name in PREDICT_CASES:
        text, cps, x, mu = _predict_case(name)
        R = O.RefCompiled(text, cps)
        cols = [np.ascontiguousarray(x[:, v]) for v in range(x.shape[1])]
        f = np.stack([R.predict_draw(cols, d, mu) for d in range(1, R.ndpost + 1)])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), text=np.frombuffer(text.encode(), np.uint8),
                            cut_flat=np.concatenate(cps), cut_len=np.array([len(c) for c in cps], np.int32), x=x,
                            mu=np.float64(mu), out=f, var=R.var, child=R.child, cut=R.cut, theta=R.theta, root=R.root)
        print(name, "draws", R.ndpost, "nodes", R.nnodes, "rows", x.shape[0])


def load_predict(name):
    """(text, cutpoints, x, mu, reference outputs [ndpost][n], reference compiled arrays) of a predict fixture."""
    z = np.load(os.path.join(HERE, name + ".npz"))
    offs = np.concatenate([[0], np.cumsum(z["cut_len"])])
    cps = [z["cut_flat"][offs[k]:offs[k + 1]] for k in range(len(z["cut_len"]))]
    arrays = {k: z[k] for k in ("var", "child", "cut", "theta", "root")}
    return bytes(z["text"]).decode(), cps, z["x"], float(z["mu"]), z["out"], arrays


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    ch = {k: z[k] for k in ("q", "y", "wt", "numcut", "pgtab", "ybin") if k in z}
    for k in SCALARS:
        v = z[f"s_{k}"]
        ch[k] = v.item()
    out = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return ch, out


if __name__ == "__main__":
    main()
    make_predict()
