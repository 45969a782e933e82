"""Generates the golden fixtures of tests/golden/ from the reference's own sampler.

The reference sampler src/bart_kernel.cpp is built from its sources by oracle/Makefile into oracle/_ref/libbartref.so
(-DFAST_CPU, the internal xoshiro128** generator) and run on small seeded chains; its outputs (sigma draws, posterior
mean, packed kept trees, move counts) and inputs are stored as .npz.  The oracle's REF mode must reproduce them bit
for bit (tests/test_oracle.py), which pins the oracle to the reference without needing the reference at test time.

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
