"""Times the reference's own GPU prototype (gpu/bart_batch.cu, built unmodified for sm_100a into oracle/_ref/bart_batch
by oracle/Makefile) on the titer-shaped workload, as the reported reference-GPU baseline.

BASELINE/TEST INFRASTRUCTURE ONLY: nothing in the product calls this.  It writes the six titer-shaped models in the
input format of fpga/host_common.h:30-48 (<prefix>_meta.txt, _q.txt row-major codes, _yw.txt "y iw" with
wt = 1/iw^2, _ref_yhat.txt, _ref_sigma.txt) and runs the prototype in its two forms:

  batched   all 6 models x `reps` replicates in one launch sequence (one fit per thread block)
  single    one fit alone (model 6, the largest shape, one replicate): the plain one-chain-per-launch GPU form

The prototype draws its own bootstrap resamples (gpu/bart_batch.cu:321-323), so only the shapes match this project's
titer workload; chain-sweeps/s is comparable, the draws are not.  Its report line compares replicate 0 with the
posterior mean written to _ref_yhat.txt, here the reference CPU sampler's (oracle/_ref/libbartref.so) on the same rows.

Usage: python oracle/ref_gpu_bench.py [--reps 16] [--threads 256] [--out DIR]   (needs a GPU and oracle/_ref/bart_batch)
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# run as a script, this folder is on sys.path and its oracle.py would shadow the oracle/ folder
sys.path = [ROOT] + [q for q in sys.path if os.path.abspath(q or ".") != HERE]

import numpy as np  # noqa: E402

from fastbart_b200 import workloads as W  # noqa: E402

NSKIP, NDPOST = 1000, 100


def write_model(d: str, k: int, ch: dict, w: np.ndarray, ref: dict | None):
    pre = os.path.join(d, f"titer{k}")
    n, p = ch["q"].shape[1], ch["q"].shape[0]
    with open(pre + "_meta.txt", "w") as f:
        f.write(f"n {n}\np {p}\nfmean {ch['fmean']!r}\ntau {ch['tau']!r}\nlambda {ch['lambda']!r}\n")
        f.write(f"sigest {ch['sigest']!r}\nnu {ch['nu']!r}\nndpost {NDPOST}\nnskip {NSKIP}\n")
        f.write("numcut " + " ".join(str(int(c)) for c in ch["numcut"]) + "\n")
    np.savetxt(pre + "_q.txt", ch["q"].T.reshape(-1), fmt="%d")
    np.savetxt(pre + "_yw.txt", np.column_stack([ch["y"], w]), fmt="%.17g")
    yhat = ref["fmean"] if ref is not None else np.zeros(n)
    sig = ref["sigma"] if ref is not None else np.zeros(NSKIP + NDPOST)
    np.savetxt(pre + "_ref_yhat.txt", np.asarray(yhat, dtype=np.float64), fmt="%.17g")
    np.savetxt(pre + "_ref_sigma.txt", np.asarray(sig, dtype=np.float64), fmt="%.17g")


def _ref_fit(ch):
    from oracle import oracle as O
    return O.ref_fit(ch) if O.ref_available() else None


def run(exe: str, d: str, reps: int, threads: int, models: str, timeout: int) -> tuple[float, str]:
    t = time.perf_counter()
    p = subprocess.run([exe, d, str(reps), str(threads), models], capture_output=True, text=True, timeout=timeout)
    wall = time.perf_counter() - t
    if p.returncode != 0:
        raise RuntimeError(f"bart_batch exited {p.returncode}: {p.stderr[-500:]}")
    m = re.search(r"GPU time ([0-9.]+) s", p.stdout)
    if not m:
        raise RuntimeError("no GPU time in the output: " + p.stdout[-500:])
    return float(m.group(1)), p.stdout + f"(wall {wall:.1f} s)\n"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=16)
    ap.add_argument("--threads", type=int, default=256)
    ap.add_argument("--out", default=None, help="folder for the input files and logs (default: a new temporary folder)")
    ap.add_argument("--no-single", action="store_true")
    args = ap.parse_args()
    exe = os.path.join(HERE, "_ref", "bart_batch")
    if not os.path.exists(exe):
        print(json.dumps({"reference_gpu": "unavailable", "why": "oracle/_ref/bart_batch was not built"}))
        return 0
    if args.out is None:
        args.out = tempfile.mkdtemp(prefix="fastbart_refgpu_")
    os.makedirs(args.out, exist_ok=True)
    import multiprocessing as mp
    bases = []
    for si in range(6):
        x, y, w = W.titer_model(si)
        ch = W.fwbart_chain(x, y, w, nskip=NSKIP, ndpost=NDPOST, seed=12345 + si)
        bases.append((ch, w))
    with mp.get_context("spawn").Pool(6) as pool:
        refs = pool.map(_ref_fit, [c for c, _ in bases])
    for si, ((ch, w), ref) in enumerate(zip(bases, refs)):
        write_model(args.out, si + 1, ch, w, ref)
    S = NSKIP + NDPOST
    res = {"metric": "chain-sweeps/s", "threads_per_fit": args.threads, "sweeps": S, "ntree": 200}
    secs, log = run(exe, args.out, args.reps, args.threads, "1,2,3,4,5,6", 1800)
    nf = 6 * args.reps
    res["batched"] = {"fits": nf, "gpu_s": secs, "value": nf * S / secs}
    open(os.path.join(args.out, "batched.log"), "w").write(log)
    if not args.no_single:
        secs1, log1 = run(exe, args.out, 1, args.threads, "6", 900)
        res["single"] = {"fits": 1, "gpu_s": secs1, "value": S / secs1, "model": "n 4,573, p 19"}
        open(os.path.join(args.out, "single.log"), "w").write(log1)
    print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
