#!/usr/bin/env python
"""Benchmark of the batched BART sampler on B200: chain-sweeps/s (and ESS/s) of the 96-chain titer bootstrap workload.

Workload (one "step"): 96 fwbart chains of uneven size run to completion in one batch -- 6 model shapes
(n 3,091-4,573, p 15-19) x 16 multinomial bootstrap resamples, ntree 200, nskip 1000, ndpost 100 (1,100 sweeps each),
seeded synthetic data with the shapes of the reference's titer models.  Every step runs the whole MCMC on the device
from the initial state, producing all outputs (sigma draws, yhat.train draws, posterior mean, kept trees).

  python bench.py [--gpus N --steps K --warmup W]          this implementation (one rank per GPU under torchrun)
  python bench.py --impl reference [--steps K --warmup W]   the reference sampler (bart_fit_cpu, built from source
                                                            into oracle/_ref) on the host cores, one chain per core
  --workload sparse | probit | predict | learned | text     the other measured configurations: 16 chains of n 65,536
                                                            on clusters; one fpbart chain (n 24,576, p 3) and the
                                                            predict_draw of its draws; bulk predict_draw; learned vs
                                                            plain proposal; tree text of the fitted 96-chain batch

Timing: W untimed warm-up steps; K timed steps, each preceded (outside its event pair) by a write of 512 MiB to flush
L2; CUDA events on the launching stream; max over ranks.  Multi-GPU: every rank runs its own 96-chain batch (different
seeds), no collective on the data path ("weak" scaling); value = all ranks' chain-sweeps / max time.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "chain-sweeps/s (96 batched fwbart chains, titer bootstrap)"
UNIT = "chain-sweeps/s"
BYTES_PER_ROW_TREE = 16   # algorithmic bytes per row-tree visit of the fused pass (leaf ids 3, residual 8, w 4, code 1)
NSKIP, NDPOST, NTREE = 1000, 100, 200
WORKLOAD_NAME = "titer_bootstrap_96"


def workload(rank: int = 0, reps: int = 16, nskip=NSKIP, ndpost=NDPOST):
    from fastbart_b200 import workloads as W
    return W.titer_bootstrap(reps=reps, seed=rank, nskip=nskip, ndpost=ndpost, ntree=NTREE)


FULL_REF = True
N_RANGE, P_RANGE = [3091, 4573], [15, 19]


def set_workload(name: str):
    """'titer96' (the benchmark), 'small' (6 chains, one per shape, 40 sweeps: the profiling case) or 'sparse'
    (16 chains, n 65,536, p 32, numcut 255, Friedman-5 signal on 5 of 32 predictors: the large-n configuration, run
    on thread-block clusters; the automatic choice is 6 CTAs per chain)."""
    global NSKIP, NDPOST, NTREE, WORKLOAD_NAME, workload, METRIC, FULL_REF, N_RANGE, P_RANGE
    if name == "probit":
        NTREE = 50
        WORKLOAD_NAME, FULL_REF, N_RANGE, P_RANGE = "fpbart_hazard_24576", False, [24576, 24576], [3, 3]
        METRIC = "chain-sweeps/s (fpbart, n 24,576 person-weeks, p 3, ntree 50; then predict_draw of its 100 draws)"

        def probit(rank: int = 0, reps: int = 0, nskip=None, ndpost=None):
            from fastbart_b200 import workloads as W
            return [W.fpbart_hazard(n=24576, seed=rank, ntree=NTREE, nskip=NSKIP, ndpost=NDPOST)]
        workload = probit
    if name == "sparse":
        WORKLOAD_NAME, FULL_REF, N_RANGE, P_RANGE = "friedman_sparse_16x65536", False, [65536, 65536], [32, 32]
        METRIC = "chain-sweeps/s (16 fwbart chains, n 65,536, p 32)"

        def sparse(rank: int = 0, reps: int = 0, nskip=None, ndpost=None):
            from fastbart_b200 import workloads as W
            out = W.friedman_large(nchains=16, n=65536, p=32, seed=rank, nskip=NSKIP, ndpost=NDPOST, ntree=NTREE)
            for k, c in enumerate(out):
                c["seed"] = 100 + 16 * rank + k
            return out
        workload = sparse
    if name == "single":
        WORKLOAD_NAME, FULL_REF, N_RANGE, P_RANGE = "friedman_single_4096x16", True, [4096, 4096], [16, 16]
        METRIC = "chain-sweeps/s (one fwbart chain, n 4,096, p 16, ntree 200)"

        def single(rank: int = 0, reps: int = 0, nskip=None, ndpost=None):
            from fastbart_b200 import workloads as W
            return [W.fwbart_friedman(n=4096, p=16, seed=rank, ntree=NTREE, nskip=NSKIP, ndpost=NDPOST)]
        workload = single
    if name == "small":
        NSKIP, NDPOST, WORKLOAD_NAME = 30, 10, "titer_small_6x40"
        base = workload

        def small(rank: int = 0, reps: int = 1, nskip=None, ndpost=None):
            return base(rank, 1, NSKIP, NDPOST)
        workload = small


LATENT_ROWS = 1 << 24   # a streaming size well beyond L2: 16,777,216 rows x 20 B


def latent_redraw(F, ch, out, stream, args):
    """fpbart's latent redraw as a streaming kernel on its own (fb_probit_latent_device): at the chain's size (its
    posterior-mean fit, 24,576 rows) and over 16,777,216 rows (the fit tiled; inputs and output beyond L2, L2 flushed
    before each timed call), CUDA-event timed after warm-up calls.  Algorithmic bytes per row: fit 8 + outcome 4 +
    z 8."""
    import torch
    res = {}
    f0 = np.asarray(out["yhat_mean"], np.float64)   # the fit of the trees (the sampler's f, without the offset)
    y0 = np.asarray(ch["ybin"], np.int32)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    peak, peak_kind = measured_peak()
    for name, n in (("chain_rows", f0.size), ("rows_16M", LATENT_ROWS)):
        reps = -(-n // f0.size)
        fd = torch.tensor(np.tile(f0, reps)[:n], device="cuda")
        yd = torch.tensor(np.tile(y0, reps)[:n], device="cuda")
        zd = torch.empty(n, dtype=torch.float64, device="cuda")
        cap = torch.zeros(1, dtype=torch.int32, device="cuda")

        def run(sweep):
            F.probit_latent_device(fd.data_ptr(), yd.data_ptr(), n, float(ch["offset"]), int(ch["seed"]), sweep,
                                   zd.data_ptr(), cap.data_ptr(), stream.cuda_stream)
        for k in range(args.warmup):
            run(k)
        torch.cuda.synchronize()
        ms = []
        for k in range(max(args.steps, 3)):
            flush.zero_()
            a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            run(100 + k)
            c.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(c))
        sec = float(np.median(ms)) / 1000.0
        gbs = 20.0 * n / sec / 1e9
        z = zd.cpu().numpy()
        ok = bool(np.all(z[yd.cpu().numpy() == 1] > -float(ch["offset"])))
        res[name] = {"rows": int(n), "ms": 1000 * sec, "rows_per_s": n / sec, "achieved_gbs": gbs, "peak": peak,
                     "frac": gbs / peak, "peak_source": peak_kind, "capped": int(cap.item()), "truncation_ok": ok}
        del fd, yd, zd
    res["note"] = ("one thread per row (grid-stride, 8 CTAs of 256 per SM); each draw runs Philox and FP64 log/exp "
                   "in a rejection loop; algorithmic bytes 20 per row")
    return res


def predict_fresh_rows(F, ch, out, stream, device):
    """The probit configuration's second half: compile_trees of the fit's 100 kept draws, then predict_draw of every
    draw on a fresh 24,576-row table from the same distribution (FP64), timed with CUDA events on the device
    (fb_predict_draws_device, x and results resident), after one untimed call."""
    import torch
    from fastbart_b200 import workloads as W
    x, _ = W.hazard_data(24576, 999)
    ct = F.CompiledTrees(F.trees_text_gpu(out["trees"], x.shape[1], device), ch["xi"], mu=ch["offset"], device=device)
    n, p = x.shape
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).to("cuda")
    od = torch.empty((NDPOST, n), dtype=torch.float64, device="cuda")
    F.predict_draws_device(ct, xd.data_ptr(), p, n, n, 1, NDPOST, od.data_ptr(), n, stream.cuda_stream)
    a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    a.record(stream)
    for _ in range(reps):
        F.predict_draws_device(ct, xd.data_ptr(), p, n, n, 1, NDPOST, od.data_ptr(), n, stream.cuda_stream)
    c.record(stream)
    torch.cuda.synchronize()
    sec = a.elapsed_time(c) / 1000.0 / reps
    chk = F.predict_draw(ct, x, NDPOST)   # the single-draw entry point agrees with the bulk one
    assert np.array_equal(chk, od[NDPOST - 1].cpu().numpy()), "bulk and single-draw predict disagree"
    return {"row_draws_per_s": NDPOST * n / sec, "ms_per_call": 1000 * sec, "draws": NDPOST, "rows": n,
            "ntree": ch["ntree"], "hbm_gbs": (n * p * 8 + NDPOST * n * 8) / sec / 1e9,
            "evaluator": ct.evaluator(n, NDPOST)[0],
            "note": "all 100 draws on fresh rows in one fb_predict_draws_device call; x read once, results written once"}


# ------------------------------------------------------------------------------------------------ CPU reference
def _ref_worker(args):
    ch, sweeps = args
    from oracle import oracle as O
    ch = dict(ch)
    ch["nskip"], ch["ndpost"] = sweeps - 10, 10
    t = time.perf_counter()
    if O.ref_available():
        O.ref_fit(ch)
        kind = "reference"
    else:
        O.fit(ch, O.MODE_REF)
        kind = "port"
    return time.perf_counter() - t, kind


def _warm_worker(_):
    """Loads the CPU reference into a pool worker, so that the timed sample excludes process start-up."""
    from oracle import oracle as O
    return O.ref_available()


def _full_ref_chain(ch):
    """One full-length chain of the reference sampler: (posterior mean of f, mean sigma over the kept draws)."""
    from oracle import oracle as O
    r = O.ref_fit(ch) if O.ref_available() else O.fit(ch, O.MODE_REF)
    return r["fmean"], float(np.mean(r["sigma"][int(ch["nskip"]):]))


def cpu_sample_plan(ncores: int):
    sweeps = 300 if ncores <= 8 else max(40, 2400 // ncores)
    return sweeps


def stratified(chains, k: int):
    """The k-th chain of a sample spread over the workload's shapes: chains are grouped by (n, p) in order of first
    appearance, and the sample takes one chain of each group in turn."""
    groups: dict = {}
    for c in chains:
        groups.setdefault(np.asarray(c["q"]).shape, []).append(c)
    g = list(groups.values())
    grp = g[k % len(g)]
    return grp[(k // len(g)) % len(grp)]


def sample_chains(chains, ncores: int) -> list:
    """ncores chains spread over the workload: one per shape in turn (stratified), or, when there are more shapes than
    cores, every (shapes / ncores)-th shape."""
    nshape = len({np.asarray(c["q"]).shape for c in chains})
    if nshape <= ncores:
        return [stratified(chains, k) for k in range(ncores)]
    return [chains[(k * len(chains)) // ncores] for k in range(ncores)]


def run_cpu_sample(pool, chains, ncores, sweeps):
    picked = sample_chains(chains, ncores)
    tasks = [(c, sweeps) for c in picked]
    t = time.perf_counter()
    res = pool.map(_ref_worker, tasks)
    wall = time.perf_counter() - t
    return ncores * sweeps / wall, res[0][1], wall


def cpu_sample_text(chains, ncores, sweeps):
    picked = sample_chains(chains, ncores)
    shapes = sorted({np.asarray(c["q"]).shape[::-1] for c in picked})
    mean_n = float(np.mean([np.asarray(c["q"]).shape[1] for c in picked]))
    listed = f" {[list(x) for x in shapes]} (n, p)" if len(shapes) <= 8 else ""
    return (f"{ncores} chains (one per core) spread over {len(shapes)} of the workload's shapes{listed}, mean n "
            f"{mean_n:.0f}, {sweeps} sweeps each")


def config_of(chains):
    """The workload description shared by both arms (launch details of this implementation go to "launch")."""
    return {"workload": WORKLOAD_NAME, "chains_per_gpu": len(chains), "ntree": NTREE, "nskip": NSKIP,
            "ndpost": NDPOST, "n_range": N_RANGE, "p_range": P_RANGE,
            "l2": "inputs resident; the GPU arm flushes L2 (512 MiB write) before every timed step"}


def agreement_plan(chains):
    """One chain of each shape (its first bootstrap resample) for the agreement check against the reference: the
    batch's own chain and a second seed on the GPU, two seeds of the reference sampler on the CPU."""
    seen, picks = set(), []
    for k, c in enumerate(chains):
        sh = np.asarray(c["q"]).shape
        if sh not in seen:
            seen.add(sh)
            picks.append(k)
    refs = []
    for k in picks:
        for s in (0, 1):
            d = dict(chains[k])
            d["seed"] = 700_001 + 2 * k + s
            d["nskip"], d["ndpost"] = NSKIP, NDPOST
            refs.append(d)
    return picks, refs


def agreement(picks, gpu_main, gpu_second, ref_results):
    """Posterior-mean f correlation and sigma ratio against the reference, per shape: single chains (the batch's chain
    vs one reference seed), the reference's own seed-to-seed correlation, and both seeds pooled on each side."""
    corr = lambda a, b: float(np.corrcoef(a, b)[0, 1])
    per = []
    for i, k in enumerate(picks):
        (fa, sa), (fb, sb) = ref_results[2 * i], ref_results[2 * i + 1]
        g1, g2 = gpu_main[k], gpu_second[i]
        sg = 0.5 * (np.mean(g1["sigma"][NSKIP:]) + np.mean(g2["sigma"][NSKIP:]))
        per.append({"n": int(len(fa)), "r_f": corr(g1["yhat_mean"], fa), "ref_seed_spread": corr(fa, fb),
                    "r_f_pooled": corr(g1["yhat_mean"] + g2["yhat_mean"], fa + fb),
                    "sigma_ratio": float(sg / (0.5 * (sa + sb))), "ref_sigma_seed_ratio": float(max(sa, sb) / min(sa, sb))})
    col = lambda key: [x[key] for x in per]
    return {"shapes": len(per), "r_f_min": min(col("r_f")), "r_f_median": float(np.median(col("r_f"))),
            "ref_seed_spread_min": min(col("ref_seed_spread")),
            "ref_seed_spread_median": float(np.median(col("ref_seed_spread"))),
            "r_f_pooled_min": min(col("r_f_pooled")), "r_f_pooled_median": float(np.median(col("r_f_pooled"))),
            "sigma_ratio_min": min(col("sigma_ratio")), "sigma_ratio_max": max(col("sigma_ratio")),
            # over all shapes (geometric mean of the per-shape ratios): the per-shape ratios scatter by the reference's
            # own seed-to-seed spread, the pooled one carries the systematic difference
            "sigma_ratio_pooled": float(np.exp(np.mean(np.log(col("sigma_ratio"))))),
            "ref_sigma_seed_ratio_max": max(col("ref_sigma_seed_ratio")),
            "per_shape": per,
            "what": "one chain per shape; r_f = corr(posterior-mean f) of this sampler's chain and one reference "
                    "chain (full length); ref_seed_spread = the same between two reference seeds; pooled = two "
                    "seeds on each side; sigma_ratio = mean sigma over the kept draws, two seeds each; ref_sigma_seed_ratio = "
                    "the larger over the smaller mean sigma of the two reference seeds (bootstrap resamples hold "
                    "duplicated rows, and chains settle at sigma levels a few percent apart)"}


# ------------------------------------------------------------------------------------------------ clocks
class Clocks:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        load = [s for s in sm if mx and s > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per full-size launch of this workload from its committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", f"sampler_kernel_{WORKLOAD_NAME}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_launch_full:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ------------------------------------------------------------------------------------------------ reference arm
def bench_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    chains = workload(0)
    ncores = os.cpu_count() or 1
    sweeps = cpu_sample_plan(ncores)
    ctx = mp.get_context("spawn")
    with ctx.Pool(ncores) as pool:
        for _ in range(args.warmup):
            run_cpu_sample(pool, chains, ncores, sweeps)
        vals, kind, walls = [], "reference", []
        for _ in range(args.steps):
            v, kind, wall = run_cpu_sample(pool, chains, ncores, sweeps)
            vals.append(v); walls.append(wall)
    tot = sum(walls)
    value = ncores * sweeps * args.steps / tot
    sample = cpu_sample_text(chains, ncores, sweeps) + ", per step"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * tot / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_of(chains),
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------ our arm
def bench_ours(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    chains = workload(rank)
    S = NSKIP + NDPOST

    # CPU baseline before any CUDA work (the pool is spawned here, rank 0, N = 1 only)
    cpu = None
    full_ref = None
    pool = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ncores = os.cpu_count() or 1
        sweeps = cpu_sample_plan(ncores)
        pool = mp.get_context("spawn").Pool(ncores)
        pool.map(_warm_worker, range(ncores), chunksize=1)
        v, kind, wall = run_cpu_sample(pool, chains, ncores, sweeps)
        cpu = {"value": v, "unit": UNIT, "cores": ncores, "kind": kind,
               "sample": cpu_sample_text(chains, ncores, sweeps) + f" ({wall:.1f} s wall)"}
        if FULL_REF:   # agreement with the reference, full-length chains, while the GPU runs
            picks, ref_chains = agreement_plan(chains)
            full_ref = pool.map_async(_full_ref_chain, ref_chains)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    import fastbart_b200 as F
    from fastbart_b200 import diagnostics

    tuned = None
    if args.autotune:   # outside the timed region
        tuned = F.autotune(chains, NSKIP, NDPOST, trial_sweeps=3, device=local)
        args.threads, args.cluster = tuned["threads"], tuned["cluster"]
    b = F.Batch(chains, NSKIP, NDPOST, threads=args.threads, device=local, cluster=args.cluster)
    info = b.launch_info()
    stream = torch.cuda.current_stream()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(args.warmup):
        flush.zero_()
        b.run(stream.cuda_stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local)
    clocks.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t0 = time.perf_counter()
    for k in range(args.steps):
        flush.zero_()
        evs[k][0].record(stream)
        b.run(stream.cuda_stream)
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    step_ms = [a.elapsed_time(c) for a, c in evs]
    tot_ms = sum(step_ms)
    from fastbart_b200 import shard
    tot_ms = shard.max_over_ranks(tot_ms, device="cuda")
    units = len(chains) * S * args.steps * world
    value = units / (tot_ms / 1000.0)

    # outputs of the last run: ESS of sigma and f (Geyer initial monotone sequence)
    outs = b.download()
    ess_s, ess_f = [], []
    for o in outs:
        e = diagnostics.chain_ess(o["sigma"][NSKIP:], o["yhat"])
        ess_s.append(e["sigma"]); ess_f.append(e["f_median"])
    per_step_s = tot_ms / 1000.0 / args.steps
    ess_line = {"sigma_per_s": sum(ess_s) * world / per_step_s, "f_median_per_s": sum(ess_f) * world / per_step_s,
                "sigma_mean_ess": float(np.mean(ess_s)), "f_median_ess": float(np.mean(ess_f)), "kept": NDPOST}
    if WORKLOAD_NAME.startswith("fpbart"):   # probit: sigma is fixed at 1
        ess_line["sigma_per_s"] = ess_line["sigma_mean_ess"] = None
    predict = latent = None
    if WORKLOAD_NAME.startswith("fpbart"):
        predict = predict_fresh_rows(F, chains[0], outs[0], stream, local)
        latent = latent_redraw(F, chains[0], outs[0], stream, args)
    b.close()

    # roofline of the sampler kernel (one launch per step)
    alg = BYTES_PER_ROW_TREE * sum(np.asarray(c["q"]).shape[1] * (c["ntree"] + 1) for c in chains) * S
    launch_s = per_step_s / info["launches"]
    achieved = alg / launch_s / 1e9
    peak, peak_kind = measured_peak()
    traffic = profiled_traffic()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_source": peak_kind,
            "note": "algorithmic bytes 16 B per row-tree visit; the kernel is bound by serial control latency"}

    # end to end through the public C ABI with host buffers (pinned), every step: H2D inputs, MCMC, D2H outputs
    e2e = None
    if not args.no_e2e:
        from fastbart_b200 import api
        import ctypes as C
        from fastbart_b200 import _lib

        def pinned(shape, dtype):
            shape = (shape,) if isinstance(shape, (int, np.integer)) else tuple(shape)
            dt = np.dtype(dtype)
            t = torch.empty(int(np.prod(shape)) * dt.itemsize, dtype=torch.uint8, pin_memory=True)
            return t.numpy().view(dt).reshape(shape)

        keep: list = []
        pin_chains = []
        for c in chains:
            d = dict(c)
            for k in ("q", "y", "wt"):
                a = np.asarray(c[k])
                p_ = pinned(a.shape, a.dtype)
                p_[...] = a
                d[k] = p_
            pin_chains.append(d)
        arr = (_lib.Chain * len(pin_chains))(*[api._as_chain(c, keep) for c in pin_chains])
        outs_p = [api._alloc_out(c, NSKIP, NDPOST, True, alloc=pinned) for c in pin_chains]
        oarr = (_lib.ChainOut * len(outs_p))(*[s_ for _, s_ in outs_p])
        opt = _lib.Options(NSKIP, NDPOST, args.threads, 0, local, args.cluster)
        h2d = sum(np.asarray(c["q"]).nbytes + 8 * len(c["y"]) + 4 * len(c["y"]) + len(c["y"]) for c in chains)
        h2d += len(chains) * 1024
        d2h = sum(8 * S + 8 * len(c["y"]) * (1 + NDPOST) + 8 * NDPOST * c["ntree"] * 64 for c in chains)
        times = []
        for k in range(args.e2e_steps + 1):
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            _lib.check(_lib.lib().fb_fit_batch(arr, len(pin_chains), C.byref(opt), oarr))
            torch.cuda.synchronize()
            if k > 0:
                times.append(time.perf_counter() - t1)
        from fastbart_b200 import shard
        e2e_s = shard.max_over_ranks(sum(times), device="cuda") / len(times)
        e2e = {"value": len(chains) * S * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": len(times), "ms_per_step": 1000 * e2e_s,
               "api": "fb_fit_batch (host buffers; allocation, H2D, MCMC, D2H of sigma/yhat/yhat_mean/trees)"}

    # the plain one-chain-per-launch form of the same chains: one chain of each shape, each alone in its launch
    # (automatic shape for one chain), outside the timed region
    per_launch = None
    if rank == 0 and world == 1 and FULL_REF and not args.no_single:
        picks1 = agreement_plan(chains)[0]
        secs = []
        for k in picks1:
            b1 = F.Batch([chains[k]], NSKIP, NDPOST, device=local)
            b1.run(stream.cuda_stream)
            a1, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a1.record(stream)
            b1.run(stream.cuda_stream)
            c1.record(stream)
            torch.cuda.synchronize()
            secs.append(a1.elapsed_time(c1) / 1000.0)
            info1 = b1.launch_info()
            b1.close()
        rate = len(picks1) * S / sum(secs)
        per_launch = {"chain_sweeps_per_s": rate, "chains_timed": len(picks1), "batched_over_per_launch": value / rate,
                      "shape": f"{info1['threads']} threads x {info1['cluster']} CTA(s) per chain (automatic)",
                      "what": "one chain of each shape per launch, device-timed: the plain one-chain-per-launch form"}

    r_f = None
    if full_ref is not None:
        ref_res = full_ref.get(timeout=900)
        picks, ref_chains = agreement_plan(chains)
        second = []
        for k in picks:   # a second GPU seed of the same chain (outside the timed region)
            d = dict(chains[k])
            d["seed"] = int(d["seed"]) + 1_000_003
            second.append(d)
        gs2 = F.fit_batch(second, NSKIP, NDPOST, device=local, trees=False)
        r_f = agreement(picks, outs, gs2, ref_res)
        pool.close()
    if pool is not None:
        pool.terminate()

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int64-fixed+f32+f64", "data": "synthetic",
                "config": config_of(chains),
                "launch": {"threads": info["threads"], "grid": info["grid"], "smem_bytes": info["smem"],
                           "ctas_per_chain": info["cluster"],
                           "shape": "autotuned" if (tuned or info["autotuned"]) else "rules"},
                "e2e": e2e, "gpu_launches": args.steps * info["launches"], "roofline": roof, "cpu_baseline": cpu,
                "clocks": clk, "ess_per_s": ess_line, "agreement_with_reference": r_f,
                "one_chain_per_launch": per_launch, "wall_s": wall}
        if predict is not None:
            line["predict_draw"] = predict
        if latent is not None:
            line["latent_redraw"] = latent
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------------------------------------ bulk predict
PRED_DRAWS, PRED_ROWS, PRED_P, PRED_CPU_ROWS = 1000, 1_000_000, 32, 100_000
PRED_METRIC = "predict_draw row-draws/s (1,000 draws x 200 trees on 1,000,000 rows x 32 FP64 columns)"
PRED_UNIT = "row-draws/s"
PRED_CHANGE = 0.15   # share of trees whose structure changes from one posterior draw to the next (posterior leg)


def _pred_newdata(rows: int, seed: int = 21):
    return np.random.default_rng(seed).random((rows, PRED_P))


def _pred_cpu_worker(a):
    """One draw of the oracle's restatement of predict_draw_cpp on a sample of rows (one core)."""
    text, cps, rows, draw, mu = a
    from oracle import oracle as O
    ct = O.compile_trees(text, cps)
    x = _pred_newdata(rows)
    cols = [np.ascontiguousarray(x[:, v]) for v in range(PRED_P)]
    t = time.perf_counter()
    O.predict_draw(ct, cols, draw, mu)
    return time.perf_counter() - t


def _pred_cpu_sample(pool, text, cps, mu, ncores):
    t = time.perf_counter()
    secs = pool.map(_pred_cpu_worker, [(text, cps, PRED_CPU_ROWS, 1 + k % PRED_DRAWS, mu) for k in range(ncores)])
    wall = time.perf_counter() - t
    return ncores * PRED_CPU_ROWS / max(max(secs), 1e-9), wall


def _pred_forest():
    """A seeded synthetic posterior of 1,000 draws x 200 trees grown from BART's tree prior (base 0.95, power 2)
    on 32 predictors with 100 uniform cutpoints each, as BART tree text with its cutpoints (no fit needed, so both
    arms see the same forest)."""
    import fastbart_b200 as F
    from fastbart_b200 import workloads as W
    trees = W.random_forest(PRED_DRAWS, 200, PRED_P, 100, seed=11)
    cps = [np.arange(1, 101, dtype=np.float64) / 101.0 for _ in range(PRED_P)]
    return F.trees_text(trees, PRED_P), cps, 0.5, trees


def walk_steps(trees: np.ndarray) -> float:
    """Node steps the code-compare evaluator executes per row and draw: per group of four consecutive trees, four
    walks of the group's deepest leaf (averaged over the draws of the packed forest [D][T][64])."""
    t = np.asarray(trees, dtype=np.uint64)
    used = (t & np.uint64(255)) != np.uint64(255)
    lch = ((t >> np.uint64(16)) & np.uint64(255)).astype(np.int64)
    rch = ((t >> np.uint64(24)) & np.uint64(255)).astype(np.int64)
    D, T, S = t.shape
    depth = np.full((D, T, S), -1, np.int64)
    depth[:, :, 0] = 0
    di, ti = np.meshgrid(np.arange(D), np.arange(T), indexing="ij")
    for _ in range(S):   # children one level below their parents, until nothing changes
        inner = used & (lch > 0) & (depth >= 0)
        if not inner.any():
            break
        old = depth.copy()
        for ch in (lch, rch):
            d_, t_, s_ = np.nonzero(inner)
            depth[d_, t_, ch[d_, t_, s_]] = depth[d_, t_, s_] + 1
        if np.array_equal(old, depth):
            break
    tdep = depth.max(axis=2)                       # [D][T]
    G = (T + 3) // 4
    pad = np.zeros((D, 4 * G), np.int64)
    pad[:, :T] = tdep
    return float((4 * pad.reshape(D, G, 4).max(axis=2)).sum(axis=1).mean())


def bench_predict(args):
    global PRED_DRAWS, PRED_ROWS
    if args.pred_rows:
        PRED_ROWS = int(args.pred_rows)
    if args.pred_draws:
        PRED_DRAWS = int(args.pred_draws)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference" and rank != 0:
        return 0
    import fastbart_b200 as F
    text, cps, mu, ptrees = _pred_forest()
    impl_ref = args.impl == "reference"
    cpu = None
    if rank == 0 and (impl_ref or (world == 1 and not args.no_cpu_baseline)):
        ncores = os.cpu_count() or 1
        with mp.get_context("spawn").Pool(ncores) as pool:
            vals, walls = [], []
            for k in range((args.warmup + args.steps) if impl_ref else 1):
                v, wall = _pred_cpu_sample(pool, text, cps, mu, ncores)
                if not impl_ref or k >= args.warmup:
                    vals.append(v); walls.append(wall)
        cpu = {"value": float(np.mean(vals)), "unit": PRED_UNIT, "cores": ncores, "kind": "port",
               "sample": f"{ncores} draws, one per core, each on {PRED_CPU_ROWS:,} rows (the oracle's C restatement "
                         f"of predict_draw_cpp; the reference's own needs Rcpp)"}
    if impl_ref:
        if rank == 0:
            line = {"metric": PRED_METRIC, "value": cpu["value"], "unit": PRED_UNIT, "n_gpus": args.gpus,
                    "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * float(np.mean(walls)),
                    "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                    "config": {"workload": "predict_bulk_1000x1M"}, "impl": "reference", "cpu_baseline": cpu,
                    "e2e": {"value": cpu["value"], "unit": PRED_UNIT, "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        return 0
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    ct = F.CompiledTrees(text, cps, mu=mu, device=local)
    # device-resident inputs: x [32][1M] column-major, out [1000][1M]
    xh = _pred_newdata(PRED_ROWS, 21 + rank)
    xd = torch.tensor(np.ascontiguousarray(xh.T), device="cuda")
    out = torch.empty((PRED_DRAWS, PRED_ROWS), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    def run():
        F.predict_draws_device(ct, xd.data_ptr(), PRED_P, PRED_ROWS, PRED_ROWS, 1, PRED_DRAWS, out.data_ptr(),
                               PRED_ROWS, stream.cuda_stream)
    for _ in range(args.warmup):
        flush.zero_()
        run()
    torch.cuda.synchronize()
    # parity spot check of two draws on the first rows against the compiled-tree host arrays is in the tests; here the
    # first draw is compared with the single-draw host call on a slice
    chk = F.predict_draw(ct, xh[:2000], 1)
    assert np.array_equal(out[0, :2000].cpu().numpy(), chk), "bulk and single-draw predict disagree"
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()
        evs[k][0].record(stream)
        run()
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    tot_ms = sum(a.elapsed_time(b) for a, b in evs)
    from fastbart_b200 import shard
    tot_ms = shard.max_over_ranks(tot_ms, device="cuda")
    per_s = tot_ms / 1000.0 / args.steps
    value = PRED_DRAWS * PRED_ROWS * world / per_s
    alg = PRED_P * PRED_ROWS * 8 + PRED_DRAWS * PRED_ROWS * 8 + ct.nnodes * 12
    peak, peak_kind = measured_peak()
    roof = {"bound": "hbm", "achieved": alg / per_s / 1e9, "peak": peak, "unit": "GB/s",
            "frac": alg / per_s / 1e9 / peak, "traffic": None, "peak_source": peak_kind,
            "algorithmic_bytes": alg,
            "node_steps_note": "x read once, every output written once, each draw's packed nodes and leaf values read"}
    roof["evaluator"] = ct.evaluator(PRED_ROWS, PRED_DRAWS)[0]
    # the rate in tree visits and in the node steps the code-compare evaluator executes (per group of four trees, four
    # walks of the group's deepest leaf): the issue-bound figure to compare kernels by
    steps = walk_steps(ptrees)
    roof["tree_visits_per_s"] = value * 200
    roof["walk_steps_per_row_draw"] = steps
    roof["node_steps_per_s"] = value * steps
    # the same call on draws shaped like one chain's consecutive posterior draws (most tree structures kept from
    # draw to draw, every leaf value redrawn): the evaluator then carries each row's leaves across draws
    post = None
    if not args.no_posterior:
        from fastbart_b200 import workloads as W
        trees2 = W.posterior_forest(PRED_DRAWS, 200, PRED_P, 100, change=PRED_CHANGE, seed=12)
        ct2 = F.CompiledTrees(F.trees_text(trees2, PRED_P), cps, mu=mu, device=local)
        ev2, shared2 = ct2.evaluator(PRED_ROWS, PRED_DRAWS)

        def run2():
            F.predict_draws_device(ct2, xd.data_ptr(), PRED_P, PRED_ROWS, PRED_ROWS, 1, PRED_DRAWS, out.data_ptr(),
                                   PRED_ROWS, stream.cuda_stream)
        for _ in range(args.warmup):
            flush.zero_()
            run2()
        torch.cuda.synchronize()
        assert np.array_equal(out[-1, :2000].cpu().numpy(), F.predict_draw(ct2, xh[:2000], PRED_DRAWS)), \
            "bulk and single-draw predict disagree (posterior draws)"
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            run2()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        ms2 = shard.max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), device="cuda") / args.steps
        post = {"row_draws_per_s": PRED_DRAWS * PRED_ROWS * world / (ms2 / 1000.0), "ms_per_call": ms2,
                "evaluator": ev2, "shared_tree_fraction": shared2 / float(PRED_DRAWS * 200), "nodes": ct2.nnodes,
                "over_tree_prior_forest": (PRED_DRAWS * PRED_ROWS * world / (ms2 / 1000.0)) / value,
                "what": f"1,000 draws shaped like one chain's consecutive posterior draws ({PRED_CHANGE:.0%} of the "
                        f"trees grown again per draw, every leaf value redrawn; workloads.posterior_forest), same rows"}
        del ct2
    # end to end with host buffers: every step copies x (column-major, pinned) to the device, evaluates all draws
    # (fb_predict_draws_device) and copies every result back to pinned host memory
    e2e = None
    if not args.no_e2e:
        xhp = torch.empty((PRED_P, PRED_ROWS), dtype=torch.float64, pin_memory=True)
        xhp.copy_(torch.from_numpy(np.ascontiguousarray(xh.T)))
        outh = torch.empty((PRED_DRAWS, PRED_ROWS), dtype=torch.float64, pin_memory=True)
        xe = torch.empty_like(xd)

        def e2e_step():
            xe.copy_(xhp, non_blocking=True)
            F.predict_draws_device(ct, xe.data_ptr(), PRED_P, PRED_ROWS, PRED_ROWS, 1, PRED_DRAWS, out.data_ptr(),
                                   PRED_ROWS, stream.cuda_stream)
            outh.copy_(out, non_blocking=True)
        e2e_step()
        torch.cuda.synchronize()
        ed = 2
        t1 = time.perf_counter()
        for _ in range(ed):
            e2e_step()
        torch.cuda.synchronize()
        e2e_s = shard.max_over_ranks((time.perf_counter() - t1) / ed, device="cuda")
        assert np.array_equal(outh[0, :2000].numpy(), chk), "host copy of the bulk result disagrees"
        e2e = {"value": PRED_DRAWS * PRED_ROWS * world / e2e_s, "unit": PRED_UNIT,
               "h2d_bytes_per_step": PRED_P * PRED_ROWS * 8, "d2h_bytes_per_step": PRED_DRAWS * PRED_ROWS * 8,
               "steps": ed, "ms_per_step": 1000 * e2e_s,
               "api": "fb_predict_draws_device with pinned host x copied in and all 1,000 x 1 M results copied out"}
    if rank == 0:
        line = {"metric": PRED_METRIC, "value": value, "unit": PRED_UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "predict_bulk_1000x1M" if (PRED_DRAWS, PRED_ROWS) == (1000, 1_000_000)
                           else f"predict_bulk_{PRED_DRAWS}x{PRED_ROWS}", "draws": PRED_DRAWS, "ntree": 200,
                           "rows": PRED_ROWS, "p": PRED_P, "nodes": ct.nnodes,
                           "l2": "flushed (512 MiB write) before every timed step; inputs and outputs exceed L2"},
                "e2e": e2e, "gpu_launches": args.steps * (2 if post else 1), "roofline": roof, "cpu_baseline": cpu,
                "clocks": clk, "posterior_draws": post}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------------------------------------ tree text
TXT_METRIC = "BART tree text of the 96 fitted titer chains, assembled on the device and delivered as host strings"


def bench_text(args):
    """The output-assembly step after a fit: BART tree text (src/glue.cpp:29-57 format) of every chain of the fitted
    96-chain titer batch (100 draws x 200 trees each), assembled on the device from the kept trees there
    (fb_batch_trees_text) and returned as host strings.  The fit itself is not timed.  Baseline: the host C++ writer
    (fb_trees_text, snprintf) on downloaded trees, one thread, on a sample of 8 chains."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    import torch
    import fastbart_b200 as F
    from fastbart_b200 import workloads as W
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    chains = W.titer_bootstrap(reps=16, seed=0, nskip=NSKIP, ndpost=NDPOST, ntree=NTREE)
    b = F.Batch(chains, NSKIP, NDPOST)
    b.run()
    b.sync()

    def step():
        return [b.trees_text(k) for k in range(len(chains))]
    for _ in range(args.warmup):
        texts = step()
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    t = time.perf_counter()
    for _ in range(args.steps):
        texts = step()
    sec = (time.perf_counter() - t) / args.steps
    clk = clocks.stop()
    mb = sum(len(x) for x in texts) / 1e6
    outs = b.download()
    cpu = None
    if not args.no_cpu_baseline:
        t = time.perf_counter()
        host = [F.trees_text(o["trees"], c["q"].shape[0]) for o, c in zip(outs[:8], chains[:8])]
        hs = time.perf_counter() - t
        assert host == texts[:8], "device and host tree text differ"
        cpu = {"value": sum(len(x) for x in host) / 1e6 / hs, "unit": "MB/s", "cores": 1, "kind": "port",
               "sample": "host C++ writer (snprintf) on the downloaded trees of the first 8 chains"}
    b.close()
    line = {"metric": TXT_METRIC, "value": mb / sec, "unit": "MB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * sec, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 trees -> text", "data": "synthetic",
            "config": {"workload": "tree_text_titer96", "chains": len(chains), "ndpost": NDPOST, "ntree": NTREE,
                       "text_mb": mb},
            "e2e": {"value": mb / sec, "unit": "MB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": int(mb * 1e6),
                    "note": "the timed step is already end to end: device trees in, host strings out"},
            "gpu_launches": 7 * len(chains) * args.steps, "roofline": None, "cpu_baseline": cpu, "clocks": clk}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------ learned proposal
LRN_N, LRN_P, LRN_CHAINS, LRN_TRAIN, LRN_NDPOST, LRN_SETS = 65_536, 32, 16, 200_000, 1000, 4
LRN_METRIC = ("ESS/s of sigma and f, learned (variable and cutpoint heads) vs plain proposal (16 fwbart chains, "
              "n 65,536, p 32, numcut 255, 27 noise predictors)")


def bench_learned(args):
    """Sparse-signal configuration: Friedman-5 on x1..x5 of 32 uniform predictors, numcut 255, 16 chains, ntree 200,
    nskip 1000, ndpost 1000.  A plain batch (other seeds) supplies accepted births as training examples of both
    heads: the variable head (node and tree features) and the cut head (node features with the residual mean and
    spread of the node's rows, drawn after the pass); each trains on up to 200,000 of them on the device.  Then, for 4
    seed sets, plain and learned batches (both heads, mix 0.5) run from the same seeds, each timed with CUDA events
    after an untimed run; ESS/s (sigma; median over 256 sampled rows of f) and the posterior agreement are reported
    per set, with the mean learned/plain ratio and a 95% t-interval over the sets, for both heads and for the variable
    head alone; seed set 0 also runs the cut head alone."""
    import torch
    import fastbart_b200 as F
    from fastbart_b200 import diagnostics, workloads as W
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    nskip, ndpost = NSKIP, LRN_NDPOST
    S = nskip + ndpost
    base = W.friedman_large(nchains=LRN_CHAINS, n=LRN_N, p=LRN_P, seed=0, nskip=nskip, ndpost=ndpost, ntree=NTREE)

    def chains(seed0):
        out = []
        for k, c in enumerate(base):
            d = dict(c)
            d["seed"] = seed0 + k
            out.append(d)
        return out

    stream = torch.cuda.current_stream()

    def timed(b):
        b.run(stream.cuda_stream)
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        b.run(stream.cuda_stream)
        c.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(c) / 1000.0

    col = F.Batch(chains(900), nskip, 100)
    col.collect(2 * LRN_TRAIN)
    col.run(stream.cuda_stream)
    col.sync()
    x, y, m, births = col.training_data()
    cx, cc, clo, chi = col.cut_training_data()
    col.close()
    k = min(LRN_TRAIN, len(y))
    t = time.perf_counter()
    vmodel, vloss = F.train_proposal(x[:k], y[:k], m[:k], epochs=10, batch=1024, lr=3e-3, seed=1)
    cmodel, closs = F.train_cut_proposal(cx[:k], cc[:k], clo[:k], chi[:k], epochs=10, batch=1024, lr=3e-3, seed=2)
    train_s = time.perf_counter() - t

    def measure(seed0, vm, cm):
        b = F.Batch(chains(seed0), nskip, ndpost)
        if vm is not None:
            b.set_proposal(dict(vm, mix=0.5))
        if cm is not None:
            b.set_cut_proposal(dict(cm, mix=0.5))
        sec = timed(b)
        info = b.launch_info()
        outs = b.download(trees=False)
        b.close()
        es = [diagnostics.chain_ess(o["sigma"][nskip:], o["yhat"]) for o in outs]
        r = {"seconds_per_batch": sec, "chain_sweeps_per_s": LRN_CHAINS * S / sec,
             "ess_sigma_per_s": float(sum(e["sigma"] for e in es) / sec),
             "ess_f_median_per_s": float(sum(e["f_median"] for e in es) / sec),
             "ess_sigma_mean": float(np.mean([e["sigma"] for e in es])),
             "ess_f_median_mean": float(np.mean([e["f_median"] for e in es])),
             "births": int(sum(o["moves"][0] for o in outs)), "deaths": int(sum(o["moves"][1] for o in outs)),
             "launch": {"threads": info["threads"], "ctas_per_chain": info["cluster"]}}
        fm = np.mean([o["yhat_mean"] for o in outs], axis=0)
        sg = float(np.mean([o["sigma"][nskip:].mean() for o in outs]))
        del outs
        return r, fm, sg

    sets = []
    for si in range(LRN_SETS):
        seed0 = 100 + 1000 * si
        rp, fp, sp = measure(seed0, None, None)
        rl, fl, sl = measure(seed0, vmodel, cmodel)
        rv, fv, sv = measure(seed0, vmodel, None)
        sets.append({"plain": rp, "learned": rl, "variable_head_only": rv,
                     "ratio_f": rl["ess_f_median_per_s"] / rp["ess_f_median_per_s"],
                     "ratio_sigma": rl["ess_sigma_per_s"] / rp["ess_sigma_per_s"],
                     "ratio_f_variable_head": rv["ess_f_median_per_s"] / rp["ess_f_median_per_s"],
                     "ratio_sigma_variable_head": rv["ess_sigma_per_s"] / rp["ess_sigma_per_s"],
                     "corr_fmean": float(np.corrcoef(fp, fl)[0, 1]), "sigma_ratio": sl / sp,
                     "corr_fmean_variable_head": float(np.corrcoef(fp, fv)[0, 1]), "sigma_ratio_variable_head": sv / sp})
    ablation = {}
    for name, vm, cm in (("cut_head_only", None, cmodel),):
        r, _, _ = measure(100, vm, cm)
        ablation[name] = {"ratio_f": r["ess_f_median_per_s"] / sets[0]["plain"]["ess_f_median_per_s"],
                          "ratio_sigma": r["ess_sigma_per_s"] / sets[0]["plain"]["ess_sigma_per_s"],
                          "chain_sweeps_per_s": r["chain_sweeps_per_s"], "births": r["births"]}

    def ci(vals):
        v = np.asarray(vals, dtype=np.float64)
        half = 3.182 * v.std(ddof=1) / np.sqrt(len(v)) if len(v) > 1 else float("nan")   # t(0.975, 3 df)
        return {"mean": float(v.mean()), "ci95": [float(v.mean() - half), float(v.mean() + half)],
                "per_set": [float(a) for a in v]}

    rf, rs = ci([x_["ratio_f"] for x_ in sets]), ci([x_["ratio_sigma"] for x_ in sets])
    rfv, rsv = ci([x_["ratio_f_variable_head"] for x_ in sets]), ci([x_["ratio_sigma_variable_head"] for x_ in sets])
    uniform_cut_loss = float(np.mean(np.log(chi[:k] - clo[:k] + 1.0)))
    line = {"metric": LRN_METRIC, "value": rf["mean"], "unit": "x (ESS/s of f, learned / plain)", "n_gpus": 1,
            "steps": 1, "warmup": 1, "ms_per_step": 1000 * sets[0]["learned"]["seconds_per_batch"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "int64-fixed+f32+f64 (MLP bf16/f32)", "data": "synthetic",
            "config": {"workload": "friedman_sparse_16x65536", "chains": LRN_CHAINS, "n": LRN_N, "p": LRN_P,
                       "numcut": 255, "ntree": NTREE, "nskip": nskip, "ndpost": ndpost, "mix": 0.5,
                       "seed_sets": LRN_SETS, "training_examples": int(k), "accepted_births_collected": int(births)},
            "ratio_f": rf, "ratio_sigma": rs, "ratio_f_variable_head": rfv, "ratio_sigma_variable_head": rsv,
            "sets": sets, "ablation_seed_set_0": ablation,
            "training": {"seconds": train_s, "epochs": 10,
                         "variable_head": {"loss_first": float(vloss[0]), "loss_last": float(vloss[-1]),
                                           "uniform_loss": float(np.log(LRN_P)),
                                           "signal_fraction_of_births": float(np.mean(y[:k] < 5))},
                         "cut_head": {"loss_first": float(closs[0]), "loss_last": float(closs[-1]),
                                      "uniform_loss": uniform_cut_loss}},
            "agreement": {"corr_fmean_min": min(x_["corr_fmean"] for x_ in sets),
                          "sigma_ratio_range": [min(x_["sigma_ratio"] for x_ in sets),
                                                max(x_["sigma_ratio"] for x_ in sets)]},
            "gpu_launches": 6 * LRN_SETS + 2 + 1}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------ mixed batch
MIX_METRIC = ("chain-sweeps/s (256 mixed chains in one launch: 128 fwbart n 2,000-65,536 p 8-32 ntree 200, "
              "128 fpbart n 4,096-24,576 ntree 50), then predict_draw of 1,000 draws x 200 trees on 1,000,000 rows")
MIX_PRED_ROWS, MIX_P = 1_000_000, 32


def _dev_oracle_fit(ch):
    from oracle import oracle as O
    o = O.fit(ch, O.MODE_DEV)
    return {k: np.asarray(o[k]) for k in ("sigma", "fmean", "trees", "moves")}


def _mix_newdata(rows: int, seed: int = 31):
    """Fresh rows of the predict fits' distribution (titer-like, p 32: half U(0,1), half integer 0..9)."""
    rng = np.random.default_rng(seed)
    x = np.empty((rows, MIX_P))
    x[:, :MIX_P // 2] = rng.random((rows, MIX_P // 2))
    x[:, MIX_P // 2:] = rng.integers(0, 10, (rows, MIX_P - MIX_P // 2))
    return x


def bench_mixed(args):
    """Config 5: the mixed 256-chain batch in one persistent launch, with BART's proposal and with the learned
    proposal (trained on this batch's accepted births from a collecting run), then compile_trees + bulk predict_draw
    of the 10 p-32 fwbart fits' pooled 1,000 kept draws (200 trees each) on 1,000,000 fresh rows x 32 FP64 columns.
    Sampled parity: the 4 smallest chains (2 fwbart, 2 fpbart) against the oracle's DEV arithmetic, full length, bit
    for bit; predict on 2,000 rows x 3 draws against the oracle's restatement of predict_draw_cpp."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from fastbart_b200 import workloads as W
    chains = W.mixed_batch(seed=0, nskip=NSKIP, ndpost=NDPOST)
    S = NSKIP + NDPOST
    ncores = os.cpu_count() or 1
    pool = mp.get_context("spawn").Pool(ncores)
    pool.map(_warm_worker, range(ncores), chunksize=1)
    sweeps = cpu_sample_plan(ncores)
    cpu = None
    if not args.no_cpu_baseline or args.impl == "reference":
        vals = []
        for _ in range((args.warmup + args.steps) if args.impl == "reference" else 1):
            v, kind, wall = run_cpu_sample(pool, chains, ncores, sweeps)
            vals.append(v)
        v = float(np.mean(vals[args.warmup:] if args.impl == "reference" else vals))
        cpu = {"value": v, "unit": UNIT, "cores": ncores, "kind": kind,
               "sample": cpu_sample_text(chains, ncores, sweeps)}
    mcfg = {"workload": "mixed_256", "chains": len(chains), "fwbart": 128, "fpbart": 128, "nskip": NSKIP,
            "ndpost": NDPOST, "n_total": int(sum(np.asarray(c["q"]).shape[1] for c in chains)),
            "predict": {"draws": 1000, "ntree": 200, "rows": MIX_PRED_ROWS, "p": MIX_P},
            "l2": "inputs resident; the GPU arm flushes L2 (512 MiB write) before every timed step"}
    if args.impl == "reference":
        line = {"metric": MIX_METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": mcfg, "impl": "reference",
                "cpu_baseline": cpu, "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                                             "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        pool.terminate()
        return 0
    order = np.argsort([np.asarray(c["q"]).shape[1] * c["ntree"] for c in chains])
    checks = [int(k) for k in order if chains[k]["probit"] == 0][:2] + \
             [int(k) for k in order if chains[k]["probit"] == 1][:2]
    dev = pool.map_async(_dev_oracle_fit, [chains[k] for k in checks])

    import torch
    import fastbart_b200 as F
    from fastbart_b200 import diagnostics
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    stream = torch.cuda.current_stream()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    b = F.Batch(chains, NSKIP, NDPOST)
    info = b.launch_info()

    def timed(steps, warmup):
        for _ in range(warmup):
            flush.zero_()
            b.run(stream.cuda_stream)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, c in evs:
            flush.zero_()
            a.record(stream)
            b.run(stream.cuda_stream)
            c.record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(c) for a, c in evs) / 1000.0 / steps

    # training examples from a collecting run, then the model
    b.collect(400_000)
    b.run(stream.cuda_stream)
    b.sync()
    x, y, m, births = b.training_data()
    b.collect(0)
    k = min(200_000, len(y))
    model, losses = F.train_proposal(x[:k], y[:k], m[:k], epochs=10, batch=1024, lr=3e-3, seed=1)

    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    res = {}
    for name, mdl in (("plain", None), ("learned", dict(model, mix=0.5))):
        b.set_proposal(mdl)
        sec = timed(args.steps, args.warmup)
        outs = b.download(trees=(name == "plain"))
        es = [diagnostics.chain_ess(o["sigma"][NSKIP:], o["yhat"]) for o in outs]
        wb = [i for i, c in enumerate(chains) if c["probit"] == 0]
        res[name] = {"seconds_per_batch": sec, "chain_sweeps_per_s": len(chains) * S / sec,
                     "ess_sigma_per_s": float(sum(es[i]["sigma"] for i in wb) / sec),
                     "ess_f_median_per_s": float(sum(e["f_median"] for e in es) / sec),
                     "births": int(sum(o["moves"][0] for o in outs))}
        if name == "plain":
            plain_outs = outs
        else:
            corr = [float(np.corrcoef(a["yhat_mean"], c["yhat_mean"])[0, 1]) for a, c in zip(plain_outs, outs)]
            res["learned"]["corr_fmean_vs_plain_median"] = float(np.median(corr))
            res["learned"]["corr_fmean_vs_plain_min"] = float(np.min(corr))
    clk = clocks.stop()
    b.set_proposal(None)

    # sampled bit-exact parity of the plain run
    parity = []
    for kk, o in zip(checks, dev.get(timeout=1200)):
        g = plain_outs[kk]
        ok = all(np.array_equal(np.asarray(g[a]), o[bk]) for a, bk in
                 (("sigma", "sigma"), ("yhat_mean", "fmean"), ("trees", "trees"), ("moves", "moves")))
        parity.append({"chain": kk, "n": int(np.asarray(chains[kk]["q"]).shape[1]), "probit": chains[kk]["probit"],
                       "bit_exact": bool(ok)})
    assert all(p_["bit_exact"] for p_ in parity), parity

    # end to end through fb_fit_batch with host buffers (allocation, H2D, MCMC, D2H of every output), one step
    e2e = None
    if not args.no_e2e:
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        F.fit_batch(chains, NSKIP, NDPOST)
        e2e_s = time.perf_counter() - t1
        d2h = sum(8 * S + 8 * np.asarray(c["q"]).shape[1] * (1 + NDPOST) + 8 * NDPOST * c["ntree"] * 64 for c in chains)
        h2d = sum(np.asarray(c["q"]).nbytes + 13 * np.asarray(c["q"]).shape[1] for c in chains)
        e2e = {"value": len(chains) * S / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": 1, "ms_per_step": 1000 * e2e_s,
               "api": "fb_fit_batch (pageable host buffers; allocation, H2D, MCMC, D2H of sigma/yhat/yhat_mean/trees)"}
    b.close()

    # bulk predict of the pooled 1,000 draws of the ten p-32 fits
    trees = np.concatenate([plain_outs[c]["trees"] for c in range(W.MIXED_PREDICT_FITS)], axis=0)
    grid = W.titer_like_grid(MIX_P)
    text = F.trees_text_gpu(trees, MIX_P)
    ct = F.CompiledTrees(text, grid, mu=0.0)
    xh = _mix_newdata(MIX_PRED_ROWS)
    xd = torch.tensor(np.ascontiguousarray(xh.T), device="cuda")
    nd = trees.shape[0]
    out = torch.empty((nd, MIX_PRED_ROWS), dtype=torch.float64, device="cuda")

    def pred():
        F.predict_draws_device(ct, xd.data_ptr(), MIX_P, MIX_PRED_ROWS, MIX_PRED_ROWS, 1, nd, out.data_ptr(),
                               MIX_PRED_ROWS, stream.cuda_stream)
    for _ in range(args.warmup):
        flush.zero_()
        pred()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for a, c in evs:
        flush.zero_()
        a.record(stream)
        pred()
        c.record(stream)
    torch.cuda.synchronize()
    psec = sum(a.elapsed_time(c) for a, c in evs) / 1000.0 / args.steps
    from oracle import oracle as O
    oct_ = O.compile_trees(text, grid)
    sub = xh[:2000]
    pparity = all(np.array_equal(out[d - 1, :2000].cpu().numpy(),
                                 O.predict_draw(oct_, [np.ascontiguousarray(sub[:, v]) for v in range(MIX_P)], d, 0.0))
                  for d in (1, 500, nd))
    assert pparity, "bulk predict differs from the oracle"
    alg = MIX_P * MIX_PRED_ROWS * 8 + nd * MIX_PRED_ROWS * 8 + ct.nnodes * 12
    peak, peak_kind = measured_peak()
    predict = {"row_draws_per_s": nd * MIX_PRED_ROWS / psec, "ms_per_call": 1000 * psec, "draws": nd,
               "nodes": ct.nnodes, "hbm_gbs": alg / psec / 1e9, "frac_of_hbm": alg / psec / 1e9 / peak,
               "peak": peak, "peak_source": peak_kind, "bit_exact_vs_oracle": bool(pparity),
               "evaluator": ct.evaluator(MIX_PRED_ROWS, nd)[0],
               "shared_tree_fraction": ct.evaluator(MIX_PRED_ROWS, nd)[1] / float(nd * 200),
               "what": "1,000 draws (10 fits x 100 kept draws) x 200 trees on 1,000,000 fresh rows, one "
                       "fb_predict_draws_device call, x and results resident"}
    pool.terminate()
    value = res["plain"]["chain_sweeps_per_s"]
    line = {"metric": MIX_METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * res["plain"]["seconds_per_batch"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64-fixed+f32+f64", "data": "synthetic",
            "config": mcfg, "launch": {"threads": info["threads"], "grid": info["grid"], "smem_bytes": info["smem"],
                                       "ctas_per_chain": info["cluster"]},
            "e2e": e2e, "gpu_launches": 2 * (args.steps + args.warmup) + 1,
            "roofline": {"bound": "hbm", "achieved": BYTES_PER_ROW_TREE * sum(np.asarray(c["q"]).shape[1] * (c["ntree"] + 1) for c in chains) * S / res["plain"]["seconds_per_batch"] / 1e9,
                         "peak": peak, "unit": "GB/s", "traffic": None, "peak_source": peak_kind},
            "cpu_baseline": cpu, "clocks": clk, "plain": res["plain"], "learned": res["learned"],
            "learned_over_plain": {"ess_f_per_s": res["learned"]["ess_f_median_per_s"] / res["plain"]["ess_f_median_per_s"],
                                   "ess_sigma_per_s": res["learned"]["ess_sigma_per_s"] / res["plain"]["ess_sigma_per_s"]},
            "training": {"examples": int(k), "accepted_births_collected": int(births), "loss_first": float(losses[0]),
                         "loss_last": float(losses[-1])},
            "parity_sample": parity, "predict_draw": predict}
    line["roofline"]["frac"] = line["roofline"]["achieved"] / peak
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------ head training
TRAIN_N = 200_000


def bench_train(args):
    """Training of both learned heads on the device (fb_train_proposal, fb_train_cut_proposal: per minibatch one
    gradient launch, whose GEMMs run on the tensor cores, and one Adam launch) on config 4's 200,000 training moves,
    synthetic features of the heads' shapes.  Metric: training examples per second (epochs x examples / wall time of
    the call, which includes one copy of the examples to the device); one full-batch gradient launch per head is also
    timed with CUDA events on its own."""
    import torch
    import fastbart_b200 as F
    from fastbart_b200 import _lib
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned proposal to train"}))
        return 0
    rng = np.random.default_rng(5)
    N, IN, O = TRAIN_N, _lib.MLP_IN, _lib.MLP_OUT
    x = rng.random((N, IN), dtype=np.float32)
    mask = rng.integers(1, 1 << 32, N, dtype=np.uint64).astype(np.uint32) | np.uint32(1)
    y = np.array([rng.choice(np.flatnonzero((int(m) >> np.arange(O)) & 1)) for m in mask[:4096]], np.int32)
    y = np.resize(y, N)
    mask = mask | (np.uint32(1) << y.astype(np.uint32))
    cx = rng.random((N, _lib.CUT_IN), dtype=np.float32)
    lo = rng.integers(0, 200, N).astype(np.int32)
    hi = np.minimum(lo + rng.integers(0, 100, N), 254).astype(np.int32)
    cc = (lo + (rng.random(N) * (hi - lo + 1)).astype(np.int32)).astype(np.int32)
    epochs = max(1, args.steps)
    F.train_proposal(x[:4096], y[:4096], mask[:4096], epochs=1, batch=512)   # warm-up (module load, first launch)
    F.train_cut_proposal(cx[:4096], cc[:4096], lo[:4096], hi[:4096], epochs=1, batch=512)
    torch.cuda.synchronize()
    out = {}
    for name, call in (("variable_head", lambda: F.train_proposal(x, y, mask, epochs=epochs, batch=512, seed=1)),
                       ("cut_head", lambda: F.train_cut_proposal(cx, cc, lo, hi, epochs=epochs, batch=512, seed=1))):
        t = time.perf_counter()
        _, losses = call()
        wall = time.perf_counter() - t
        out[name] = {"examples_per_s": N * epochs / wall, "seconds": wall, "epochs": epochs,
                     "loss_first": float(losses[0]), "loss_last": float(losses[-1])}
    # one gradient launch over all examples (6,250 tiles of 32), device time from CUDA events around the call's copy
    # and kernel (the call copies its inputs and results synchronously)
    model = {k: np.zeros(v.shape, v.dtype) for k, v in F.api._empty_model().items()}
    gflop = 2.0 * (IN * 64 + 64 * 64 + 64 * O) * 3 * N / 1e9
    t = time.perf_counter()
    F.mlp_loss_grad(model, x, y, mask)
    out["variable_head"]["full_batch_gradient_s"] = time.perf_counter() - t
    out["variable_head"]["gemm_gflop_per_pass"] = gflop
    value = out["variable_head"]["examples_per_s"]
    line = {"metric": "training examples/s of the learned variable head (config 4's 200,000 moves, minibatch 512)",
            "value": value, "unit": "examples/s", "n_gpus": 1, "steps": epochs, "warmup": 1,
            "ms_per_step": 1000 * out["variable_head"]["seconds"] / epochs, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "tf32x3 (f32 accuracy) on tensor cores, bf16 weights",
            "data": "synthetic", "config": {"workload": "train_heads_200k", "examples": N, "batch": 512},
            "e2e": {"value": value, "unit": "examples/s", "h2d_bytes_per_step": int(x.nbytes + y.nbytes + mask.nbytes),
                    "d2h_bytes_per_step": 0, "api": "fb_train_proposal (host arrays in, model out)"},
            "gpu_launches": int(2 * epochs * ((N + 511) // 512)), "heads": out}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--cluster", type=int, default=0, help="CTAs per chain (0: automatic, 1: no clusters)")
    ap.add_argument("--autotune", action="store_true", help="time candidate launch shapes first (fb_autotune)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-posterior", action="store_true", help="predict: skip the posterior-shaped forest leg")
    ap.add_argument("--pred-rows", type=int, default=0, help="predict: rows (default 1,000,000; smaller for profiling)")
    ap.add_argument("--pred-draws", type=int, default=0, help="predict: draws (default 1,000)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-single", action="store_true", help="skip the one-chain-per-launch comparison")
    ap.add_argument("--workload", default="titer96",
                    choices=["titer96", "small", "single", "sparse", "probit", "predict", "learned", "text",
                             "mixed", "train"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "predict":
        return bench_predict(args)
    if args.workload == "learned":
        return bench_learned(args)
    if args.workload == "text":
        return bench_text(args)
    if args.workload == "mixed":
        return bench_mixed(args)
    if args.workload == "train":
        return bench_train(args)
    set_workload(args.workload)
    if args.impl == "reference":
        return bench_reference(args)
    return bench_ours(args)


if __name__ == "__main__":
    sys.exit(main())
