"""Python mirror of fastbart's R interface (R/fwbart.R, R/fpbart.R, R/predict_draw.R) on the B200 library.

fwbart()/fpbart() take BART's arguments and return the fields of BART's "wbart"/"pbart" objects (R names, dots
included); compile_trees()/predict_draw() reproduce the fast single-draw evaluator.  All compute runs in
libfastbart_b200.so on the GPU; there is no CPU fallback (the reference falls back to BART::wbart / BART::pbart for
unsupported settings; BART is not available here, so those settings raise FastbartError(FB_ERR_LIMIT)).
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np
from scipy import stats

from . import _lib, prep, workloads
from ._lib import NODES, FastbartError, check, ptr

__all__ = ["fwbart", "fpbart", "compile_trees", "predict_draw", "fit_batch", "Batch", "trees_text", "trees_text_gpu",
           "varcount", "release_cached_memory",
           "FastbartError"]


class BartFit(dict):
    """A fitted model: a dict with the R object's fields; .cls is "wbart" or "pbart"."""

    def __init__(self, cls: str, **kw):
        super().__init__(**kw)
        self.cls = cls


# ------------------------------------------------------------------------------------------------ batches
def _as_chain(ch: dict, keep: list) -> _lib.Chain:
    q = np.ascontiguousarray(ch["q"], dtype=np.uint8)
    p, n = q.shape
    probit = int(ch.get("probit", 0))
    y = None if probit else np.ascontiguousarray(ch["y"], dtype=np.float64)
    wt = ch.get("wt")
    wt = None if wt is None else np.ascontiguousarray(wt, dtype=np.float64)
    ybin = np.ascontiguousarray(ch["ybin"], dtype=np.int32) if probit else None
    numcut = np.ascontiguousarray(ch["numcut"], dtype=np.int32)
    pg = np.ascontiguousarray(ch["pgtab"], dtype=np.float64)
    keep += [q, y, wt, ybin, numcut, pg]
    return _lib.Chain(n, p, int(ch["ntree"]), ptr(q), ptr(y), ptr(wt), ptr(ybin), ptr(numcut), ptr(pg),
                      float(ch["tau"]), float(ch["lambda"]), float(ch["nu"]), float(ch["sigest"]),
                      float(ch.get("offset", 0.0)), int(ch["seed"]) & 0xFFFFFFFFFFFFFFFF, probit,
                      int(ch.get("fx_shift", 0)), int(ch.get("rss_shift", 0)))


def _alloc_out(ch: dict, nskip: int, ndpost: int, trees: bool = True, alloc=np.empty):
    n = np.asarray(ch["q"]).shape[1]
    m = int(ch["ntree"])
    o = dict(sigma=alloc(nskip + ndpost, dtype=np.float64), yhat_mean=alloc(n, dtype=np.float64),
             yhat=alloc((ndpost, n), dtype=np.float64),
             trees=alloc((ndpost, m, NODES), dtype=np.uint64) if trees else None)
    s = _lib.ChainOut(ptr(o["sigma"]), ptr(o["yhat_mean"]), ptr(o["yhat"]), ptr(o["trees"]))
    return o, s


def _collect(o: dict, s: _lib.ChainOut) -> dict:
    o["moves"] = np.array(list(s.moves), dtype=np.int32)
    o["rtnorm_caps"] = int(s.rtnorm_caps)
    return o


def _options(nskip, ndpost, threads=0, sweeps_per_launch=0, device=0, cluster=0) -> _lib.Options:
    return _lib.Options(int(nskip), int(ndpost), int(threads), int(sweeps_per_launch), int(device), int(cluster))


def fit_batch(chains: Sequence[dict], nskip: int, ndpost: int, threads: int = 0, sweeps_per_launch: int = 0,
              device: int = 0, trees: bool = True, cluster: int = 0, devices: Sequence[int] | None = None) -> list:
    """Runs prepared chains (dicts as built by workloads.fwbart_chain / fpbart_chain) in one device batch.  With
    `devices` (several GPU ordinals) the chains are partitioned across those GPUs, one batch per GPU run from its own
    host thread, and the outputs are returned in the order of `chains` (shard.fit_sharded)."""
    if devices is not None and len(devices) > 1:
        from . import shard
        return shard.fit_sharded(chains, nskip, ndpost, devices, threads=threads, sweeps_per_launch=sweeps_per_launch,
                                 trees=trees, cluster=cluster)
    if devices is not None and len(devices) == 1:
        device = int(devices[0])
    keep: list = []
    arr = (_lib.Chain * len(chains))(*[_as_chain(c, keep) for c in chains])
    outs = [_alloc_out(c, nskip, ndpost, trees) for c in chains]
    oarr = (_lib.ChainOut * len(chains))(*[s for _, s in outs])
    opt = _options(nskip, ndpost, threads, sweeps_per_launch, device, cluster)
    check(_lib.lib().fb_fit_batch(arr, len(chains), C.byref(opt), oarr))
    return [_collect(o, oarr[k]) for k, (o, _) in enumerate(outs)]


def autotune(chains: Sequence[dict], nskip: int, ndpost: int, trial_sweeps: int = 3, device: int = 0) -> dict:
    """Fastest launch shape for these chains (fb_autotune): {"threads", "cluster", "trial_ms"}, to pass to Batch /
    fit_batch."""
    keep: list = []
    arr = (_lib.Chain * len(chains))(*[_as_chain(c, keep) for c in chains])
    opt = _options(nskip, ndpost, 0, 0, device, 0)
    best = _lib.Options()
    ms = C.c_double()
    check(_lib.lib().fb_autotune(arr, len(chains), C.byref(opt), int(trial_sweeps), C.byref(best), C.byref(ms)))
    return dict(threads=best.threads, cluster=best.cluster, trial_ms=ms.value)


class Batch:
    """Staged batch: inputs uploaded once; run() repeats the full MCMC on the device; download() copies outputs."""

    def __init__(self, chains: Sequence[dict], nskip: int, ndpost: int, threads: int = 0, sweeps_per_launch: int = 0,
                 device: int = 0, cluster: int = 0):
        self._keep: list = []
        self.chains = list(chains)
        self.nskip, self.ndpost = int(nskip), int(ndpost)
        arr = (_lib.Chain * len(chains))(*[_as_chain(c, self._keep) for c in chains])
        opt = _options(nskip, ndpost, threads, sweeps_per_launch, device, cluster)
        h = C.c_void_p()
        check(_lib.lib().fb_batch_create(arr, len(chains), C.byref(opt), C.byref(h)))
        self._h = h

    def run(self, stream: int | None = None):
        check(_lib.lib().fb_batch_run(self._h, stream))

    def sync(self):
        check(_lib.lib().fb_batch_sync(self._h))

    def launch_info(self) -> dict:
        a, b, c, d, e = C.c_int(), C.c_int(), C.c_int(), C.c_size_t(), C.c_int()
        check(_lib.lib().fb_batch_launch_info(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d), C.byref(e)))
        return dict(launches=a.value, threads=b.value, grid=c.value, smem=d.value, cluster=e.value,
                    autotuned=bool(_lib.lib().fb_batch_autotuned(self._h)))

    def download(self, trees: bool = True, alloc=np.empty) -> list:
        outs = [_alloc_out(c, self.nskip, self.ndpost, trees, alloc) for c in self.chains]
        oarr = (_lib.ChainOut * len(outs))(*[s for _, s in outs])
        check(_lib.lib().fb_batch_download(self._h, oarr))
        return [_collect(o, oarr[k]) for k, (o, _) in enumerate(outs)]

    def trees_text(self, chain: int) -> str:
        """BART tree text of one chain's kept draws, assembled on the device from its trees there."""
        L, ln = _lib.lib(), C.c_size_t()
        check(L.fb_batch_trees_text(self._h, chain, None, 0, C.byref(ln)))
        buf = C.create_string_buffer(ln.value + 1)
        check(L.fb_batch_trees_text(self._h, chain, buf, ln.value + 1, C.byref(ln)))
        return buf.raw[:ln.value].decode()

    def set_proposal(self, model: dict | None):
        """Learned split-variable proposal for the next runs (see `train_proposal`); None restores BART's."""
        if model is None:
            check(_lib.lib().fb_batch_set_proposal(self._h, None))
            return
        ms = _model_struct(model, self._keep)
        check(_lib.lib().fb_batch_set_proposal(self._h, C.byref(ms)))

    def set_cut_proposal(self, model: dict | None):
        """Learned cutpoint proposal for the next runs (see `train_cut_proposal`); None restores BART's uniform cut."""
        if model is None:
            check(_lib.lib().fb_batch_set_cut_proposal(self._h, None))
            return
        ms = _cut_struct(model, self._keep)
        check(_lib.lib().fb_batch_set_cut_proposal(self._h, C.byref(ms)))

    def cut_training_data(self) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
        """(x [k][40] float32, cut [k], lo [k], hi [k] int32) of the births training_data() returns, same order."""
        cap = getattr(self, "_cap", 0)
        x = np.zeros((max(cap, 1), _lib.CUT_IN), np.float32)
        c, lo, hi = (np.zeros(max(cap, 1), np.int32) for _ in range(3))
        cnt = C.c_int()
        check(_lib.lib().fb_batch_cut_training_data(self._h, ptr(x), ptr(c), ptr(lo), ptr(hi), cap, C.byref(cnt)))
        k = min(cnt.value, cap)
        return x[:k], c[:k], lo[:k], hi[:k]

    def collect(self, capacity: int):
        """Collect the accepted births of the next runs as training examples (at most `capacity` per run)."""
        self._cap = int(capacity)
        check(_lib.lib().fb_batch_collect(self._h, self._cap))

    def training_data(self) -> tuple[np.ndarray, np.ndarray, np.ndarray, int]:
        """(x [k][98] float32, y [k] int32, mask [k] uint32, accepted births of the run) of the last run."""
        cap = getattr(self, "_cap", 0)
        x = np.zeros((max(cap, 1), _lib.MLP_IN), np.float32)
        y = np.zeros(max(cap, 1), np.int32)
        m = np.zeros(max(cap, 1), np.uint32)
        cnt = C.c_int()
        check(_lib.lib().fb_batch_training_data(self._h, ptr(x), ptr(y), ptr(m), cap, C.byref(cnt)))
        k = min(cnt.value, cap)
        return x[:k], y[:k], m[:k], cnt.value

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().fb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------------------------------ learned proposal
def _model_struct(model: dict, keep: list) -> _lib.ProposalModel:
    arrs = []
    for k, dt in (("w1", np.uint16), ("b1", np.float32), ("w2", np.uint16), ("b2", np.float32), ("w3", np.uint16),
                  ("b3", np.float32)):
        a = np.ascontiguousarray(model[k], dtype=dt)
        keep.append(a)
        arrs.append(a.ctypes.data)
    ms = _lib.ProposalModel(*arrs, float(model.get("mix", 0.5)))
    keep.append(ms)
    return ms


CUT_KEYS = (("w1", np.uint16), ("b1", np.float32), ("w2", np.uint16), ("b2", np.float32), ("w3", np.uint16),
            ("b3", np.float32), ("emb", np.uint16), ("be", np.float32))


def _cut_struct(model: dict, keep: list) -> _lib.CutModel:
    arrs = []
    for k, dt in CUT_KEYS:
        a = np.ascontiguousarray(model[k], dtype=dt)
        keep.append(a)
        arrs.append(a.ctypes.data)
    ms = _lib.CutModel(*arrs, float(model.get("mix", 0.5)))
    keep.append(ms)
    return ms


def _cut_shapes() -> dict:
    H, I, E, NB = _lib.CUT_H, _lib.CUT_IN, _lib.CUT_E, _lib.CUT_BINS
    return dict(w1=(H, I), b1=(H,), w2=(H, H), b2=(H,), w3=(E, H), b3=(E,), emb=(NB, E), be=(NB,))


def train_cut_proposal(x, c, lo, hi, epochs: int = 10, batch: int = 512, lr: float = 2e-3, seed: int = 0,
                       init: dict | None = None, mix: float = 0.5, device: int = 0) -> tuple[dict, np.ndarray]:
    """Trains the cut head on the device (softmax cross-entropy over each example's cut range, Adam); returns
    (model, epoch losses)."""
    x = np.ascontiguousarray(x, np.float32)
    c, lo, hi = (np.ascontiguousarray(a, np.int32) for a in (c, lo, hi))
    out = {k: np.zeros(sh, dtype=dt) for (k, dt), sh in zip(CUT_KEYS, _cut_shapes().values())}
    losses = np.zeros(int(epochs))
    keep: list = []
    opt = _lib.TrainOptions(int(epochs), int(batch), float(lr), int(seed) & 0xFFFFFFFFFFFFFFFF, int(device))
    ini = C.byref(_cut_struct(init, keep)) if init is not None else None
    check(_lib.lib().fb_train_cut_proposal(ptr(x), ptr(c), ptr(lo), ptr(hi), len(c), C.byref(opt), ini,
                                           *(ptr(out[k]) for k, _ in CUT_KEYS), ptr(losses)))
    out["mix"] = float(mix)
    return out, losses


def cut_loss_grad(model: dict, x, c, lo, hi, device: int = 0) -> tuple[float, dict]:
    """One forward/backward of the cut head's training kernels: mean loss and gradients (FP32)."""
    x = np.ascontiguousarray(x, np.float32)
    c, lo, hi = (np.ascontiguousarray(a, np.int32) for a in (c, lo, hi))
    keep: list = []
    ms = _cut_struct(model, keep)
    g = {k: np.zeros(sh, np.float32) for k, sh in _cut_shapes().items()}
    loss = C.c_double()
    check(_lib.lib().fb_cut_loss_grad(C.byref(ms), ptr(x), ptr(c), ptr(lo), ptr(hi), len(c), int(device),
                                      C.byref(loss), *(ptr(g[k]) for k, _ in CUT_KEYS)))
    return loss.value, g


def _empty_model() -> dict:
    H, I, O = _lib.MLP_H, _lib.MLP_IN, _lib.MLP_OUT
    return dict(w1=np.zeros((H, I), np.uint16), b1=np.zeros(H, np.float32), w2=np.zeros((H, H), np.uint16),
                b2=np.zeros(H, np.float32), w3=np.zeros((O, H), np.uint16), b3=np.zeros(O, np.float32))


def train_proposal(x, y, mask, epochs: int = 10, batch: int = 512, lr: float = 2e-3, seed: int = 0,
                   init: dict | None = None, mix: float = 0.5, device: int = 0) -> tuple[dict, np.ndarray]:
    """Trains the proposal MLP on the device (masked softmax cross-entropy, Adam); returns (model, epoch losses)."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.int32)
    mask = np.ascontiguousarray(mask, np.uint32)
    out = _empty_model()
    losses = np.zeros(int(epochs))
    keep: list = []
    opt = _lib.TrainOptions(int(epochs), int(batch), float(lr), int(seed) & 0xFFFFFFFFFFFFFFFF, int(device))
    ini = C.byref(_model_struct(init, keep)) if init is not None else None
    check(_lib.lib().fb_train_proposal(ptr(x), ptr(y), ptr(mask), len(y), C.byref(opt), ini,
                                       *(ptr(out[k]) for k in ("w1", "b1", "w2", "b2", "w3", "b3")), ptr(losses)))
    out["mix"] = float(mix)
    return out, losses


def mlp_loss_grad(model: dict, x, y, mask, device: int = 0) -> tuple[float, dict]:
    """One forward/backward of the device training kernels: mean loss and gradients (FP32)."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.int32)
    mask = np.ascontiguousarray(mask, np.uint32)
    keep: list = []
    ms = _model_struct(model, keep)
    H, I, O = _lib.MLP_H, _lib.MLP_IN, _lib.MLP_OUT
    g = dict(w1=np.zeros((H, I), np.float32), b1=np.zeros(H, np.float32), w2=np.zeros((H, H), np.float32),
             b2=np.zeros(H, np.float32), w3=np.zeros((O, H), np.float32), b3=np.zeros(O, np.float32))
    loss = C.c_double()
    check(_lib.lib().fb_mlp_loss_grad(C.byref(ms), ptr(x), ptr(y), ptr(mask), len(y), int(device), C.byref(loss),
                                      *(ptr(g[k]) for k in ("w1", "b1", "w2", "b2", "w3", "b3"))))
    return loss.value, g


def probit_latent_device(fit_ptr: int, ybin_ptr: int, n: int, offset: float, seed: int, sweep: int, z_ptr: int,
                         capped_ptr: int = 0, stream: int = 0):
    """fpbart's latent redraw on device arrays (fb_probit_latent_device): z[i] for fits fit[i] (FP64) and outcomes
    ybin[i] (int32) as the sampler draws it for that row at the end of 0-based sweep `sweep` (-1: the initial draw)."""
    check(_lib.lib().fb_probit_latent_device(fit_ptr, ybin_ptr, int(n), float(offset), int(seed) & (2**64 - 1),
                                             int(sweep), z_ptr, capped_ptr or None, stream or None))


def sigma_estimate(x, yc, device: int = 0) -> tuple[float, int]:
    """(sigest, rank): the residual standard error of the least-squares fit yc ~ 1 + x computed from device Gram
    sums (fb_sigma_estimate; R/fwbart.R:22), or sd(yc) when x has at least as many columns as rows."""
    X = np.asarray(x, dtype=np.float64)
    if X.ndim == 1:
        X = X[:, None]
    cols = [np.ascontiguousarray(X[:, v]) for v in range(X.shape[1])]
    ptrs = (C.c_void_p * max(1, len(cols)))(*[c.ctypes.data for c in cols])
    y = np.ascontiguousarray(yc, dtype=np.float64)
    out, rank = C.c_double(), C.c_int()
    check(_lib.lib().fb_sigma_estimate(ptrs, len(cols), y.size, ptr(y), int(device), C.byref(out), C.byref(rank)))
    return out.value, rank.value


def cut_codes(x, cutpoints: Sequence[np.ndarray], device: int = 0) -> np.ndarray:
    """Cutpoint codes on the device (fb_cut_codes): q [p][n] uint8 with x < cutpoints[v][c] <=> q <= c."""
    X = np.asarray(x, dtype=np.float64)
    if X.ndim == 1:
        X = X[:, None]
    n, p = X.shape
    cols = [np.ascontiguousarray(X[:, j]) for j in range(p)]
    cps = [np.ascontiguousarray(c, dtype=np.float64) for c in cutpoints]
    cp = (C.c_void_p * max(1, p))(*[c.ctypes.data for c in cols])
    kp = (C.c_void_p * max(1, p))(*[c.ctypes.data for c in cps])
    nc = np.array([c.size for c in cps], dtype=np.int32)
    q = np.zeros((p, n), dtype=np.uint8)
    check(_lib.lib().fb_cut_codes(cp, p, n, kp, ptr(nc), int(device), ptr(q)))
    return q


# ------------------------------------------------------------------------------------------------ tree text
def trees_text(trees: np.ndarray, p: int) -> str:
    t = np.ascontiguousarray(trees, dtype=np.uint64)
    nd, m = t.shape[0], t.shape[1]
    L = _lib.lib()
    ln = L.fb_trees_text(ptr(t), nd, m, p, None, 0)
    buf = C.create_string_buffer(ln + 1)
    L.fb_trees_text(ptr(t), nd, m, p, buf, ln + 1)
    return buf.raw[:ln].decode()


def release_cached_memory(device: int = 0):
    """Returns the device memory kept by finished batches (for the next batch) to the driver."""
    check(_lib.lib().fb_release_cached_memory(device))


def trees_text_gpu(trees: np.ndarray, p: int, device: int = 0) -> str:
    """`trees_text` assembled on the device (the same bytes), for host arrays of packed draws."""
    t = np.ascontiguousarray(trees, dtype=np.uint64)
    nd, m = t.shape[0], t.shape[1]
    L, ln = _lib.lib(), C.c_size_t()
    check(L.fb_trees_text_gpu(ptr(t), nd, m, p, device, None, 0, C.byref(ln)))
    buf = C.create_string_buffer(ln.value + 1)
    check(L.fb_trees_text_gpu(ptr(t), nd, m, p, device, buf, ln.value + 1, C.byref(ln)))
    return buf.raw[:ln.value].decode()


def varcount(trees: np.ndarray, p: int) -> np.ndarray:
    t = np.ascontiguousarray(trees, dtype=np.uint64)
    out = np.zeros((t.shape[0], p), dtype=np.int32)
    check(_lib.lib().fb_varcount(ptr(t), t.shape[0], t.shape[1], p, ptr(out)))
    return out


# ------------------------------------------------------------------------------------------------ R-shaped API
def _unsupported(name, sparse, x_test, n, p, ntree, numcut_v, extra):
    if sparse or (x_test is not None and np.size(x_test) > 0) or n > prep.NMAX or p > prep.PMAX or \
            ntree > prep.MMAX or (numcut_v.size and numcut_v.max() > prep.NUMCUT_MAX) or extra:
        raise FastbartError(_lib.FB_ERR_LIMIT, f"{name}: unsupported settings (sparse, x.test, n > 65536, p > 32, "
                                               f"ntree > 200, numcut > 255 or extra arguments)")


def fwbart(x_train, y_train, x_test=None, sparse=False, xinfo=None, usequants=False, cont=False, rm_const=True,
           sigest=None, sigdf=3, sigquant=0.90, k=2.0, power=2.0, base=0.95, sigmaf=None, lambda_=None, fmean=None,
           w=None, ntree=200, numcut=100, ndpost=1000, nskip=100, printevery=100, seed=None, device=0, **extra) -> BartFit:
    """Drop-in for BART::wbart (R/fwbart.R:4-45).  Returns the "wbart" fields."""
    d = prep.model_matrix(x_train, numcut, rm_const, xinfo)
    y = np.asarray(y_train, dtype=np.float64)
    n, p = y.size, d.X.shape[1]
    _unsupported("fwbart", sparse, x_test, n, p, ntree, d.numcut, extra)
    fm = float(np.mean(y)) if fmean is None else float(fmean)
    w = np.ones(n) if w is None else np.asarray(w, dtype=np.float64)
    yc = y - fm
    nu = float(sigdf)
    if lambda_ is None:
        if sigest is None:   # lm's residual standard error (sd(yc) when p >= n), from Gram sums on the device
            sigest = sigma_estimate(d.X, yc, device)[0]
        lambda_ = sigest * sigest * stats.chi2.ppf(1.0 - sigquant, nu) / nu
    else:
        sigest = float(np.sqrt(lambda_))
    tau = (yc.max() - yc.min()) / (2 * k * np.sqrt(ntree)) if sigmaf is None else sigmaf / np.sqrt(ntree)
    if seed is None:
        seed = int(np.random.default_rng().integers(1, 2**63))
    ch = dict(q=d.q, y=yc, wt=1.0 / (w * w), numcut=d.numcut, pgtab=prep.pg_table(base, power), tau=float(tau),
              nu=nu, sigest=float(sigest), offset=0.0, seed=int(seed), probit=0, ntree=int(ntree))
    ch["lambda"] = float(lambda_)
    o = fit_batch([ch], nskip, ndpost, device=device)[0]
    names = d.colnames
    xi = {nm: d.xi[v] for v, nm in enumerate(names)}
    return BartFit("wbart", sigma=o["sigma"], **{"yhat.train.mean": o["yhat_mean"] + fm,
                                                "yhat.train": o["yhat"] + fm},
                   varcount=varcount(o["trees"], p), varprob=np.full((ndpost, p), 1.0 / p),
                   treedraws=dict(cutpoints=xi, trees=trees_text_gpu(o["trees"], p, device)), mu=fm, moves=o["moves"],
                   **{"rm.const": d.rm_const, "varcount.mean": varcount(o["trees"], p).mean(axis=0),
                      "varprob.mean": np.full(p, 1.0 / p)}, colnames=names)


def fpbart(x_train, y_train, x_test=None, sparse=False, xinfo=None, usequants=False, cont=False, rm_const=True,
           k=2.0, power=2.0, base=0.95, binaryOffset=None, ntree=50, numcut=100, ndpost=1000, nskip=100,
           printevery=100, seed=None, device=0, **extra) -> BartFit:
    """Drop-in for BART::pbart (R/fpbart.R:4-41).  Returns the "pbart" fields."""
    y = np.asarray(y_train).astype(np.int32)
    off = float(stats.norm.ppf(np.mean(y))) if binaryOffset is None else float(binaryOffset)
    d = prep.model_matrix(x_train, numcut, rm_const, xinfo)
    n, p = y.size, d.X.shape[1]
    _unsupported("fpbart", sparse, x_test, n, p, ntree, d.numcut, extra)
    tau = 3.0 / (k * np.sqrt(ntree))
    if seed is None:
        seed = int(np.random.default_rng().integers(1, 2**63))
    ch = dict(q=d.q, ybin=y, numcut=d.numcut, pgtab=prep.pg_table(base, power), tau=float(tau), nu=3.0, sigest=1.0,
              offset=off, seed=int(seed), probit=1, ntree=int(ntree))
    ch["lambda"] = 1.0
    o = fit_batch([ch], nskip, ndpost, device=device)[0]
    names = d.colnames
    yh = o["yhat"] + off
    prob = stats.norm.cdf(yh)
    vc = varcount(o["trees"], p)
    return BartFit("pbart", **{"yhat.train": yh, "prob.train": prob, "prob.train.mean": prob.mean(axis=0)},
                   varcount=vc, varprob=np.full((ndpost, p), 1.0 / p),
                   treedraws=dict(cutpoints={nm: d.xi[v] for v, nm in enumerate(names)},
                                  trees=trees_text_gpu(o["trees"], p, device)),
                   binaryOffset=off, moves=o["moves"],
                   **{"rm.const": d.rm_const, "varcount.mean": vc.mean(axis=0), "varprob.mean": np.full(p, 1.0 / p)},
                   colnames=names)


class CompiledTrees:
    """Result of compile_trees(): flat node arrays on the device (and host copies, as compile_trees_cpp returns)."""

    def __init__(self, text: str, cutpoints: Sequence[np.ndarray], mu: float = 0.0, rm_const=None,
                 probit: bool = False, device: int = 0):
        xs = [np.ascontiguousarray(c, dtype=np.float64) for c in cutpoints]
        self._xs = xs
        ptrs = (C.c_void_p * max(1, len(xs)))(*[x.ctypes.data for x in xs])
        nc = np.array([x.size for x in xs], dtype=np.int32)
        h = C.c_void_p()
        raw = text.encode()
        check(_lib.lib().fb_compile_trees(raw, len(raw), ptrs, ptr(nc), len(xs), int(device), C.byref(h)))
        self._h = h
        nd, m, p, nn = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(_lib.lib().fb_compiled_info(h, C.byref(nd), C.byref(m), C.byref(p), C.byref(nn)))
        self.ndpost, self.ntree, self.p, self.nnodes = nd.value, m.value, p.value, nn.value
        self.mu, self.rm_const, self.probit = float(mu), rm_const, bool(probit)

    def arrays(self) -> dict:
        N = self.nnodes
        var, child = np.zeros(N, np.int32), np.zeros(N, np.int32)
        cut, theta = np.zeros(N), np.zeros(N)
        root = np.zeros(self.ndpost * self.ntree, np.int32)
        check(_lib.lib().fb_compiled_arrays(self._h, ptr(var), ptr(child), ptr(cut), ptr(theta), ptr(root)))
        return dict(ndpost=self.ndpost, ntree=self.ntree, p=self.p, var=var, child=child, cut=cut, theta=theta,
                    root=root)

    EVALUATORS = ("streaming", "tiled", "codes", "codes_carry")

    def evaluator(self, n: int, ndraws: int) -> tuple[str, int]:
        """(name of the device evaluator a bulk call of ndraws draws on n rows runs, trees that share their structure
        with the previous draw's tree of the same index)."""
        ev, sh = C.c_int(), C.c_longlong()
        check(_lib.lib().fb_predict_evaluator(self._h, int(n), int(ndraws), C.byref(ev), C.byref(sh)))
        return self.EVALUATORS[ev.value], sh.value

    def handle(self):
        return self._h

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                _lib.lib().fb_compiled_free(self._h)
                self._h = None
        except Exception:
            pass


def compile_trees(fit: BartFit, device: int = 0) -> CompiledTrees:
    """compile_trees() of R/predict_draw.R:3-10."""
    cps = list(fit["treedraws"]["cutpoints"].values())
    if fit.get("binaryOffset") is not None:
        mu = fit["binaryOffset"]
    else:
        mu = fit.get("mu", fit.get("offset", 0.0))
    return CompiledTrees(fit["treedraws"]["trees"], cps, mu, fit.get("rm.const"), getattr(fit, "cls", "") == "pbart",
                         device)


def predict_draws_device(ct: CompiledTrees, x_ptr: int, ncol: int, n: int, ld: int, draw0: int, ndraws: int,
                         out_ptr: int, ldo: int, stream: int = 0) -> None:
    """Bulk predict_draw on device memory (fb_predict_draws_device): column v of x at x_ptr + 8*v*ld, draw
    draw0 + d (1-based) written to out_ptr + 8*d*ldo; enqueued on `stream` (a CUDA stream handle, 0 = default)."""
    check(_lib.lib().fb_predict_draws_device(ct.handle(), x_ptr, int(ncol), int(n), int(ld), int(draw0), int(ndraws),
                                             ct.mu, out_ptr, int(ldo), stream or None))


def predict_draw(ct: CompiledTrees, newdata, m: int) -> np.ndarray:
    """predict_draw() of R/predict_draw.R:13-18: f (+ mu) of posterior draw m (1-based) on the rows of newdata."""
    X = np.asarray(newdata, dtype=np.float64)
    if X.ndim == 1:
        X = X[:, None]
    if ct.rm_const is not None and len(ct.rm_const) < X.shape[1]:
        X = X[:, np.asarray(ct.rm_const) - 1]
    cols = [np.ascontiguousarray(X[:, j]) for j in range(X.shape[1])]
    n = X.shape[0]
    ptrs = (C.c_void_p * max(1, len(cols)))(*[c.ctypes.data for c in cols])
    out = np.zeros(n)
    check(_lib.lib().fb_predict_draw(ct.handle(), ptrs, len(cols), n, int(m), ct.mu, ptr(out)))
    return out
