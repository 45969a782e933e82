"""ctypes front end of the CPU oracle (oracle/liborc.so) and of the reference library built from source
(oracle/_ref/libbartref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg as
the checker.  The product package fastbart_b200 never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBORC = os.path.join(HERE, "liborc.so")
LIBREF = os.path.join(HERE, "_ref", "libbartref.so")
REF_BATCH = os.path.join(HERE, "_ref", "bart_batch")
LIBPREDREF = os.path.join(HERE, "_ref", "libpredref.so")

NODES = 64
MODE_REF, MODE_DEV = 0, 1

_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C")


class _Chain(C.Structure):
    _fields_ = [("n", C.c_int), ("p", C.c_int), ("m", C.c_int), ("nskip", C.c_int), ("ndpost", C.c_int),
                ("q", C.c_void_p), ("y", C.c_void_p), ("wt", C.c_void_p), ("ybin", C.c_void_p),
                ("numcut", C.c_void_p), ("pgtab", C.c_void_p),
                ("tau", C.c_double), ("lambda_", C.c_double), ("nu", C.c_double), ("sigest", C.c_double),
                ("offset", C.c_double), ("seed", C.c_uint64), ("probit", C.c_int), ("fx_shift", C.c_int),
                ("rss_shift", C.c_int), ("model", C.c_void_p), ("cut", C.c_void_p)]


class _Out(C.Structure):
    _fields_ = [("sigma", C.c_void_p), ("fmean", C.c_void_p), ("yhat", C.c_void_p), ("trees", C.c_void_p),
                ("moves", C.c_int * 3), ("rtnorm_caps", C.c_int), ("train_x", C.c_void_p), ("train_y", C.c_void_p),
                ("train_mask", C.c_void_p), ("train_cap", C.c_int), ("train_count", C.c_int),
                ("train_cx", C.c_void_p), ("train_c", C.c_void_p), ("train_lo", C.c_void_p), ("train_hi", C.c_void_p)]


MLP_IN, MLP_H, MLP_OUT = 98, 64, 32
CUT_IN, CUT_H, CUT_E, CUT_BINS = 40, 64, 16, 255


class _CutModel(C.Structure):
    _fields_ = [("w1", C.c_void_p), ("b1", C.c_void_p), ("w2", C.c_void_p), ("b2", C.c_void_p),
                ("w3", C.c_void_p), ("b3", C.c_void_p), ("emb", C.c_void_p), ("be", C.c_void_p), ("mix", C.c_double)]


CUT_KEYS = (("w1", np.uint16), ("b1", np.float32), ("w2", np.uint16), ("b2", np.float32), ("w3", np.uint16),
            ("b3", np.float32), ("emb", np.uint16), ("be", np.float32))


def _cut_struct(model: dict, keep: list):
    """orc_cut_model from a dict of w1 [64][40], w2 [64][64], w3 [16][64], emb [255][16] (uint16 BF16 bits), b1, b2, b3,
    be (float32), mix."""
    arrs = {k: np.ascontiguousarray(model[k], dtype=dt) for k, dt in CUT_KEYS}
    keep += list(arrs.values())
    return _CutModel(*(arrs[k].ctypes.data for k, _ in CUT_KEYS), float(model.get("mix", 0.5)))


class _Model(C.Structure):
    _fields_ = [("w1", C.c_void_p), ("b1", C.c_void_p), ("w2", C.c_void_p), ("b2", C.c_void_p),
                ("w3", C.c_void_p), ("b3", C.c_void_p), ("mix", C.c_double)]


def _model_struct(model: dict, keep: list):
    """orc_model from a dict of w1 [64][98], w2 [64][64], w3 [32][64] (uint16 BF16 bits), b1, b2, b3 (float32), mix."""
    arrs = {}
    for k, dt in (("w1", np.uint16), ("w2", np.uint16), ("w3", np.uint16), ("b1", np.float32), ("b2", np.float32),
                  ("b3", np.float32)):
        arrs[k] = np.ascontiguousarray(model[k], dtype=dt)
        keep.append(arrs[k])
    return _Model(*(arrs[k].ctypes.data for k in ("w1", "b1", "w2", "b2", "w3", "b3")), float(model.get("mix", 0.5)))


class _Upd(C.Structure):
    _fields_ = [(k, C.c_int) for k in ("mode", "nx", "v", "c", "L", "R", "l", "r")]


class _Prop(C.Structure):
    _fields_ = [(k, C.c_int) for k in ("mode", "nx", "v", "c")]


class _Stats(C.Structure):
    _fields_ = [("S0", C.c_int64 * NODES), ("S1", C.c_int64 * NODES), ("sL0", C.c_int64), ("sL1", C.c_int64),
                ("sR0", C.c_int64), ("sR1", C.c_int64), ("nL", C.c_int), ("nR", C.c_int)]


class _CT(C.Structure):
    _fields_ = [("ndpost", C.c_int), ("ntree", C.c_int), ("p", C.c_int), ("nnodes", C.c_int),
                ("var", C.POINTER(C.c_int)), ("child", C.POINTER(C.c_int)), ("cut", C.POINTER(C.c_double)),
                ("theta", C.POINTER(C.c_double)), ("root", C.POINTER(C.c_int))]


_lib = None
_ref = None


def build():
    """Builds liborc.so (and oracle/_ref when the reference sources are present) with make."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBORC):
            build()
        L = C.CDLL(LIBORC)
        L.orc_fit.argtypes = [C.POINTER(_Chain), C.c_int, C.POINTER(_Out)]
        L.orc_fit.restype = C.c_int
        L.orc_pass_dev.argtypes = [C.c_int, C.c_void_p, C.c_void_p, _f32p, _f32p, C.c_void_p, C.c_void_p,
                                   C.POINTER(_Upd), _f32p, _f32p, C.c_int, C.POINTER(_Prop), _f32p, C.c_int,
                                   C.POINTER(_Stats)]
        L.orc_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        for f in ("orc_log", "orc_exp"):
            getattr(L, f).argtypes = [C.c_double]
            getattr(L, f).restype = C.c_double
        L.orc_normal.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_normal.restype = C.c_double
        L.orc_gamma.argtypes = [C.c_uint64, C.c_uint32, C.c_double]
        L.orc_gamma.restype = C.c_double
        L.orc_rtnorm.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.POINTER(C.c_int)]
        L.orc_rtnorm.restype = C.c_double
        L.orc_probit_latent.argtypes = [C.c_uint64, C.c_uint32, C.c_double, C.c_void_p, C.c_void_p, C.c_longlong,
                                        C.c_void_p]
        L.orc_probit_latent.restype = C.c_int
        L.orc_compile_trees.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(_CT)]
        L.orc_compile_trees.restype = C.c_int
        L.orc_ct_free.argtypes = [C.POINTER(_CT)]
        L.orc_mlp_logits.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_mlp_logits.restype = None
        L.orc_mlp_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int] + [C.c_void_p] * 6
        L.orc_mlp_loss_grad.restype = C.c_double
        L.orc_cut_logits.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.orc_cut_logits.restype = None
        L.orc_cut_loss_grad.argtypes = [C.c_void_p] * 5 + [C.c_int] + [C.c_void_p] * 8
        L.orc_cut_loss_grad.restype = C.c_double
        L.orc_predict_draw.argtypes = [C.POINTER(_CT), C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, _f64p]
        L.orc_predict_draw.restype = C.c_int
        L.orc_trees_text.argtypes = [_u64p, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_size_t]
        L.orc_trees_text.restype = C.c_size_t
        L.orc_varcount.argtypes = [_u64p, C.c_int, C.c_int, C.c_int, _i32p]
        L.orc_yhat_from_trees.argtypes = [_u64p, C.c_int, C.c_int, _u8p, C.c_int, _f64p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(LIBREF)


def reflib():
    global _ref
    if _ref is None:
        R = C.CDLL(LIBREF)
        R.bart_fit_cpu.argtypes = [_u8p, _f32p, _f32p, _i32p, _f32p, _f32p, _f32p, _u64p, C.c_int, C.c_int, C.c_int,
                                   C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_uint, C.c_int,
                                   _i32p, C.c_int, C.c_void_p, C.c_float]
        R.bart_set_rng.argtypes = [C.c_void_p] * 4
        R.bart_set_rng(None, None, None, None)
        _ref = R
    return _ref


def _keep(*arrs):
    return [np.ascontiguousarray(a) for a in arrs]


def fit(ch: dict, mode: int, want_trees: bool = True, model: dict | None = None, train_cap: int = 0,
        cut: dict | None = None) -> dict:
    """Runs one chain in the oracle.  ch keys: q [p][n] u8, y, wt, ybin, numcut, pgtab, tau, lambda, nu, sigest,
    offset, seed, probit, nskip, ndpost, ntree, fx_shift, rss_shift.  DEV mode: `model` = learned proposal (see
    _model_struct); train_cap > 0 collects accepted births as training examples (train_x, train_y, train_mask)."""
    q = np.ascontiguousarray(ch["q"], dtype=np.uint8)
    p, n = q.shape
    m, nskip, ndpost = int(ch["ntree"]), int(ch["nskip"]), int(ch["ndpost"])
    probit = int(ch.get("probit", 0))
    y = np.ascontiguousarray(ch.get("y", np.zeros(n)), dtype=np.float64)
    wt = np.ascontiguousarray(ch.get("wt", np.ones(n)), dtype=np.float64)
    ybin = np.ascontiguousarray(ch.get("ybin", np.zeros(n)), dtype=np.int32)
    numcut = np.ascontiguousarray(ch["numcut"], dtype=np.int32)
    pg = np.ascontiguousarray(ch["pgtab"], dtype=np.float64)
    c = _Chain(n, p, m, nskip, ndpost, q.ctypes.data, y.ctypes.data, wt.ctypes.data, ybin.ctypes.data,
               numcut.ctypes.data, pg.ctypes.data, ch["tau"], ch["lambda"], ch["nu"], ch["sigest"],
               ch.get("offset", 0.0), int(ch["seed"]) & 0xFFFFFFFFFFFFFFFF, probit, int(ch.get("fx_shift", 32)),
               int(ch.get("rss_shift", 24)), None)
    keep: list = []
    if model is not None:
        ms = _model_struct(model, keep)
        keep.append(ms)
        c.model = C.cast(C.pointer(ms), C.c_void_p)
    if cut is not None:
        cs = _cut_struct(cut, keep)
        keep.append(cs)
        c.cut = C.cast(C.pointer(cs), C.c_void_p)
    S = nskip + ndpost
    sigma = np.zeros(S)
    fmean = np.zeros(n)
    yhat = np.zeros((ndpost, n))
    trees = np.zeros((ndpost, m, NODES), dtype=np.uint64) if want_trees or mode == MODE_REF else None
    tx = np.zeros((max(train_cap, 1), MLP_IN), dtype=np.float32)
    ty = np.zeros(max(train_cap, 1), dtype=np.int32)
    tm = np.zeros(max(train_cap, 1), dtype=np.uint32)
    o = _Out(sigma.ctypes.data, fmean.ctypes.data, yhat.ctypes.data, trees.ctypes.data if trees is not None else None)
    o.train_x, o.train_y, o.train_mask, o.train_cap = tx.ctypes.data, ty.ctypes.data, tm.ctypes.data, int(train_cap)
    cx = np.zeros((max(train_cap, 1), CUT_IN), dtype=np.float32)
    cc, clo, chi = (np.zeros(max(train_cap, 1), dtype=np.int32) for _ in range(3))
    o.train_cx, o.train_c, o.train_lo, o.train_hi = cx.ctypes.data, cc.ctypes.data, clo.ctypes.data, chi.ctypes.data
    rc = lib().orc_fit(C.byref(c), mode, C.byref(o))
    if rc != 0:
        raise ValueError(f"orc_fit returned {rc}")
    k = o.train_count
    return dict(sigma=sigma, fmean=fmean, yhat=yhat, trees=trees, moves=np.array(list(o.moves)),
                rtnorm_caps=o.rtnorm_caps, train_x=tx[:k], train_y=ty[:k], train_mask=tm[:k], train_cx=cx[:k],
                train_c=cc[:k], train_lo=clo[:k], train_hi=chi[:k])


def cut_logits(cut: dict, x: np.ndarray, lo: int, hi: int) -> np.ndarray:
    """The cut head's logits over [lo, hi] (float32, other entries 0)."""
    keep: list = []
    cs = _cut_struct(cut, keep)
    xs = np.ascontiguousarray(x, dtype=np.float32)
    z = np.zeros(CUT_BINS, dtype=np.float32)
    lib().orc_cut_logits(C.byref(cs), xs.ctypes.data, int(lo), int(hi), z.ctypes.data)
    return z


def cut_loss_grad(cut: dict, X, c, lo, hi) -> tuple[float, dict]:
    keep: list = []
    cs = _cut_struct(cut, keep)
    X = np.ascontiguousarray(X, dtype=np.float32)
    c, lo, hi = (np.ascontiguousarray(a, dtype=np.int32) for a in (c, lo, hi))
    shapes = dict(w1=(CUT_H, CUT_IN), b1=(CUT_H,), w2=(CUT_H, CUT_H), b2=(CUT_H,), w3=(CUT_E, CUT_H), b3=(CUT_E,),
                  emb=(CUT_BINS, CUT_E), be=(CUT_BINS,))
    g = {k: np.zeros(v) for k, v in shapes.items()}
    loss = lib().orc_cut_loss_grad(C.byref(cs), X.ctypes.data, c.ctypes.data, lo.ctypes.data, hi.ctypes.data, len(c),
                                   *(g[k].ctypes.data for k in ("w1", "b1", "w2", "b2", "w3", "b3", "emb", "be")))
    return float(loss), g


def mlp_logits(model: dict, x: np.ndarray) -> np.ndarray:
    keep: list = []
    ms = _model_struct(model, keep)
    xs = np.ascontiguousarray(x, dtype=np.float32)
    z = np.zeros(MLP_OUT, dtype=np.float32)
    lib().orc_mlp_logits(C.byref(ms), xs.ctypes.data, z.ctypes.data)
    return z


def mlp_loss_grad(model: dict, X, y, mask) -> tuple[float, dict]:
    """Mean masked cross-entropy and its FP64 gradients (the checker of the device training kernels)."""
    keep: list = []
    ms = _model_struct(model, keep)
    X = np.ascontiguousarray(X, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.int32)
    mask = np.ascontiguousarray(mask, dtype=np.uint32)
    g = {k: np.zeros(sh) for k, sh in (("w1", (MLP_H, MLP_IN)), ("b1", MLP_H), ("w2", (MLP_H, MLP_H)), ("b2", MLP_H),
                                      ("w3", (MLP_OUT, MLP_H)), ("b3", MLP_OUT))}
    loss = lib().orc_mlp_loss_grad(C.byref(ms), X.ctypes.data, y.ctypes.data, mask.ctypes.data, len(y),
                                   *(g[k].ctypes.data for k in ("w1", "b1", "w2", "b2", "w3", "b3")))
    return float(loss), g


def ref_fit(ch: dict) -> dict:
    """Runs the reference bart_fit_cpu (oracle/_ref/libbartref.so) with glue.cpp's float conversions."""
    R = reflib()
    q = np.ascontiguousarray(ch["q"], dtype=np.uint8)
    p, n = q.shape
    m, nskip, ndpost = int(ch["ntree"]), int(ch["nskip"]), int(ch["ndpost"])
    probit = int(ch.get("probit", 0))
    y = np.ascontiguousarray(ch.get("y", np.zeros(n)), dtype=np.float32) if not probit else np.zeros(n, np.float32)
    wt = np.ascontiguousarray(ch.get("wt", np.ones(n)), dtype=np.float32)
    ybin = np.ascontiguousarray(ch.get("ybin", np.zeros(n)), dtype=np.int32)
    numcut = np.ascontiguousarray(ch["numcut"], dtype=np.int32)
    pg = np.ascontiguousarray(ch["pgtab"], dtype=np.float32)
    sig = np.zeros(nskip + ndpost, np.float32)
    trm = np.zeros(n, np.float32)
    trees = np.zeros((ndpost, m, NODES), np.uint64)
    st = np.zeros(8, np.int32)
    R.bart_fit_cpu(q, y, wt, numcut, pg, sig, trm, trees, n, p, m, nskip, ndpost, ch["tau"], ch["lambda"], ch["nu"],
                   ch["sigest"], int(ch["seed"]) & 0xFFFFFFFF, 1, st, probit, ybin.ctypes.data, ch.get("offset", 0.0))
    return dict(sigma=sig.astype(np.float64), fmean=trm.astype(np.float64), trees=trees, moves=st[:3].copy())


def pass_dev(n, leaf_prev, leaf_cur, r, w, qprev, qcur, upd, tho, thn, apply, prop, thc, fx_shift):
    """Per-tree fused pass in DEV arithmetic.  Mutates leaf_prev and r in place; returns the stats dict."""
    st = _Stats()
    u = _Upd(*[int(upd.get(k, 0)) for k in ("mode", "nx", "v", "c", "L", "R", "l", "r")])
    pr = _Prop(*[int(prop.get(k, 0)) for k in ("mode", "nx", "v", "c")])
    lib().orc_pass_dev(n, leaf_prev.ctypes.data if leaf_prev is not None else None,
                       leaf_cur.ctypes.data if leaf_cur is not None else None, r, w,
                       qprev.ctypes.data if qprev is not None else None, qcur.ctypes.data if qcur is not None else None,
                       C.byref(u), tho, thn, int(apply), C.byref(pr), thc, int(fx_shift), C.byref(st))
    return dict(S0=np.array(st.S0[:], dtype=np.int64), S1=np.array(st.S1[:], dtype=np.int64),
                split=np.array([st.sL0, st.sL1, st.sR0, st.sR1], dtype=np.int64), nL=st.nL, nR=st.nR)


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox(c, k, o)
    return list(o)


def log(x):
    return lib().orc_log(float(x))


def exp(x):
    return lib().orc_exp(float(x))


def normal(seed, c0, c1, c2, tag):
    return lib().orc_normal(seed, c0, c1, c2, tag)


def gamma(seed, it, a):
    return lib().orc_gamma(seed, it, a)


def probit_latent(seed, it, offset, fit, ybin):
    """z of every row at sweep `it` (-1: the initial draw) as the sampler draws it, and the capped draw count."""
    f = np.ascontiguousarray(fit, dtype=np.float64)
    y = np.ascontiguousarray(ybin, dtype=np.int32)
    z = np.empty_like(f)
    caps = lib().orc_probit_latent(int(seed) & (2**64 - 1), int(it) & 0xFFFFFFFF, float(offset), f.ctypes.data,
                                   y.ctypes.data, f.size, z.ctypes.data)
    return z, caps


def rtnorm(seed, row, it, mean, tau):
    cap = C.c_int(0)
    v = lib().orc_rtnorm(seed, row, it, mean, tau, C.byref(cap))
    return v, cap.value


class Compiled:
    def __init__(self, ct: _CT):
        self._ct = ct
        N = ct.nnodes
        self.ndpost, self.ntree, self.p = ct.ndpost, ct.ntree, ct.p
        self.var = np.ctypeslib.as_array(ct.var, (N,)).copy()
        self.child = np.ctypeslib.as_array(ct.child, (N,)).copy()
        self.cut = np.ctypeslib.as_array(ct.cut, (N,)).copy()
        self.theta = np.ctypeslib.as_array(ct.theta, (N,)).copy()
        self.root = np.ctypeslib.as_array(ct.root, (ct.ndpost * ct.ntree,)).copy()

    def __del__(self):
        try:
            lib().orc_ct_free(C.byref(self._ct))
        except Exception:
            pass


def compile_trees(text: str, cutpoints) -> Compiled:
    xs = [np.ascontiguousarray(c, dtype=np.float64) for c in cutpoints]
    ptrs = (C.c_void_p * max(1, len(xs)))(*[x.ctypes.data for x in xs])
    nc = np.array([len(x) for x in xs], dtype=np.int32)
    ct = _CT()
    rc = lib().orc_compile_trees(text.encode(), ptrs, nc.ctypes.data, len(xs), C.byref(ct))
    if rc != 0:
        raise ValueError("bad tree text")
    obj = Compiled(ct)
    obj._keep = (xs, ptrs, nc)
    return obj


def predict_draw(ct: Compiled, cols, draw1: int, mu: float) -> np.ndarray:
    xs = [np.ascontiguousarray(c, dtype=np.float64) for c in cols]
    n = len(xs[0]) if xs else 0
    ptrs = (C.c_void_p * max(1, len(xs)))(*[x.ctypes.data for x in xs])
    out = np.zeros(n)
    rc = lib().orc_predict_draw(C.byref(ct._ct), ptrs, len(xs), n, int(draw1), float(mu), out)
    if rc == -1:
        raise ValueError(f"newdata has {len(xs)} columns, the trees use {ct.p}")
    if rc == -2:
        raise ValueError(f"draw {draw1} out of range 1..{ct.ndpost}")
    return out


# ---- the reference's own evaluator (src/predict.cpp built from source into oracle/_ref/libpredref.so)
_predref = None


def ref_predict_available() -> bool:
    return os.path.exists(LIBPREDREF)


def predreflib():
    global _predref
    if _predref is None:
        R = C.CDLL(LIBPREDREF)
        R.refp_compile.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_int, C.c_char_p, C.c_int]
        R.refp_compile.restype = C.c_void_p
        R.refp_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 4
        R.refp_info.restype = None
        R.refp_arrays.argtypes = [C.c_void_p] * 6
        R.refp_arrays.restype = None
        R.refp_predict.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p,
                                   C.c_char_p, C.c_int]
        R.refp_predict.restype = C.c_int
        R.refp_free.argtypes = [C.c_void_p]
        R.refp_free.restype = None
        _predref = R
    return _predref


class RefCompiled:
    """compile_trees_cpp's result list as computed by the reference's own code: the node arrays, and a handle for
    predict_draw_cpp."""

    def __init__(self, text: str, cutpoints):
        R = predreflib()
        xs = [np.ascontiguousarray(c, dtype=np.float64) for c in cutpoints]
        ptrs = (C.c_void_p * max(1, len(xs)))(*[x.ctypes.data for x in xs])
        nc = np.array([len(x) for x in xs], dtype=np.int32)
        err = C.create_string_buffer(256)
        self._h = R.refp_compile(text.encode(), ptrs, nc.ctypes.data, len(xs), err, 256)
        if not self._h:
            raise ValueError(err.value.decode())
        nd, m, p, nn = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        R.refp_info(self._h, C.byref(nd), C.byref(m), C.byref(p), C.byref(nn))
        self.ndpost, self.ntree, self.p, self.nnodes = nd.value, m.value, p.value, nn.value
        self.var, self.child = np.zeros(nn.value, np.int32), np.zeros(nn.value, np.int32)
        self.cut, self.theta = np.zeros(nn.value), np.zeros(nn.value)
        self.root = np.zeros(nd.value * m.value, np.int32)
        R.refp_arrays(self._h, *(a.ctypes.data for a in (self.var, self.child, self.cut, self.theta, self.root)))

    def predict_draw(self, cols, draw1: int, mu: float) -> np.ndarray:
        xs = [np.ascontiguousarray(c, dtype=np.float64) for c in cols]
        n = len(xs[0]) if xs else 0
        ptrs = (C.c_void_p * max(1, len(xs)))(*[x.ctypes.data for x in xs])
        out = np.zeros(n)
        err = C.create_string_buffer(256)
        if predreflib().refp_predict(self._h, ptrs, len(xs), n, int(draw1), float(mu), out.ctypes.data, err, 256):
            raise ValueError(err.value.decode())
        return out

    def __del__(self):
        if getattr(self, "_h", None) and _predref is not None:
            _predref.refp_free(self._h)
            self._h = None


def trees_text(trees: np.ndarray, p: int) -> str:
    t = np.ascontiguousarray(trees, dtype=np.uint64)
    nd, m = t.shape[0], t.shape[1]
    ln = lib().orc_trees_text(t, nd, m, p, None, 0)
    buf = C.create_string_buffer(ln + 1)
    lib().orc_trees_text(t, nd, m, p, buf, ln + 1)
    return buf.raw[:ln].decode()


def varcount(trees: np.ndarray, p: int) -> np.ndarray:
    t = np.ascontiguousarray(trees, dtype=np.uint64)
    out = np.zeros((t.shape[0], p), dtype=np.int32)
    lib().orc_varcount(t, t.shape[0], t.shape[1], p, out)
    return out


def yhat_from_trees(trees: np.ndarray, q: np.ndarray) -> np.ndarray:
    t = np.ascontiguousarray(trees, dtype=np.uint64)
    qq = np.ascontiguousarray(q, dtype=np.uint8)
    out = np.zeros((t.shape[0], qq.shape[1]))
    lib().orc_yhat_from_trees(t, t.shape[0], t.shape[1], qq, qq.shape[1], out)
    return out
