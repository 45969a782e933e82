"""ctypes binding of libfastbart_b200.so (include/fastbart_b200.h).

The library is built in-tree (fastbart_b200/lib/) by fastbart_b200._build; importing this module never falls back to a
CPU implementation: if the library is missing or cannot be loaded, lib() raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _build

NODES = 64
FB_OK, FB_ERR_ARG, FB_ERR_LIMIT, FB_ERR_CUDA, FB_ERR_PARSE, FB_ERR_SHAPE, FB_ERR_RANGE = range(7)

EXPORTS = ["fb_last_error", "fb_version", "fb_fit_batch", "fb_batch_create", "fb_batch_run", "fb_batch_sync",
           "fb_batch_download", "fb_batch_launch_info", "fb_batch_destroy", "fb_fbart", "fb_trees_text",
           "fb_varcount", "fb_compile_trees", "fb_compiled_info", "fb_predict_evaluator", "fb_probit_latent_device", "fb_sigma_estimate", "fb_compiled_arrays", "fb_compiled_free",
           "fb_predict_draw", "fb_predict_draws_device", "fb_predict_draw_static", "fb_debug_tree_pass",
           "fb_batch_set_proposal", "fb_batch_collect", "fb_batch_training_data", "fb_train_proposal",
           "fb_mlp_loss_grad", "fb_autotune", "fb_cut_codes", "fb_trees_text_gpu", "fb_batch_trees_text",
           "fb_release_cached_memory", "fb_batch_autotuned", "fb_batch_set_cut_proposal",
           "fb_batch_cut_training_data", "fb_train_cut_proposal", "fb_cut_loss_grad"]

MLP_IN, MLP_H, MLP_OUT = 98, 64, 32


class ProposalModel(C.Structure):
    _fields_ = [("w1", C.c_void_p), ("b1", C.c_void_p), ("w2", C.c_void_p), ("b2", C.c_void_p),
                ("w3", C.c_void_p), ("b3", C.c_void_p), ("mix", C.c_double)]


class CutModel(C.Structure):
    _fields_ = [("w1", C.c_void_p), ("b1", C.c_void_p), ("w2", C.c_void_p), ("b2", C.c_void_p),
                ("w3", C.c_void_p), ("b3", C.c_void_p), ("emb", C.c_void_p), ("be", C.c_void_p),
                ("mix", C.c_double)]


CUT_IN, CUT_H, CUT_E, CUT_BINS = 40, 64, 16, 255


class TrainOptions(C.Structure):
    _fields_ = [("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_double), ("seed", C.c_uint64),
                ("device", C.c_int)]


class FastbartError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(msg)
        self.status = status


class Chain(C.Structure):
    _fields_ = [("n", C.c_int), ("p", C.c_int), ("ntree", C.c_int), ("q", C.c_void_p), ("y", C.c_void_p),
                ("wt", C.c_void_p), ("ybin", C.c_void_p), ("numcut", C.c_void_p), ("pgtab", C.c_void_p),
                ("tau", C.c_double), ("lambda_", C.c_double), ("nu", C.c_double), ("sigest", C.c_double),
                ("offset", C.c_double), ("seed", C.c_uint64), ("probit", C.c_int), ("fx_shift", C.c_int),
                ("rss_shift", C.c_int)]


class Options(C.Structure):
    _fields_ = [("nskip", C.c_int), ("ndpost", C.c_int), ("threads", C.c_int), ("sweeps_per_launch", C.c_int),
                ("device", C.c_int), ("cluster", C.c_int)]


class ChainOut(C.Structure):
    _fields_ = [("sigma", C.c_void_p), ("yhat_mean", C.c_void_p), ("yhat", C.c_void_p), ("trees", C.c_void_p),
                ("moves", C.c_int * 3), ("rtnorm_caps", C.c_int)]


class PassState(C.Structure):
    _fields_ = [(k, C.c_int) for k in ("n", "apply", "stats", "fx_shift", "threads", "pmode", "pnx", "pc", "pL",
                                       "pR", "pl", "pr", "cmode", "cnx", "cc")] + \
               [("leafmask", C.c_uint64)] + \
               [(k, C.c_void_p) for k in ("leaf_prev", "leaf_cur", "qprev", "qcur", "r", "w", "tho", "thn", "thc")]


_lib = None


def lib_path() -> str:
    return _build.LIB


def lib() -> C.CDLL:
    """Loads the library, building it first if the in-tree copy is missing or older than its sources."""
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path) or _build._stale():
            try:
                _build.build()
            except Exception as e:   # no toolchain: only a prebuilt library can be used
                if not os.path.exists(path):
                    raise FastbartError(FB_ERR_CUDA, f"libfastbart_b200.so is missing and cannot be built: {e}")
        L = C.CDLL(path)
        vp, i, d, sz = C.c_void_p, C.c_int, C.c_double, C.c_size_t
        L.fb_last_error.restype = C.c_char_p
        L.fb_version.restype = C.c_char_p
        L.fb_fit_batch.argtypes = [C.POINTER(Chain), i, C.POINTER(Options), C.POINTER(ChainOut)]
        L.fb_batch_create.argtypes = [C.POINTER(Chain), i, C.POINTER(Options), C.POINTER(vp)]
        L.fb_batch_run.argtypes = [vp, vp]
        L.fb_batch_sync.argtypes = [vp]
        L.fb_batch_download.argtypes = [vp, C.POINTER(ChainOut)]
        L.fb_batch_launch_info.argtypes = [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(sz), C.POINTER(i)]
        L.fb_batch_destroy.argtypes = [vp]
        L.fb_batch_destroy.restype = None
        L.fb_batch_autotuned.argtypes = [vp]
        L.fb_batch_set_cut_proposal.argtypes = [vp, C.POINTER(CutModel)]
        L.fb_batch_cut_training_data.argtypes = [vp, vp, vp, vp, vp, i, C.POINTER(i)]
        L.fb_train_cut_proposal.argtypes = [vp, vp, vp, vp, i, C.POINTER(TrainOptions), C.POINTER(CutModel)] + [vp] * 9
        L.fb_cut_loss_grad.argtypes = [C.POINTER(CutModel), vp, vp, vp, vp, i, i, C.POINTER(d)] + [vp] * 8
        L.fb_fbart.argtypes = [vp, i, i, vp, vp, vp, vp, vp, i, i, i, d, d, d, d, C.c_uint64, i, d, vp, vp, vp, vp,
                               C.c_char_p, sz, C.POINTER(sz), vp]
        L.fb_trees_text.argtypes = [vp, i, i, i, C.c_char_p, sz]
        L.fb_trees_text.restype = sz
        L.fb_varcount.argtypes = [vp, i, i, i, vp]
        L.fb_trees_text_gpu.argtypes = [vp, i, i, i, i, C.c_char_p, sz, C.POINTER(sz)]
        L.fb_batch_trees_text.argtypes = [vp, i, C.c_char_p, sz, C.POINTER(sz)]
        L.fb_release_cached_memory.argtypes = [i]
        L.fb_compile_trees.argtypes = [C.c_char_p, sz, vp, vp, i, i, C.POINTER(vp)]
        L.fb_compiled_info.argtypes = [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i)]
        L.fb_predict_evaluator.argtypes = [vp, i, i, C.POINTER(i), C.POINTER(C.c_longlong)]
        L.fb_probit_latent_device.argtypes = [vp, vp, C.c_longlong, d, C.c_uint64, i, vp, vp, vp]
        L.fb_sigma_estimate.argtypes = [vp, i, i, vp, i, C.POINTER(d), C.POINTER(i)]
        L.fb_compiled_arrays.argtypes = [vp, vp, vp, vp, vp, vp]
        L.fb_compiled_free.argtypes = [vp]
        L.fb_compiled_free.restype = None
        L.fb_predict_draw.argtypes = [vp, vp, i, i, i, d, vp]
        L.fb_predict_draws_device.argtypes = [vp, vp, i, i, i, i, i, d, vp, i, vp]
        L.fb_predict_draw_static.argtypes = [vp, vp, i, i, i, d, vp]
        L.fb_debug_tree_pass.argtypes = [C.POINTER(PassState), vp]
        L.fb_batch_set_proposal.argtypes = [vp, C.POINTER(ProposalModel)]
        L.fb_cut_codes.argtypes = [vp, i, i, vp, vp, i, vp]
        L.fb_autotune.argtypes = [C.POINTER(Chain), i, C.POINTER(Options), i, C.POINTER(Options), C.POINTER(d)]
        L.fb_batch_collect.argtypes = [vp, i]
        L.fb_batch_training_data.argtypes = [vp, vp, vp, vp, i, C.POINTER(i)]
        L.fb_train_proposal.argtypes = [vp, vp, vp, i, C.POINTER(TrainOptions), C.POINTER(ProposalModel),
                                        vp, vp, vp, vp, vp, vp, vp]
        L.fb_mlp_loss_grad.argtypes = [C.POINTER(ProposalModel), vp, vp, vp, i, i, C.POINTER(d), vp, vp, vp, vp, vp,
                                       vp]
        for f in EXPORTS:
            if f not in ("fb_last_error", "fb_version", "fb_trees_text", "fb_batch_destroy", "fb_compiled_free"):
                getattr(L, f).restype = C.c_int
        _lib = L
    return _lib


def check(status: int):
    if status != FB_OK:
        raise FastbartError(status, lib().fb_last_error().decode())


def ptr(a) -> int | None:
    return None if a is None else a.ctypes.data


def version() -> str:
    return lib().fb_version().decode()
