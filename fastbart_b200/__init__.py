"""fastbart_b200: B200-native (sm_100a) restructured BART backfitting sampler (fwbart / fpbart) and the
compile_trees / predict_draw evaluator, behind the C ABI of include/fastbart_b200.h."""
from ._lib import FastbartError, lib, lib_path, version
from .api import (Batch, CompiledTrees, autotune, compile_trees, cut_codes, cut_loss_grad, fit_batch, fpbart, fwbart,
                  mlp_loss_grad, predict_draw, predict_draws_device, probit_latent_device, release_cached_memory, sigma_estimate,
                  train_cut_proposal, train_proposal, trees_text, trees_text_gpu, varcount)

__all__ = ["FastbartError", "lib", "lib_path", "version", "Batch", "CompiledTrees", "compile_trees", "fit_batch",
           "fpbart", "fwbart", "predict_draw", "predict_draws_device", "trees_text", "trees_text_gpu", "varcount",
           "train_proposal", "mlp_loss_grad", "autotune", "cut_codes", "release_cached_memory", "train_cut_proposal",
           "cut_loss_grad", "probit_latent_device", "sigma_estimate"]
