/*
 * fastbart_b200.h -- C ABI of the B200 implementation of fastbart's hot path.
 *
 * One shared library (libfastbart_b200.so) replaces the native side of the reference R package:
 *   - the sampler call that src/glue.cpp:26-27 makes into bart_fit_cpu (src/bart_kernel.h:63-66) and the output
 *     assembly around it (src/glue.cpp:29-61);
 *   - compile_trees_cpp / predict_draw_cpp (src/predict.cpp:11-73);
 *   - the batch GPU prototype's fit list (gpu/bart_gpu.cu:326-404) via fb_fit_batch.
 *
 * Conventions: plain C types; every buffer is owned by the caller; sizes are element counts.  Functions return an
 * fb_status; on failure fb_last_error() returns a message for the calling thread.  Calls are thread-safe as long as
 * different threads use different fb_batch / fb_compiled objects.  Results are bit-for-bit deterministic for a given
 * input and seed.  The product never falls back to a CPU path: without a usable CUDA device every compute entry point
 * returns FB_ERR_CUDA.
 */
#ifndef FASTBART_B200_H
#define FASTBART_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef enum fb_status {
  FB_OK = 0,
  FB_ERR_ARG = 1,     /* null pointer or invalid argument */
  FB_ERR_LIMIT = 2,   /* n > 65536, p > 32, ntree > 200, numcut > 255, ... (R/fwbart.R:11-17 falls back to BART) */
  FB_ERR_CUDA = 3,    /* no device, out of device memory, launch or runtime error */
  FB_ERR_PARSE = 4,   /* malformed tree text */
  FB_ERR_SHAPE = 5,   /* predict: newdata has the wrong number of columns (src/predict.cpp:51) */
  FB_ERR_RANGE = 6    /* predict: draw out of range (src/predict.cpp:52) */
} fb_status;

#define FB_NODES 64   /* node slots per tree in the packed tree format (src/bart_kernel.h:23) */

/* Message describing the last failure on the calling thread ("" if none). */
const char* fb_last_error(void);
/* Library version string. */
const char* fb_version(void);

/* ------------------------------------------------------------------------------------------------ sampler */

/* One chain (fit).  Field meanings follow fbart_cpp's arguments (src/glue.cpp:10-12, R/fwbart.R:31-32,
 * R/fpbart.R:24-26). */
typedef struct fb_chain {
  int n, p, ntree;          /* rows (<= 65536), predictors (<= 32), trees (<= 200) */
  const uint8_t* q;         /* [p][n] cutpoint codes: x < cutpoints[v][c]  <=>  q <= c */
  const double* y;          /* [n] centred y (fwbart); ignored when probit */
  const double* wt;         /* [n] 1/w^2 (fwbart); NULL means all ones */
  const int* ybin;          /* [n] 0/1 outcomes (fpbart); NULL unless probit */
  const int* numcut;        /* [p] number of cutpoints of each predictor (1..255) */
  const double* pgtab;      /* [64] base / (1 + depth)^power */
  double tau, lambda, nu, sigest, offset;  /* offset = binaryOffset (fpbart) */
  uint64_t seed;            /* Philox key of the chain */
  int probit;               /* 0: fwbart (weighted continuous), 1: fpbart (probit; sigma fixed at 1) */
  int fx_shift, rss_shift;  /* fixed-point scales 2^fx_shift / 2^rss_shift of the exact sums; 0 = automatic */
} fb_chain;

typedef struct fb_options {
  int nskip, ndpost;        /* burn-in and kept sweeps (shared by all chains of a batch) */
  int threads;              /* threads per CTA; 0 = automatic (with cluster 0: picked by fb_autotune, cached) */
  int sweeps_per_launch;    /* 0 = the whole MCMC in one launch; k > 0 = launches of k sweeps */
  int device;               /* CUDA device ordinal */
  int cluster;              /* CTAs per chain (a thread-block cluster sharing the rows): 0 = automatic, 1 = one CTA,
                               2..16 = that many when they can be resident (above 8: non-portable cluster sizes);
                               results are identical for every value */
} fb_options;

/* Caller-owned host outputs of one chain; a NULL pointer skips that copy. */
typedef struct fb_chain_out {
  double* sigma;            /* [nskip + ndpost] every sigma draw (sigest for probit) */
  double* yhat_mean;        /* [n] posterior mean of f over kept draws, without fmean / binaryOffset */
  double* yhat;             /* [ndpost][n] f of every kept draw: FP64 sum of leaf values in tree order */
  uint64_t* trees;          /* [ndpost][ntree][64] packed nodes (src/bart_kernel.cpp:559-571 format) */
  int moves[3];             /* births, deaths, node-cap hits (src/glue.cpp:61 "moves") */
  int rtnorm_caps;          /* truncated-normal draws that reached their iteration cap (probit) */
} fb_chain_out;

/* Runs every chain's full MCMC (nskip + ndpost sweeps) in one batch on the device and copies the outputs back.
 * Replaces the fit call of src/glue.cpp:26-27 (bart_fit_cpu, src/bart_kernel.h:63-66) and the batch runner of
 * gpu/bart_gpu.cu:366-390. */
fb_status fb_fit_batch(const fb_chain* chains, int nchains, const fb_options* opt, fb_chain_out* outs);

/* Staged use of the same sampler: inputs are uploaded once, fb_batch_run() repeats the full MCMC from the initial
 * state on the device (results are identical every run), fb_batch_download() copies the outputs of the last run. */
typedef struct fb_batch fb_batch;
fb_status fb_batch_create(const fb_chain* chains, int nchains, const fb_options* opt, fb_batch** out);
fb_status fb_batch_run(fb_batch* b, void* cuda_stream);        /* enqueues on cuda_stream (NULL: default stream) */
fb_status fb_batch_sync(fb_batch* b);
fb_status fb_batch_download(fb_batch* b, fb_chain_out* outs);
/* Batches take device memory from a per-device pool that keeps freed blocks for the next batch (no unmapping and
 * remapping between fits); this returns the kept blocks of `device` to the driver.  No counterpart in the reference. */
fb_status fb_release_cached_memory(int device);
/* number of sampler kernel launches per fb_batch_run, the dynamic shared memory / threads / grid of each, and the
 * CTAs per chain (thread-block cluster size; 1 without clusters).  Outputs may be NULL. */
fb_status fb_batch_launch_info(const fb_batch* b, int* launches, int* threads, int* grid, size_t* smem_bytes,
                               int* cluster);
/* 1 when the batch's launch shape was picked by the autotuner (options threads = cluster = 0, the default), 0 when
 * it was given or picked by the built-in rules (environment FASTBART_AUTOTUNE=0).  The autotuner's choice is timed
 * once per device and batch signature (chain count, rows, trees, largest n / ntree / p, probit chains) and reused. */
int fb_batch_autotuned(const fb_batch* b);
void fb_batch_destroy(fb_batch* b);
/* Autotuner of the launch shape: runs trial_sweeps sweeps of the given chains for every candidate shape (threads per
 * CTA 256, 384, 416, 448, 512 x CTAs per chain 1..16 whose clusters are all resident at once), timed with CUDA
 * events, and writes to *best a copy of *opt with the fastest threads and cluster (and its trial time to *best_ms
 * when non-NULL).
 * No counterpart in the reference, whose GPU prototype takes the block size on its command line
 * (gpu/bart_batch.cu:302-308). */
fb_status fb_autotune(const fb_chain* chains, int nchains, const fb_options* opt, int trial_sweeps, fb_options* best,
                      double* best_ms);

/* ---------------------------------------------------------------------------- learned split-variable proposal */

/* Small MLP that proposes the split variable of a birth from node features (depth, row count, per-predictor use in
 * the tree and cut range at the node): FB_MLP_IN -> FB_MLP_H -> FB_MLP_H -> FB_MLP_OUT logits, ReLU between, BF16
 * weights (raw bits), FP32 biases.  A birth draws its variable from the masked softmax with probability mix, else
 * uniformly as BART (src/bart_kernel.cpp:434); the Metropolis-Hastings ratio carries the exact proposal probabilities
 * of the birth and of the reverse birth of a death, so the chain targets the same posterior as BART's proposal.
 * No counterpart in the reference, which always proposes uniformly. */
#define FB_MLP_IN 98
#define FB_MLP_H 64
#define FB_MLP_OUT 32
typedef struct fb_proposal_model {
  const uint16_t* w1; const float* b1;   /* [FB_MLP_H][FB_MLP_IN], [FB_MLP_H] */
  const uint16_t* w2; const float* b2;   /* [FB_MLP_H][FB_MLP_H], [FB_MLP_H] */
  const uint16_t* w3; const float* b3;   /* [FB_MLP_OUT][FB_MLP_H], [FB_MLP_OUT] */
  double mix;                            /* probability of the model component, in (0, 1]; <= 0: BART's proposal */
} fb_proposal_model;
/* Uses `model` (copied to the device) for the batch's next runs; NULL or mix <= 0 restores BART's proposal. */
fb_status fb_batch_set_proposal(fb_batch* b, const fb_proposal_model* model);
/* Collects every accepted birth of the next runs as a training example (features of the node before the birth, the
 * split variable, the mask of predictors with a non-empty cut range there), up to `capacity` per run; 0 stops. */
fb_status fb_batch_collect(fb_batch* b, int capacity);
/* Copies up to cap examples of the last run (x [cap][FB_MLP_IN], y, mask); *count receives the number of accepted
 * births of the run (it can exceed the capacity). */
fb_status fb_batch_training_data(fb_batch* b, float* x, int* y, uint32_t* mask, int cap, int* count);

/* Learned cutpoint proposal, the second head of the learned proposal: once the tree's fused pass has run, a birth
 * draws its cutpoint index c from a small MLP over features of the node that include the weighted mean and spread of
 * the node's current residuals (exact fixed-point sums from that pass): FB_CUT_IN features -> FB_CUT_H -> FB_CUT_H ->
 * FB_CUT_E (ReLU between the hidden layers), then the logit of cut c is be[c] + emb[c] . e, a softmax over the cut
 * range of the birth's variable at the node, mixed with BART's uniform cut (src/bart_kernel.cpp:437) with probability
 * 1 - mix.  The pass keeps a histogram of the node's rows over the variable's codes, so the split sums of the drawn cut
 * are exact prefix sums.  The Metropolis-Hastings ratio carries the exact probability of the drawn cut and, for a
 * death, of the reverse birth's cut at the collapsed node, so the posterior is unchanged.  Features: depth / 8,
 * floor(log2(rows + 1)) / 16, clamp(mean / sigma, -4, 4) / 4, min(sd / sigma, 4) / 4, (U - L + 1) / numcut,
 * L / numcut, min(uses of the variable in the tree, 8) / 8, 0, then the variable one-hot (32).
 * Needs CTAs of at least 256 threads.  No counterpart in the reference. */
#define FB_CUT_IN 40
#define FB_CUT_H 64
#define FB_CUT_E 16
#define FB_CUT_BINS 255
typedef struct fb_cut_model {
  const uint16_t* w1; const float* b1;    /* [FB_CUT_H][FB_CUT_IN], [FB_CUT_H] */
  const uint16_t* w2; const float* b2;    /* [FB_CUT_H][FB_CUT_H], [FB_CUT_H] */
  const uint16_t* w3; const float* b3;    /* [FB_CUT_E][FB_CUT_H], [FB_CUT_E] */
  const uint16_t* emb; const float* be;   /* [FB_CUT_BINS][FB_CUT_E], [FB_CUT_BINS] */
  double mix;                             /* probability of the head's component, in (0, 1]; <= 0: BART's cut */
} fb_cut_model;
/* Uses `model` (copied to the device) for the batch's next runs; NULL or mix <= 0 restores BART's uniform cut. */
fb_status fb_batch_set_cut_proposal(fb_batch* b, const fb_cut_model* model);
/* The cut examples of the births fb_batch_training_data returns, in the same order: features x [cap][FB_CUT_IN], the
 * accepted cut c and the cut range [lo, hi] of its variable at the node. */
fb_status fb_batch_cut_training_data(fb_batch* b, float* x, int* c, int* lo, int* hi, int cap, int* count);

/* Training of the proposal MLP on the device (masked softmax cross-entropy, Adam, minibatches in a fixed seeded
 * order).  Weights start from `init` when non-NULL (else a seeded scaled-uniform initialisation); the trained model
 * is written to out_* (host arrays of the fb_proposal_model shapes, FP32 master weights rounded to BF16).
 * losses[e] receives the mean loss of epoch e when non-NULL. */
typedef struct fb_train_options {
  int epochs, batch;        /* passes over the examples, examples per step */
  double lr;                /* Adam step size */
  uint64_t seed;            /* initialisation and shuffling */
  int device;
} fb_train_options;
fb_status fb_train_proposal(const float* x, const int* y, const uint32_t* mask, int count,
                            const fb_train_options* opt, const fb_proposal_model* init, uint16_t* out_w1,
                            float* out_b1, uint16_t* out_w2, float* out_b2, uint16_t* out_w3, float* out_b3,
                            double* losses);
/* One forward and backward pass of the training kernels on `count` examples: mean loss and the gradients of the
 * loss with respect to the (BF16-valued) weights and biases, in the shapes of fb_proposal_model (FP32). */
fb_status fb_mlp_loss_grad(const fb_proposal_model* model, const float* x, const int* y, const uint32_t* mask,
                           int count, int device, double* loss, float* gw1, float* gb1, float* gw2, float* gb2,
                           float* gw3, float* gb3);

/* Training of the cut head on the device, as fb_train_proposal: softmax cross-entropy over each example's cut range
 * [lo, hi], Adam, minibatches in a fixed seeded order; the trained head goes to out_* (host arrays of the
 * fb_cut_model shapes). */
fb_status fb_train_cut_proposal(const float* x, const int* c, const int* lo, const int* hi, int count,
                                const fb_train_options* opt, const fb_cut_model* init, uint16_t* out_w1, float* out_b1,
                                uint16_t* out_w2, float* out_b2, uint16_t* out_w3, float* out_b3, uint16_t* out_emb,
                                float* out_be, double* losses);
/* One forward and backward pass of the cut head's training kernels: mean loss and FP32 gradients (fb_cut_model
 * shapes). */
fb_status fb_cut_loss_grad(const fb_cut_model* model, const float* x, const int* c, const int* lo, const int* hi,
                           int count, int device, double* loss, float* gw1, float* gb1, float* gw2, float* gb2,
                           float* gw3, float* gb3, float* gemb, float* gbe);

/* fbart_cpp (src/glue.cpp:10-62) with R's memory layouts: q is the n x p integer code matrix (column-major), yhat is
 * ndpost x n and varcount ndpost x p (column-major, as Rcpp::NumericMatrix / IntegerMatrix).  trees_text receives
 * BART's tree text when non-NULL; *text_len always receives its length (call once with trees_text = NULL to size the
 * buffer, which must hold text_len + 1 bytes).  Outputs may be NULL.  seed is the chain's Philox key (the R
 * generator of use_r_rng = 1 is not available on the device). */
fb_status fb_fbart(const int* q, int n, int p, const double* y, const double* wt, const int* ybin, const int* numcut,
                   const double* pgtab, int ntree, int nskip, int ndpost, double tau, double lambda, double nu,
                   double sigest, uint64_t seed, int probit, double offset, double* sigma, double* yhat_train_mean,
                   double* yhat_train, int* varcount, char* trees_text, size_t text_cap, size_t* text_len, int* moves);

/* BART's tree text of packed draws (src/glue.cpp:32-50): header "ndpost ntree p", then per draw and tree the node
 * count and pre-order "id v c theta" lines (root id 1, children 2id / 2id+1, 10 significant digits).  Writes at most
 * cap bytes (NUL-terminated when cap > 0) and returns the full length. */
size_t fb_trees_text(const uint64_t* trees, int ndpost, int ntree, int p, char* buf, size_t cap);
/* The same text assembled on the device (one thread per tree), byte for byte what fb_trees_text writes: trees are
 * host arrays copied to `device`.  *len receives the full length; buf (cap bytes, NUL-terminated when cap > 0) may be
 * NULL to size it.  Replaces the host loop of src/glue.cpp:29-57 (F1: device-side output assembly). */
fb_status fb_trees_text_gpu(const uint64_t* trees, int ndpost, int ntree, int p, int device, char* buf, size_t cap,
                            size_t* len);
/* Tree text of chain `chain` of a batch from its kept draws in device memory (after fb_batch_sync), as
 * fb_trees_text would write it from the downloaded trees; only the text crosses to the host. */
fb_status fb_batch_trees_text(fb_batch* b, int chain, char* buf, size_t cap, size_t* len);
/* varcount[dr][v] = number of internal nodes splitting on v in draw dr (src/glue.cpp:49). */
fb_status fb_varcount(const uint64_t* trees, int ndpost, int ntree, int p, int* varcount);

/* ------------------------------------------------------------------------------------------------ evaluator */

/* compile_trees_cpp (src/predict.cpp:12-45): parses tree text once into flat breadth-first node arrays (children
 * adjacent, cut = cutpoints[v][c]) and uploads them to the device.  cutpoints[v] has ncut[v] values. */
typedef struct fb_compiled fb_compiled;
fb_status fb_compile_trees(const char* text, size_t len, const double* const* cutpoints, const int* ncut, int ncol,
                           int device, fb_compiled** out);
fb_status fb_compiled_info(const fb_compiled* ct, int* ndpost, int* ntree, int* p, int* nnodes);
/* Which device evaluator a bulk call of ndraws draws on n rows runs (0 streaming FP64 compares, 1 tiled FP64
 * compares, 2 cutpoint codes, 3 cutpoint codes carrying each row's leaves across consecutive draws), and how many
 * trees have the structure of the previous draw's tree of the same index (the leaves the carrying evaluator reuses;
 * 0 when it is not applicable).  Every evaluator gives the same results. */
fb_status fb_predict_evaluator(const fb_compiled* ct, int n, int ndraws, int* evaluator, long long* shared_trees);
/* Copies the host arrays of compile_trees_cpp's result list (var, child, cut, theta [nnodes]; root [ndpost*ntree]). */
fb_status fb_compiled_arrays(const fb_compiled* ct, int* var, int* child, double* cut, double* theta, int* root);
void fb_compiled_free(fb_compiled* ct);

/* predict_draw_cpp (src/predict.cpp:49-73): f[i] = sum over trees, in tree order, of the leaf value reached by row i
 * (left when x < cut), plus mu; draw is 1-based.  cols[v] are host columns of n doubles.  Bit-identical to the
 * reference loop. */
fb_status fb_predict_draw(const fb_compiled* ct, const double* const* cols, int ncol, int n, int draw, double mu,
                          double* out);
/* Bulk form on device memory: x_dev is [ncol][ld] (column v at x_dev + v*ld), out_dev receives ndraws rows of n
 * values at out_dev + d*ldo, for draws draw0 .. draw0+ndraws-1 (1-based).  Enqueued on cuda_stream. */
fb_status fb_predict_draws_device(const fb_compiled* ct, const double* x_dev, int ncol, int n, int ld, int draw0,
                                  int ndraws, double mu, double* out_dev, int ldo, void* cuda_stream);
/* fb_predict_draw without any device allocation.  No counterpart in the reference (its predict_draw_cpp runs on the
 * host).  Same arguments, results and errors as fb_predict_draw, which allocates and frees device buffers for the
 * columns and the result on every call.  This form stages them in a fixed 8 MiB device array instead; every device
 * that loads the library holds that array until the process exits.  It is meant for callers that cannot call
 * cudaMalloc: a process whose device memory is already held by another framework's caching allocator or by a fixed
 * budget, where a new allocation can fail, and latency-sensitive loops, where cudaFree synchronizes the whole device
 * and stalls every other stream.
 * Limits: n * (ncol + 1) <= 1048576 doubles, and device ordinals 0..63; beyond either the call fails with
 * FB_ERR_LIMIT (split the rows over several calls).
 * The first call on a device does the set-up: it looks up the array's device address with that device current and
 * keeps it for the life of the process, so the process must not reset that device (cudaDeviceReset) afterwards.
 * Make that first call before any stream capture.  Nothing in the array needs to start at zero, because each call
 * copies in all its columns and the kernel writes every result.  All calls on a device share the one array, so calls
 * that overlap on the GPU (from several host threads) race; serialize them. */
fb_status fb_predict_draw_static(const fb_compiled* ct, const double* const* cols, int ncol, int n, int draw,
                                 double mu, double* out);

/* The probit latent redraw of fpbart (src/bart_kernel.cpp:280-292, 543-547) on its own, over device arrays:
 * z_dev[i] = N(fit_dev[i], 1) truncated to z > -offset when ybin_dev[i] is 1 and to z < -offset when it is 0, the
 * value the sampler draws for row i of the chain with this seed at the end of 0-based sweep `sweep` (-1: the
 * initial draw, whose fit is 0).  fit excludes the offset, as the sampler's fit does.  Draws that hit the 64-try cap
 * are counted into *capped_dev when it is not NULL.  Enqueued on cuda_stream; rows up to 2^32. */
fb_status fb_probit_latent_device(const double* fit_dev, const int* ybin_dev, long long n, double offset,
                                  uint64_t seed, int sweep, double* z_dev, int* capped_dev, void* cuda_stream);
/* sigest of the preprocessing (R/fwbart.R:22): the residual standard error of the least-squares fit of y on an
 * intercept and the columns (summary(lm(yc ~ X))$sigma), from FP64 Gram sums computed on the device; aliased columns
 * are dropped as lm drops them (*rank = the columns kept, intercept included).  When ncol >= n it is sd(y), as in
 * the reference (*rank = 0).  cols[v] are host columns of n doubles, at most 32. */
fb_status fb_sigma_estimate(const double* const* cols, int ncol, int n, const double* y, int device, double* sigest,
                            int* rank);
/* Cutpoint codes on the device, the findInterval step of R/fwbart.R:19 and R/fpbart.R:13: q[v][i] = number of
 * cutpoints of predictor v that are <= cols[v][i] (so x < cutpoints[v][c] <=> q <= c; NaN gives 0).  cutpoints[v]
 * has ncut[v] (0..255) strictly increasing values; q is [ncol][n] bytes (host). */
fb_status fb_cut_codes(const double* const* cols, int ncol, int n, const double* const* cutpoints, const int* ncut,
                       int device, uint8_t* q);

/* ------------------------------------------------------------------------------------------------ diagnostics */

/* One fused per-tree data pass on explicit state (the pass of src/bart_kernel.cpp:131-213), run by the same device
 * code as the sampler.  Host buffers of n rows: leaf_prev and r are updated in place; out receives 70 int64 values:
 * S1 (sum of fx(w*R)) per leaf slot [64], the birth split sums sL0 sL1 sR0 sR1, and the counts nL nR. */
typedef struct fb_pass_state {
  int n, apply, stats, fx_shift, threads;
  int pmode, pnx, pc, pL, pR, pl, pr;   /* previous tree's move */
  int cmode, cnx, cc;                   /* current tree's proposal */
  uint64_t leafmask;                    /* leaf slots of the current tree */
  uint8_t* leaf_prev; const uint8_t* leaf_cur; const uint8_t* qprev; const uint8_t* qcur;
  float* r; const float* w;
  const float* tho; const float* thn; const float* thc;   /* [64] each */
} fb_pass_state;
fb_status fb_debug_tree_pass(const fb_pass_state* s, int64_t* out);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
