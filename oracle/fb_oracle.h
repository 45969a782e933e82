/*
 * fb_oracle.h -- CPU oracle for fastbart_b200.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/, __graft_entry__.smoke() and the cpu_baseline leg
 * of bench.py load it to compute the expected answer on the CPU.  The product (fastbart_b200/, libfastbart_b200.so)
 * never links, loads or calls it.
 *
 * It restates, in plain C, the reference's algorithms for the hot path:
 *
 *   - the sampler of src/bart_kernel.cpp:304-580 (bart_fit_cpu), in two arithmetic modes:
 *       ORC_MODE_REF  the reference's own arithmetic: xoshiro128** RNG (bart_kernel.cpp:53-83), FP64 row sums in
 *                     KL = 16 lanes summed lane by lane (bart_kernel.cpp:131-213).  Bit-exact to bart_fit_cpu built
 *                     with -DFAST_CPU and run with bart_set_rng(NULL, ...) (the internal generator), which pins this
 *                     restatement to the reference itself (oracle/_ref).
 *       ORC_MODE_DEV  the arithmetic of the B200 kernels: counter-based Philox4x32-10 RNG, FP32 row residuals, exact
 *                     int64 fixed-point sums, FP64 control math with this project's own log/exp (atanh-series log,
 *                     Taylor exp with Cody-Waite reduction), polar-method normals, FP64 tree-order refresh of
 *                     y - sum(trees) once per sweep.  The CUDA sampler must reproduce this mode bit for bit.
 *   - the per-tree fused data pass (bart_kernel.cpp:131-213 semantics, gpu/bart_batch.cu:184-227 fixed-point
 *     semantics) on explicit state, in DEV arithmetic (orc_pass_dev);
 *   - compile_trees_cpp / predict_draw_cpp of src/predict.cpp:11-73 without Rcpp;
 *   - the BART tree-text writer, varcount and yhat.train re-sum of src/glue.cpp:29-57.
 */
#ifndef FB_ORACLE_H
#define FB_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#define ORC_NODES 64      /* node slots per tree (bart_kernel.h:23) */
#define ORC_MAXDEPTH 24   /* bart_kernel.h:33 */
#define ORC_PMAX 32       /* bart_kernel.h:20 */
#define ORC_MMAX 200      /* bart_kernel.h:21 */
#define ORC_KL 16         /* lanes of the reference CPU build (bart_kernel.h:26) */

enum { ORC_MODE_REF = 0, ORC_MODE_DEV = 1 };

/* Philox counter tags (word 3 of the counter) used by the DEV arithmetic. */
enum { ORC_TAG_PROP = 1, ORC_TAG_MH = 2, ORC_TAG_MU = 3, ORC_TAG_SIG_N = 4, ORC_TAG_SIG_U = 5, ORC_TAG_Z_N = 6,
       ORC_TAG_Z_E = 7, ORC_TAG_PROP2 = 8, ORC_TAG_PROP3 = 9 };
#define ORC_INIT_SWEEP 0xFFFFFFFFu

/* Learned split-variable proposal (DEV mode): an MLP of ORC_MLP_IN node features -> ORC_MLP_H -> ORC_MLP_H ->
 * ORC_MLP_OUT logits (ReLU between), BF16 weights, FP32 arithmetic without fused multiply-add.  A birth draws its
 * variable from the model's masked softmax with probability mix, else uniformly as BART does; the MH ratio carries
 * the exact proposal probabilities (birth and reverse death), so the chain targets the same posterior. */
#define ORC_MLP_IN 98
#define ORC_MLP_H 64
#define ORC_MLP_OUT 32
typedef struct {
  const uint16_t* w1; const float* b1;   /* [H][IN] bf16, [H] */
  const uint16_t* w2; const float* b2;   /* [H][H], [H] */
  const uint16_t* w3; const float* b3;   /* [OUT][H], [OUT] */
  double mix;                            /* probability of the model component (0: plain proposal) */
} orc_model;

/* Learned cutpoint proposal (DEV mode), drawn after the tree's fused pass: node features including the residual
 * mean and spread of the node's rows (ORC_CUT_IN) -> ORC_CUT_H -> ORC_CUT_H -> ORC_CUT_E (ReLU between the hidden
 * layers), then one logit per cutpoint index c, be[c] + emb[c] . e; BF16 weights, FP32 sums without fused
 * multiply-add.  A birth draws its cutpoint from the softmax over the variable's cut range at the node with probability
 * mix, else uniformly as BART does; the MH ratio carries the exact probabilities of the birth's cut and of the
 * reverse birth's cut of a death.  Features (orc_cut_features): x[0] depth / 8, x[1] floor(log2(cnt + 1)) / 16,
 * x[2] clamp(mean / sigma, -4, 4) / 4, x[3] min(sd / sigma, 4) / 4 (weighted residual mean and sd of the node's rows),
 * x[4] (U - L + 1) / numcut, x[5] L / numcut, x[6] min(uses of v, 8) / 8, x[7] 0, x[8 + k] = (k == v). */
#define ORC_CUT_IN 40
#define ORC_CUT_H 64
#define ORC_CUT_E 16
#define ORC_CUT_BINS 255
typedef struct {
  const uint16_t* w1; const float* b1;   /* [H][IN], [H] */
  const uint16_t* w2; const float* b2;   /* [H][H], [H] */
  const uint16_t* w3; const float* b3;   /* [E][H], [E] */
  const uint16_t* emb; const float* be;  /* [BINS][E], [BINS] */
  double mix;
} orc_cut_model;

typedef struct {
  int n, p, m, nskip, ndpost;
  const uint8_t* q;       /* [p][n] cutpoint codes: x < xi[v][c]  <=>  q <= c */
  const double* y;        /* [n] centred y (wbart); unused when probit */
  const double* wt;       /* [n] 1/w^2 (wbart); NULL means all ones */
  const int* ybin;        /* [n] 0/1 outcomes (probit), else NULL */
  const int* numcut;      /* [p] */
  const double* pgtab;    /* [64] base/(1+d)^power */
  double tau, lambda, nu, sigest, offset;
  uint64_t seed;          /* REF: low 32 bits are bart_fit_cpu's seed; DEV: the Philox key */
  int probit;
  int fx_shift;           /* DEV: w and w*r are summed as llrint(x * 2^fx_shift) */
  int rss_shift;          /* DEV: w*e^2 is summed as llrint(x * 2^rss_shift) */
  const orc_model* model; /* DEV: learned proposal, or NULL */
  const orc_cut_model* cut; /* DEV: learned cutpoint proposal, or NULL */
} orc_chain;

typedef struct {
  double* sigma;          /* [nskip+ndpost] (REF: float-rounded like sigma_out) */
  double* fmean;          /* [n] posterior mean of f (REF: float TM/ndpost like trmean_out) */
  double* yhat;           /* [ndpost][n] FP64 tree-order sum of each kept draw (glue.cpp:52-56); may be NULL */
  uint64_t* trees;        /* [ndpost][m][64] packed nodes (bart_kernel.cpp:559-571); may be NULL */
  int moves[3];           /* births, deaths, node-cap hits */
  int rtnorm_caps;        /* DEV: truncated-normal draws that hit their iteration cap */
  /* DEV: accepted births as training examples (features at the node before the birth, split variable, mask of the
   * variables with a non-empty cut range there), in step order; train_cap 0 disables */
  float* train_x;         /* [train_cap][ORC_MLP_IN] */
  int* train_y;
  uint32_t* train_mask;
  int train_cap, train_count;
  /* DEV: the cutpoint examples of the same accepted births: features, cut, cut range [lo, hi] (when train_cx set) */
  float* train_cx;        /* [train_cap][ORC_CUT_IN] */
  int* train_c;
  int* train_lo;
  int* train_hi;
} orc_out;

/* Whole-chain sampler.  Returns 0 on success, <0 on a bad shape. */
int orc_fit(const orc_chain* c, int mode, orc_out* o);

/* ---------------------------------------------------------------- per-tree pass on explicit state (DEV arithmetic) */
typedef struct { int mode, nx, v, c, L, R, l, r; } orc_upd;   /* previous tree's accepted move (0 none, 1 birth, 2 death) */
typedef struct { int mode, nx, v, c; } orc_prop;              /* current tree's proposal (0 none, 1 birth, 2 death) */
typedef struct {
  int64_t S0[ORC_NODES], S1[ORC_NODES];                       /* per leaf slot: sum fx(w), sum fx(w*R) */
  int64_t sL0, sL1, sR0, sR1;                                 /* birth split sums */
  int nL, nR;
} orc_stats;

void orc_pass_dev(int n, uint8_t* leaf_prev, const uint8_t* leaf_cur, float* r, const float* w,
                  const uint8_t* qprev, const uint8_t* qcur, const orc_upd* pu, const float* tho, const float* thn,
                  int apply, const orc_prop* cp, const float* thc, int fx_shift, orc_stats* st);

/* ---------------------------------------------------------------- DEV arithmetic primitives (exported for tests) */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* MLP forward on one feature vector: logits [ORC_MLP_OUT]. */
void orc_mlp_logits(const orc_model* M, const float* x, float* z);
/* Masked softmax of the logits in FP64 with orc_exp; q[v] = 0 for masked v. */
void orc_mlp_probs(const float* z, uint32_t valid, double* q);
/* Mean masked cross-entropy over a batch and its gradients with respect to the (BF16-valued) weights and biases,
 * computed in FP64 from the same BF16 weights (the checker of the device training kernels). */
double orc_mlp_loss_grad(const orc_model* M, const float* X, const int* y, const uint32_t* mask, int B,
                         double* gw1, double* gb1, double* gw2, double* gb2, double* gw3, double* gb3);
/* Cutpoint-proposal features, logits over c in [L, U] (z[c]; other entries untouched) and the masked softmax in the
 * device's summation order (blocks of 8 consecutive c from L, each summed in order, block sums in order); ex[c]
 * receives exp(z[c] - max), the return value is the sum. */
void orc_cut_features(int depth, int cnt, int64_t S0, int64_t S1, int64_t Q, int fx_shift, int rss_shift,
                      double sigma, int L, int U, int nc, int uses, int v, float* x);
void orc_cut_logits(const orc_cut_model* M, const float* x, int L, int U, float* z);
double orc_cut_softmax(const float* z, int L, int U, double* ex);
/* Mean cross-entropy of the cut head over a batch (softmax over [lo, hi] of each example) and its gradients. */
double orc_cut_loss_grad(const orc_cut_model* M, const float* X, const int* c, const int* lo, const int* hi, int B,
                         double* gw1, double* gb1, double* gw2, double* gb2, double* gw3, double* gb3, double* gemb,
                         double* gbe);
double orc_log(double x);
double orc_exp(double x);
double orc_normal(uint64_t seed, uint32_t c0base, uint32_t c1, uint32_t c2, uint32_t tag);
double orc_gamma(uint64_t seed, uint32_t it, double a);
double orc_rtnorm(uint64_t seed, uint32_t row, uint32_t it, double mean, double tau, int* capped);
int orc_probit_latent(uint64_t seed, uint32_t it, double offset, const double* fit, const int* ybin, long long n,
                      double* z);

/* ---------------------------------------------------------------- evaluator (src/predict.cpp) */
typedef struct {
  int ndpost, ntree, p, nnodes;
  int* var; int* child; double* cut; double* theta; int* root;
} orc_ct;
int orc_compile_trees(const char* text, const double* const* xi, const int* ncut, int ncol, orc_ct* out);
void orc_ct_free(orc_ct* ct);
int orc_predict_draw(const orc_ct* ct, const double* const* cols, int ncol, int n, int draw1, double mu, double* out);

/* ---------------------------------------------------------------- output assembly (src/glue.cpp:29-57) */
/* Writes BART tree text into buf (if non-NULL, up to cap bytes) and returns the full length (excluding NUL). */
size_t orc_trees_text(const uint64_t* trees, int ndpost, int m, int p, char* buf, size_t cap);
void orc_varcount(const uint64_t* trees, int ndpost, int m, int p, int* varcount /* [ndpost][p] */);
void orc_yhat_from_trees(const uint64_t* trees, int ndpost, int m, const uint8_t* q, int n, double* yhat /* [ndpost][n] */);

#endif
