// fb_internal.h -- layouts shared by the host code (host.cpp) and the CUDA kernels (sampler.cu, predict.cu).
#pragma once
#include <cstdint>

namespace fb {

constexpr int NODES = 64;      // node slots per tree (src/bart_kernel.h:23)
constexpr int PMAX = 32;       // predictors (src/bart_kernel.h:20)
constexpr int MMAX = 200;      // trees (src/bart_kernel.h:21)
constexpr int NMAX = 65536;    // rows per chain (src/bart_kernel.h:16)
constexpr int MAXDEPTH = 24;   // src/bart_kernel.h:33
constexpr int NB_MAX = 8;      // per-thread register bins of the fused pass; leaves beyond use shared atomics
constexpr int MAX_THREADS = 512;
constexpr int LEAF_STAT_WORDS = 96;   // per tree, 8-byte words: leaf sums of fx(w) [64], then row counts (int) [64]
constexpr int MIN_THREADS = 64;
// learned proposal MLP: node features -> hidden -> hidden -> one logit per predictor
constexpr int MLP_IN = 98;
constexpr int MLP_H = 64;
constexpr int MLP_OUT = 32;   // warp 0 is the control warp; at least one row warp

// Topology of one tree: 64 node slots (leaf values are kept apart, in th[]).  464 bytes, 16-byte multiple.
struct DTree {
  uint8_t l[NODES], r[NODES], par[NODES], v[NODES], c[NODES], d[NODES], ngv[NODES];
  unsigned long long used, leaf;
};
static_assert(sizeof(DTree) == 464, "DTree layout");

// Per-chain descriptor (device resident, read-only while sampling).  Offsets are in elements of the batch arrays.
struct DChain {
  int n, p, m, n_pad;
  int probit, fx_shift, rss_shift, root_ngv;
  int nskip, ndpost, pad0, pad1;
  int numcut[PMAX];
  double tau, lambda, nu, sigest, offset;
  double pg[NODES];
  unsigned long long seed;
  long long off_row;    // y, w, ybin, tm, rsave: [n_pad]
  long long off_q;      // codes [p][n_pad]
  long long off_leaf;   // leaf ids [m][n_pad]
  long long off_tree;   // trees, th [m][64], s0 [m][LEAF_STAT_WORDS]
  long long off_sigma;  // [nskip + ndpost]
  long long off_yhat;   // [ndpost][n]
  long long off_tout;   // [ndpost][m][64]
};

// Mutable per-chain state kept between launches.
struct DState {
  double sigma;
  int births, deaths, caps, rtcaps;
  int it_done, status, pad0, pad1;
};

// Device buffers of one batch.
struct DBufs {
  const DChain* chains;
  DState* states;
  const uint8_t* q;
  const double* yin;
  double* ywork;
  const float* win;
  const int8_t* ybin;
  float* rsave;
  float* wsave;
  uint8_t* leaf;
  DTree* trees;
  long long* s0;                   // per tree: leaf sums of fx(w) [64] (int64), then leaf row counts [64] (int32)
  float* th;
  double* tm;
  double* sigma_out;
  double* yhat_out;
  unsigned long long* trees_out;
  const int* order;
  int* queue;
  int nchains;
  int m_max;
  int n_pad_max;                   // rows of one CTA's slice (shared-memory capacity)
  int rows_in_smem;                // 1: residuals and weights in shared memory, 2: residuals only, 0: neither
  int cluster;                     // CTAs per chain (a thread-block cluster when > 1)
  // learned split-variable proposal (null mvar: BART's uniform proposal): the model's weight image (see MIMG_*),
  // staged in shared memory behind the sampler's own layout when model_smem is set, else read from global memory
  const uint32_t* mimg;
  int model_smem;
  double mix;                              // probability of the model component, in (0, 1]
  int* mvar; double* mcorr;                // [trees] the model's choices of the current sweep: variable, correction
  // accepted births as training examples (train_cap 0: off)
  float* feat;                             // [trees][MLP_IN] features of each tree's birth proposal
  unsigned* feat_valid;                    // [trees] valid-variable mask of that proposal
  float* train_x;                          // [train_cap][MLP_IN]
  int* train_y;
  unsigned* train_mask;
  int* train_count;
  int train_cap;
  // learned cutpoint proposal (null cimg: BART's uniform cut): the cut head's weight image (see CIMG_*), staged in
  // shared memory when cut_smem is set, else read from global memory; a birth's cut is then drawn after the pass
  const uint32_t* cimg;
  int cut_smem;
  double cmix;                             // probability of the cut head's component, in (0, 1]
  // the cut examples of the collected births (train_cx null: none): per tree, the features and (cut, lo, hi) of its
  // accepted birth of the current step, copied to the example arrays with the variable example
  float* cfeat;                            // [trees][CUT_IN]
  int* cinfo;                              // [trees][3]
  float* train_cx;                         // [train_cap][CUT_IN]
  int* train_c;
  int* train_lo;
  int* train_hi;
};

// learned cutpoint proposal: CUT_IN node features (with the node's residual mean and spread) -> CUT_H -> CUT_H ->
// CUT_E, then one logit per cutpoint index c < CUT_BINS: be[c] + emb[c] . e
constexpr int CUT_IN = 40, CUT_H = 64, CUT_E = 16, CUT_BINS = 255;
// the sampler's image of a cut head (32-bit words): BF16 pairs row by row, rows padded to an odd word count (distinct
// banks for the threads reading one row each), then the FP32 biases b1 [H], b2 [H], b3 [E], be [BINS]
constexpr int CIMG_W1S = CUT_IN / 2 + 1, CIMG_W2S = CUT_H / 2 + 1, CIMG_ES = CUT_E / 2 + 1;
constexpr int CIMG_W2 = CUT_H * CIMG_W1S, CIMG_W3 = CIMG_W2 + CUT_H * CIMG_W2S, CIMG_EMB = CIMG_W3 + CUT_E * CIMG_W2S;
constexpr int CIMG_B = CIMG_EMB + CUT_BINS * CIMG_ES;
constexpr int CIMG_WORDS = (CIMG_B + 2 * CUT_H + CUT_E + CUT_BINS + 3) / 4 * 4;
constexpr int CUT_NPARAM = CUT_H * CUT_IN + CUT_H + CUT_H * CUT_H + CUT_H + CUT_E * CUT_H + CUT_E + CUT_BINS * CUT_E +
                           CUT_BINS;

// cut: the layout of a launch with the learned cut proposal (its per-tree ratios, histograms and head)
size_t sampler_smem_bytes(int threads, int m_max, int n_pad_max, int rows_in_smem, int cluster, int cut = 0);
// Tree text (without its header) of ntrees consecutive device trees: *total receives its length; with d_out
// non-null, *d_out is allocated (cudaMalloc, caller frees) and receives the text.  0 on success.
int trees_text_device(const uint64_t* d_trees, long long ntrees, char** d_out, unsigned long long* total,
                      void* stream);
// whether the sampler stages the proposal model's weights in its pass bins (no extra shared memory needed)
bool sampler_bins_hold_model(int threads);
// groups of 4 rows per row thread held in registers (1, 2, 3, 4, 6, 8), or 0 when the rows stream from L2 in the pass
int sampler_gmax(int threads, int n_pad_max);
int launch_sampler(const DBufs& b, int it0, int it1, int threads, int grid, size_t smem, int gmax, int cluster,
                   void* stream);
// CTAs that can be resident at once (a multiple of cluster), 0 when none
int sampler_max_grid(int threads, size_t smem, int device, int gmax, int cluster);

// Per-tree pass on explicit state (diagnostics / parity tests): one CTA.
struct DPassArgs {
  int n, n_pad, apply, stats;
  int pmode, pnx, pc, pL, pR, pl, pr;
  int cmode, cnx, cc;
  int fx_shift, rows_in_smem;
  unsigned long long leafmask;   // leaves of the current tree
  uint8_t* leaf_prev;            // [n_pad] in/out
  const uint8_t* leaf_cur;       // [n_pad]
  const uint8_t* qprev;          // [n_pad]
  const uint8_t* qcur;           // [n_pad]
  float* r;                      // [n_pad] in/out
  const float* w;                // [n_pad]
  float* wscratch;               // [n_pad] scaled weights when rows stay in global memory
  const float* tho;              // [64]
  const float* thn;              // [64]
  const float* thc;              // [64]
  long long* out;                // [64 + 4 + 2]: S1 per slot, sL0 sL1 sR0 sR1, nL nR
};
int launch_debug_pass(DPassArgs a, int threads, void* stream);

// Evaluator (predict_draw) on device.
// One node of the tiled evaluator's packed layout (16 bytes, one load per step).  Internal node: v = cut, children at
// child and child + 1, split variable var.  Leaf: v = leaf value, child = its own index, var = p (a column that is
// -inf in the evaluator's tile, so the step x >= v never leaves the leaf).
struct PNode { double v; int child; int var; };
static_assert(sizeof(PNode) == 16, "PNode layout");
struct DForest {
  const int* var; const int* child; const double* cut; const double* theta; const int* root;
  const PNode* nodes;
  const uint8_t* gdepth;   // [ndpost][ceil(ntree / 4)] deepest leaf of each group of 4 consecutive trees
  // code-compare layout (null when not applicable): nodes packed in 32 bits, relative to their draw's first node
  // (child | var << 16 | c << 24; leaves point to themselves with c = 255), and the cutpoints of every predictor
  // (cuts[cutoff[v] .. cutoff[v + 1]), strictly increasing)
  const uint32_t* n32; const double* cuts; const int* cutoff;
  // reuse across consecutive draws (code-compare layout): bit t of same[d][.] says tree t of draw d has the structure
  // of tree t of draw d - 1 (node count, splits and children relative to its root; leaf values may differ), so a row
  // reaches the same leaf offset in both; tdep[d][t] is the tree's deepest leaf; nsame counts the set bits
  const uint32_t* same; const uint8_t* tdep; long long nsame;
  int maxnd;               // most nodes of one draw
  int ntree, ndpost, p, nnodes;
};
// Learned-proposal training (mlp.cu).  Flat FP32 parameter vector: w1 [H][IN], b1 [H], w2 [H][H], b2 [H],
// w3 [OUT][H], b3 [OUT]; the forward pass reads BF16 copies of the weights.
constexpr int MLP_NPARAM = MLP_H * MLP_IN + MLP_H + MLP_H * MLP_H + MLP_H + MLP_OUT * MLP_H + MLP_OUT;
// The sampler's image of a proposal model (32-bit words): BF16 weight pairs row by row, rows padded to an odd
// number of words so that the lanes of a warp reading one row each hit distinct shared-memory banks, then the
// FP32 biases.  W1 rows [MLP_H][MIMG_W1S], W2 rows [MLP_H][MIMG_W2S], W3 rows [MLP_OUT][MIMG_W2S], b1, b2, b3.
constexpr int MIMG_W1S = MLP_IN / 2, MIMG_W2S = MLP_H / 2 + 1;
constexpr int MIMG_W2 = MLP_H * MIMG_W1S, MIMG_W3 = MIMG_W2 + MLP_H * MIMG_W2S, MIMG_B = MIMG_W3 + MLP_OUT * MIMG_W2S;
constexpr int MIMG_WORDS = (MIMG_B + 2 * MLP_H + MLP_OUT + 3) / 4 * 4;   // a multiple of 16 bytes
struct MlpParams {
  uint16_t* w1; uint16_t* w2; uint16_t* w3;   // BF16 weights (device)
  const float* b1; const float* b2; const float* b3;
};
size_t mlp_grad_smem();
// summed gradients (and summed loss) of examples idx[0..B) (or 0..B when idx is null), added into grad / *loss
int mlp_grad_launch(const MlpParams& P, const float* X, const int* Y, const unsigned* M, const int* idx, int B,
                    float* grad, float* loss, void* stream);
// Adam step `step` (1-based) with gradient grad * inv_batch; refreshes the BF16 weights of P
int mlp_adam_launch(float* p, float* m1, float* m2, const float* g, float inv_batch, float lr, int step,
                    const MlpParams& P, void* stream);

// Training of the cut head (mlp.cu); flat FP32 parameters in the order of CUT_NPARAM (see mlp.cu)
struct CutParams {
  uint16_t* w1; uint16_t* w2; uint16_t* w3; uint16_t* emb;   // BF16 weights (device)
  const float* b1; const float* b2; const float* b3; const float* be;
};
int cut_grad_launch(const CutParams& P, const float* X, const int* Yc, const int* LO, const int* HI, const int* idx,
                    int B, float* grad, float* loss, void* stream);
int cut_adam_launch(float* p, float* m1, float* m2, const float* g, float inv_batch, float lr, int step,
                    const CutParams& P, void* stream);

// cutpoint codes of p columns of n values (x [p][n], cutpoints cuts[cutoff[v] .. cutoff[v + 1]), q [p][n])
int launch_cut_codes(const double* x, int n, int p, const double* cuts, const int* cutoff, uint8_t* q, void* stream);
// fixed device scratch of the allocation-free predict call: n * (ncol + 1) doubles at most (8 MiB per device)
constexpr size_t PREDICT_SCRATCH_DOUBLES = size_t(1) << 20;
// 0: *ptr = the scratch's address on `device` (the current device); -1: CUDA error; -2: device ordinal not tracked
int predict_scratch_address(int device, double** ptr);
// the probit latent redraw on its own (latent.cu): z[i] for fits fit[i] and outcomes ybin[i] at `sweep`
int launch_probit_latent(const double* fit, const int* ybin, long long n, double offset, uint64_t seed, uint32_t sweep,
                         double* z, int* capped, void* stream);
// Gram sums of [1, x_1 .. x_p, y] for the least-squares sigest (latent.cu): part[block][pair], x column-major [p][n]
int launch_gram(const double* x, int n, int p, const double* y, int nblocks, int chunk, double* part, void* stream);
// evaluator launch_predict uses for f: 0 streaming, 1 tiled, 2 code-compare, 3 code-compare carrying leaves across draws
int predict_evaluator(const DForest& f, int n, int ndraws);
int launch_predict(const DForest& f, const double* x, int n, int ld, int draw0, int ndraws, double mu, double* out,
                   int ldo, void* stream);

}  // namespace fb
