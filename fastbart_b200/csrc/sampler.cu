// sampler.cu -- the restructured BART backfitting sampler (fwbart / fpbart) as one persistent sm_100a kernel.
//
// Reference algorithm: src/bart_kernel.cpp:304-580 (bart_fit_cpu); the one-fit-per-block CUDA prototype
// gpu/bart_batch.cu:101-298 is the design this kernel replaces.
//
// Layout and execution
//   * One CTA runs one chain at a time; CTAs pull chains from a device work queue (atomic counter over a host-sorted
//     order, largest n*ntree first), so chains of uneven n, p and ntree share one launch.
//   * Warp 0 is the control warp; warps 1.. stream the rows.  Rows live in shared memory (FP32 residual r and the
//     weight pre-scaled to fixed point, ws = w * 2^S, one float4 per group of 4 rows); leaf ids [ntree][n] and
//     cutpoint codes [p][n] stream from L2 as one 32-bit word per group.  Each row thread owns fixed groups and keeps
//     their leaf ids and codes in registers: the words it needs for the next tree are loaded at the end of the
//     current pass, so the loads overlap the control phase instead of delaying the next pass.
//   * Per tree step j, two phases separated by barriers:
//     A. the row warps make ONE fused pass that applies tree j-1's accepted move (leaf ids updated four at a time
//        with byte-SIMD compares, r -= delta from a 64-entry table) and accumulates tree j's per-leaf sum of
//        fx(w*R) in per-thread shared-memory bins (one column of the bin matrix per row thread; leaves beyond the
//        8th by shared atomics) plus the left child's sums and count of a birth proposal, all exact int64 (order
//        independent, hence bit-exact).  After a barrier every warp forms one CTA total from the per-thread
//        partials (coalesced shared loads, then a warp sum by redux.sync on three 21-bit limbs).
//        Meanwhile the control warp writes tree j-1's topology update back to global memory and fetches tree j+1
//        (cp.async).
//     B. 64 threads, one per node slot, decide Metropolis-Hastings (warps 0 and 1 each evaluate the three log
//        marginal likelihoods on lanes 0..2) and draw the new leaf values in FP64; they publish the apply deltas of
//        the move and tree j+1's leaf table for the next pass.
//   * Per sweep: all proposals are drawn at the start, one thread per tree (a proposal depends only on its own tree
//     and on counter-based random numbers), together with the leaf-mu normals of every slot that can be a leaf of
//     that tree after its move, and the goodvar counts of new leaves; at the end one pass refreshes every row's fit as an FP64 tree-order sum
//     of leaf values (which is also the draw's yhat.train), redraws the probit latent z, and sums rss for sigma.
//   * sum(fx(w)) and the row count of every leaf are kept exactly with each tree (root: all rows; birth: the split
//     sums; death: the two children), so the pass reduces only sum(fx(w * R)) per leaf, and a birth's right child
//     follows from its node's totals minus the left child's.
//   * Random numbers: Philox4x32-10 keyed by the chain seed, counter = (draw index, tree or row, sweep, purpose).
//   * All control arithmetic is IEEE FP64 through fb_math.cuh; the file is compiled with -fmad=false.  The oracle's
//     DEV mode (oracle/fb_oracle.c) restates exactly this arithmetic on the CPU.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "fb_internal.h"
#include "fb_math.cuh"

namespace fb {

constexpr int NBS = NB_MAX;   // per-thread shared-memory bins (compact leaf index < NBS); beyond: shared atomics
constexpr int TOT = 16;       // CTA totals per tree: [0, NBS) leaf sums, NBS.. sL0 sL1 nL
constexpr int NSPLIT = 4;     // split partials per row thread: sum fx(w), sum fx(w*R), count of the left child, and
                              // sum fx2(w*R^2) of the rows of the learned cut proposal's node
constexpr int LST = LEAF_STAT_WORDS;
constexpr int ZMAX = 16;      // leaf-mu normals drawn ahead per tree (candidate slots beyond are drawn in the step)
constexpr int ZMAX_CUT = 8;   // the same in cut layouts (smaller; the normals are the same counter-based draws)
constexpr int MODE_PLAIN = 0, MODE_MODEL = 1, MODE_COLLECT = 2;   // sampler kernel variants (see sampler_kernel)
constexpr int BIN_ROWS = NBS + 3;       // rows of the bin matrix: leaf rows, split rows (sum fx(w), fx(w R), count)
constexpr int BIN_ROWS_CUT = NBS + 4;   // with the learned cut proposal: and sum fx2(w R^2) of its node's rows
// the pass bins of a CTA of `threads` can hold the proposal model's weight image at sweep start
__host__ __device__ inline bool bins_hold_model(int threads) {
  return (size_t)BIN_ROWS * (size_t)(threads - 32) * 8 >= (size_t)MIMG_WORDS * 4;
}
// the split rows of the bins hold the cut proposal's code histogram (cut launches accumulate no split sums)
__host__ __device__ inline bool bins_hold_hist(int threads) { return (size_t)3 * (threads - 32) * 8 >= 256 * 20; }

struct Prop {                 // proposal of one tree for the current sweep
  double logpr, lu;
  unsigned long long cand;    // slots that can be leaves after the move (normals drawn ahead, in slot order)
  uint8_t mode, nx, v, c, l, r, dnx, flags;   // dnx: depth of node nx; flags bit 0: the cut is drawn after the pass
};
constexpr int PROP_DEFER = 1;
// What the learned cut proposal needs of tree j's proposal beyond Prop (launches with a cut head, and collecting
// launches): for a birth, BART's ratio (times the variable proposal's factor) for a cut at the inside of the range or
// at its ends, pr4[(c == L) + 2 (c == U)]; for a death, pr4[0] is the ratio; L, U: the cut range of the variable at
// the node; uses: internal nodes splitting on the variable (other than the node itself).
struct PropX {
  double pr4[4];
  uint8_t L, U, uses, pad[5];
};
struct Masks { unsigned long long used, leaf; };
struct Ctl {                  // CTA-shared control state
  int pmode, pnx, pv, pc, pL, pR, pl, pr;   // the last decided move (tree j during pass j+1)
  float DL, DR;                             // apply deltas of a birth's left / right rows
  long long sL0, sR0;                       // leaf weight sums of a birth's children (death: sL0 of the merged node)
  int nL, nR;                               // and their row counts (death: nL of the merged node)
  int pd;                                   // depth of the decided move's node
  unsigned long long used, leaf;            // node masks of the tree after the move
  int nleaf[2];                             // leaves of the tree whose table is in buffer 0 / 1
  int births, deaths, caps, rtcaps;
  int chain;
  int accept;                               // MH decision of the current tree (handed from warp 2 to warps 0-1)
  int err;                                  // a bounded wait gave up (reported in the chain's state)
  unsigned fetches[2];                      // leaf-statistics copies issued into buffer 0 / 1 (mbarrier phases)
  double sigma;
};

__device__ __forceinline__ long long warp_sum64(long long x) {
  // exact int64 warp sum with three 32-bit redux.sync: x = a*2^42 + b*2^21 + c, b and c in [0, 2^21)
  const unsigned c = (unsigned)(x & 0x1FFFFF), b = (unsigned)((x >> 21) & 0x1FFFFF);
  const int a = (int)(x >> 42);
  const unsigned sc = __reduce_add_sync(0xffffffffu, c);
  const unsigned sb = __reduce_add_sync(0xffffffffu, b);
  const int sa = __reduce_add_sync(0xffffffffu, a);
  return (long long)((unsigned long long)(long long)sa << 42) + ((long long)sb << 21) + (long long)sc;
}

__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(1023 + e) << 52); }

// ---- bulk asynchronous copies (the copy engine writes shared memory and completes an mbarrier transaction; the
// issuing warp's own shared-memory accesses do not queue behind the copy)
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// one arrival that also expects `bytes` of copy transactions, then the copy of `bytes` (16-byte aligned, a multiple
// of 16) from global memory into this CTA's shared memory, completing on `bar`
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
               ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
               : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Waits for the completion of phase `parity` of bar for at most MBAR_WAIT_NS nanoseconds; false when it gave up.
constexpr unsigned long long MBAR_WAIT_NS = 2000000000ull;
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (global_ns() - t0 < MBAR_WAIT_NS)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// generic-proxy global stores of this thread become visible to later bulk copies (async proxy)
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }

__device__ __forceinline__ uint32_t bcast4(int v) { return (uint32_t)v * 0x01010101u; }
__device__ __forceinline__ int byte_of(uint32_t w, int e) { return (int)((w >> (8 * e)) & 255u); }
__device__ __forceinline__ uint32_t ld_u32(const uint8_t* p) { return *reinterpret_cast<const uint32_t*>(p); }

// ------------------------------------------------------------------------------------------------ fused row pass
struct PassU {
  uint8_t* leaf_prev;         // tree j-1 leaf ids (written back after the move)
  const uint8_t* leaf_cur;    // tree j leaf ids
  const uint8_t* qprev;       // codes of tree j-1's split variable
  const uint8_t* qcur;        // codes of tree j's proposed split variable
  const uint8_t* leaf_next;   // tree j+1 leaf ids (prefetch), or null
  const uint8_t* qnext;       // codes of tree j+1's proposed split variable (prefetch), or null
  float* r;
  const float* ws;
  const float* D;             // [64] apply deltas
  const float2* tc;           // [64] {theta of tree j, compact leaf index as int bits}
  long long* bins;            // [NBS + NSPLIT][RT]: per-thread leaf sums, then split partials
  unsigned long long* ovb;    // [64] leaves with compact index >= NBS
  long long* tot;             // [TOT] CTA totals
  unsigned long long* h0;     // learned cut proposal: per code of the birth variable, sum fx(w) / sum fx(w*R) [256]
  unsigned long long* h1;
  int* hc;                    // and the row count [256]
  float sqs;                  // 2^(rss_shift - fx_shift): fx2(w R^2) = llrint(w 2^S R R sqs)
  int xhist;                  // accumulate the histogram of the rows of leaf sqa
  int sqa, sqb;               // rows of leaves sqa and sqb accumulate fx2(w R^2) (-1: none)
  float DL, DR;
  int n, g0, g1, rt, RT, nleaf;   // rows: groups [g0, g1) of this CTA (r and ws are indexed from group g0)
  int apply, pmode, pnx, pc, pL, pR, pl, pr;
  int cmode, cnx, cc;
};

// The words of one group that the pass of tree j consumes: leaf ids of trees j-1 (lp) and j (lc), codes of the
// previous (qp) and current (qc) split variables.
struct GroupWords { uint32_t lp, lc, qp, qc; };

// One group of 4 rows: apply tree j-1's move, accumulate tree j's statistics (src/bart_kernel.cpp:164-201
// semantics; gpu/bart_batch.cu:184-227 fixed-point semantics).  Leaf sums go to this thread's column of the bin
// matrix (compact leaf index < NBS; conflict-free, RT * 8 bytes is a multiple of the 32 banks), leaves beyond to
// shared atomics.  For a birth proposal only the left child's sums and count are accumulated: the right child's
// follow from the node's totals.
template <bool XP>
__device__ __forceinline__ void pass_group(const PassU& P, int g, const GroupWords& W, long long& sl0, long long& sl1,
                                           int& nl, long long& sq) {
  float* __restrict__ rp = P.r;
  const float* __restrict__ wp = P.ws;
  const float* __restrict__ Dp = P.D;
  const float2* __restrict__ tcp = P.tc;
  const float4 r4 = reinterpret_cast<const float4*>(rp)[g - P.g0];
  const float4 w4 = reinterpret_cast<const float4*>(wp)[g - P.g0];
  float rr[4] = {r4.x, r4.y, r4.z, r4.w};
  const float ww[4] = {w4.x, w4.y, w4.z, w4.w};
  if (P.apply) {
    uint32_t lpn = W.lp, mv = 0u, side = 0u;
    if (P.pmode == 1) {
      mv = __vcmpeq4(W.lp, bcast4(P.pnx));
      side = __vcmpleu4(W.qp, bcast4(P.pc));                // 0xFF where the row goes left
      lpn = (W.lp & ~mv) | (mv & ((side & bcast4(P.pL)) | (~side & bcast4(P.pR))));
    } else if (P.pmode == 2) {
      const uint32_t md = __vcmpeq4(W.lp, bcast4(P.pl)) | __vcmpeq4(W.lp, bcast4(P.pr));
      lpn = (W.lp & ~md) | (md & bcast4(P.pnx));          // death deltas come from the table
    }
#pragma unroll
    for (int e = 0; e < 4; e++) {
      float delta = Dp[byte_of(W.lp, e)];
      if (byte_of(mv, e)) delta = byte_of(side, e) ? P.DL : P.DR;
      rr[e] = __fsub_rn(rr[e], delta);
    }
    reinterpret_cast<float4*>(rp)[g - P.g0] = make_float4(rr[0], rr[1], rr[2], rr[3]);
    if (lpn != W.lp) *reinterpret_cast<uint32_t*>(P.leaf_prev + 4 * g) = lpn;
  }
  // rows of a birth proposal's node that go left (padding rows beyond n excluded)
  uint32_t inl = 0u;
  if (P.cmode == 1) {
    inl = __vcmpeq4(W.lc, bcast4(P.cnx)) & __vcmpleu4(W.qc, bcast4(P.cc));
    const int left = P.n - 4 * g;
    if (left < 4) inl &= (1u << (8 * (left > 0 ? left : 0))) - 1u;
    nl += __popc(inl) >> 3;
  }
  // rows of the learned cut proposal's node (extras kernels only): fx2(w R^2), and the code histogram of a birth
  uint32_t insq = 0u;
  if constexpr (XP) {
    if (P.sqa >= 0) {
      insq = __vcmpeq4(W.lc, bcast4(P.sqa)) | __vcmpeq4(W.lc, bcast4(P.sqb));
      const int left = P.n - 4 * g;
      if (left < 4) insq &= (1u << (8 * (left > 0 ? left : 0))) - 1u;
    }
  }
  long long* mybins = P.bins + P.rt;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const int lc = byte_of(W.lc, e);
    const float2 t = tcp[lc];
    const float R = __fadd_rn(rr[e], t.x);
    const float wrf = __fmul_rn(ww[e], R);
    const long long wr = __float2ll_rn(wrf);
    const int ci = __float_as_int(t.y);
    if (ci < NBS) mybins[ci * P.RT] += wr;
    else atomicAdd(&P.ovb[lc], (unsigned long long)wr);
    if (byte_of(inl, e)) { sl0 += __float2ll_rn(ww[e]); sl1 += wr; }
    if constexpr (XP) {
      if (byte_of(insq, e)) {
        sq += __float2ll_rn(__fmul_rn(__fmul_rn(wrf, R), P.sqs));
        if (P.xhist) {
          const int cd = byte_of(W.qc, e);
          atomicAdd(&P.h0[cd], (unsigned long long)__float2ll_rn(ww[e]));
          atomicAdd(&P.h1[cd], (unsigned long long)wr);
          atomicAdd(&P.hc[cd], 1);
        }
      }
    }
  }
}

// End of the pass: the split partials join this thread's column of the bin matrix (rows NBS..); the CTA totals are
// formed afterwards by reduce_totals(), one warp per total.
template <bool XP>
__device__ __forceinline__ void pass_store(const PassU& P, long long sl0, long long sl1, int nl, long long sq) {
  long long* mybins = P.bins + P.rt;
  if (P.cmode == 1) {
    mybins[(NBS + 0) * P.RT] = sl0; mybins[(NBS + 1) * P.RT] = sl1; mybins[(NBS + 2) * P.RT] = nl;
  }
  if constexpr (XP) {
    if (P.sqa >= 0) mybins[(NBS + 3) * P.RT] = sq;
  }
}

// CTA totals of one pass: warp w sums row w of the bin matrix over the RT row threads (lanes read consecutive
// threads' partials, and clears the leaf rows for the next pass), then reduces across the warp.  Exact int64.  Called
// by every warp of the CTA after the pass and a barrier.
__device__ __forceinline__ void reduce_totals(long long* bins, int RT, int nleaf, int cmode, long long* tot,
                                              bool sq = false) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, NW = blockDim.x >> 5;
  const int nb = nleaf < NBS ? nleaf : NBS;
  for (int row = warp; row < NBS + NSPLIT; row += NW) {
    const bool leafrow = row < NBS;
    if (leafrow ? row >= nb : (row < NBS + 3 ? cmode != 1 : !sq)) continue;
    long long* br = bins + (long long)row * RT;
    long long v = 0;
    for (int k = lane; k < RT; k += 32) {
      v += br[k];
      if (leafrow) br[k] = 0;
    }
    const long long t = warp_sum64(v);
    if (lane == 0) tot[row] = t;
  }
}

// Pass with words streamed from L2 in the pass itself (any n).
template <bool XP>
__device__ void pass_rows_stream(const PassU& P) {
  long long sl0 = 0, sl1 = 0, sq = 0;
  int nl = 0;
  for (int g = P.g0 + P.rt; g < P.g1; g += P.RT) {
    GroupWords W;
    W.lc = ld_u32(P.leaf_cur + 4 * g);
    W.lp = P.apply ? ld_u32(P.leaf_prev + 4 * g) : 0u;
    W.qp = (P.apply && P.pmode == 1) ? __ldg(reinterpret_cast<const uint32_t*>(P.qprev + 4 * g)) : 0u;
    W.qc = (P.cmode == 1 || P.xhist) ? __ldg(reinterpret_cast<const uint32_t*>(P.qcur + 4 * g)) : 0u;
    pass_group<XP>(P, g, W, sl0, sl1, nl, sq);
  }
  pass_store<XP>(P, sl0, sl1, nl, sq);
}

// Pass with register-held words (each row thread owns at most G groups).  lcr/qcr hold tree j-1's words on entry
// (tree j's on exit); nlc/nqc hold tree j's prefetched words on entry (tree j+1's on exit).  first: tree 0 of a
// sweep (no prefetch available, nothing to apply).
template <int G, bool XP>
__device__ __forceinline__ void pass_rows_regs(const PassU& P, bool first, uint32_t (&lcr)[G], uint32_t (&qcr)[G],
                                               uint32_t (&nlc)[G], uint32_t (&nqc)[G]) {
  long long sl0 = 0, sl1 = 0, sq = 0;
  int nl = 0;
#pragma unroll
  for (int k = 0; k < G; k++) {
    const int g = P.g0 + P.rt + k * P.RT;
    if (g < P.g1) {
      GroupWords W;
      if (first) {
        W.lc = ld_u32(P.leaf_cur + 4 * g);
        W.qc = (P.cmode == 1 || P.xhist) ? __ldg(reinterpret_cast<const uint32_t*>(P.qcur + 4 * g)) : 0u;
      } else {
        W.lc = nlc[k];
        W.qc = nqc[k];
      }
      W.lp = lcr[k];
      W.qp = qcr[k];
      pass_group<XP>(P, g, W, sl0, sl1, nl, sq);
      lcr[k] = W.lc;
      qcr[k] = W.qc;
    }
  }
  // the next tree's words: in flight while the control phase runs
#pragma unroll
  for (int k = 0; k < G; k++) {
    const int g = P.g0 + P.rt + k * P.RT;
    if (g < P.g1 && P.leaf_next) {
      nlc[k] = ld_u32(P.leaf_next + 4 * g);
      nqc[k] = P.qnext ? __ldg(reinterpret_cast<const uint32_t*>(P.qnext + 4 * g)) : 0u;
    }
  }
  pass_store<XP>(P, sl0, sl1, nl, sq);
}

// ------------------------------------------------------------------------------------------------ tree helpers
__device__ __forceinline__ int select_kth(unsigned long long m, int k) {   // src/bart_kernel.cpp:94-101
  for (int i = 0; i < k && m; i++) m &= m - 1ull;
  return m ? __ffsll((long long)m) - 1 : 0;
}
__device__ __forceinline__ int first_free(unsigned long long used, int skip) {   // src/bart_kernel.cpp:102-109
  unsigned long long f = ~used & ~1ull;
  if (skip >= 0) f &= ~(1ull << skip);
  return f ? __ffsll((long long)f) - 1 : -1;
}
__device__ void node_range(const DTree* t, int x, int v, int nc, int& L, int& U) {   // src/bart_kernel.cpp:238-251
  L = 0; U = nc - 1;
  int node = x;
  for (int s = 0; s < MAXDEPTH; s++) {
    if (node == 0) break;
    const int pa = t->par[node];
    if ((int)t->v[pa] == v) {
      if ((int)t->l[pa] == node) { if ((int)t->c[pa] - 1 < U) U = (int)t->c[pa] - 1; }
      else { if ((int)t->c[pa] + 1 > L) L = (int)t->c[pa] + 1; }
    }
    node = pa;
  }
}
__device__ int count_goodvars(const DTree* t, int x, const int* nc, int p) {   // src/bart_kernel.cpp:253-276
  int g = 0;
  for (int v = 0; v < p; v++) {
    int L, U;
    node_range(t, x, v, nc[v], L, U);
    g += (U >= L);
  }
  return g;
}
__device__ __noinline__ double lh(double b, double M, double t2) {   // src/bart_kernel.cpp:278
  const double k = b * t2 + 1.0;
  return -0.5 * fbm::fb_log_inl(k) + 0.5 * M * M * t2 / k;   // inlined log: its division overlaps the one here
}

// ------------------------------------------------------------------------------------------------ learned proposal
// Features of node nx of tree t for the learned split-variable proposal (functions of the tree and the node's row
// count only, so the forward and the reverse move see the same inputs):
//   x[0] depth / 8;  x[1] floor(log2(cnt + 1)) / 16;
//   x[2 + v]  min(internal nodes other than `exclude` splitting on v, 8) / 8;
//   x[34 + v] cut range of v at nx, (U - L + 1) / numcut[v];  x[66 + v] L / numcut[v]  (0 when empty).
// Returns the mask of predictors whose range at nx is non-empty.
__device__ __noinline__ unsigned node_features(const DTree* t, int nx, int cnt, int exclude, const DChain& C, float* x) {
  for (int k = 0; k < MLP_IN; k++) x[k] = 0.0f;
  x[0] = __fdiv_rn((float)t->d[nx], 8.0f);
  x[1] = __fdiv_rn((float)(31 - __clz(cnt + 1)), 16.0f);
  int use[PMAX];
  for (int v = 0; v < PMAX; v++) use[v] = 0;
  const unsigned long long inner = t->used & ~t->leaf;
  for (unsigned long long im = inner; im; im &= im - 1ull) {
    const int sl = __ffsll((long long)im) - 1;
    if (sl != exclude) use[t->v[sl]]++;
  }
  unsigned valid = 0u;
  for (int v = 0; v < PMAX; v++) {
    x[2 + v] = __fdiv_rn((float)(use[v] < 8 ? use[v] : 8), 8.0f);
    if (v < C.p && C.numcut[v] > 0) {
      int L, U;
      node_range(t, nx, v, C.numcut[v], L, U);
      if (U >= L) {
        x[34 + v] = __fdiv_rn((float)(U - L + 1), (float)C.numcut[v]);
        x[66 + v] = __fdiv_rn((float)L, (float)C.numcut[v]);
        valid |= 1u << v;
      }
    }
  }
  return valid;
}

// ---- the learned model's phase at sweep start: one warp per tree, up to MP_NB trees of a warp at once
// A tree held across a warp's registers: lane i holds bytes [16 i, 16 i + 16) of the DTree, and a field is read by a
// warp-uniform shuffle.  The proposal's tree walks then cost shuffles instead of dependent global loads.
namespace wt {
constexpr int L = 0, R = NODES, PAR = 2 * NODES, V = 3 * NODES, C = 4 * NODES, D = 5 * NODES, NGV = 6 * NODES;
constexpr int USED = 7 * NODES, LEAF = 7 * NODES + 8, UNITS = (int)(sizeof(DTree) / 16);
static_assert(sizeof(DTree) % 16 == 0 && UNITS <= 32, "a tree fits one 16-byte unit per lane");
__device__ __forceinline__ uint4 load(const DTree* t, int lane) {
  return lane < UNITS ? reinterpret_cast<const uint4*>(t)[lane] : make_uint4(0u, 0u, 0u, 0u);
}
__device__ __forceinline__ uint32_t word(const uint4& q, int off) {   // the 32-bit word at byte offset off (uniform)
  const int c = (off >> 2) & 3;
  const uint32_t w = c == 0 ? q.x : c == 1 ? q.y : c == 2 ? q.z : q.w;
  return __shfl_sync(0xffffffffu, w, off >> 4);
}
__device__ __forceinline__ int byte(const uint4& q, int field, int s) {
  const int off = field + s;
  return (int)((word(q, off & ~3) >> (8 * (off & 3))) & 0xffu);
}
__device__ __forceinline__ unsigned long long mask(const uint4& q, int off) {
  return (unsigned long long)word(q, off) | ((unsigned long long)word(q, off + 4) << 32);
}
// node_range (src/bart_kernel.cpp:238-251) of node x for predictor v with nc cutpoints; the walk is warp-uniform
__device__ __forceinline__ void node_range(const uint4& q, int x, int v, int nc, int& L, int& U) {
  L = 0; U = nc - 1;
  int node = x;
  for (int s = 0; s < MAXDEPTH; s++) {
    if (node == 0) break;
    const int pa = byte(q, PAR, node);
    const int vp = byte(q, V, pa), lp = byte(q, wt::L, pa), cp = byte(q, wt::C, pa);
    if (vp == v) {
      if (lp == node) { if (cp - 1 < U) U = cp - 1; }
      else { if (cp + 1 > L) L = cp + 1; }
    }
    node = pa;
  }
}
}  // namespace wt

constexpr int MP_NB = 1;   // trees of one warp evaluated together (each weight load serves all of them)

// node_features with lane v on predictor v, from a warp-held tree: lane v returns x[2 + v], x[34 + v], x[66 + v] in
// xa, xb, xc and every lane x[0], x[1]; returns the valid mask
__device__ __forceinline__ unsigned node_features_wt(const uint4& q, int nx, int cnt, int exclude, const DChain& C,
                                                     int lane, float& x0, float& x1, float& xa, float& xb, float& xc) {
  x0 = __fdiv_rn((float)wt::byte(q, wt::D, nx), 8.0f);
  x1 = __fdiv_rn((float)(31 - __clz(cnt + 1)), 16.0f);
  int use = 0;
  const unsigned long long inner = wt::mask(q, wt::USED) & ~wt::mask(q, wt::LEAF);
  for (unsigned long long im = inner; im; im &= im - 1ull) {
    const int sl = __ffsll((long long)im) - 1;
    if (sl != exclude && wt::byte(q, wt::V, sl) == lane) use++;
  }
  xa = __fdiv_rn((float)(use < 8 ? use : 8), 8.0f);
  const int nc = lane < C.p ? C.numcut[lane] : 0;
  int L, U;
  wt::node_range(q, nx, lane, nc, L, U);
  const bool ok = nc > 0 && U >= L;
  xb = ok ? __fdiv_rn((float)(U - L + 1), (float)nc) : 0.0f;
  xc = ok ? __fdiv_rn((float)L, (float)nc) : 0.0f;
  return __ballot_sync(0xffffffffu, ok);
}

// The model at NB nodes, evaluated by one warp from the weight image W (shared or global memory).  Lane o computes
// hidden outputs o and o + 32, then logit o, of every node; each output is the sequential sum bias + w[0] x[0] +
// w[1] x[1] + ... in FP32 without fused multiply-add.  The masked softmax is in FP64 (max over the valid logits, 0
// when none; exp of the differences; their sum in predictor order).  q[b] = q_lane of node b (0 when invalid).
__device__ __forceinline__ float feat_k(int k, float x0, float x1, float xa, float xb, float xc) {
  return k == 0 ? x0 : k == 1 ? x1 : __shfl_sync(0xffffffffu, k < 34 ? xa : k < 66 ? xb : xc, (k - 2) & 31);
}
__device__ __forceinline__ float acc2(float a, uint32_t pw, float xlo, float xhi) {
  a = __fadd_rn(a, __fmul_rn(__uint_as_float(pw << 16), xlo));
  return __fadd_rn(a, __fmul_rn(__uint_as_float(pw & 0xFFFF0000u), xhi));
}
template <int NB>
__device__ __forceinline__ void model_q_batch(const uint32_t* W, const float (&x0)[NB], const float (&x1)[NB],
                                              const float (&xa)[NB], const float (&xb)[NB], const float (&xc)[NB],
                                              const unsigned (&valid)[NB], int lane, double (&q)[NB]) {
  const float* bias = reinterpret_cast<const float*>(W + MIMG_B);
  float a0[NB], a1[NB], h1a[NB], h1b[NB];
  const uint32_t* r0 = W + lane * MIMG_W1S;
  const uint32_t* r1 = W + (lane + 32) * MIMG_W1S;
#pragma unroll
  for (int b = 0; b < NB; b++) { a0[b] = bias[lane]; a1[b] = bias[lane + 32]; }
#pragma unroll
  for (int kk = 0; kk < MIMG_W1S; kk++) {
    const uint32_t p0 = r0[kk], p1 = r1[kk];
#pragma unroll
    for (int b = 0; b < NB; b++) {
      const float xl = feat_k(2 * kk, x0[b], x1[b], xa[b], xb[b], xc[b]);
      const float xh = feat_k(2 * kk + 1, x0[b], x1[b], xa[b], xb[b], xc[b]);
      a0[b] = acc2(a0[b], p0, xl, xh);
      a1[b] = acc2(a1[b], p1, xl, xh);
    }
  }
#pragma unroll
  for (int b = 0; b < NB; b++) {
    h1a[b] = a0[b] > 0.0f ? a0[b] : 0.0f; h1b[b] = a1[b] > 0.0f ? a1[b] : 0.0f;
    a0[b] = bias[MLP_H + lane]; a1[b] = bias[MLP_H + lane + 32];
  }
  r0 = W + MIMG_W2 + lane * MIMG_W2S;
  r1 = W + MIMG_W2 + (lane + 32) * MIMG_W2S;
#pragma unroll
  for (int kk = 0; kk < MLP_H / 2; kk++) {
    const uint32_t p0 = r0[kk], p1 = r1[kk];
#pragma unroll
    for (int b = 0; b < NB; b++) {
      const float hl = __shfl_sync(0xffffffffu, kk < 16 ? h1a[b] : h1b[b], (2 * kk) & 31);
      const float hh = __shfl_sync(0xffffffffu, kk < 16 ? h1a[b] : h1b[b], (2 * kk + 1) & 31);
      a0[b] = acc2(a0[b], p0, hl, hh);
      a1[b] = acc2(a1[b], p1, hl, hh);
    }
  }
#pragma unroll
  for (int b = 0; b < NB; b++) {
    h1a[b] = a0[b] > 0.0f ? a0[b] : 0.0f; h1b[b] = a1[b] > 0.0f ? a1[b] : 0.0f;   // now the second hidden layer
    a0[b] = bias[2 * MLP_H + lane];
  }
  r0 = W + MIMG_W3 + lane * MIMG_W2S;
#pragma unroll
  for (int kk = 0; kk < MLP_H / 2; kk++) {
    const uint32_t p0 = r0[kk];
#pragma unroll
    for (int b = 0; b < NB; b++) {
      const float hl = __shfl_sync(0xffffffffu, kk < 16 ? h1a[b] : h1b[b], (2 * kk) & 31);
      const float hh = __shfl_sync(0xffffffffu, kk < 16 ? h1a[b] : h1b[b], (2 * kk + 1) & 31);
      a0[b] = acc2(a0[b], p0, hl, hh);
    }
  }
#pragma unroll
  for (int b = 0; b < NB; b++) {
    const double z = (double)a0[b];
    const bool vl = (valid[b] >> lane) & 1u;
    double zmax = vl ? z : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double other = __shfl_xor_sync(0xffffffffu, zmax, o);
      zmax = other > zmax ? other : zmax;
    }
    if (!valid[b]) zmax = 0.0;
    const double e = vl ? fbm::fb_exp(z - zmax) : 0.0;
    double sum = 0.0;
#pragma unroll
    for (int v = 0; v < MLP_OUT; v++) sum = sum + __shfl_sync(0xffffffffu, e, v);
    q[b] = sum > 0.0 ? e / sum : 0.0;
  }
}

// probability that the mixture proposes valid predictor v: mix * q_v + (1 - mix) / p
__device__ __forceinline__ double mix_prob(double mix, double qv, int p) {
  return mix * qv + (1.0 - mix) * (1.0 / (double)p);
}

// The learned model's part of every proposal of sweep it, at sweep start (trees j = crank, crank + CS, ... of the
// chain are this CTA's share; a warp takes every (CS * warps)-th of them, MP_NB at a time): the same node choice as
// propose() makes from the trees at sweep start, then for a birth the model's variable (with probability mix from
// the masked softmax, else uniformly, as BART) and the proposal-ratio correction (1/p) / (mix q_v + (1 - mix)/p); for
// a death the correction of the reverse birth, the model evaluated at the collapsed node with the node's own split
// left out of the use counts.  Results go to B.mvar / B.mcorr, which propose() reads after a barrier.
__device__ __forceinline__ void model_phase(const DBufs& B, const DChain& C, const DTree* trees, const long long* s0g,
                                            const uint32_t* W, int it, int crank, int CS) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, NW = blockDim.x >> 5;
  const int step = CS * NW;
  for (int j0 = crank + CS * warp; j0 < C.m; j0 += MP_NB * step) {   // warp-uniform loop
    float x0[MP_NB], x1[MP_NB], xa[MP_NB], xb[MP_NB], xc[MP_NB];
    unsigned valid[MP_NB];
    int kind[MP_NB], vdeath[MP_NB];
    double uvb[MP_NB];
#pragma unroll
    for (int b = 0; b < MP_NB; b++) {
      const int j = j0 + b * step;
      x0[b] = x1[b] = xa[b] = xb[b] = xc[b] = 0.0f;
      valid[b] = 0u; kind[b] = 0; vdeath[b] = 0; uvb[b] = 0.0;
      if (j >= C.m) continue;
      const uint4 q = wt::load(trees + j, lane);
      const int* cnt = reinterpret_cast<const int*>(s0g + (long long)j * LST + NODES);
      const unsigned long long used = wt::mask(q, wt::USED), leafm = wt::mask(q, wt::LEAF);
      unsigned long long goodm = 0, nogm = 0;
      for (unsigned long long um = used; um; um &= um - 1ull) {
        const int s = __ffsll((long long)um) - 1;
        if ((leafm >> s) & 1ull) {
          int g = wt::byte(q, wt::NGV, s);
          if (g == 255) {
            const int nc = lane < C.p ? C.numcut[lane] : 0;
            int L, U;
            wt::node_range(q, s, lane, nc, L, U);
            g = __popc(__ballot_sync(0xffffffffu, lane < C.p && U >= L));
          }
          if (g > 0) goodm |= 1ull << s;
        } else if (((leafm >> wt::byte(q, wt::L, s)) & 1ull) && ((leafm >> wt::byte(q, wt::R, s)) & 1ull)) {
          nogm |= 1ull << s;
        }
      }
      const int ngood = __popcll(goodm), nnogs = __popcll(nogm);
      const double PBx = ngood == 0 ? 0 : (used == 1ull ? 1 : 0.5);
      const fbm::U4 xr = fbm::philox(0u, (uint32_t)j, (uint32_t)it, fbm::TAG_PROP, C.seed);
      const double ub = fbm::u32d(xr.x), un = fbm::u32d(xr.y);
      uvb[b] = fbm::u32d(xr.z);
      if (ub < PBx) {
        const int nx = select_kth(goodm, (int)(un * ngood));
        kind[b] = 1;
        valid[b] = node_features_wt(q, nx, cnt[nx], -1, C, lane, x0[b], x1[b], xa[b], xb[b], xc[b]);
      } else if (nnogs > 0) {
        const int nx = select_kth(nogm, (int)(un * nnogs));
        kind[b] = 2;
        vdeath[b] = wt::byte(q, wt::V, nx);
        const int lr = cnt[wt::byte(q, wt::L, nx)] + cnt[wt::byte(q, wt::R, nx)];
        valid[b] = node_features_wt(q, nx, lr, nx, C, lane, x0[b], x1[b], xa[b], xb[b], xc[b]);
      }
    }
    double qb[MP_NB];
    model_q_batch<MP_NB>(W, x0, x1, xa, xb, xc, valid, lane, qb);
#pragma unroll
    for (int b = 0; b < MP_NB; b++) {
      const int j = j0 + b * step;
      if (j >= C.m) continue;
      int v = 0;
      double corr = 1.0;
      if (kind[b] == 1) {
        const fbm::U4 y2 = fbm::philox(0u, (uint32_t)j, (uint32_t)it, fbm::TAG_PROP2, C.seed);
        const double umix = fbm::u32d(y2.x), uvm = fbm::u32d(y2.y);
        if (umix < B.mix && valid[b]) {   // the first valid k whose cumulative q exceeds uvm, else the last valid
          double cum = 0.0;
          int last = 0;
          v = -1;
#pragma unroll
          for (int k = 0; k < MLP_OUT; k++) {
            const double qk = __shfl_sync(0xffffffffu, qb[b], k);
            if ((valid[b] >> k) & 1u) { cum = cum + qk; last = k; if (v < 0 && uvm < cum) v = k; }
          }
          if (v < 0) v = last;
        } else {
          v = (int)(uvb[b] * C.p); if (v >= C.p) v = C.p - 1;
        }
        const double qv = __shfl_sync(0xffffffffu, qb[b], v);
        corr = ((valid[b] >> v) & 1u) ? (1.0 / (double)C.p) / mix_prob(B.mix, qv, C.p) : 1.0;
      } else if (kind[b] == 2) {
        const double qv = __shfl_sync(0xffffffffu, qb[b], vdeath[b]);
        corr = mix_prob(B.mix, qv, C.p) * (double)C.p;
      }
      if (lane == 0) { B.mvar[C.off_tree + j] = v; B.mcorr[C.off_tree + j] = corr; }
    }
  }
}

// Proposal of tree j at sweep it (src/bart_kernel.cpp:413-464); also resolves unknown goodvar counts of leaves.
// With a learned model (B.mvar), the birth variable and the proposal-probability correction of the birth, or of the
// reverse birth of a death, come from model_phase, and pr carries the correction, so the chain keeps BART's target.
// cnt: the tree's per-slot row counts.  When training examples are collected, the birth node's features go to
// feat / *fvalid.
// internal nodes of t splitting on v, other than `exclude`
__device__ __forceinline__ int uses_of(const DTree* t, int v, int exclude) {
  int u = 0;
  for (unsigned long long im = t->used & ~t->leaf; im; im &= im - 1ull) {
    const int s = __ffsll((long long)im) - 1;
    u += s != exclude && (int)t->v[s] == v;
  }
  return u;
}

// With px (model and collecting kernels) the learned cut proposal's view of the proposal is filled in, and with a
// cut head (B.cimg) a birth's cut is left to the step (PROP_DEFER).
template <bool LP, bool MP>
__device__ Prop propose(DTree* t, const DChain& C, const DBufs& B, const int* cnt, int j, int it, Masks& mk,
                        float* feat, unsigned* fvalid, PropX* px) {
  const double pb = 0.5;
  const unsigned long long used = t->used, leafm = t->leaf;
  mk.used = used; mk.leaf = leafm;
  for (unsigned long long lm = used & leafm; lm; lm &= lm - 1ull) {
    const int s = __ffsll((long long)lm) - 1;
    if (t->ngv[s] == 255) t->ngv[s] = (uint8_t)count_goodvars(t, s, C.numcut, C.p);
  }
  unsigned long long goodm = 0, nogm = 0;
  for (unsigned long long um = used; um; um &= um - 1ull) {
    const int s = __ffsll((long long)um) - 1;
    if ((leafm >> s) & 1ull) { if (t->ngv[s] > 0) goodm |= 1ull << s; }
    else if (((leafm >> t->l[s]) & 1ull) && ((leafm >> t->r[s]) & 1ull)) nogm |= 1ull << s;
  }
  const int ngood = __popcll(goodm), nnogs = __popcll(nogm);
  const bool single = (used == 1ull);
  const double PBx = ngood == 0 ? 0 : (single ? 1 : pb);
  const fbm::U4 x = fbm::philox(0u, (uint32_t)j, (uint32_t)it, fbm::TAG_PROP, C.seed);
  const double ub = fbm::u32d(x.x), un = fbm::u32d(x.y), uv = fbm::u32d(x.z), uc = fbm::u32d(x.w);
  const bool model = MP && B.mvar != nullptr;
  Prop P;
  P.mode = 0; P.nx = 0; P.v = 0; P.c = 0; P.l = 0; P.r = 0; P.dnx = P.flags = 0; P.logpr = 0; P.lu = 0;
  double pr = 0;
  if (ub < PBx) {
    const int nx = select_kth(goodm, (int)(un * ngood));
    int v;
    double corr = 1.0;
    if (model) { v = B.mvar[C.off_tree + j]; corr = B.mcorr[C.off_tree + j]; }
    else { v = (int)(uv * C.p); if (v >= C.p) v = C.p - 1; }
    if constexpr (LP) {
      if (feat) *fvalid = node_features(t, nx, cnt[nx], -1, C, feat);
    }
    int bL, bU;
    node_range(t, nx, v, C.numcut[v], bL, bU);
    if (bU >= bL && (int)t->d[nx] + 1 < MAXDEPTH) {
      int c = bL + (int)(uc * (bU - bL + 1)); if (c > bU) c = bU;
      const int dnx = t->d[nx];
      const double PGnx = C.pg[dnx];
      double PGly, PGry;
      if (t->ngv[nx] > 1) { PGly = PGry = C.pg[dnx + 1]; }
      else { PGly = (c - 1 < bL) ? 0 : C.pg[dnx + 1]; PGry = (bU < c + 1) ? 0 : C.pg[dnx + 1]; }
      const double PDy = (ngood > 1) ? 1 - pb : ((PGry == 0 && PGly == 0) ? 1 : 1 - pb);
      double Pnogy;
      if (nx == 0) Pnogy = 1;
      else {
        const int pa = t->par[nx];
        const bool panog = ((leafm >> t->l[pa]) & 1ull) && ((leafm >> t->r[pa]) & 1ull);
        Pnogy = panog ? (double)1 / nnogs : (double)1 / (nnogs + 1);
      }
      const double Pbotx = (double)1 / ngood;
      pr = (PGnx * (1 - PGly) * (1 - PGry) * PDy * Pnogy) / ((1 - PGnx) * Pbotx * PBx);
      if (model) pr = pr * corr;
      P.mode = 1; P.nx = (uint8_t)nx; P.v = (uint8_t)v; P.c = (uint8_t)c; P.dnx = (uint8_t)dnx;
      if (MP && px) {   // the ratio for a cut inside the range or at either end (c == bL: k & 1, c == bU: k & 2)
        px->L = (uint8_t)bL; px->U = (uint8_t)bU; px->uses = (uint8_t)uses_of(t, v, -1);
        for (int k = 0; k < 4; k++) {
          double gl, gr;
          if (t->ngv[nx] > 1) { gl = gr = C.pg[dnx + 1]; }
          else { gl = (k & 1) ? 0 : C.pg[dnx + 1]; gr = (k & 2) ? 0 : C.pg[dnx + 1]; }
          const double pdy = (ngood > 1) ? 1 - pb : ((gr == 0 && gl == 0) ? 1 : 1 - pb);
          double prk = (PGnx * (1 - gl) * (1 - gr) * pdy * Pnogy) / ((1 - PGnx) * Pbotx * PBx);
          if (model) prk = prk * corr;
          px->pr4[k] = prk;
        }
        if (B.cimg) P.flags = PROP_DEFER;
      }
    }
  } else if (nnogs > 0) {
    const int nx = select_kth(nogm, (int)(un * nnogs));
    const int dny = t->d[nx], l = t->l[nx], r = t->r[nx];
    const double PGny = C.pg[dny];
    const double PGlx = t->ngv[l] > 0 ? C.pg[dny + 1] : 0, PGrx = t->ngv[r] > 0 ? C.pg[dny + 1] : 0;
    const double PBy = (nx == 0) ? 1 : pb;
    const int ng2 = ngood - (t->ngv[l] > 0) - (t->ngv[r] > 0) + 1;
    const double Pboty = (double)1 / ng2, PDx = 1 - PBx, Pnogx = (double)1 / nnogs;
    pr = ((1 - PGny) * PBy * Pboty) / (PGny * (1 - PGlx) * (1 - PGrx) * PDx * Pnogx);
    if (model) pr = pr * B.mcorr[C.off_tree + j];   // the reverse birth
    P.mode = 2; P.nx = (uint8_t)nx; P.l = (uint8_t)l; P.r = (uint8_t)r;
    if (MP && px) {   // the reverse birth's variable, cut and cut range
      const int vn = t->v[nx];
      int Ln, Un;
      node_range(t, nx, vn, C.numcut[vn], Ln, Un);
      P.v = (uint8_t)vn; P.c = t->c[nx]; P.dnx = (uint8_t)dny;
      px->L = (uint8_t)Ln; px->U = (uint8_t)Un; px->uses = (uint8_t)uses_of(t, vn, nx);
      px->pr4[0] = pr;
    }
  }
  if (P.mode) {
    P.logpr = fbm::fb_log(pr);
    const fbm::U4 y = fbm::philox(0u, (uint32_t)j, (uint32_t)it, fbm::TAG_MH, C.seed);
    P.lu = fbm::fb_log(fbm::u32d(y.x));
  }
  // every slot that can be a leaf after the move: the current leaves, the two slots a birth would take, the node a
  // death would restore
  unsigned long long cand = used & leafm;
  if (P.mode == 1) {
    const int L = first_free(used, -1), R = L >= 0 ? first_free(used, L) : -1;
    if (L >= 0 && R >= 0) cand |= (1ull << L) | (1ull << R);
  } else if (P.mode == 2) {
    cand |= 1ull << P.nx;
  }
  P.cand = cand;
  return P;
}

// ------------------------------------------------------------------------------------------------ shared layout
struct Smem {
  float* r; float* ws;          // [n_pad] (shared, or global when rows do not fit)
  float* th;                    // [m][64]
  Prop* prop;                   // [m]
  Masks* masks;                 // [m]
  unsigned long long* bar;      // [2] mbarriers of the leaf-statistics buffers
  long long* s0t;               // [2][LST] leaf statistics of trees j and j+1 (buffer j & 1: S0 [64], counts int [64])
  float* D;                     // [64] apply deltas of the last decided move
  float2* tc;                   // [2][64] theta and compact leaf index
  double* z;                    // [64] mu normals of tree j beyond the first ZMAX candidates
  double* zall;                 // [m][zmax] mu normals drawn ahead
  int zmax;                     // normals drawn ahead per tree in this layout
  long long* bins;              // [NBS + NSPLIT][RT]
  long long* tot;               // [2][TOT]
  unsigned long long* ovb;      // [2][64]
  long long* red;               // [NW]
  Ctl* ctl;
  long long* ctot;              // [2][TOT] cluster totals (sum over the cluster's CTAs)
  unsigned long long* covb;     // [2][64]
  long long* xch;               // [2][4] per-CTA values exchanged across the cluster (rss, latent-z caps, sum w)
  long long* xtot;              // [2][cluster][TOT] every CTA's pass totals, pushed by their owners
  unsigned long long* xovb;     // [2][cluster][64]
  uint32_t* mimg;               // [MIMG_WORDS] the proposal model's weight image, behind the layout (B.model_smem)
  int binrows;                  // rows of the bin matrix in this layout
  // learned cut proposal (cut layouts)
  PropX* px;                    // [m]
  struct CutScr* cs;            // the cut stage's scratch
  unsigned long long* h0;       // [256] code histogram of the birth node (in the split rows of the bins)
  unsigned long long* h1;       // [256]
  int* hc;                      // [256]
  uint32_t* cimg;               // [CIMG_WORDS] the cut head's weight image, behind mimg (B.cut_smem)
  long long* xcut;              // [cluster][4] every CTA's split sums of the drawn cut, pushed by their owners
};
// scratch of the cut stage (in the bins' leaf rows, which are zero between passes; cleared again after the stage):
// features, hidden layers, logits, exponentials, block sums; the decision
struct CutScr {
  float cx[CUT_IN], h1[CUT_H], h2[CUT_H], e[CUT_E], z[256];
  double ex[256], bs[32];
  double zmax, logpr;
  long long sL0, sL1;
  int nL, c, pad0, pad1;
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

__host__ __device__ inline size_t smem_layout(int threads, int m_max, int n_pad_max, int rows_in_smem, int cluster,
                                               size_t* off, int cut = 0) {
  const int NW = threads / 32, RT = threads - 32;
  size_t o = 0;
  off[0] = o; o += rows_in_smem ? align_up((size_t)n_pad_max * 4, 16) : 0;   // r
  off[1] = o; o += rows_in_smem == 1 ? align_up((size_t)n_pad_max * 4, 16) : 0;   // ws
  off[2] = o; o += align_up((size_t)m_max * NODES * 4, 16);                  // th
  off[3] = o; o += align_up((size_t)m_max * sizeof(Prop), 16);               // prop
  off[4] = o; o += align_up((size_t)m_max * sizeof(Masks), 16);              // masks
  off[5] = o; o += 16;                                                       // bar[2]
  off[6] = o; o += 2 * LST * 8;                                              // s0t[2]
  off[7] = o; o += NODES * 4;                                                // D
  off[8] = o; o += 2 * NODES * 8;                                            // tc[2]
  off[9] = o; o += NODES * 8;                                                // z
  off[10] = o; o += (size_t)(cut ? BIN_ROWS_CUT : BIN_ROWS) * RT * 8;         // bins (leaf rows, split rows)
  off[11] = o; o += 2 * TOT * 8;                                             // tot[2]
  off[12] = o; o += 2 * NODES * 8;                                           // ovb[2]
  off[13] = o; o += align_up((size_t)NW * 8, 16);                            // red
  off[14] = o; o += align_up(sizeof(Ctl), 16);                               // ctl
  off[15] = o; o += (size_t)m_max * (cut ? ZMAX_CUT : ZMAX) * 8;            // zall
  off[16] = o; o += 2 * TOT * 8;                                             // ctot[2]
  off[17] = o; o += 2 * NODES * 8;                                           // covb[2]
  off[18] = o; o += 2 * 4 * 8;                                               // xch[2][4]
  const size_t cs = cluster > 1 ? (size_t)cluster : 0;
  off[19] = o; o += 2 * cs * TOT * 8;                                        // xtot[2][cluster][TOT]
  off[20] = o; o += 2 * cs * NODES * 8;                                      // xovb[2][cluster][64]
  off[21] = o; o += cut ? align_up((size_t)m_max * sizeof(PropX), 16) : 0;  // px
  off[22] = o; o += cut ? (size_t)(cs ? cs : 1) * 4 * 8 : 0;                   // xcut[cluster][4]
  return o;
}
constexpr int NOFF = 23;
// words staged behind the layout: the proposal model's image (when the bins cannot hold it), then the cut head's
__host__ __device__ inline size_t model_words(int threads, bool mimg_smem) {
  return mimg_smem && !bins_hold_model(threads) ? (size_t)MIMG_WORDS : 0;
}

__device__ Smem carve(unsigned char* base, int threads, int m_max, int n_pad_max, int rows_in_smem, int cluster,
                      int cut, bool mimg_smem) {
  size_t off[NOFF];
  const size_t end = smem_layout(threads, m_max, n_pad_max, rows_in_smem, cluster, off, cut);
  Smem S;
  S.r = reinterpret_cast<float*>(base + off[0]);
  S.ws = reinterpret_cast<float*>(base + off[1]);
  S.th = reinterpret_cast<float*>(base + off[2]);
  S.prop = reinterpret_cast<Prop*>(base + off[3]);
  S.masks = reinterpret_cast<Masks*>(base + off[4]);
  S.bar = reinterpret_cast<unsigned long long*>(base + off[5]);
  S.s0t = reinterpret_cast<long long*>(base + off[6]);
  S.D = reinterpret_cast<float*>(base + off[7]);
  S.tc = reinterpret_cast<float2*>(base + off[8]);
  S.z = reinterpret_cast<double*>(base + off[9]);
  S.bins = reinterpret_cast<long long*>(base + off[10]);
  S.tot = reinterpret_cast<long long*>(base + off[11]);
  S.ovb = reinterpret_cast<unsigned long long*>(base + off[12]);
  S.red = reinterpret_cast<long long*>(base + off[13]);
  S.ctl = reinterpret_cast<Ctl*>(base + off[14]);
  S.zall = reinterpret_cast<double*>(base + off[15]);
  S.ctot = reinterpret_cast<long long*>(base + off[16]);
  S.covb = reinterpret_cast<unsigned long long*>(base + off[17]);
  S.xch = reinterpret_cast<long long*>(base + off[18]);
  S.xtot = reinterpret_cast<long long*>(base + off[19]);
  S.xovb = reinterpret_cast<unsigned long long*>(base + off[20]);
  S.mimg = reinterpret_cast<uint32_t*>(base + align_up(end, 16));
  S.binrows = cut ? BIN_ROWS_CUT : BIN_ROWS;
  S.px = cut ? reinterpret_cast<PropX*>(base + off[21]) : nullptr;
  S.cs = cut ? reinterpret_cast<CutScr*>(S.bins) : nullptr;   // in the leaf rows of the bins, zeroed after use
  S.zmax = cut ? ZMAX_CUT : ZMAX;
  S.xcut = reinterpret_cast<long long*>(base + off[22]);
  const int RT = threads - 32;
  S.h0 = reinterpret_cast<unsigned long long*>(S.bins + (size_t)NBS * RT);
  S.h1 = S.h0 + 256;
  S.hc = reinterpret_cast<int*>(S.h1 + 256);
  S.cimg = S.mimg + model_words(threads, mimg_smem);
  return S;
}

// block-wide exact int64 sum (all threads call; result valid in every thread)
__device__ long long block_sum64(long long x, long long* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, NW = blockDim.x >> 5;
  const long long s = warp_sum64(x);
  __syncthreads();
  if (lane == 0) red[warp] = s;
  __syncthreads();
  long long t = 0;
  for (int w = 0; w < NW; w++) t += red[w];
  __syncthreads();
  return t;
}

// theta / compact-index table of tree j into buffer j & 1 (one slot per thread: s = 0..63)
__device__ __forceinline__ void build_tc_slot(const Smem& S, int j, int s) {
  const unsigned long long lm = S.masks[j].leaf & S.masks[j].used;
  const int ci = ((lm >> s) & 1ull) ? __popcll(lm & ((1ull << s) - 1ull)) : 255;
  S.tc[(j & 1) * NODES + s] = make_float2(S.th[j * NODES + s], __int_as_float(ci));
  if (s == 0) S.ctl->nleaf[j & 1] = __popcll(lm);
}

// copy tree j's leaf statistics from global memory into buffer j & 1: one bulk copy issued by lane 0 of the control
// warp, completing on the buffer's mbarrier (the topology stays in global memory: phase B needs only the statistics,
// and a move's changes to the topology are known without reading it)
__device__ __forceinline__ void fetch_stats(const Smem& S, const long long* s0g, int j, int lane) {
  if (lane == 0) {
    const int b = j & 1;
    S.ctl->fetches[b]++;
    bulk_copy_g2s(S.s0t + b * LST, s0g + (long long)j * LST, LST * 8, S.bar + b);
  }
  __syncwarp();
}
// wait for tree j's statistics in buffer j & 1 (the phase of its last copy); a wait that gives up is recorded
// (after a wait has given up, later waits are skipped: the chain's results are then flagged as failed)
__device__ __forceinline__ void wait_stats(const Smem& S, int j) {
  const int b = j & 1;
  if (S.ctl->err) return;
  if (!mbar_wait(S.bar + b, (S.ctl->fetches[b] - 1u) & 1u)) S.ctl->err = 1;
}

// An accepted birth of tree j becomes a training example (control warp).
__device__ __forceinline__ void collect_example(const DBufs& B, const DChain& C, int j, int v, int lane) {
  int idx = 0;
  if (lane == 0) idx = atomicAdd(B.train_count, 1);
  idx = __shfl_sync(0xffffffffu, idx, 0);
  if (idx < B.train_cap) {
    const float* f = B.feat + (C.off_tree + j) * MLP_IN;
    for (int k = lane; k < MLP_IN; k += 32) B.train_x[(long long)idx * MLP_IN + k] = f[k];
    if (lane == 0) { B.train_y[idx] = v; B.train_mask[idx] = B.feat_valid[C.off_tree + j]; }
    if (B.train_cx) {   // the same birth's cut example, written by its step
      const float* cf = B.cfeat + (C.off_tree + j) * CUT_IN;
      for (int k = lane; k < CUT_IN; k += 32) B.train_cx[(long long)idx * CUT_IN + k] = cf[k];
      if (lane == 0) {
        const int* ci3 = B.cinfo + (C.off_tree + j) * 3;
        B.train_c[idx] = ci3[0]; B.train_lo[idx] = ci3[1]; B.train_hi[idx] = ci3[2];
      }
    }
  }
}

// Write the decided move of tree j (ctl) into its topology and leaf statistics in global memory (control warp).  Only
// what the move changes is stored, one field per lane: nothing for a rejected move; for a birth the node's split and
// children, the children's parent, depth, children and unknown goodvar count, both masks and the children's sums and
// counts; for a death the node's split fields, masks, sum and count.  The move is src/bart_kernel.cpp:492-500 / 509-512;
// the reference stores its whole tree after every step instead (store_tree, :229-236, called at :533).
template <bool LP>
__device__ void commit_tree(const Smem& S, const DChain& C, const DBufs& B, DTree* trees, long long* s0g, int j,
                            int lane, bool lead) {
  const Ctl& ctl = *S.ctl;
  if constexpr (LP) {
    if (B.train_cap > 0 && lead && ctl.pmode == 1) collect_example(B, C, j, ctl.pv, lane);
  }
  const int mode = ctl.pmode;
  if (mode == 0) return;
  uint8_t* tb = reinterpret_cast<uint8_t*>(trees + j);
  long long* s0 = s0g + (long long)j * LST;
  int* cnt = reinterpret_cast<int*>(s0 + NODES);
  const int nx = ctl.pnx;
  constexpr int FL = 0, FR = NODES, FPAR = 2 * NODES, FV = 3 * NODES, FC = 4 * NODES, FD = 5 * NODES,
                FNGV = 6 * NODES, FUSED = 7 * NODES;
  if (mode == 1) {
    const int L = ctl.pL, R = ctl.pR;
    const uint8_t d1 = (uint8_t)(ctl.pd + 1);
    switch (lane) {
      case 0: tb[FV + nx] = (uint8_t)ctl.pv; break;
      case 1: tb[FC + nx] = (uint8_t)ctl.pc; break;
      case 2: tb[FL + nx] = (uint8_t)L; break;
      case 3: tb[FR + nx] = (uint8_t)R; break;
      case 4: tb[FPAR + L] = (uint8_t)nx; break;
      case 5: tb[FPAR + R] = (uint8_t)nx; break;
      case 6: tb[FL + L] = 0; break;
      case 7: tb[FR + L] = 0; break;
      case 8: tb[FL + R] = 0; break;
      case 9: tb[FR + R] = 0; break;
      case 10: tb[FD + L] = d1; break;
      case 11: tb[FD + R] = d1; break;
      case 12: tb[FNGV + L] = 255; break;   // counted by the next sweep's proposal step
      case 13: tb[FNGV + R] = 255; break;
      case 14: reinterpret_cast<unsigned long long*>(tb + FUSED)[0] = ctl.used; break;
      case 15: reinterpret_cast<unsigned long long*>(tb + FUSED)[1] = ctl.leaf; break;
      case 16: s0[L] = ctl.sL0; break;
      case 17: s0[R] = ctl.sR0; break;
      case 18: cnt[L] = ctl.nL; break;
      case 19: cnt[R] = ctl.nR; break;
      default: break;
    }
  } else {
    switch (lane) {
      case 0: tb[FL + nx] = 0; break;
      case 1: tb[FR + nx] = 0; break;
      case 2: tb[FV + nx] = 0; break;
      case 3: tb[FC + nx] = 0; break;
      case 4: reinterpret_cast<unsigned long long*>(tb + FUSED)[0] = ctl.used; break;
      case 5: reinterpret_cast<unsigned long long*>(tb + FUSED)[1] = ctl.leaf; break;
      case 6: s0[nx] = ctl.sL0; break;
      case 7: cnt[nx] = ctl.nL; break;
      default: break;
    }
  }
  __syncwarp();
}

// ------------------------------------------------------------------------------------------------ cut proposal
namespace cg = cooperative_groups;

// Features of the learned cut proposal at a node (see the oracle's orc_cut_features): depth, row count, the weighted
// residual mean and sd of the node's rows from its exact sums (S0 = sum fx(w), S1 = sum fx(w R), Q = sum fx2(w R^2))
// relative to sigma, the cut range [L, U] of v and v's uses in the tree, and v one-hot.
__device__ void cut_features(int depth, int cnt, long long S0, long long S1, long long Q, int fx_shift, int rss_shift,
                             double sigma, int L, int U, int nc, int uses, int v, float* x) {
  for (int k = 0; k < CUT_IN; k++) x[k] = 0.0f;
  x[0] = __fdiv_rn((float)depth, 8.0f);
  x[1] = __fdiv_rn((float)(31 - __clz(cnt + 1)), 16.0f);
  double mean = 0.0, sd = 0.0;
  if (S0 > 0) {
    const double w = (double)S0 * pow2(-fx_shift);
    mean = (double)S1 / (double)S0;
    const double msq = ((double)Q * pow2(-rss_shift)) / w;
    const double var = msq - mean * mean;
    sd = var > 0.0 ? sqrt(var) : 0.0;
  }
  double fm = mean / sigma;
  fm = fm < -4.0 ? -4.0 : (fm > 4.0 ? 4.0 : fm);
  double fs = sd / sigma;
  fs = fs > 4.0 ? 4.0 : fs;
  x[2] = (float)(fm * 0.25);
  x[3] = (float)(fs * 0.25);
  x[4] = __fdiv_rn((float)(U - L + 1), (float)nc);
  x[5] = __fdiv_rn((float)L, (float)nc);
  x[6] = __fdiv_rn((float)(uses < 8 ? uses : 8), 8.0f);
  if (v >= 0 && v < 32) x[8 + v] = 1.0f;
}

__device__ __forceinline__ float cimg_w(const uint32_t* row, int k) {   // BF16 element k of a packed row
  const uint32_t w = row[k >> 1];
  return __uint_as_float((k & 1) ? (w & 0xFFFF0000u) : (w << 16));
}

// The learned cut proposal of tree j's step, after the pass totals (every thread of the CTA calls it; it ends with a
// barrier).  A deferred birth draws its cut from the mixture of the head's softmax over [L, U] and the uniform cut
// (Philox tag PROP3), takes the split sums of that cut from the code histogram of the node's rows (in cluster mode
// every CTA pushes its three sums to every CTA, and a cluster barrier precedes their sum), and scales BART's ratio by
// (1 / range) / q(c); a death scales its ratio by
// q(c of the node) * range, the reverse birth's cut probability at the collapsed node.  Results in S.cs: c, logpr,
// sL0, sL1, nL.  Every sum runs in the oracle's order, so the decision is bit-exact.
struct CutOut { double logpr; long long sL0, sL1; int nL, c; };
template <bool CL>
__device__ void cut_stage(const Smem& S, const DBufs& B, const DChain& C, const Prop& P, int j, int it, int cur, int CS,
                          double sigma, bool birth, bool lead, CutOut& out) {
  const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
  CutScr& cs = *S.cs;
  const PropX px = S.px[j];
  const int L = px.L, U = px.U, range = U - L + 1, v = P.v;
  const uint32_t* W = B.cut_smem ? S.cimg : B.cimg;
  if (tid == 0) {
    wait_stats(S, j);
    const long long* tot = (CL ? S.ctot : S.tot) + cur * TOT;
    const unsigned long long* ovb = (CL ? S.covb : S.ovb) + cur * NODES;
    const float2* tcj = S.tc + cur * NODES;
    const long long* s0 = S.s0t + cur * LST;
    const int* cnt = reinterpret_cast<const int*>(s0 + NODES);
    auto s1of = [&](int slot) -> long long {
      const int c = __float_as_int(tcj[slot].y);
      return c < NBS ? tot[c] : (long long)ovb[slot];
    };
    long long S0, S1;
    int n;
    if (birth) { S0 = s0[P.nx]; S1 = s1of(P.nx); n = cnt[P.nx]; }
    else { S0 = s0[P.l] + s0[P.r]; S1 = s1of(P.l) + s1of(P.r); n = cnt[P.l] + cnt[P.r]; }
    cut_features(P.dnx, n, S0, S1, tot[NBS + 3], C.fx_shift, C.rss_shift, sigma, L, U, C.numcut[v], px.uses, v, cs.cx);
  }
  __syncthreads();
  const float* b = reinterpret_cast<const float*>(W + CIMG_B);
  if (tid < CUT_H) {
    const uint32_t* row = W + tid * CIMG_W1S;
    float a = b[tid];
#pragma unroll   // (every weight load issued ahead: the image may be in global memory)
    for (int f = 0; f < CUT_IN; f++) a = __fadd_rn(a, __fmul_rn(cimg_w(row, f), cs.cx[f]));
    cs.h1[tid] = a > 0.0f ? a : 0.0f;
  }
  __syncthreads();
  if (tid < CUT_H) {
    const uint32_t* row = W + CIMG_W2 + tid * CIMG_W2S;
    float a = b[CUT_H + tid];
#pragma unroll
    for (int f = 0; f < CUT_H; f++) a = __fadd_rn(a, __fmul_rn(cimg_w(row, f), cs.h1[f]));
    cs.h2[tid] = a > 0.0f ? a : 0.0f;
  }
  __syncthreads();
  if (tid < CUT_E) {
    const uint32_t* row = W + CIMG_W3 + tid * CIMG_W2S;
    float a = b[2 * CUT_H + tid];
#pragma unroll
    for (int f = 0; f < CUT_H; f++) a = __fadd_rn(a, __fmul_rn(cimg_w(row, f), cs.h2[f]));
    cs.e[tid] = a;
  }
  __syncthreads();
  for (int k = tid; k < range; k += T) {
    const int c = L + k;
    const uint32_t* row = W + CIMG_EMB + c * CIMG_ES;
    float a = b[2 * CUT_H + CUT_E + c];
#pragma unroll
    for (int f = 0; f < CUT_E; f++) a = __fadd_rn(a, __fmul_rn(cimg_w(row, f), cs.e[f]));
    cs.z[c] = a;
  }
  __syncthreads();
  if (warp == 2) {   // the largest logit: lane l takes block l (cuts L + 8l .. L + 8l + 7)
    double zm = -INFINITY;
    for (int k = 8 * lane; k < 8 * lane + 8 && k < range; k++) zm = fmax(zm, (double)cs.z[L + k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) zm = fmax(zm, __shfl_xor_sync(0xffffffffu, zm, o));
    if (lane == 0) cs.zmax = zm;
  }
  __syncthreads();
  for (int k = tid; k < range; k += T) cs.ex[L + k] = fbm::fb_exp((double)cs.z[L + k] - cs.zmax);
  __syncthreads();
  if (warp == 2) {
    const int nb = (range + 7) / 8;
    double bs = 0.0;
    for (int k = 8 * lane; k < 8 * lane + 8 && k < range; k++) bs = bs + cs.ex[L + k];
    if (lane < nb) cs.bs[lane] = bs;
    __syncwarp();
    int c = 0;
    if (lane == 0) {
      double Ssum = 0.0;
      for (int k = 0; k < nb; k++) Ssum = Ssum + cs.bs[k];
      const double mix = B.cmix;
      double pr;
      if (birth) {
        const fbm::U4 x3 = fbm::philox(0u, (uint32_t)j, (uint32_t)it, fbm::TAG_PROP3, C.seed);
        const double umix = fbm::u32d(x3.x), uc = fbm::u32d(x3.y);
        c = U;
        if (umix < mix) {
          const double target = uc * Ssum;
          double Pp = 0.0;
          for (int bk = 0; bk < nb; bk++) {
            const double P1 = Pp + cs.bs[bk];
            if (P1 > target) {
              double run = Pp;
              const int c0 = L + 8 * bk;
              c = c0 + 7 < U ? c0 + 7 : U;
              for (int cc = c0; cc < c0 + 8 && cc <= U; cc++) {
                run = run + cs.ex[cc];
                if (run > target) { c = cc; break; }
              }
              break;
            }
            Pp = P1;
          }
        } else {
          c = L + (int)(uc * range);
          if (c > U) c = U;
        }
        const double q = mix * (cs.ex[c] / Ssum) + (1.0 - mix) * (1.0 / (double)range);
        const double corr = (1.0 / (double)range) / q;
        pr = px.pr4[(c == L ? 1 : 0) + (c == U ? 2 : 0)] * corr;
      } else {
        c = P.c;
        const double q = mix * (cs.ex[c] / Ssum) + (1.0 - mix) * (1.0 / (double)range);
        pr = px.pr4[0] * (q * (double)range);
      }
      cs.c = c;
      cs.logpr = fbm::fb_log(pr);
    }
    c = __shfl_sync(0xffffffffu, c, 0);
    if (birth) {   // split sums of the cut: codes <= c of this CTA's rows of the node
      unsigned long long a0 = 0, a1 = 0;
      int ac = 0;
      for (int k = lane; k <= c; k += 32) { a0 += S.h0[k]; a1 += S.h1[k]; ac += S.hc[k]; }
      const long long t0 = warp_sum64((long long)a0), t1 = warp_sum64((long long)a1);
      const int tc = __reduce_add_sync(0xffffffffu, ac);
      if (lane == 0) {
        if constexpr (CL) {   // every CTA's three sums to every CTA (remote stores), summed after a cluster barrier
          cg::cluster_group cl = cg::this_cluster();
          const int me = (int)cl.block_rank();
          for (int d = 0; d < CS; d++) {
            long long* x = cl.map_shared_rank(S.xcut + 4 * me, d);
            x[0] = t0; x[1] = t1; x[2] = tc;
          }
        } else {
          cs.sL0 = t0; cs.sL1 = t1; cs.nL = tc;
        }
      }
    }
  }
  if constexpr (CL) {
    if (birth) {
      cg::this_cluster().sync();
      if (tid == 0) {
        long long s0 = 0, s1 = 0, sc = 0;
        for (int r = 0; r < CS; r++) { s0 += S.xcut[4 * r]; s1 += S.xcut[4 * r + 1]; sc += S.xcut[4 * r + 2]; }
        cs.sL0 = s0; cs.sL1 = s1; cs.nL = (int)sc;
      }
    }
  }
  __syncthreads();
  out.c = cs.c; out.logpr = cs.logpr; out.sL0 = cs.sL0; out.sL1 = cs.sL1; out.nL = cs.nL;
  if (B.train_cx && lead && birth && tid < CUT_IN) B.cfeat[(C.off_tree + j) * CUT_IN + tid] = cs.cx[tid];
  __syncthreads();
  // the scratch's bin rows back to zero for the next pass, and the histogram for the next birth (only this CTA reads
  // its own histogram)
  for (int k = tid; k < (int)(sizeof(CutScr) / 8); k += T) S.bins[k] = 0;
  if (birth)
    for (int k = tid; k < 256; k += T) { S.h0[k] = 0ull; S.h1[k] = 0ull; S.hc[k] = 0; }
}

// ------------------------------------------------------------------------------------------------ one chain

// Proposals of every tree of sweep it (one thread per tree) with the leaf-mu normals drawn ahead.
template <bool LP, bool MP>
__device__ __forceinline__ void proposals_body(const Smem& S, const DBufs& B, const DChain& C, DTree* trees,
                                               const long long* s0g, int it, bool lead) {
  const int m = C.m;
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    Masks mk;
    float* featj = (LP && B.train_cap > 0 && lead) ? B.feat + (C.off_tree + j) * MLP_IN : nullptr;
    const Prop P = propose<LP, MP>(trees + j, C, B, reinterpret_cast<const int*>(s0g + (long long)j * LST + NODES), j, it,
                               mk, featj, B.feat_valid + (C.off_tree + j), S.px ? S.px + j : nullptr);
    S.prop[j] = P;
    S.masks[j] = mk;
    int k = 0;
    for (unsigned long long cm = P.cand; cm && k < S.zmax; cm &= cm - 1ull, k++) {
      const int sl = __ffsll((long long)cm) - 1;
      S.zall[j * S.zmax + k] = fbm::fb_normal(C.seed, (uint32_t)sl << 8, (uint32_t)j, (uint32_t)it, fbm::TAG_MU);
    }
  }
}
// Out of line for the collecting kernels: the feature calls then save only this function's few live registers, not
// the chain loop's.
__device__ __noinline__ void proposals_collect(const Smem& S, const DBufs& B, const DChain& C, DTree* trees,
                                             const long long* s0g, int it, bool lead) {
  proposals_body<true, true>(S, B, C, trees, s0g, it, lead);
}

// Cluster exchange of the pass totals (buffer cur), push style: every CTA stores its totals into slot [crank] of every
// CTA's xtot / xovb (remote stores do not wait), a cluster barrier publishes them, and each CTA then sums the slots
// in its own shared memory.  The ovb partials (leaves beyond the register bins) are exchanged only when used.
__device__ __forceinline__ void cluster_push(const Smem& S, int cur, int CS, int crank, bool ovf) {
  cg::cluster_group cl = cg::this_cluster();
  const int k = threadIdx.x;
  if (k < TOT) {
    const long long v = S.tot[cur * TOT + k];
    for (int d = 0; d < CS; d++) *cl.map_shared_rank(S.xtot + (cur * CS + crank) * TOT + k, d) = v;
  } else if (ovf && k < TOT + NODES) {
    const unsigned long long v = S.ovb[cur * NODES + k - TOT];
    for (int d = 0; d < CS; d++) *cl.map_shared_rank(S.xovb + (cur * CS + crank) * NODES + k - TOT, d) = v;
  }
}
__device__ __forceinline__ void cluster_sum(const Smem& S, int cur, int CS, bool ovf) {
  const int k = threadIdx.x;
  if (k < TOT) {
    long long t = 0;
    for (int r = 0; r < CS; r++) t += S.xtot[(cur * CS + r) * TOT + k];
    S.ctot[cur * TOT + k] = t;
  } else if (ovf && k < TOT + NODES) {
    unsigned long long t = 0;
    for (int r = 0; r < CS; r++) t += S.xovb[(cur * CS + r) * NODES + k - TOT];
    S.covb[cur * NODES + k - TOT] = t;
  }
}

// Sum over the cluster of one exchanged value (slot k of xch) of every CTA; after a cluster barrier.
__device__ __forceinline__ long long cluster_value(const Smem& S, int k, int CS) {
  cg::cluster_group cl = cg::this_cluster();
  long long t = 0;
  for (int r = 0; r < CS; r++) t += *cl.map_shared_rank(S.xch + k, r);
  return t;
}

// One chain.  With B.cluster = CS > 1 the chain runs on a cluster of CS CTAs: each CTA owns a contiguous slice of the
// rows (groups [g0, g1)) in its shared memory and runs every control step itself on identical inputs (the proposals,
// Metropolis-Hastings, leaf draws and sigma come out bit-identical in every CTA, each on its own copy of the trees);
// only the exact integer pass totals and the end-of-sweep rss cross the cluster, through distributed shared memory,
// once per tree step.  Integer sums do not depend on order, so the results equal the one-CTA run bit for bit.
template <int G, bool CL, int MODE>
__device__ void run_chain(const DBufs& B, int ci, int it0, int it1, const Smem& S) {
  constexpr bool LP = MODE == MODE_COLLECT, MP = MODE != MODE_PLAIN;
  const DChain& C = B.chains[ci];
  const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int RT = T - 32;
  const int n = C.n, m = C.m, n_pad = C.n_pad, ngroups = n_pad / 4;
  const int CS = CL ? B.cluster : 1;
  const int crank = CL ? (int)cg::this_cluster().block_rank() : 0;
  const bool lead = crank == 0;   // writes the chain's outputs
  const int per = (ngroups + CS - 1) / CS;
  const int g0 = min(ngroups, crank * per), g1 = min(ngroups, g0 + per);
  const int ns = 4 * (g1 - g0);   // this CTA's rows (padded)
  const unsigned long long seed = C.seed;
  const double t2 = C.tau * C.tau, a_prior = 1.0 / t2;
  const double sci = pow2(-C.fx_shift), rscale = pow2(C.rss_shift), rsci = pow2(-C.rss_shift);
  const float scale = (float)pow2(C.fx_shift);
  const uint8_t* q = B.q + C.off_q;
  uint8_t* leaf = B.leaf + C.off_leaf;
  const long long tb = C.off_tree * CS + (long long)crank * m;   // this CTA's copy of the chain's trees
  DTree* trees = B.trees + tb;
  long long* s0g = B.s0 + tb * LST;
  float* thg = B.th + tb * NODES;
  double* ywork = B.ywork + C.off_row;
  const float* wg = B.win + C.off_row;
  float* rg = B.rsave + C.off_row + 4 * g0;   // this CTA's rows
  float* wsg = B.wsave + C.off_row + 4 * g0;
  double* tm = B.tm + C.off_row;
  float* r = B.rows_in_smem ? S.r : rg;       // indexed from row 4 * g0
  float* ws = B.rows_in_smem == 1 ? S.ws : wsg;
  Ctl& ctl = *S.ctl;
  DState& st = B.states[ci];
  const bool regs = G > 0 && (g1 - g0) <= G * RT;   // register-held words for this CTA's groups

  // ---------------------------------------------------------------- chain start or resume
  if (tid == 0) {
    if (it0 == 0) { ctl.sigma = C.sigest; ctl.births = ctl.deaths = ctl.caps = ctl.rtcaps = 0; }
    else {
      ctl.sigma = st.sigma; ctl.births = st.births; ctl.deaths = st.deaths; ctl.caps = st.caps;
      ctl.rtcaps = lead ? st.rtcaps : 0;   // latent-z caps are counted per CTA and summed at the end
    }
    ctl.pmode = 0;
    ctl.err = 0;
  }
  for (int k = tid; k < S.binrows * RT; k += T) S.bins[k] = 0;
  __syncthreads();
  for (int li = tid; li < ns; li += T) ws[li] = __fmul_rn(wg[4 * g0 + li], scale);   // exact: power-of-two scaling
  if (it0 == 0) {
    int caps = 0;
    for (int li = tid; li < ns; li += T) {
      const int i = 4 * g0 + li;
      double y = 0.0;
      if (i < n) {
        if (C.probit)
          y = B.ybin[C.off_row + i] == 0 ? -fbm::fb_rtnorm(seed, (uint32_t)i, fbm::INIT_SWEEP, 0.0, C.offset, &caps)
                                         : fbm::fb_rtnorm(seed, (uint32_t)i, fbm::INIT_SWEEP, 0.0, -C.offset, &caps);
        else y = B.yin[C.off_row + i];
      }
      ywork[i] = y;
      r[li] = (float)y;
      tm[i] = 0.0;
    }
    if (caps) atomicAdd(&ctl.rtcaps, caps);
    const int sg = g1 - g0;   // this CTA's groups of every tree's leaf ids
    for (long long k = tid; k < (long long)m * sg; k += T)
      *reinterpret_cast<uint32_t*>(leaf + (k / sg) * n_pad + 4 * (g0 + k % sg)) = 0u;
    for (int k = tid; k < m * NODES; k += T) S.th[k] = 0.0f;
    long long sw = 0;
    for (int li = tid; li < ns; li += T)
      if (4 * g0 + li < n) sw += __float2ll_rn(__fmul_rn(wg[4 * g0 + li], scale));
    long long swt = block_sum64(sw, S.red);
    if (CL) {   // sum of w over the whole chain
      if (tid == 0) S.xch[4 + 2] = swt;
      cg::this_cluster().sync();
      swt = cluster_value(S, 4 + 2, CS);
    }
    // root-only trees: every word zero except ngv[0] (byte 384), used (byte 448) and leaf (byte 456)
    constexpr int TWORDS = (int)(sizeof(DTree) / 4);
    for (int k = tid; k < m * TWORDS; k += T) {
      const int j = k / TWORDS, byte0 = (k % TWORDS) * 4;
      uint32_t val = 0u;
      if (byte0 == 6 * NODES) val = (uint32_t)C.root_ngv;
      else if (byte0 == 7 * NODES || byte0 == 7 * NODES + 8) val = 1u;
      reinterpret_cast<uint32_t*>(trees + j)[k % TWORDS] = val;
    }
    for (int k = tid; k < m * LST; k += T) {   // root: all rows; counts are ints in words 64..95
      const int w = k % LST;
      long long v = 0;
      if (w == 0) v = swt;
      else if (w == NODES) v = (long long)(unsigned)n;   // cnt[0] = n (little endian: low half of word 64)
      s0g[k] = v;
    }
    fence_proxy_async_global();   // the bulk copies of the first sweep see these statistics
  } else {
    if (B.rows_in_smem)
      for (int li = tid; li < ns; li += T) S.r[li] = rg[li];
    for (int k = tid; k < m * NODES; k += T) S.th[k] = thg[k];
  }
  __syncthreads();

  // words of the row thread's groups (register path)
  uint32_t lcr[G > 0 ? G : 1], qcr[G > 0 ? G : 1], nlc[G > 0 ? G : 1], nqc[G > 0 ? G : 1];

  for (int it = it0; it < it1; it++) {
    // a bounded wait gave up: a chain on one CTA stops here (its state says so); the CTAs of a cluster keep their
    // barriers in step and finish with the error recorded
    if (!CL && ctl.err) break;
    const double inv_s2 = 1.0 / (ctl.sigma * ctl.sigma);
    // ---------------------------------------------------------------- learned model, one warp per tree
    if (MP && B.mvar) {
      // the weights in shared memory: in the pass bins, free at sweep start when they are large enough (the leaf
      // rows, which the pass accumulates into, are zeroed again afterwards), else behind the layout, else global
      const bool in_bins = bins_hold_model(T);
      const uint32_t* W = B.model_smem ? S.mimg : B.mimg;
      if (in_bins) {
        for (int k = tid; k < MIMG_WORDS / 4; k += T)
          reinterpret_cast<uint4*>(S.bins)[k] = __ldg(reinterpret_cast<const uint4*>(B.mimg) + k);
        __syncthreads();
        W = reinterpret_cast<const uint32_t*>(S.bins);
      }
      model_phase(B, C, trees, s0g, W, it, crank, CS);
      if (in_bins) {
        __syncthreads();
        for (int k = tid; k < (S.px ? BIN_ROWS : NBS) * RT; k += T) S.bins[k] = 0;
      }
      if constexpr (CL) { __threadfence(); cg::this_cluster().sync(); }   // every CTA's share, in global memory
      else __syncthreads();
    }
    // ---------------------------------------------------------------- proposals, one thread per tree
    if constexpr (LP) proposals_collect(S, B, C, trees, s0g, it, lead);
    else proposals_body<false, MP>(S, B, C, trees, s0g, it, lead);
    for (int k = tid; k < 2 * TOT; k += T) S.tot[k] = 0;
    for (int k = tid; k < 2 * NODES; k += T) S.ovb[k] = 0ull;
    __syncthreads();
    if (warp == 0) {
      fetch_stats(S, s0g, 0, lane);
      if (m > 1) fetch_stats(S, s0g, 1, lane);
      build_tc_slot(S, 0, lane);
      build_tc_slot(S, 0, lane + 32);
      if (lane == 0) ctl.pmode = 0;
    }
    __syncthreads();
    // the first pass of a sweep loads its words itself: the held words are dead until here (keeps them out of the
    // registers live across the proposal step's calls)
#pragma unroll
    for (int k = 0; k < (G > 0 ? G : 1); k++) lcr[k] = qcr[k] = nlc[k] = nqc[k] = 0u;
    // ---------------------------------------------------------------- trees
    for (int j = 0; j < m; j++) {
      Prop P = S.prop[j];
      const int cur = j & 1;
      // learned cut proposal: a deferred birth, or a death whose reverse birth's cut is scored; collecting launches
      // also sum the squared residuals of a birth node for its cut example
      const bool cutb = MP && (P.flags & PROP_DEFER);
      const bool cutd = MP && B.cimg && P.mode == 2;
      const bool csq = LP && B.train_cx && P.mode == 1 && !cutb;
      const bool sqon = cutb || cutd || csq;
      const int cmode = cutb ? 0 : P.mode;
      CutOut co{0.0, 0, 0, 0, 0};
      // ------------------------------------------------------------ phase A: row pass | control prefetch
      if (warp > 0) {
        PassU U;
        U.leaf_prev = j > 0 ? leaf + (long long)(j - 1) * n_pad : nullptr;
        U.leaf_cur = leaf + (long long)j * n_pad;
        U.qprev = q + (long long)ctl.pv * n_pad;
        U.qcur = q + (long long)P.v * n_pad;
        if (j + 1 < m) {
          const Prop Pn = S.prop[j + 1];
          U.leaf_next = leaf + (long long)(j + 1) * n_pad;
          U.qnext = Pn.mode == 1 ? q + (long long)Pn.v * n_pad : nullptr;
        } else {
          U.leaf_next = nullptr;
          U.qnext = nullptr;
        }
        U.r = r; U.ws = ws; U.D = S.D; U.tc = S.tc + cur * NODES; U.bins = S.bins; U.ovb = S.ovb + cur * NODES;
        U.tot = S.tot + cur * TOT;
        U.DL = ctl.DL; U.DR = ctl.DR;
        U.n = n; U.g0 = g0; U.g1 = g1; U.rt = tid - 32; U.RT = RT; U.nleaf = ctl.nleaf[cur];
        U.apply = j > 0; U.pmode = ctl.pmode; U.pnx = ctl.pnx; U.pc = ctl.pc; U.pL = ctl.pL; U.pR = ctl.pR;
        U.pl = ctl.pl; U.pr = ctl.pr;
        U.cmode = cmode; U.cnx = P.nx; U.cc = P.c;
        U.h0 = S.h0; U.h1 = S.h1; U.hc = S.hc;
        U.sqs = (float)pow2(C.rss_shift - C.fx_shift);
        U.xhist = cutb ? 1 : 0;
        U.sqa = (cutb || csq) ? P.nx : cutd ? P.l : -1;
        U.sqb = cutd ? P.r : U.sqa;
        // the pass with the cut proposal's extras (squared residuals, code histogram) only in the steps that use
        // them: a step of a chain without a cut head runs the plain pass
        if constexpr (G > 0) {
          if (regs) {
            if (MP && sqon) pass_rows_regs<G, MP>(U, j == 0, lcr, qcr, nlc, nqc);
            else pass_rows_regs<G, false>(U, j == 0, lcr, qcr, nlc, nqc);
          } else {
            if (MP && sqon) pass_rows_stream<MP>(U);
            else pass_rows_stream<false>(U);
          }
        } else {
          if (MP && sqon) pass_rows_stream<MP>(U);
          else pass_rows_stream<false>(U);
        }
      } else {
        // control warp: commit tree j-1, fetch tree j+1 into the freed buffer, draw the normals of every slot that
        // can be a leaf of tree j after its move (current leaves, the two slots a birth would take, the node a death
        // would restore)
        if (j > 0) commit_tree<LP>(S, C, B, trees, s0g, j - 1, lane, lead);
        if (j + 1 < m && j > 0) fetch_stats(S, s0g, j + 1, lane);
        const unsigned long long cand = P.cand;
        if (__popcll(cand) > S.zmax)
          for (int s = lane; s < NODES; s += 32)
            if (((cand >> s) & 1ull) && __popcll(cand & ((1ull << s) - 1ull)) >= S.zmax)
              S.z[s] = fbm::fb_normal(seed, (uint32_t)s << 8, (uint32_t)j, (uint32_t)it, fbm::TAG_MU);
      }
      __syncthreads();
      reduce_totals(S.bins, RT, ctl.nleaf[cur], cmode, S.tot + cur * TOT, sqon);
      if (CL) {   // the chain's totals: every CTA's partial totals, pushed through distributed shared memory
        const bool ovf = ctl.nleaf[cur] > NBS;
        __syncthreads();
        cluster_push(S, cur, CS, crank, ovf);
        cg::this_cluster().sync();
        cluster_sum(S, cur, CS, ovf);
      }
      __syncthreads();
      if constexpr (MP) {
        if (cutb || cutd) {   // the learned cut (all threads; ends with a barrier)
          cut_stage<CL>(S, B, C, P, j, it, cur, CS, ctl.sigma, cutb, lead, co);
          if (cutb) P.c = (uint8_t)co.c;
          P.logpr = co.logpr;
        }
      }
      // ------------------------------------------------------------ phase B: MH and leaf draws, one thread per slot
      // With at least 3 warps, warp 2 evaluates Metropolis-Hastings while warps 0-1 draw every slot's leaf value for
      // the outcome in which that slot is a leaf (a slot is a leaf with the same statistics in both outcomes, or in
      // one outcome only), so the two overlap; a named barrier of the 3 warps then hands over the decision.
      const bool sep = T >= 96;
      if (tid < (sep ? NODES + 32 : NODES)) {
        const int s = tid;
        wait_stats(S, j);   // tree j's statistics (copy issued one step earlier, normally landed long ago)
        const Masks mk = S.masks[j];
        const long long* tot = (CL ? S.ctot : S.tot) + cur * TOT;
        const unsigned long long* ovb = (CL ? S.covb : S.ovb) + cur * NODES;
        const float2* tcj = S.tc + cur * NODES;
        const long long* s0 = S.s0t + cur * LST;
        const int* cnt = reinterpret_cast<const int*>(s0 + NODES);
        float* thj = S.th + j * NODES;
        auto s1of = [&](int slot) -> long long {
          const int c = __float_as_int(tcj[slot].y);
          return c < NBS ? tot[c] : (long long)ovb[slot];
        };
        // birth split: the left child's sums come from the pass, the right child's from the node's totals
        long long sL0 = 0, sL1 = 0, sR0 = 0, sR1 = 0;
        int nL = 0, nR = 0;
        if (P.mode == 1) {
          if (cutb) { sL0 = co.sL0; sL1 = co.sL1; nL = co.nL; }
          else { sL0 = tot[NBS + 0]; sL1 = tot[NBS + 1]; nL = (int)tot[NBS + 2]; }
          sR0 = s0[P.nx] - sL0; sR1 = s1of(P.nx) - sL1; nR = cnt[P.nx] - nL;
        }
        const bool eval = (P.mode == 1 && nL >= 5 && nR >= 5) || P.mode == 2;
        bool accept = false;
        if (!sep || warp == 2) {
          if (eval) {
            double bl, Ml, br, Mr;
            if (P.mode == 1) {
              bl = (double)sL0 * sci * inv_s2; Ml = (double)sL1 * sci * inv_s2;
              br = (double)sR0 * sci * inv_s2; Mr = (double)sR1 * sci * inv_s2;
            } else {
              bl = (double)s0[P.l] * sci * inv_s2; Ml = (double)s1of(P.l) * sci * inv_s2;
              br = (double)s0[P.r] * sci * inv_s2; Mr = (double)s1of(P.r) * sci * inv_s2;
            }
            // lanes 0..2 evaluate the three log marginal likelihoods at one call site: birth (l, r, l+r),
            // death (l+r, l, r), in the order the ratio adds them
            const int which = P.mode == 1 ? lane : (lane == 0 ? 2 : lane - 1);
            const double hb = which == 0 ? bl : (which == 1 ? br : bl + br);
            const double hM = which == 0 ? Ml : (which == 1 ? Mr : Ml + Mr);
            double hv = 0.0;
            if (lane < 3) hv = lh(hb, hM, t2);
            const double h0 = __shfl_sync(0xffffffffu, hv, 0), h1 = __shfl_sync(0xffffffffu, hv, 1),
                         h2 = __shfl_sync(0xffffffffu, hv, 2);
            double lalpha = (P.mode == 1) ? P.logpr + h0 + h1 - h2 : P.logpr + h0 - h1 - h2;
            if (lalpha > 0) lalpha = 0;
            accept = P.lu < lalpha;
          }
          if (sep && lane == 0) ctl.accept = accept ? 1 : 0;
        }
        // slots a birth would take (lowest free slots), decided before the outcome is known
        int Lc = -1, Rc = -1;
        if (P.mode == 1) { Lc = first_free(mk.used, -1); Rc = Lc >= 0 ? first_free(mk.used, Lc) : -1; }
        const unsigned long long lm0 = mk.used & mk.leaf;
        float nws = 0.0f;   // this slot's leaf value in the outcome where it is a leaf
        if (s < NODES) {
          bool has = true;
          long long S0s = 0, S1s = 0;
          if ((lm0 >> s) & 1ull) { S0s = s0[s]; S1s = s1of(s); }
          else if (eval && P.mode == 1 && Lc >= 0 && Rc >= 0 && s == Lc) { S0s = sL0; S1s = sL1; }
          else if (eval && P.mode == 1 && Lc >= 0 && Rc >= 0 && s == Rc) { S0s = sR0; S1s = sR1; }
          else if (eval && P.mode == 2 && s == P.nx) { S0s = s0[P.l] + s0[P.r]; S1s = s1of(P.l) + s1of(P.r); }
          else has = false;
          if (has) {
            const double b = (double)S0s * sci * inv_s2, M = (double)S1s * sci * inv_s2;
            const int zi = __popcll(P.cand & ((1ull << s) - 1ull));
            const double z = zi < S.zmax ? S.zall[j * S.zmax + zi] : S.z[s];
            nws = (float)(M / (a_prior + b) + z / sqrt(a_prior + b));
          }
        }
        if (s < NODES) {   // the next tree's table (its accumulators start at zero) does not depend on this decision
          if (j + 1 < m) build_tc_slot(S, j + 1, s);
          S.ovb[(cur ^ 1) * NODES + s] = 0ull;
        }
        if (sep) {
          asm volatile("bar.sync 1, 96;" ::: "memory");   // warps 0-2: the decision is published
          accept = ctl.accept != 0;
        }
        if (s < NODES) {
          int nmode = 0, L = 0, R = 0;
          bool cap = false;
          unsigned long long used = mk.used, leafm = mk.leaf;
          if (accept && P.mode == 1) {
            L = Lc; R = Rc;
            if (L < 0 || R < 0) { cap = true; L = R = 0; }
            else {
              nmode = 1;
              used |= (1ull << L) | (1ull << R);
              leafm = (leafm & ~(1ull << P.nx)) | (1ull << L) | (1ull << R);
            }
          } else if (accept && P.mode == 2) {
            nmode = 2;
            used &= ~((1ull << P.l) | (1ull << P.r));
            leafm = (leafm & ~((1ull << P.l) | (1ull << P.r))) | (1ull << P.nx);
          }
          // this thread's slot: new leaf value (DRMU) and apply delta
          const unsigned long long lm1 = used & leafm;
          const float old = thj[s];
          float nw = old;
          if ((lm1 >> s) & 1ull) {
            nw = nws;
            thj[s] = nw;
          }
          // leaf values of slots that stop being leaves do not change, so the reads below see old values
          if (!(nmode == 2 && (s == P.l || s == P.r))) S.D[s] = __fsub_rn(nw, old);
          if (nmode == 2 && s == P.nx) { S.D[P.l] = __fsub_rn(nw, thj[P.l]); S.D[P.r] = __fsub_rn(nw, thj[P.r]); }
          if (nmode == 1 && s == L) ctl.DL = __fsub_rn(nw, thj[P.nx]);
          if (nmode == 1 && s == R) ctl.DR = __fsub_rn(nw, thj[P.nx]);
          if (s == 0) {
            if constexpr (LP) {   // the cut example of an accepted birth (features of the node before the split)
              if (B.train_cx && lead && nmode == 1) {
                const PropX px = S.px[j];
                float* xf = B.cfeat + (C.off_tree + j) * CUT_IN;
                if (!cutb) {   // (a deferred birth's features were written by its cut stage)
                  float xl[CUT_IN];
                  cut_features(P.dnx, cnt[P.nx], s0[P.nx], s1of(P.nx), tot[NBS + 3], C.fx_shift, C.rss_shift,
                               ctl.sigma, px.L, px.U, C.numcut[P.v], px.uses, P.v, xl);
                  for (int k = 0; k < CUT_IN; k++) xf[k] = xl[k];
                }
                int* ci3 = B.cinfo + (C.off_tree + j) * 3;
                ci3[0] = P.c; ci3[1] = px.L; ci3[2] = px.U;
              }
            }
            if (cap) ctl.caps++;
            if (nmode == 1) ctl.births++;
            if (nmode == 2) ctl.deaths++;
            ctl.pmode = nmode; ctl.pnx = P.nx; ctl.pv = P.v; ctl.pc = P.c; ctl.pL = L; ctl.pR = R;
            ctl.pl = P.l; ctl.pr = P.r; ctl.sL0 = sL0; ctl.sR0 = sR0; ctl.nL = nL; ctl.nR = nR; ctl.pd = P.dnx;
            if (nmode == 2) { ctl.sL0 = s0[P.l] + s0[P.r]; ctl.nL = cnt[P.l] + cnt[P.r]; }   // the merged node
            ctl.used = used; ctl.leaf = leafm;
          }
        }
      }
      __syncthreads();
    }
    // ---------------------------------------------------------------- end of sweep
    if (warp == 0) {
      commit_tree<LP>(S, C, B, trees, s0g, m - 1, lane, lead);
      // the next sweep's bulk copies see every statistic this sweep's commits stored: each storing lane orders its
      // own generic-proxy stores before the async proxy once, here, and the barrier below orders them before lane 0's
      // copies (no statistic is fetched again within the sweep that stores it)
      fence_proxy_async_global();
    }
    __syncthreads();
    const bool keep = it >= C.nskip;
    const int dr = it - C.nskip;
    int caps = 0;
    long long rssfx = 0;
    {
      const int pmode = ctl.pmode;
      const uint32_t pnx4 = bcast4(ctl.pnx), pc4 = bcast4(ctl.pc), pL4 = bcast4(ctl.pL), pR4 = bcast4(ctl.pR),
                     pl4 = bcast4(ctl.pl), pr4 = bcast4(ctl.pr);
      uint8_t* lp = leaf + (long long)(m - 1) * n_pad;
      const uint8_t* qp = q + (long long)ctl.pv * n_pad;
      for (int g = g0 + tid; g < g1; g += T) {
        const uint32_t lp4 = ld_u32(lp + 4 * g);
        uint32_t lpn = lp4;
        if (pmode == 1) {
          const uint32_t mv = __vcmpeq4(lp4, pnx4), side = __vcmpleu4(__ldg(reinterpret_cast<const uint32_t*>(qp + 4 * g)), pc4);
          lpn = (lp4 & ~mv) | (mv & ((side & pL4) | (~side & pR4)));
        } else if (pmode == 2) {
          const uint32_t mv = __vcmpeq4(lp4, pl4) | __vcmpeq4(lp4, pr4);
          lpn = (lp4 & ~mv) | (mv & pnx4);
        }
        if (lpn != lp4) *reinterpret_cast<uint32_t*>(lp + 4 * g) = lpn;
        // FP64 refresh: f = sum over trees, in tree order, of the row's leaf value
        double f0 = 0.0, f1 = 0.0, f2 = 0.0, f3 = 0.0;
        int jj = 0;
        for (; jj + 16 <= m - 1; jj += 16) {
          uint32_t l4[16];
#pragma unroll
          for (int u = 0; u < 16; u++) l4[u] = ld_u32(leaf + (long long)(jj + u) * n_pad + 4 * g);
#pragma unroll
          for (int u = 0; u < 16; u++) {
            const float* thj = S.th + (jj + u) * NODES;
            f0 += (double)thj[l4[u] & 255u]; f1 += (double)thj[(l4[u] >> 8) & 255u];
            f2 += (double)thj[(l4[u] >> 16) & 255u]; f3 += (double)thj[l4[u] >> 24];
          }
        }
        for (; jj < m; jj++) {
          const uint32_t l4 = jj == m - 1 ? lpn : ld_u32(leaf + (long long)jj * n_pad + 4 * g);
          const float* thj = S.th + jj * NODES;
          f0 += (double)thj[l4 & 255u]; f1 += (double)thj[(l4 >> 8) & 255u];
          f2 += (double)thj[(l4 >> 16) & 255u]; f3 += (double)thj[l4 >> 24];
        }
        const double fe[4] = {f0, f1, f2, f3};
        const float4 w4 = reinterpret_cast<const float4*>(ws)[g - g0];
        const float wwe[4] = {w4.x, w4.y, w4.z, w4.w};
        float rn[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int i = 4 * g + e;
          rn[e] = 0.0f;
          if (i < n) {
            const double f = fe[e];
            double y = ywork[i];
            if (C.probit) {
              y = B.ybin[C.off_row + i] == 0 ? -fbm::fb_rtnorm(seed, (uint32_t)i, (uint32_t)it, -f, C.offset, &caps)
                                             : fbm::fb_rtnorm(seed, (uint32_t)i, (uint32_t)it, f, -C.offset, &caps);
              ywork[i] = y;
            }
            const double ee = y - f;
            rn[e] = (float)ee;
            if (!C.probit) {
              const double we = ((double)wwe[e] * sci) * ee;
              rssfx += __double2ll_rn(we * ee * rscale);
            }
            if (keep) {
              tm[i] += f;
              B.yhat_out[C.off_yhat + (long long)dr * n + i] = f;
            }
          }
        }
        reinterpret_cast<float4*>(r)[g - g0] = make_float4(rn[0], rn[1], rn[2], rn[3]);
      }
    }
    if (caps) atomicAdd(&ctl.rtcaps, caps);
    long long rss = C.probit ? 0 : block_sum64(rssfx, S.red);
    if (CL && !C.probit) {   // the chain's rss: every CTA's partial sum
      if (tid == 0) S.xch[(it & 1) * 4] = rss;
      cg::this_cluster().sync();
      if (tid == 0) rss = cluster_value(S, (it & 1) * 4, CS);
    }
    if (tid == 0) {
      if (!C.probit) {
        const double rssd = (double)rss * rsci;
        ctl.sigma = sqrt((C.nu * C.lambda + rssd) / (2.0 * fbm::fb_gamma(seed, (uint32_t)it, ((double)n + C.nu) / 2.0)));
      }
      if (lead) B.sigma_out[C.off_sigma + it] = ctl.sigma;
      ctl.pmode = 0;
    }
    if (keep && lead) {   // kept draw: packed nodes (src/bart_kernel.cpp:559-571)
      unsigned long long* out = B.trees_out + C.off_tout + (long long)dr * m * NODES;
      for (int k = tid; k < m * NODES; k += T) {
        const int j = k / NODES, s = k % NODES;
        const DTree* t = trees + j;
        const bool used = (t->used >> s) & 1ull;
        const uint32_t thu = __float_as_uint(S.th[k]);
        out[k] = (unsigned long long)(used ? (unsigned)t->v[s] : 255u) | ((unsigned long long)t->c[s] << 8) |
                 ((unsigned long long)t->l[s] << 16) | ((unsigned long long)t->r[s] << 24) |
                 ((unsigned long long)thu << 32);
      }
    }
    __syncthreads();
  }
  // ---------------------------------------------------------------- save state
  for (int k = tid; k < m * NODES; k += T) thg[k] = S.th[k];
  if (B.rows_in_smem)
    for (int li = tid; li < ns; li += T) rg[li] = S.r[li];
  int rtcaps = ctl.rtcaps;
  if (CL) {   // latent-z caps of the whole chain
    __syncthreads();
    if (tid == 0) S.xch[4 + 3] = ctl.rtcaps;
    cg::this_cluster().sync();
    if (tid == 0) rtcaps = (int)cluster_value(S, 4 + 3, CS);
  }
  if (tid == 0 && lead) {
    st.sigma = ctl.sigma; st.births = ctl.births; st.deaths = ctl.deaths; st.caps = ctl.caps; st.rtcaps = rtcaps;
    st.it_done = it1;
    st.status = (it0 == 0 ? 0 : st.status) | ctl.err;
  }
  __syncthreads();
  if (CL) cg::this_cluster().sync();   // no CTA reuses or leaves its shared memory while others read it
}

// G: groups of 4 rows held in registers per row thread (0: streamed); CL: a cluster of CTAs per chain; MODE: plain,
// with the learned proposal's model phase, or with training-example collection (and the model phase).  Each feature
// lives in its own variant: compiled into the plain kernels, its code would cost them registers.
template <int G, bool CL, int MODE>
__global__ void __launch_bounds__(MAX_THREADS, 1) sampler_kernel(DBufs B, int it0, int it1) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int cutl = (MODE != MODE_PLAIN && (B.cimg || B.train_cap > 0)) ? 1 : 0;   // the cut layout
  const Smem S = carve(smem, blockDim.x, B.m_max, B.n_pad_max, B.rows_in_smem, B.cluster, cutl,
                       B.mvar && B.model_smem);
  if (threadIdx.x == 0) {   // the leaf-statistics buffers' mbarriers, once per launch
    mbar_init(S.bar, 1);
    mbar_init(S.bar + 1, 1);
    S.ctl->fetches[0] = S.ctl->fetches[1] = 0u;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if constexpr (MODE != MODE_PLAIN) {   // the cut head's weights, once per launch
    if (B.cimg && B.cut_smem) {
      for (int k = threadIdx.x; k < CIMG_WORDS / 4; k += blockDim.x)
        reinterpret_cast<uint4*>(S.cimg)[k] = __ldg(reinterpret_cast<const uint4*>(B.cimg) + k);
      __syncthreads();
    }
  }
  if constexpr (MODE != MODE_PLAIN) {   // the proposal model's weights, once per launch
    if (B.mvar && B.model_smem && !bins_hold_model(blockDim.x)) {
      for (int k = threadIdx.x; k < MIMG_WORDS / 4; k += blockDim.x)
        reinterpret_cast<uint4*>(S.mimg)[k] = __ldg(reinterpret_cast<const uint4*>(B.mimg) + k);
      __syncthreads();
    }
  }
  if constexpr (CL) {   // one chain per cluster at a time, in the host's order; every CTA of a cluster agrees
    const int ncl = gridDim.x / B.cluster, cid = blockIdx.x / B.cluster;
    for (int qi = cid; qi < B.nchains; qi += ncl) run_chain<G, CL, MODE>(B, B.order[qi], it0, it1, S);
  } else {
    for (;;) {
      if (threadIdx.x == 0) S.ctl->chain = atomicAdd(B.queue, 1);
      __syncthreads();
      const int qi = S.ctl->chain;
      __syncthreads();
      if (qi >= B.nchains) break;
      run_chain<G, CL, MODE>(B, B.order[qi], it0, it1, S);
    }
  }
}

using KernelFn = void (*)(DBufs, int, int);
template <bool CL, int MODE>
static KernelFn kernel_g(int gmax) {
  switch (gmax) {
    case 1: return sampler_kernel<1, CL, MODE>;
    case 2: return sampler_kernel<2, CL, MODE>;
    case 3: return sampler_kernel<3, CL, MODE>;
    case 4: return sampler_kernel<4, CL, MODE>;
    case 6: return sampler_kernel<6, CL, MODE>;
    case 8: return sampler_kernel<8, CL, MODE>;
    default: return sampler_kernel<0, CL, MODE>;
  }
}
// Collecting runs (training data for the learned proposal, not timed work) take fewer register variants: 3 groups
// serve 1..3, 6 serve 4..6, larger slices stream.
template <bool CL>
static KernelFn kernel_collect(int gmax) {
  return (gmax >= 1 && gmax <= 3) ? sampler_kernel<3, CL, MODE_COLLECT>
       : (gmax == 4 || gmax == 6) ? sampler_kernel<6, CL, MODE_COLLECT> : sampler_kernel<0, CL, MODE_COLLECT>;
}
static KernelFn kernel_for(int gmax, bool cluster, int mode) {
  if (cluster)
    return mode == MODE_COLLECT ? kernel_collect<true>(gmax)
         : mode == MODE_MODEL ? kernel_g<true, MODE_MODEL>(gmax) : kernel_g<true, MODE_PLAIN>(gmax);
  return mode == MODE_COLLECT ? kernel_collect<false>(gmax)
       : mode == MODE_MODEL ? kernel_g<false, MODE_MODEL>(gmax) : kernel_g<false, MODE_PLAIN>(gmax);
}

int sampler_gmax(int threads, int n_pad_max) {
  const int RT = threads - 32;
  const int g = (n_pad_max / 4 + RT - 1) / RT;
  return g <= 1 ? 1 : g <= 2 ? 2 : g <= 3 ? 3 : g <= 4 ? 4 : g <= 6 ? 6 : g <= 8 ? 8 : 0;
}

bool sampler_bins_hold_model(int threads) { return bins_hold_model(threads); }

size_t sampler_smem_bytes(int threads, int m_max, int n_pad_max, int rows_in_smem, int cluster, int cut) {
  size_t off[NOFF];
  return smem_layout(threads, m_max, n_pad_max, rows_in_smem, cluster, off, cut);
}

int sampler_max_grid(int threads, size_t smem, int device, int gmax, int cluster) {
  // every variant needs the same shared memory; residency is the same for all
  const KernelFn k = kernel_for(gmax, cluster > 1, MODE_COLLECT);
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  // clusters of 9..16 CTAs are beyond the portable size: allowed per kernel
  if (cluster > 8 && cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
  if (cluster <= 1) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem) != cudaSuccess) return 0;
    return per_sm * nsm;
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(cluster * ((nsm + cluster - 1) / cluster), 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int ncl = 0;
  if (cudaOccupancyMaxActiveClusters(&ncl, k, &cfg) != cudaSuccess) { cudaGetLastError(); return 0; }
  return ncl * cluster;
}

int launch_sampler(const DBufs& b, int it0, int it1, int threads, int grid, size_t smem, int gmax, int cluster,
                   void* stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int mode = b.train_cap > 0 ? MODE_COLLECT : (b.mvar || b.cimg) ? MODE_MODEL : MODE_PLAIN;
  const KernelFn k = kernel_for(gmax, cluster > 1, mode);
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return -1;
  if (cluster > 8 && cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    return -1;
  if (cudaMemsetAsync(b.queue, 0, sizeof(int), s) != cudaSuccess) return -1;
  if (cluster <= 1) {
    k<<<grid, threads, smem, s>>>(b, it0, it1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cluster; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(grid, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, b, it0, it1) == cudaSuccess ? 0 : -1;
}

// ------------------------------------------------------------------------------------------------ diagnostics
// One pass on explicit state, run by the same pass code as the sampler (streaming form): warp 0 builds the tables,
// warps 1.. stream the rows.
__global__ void __launch_bounds__(MAX_THREADS, 1) debug_pass_kernel(DPassArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x, T = blockDim.x, RT = T - 32, lane = tid & 31;
  const int rows_smem = a.rows_in_smem;
  unsigned char* p = smem;
  float* r = rows_smem ? reinterpret_cast<float*>(p) : a.r;
  float* ws = rows_smem ? reinterpret_cast<float*>(p) + a.n_pad : a.wscratch;
  p += rows_smem ? (size_t)a.n_pad * 8 : 0;
  float* D = reinterpret_cast<float*>(p); p += NODES * 4;
  float2* tc = reinterpret_cast<float2*>(p); p += NODES * 8;
  long long* bins = reinterpret_cast<long long*>(p); p += (size_t)(NBS + NSPLIT) * RT * 8;
  long long* tot = reinterpret_cast<long long*>(p); p += TOT * 8;
  unsigned long long* ovb = reinterpret_cast<unsigned long long*>(p); p += NODES * 8;
  float* dlr = reinterpret_cast<float*>(p); p += 16;
  unsigned long long* nodesum = reinterpret_cast<unsigned long long*>(p);   // sum fx(w), row count of the birth node
  const float scale = (float)pow2(a.fx_shift);
  for (int i = tid; i < a.n_pad; i += T) {
    if (rows_smem) r[i] = a.r[i];
    ws[i] = __fmul_rn(a.w[i], scale);
  }
  for (int k = tid; k < (NBS + NSPLIT) * RT; k += T) bins[k] = 0;
  for (int s = tid; s < NODES; s += T) ovb[s] = 0;
  if (tid < TOT) tot[tid] = 0;
  if (tid < 2) nodesum[tid] = 0;
  if (tid < 32) {
    const unsigned long long lm = a.leafmask;
    for (int s = lane; s < NODES; s += 32) {
      const int ci = ((lm >> s) & 1ull) ? __popcll(lm & ((1ull << s) - 1ull)) : 255;
      tc[s] = make_float2(a.thc[s], __int_as_float(ci));
      D[s] = __fsub_rn(a.thn[s], a.tho[s]);
    }
    __syncwarp();
    if (lane == 0) {
      dlr[0] = dlr[1] = 0.0f;
      if (a.pmode == 1) { dlr[0] = __fsub_rn(a.thn[a.pL], a.tho[a.pnx]); dlr[1] = __fsub_rn(a.thn[a.pR], a.tho[a.pnx]); }
      else if (a.pmode == 2) { D[a.pl] = __fsub_rn(a.thn[a.pnx], a.tho[a.pl]); D[a.pr] = __fsub_rn(a.thn[a.pnx], a.tho[a.pr]); }
    }
  }
  __syncthreads();
  const int nleaf = __popcll(a.leafmask);
  if (tid >= 32) {
    PassU U;
    U.leaf_prev = a.leaf_prev; U.leaf_cur = a.leaf_cur; U.qprev = a.qprev; U.qcur = a.qcur;
    U.leaf_next = nullptr; U.qnext = nullptr;
    U.r = r; U.ws = ws; U.D = D; U.tc = tc; U.bins = bins; U.ovb = ovb; U.tot = tot;
    U.DL = dlr[0]; U.DR = dlr[1];
    U.n = a.n; U.g0 = 0; U.g1 = a.n_pad / 4; U.rt = tid - 32; U.RT = RT; U.nleaf = nleaf;
    U.apply = a.apply; U.pmode = a.pmode; U.pnx = a.pnx; U.pc = a.pc; U.pL = a.pL; U.pR = a.pR; U.pl = a.pl; U.pr = a.pr;
    U.cmode = a.stats ? a.cmode : 0; U.cnx = a.cnx; U.cc = a.cc;
    U.h0 = U.h1 = nullptr; U.hc = nullptr; U.sqs = 0.0f; U.xhist = 0; U.sqa = U.sqb = -1;
    pass_rows_stream<false>(U);
  }
  __syncthreads();
  reduce_totals(bins, RT, nleaf, a.stats ? a.cmode : 0, tot);
  __syncthreads();
  for (int s = tid; s < NODES; s += T) {
    long long v = 0;
    if ((a.leafmask >> s) & 1ull) {
      const int ci = __float_as_int(tc[s].y);
      v = ci < NBS ? tot[ci] : (long long)ovb[s];
    }
    a.out[s] = v;
  }
  // The sampler keeps each leaf's sum fx(w) and row count with its tree; here they are counted directly, and the
  // right child's statistics follow from them as in the sampler.
  const bool sp = a.stats && a.cmode == 1;
  if (sp) {
    long long s0 = 0, c = 0;
    for (int i = tid; i < a.n; i += T)
      if (a.leaf_cur[i] == a.cnx) { s0 += __float2ll_rn(ws[i]); c++; }
    atomicAdd(&nodesum[0], (unsigned long long)s0);
    atomicAdd(&nodesum[1], (unsigned long long)c);
  }
  __syncthreads();
  if (tid == 0) {
    for (int k = 0; k < 6; k++) a.out[NODES + k] = 0;
    if (sp) {
      const long long sL0 = tot[NBS + 0], sL1 = tot[NBS + 1], nL = tot[NBS + 2];
      a.out[NODES + 0] = sL0; a.out[NODES + 1] = sL1;
      a.out[NODES + 2] = (long long)nodesum[0] - sL0; a.out[NODES + 3] = a.out[a.cnx] - sL1;
      a.out[NODES + 4] = nL; a.out[NODES + 5] = (long long)nodesum[1] - nL;
    }
  }
  if (rows_smem)
    for (int i = tid; i < a.n_pad; i += T) a.r[i] = r[i];
}

int launch_debug_pass(DPassArgs a, int threads, void* stream) {
  const int RT = threads - 32;
  const size_t rest = NODES * 4 + NODES * 8 + (size_t)(NBS + NSPLIT) * RT * 8 + TOT * 8 + NODES * 8 + 32;
  a.rows_in_smem = (size_t)a.n_pad * 8 + rest <= 200 * 1024;
  const size_t smem = (a.rows_in_smem ? (size_t)a.n_pad * 8 : 0) + rest;
  if (cudaFuncSetAttribute(debug_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return -1;
  debug_pass_kernel<<<1, threads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace fb
