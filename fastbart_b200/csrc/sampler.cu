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
//     cutpoint codes [p][n] stream from L2 as one 32-bit word per group.
//   * Per sweep: (1) all proposals are drawn in parallel, one thread per tree (a proposal depends only on its own
//     tree and on counter-based random numbers); (2) for each tree j the row warps make ONE fused pass that applies
//     tree j-1's accepted move (leaf ids updated four at a time with byte-SIMD compares, r -= delta from a 64-entry
//     table) and accumulates tree j's per-leaf sum of fx(w*R) into per-thread shared-memory bins plus the birth split
//     sums, all exact int64 (order independent, hence bit-exact); warp sums use redux.sync on three 21-bit limbs.
//     Meanwhile the control warp prefetches tree j's topology (cp.async) and draws the leaf-mu normals of every slot
//     that can be a leaf after the move.  Then the control warp runs Metropolis-Hastings, the tree update and the mu
//     draws in FP64, lanes in parallel; (3) an end-of-sweep pass refreshes every row's fit as an FP64 tree-order sum
//     of leaf values (which is also the draw's yhat.train), redraws the probit latent z, and sums rss for sigma.
//   * sum(w) per leaf is maintained exactly per tree (root: all rows; birth: the split sums; death: the two
//     children), so the pass reduces only sum(fx(w * R)).
//   * Random numbers: Philox4x32-10 keyed by the chain seed, counter = (draw index, tree or row, sweep, purpose).
//   * All control arithmetic is IEEE FP64 through fb_math.cuh; the file is compiled with -fmad=false.  The oracle's
//     DEV mode (oracle/fb_oracle.c) restates exactly this arithmetic on the CPU.
#include <cuda_runtime.h>

#include <cstdint>

#include "fb_internal.h"
#include "fb_math.cuh"

namespace fb {

constexpr int NBS = NB_MAX;   // per-thread shared-memory bins (compact leaf index < NBS); beyond: shared atomics

struct Prop {                 // proposal of one tree for the current sweep
  double logpr, lu;
  uint8_t mode, nx, v, c, l, r, pad0, pad1;
};
struct Masks { unsigned long long used, leaf; };
struct Ctl {                  // CTA-shared control state
  int pmode, pnx, pv, pc, pL, pR, pl, pr;   // tree j-1's applied move
  float DL, DR;                             // apply deltas of a birth's left / right rows
  int nleaf;                                // leaves of tree j
  int births, deaths, caps, rtcaps;
  int chain;
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

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ uint32_t bcast4(int v) { return (uint32_t)v * 0x01010101u; }
__device__ __forceinline__ int byte_of(uint32_t w, int e) { return (int)((w >> (8 * e)) & 255u); }

// ------------------------------------------------------------------------------------------------ fused row pass
struct PassU {
  uint8_t* leaf_prev;
  const uint8_t* leaf_cur;
  const uint8_t* qprev;
  const uint8_t* qcur;
  float* r;
  const float* ws;
  const float* D;       // [64] apply deltas
  const float2* tc;     // [64] {theta of tree j, compact leaf index as int bits}
  long long* bins;      // [NBS][RT]
  unsigned long long* ovb;
  long long* s1c;       // [NBS] CTA totals of sum fx(w*R) per compact leaf
  long long* split;     // [6] CTA totals sL0 sL1 sR0 sR1 nL nR
  float DL, DR;
  int n, ngroups, rt, RT, rwarp, nleaf;
  int apply, pmode, pnx, pc, pL, pR, pl, pr;
  int cmode, cnx, cc;
};

// Applies tree j-1's move to its leaf ids and to r, accumulates tree j's statistics (src/bart_kernel.cpp:164-201
// semantics; gpu/bart_batch.cu:184-227 fixed-point semantics).  Called by the row warps only; every lane of a row
// warp must call it (warp-wide reductions at the end).
__device__ __forceinline__ void pass_rows(const PassU& P) {
  const int lane = threadIdx.x & 31;
  long long* mybins = P.bins + P.rt;
  long long sl0 = 0, sl1 = 0, sr0 = 0, sr1 = 0;
  int nl = 0, nr = 0;
  const uint32_t pnx4 = bcast4(P.pnx), pc4 = bcast4(P.pc), pl4 = bcast4(P.pl), pr4 = bcast4(P.pr);
  const uint32_t pL4 = bcast4(P.pL), pR4 = bcast4(P.pR), cnx4 = bcast4(P.cnx), cc4 = bcast4(P.cc);
  for (int g = P.rt; g < P.ngroups; g += P.RT) {
    const uint32_t lc4 = *reinterpret_cast<const uint32_t*>(P.leaf_cur + 4 * g);
    const uint32_t lp4 = P.apply ? *reinterpret_cast<const uint32_t*>(P.leaf_prev + 4 * g) : 0u;
    const uint32_t qp4 = (P.apply && P.pmode == 1) ? __ldg(reinterpret_cast<const uint32_t*>(P.qprev + 4 * g)) : 0u;
    const uint32_t qc4 = P.cmode == 1 ? __ldg(reinterpret_cast<const uint32_t*>(P.qcur + 4 * g)) : 0u;
    const float4 r4 = reinterpret_cast<const float4*>(P.r)[g];
    const float4 w4 = reinterpret_cast<const float4*>(P.ws)[g];
    float rr[4] = {r4.x, r4.y, r4.z, r4.w};
    const float ww[4] = {w4.x, w4.y, w4.z, w4.w};
    if (P.apply) {
      uint32_t lpn = lp4, mv = 0u, side = 0u;
      if (P.pmode == 1) {
        mv = __vcmpeq4(lp4, pnx4);
        side = __vcmpleu4(qp4, pc4);                       // 0xFF where the row goes left
        lpn = (lp4 & ~mv) | (mv & ((side & pL4) | (~side & pR4)));
      } else if (P.pmode == 2) {
        const uint32_t md = __vcmpeq4(lp4, pl4) | __vcmpeq4(lp4, pr4);
        lpn = (lp4 & ~md) | (md & pnx4);                   // death deltas come from the table
      }
#pragma unroll
      for (int e = 0; e < 4; e++) {
        float delta = P.D[byte_of(lp4, e)];
        if (byte_of(mv, e)) delta = byte_of(side, e) ? P.DL : P.DR;
        rr[e] = __fsub_rn(rr[e], delta);
      }
      reinterpret_cast<float4*>(P.r)[g] = make_float4(rr[0], rr[1], rr[2], rr[3]);
      if (lpn != lp4) *reinterpret_cast<uint32_t*>(P.leaf_prev + 4 * g) = lpn;
    }
    long long wr[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const int lc = byte_of(lc4, e);
      const float2 t = P.tc[lc];
      const float R = __fadd_rn(rr[e], t.x);
      wr[e] = __float2ll_rn(__fmul_rn(ww[e], R));
      const int ci = __float_as_int(t.y);
      if (ci < NBS) mybins[ci * P.RT] += wr[e];
      else atomicAdd(&P.ovb[lc], (unsigned long long)wr[e]);
    }
    if (P.cmode == 1) {
      uint32_t inx = __vcmpeq4(lc4, cnx4);
      const int left = P.n - 4 * g;
      if (left < 4) inx &= (1u << (8 * (left > 0 ? left : 0))) - 1u;   // rows beyond n are padding
      if (inx) {
        const uint32_t lq = __vcmpleu4(qc4, cc4);
#pragma unroll
        for (int e = 0; e < 4; e++) {
          if (byte_of(inx, e)) {
            const long long wfx = __float2ll_rn(ww[e]);
            if (byte_of(lq, e)) { nl++; sl0 += wfx; sl1 += wr[e]; }
            else { nr++; sr0 += wfx; sr1 += wr[e]; }
          }
        }
      }
    }
  }
  // per-warp reductions of the private bins (reset for the next pass), then one shared atomic per warp and leaf into
  // the CTA totals (integer adds: the order of the atomics does not matter)
  const int nb = P.nleaf < NBS ? P.nleaf : NBS;
  for (int b = 0; b < nb; b++) {
    const long long v = mybins[b * P.RT];
    mybins[b * P.RT] = 0;
    const long long s = warp_sum64(v);
    if (lane == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&P.s1c[b]), (unsigned long long)s);
  }
  if (P.cmode == 1) {
    const long long a0 = warp_sum64(sl0), a1 = warp_sum64(sl1), a2 = warp_sum64(sr0), a3 = warp_sum64(sr1);
    const int c0 = __reduce_add_sync(0xffffffffu, nl), c1 = __reduce_add_sync(0xffffffffu, nr);
    if (lane == 0) {
      unsigned long long* sp = reinterpret_cast<unsigned long long*>(P.split);
      atomicAdd(sp + 0, (unsigned long long)a0); atomicAdd(sp + 1, (unsigned long long)a1);
      atomicAdd(sp + 2, (unsigned long long)a2); atomicAdd(sp + 3, (unsigned long long)a3);
      atomicAdd(sp + 4, (unsigned long long)c0); atomicAdd(sp + 5, (unsigned long long)c1);
    }
  }
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
  return -0.5 * fbm::fb_log(k) + 0.5 * M * M * t2 / k;
}

// Proposal of tree j at sweep it (src/bart_kernel.cpp:413-464); also resolves unknown goodvar counts of leaves.
__device__ Prop propose(DTree* t, const DChain& C, int j, int it, Masks& mk) {
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
  Prop P;
  P.mode = 0; P.nx = 0; P.v = 0; P.c = 0; P.l = 0; P.r = 0; P.pad0 = P.pad1 = 0; P.logpr = 0; P.lu = 0;
  double pr = 0;
  if (ub < PBx) {
    const int nx = select_kth(goodm, (int)(un * ngood));
    int v = (int)(uv * C.p); if (v >= C.p) v = C.p - 1;
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
      P.mode = 1; P.nx = (uint8_t)nx; P.v = (uint8_t)v; P.c = (uint8_t)c;
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
    P.mode = 2; P.nx = (uint8_t)nx; P.l = (uint8_t)l; P.r = (uint8_t)r;
  }
  if (P.mode) {
    P.logpr = fbm::fb_log(pr);
    const fbm::U4 y = fbm::philox(0u, (uint32_t)j, (uint32_t)it, fbm::TAG_MH, C.seed);
    P.lu = fbm::fb_log(fbm::u32d(y.x));
  }
  return P;
}

// ------------------------------------------------------------------------------------------------ shared layout
struct Smem {
  float* r; float* ws;          // [n_pad] (shared, or global when rows do not fit)
  float* th;                    // [m][64]
  Prop* prop;                   // [m]
  Masks* masks;                 // [m]
  DTree* tcur;                  // tree j (copy)
  long long* s0cur;             // [64]
  long long* s1;                // [64]
  float* tho;                   // [64] leaf values of tree j before its mu draw
  float* D;                     // [64] apply deltas of tree j-1's update
  float2* tc;                   // [64] theta and compact leaf index of tree j
  double* z;                    // [64] mu normals of tree j
  long long* bins;              // [NBS][RT]
  long long* s1c;               // [NBS]
  long long* split;             // [8]
  unsigned long long* ovb;      // [64]
  long long* red;               // [NW]
  Ctl* ctl;
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

__host__ __device__ inline size_t smem_layout(int threads, int m_max, int n_pad_max, int rows_in_smem, size_t* off) {
  const int NW = threads / 32, RT = threads - 32;
  size_t o = 0;
  off[0] = o; o += rows_in_smem ? align_up((size_t)n_pad_max * 4, 16) : 0;   // r
  off[1] = o; o += rows_in_smem ? align_up((size_t)n_pad_max * 4, 16) : 0;   // ws
  off[2] = o; o += align_up((size_t)m_max * NODES * 4, 16);                  // th
  off[3] = o; o += align_up((size_t)m_max * sizeof(Prop), 16);               // prop
  off[4] = o; o += align_up((size_t)m_max * sizeof(Masks), 16);              // masks
  off[5] = o; o += align_up(sizeof(DTree), 16);                              // tcur
  off[6] = o; o += NODES * 8;                                                // s0cur
  off[7] = o; o += NODES * 8;                                                // s1
  off[8] = o; o += NODES * 4;                                                // tho
  off[9] = o; o += NODES * 4;                                                // D
  off[10] = o; o += NODES * 8;                                               // tc
  off[11] = o; o += NODES * 8;                                               // z
  off[12] = o; o += (size_t)NBS * RT * 8;                                    // bins
  off[13] = o; o += (size_t)NBS * 8;                                         // s1c
  off[14] = o; o += 8 * 8;                                                   // split
  off[15] = o; o += 0;                                                       // (unused)
  off[16] = o; o += NODES * 8;                                               // ovb
  off[17] = o; o += align_up((size_t)NW * 8, 16);                            // red
  off[18] = o; o += align_up(sizeof(Ctl), 16);                               // ctl
  return o;
}
constexpr int NOFF = 19;

__device__ Smem carve(unsigned char* base, int threads, int m_max, int n_pad_max, int rows_in_smem) {
  size_t off[NOFF];
  smem_layout(threads, m_max, n_pad_max, rows_in_smem, off);
  Smem S;
  S.r = reinterpret_cast<float*>(base + off[0]);
  S.ws = reinterpret_cast<float*>(base + off[1]);
  S.th = reinterpret_cast<float*>(base + off[2]);
  S.prop = reinterpret_cast<Prop*>(base + off[3]);
  S.masks = reinterpret_cast<Masks*>(base + off[4]);
  S.tcur = reinterpret_cast<DTree*>(base + off[5]);
  S.s0cur = reinterpret_cast<long long*>(base + off[6]);
  S.s1 = reinterpret_cast<long long*>(base + off[7]);
  S.tho = reinterpret_cast<float*>(base + off[8]);
  S.D = reinterpret_cast<float*>(base + off[9]);
  S.tc = reinterpret_cast<float2*>(base + off[10]);
  S.z = reinterpret_cast<double*>(base + off[11]);
  S.bins = reinterpret_cast<long long*>(base + off[12]);
  S.s1c = reinterpret_cast<long long*>(base + off[13]);
  S.split = reinterpret_cast<long long*>(base + off[14]);
  S.ovb = reinterpret_cast<unsigned long long*>(base + off[16]);
  S.red = reinterpret_cast<long long*>(base + off[17]);
  S.ctl = reinterpret_cast<Ctl*>(base + off[18]);
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

// theta / compact-index table of tree j (control warp)
__device__ __forceinline__ void build_tc(const Smem& S, int j, int lane) {
  const unsigned long long lm = S.masks[j].leaf & S.masks[j].used;
  const float* thj = S.th + j * NODES;
  for (int s = lane; s < NODES; s += 32) {
    const int ci = ((lm >> s) & 1ull) ? __popcll(lm & ((1ull << s) - 1ull)) : 255;
    S.tc[s] = make_float2(thj[s], __int_as_float(ci));
  }
  if (lane == 0) S.ctl->nleaf = __popcll(lm);
}

// ------------------------------------------------------------------------------------------------ one chain
__device__ void run_chain(const DBufs& B, int ci, int it0, int it1, const Smem& S) {
  const DChain& C = B.chains[ci];
  const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int RT = T - 32;
  const int n = C.n, m = C.m, n_pad = C.n_pad, ngroups = n_pad / 4;
  const unsigned long long seed = C.seed;
  const double t2 = C.tau * C.tau, a_prior = 1.0 / t2;
  const double sci = pow2(-C.fx_shift), rscale = pow2(C.rss_shift), rsci = pow2(-C.rss_shift);
  const float scale = (float)pow2(C.fx_shift);
  const uint8_t* q = B.q + C.off_q;
  uint8_t* leaf = B.leaf + C.off_leaf;
  DTree* trees = B.trees + C.off_tree;
  long long* s0g = B.s0 + C.off_tree * NODES;
  float* thg = B.th + C.off_tree * NODES;
  double* ywork = B.ywork + C.off_row;
  const float* wg = B.win + C.off_row;
  float* rg = B.rsave + C.off_row;
  float* wsg = B.wsave + C.off_row;
  double* tm = B.tm + C.off_row;
  float* r = B.rows_in_smem ? S.r : rg;
  float* ws = B.rows_in_smem ? S.ws : wsg;
  Ctl& ctl = *S.ctl;
  DState& st = B.states[ci];

  // ---------------------------------------------------------------- chain start or resume
  if (tid == 0) {
    if (it0 == 0) { ctl.sigma = C.sigest; ctl.births = ctl.deaths = ctl.caps = ctl.rtcaps = 0; }
    else { ctl.sigma = st.sigma; ctl.births = st.births; ctl.deaths = st.deaths; ctl.caps = st.caps; ctl.rtcaps = st.rtcaps; }
    ctl.pmode = 0;
  }
  for (int k = tid; k < NBS * RT; k += T) S.bins[k] = 0;
  for (int s = tid; s < NODES; s += T) S.ovb[s] = 0ull;
  if (tid < NBS) S.s1c[tid] = 0;
  if (tid < 8) S.split[tid] = 0;
  __syncthreads();
  for (int i = tid; i < n_pad; i += T) ws[i] = __fmul_rn(wg[i], scale);   // exact: power-of-two scaling
  if (it0 == 0) {
    int caps = 0;
    for (int i = tid; i < n_pad; i += T) {
      double y = 0.0;
      if (i < n) {
        if (C.probit)
          y = B.ybin[C.off_row + i] == 0 ? -fbm::fb_rtnorm(seed, (uint32_t)i, fbm::INIT_SWEEP, 0.0, C.offset, &caps)
                                         : fbm::fb_rtnorm(seed, (uint32_t)i, fbm::INIT_SWEEP, 0.0, -C.offset, &caps);
        else y = B.yin[C.off_row + i];
      }
      ywork[i] = y;
      r[i] = (float)y;
      tm[i] = 0.0;
    }
    if (caps) atomicAdd(&ctl.rtcaps, caps);
    for (long long k = tid; k < (long long)m * n_pad / 16; k += T)
      reinterpret_cast<uint4*>(leaf)[k] = make_uint4(0u, 0u, 0u, 0u);
    for (int k = tid; k < m * NODES; k += T) S.th[k] = 0.0f;
    long long sw = 0;
    for (int i = tid; i < n; i += T) sw += __float2ll_rn(__fmul_rn(wg[i], scale));
    const long long swt = block_sum64(sw, S.red);
    // root-only trees: every word zero except ngv[0] (byte 384), used (byte 448) and leaf (byte 456)
    constexpr int TWORDS = (int)(sizeof(DTree) / 4);
    for (int k = tid; k < m * TWORDS; k += T) {
      const int j = k / TWORDS, byte0 = (k % TWORDS) * 4;
      uint32_t val = 0u;
      if (byte0 == 6 * NODES) val = (uint32_t)C.root_ngv;
      else if (byte0 == 7 * NODES || byte0 == 7 * NODES + 8) val = 1u;
      reinterpret_cast<uint32_t*>(trees + j)[k % TWORDS] = val;
    }
    for (int k = tid; k < m * NODES; k += T) s0g[k] = (k % NODES == 0) ? swt : 0ll;
  } else {
    if (B.rows_in_smem)
      for (int i = tid; i < n_pad; i += T) S.r[i] = rg[i];
    for (int k = tid; k < m * NODES; k += T) S.th[k] = thg[k];
  }
  __syncthreads();

  for (int it = it0; it < it1; it++) {
    const double inv_s2 = 1.0 / (ctl.sigma * ctl.sigma);
    // ---------------------------------------------------------------- (1) proposals, one thread per tree
    for (int j = tid; j < m; j += T) {
      Masks mk;
      S.prop[j] = propose(trees + j, C, j, it, mk);
      S.masks[j] = mk;
    }
    __syncthreads();
    if (warp == 0) {
      build_tc(S, 0, lane);
      if (lane == 0) ctl.pmode = 0;
    }
    __syncthreads();
    // ---------------------------------------------------------------- (2) trees
    for (int j = 0; j < m; j++) {
      const Prop P = S.prop[j];
      if (warp > 0) {
        PassU U;
        U.leaf_prev = j > 0 ? leaf + (long long)(j - 1) * n_pad : nullptr;
        U.leaf_cur = leaf + (long long)j * n_pad;
        U.qprev = q + (long long)ctl.pv * n_pad;
        U.qcur = q + (long long)P.v * n_pad;
        U.r = r; U.ws = ws; U.D = S.D; U.tc = S.tc; U.bins = S.bins; U.ovb = S.ovb;
        U.s1c = S.s1c; U.split = S.split;
        U.DL = ctl.DL; U.DR = ctl.DR;
        U.n = n; U.ngroups = ngroups; U.rt = tid - 32; U.RT = RT; U.rwarp = warp - 1; U.nleaf = ctl.nleaf;
        U.apply = j > 0; U.pmode = ctl.pmode; U.pnx = ctl.pnx; U.pc = ctl.pc; U.pL = ctl.pL; U.pR = ctl.pR;
        U.pl = ctl.pl; U.pr = ctl.pr;
        U.cmode = P.mode; U.cnx = P.nx; U.cc = P.c;
        pass_rows(U);
      } else {
        // control warp during the pass: prefetch tree j, draw the normals of every slot that can be a leaf after
        // this step's move (current leaves, the two slots a birth would take, the node a death would restore)
        constexpr int TW = (int)(sizeof(DTree) / 16), SW = NODES * 8 / 16;
        for (int k = lane; k < TW + SW; k += 32) {
          if (k < TW) cp_async16(reinterpret_cast<unsigned char*>(S.tcur) + 16 * k, reinterpret_cast<const unsigned char*>(trees + j) + 16 * k);
          else cp_async16(reinterpret_cast<unsigned char*>(S.s0cur) + 16 * (k - TW), reinterpret_cast<const unsigned char*>(s0g + (long long)j * NODES) + 16 * (k - TW));
        }
        const Masks mk = S.masks[j];
        unsigned long long cand = mk.leaf & mk.used;
        if (P.mode == 1) {
          const int L = first_free(mk.used, -1), R = L >= 0 ? first_free(mk.used, L) : -1;
          if (L >= 0 && R >= 0) cand |= (1ull << L) | (1ull << R);
        } else if (P.mode == 2) {
          cand |= 1ull << P.nx;
        }
        for (int s = lane; s < NODES; s += 32)
          if ((cand >> s) & 1ull) S.z[s] = fbm::fb_normal(seed, (uint32_t)s << 8, (uint32_t)j, (uint32_t)it, fbm::TAG_MU);
        cp_async_wait_all();
      }
      __syncthreads();
      // ---------------------------------------------------------------- control: MH, tree update, mu draws
      if (warp == 0) {
        const int nleaf = ctl.nleaf;
        const Masks mk = S.masks[j];
        unsigned long long used = mk.used, leafm = mk.leaf;
        const unsigned long long lm0 = used & leafm;
        for (int s = lane; s < NODES; s += 32) {
          if ((lm0 >> s) & 1ull) {
            const int ci2 = __float_as_int(S.tc[s].y);
            S.s1[s] = ci2 < NBS ? S.s1c[ci2] : (long long)S.ovb[s];
          }
          if (nleaf > NBS) S.ovb[s] = 0ull;
        }
        const long long sL0 = S.split[0], sL1 = S.split[1], sR0 = S.split[2], sR1 = S.split[3];
        const int nL = (int)S.split[4], nR = (int)S.split[5];
        __syncwarp();
        if (lane < NBS) S.s1c[lane] = 0;
        if (lane < 8) S.split[lane] = 0;
        __syncwarp();
        bool eval = false;
        double bl = 0, Ml = 0, br = 0, Mr = 0;
        if (P.mode == 1 && nL >= 5 && nR >= 5) {
          eval = true;
          bl = (double)sL0 * sci * inv_s2; Ml = (double)sL1 * sci * inv_s2;
          br = (double)sR0 * sci * inv_s2; Mr = (double)sR1 * sci * inv_s2;
        } else if (P.mode == 2) {
          eval = true;
          bl = (double)S.s0cur[P.l] * sci * inv_s2; Ml = (double)S.s1[P.l] * sci * inv_s2;
          br = (double)S.s0cur[P.r] * sci * inv_s2; Mr = (double)S.s1[P.r] * sci * inv_s2;
        }
        bool accept = false;
        if (eval) {
          // lanes 0..2 evaluate the three log marginal likelihoods at one call site: birth (l, r, l+r), death
          // (l+r, l, r), in the order the ratio adds them
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
        int nmode = 0, L = 0, R = 0, l = 0, rr = 0;
        DTree* t = S.tcur;
        if (accept && P.mode == 1) {
          L = first_free(used, -1);
          R = L >= 0 ? first_free(used, L) : -1;
          if (L < 0 || R < 0) {
            if (lane == 0) ctl.caps++;
            L = R = 0;
          } else {
            const int nx = P.nx;
            if (lane == 0) {
              t->v[nx] = P.v; t->c[nx] = P.c; t->l[nx] = (uint8_t)L; t->r[nx] = (uint8_t)R;
              t->par[L] = (uint8_t)nx; t->par[R] = (uint8_t)nx; t->l[L] = t->r[L] = t->l[R] = t->r[R] = 0;
              t->d[L] = t->d[R] = (uint8_t)(t->d[nx] + 1);
              t->ngv[L] = t->ngv[R] = 255;   // resolved by the next sweep's proposal step
              S.s0cur[L] = sL0; S.s0cur[R] = sR0; S.s1[L] = sL1; S.s1[R] = sR1;
              ctl.births++;
            }
            used |= (1ull << L) | (1ull << R);
            leafm = (leafm & ~(1ull << nx)) | (1ull << L) | (1ull << R);
            nmode = 1;
          }
        } else if (accept && P.mode == 2) {
          const int nx = P.nx;
          l = P.l; rr = P.r;
          if (lane == 0) {
            S.s0cur[nx] = S.s0cur[l] + S.s0cur[rr]; S.s1[nx] = S.s1[l] + S.s1[rr];
            t->l[nx] = 0; t->r[nx] = 0; t->v[nx] = 0; t->c[nx] = 0;
            ctl.deaths++;
          }
          used &= ~((1ull << l) | (1ull << rr));
          leafm = (leafm & ~((1ull << l) | (1ull << rr))) | (1ull << nx);
          nmode = 2;
        }
        if (lane == 0) { t->used = used; t->leaf = leafm; S.masks[j].used = used; S.masks[j].leaf = leafm; }
        __syncwarp();
        // leaf mu draws (DRMU), lanes in parallel over slots; apply deltas D[s] = new - old
        const unsigned long long lm = used & leafm;
        float* thj = S.th + j * NODES;
        for (int s = lane; s < NODES; s += 32) {
          const float old = thj[s];
          S.tho[s] = old;
          float nw = old;
          if ((lm >> s) & 1ull) {
            const double b = (double)S.s0cur[s] * sci * inv_s2, M = (double)S.s1[s] * sci * inv_s2;
            nw = (float)(M / (a_prior + b) + S.z[s] / sqrt(a_prior + b));
          }
          thj[s] = nw;
          S.D[s] = __fsub_rn(nw, old);
        }
        __syncwarp();
        if (lane == 0) {
          float DL = 0.0f, DR = 0.0f;
          if (nmode == 1) { DL = __fsub_rn(thj[L], S.tho[P.nx]); DR = __fsub_rn(thj[R], S.tho[P.nx]); }
          else if (nmode == 2) { S.D[l] = __fsub_rn(thj[P.nx], S.tho[l]); S.D[rr] = __fsub_rn(thj[P.nx], S.tho[rr]); }
          ctl.DL = DL; ctl.DR = DR;
          ctl.pmode = nmode; ctl.pnx = P.nx; ctl.pv = P.v; ctl.pc = P.c; ctl.pL = L; ctl.pR = R; ctl.pl = l; ctl.pr = rr;
        }
        // write tree j back
        {
          const uint32_t* src = reinterpret_cast<const uint32_t*>(t);
          uint32_t* dst = reinterpret_cast<uint32_t*>(trees + j);
          for (int k = lane; k < (int)(sizeof(DTree) / 4); k += 32) dst[k] = src[k];
          for (int k = lane; k < NODES; k += 32) s0g[(long long)j * NODES + k] = S.s0cur[k];
        }
        if (j + 1 < m) build_tc(S, j + 1, lane);
      }
      __syncthreads();
    }
    // ---------------------------------------------------------------- (3) end of sweep
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
      for (int g = tid; g < ngroups; g += T) {
        const uint32_t lp4 = *reinterpret_cast<const uint32_t*>(lp + 4 * g);
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
          for (int u = 0; u < 16; u++) l4[u] = *reinterpret_cast<const uint32_t*>(leaf + (long long)(jj + u) * n_pad + 4 * g);
#pragma unroll
          for (int u = 0; u < 16; u++) {
            const float* thj = S.th + (jj + u) * NODES;
            f0 += (double)thj[l4[u] & 255u]; f1 += (double)thj[(l4[u] >> 8) & 255u];
            f2 += (double)thj[(l4[u] >> 16) & 255u]; f3 += (double)thj[l4[u] >> 24];
          }
        }
        for (; jj < m; jj++) {
          const uint32_t l4 = jj == m - 1 ? lpn : *reinterpret_cast<const uint32_t*>(leaf + (long long)jj * n_pad + 4 * g);
          const float* thj = S.th + jj * NODES;
          f0 += (double)thj[l4 & 255u]; f1 += (double)thj[(l4 >> 8) & 255u];
          f2 += (double)thj[(l4 >> 16) & 255u]; f3 += (double)thj[l4 >> 24];
        }
        const double fe[4] = {f0, f1, f2, f3};
        const float4 w4 = reinterpret_cast<const float4*>(ws)[g];
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
        reinterpret_cast<float4*>(r)[g] = make_float4(rn[0], rn[1], rn[2], rn[3]);
      }
    }
    if (caps) atomicAdd(&ctl.rtcaps, caps);
    const long long rss = C.probit ? 0 : block_sum64(rssfx, S.red);
    if (tid == 0) {
      if (!C.probit) {
        const double rssd = (double)rss * rsci;
        ctl.sigma = sqrt((C.nu * C.lambda + rssd) / (2.0 * fbm::fb_gamma(seed, (uint32_t)it, ((double)n + C.nu) / 2.0)));
      }
      B.sigma_out[C.off_sigma + it] = ctl.sigma;
      ctl.pmode = 0;
    }
    if (keep) {   // kept draw: packed nodes (src/bart_kernel.cpp:559-571)
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
    for (int i = tid; i < n_pad; i += T) rg[i] = S.r[i];
  if (tid == 0) {
    st.sigma = ctl.sigma; st.births = ctl.births; st.deaths = ctl.deaths; st.caps = ctl.caps; st.rtcaps = ctl.rtcaps;
    st.it_done = it1;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(MAX_THREADS, 1) sampler_kernel(DBufs B, int it0, int it1) {
  extern __shared__ __align__(16) unsigned char smem[];
  const Smem S = carve(smem, blockDim.x, B.m_max, B.n_pad_max, B.rows_in_smem);
  for (;;) {
    if (threadIdx.x == 0) S.ctl->chain = atomicAdd(B.queue, 1);
    __syncthreads();
    const int qi = S.ctl->chain;
    __syncthreads();
    if (qi >= B.nchains) break;
    run_chain(B, B.order[qi], it0, it1, S);
  }
}

size_t sampler_smem_bytes(int threads, int m_max, int n_pad_max, int rows_in_smem) {
  size_t off[NOFF];
  return smem_layout(threads, m_max, n_pad_max, rows_in_smem, off);
}

int sampler_max_grid(int threads, size_t smem, int device) {
  int per_sm = 0, nsm = 0;
  cudaFuncSetAttribute(sampler_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sampler_kernel, threads, smem) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return -1;
  return per_sm * nsm;
}

int launch_sampler(const DBufs& b, int it0, int it1, int threads, int grid, size_t smem, void* stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (cudaFuncSetAttribute(sampler_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return -1;
  if (cudaMemsetAsync(b.queue, 0, sizeof(int), s) != cudaSuccess) return -1;
  sampler_kernel<<<grid, threads, smem, s>>>(b, it0, it1);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// ------------------------------------------------------------------------------------------------ diagnostics
// One pass on explicit state, run by the same pass_rows() as the sampler: warp 0 builds the tables, warps 1.. stream.
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
  long long* bins = reinterpret_cast<long long*>(p); p += (size_t)NBS * RT * 8;
  long long* s1c = reinterpret_cast<long long*>(p); p += NBS * 8;
  long long* split = reinterpret_cast<long long*>(p); p += 8 * 8;
  unsigned long long* ovb = reinterpret_cast<unsigned long long*>(p); p += NODES * 8;
  float* dlr = reinterpret_cast<float*>(p);
  const float scale = (float)pow2(a.fx_shift);
  for (int i = tid; i < a.n_pad; i += T) {
    if (rows_smem) r[i] = a.r[i];
    ws[i] = __fmul_rn(a.w[i], scale);
  }
  for (int k = tid; k < NBS * RT; k += T) bins[k] = 0;
  for (int s = tid; s < NODES; s += T) ovb[s] = 0;
  if (tid < NBS) s1c[tid] = 0;
  if (tid < 8) split[tid] = 0;
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
    U.r = r; U.ws = ws; U.D = D; U.tc = tc; U.bins = bins; U.ovb = ovb; U.s1c = s1c; U.split = split;
    U.DL = dlr[0]; U.DR = dlr[1];
    U.n = a.n; U.ngroups = a.n_pad / 4; U.rt = tid - 32; U.RT = RT; U.rwarp = (tid >> 5) - 1; U.nleaf = nleaf;
    U.apply = a.apply; U.pmode = a.pmode; U.pnx = a.pnx; U.pc = a.pc; U.pL = a.pL; U.pR = a.pR; U.pl = a.pl; U.pr = a.pr;
    U.cmode = a.stats ? a.cmode : 0; U.cnx = a.cnx; U.cc = a.cc;
    pass_rows(U);
  }
  __syncthreads();
  for (int s = tid; s < NODES; s += T) {
    long long v = 0;
    if ((a.leafmask >> s) & 1ull) {
      const int ci = __float_as_int(tc[s].y);
      v = ci < NBS ? s1c[ci] : (long long)ovb[s];
    }
    a.out[s] = v;
  }
  if (tid == 0) {
    const bool sp = a.stats && a.cmode == 1;
    for (int k = 0; k < 6; k++) a.out[NODES + k] = sp ? split[k] : 0;
  }
  if (rows_smem)
    for (int i = tid; i < a.n_pad; i += T) a.r[i] = r[i];
}

int launch_debug_pass(DPassArgs a, int threads, void* stream) {
  const int RT = threads - 32;
  const size_t rest = NODES * 4 + NODES * 8 + (size_t)NBS * RT * 8 + NBS * 8 + 64 + NODES * 8 + 16;
  a.rows_in_smem = (size_t)a.n_pad * 8 + rest <= 200 * 1024;
  const size_t smem = (a.rows_in_smem ? (size_t)a.n_pad * 8 : 0) + rest;
  if (cudaFuncSetAttribute(debug_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return -1;
  debug_pass_kernel<<<1, threads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace fb
