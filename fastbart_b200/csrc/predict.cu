// predict.cu -- predict_draw on the device (src/predict.cpp:49-73).
//
// Two evaluators with the same arithmetic.  The tiled one (predict_tiled_kernel, used when the columns of a row tile
// fit in shared memory) is described at its definition.  The streaming one (predict_kernel, any p):
// each thread owns one row of one draw and walks the draw's trees in order 1..ntree with the
// branch-free step k = child[k] + (x[var[k]] >= cut[k]) over the breadth-first node arrays (children adjacent), adding
// leaf values to an FP64 accumulator that starts at 0; mu is added last.  That is the reference's summation order, so
// results are bit-identical to predict_draw_cpp / pwbart.  Rows of a warp are consecutive, so the x reads of each
// node visit are coalesced (column-major x); node arrays are read through the read-only cache, where all threads of a
// draw share them.  The grid's y dimension enumerates draws, so a bulk call (many draws) runs in one launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "fb_internal.h"

namespace fb {

__global__ void __launch_bounds__(256) predict_kernel(DForest f, const double* __restrict__ x, int n, int ld, int draw0,
                                                      double mu, double* __restrict__ out, int ldo) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int d = draw0 + blockIdx.y;   // 0-based draw
  if (i >= n) return;
  const int* __restrict__ root = f.root + (long long)d * f.ntree;
  double acc = 0.0;
  for (int t = 0; t < f.ntree; t++) {
    int k = __ldg(root + t);
    int ch = __ldg(f.child + k);
    while (ch >= 0) {
      const int v = __ldg(f.var + k);
      const double xv = __ldg(x + (long long)v * ld + i);
      k = ch + (xv >= __ldg(f.cut + k) ? 1 : 0);
      ch = __ldg(f.child + k);
    }
    acc = __dadd_rn(acc, __ldg(f.theta + k));
  }
  out[(long long)blockIdx.y * ldo + i] = __dadd_rn(acc, mu);
}

// Tiled evaluator for inputs whose columns fit in shared memory (p < PT_MAXP).  A CTA stages the x of PT_ROWS
// consecutive rows in shared memory once ([p + 1][PT_ROWS], coalesced; column p is -inf), then evaluates a range of
// draws for them, so x crosses HBM once however many draws are evaluated.  A thread walks four trees at a time with a
// fixed number of steps, the deepest leaf of the four (leaves loop on themselves, see PNode): no data-dependent
// branches, and the four node chains overlap.  Leaf values are added in tree order, so the FP64 sum is the same
// sequence of additions as the one-tree-at-a-time loop of src/predict.cpp:62-70.
constexpr int PT_ROWS = 128;
constexpr int PT_MAXP = 96;

struct NodeReg { double v; int child, var; };

__device__ __forceinline__ NodeReg load_node(const PNode* __restrict__ nodes, int k) {
  const double2 q = __ldg(reinterpret_cast<const double2*>(nodes + k));
  return NodeReg{q.x, __double2loint(q.y), __double2hiint(q.y)};
}
__device__ __forceinline__ void step(NodeReg& a, const PNode* __restrict__ nodes, const double* xr) {
  a = load_node(nodes, a.child + (xr[a.var * PT_ROWS] >= a.v ? 1 : 0));
}

__global__ void __launch_bounds__(PT_ROWS) predict_tiled_kernel(DForest f, const double* __restrict__ x, int n, int ld,
                                                                int draw0, int ndraws, int dpc, double mu,
                                                                double* __restrict__ out, int ldo) {
  extern __shared__ double xs[];   // [p + 1][PT_ROWS]
  const int tid = threadIdx.x;
  const int i = blockIdx.x * PT_ROWS + tid;
  for (int v = 0; v < f.p; v++) xs[v * PT_ROWS + tid] = i < n ? x[(long long)v * ld + i] : 0.0;
  xs[f.p * PT_ROWS + tid] = -__longlong_as_double(0x7FF0000000000000LL);
  __syncthreads();
  if (i >= n) return;
  const double* xr = xs + tid;
  const PNode* __restrict__ nodes = f.nodes;
  const int m = f.ntree, G = (m + 3) / 4, m4 = m & ~3;
  const int d0 = blockIdx.y * dpc, d1 = min(ndraws, d0 + dpc);
  for (int d = d0; d < d1; d++) {
    const int* __restrict__ root = f.root + (long long)(draw0 + d) * m;
    const uint8_t* __restrict__ gdep = f.gdepth + (long long)(draw0 + d) * G;
    double acc = 0.0;
    for (int t = 0; t < m4; t += 4) {
      NodeReg a = load_node(nodes, __ldg(root + t)), b = load_node(nodes, __ldg(root + t + 1));
      NodeReg c = load_node(nodes, __ldg(root + t + 2)), e = load_node(nodes, __ldg(root + t + 3));
      const int depth = __ldg(gdep + (t >> 2));
      for (int s = 0; s < depth; s++) {
        step(a, nodes, xr);
        step(b, nodes, xr);
        step(c, nodes, xr);
        step(e, nodes, xr);
      }
      acc = __dadd_rn(acc, a.v);
      acc = __dadd_rn(acc, b.v);
      acc = __dadd_rn(acc, c.v);
      acc = __dadd_rn(acc, e.v);
    }
    if (m4 < m) {
      const int depth = __ldg(gdep + (m4 >> 2));
      for (int t = m4; t < m; t++) {
        NodeReg a = load_node(nodes, __ldg(root + t));
        for (int s = 0; s < depth; s++) step(a, nodes, xr);
        acc = __dadd_rn(acc, a.v);
      }
    }
    out[(long long)d * ldo + i] = __dadd_rn(acc, mu);
  }
}

// Code-compare evaluator, the default when the cutpoints allow it (DForest::n32).  A CTA of PC_ROWS threads (one row
// each) first turns its rows' x into cutpoint codes, code_v(x) = number of cutpoints of v that are <= x (binary
// search; NaN gives 0), kept in shared memory as bytes [p][PC_ROWS]: then x >= cut[v][c] is code_v(x) > c exactly.
// For each draw of its range it stages that draw's packed nodes (4 bytes each) and leaf values in shared memory, and
// every thread walks four trees at a time for the group's fixed depth (leaves loop on themselves): per step one
// broadcast node load and one byte load, both from shared memory.  Leaf values are added in tree order, the same
// FP64 additions as src/predict.cpp:62-70.
constexpr int PC_ROWS = 256;

__device__ __forceinline__ int cstep(int k, const uint32_t* nd, const uint8_t* cr) {
  const uint32_t w = nd[k];
  return (int)(w & 0xFFFFu) + (cr[((w >> 16) & 0xFFu) * PC_ROWS] > (w >> 24) ? 1 : 0);
}

__global__ void __launch_bounds__(PC_ROWS) predict_codes_kernel(DForest f, const double* __restrict__ x, int n, int ld,
                                                                int draw0, int ndraws, int dpc, double mu,
                                                                double* __restrict__ out, int ldo, int ncodes) {
  extern __shared__ __align__(16) unsigned char pc_smem[];
  double* th_s = reinterpret_cast<double*>(pc_smem);                   // [maxnd]
  uint32_t* nd_s = reinterpret_cast<uint32_t*>(th_s + f.maxnd);       // [maxnd]
  uint8_t* code_s = reinterpret_cast<uint8_t*>(nd_s + f.maxnd);        // [ncodes][PC_ROWS]
  const int tid = threadIdx.x;
  const int i = blockIdx.x * PC_ROWS + tid;
  const bool live = i < n;
  for (int v = 0; v < ncodes; v++) {
    int lo = 0;
    if (live) {
      const double xv = x[(long long)v * ld + i];
      const double* __restrict__ cv = f.cuts + f.cutoff[v];
      int hi = f.cutoff[v + 1] - f.cutoff[v];
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(cv + mid) <= xv) lo = mid + 1;
        else hi = mid;
      }
    }
    code_s[v * PC_ROWS + tid] = (uint8_t)lo;
  }
  const uint8_t* cr = code_s + tid;
  const int m = f.ntree, G = (m + 3) / 4, m4 = m & ~3;
  const long long ntot = (long long)f.ndpost * m;
  const int d0 = blockIdx.y * dpc, d1 = min(ndraws, d0 + dpc);
  for (int d = d0; d < d1; d++) {
    const long long t0 = (long long)(draw0 + d) * m;
    const int base = __ldg(f.root + t0);
    const int cnt = (t0 + m < ntot ? __ldg(f.root + t0 + m) : f.nnodes) - base;
    __syncthreads();   // the previous draw's nodes are no longer read
    for (int k = tid; k < cnt; k += PC_ROWS) {
      nd_s[k] = __ldg(f.n32 + base + k);
      th_s[k] = __ldg(f.theta + base + k);
    }
    __syncthreads();
    if (!live) continue;
    const int* __restrict__ root = f.root + t0;
    const uint8_t* __restrict__ gdep = f.gdepth + (long long)(draw0 + d) * G;
    double acc = 0.0;
    for (int t = 0; t < m4; t += 4) {
      int a = __ldg(root + t) - base, b = __ldg(root + t + 1) - base;
      int c = __ldg(root + t + 2) - base, e = __ldg(root + t + 3) - base;
      const int depth = __ldg(gdep + (t >> 2));
      for (int s = 0; s < depth; s++) {
        a = cstep(a, nd_s, cr);
        b = cstep(b, nd_s, cr);
        c = cstep(c, nd_s, cr);
        e = cstep(e, nd_s, cr);
      }
      acc = __dadd_rn(acc, th_s[a]);
      acc = __dadd_rn(acc, th_s[b]);
      acc = __dadd_rn(acc, th_s[c]);
      acc = __dadd_rn(acc, th_s[e]);
    }
    if (m4 < m) {
      const int depth = __ldg(gdep + (m4 >> 2));
      for (int t = m4; t < m; t++) {
        int a = __ldg(root + t) - base;
        for (int s = 0; s < depth; s++) a = cstep(a, nd_s, cr);
        acc = __dadd_rn(acc, th_s[a]);
      }
    }
    out[(long long)d * ldo + i] = __dadd_rn(acc, mu);
  }
}

// Code-compare evaluator that carries each row's leaves from one draw to the next (DForest::same).  BART changes a
// few trees per sweep and redraws every leaf value, so consecutive posterior draws share the structure of most
// trees: a row then reaches the same leaf, at the same offset from the tree's root, and only the leaf value differs.
// A CTA of PC_ROWS rows evaluates a contiguous range of draws; it keeps, per row and tree, the offset of the row's
// leaf from the tree's root (one byte, four trees to a shared-memory word).  Its first draw walks every tree; a later
// draw walks only the trees whose structure changed (the flags are per draw and tree, so the branch is uniform across
// the CTA), each for its own depth, and reads the other leaves' offsets.  Leaf values are added in tree order, the
// same FP64 additions as src/predict.cpp:62-70, so the results equal the other evaluators' bit for bit.
__global__ void __launch_bounds__(PC_ROWS, 3) predict_carry_kernel(DForest f, const double* __restrict__ x, int n, int ld,
                                                                int draw0, int ndraws, int dpc, double mu,
                                                                double* __restrict__ out, int ldo, int ncodes) {
  extern __shared__ __align__(16) unsigned char pc_smem[];
  const int m = f.ntree, G = (m + 3) / 4;
  double* th_s = reinterpret_cast<double*>(pc_smem);                   // [maxnd]
  uint32_t* nd_s = reinterpret_cast<uint32_t*>(th_s + f.maxnd);       // [maxnd]
  uint32_t* lf_s = reinterpret_cast<uint32_t*>(pc_smem + (((size_t)f.maxnd * 12 + 15) & ~(size_t)15));
                                                                       // [G][PC_ROWS] leaf offsets, 4 trees a word
  uint16_t* rt_s = reinterpret_cast<uint16_t*>(lf_s + (size_t)G * PC_ROWS);   // [4 G] roots of the draw's trees
  uint8_t* td_s = reinterpret_cast<uint8_t*>(rt_s + 4 * G);           // [4 G] their depths
  uint8_t* sg_s = td_s + 4 * G;                                        // [G] bit u: tree 4 g + u keeps its leaves
  uint8_t* code_s = sg_s + ((G + 7) & ~7);                             // [ncodes][PC_ROWS]
  const int tid = threadIdx.x;
  const int i = blockIdx.x * PC_ROWS + tid;
  const bool live = i < n;
  for (int v = 0; v < ncodes; v++) {
    int lo = 0;
    if (live) {
      const double xv = x[(long long)v * ld + i];
      const double* __restrict__ cv = f.cuts + f.cutoff[v];
      int hi = f.cutoff[v + 1] - f.cutoff[v];
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(cv + mid) <= xv) lo = mid + 1;
        else hi = mid;
      }
    }
    code_s[v * PC_ROWS + tid] = (uint8_t)lo;
  }
  const uint8_t* cr = code_s + tid;
  uint32_t* lf = lf_s + tid;
  for (int g = 0; g < G; g++) lf[g * PC_ROWS] = 0u;
  const long long ntot = (long long)f.ndpost * m;
  const int SW = (m + 31) / 32;
  const int d0 = blockIdx.y * dpc, d1 = min(ndraws, d0 + dpc);
  // a range's first draw walks every tree; trees past ntree (padding of the last group) never walk
  auto keep_bits = [&](int d, int g) {
    uint32_t keep = d == d0 ? 0u : (__ldg(f.same + (long long)(draw0 + d) * SW + (g >> 3)) >> ((g & 7) * 4)) & 15u;
    for (int u = 0; u < 4; u++)
      if (4 * g + u >= m) keep |= 1u << u;
    return keep;
  };
  // When a draw has at most PF x PC_ROWS nodes (4 G <= 200 < PC_ROWS always), each thread loads its share of the next
  // draw's tables into registers while the current draw is evaluated, and stores them after the next barrier, so
  // the tables' global-memory latency is not exposed once per draw.
  constexpr int PF = 4;
  const bool pipe = f.maxnd <= PF * PC_ROWS;
  uint32_t pn[PF];
  double pt[PF];
  uint32_t prt = 0, ptd = 0, psg = 0;
  int pcnt = 0;
  auto load_next = [&](int d) {
    const long long t0 = (long long)(draw0 + d) * m;
    const int base = __ldg(f.root + t0);
    pcnt = (t0 + m < ntot ? __ldg(f.root + t0 + m) : f.nnodes) - base;
#pragma unroll
    for (int u = 0; u < PF; u++) {
      const int k = tid + u * PC_ROWS;
      if (k < pcnt) { pn[u] = __ldg(f.n32 + base + k); pt[u] = __ldg(f.theta + base + k); }
    }
    if (tid < 4 * G) {
      prt = tid < m ? (uint32_t)(__ldg(f.root + t0 + tid) - base) : 0u;
      ptd = tid < m ? (uint32_t)__ldg(f.tdep + t0 + tid) : 0u;
    }
    if (tid < G) psg = keep_bits(d, tid);
  };
  if (pipe && d0 < d1) load_next(d0);
  for (int d = d0; d < d1; d++) {
    __syncthreads();   // the previous draw's tables are no longer read
    if (pipe) {
#pragma unroll
      for (int u = 0; u < PF; u++) {
        const int k = tid + u * PC_ROWS;
        if (k < pcnt) { nd_s[k] = pn[u]; th_s[k] = pt[u]; }
      }
      if (tid < 4 * G) { rt_s[tid] = (uint16_t)prt; td_s[tid] = (uint8_t)ptd; }
      if (tid < G) sg_s[tid] = (uint8_t)psg;
    } else {
      const long long t0 = (long long)(draw0 + d) * m;
      const int base = __ldg(f.root + t0);
      const int cnt = (t0 + m < ntot ? __ldg(f.root + t0 + m) : f.nnodes) - base;
      for (int k = tid; k < cnt; k += PC_ROWS) {
        nd_s[k] = __ldg(f.n32 + base + k);
        th_s[k] = __ldg(f.theta + base + k);
      }
      for (int t = tid; t < 4 * G; t += PC_ROWS) {
        rt_s[t] = t < m ? (uint16_t)(__ldg(f.root + t0 + t) - base) : (uint16_t)0;
        td_s[t] = t < m ? __ldg(f.tdep + t0 + t) : (uint8_t)0;
      }
      for (int g = tid; g < G; g += PC_ROWS) sg_s[g] = (uint8_t)keep_bits(d, g);
    }
    __syncthreads();
    if (pipe && d + 1 < d1) load_next(d + 1);
    if (!live) continue;
    double acc = 0.0;
    uint32_t wn = lf[0];
    for (int g = 0; g < G; g++) {
      uint32_t w = wn;
      if (g + 1 < G) wn = lf[(g + 1) * PC_ROWS];   // the next group's offsets, loaded ahead
      const uint2 rr = *reinterpret_cast<const uint2*>(rt_s + 4 * g);
      const int r[4] = {(int)(rr.x & 0xFFFFu), (int)(rr.x >> 16), (int)(rr.y & 0xFFFFu), (int)(rr.y >> 16)};
      const uint32_t keep = sg_s[g];
      if (keep != 15u) {   // some structure changed (the flags are the CTA's, so the branch is uniform)
#pragma unroll
        for (int u = 0; u < 4; u++) {
          if (!((keep >> u) & 1u)) {
            int a = r[u];
            const int depth = td_s[4 * g + u];
            for (int st = 0; st < depth; st++) a = cstep(a, nd_s, cr);
            w = (w & ~(0xFFu << (8 * u))) | ((uint32_t)(a - r[u]) << (8 * u));
          }
        }
        lf[g * PC_ROWS] = w;
      }
      // the four leaf values, loaded together, then added in tree order
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) v[u] = th_s[r[u] + (int)((w >> (8 * u)) & 0xFFu)];
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (4 * g + u < m) acc = __dadd_rn(acc, v[u]);
    }
    out[(long long)d * ldo + i] = __dadd_rn(acc, mu);
  }
}

// Draws that share the structure of most trees with their predecessor make the carrying evaluator pay: on B200 it
// ran 1.19x the code-compare evaluator's rate with 85% of the trees shared (262,144 rows x 200 draws x 200 trees),
// and at 3 CTAs per SM (the leaf table's shared memory) it loses to it when few trees are shared.
__host__ __device__ inline bool carry_pays(const DForest& f) {
  return f.same && f.tdep && f.nsame * 5 >= 3 * (long long)f.ndpost * f.ntree;
}
size_t carry_smem(const DForest& f) {
  const size_t G = (size_t)(f.ntree + 3) / 4;
  return (((size_t)f.maxnd * 12 + 15) & ~(size_t)15) + G * PC_ROWS * 4 + G * 12 + ((G + 7) & ~(size_t)7) +
         (size_t)f.p * PC_ROWS;
}

int predict_evaluator(const DForest& f, int n, int ndraws) {
  (void)n;
  const size_t csmem = (size_t)f.maxnd * 12 + (size_t)f.p * PC_ROWS;
  if (f.n32 && f.gdepth && csmem <= 160 * 1024) {
    if (ndraws > 1 && carry_pays(f) && carry_smem(f) <= 200 * 1024) return 3;
    return 2;
  }
  if (f.p < PT_MAXP && f.nodes && f.gdepth) return 1;
  return 0;
}

int launch_predict(const DForest& f, const double* x, int n, int ld, int draw0, int ndraws, double mu, double* out,
                   int ldo, void* stream) {
  if (n <= 0 || ndraws <= 0) return 0;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int ev = predict_evaluator(f, n, ndraws);
  if (ev == 3) {
    const int tiles = (n + PC_ROWS - 1) / PC_ROWS;
    // one CTA per row tile and as long a range of draws as the SMs allow (every range starts with a full walk)
    const long long target = 2ll * nsm;
    const int chunks = (int)std::min<long long>(ndraws, std::max<long long>(1, (target + tiles - 1) / tiles));
    const int dpc = (ndraws + chunks - 1) / chunks;
    const int ny = (ndraws + dpc - 1) / dpc;
    const size_t smem = carry_smem(f);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(predict_carry_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
      return -1;
    predict_carry_kernel<<<dim3(tiles, ny), PC_ROWS, smem, st>>>(f, x, n, ld, draw0, ndraws, dpc, mu, out, ldo, f.p);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }
  const size_t csmem = (size_t)f.maxnd * 12 + (size_t)f.p * PC_ROWS;
  if (ev == 2) {
    const int tiles = (n + PC_ROWS - 1) / PC_ROWS;
    // enough CTAs for every SM (8 per SM), each taking a contiguous range of draws
    const long long target = 8ll * nsm;
    const int chunks = (int)std::min<long long>(ndraws, std::max<long long>(1, (target + tiles - 1) / tiles));
    const int dpc = (ndraws + chunks - 1) / chunks;
    const int ny = (ndraws + dpc - 1) / dpc;
    if (csmem > 48 * 1024 &&
        cudaFuncSetAttribute(predict_codes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)csmem) !=
            cudaSuccess)
      return -1;
    predict_codes_kernel<<<dim3(tiles, ny), PC_ROWS, csmem, st>>>(f, x, n, ld, draw0, ndraws, dpc, mu, out, ldo,
                                                                  f.p);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }
  if (ev == 1) {
    const int tiles = (n + PT_ROWS - 1) / PT_ROWS;
    // enough CTAs for every SM (16 per SM), each taking a contiguous range of draws
    const long long target = 16ll * nsm;
    const int chunks = (int)std::min<long long>(ndraws, std::max<long long>(1, (target + tiles - 1) / tiles));
    const int dpc = (ndraws + chunks - 1) / chunks;
    const int ny = (ndraws + dpc - 1) / dpc;
    const size_t smem = (size_t)(f.p + 1) * PT_ROWS * sizeof(double);
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(predict_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
      return -1;
    predict_tiled_kernel<<<dim3(tiles, ny), PT_ROWS, smem, st>>>(f, x, n, ld, draw0, ndraws, dpc, mu, out, ldo);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }
  const int T = 256;
  for (int d0 = 0; d0 < ndraws; d0 += 65535) {
    const int nd = ndraws - d0 < 65535 ? ndraws - d0 : 65535;
    dim3 grid((n + T - 1) / T, nd);
    predict_kernel<<<grid, T, 0, st>>>(f, x, n, ld, draw0 + d0, mu, out + (long long)d0 * ldo, ldo);
    if (cudaGetLastError() != cudaSuccess) return -1;
  }
  return 0;
}

// Cutpoint codes (the findInterval step of R/fwbart.R:19): q[v][i] = number of cutpoints of v that are <= x[v][i]
// (binary search; NaN gives 0), so that x < cut[v][c] <=> q <= c.  One thread per value, columns along grid y.
__global__ void cut_codes_kernel(const double* __restrict__ x, int n, const double* __restrict__ cuts,
                                 const int* __restrict__ cutoff, uint8_t* __restrict__ q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int v = blockIdx.y;
  if (i >= n) return;
  const double xv = x[(long long)v * n + i];
  const double* cv = cuts + cutoff[v];
  int lo = 0, hi = cutoff[v + 1] - cutoff[v];
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(cv + mid) <= xv) lo = mid + 1;
    else hi = mid;
  }
  q[(long long)v * n + i] = (uint8_t)lo;
}

int launch_cut_codes(const double* x, int n, int p, const double* cuts, const int* cutoff, uint8_t* q, void* stream) {
  if (n <= 0 || p <= 0) return 0;
  cut_codes_kernel<<<dim3((n + 255) / 256, p), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(x, n, cuts, cutoff,
                                                                                               q);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// Fixed device scratch of fb_predict_draw_static: the newdata columns and the result are staged here instead of in
// device memory allocated per call.  It belongs to the library's module, so every device that loads the library
// holds it until the process exits.  Nothing in it needs to start at zero: each call copies in all the columns it
// reads, and the kernel writes every result it returns.
static __device__ __align__(256) double g_predict_scratch[PREDICT_SCRATCH_DOUBLES];

namespace {
constexpr int kScratchDevices = 64;
std::atomic<double*> g_scratch_addr[kScratchDevices];
std::mutex g_scratch_mu;
}  // namespace

// Device address of the scratch on `device`, which must be the current device.  The first call on a device resolves
// it (host code only knows the array's host-side stand-in); later calls return the cached address.
int predict_scratch_address(int device, double** ptr) {
  if (device < 0 || device >= kScratchDevices) return -2;
  double* a = g_scratch_addr[device].load(std::memory_order_acquire);
  if (!a) {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    a = g_scratch_addr[device].load(std::memory_order_relaxed);
    if (!a) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_predict_scratch) != cudaSuccess || !p) return -1;
      a = static_cast<double*>(p);
      g_scratch_addr[device].store(a, std::memory_order_release);
    }
  }
  *ptr = a;
  return 0;
}

}  // namespace fb
