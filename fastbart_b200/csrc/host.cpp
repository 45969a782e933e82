// host.cpp -- C ABI of libfastbart_b200.so (include/fastbart_b200.h): batch set-up and transfers for the sampler
// kernel, BART tree-text assembly, compile_trees parsing and predict_draw launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../../include/fastbart_b200.h"
#include "fb_internal.h"

using namespace fb;

namespace {

thread_local std::string g_err;

fb_status fail(fb_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return s;
}

#define CK(call)                                                                                     \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess) return fail(FB_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));        \
  } while (0)

long long round_up(long long x, long long a) { return (x + a - 1) / a * a; }

// Fixed-point scales: every per-row term llrint(w*R*2^S) (and llrint(w*e^2*2^Srss)) summed over n rows stays below
// 2^61 even for residuals 64 times the data range.
void auto_shifts(const fb_chain& c, int* s, int* srss) {
  double wmax = 1.0, ymax = 10.0;
  if (c.wt) { wmax = 0.0; for (int i = 0; i < c.n; i++) wmax = std::max(wmax, c.wt[i]); }
  if (!c.probit && c.y) { ymax = 0.0; for (int i = 0; i < c.n; i++) ymax = std::max(ymax, std::fabs(c.y[i])); }
  const double rb = 64.0 * (ymax + 1.0);
  int a = 61 - (int)std::ceil(std::log2((double)c.n * std::max(wmax, 1e-300) * rb + 1.0));
  int b = 61 - (int)std::ceil(std::log2((double)c.n * std::max(wmax, 1e-300) * rb * rb + 1.0));
  *s = std::min(std::max(a, 8), 40);
  *srss = std::min(std::max(b, 0), 40);
}

fb_status check_chain(const fb_chain& c, int k) {
  if (c.n < 1 || c.p < 1 || c.ntree < 1) return fail(FB_ERR_ARG, "chain %d: n, p and ntree must be positive", k);
  if (c.n > NMAX) return fail(FB_ERR_LIMIT, "chain %d: n = %d exceeds %d rows", k, c.n, NMAX);
  if (c.p > PMAX) return fail(FB_ERR_LIMIT, "chain %d: p = %d exceeds %d predictors", k, c.p, PMAX);
  if (c.ntree > MMAX) return fail(FB_ERR_LIMIT, "chain %d: ntree = %d exceeds %d trees", k, c.ntree, MMAX);
  if (!c.q || !c.numcut || !c.pgtab) return fail(FB_ERR_ARG, "chain %d: q, numcut and pgtab are required", k);
  if (c.probit ? !c.ybin : !c.y) return fail(FB_ERR_ARG, "chain %d: %s is required", k, c.probit ? "ybin" : "y");
  int any = 0;
  for (int v = 0; v < c.p; v++) {
    if (c.numcut[v] < 0 || c.numcut[v] > 255)
      return fail(FB_ERR_LIMIT, "chain %d: numcut[%d] = %d is outside 0..255", k, v, c.numcut[v]);
    any |= c.numcut[v] > 0;
  }
  if (!any) return fail(FB_ERR_ARG, "chain %d: no predictor has a cutpoint", k);
  if (!(c.tau > 0) || !std::isfinite(c.tau)) return fail(FB_ERR_ARG, "chain %d: tau must be positive", k);
  if (!c.probit) {
    if (!(c.sigest > 0) || !std::isfinite(c.sigest)) return fail(FB_ERR_ARG, "chain %d: sigest must be positive", k);
    for (int i = 0; i < c.n; i++)
      if (!std::isfinite(c.y[i])) return fail(FB_ERR_ARG, "chain %d: y[%d] is not finite", k, i);
  }
  if (c.wt)
    for (int i = 0; i < c.n; i++)
      if (!(c.wt[i] >= 0) || !std::isfinite(c.wt[i])) return fail(FB_ERR_ARG, "chain %d: wt[%d] is invalid", k, i);
  return FB_OK;
}

// Device memory of batches comes from one pool per device that keeps what is freed (release threshold unlimited):
// a fit's arrays (1.5 GB for 96 titer chains) are then reused by the next fit instead of being unmapped by cudaFree
// and mapped again, which took 0.5-0.7 s per fit.  fb_release_cached_memory() returns the cache to the device.
std::mutex g_pool_mu;
std::unordered_map<int, cudaMemPool_t> g_pools;

cudaMemPool_t batch_pool(int device) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto it = g_pools.find(device);
  if (it != g_pools.end()) return it->second;
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof props);
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  g_pools[device] = pool;
  return pool;
}

// Narrowest CTA (whole warps, 256..512 threads) whose row threads hold a slice of `groups` 4-row groups in as few
// groups each as a 512-thread CTA does: the pass's longest thread is unchanged, while the barriers and the bin
// reductions span fewer warps.  Measured on B200: the titer chains (1,144 groups) run 3.6% faster on 416 threads.
int fitted_threads(int groups) {
  const int g = (groups + 479) / 480;   // groups per row thread at 512 threads
  if (g > 8) return 512;                 // rows streamed from L2: widest
  const int rt = ((groups + g - 1) / g + 31) / 32 * 32;
  return std::max(256, std::min(512, rt + 32));
}

// bytes from the batch pool, ordered on the legacy stream (the caller synchronises it before other streams use them);
// when the device is full, the pool's cache is trimmed and the allocation tried once more
void* pool_alloc(size_t bytes, int device) {
  cudaMemPool_t pool = batch_pool(device);
  if (!pool) return nullptr;
  void* p = nullptr;
  if (bytes == 0) bytes = 1;
  if (cudaMallocFromPoolAsync(&p, bytes, pool, 0) == cudaSuccess) return p;
  cudaGetLastError();
  cudaStreamSynchronize(0);
  cudaMemPoolTrimTo(pool, 0);
  if (cudaMallocFromPoolAsync(&p, bytes, pool, 0) == cudaSuccess) return p;
  cudaGetLastError();
  return nullptr;
}

}  // namespace

struct fb_batch {
  int device = 0, nchains = 0, nskip = 0, ndpost = 0;
  int threads = 256, grid = 0, spl = 0, launches = 0, gmax = 0;
  size_t smem = 0;
  std::vector<DChain> hch;
  std::vector<int> order;
  DBufs d{};
  std::vector<void*> allocs;
  long long rows = 0, qbytes = 0, leafbytes = 0, ntrees = 0, nsig = 0, nyhat = 0, ntout = 0;
  cudaStream_t stream = nullptr;
  void* model_mem = nullptr;   // learned proposal weights (owned; also listed in allocs)
  int* mvar = nullptr;         // learned proposal: per-tree choices of the current sweep (owned)
  size_t smem_model = 0;       // the sampler's shared memory of model, cut and collecting launches (update_launch)
  int rows_plain = 1;          // rows in shared memory in the plain layout
  void* cut_mem = nullptr;     // the cut head's weight image (owned; also listed in allocs)
  int cut_cap = 0;             // allocated capacity of the cut-example buffers
  double* mcorr = nullptr;
  int cluster = 1;             // CTAs per chain
  int slice_rows = 0;          // rows of one CTA's slice (shared-memory capacity)
  int collect_cap = 0;         // allocated capacity of the training-example buffers
  // n elements of T from the batch pool, owned by the batch; null when the device is full
  template <class T>
  T* alloc(size_t n) {
    void* p = pool_alloc(n * sizeof(T), device);
    if (p) allocs.push_back(p);
    return static_cast<T*>(p);
  }
  cudaEvent_t done = nullptr;  // recorded on the caller's stream after every run's launches
  int autotuned = 0;           // the launch shape came from the autotuner
  ~fb_batch() {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    // the last run may still be in flight on the caller's stream: wait for it alone, not for the whole device
    if (done) { cudaEventSynchronize(done); cudaEventDestroy(done); }
    for (void* p : allocs) cudaFreeAsync(p, 0);
    cudaStreamSynchronize(0);
    cudaSetDevice(cur);
  }
};

extern "C" {

const char* fb_last_error(void) { return g_err.c_str(); }
const char* fb_version(void) { return "fastbart_b200 0.1.0 (sm_100a)"; }

}  // extern "C"

namespace {
// Launch shapes chosen by the autotuner, per device and batch signature, for the life of the process.
std::mutex g_tune_mu;
std::unordered_map<std::string, std::pair<int, int>> g_tuned;

std::string batch_signature(const fb_chain* chains, int nchains, int device) {
  long long rows = 0, trees = 0;
  int nmax = 0, mmax = 0, pmax = 0, probit = 0;
  for (int k = 0; k < nchains; k++) {
    rows += chains[k].n; trees += chains[k].ntree; probit += chains[k].probit ? 1 : 0;
    nmax = std::max(nmax, chains[k].n); mmax = std::max(mmax, chains[k].ntree); pmax = std::max(pmax, chains[k].p);
  }
  char buf[160];
  std::snprintf(buf, sizeof buf, "%d:%d:%lld:%lld:%d:%d:%d:%d", device, nchains, rows, trees, nmax, mmax, pmax, probit);
  return buf;
}

// Shared memory and staging of the batch's model, cut and collecting launches: the cut layout (per-tree ratios,
// scratch, one more bin row) when a cut head or collection is set, the proposal model's image behind the layout when
// the bins cannot hold it, then the cut head's image, each staged only while every CTA of the launch stays resident
// (else read from global memory); rows move to global memory when the cut layout cannot keep them in shared memory.
fb_status update_launch(fb_batch* b) {
  DBufs& d = b->d;
  const bool special = d.mvar || d.cimg || d.train_cap > 0;
  d.rows_in_smem = b->rows_plain;
  d.model_smem = 0; d.cut_smem = 0;
  b->smem_model = b->smem;
  if (!special) return FB_OK;
  int optin = 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device) != cudaSuccess) optin = 0;
  const int cutl = (d.cimg || d.train_cap > 0) ? 1 : 0;
  size_t base = sampler_smem_bytes(b->threads, d.m_max, d.n_pad_max, d.rows_in_smem, b->cluster, cutl);
  auto resident = [&](size_t sm) {
    return sm <= (size_t)optin && sampler_max_grid(b->threads, sm, b->device, b->gmax, b->cluster) >= b->grid;
  };
  if (!resident(base) && d.rows_in_smem == 1) {   // the weights to global memory
    d.rows_in_smem = 2;
    base = sampler_smem_bytes(b->threads, d.m_max, d.n_pad_max, 2, b->cluster, cutl);
  }
  if (!resident(base) && d.rows_in_smem == 2) {   // and the residuals
    d.rows_in_smem = 0;
    base = sampler_smem_bytes(b->threads, d.m_max, d.n_pad_max, 0, b->cluster, cutl);
  }
  if (!resident(base)) return fail(FB_ERR_LIMIT, "shared memory %zu of the learned proposal's layout does not fit", base);
  size_t sm = (base + 15) / 16 * 16;
  if (d.mvar && !sampler_bins_hold_model(b->threads) && resident(sm + 4 * (size_t)MIMG_WORDS)) {
    d.model_smem = 1;
    sm += 4 * (size_t)MIMG_WORDS;
  }
  if (d.cimg && resident(sm + 4 * (size_t)CIMG_WORDS)) {
    d.cut_smem = 1;
    sm += 4 * (size_t)CIMG_WORDS;
  }
  b->smem_model = sm;
  return FB_OK;
}

// whether an automatic launch shape (threads = cluster = 0) is picked by the autotuner (default) or by the measured
// rules of fb_batch_create (FASTBART_AUTOTUNE=0)
bool autotune_by_default() {
  const char* e = std::getenv("FASTBART_AUTOTUNE");
  return !(e && e[0] == '0');
}
}  // namespace

extern "C" {

fb_status fb_batch_create(const fb_chain* chains, int nchains, const fb_options* opt, fb_batch** out) {
  if (!out) return fail(FB_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!chains || nchains < 1 || !opt) return fail(FB_ERR_ARG, "chains, nchains >= 1 and opt are required");
  if (opt->nskip < 0 || opt->ndpost < 1) return fail(FB_ERR_ARG, "nskip must be >= 0 and ndpost >= 1");
  if (opt->threads != 0 && (opt->threads < MIN_THREADS || opt->threads > MAX_THREADS || opt->threads % 32))
    return fail(FB_ERR_ARG, "threads must be a multiple of 32 in %d..%d", MIN_THREADS, MAX_THREADS);
  for (int k = 0; k < nchains; k++) {
    fb_status s = check_chain(chains[k], k);
    if (s != FB_OK) return s;
  }
  // automatic shape: the autotuner's choice for this batch signature (timed once per process), else the rules below
  if (opt->threads == 0 && opt->cluster == 0 && autotune_by_default()) {
    const std::string sig = batch_signature(chains, nchains, opt->device);
    std::pair<int, int> shape{0, 0};
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tuned.find(sig);
      if (it != g_tuned.end()) shape = it->second;
    }
    if (shape.first == 0) {
      fb_options best;
      if (fb_autotune(chains, nchains, opt, 2, &best, nullptr) == FB_OK) {
        shape = {best.threads, best.cluster};
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[sig] = shape;
      } else {
        g_err.clear();   // no trial shape worked: the rules decide
      }
    }
    if (shape.first > 0) {
      fb_options o = *opt;
      o.threads = shape.first; o.cluster = shape.second;
      fb_status s = fb_batch_create(chains, nchains, &o, out);
      if (s == FB_OK) (*out)->autotuned = 1;
      return s;
    }
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FB_ERR_CUDA, "no CUDA device is available");
  if (opt->device < 0 || opt->device >= ndev) return fail(FB_ERR_ARG, "device %d does not exist", opt->device);
  CK(cudaSetDevice(opt->device));

  auto* b = new fb_batch();
  b->device = opt->device; b->nchains = nchains; b->nskip = opt->nskip; b->ndpost = opt->ndpost;
  const int S = opt->nskip + opt->ndpost;
  b->hch.resize(nchains);
  int m_max = 0, n_pad_max = 0;
  for (int k = 0; k < nchains; k++) {
    const fb_chain& c = chains[k];
    DChain& D = b->hch[k];
    std::memset(&D, 0, sizeof D);
    D.n = c.n; D.p = c.p; D.m = c.ntree; D.n_pad = (int)round_up(c.n, 16);
    D.probit = c.probit ? 1 : 0;
    int s1, s2;
    auto_shifts(c, &s1, &s2);
    D.fx_shift = c.fx_shift > 0 ? c.fx_shift : s1;
    D.rss_shift = c.rss_shift > 0 ? c.rss_shift : s2;
    int rn = 0;
    for (int v = 0; v < c.p; v++) { D.numcut[v] = c.numcut[v]; rn += c.numcut[v] >= 1; }
    D.root_ngv = rn;
    D.nskip = opt->nskip; D.ndpost = opt->ndpost;
    D.tau = c.tau; D.lambda = c.lambda; D.nu = c.nu; D.sigest = c.probit ? (c.sigest > 0 ? c.sigest : 1.0) : c.sigest;
    D.offset = c.offset;
    for (int d = 0; d < NODES; d++) D.pg[d] = c.pgtab[d];
    D.seed = c.seed;
    D.off_row = b->rows; D.off_q = b->qbytes; D.off_leaf = b->leafbytes; D.off_tree = b->ntrees;
    D.off_sigma = b->nsig; D.off_yhat = b->nyhat; D.off_tout = b->ntout;
    b->rows += D.n_pad; b->qbytes += (long long)c.p * D.n_pad; b->leafbytes += (long long)c.ntree * D.n_pad;
    b->ntrees += c.ntree; b->nsig += S; b->nyhat += (long long)opt->ndpost * c.n;
    b->ntout += (long long)opt->ndpost * c.ntree * NODES;
    m_max = std::max(m_max, c.ntree); n_pad_max = std::max(n_pad_max, D.n_pad);
  }
  // largest chains first (n * ntree), then the queue hands them out as CTAs free up
  b->order.resize(nchains);
  for (int k = 0; k < nchains; k++) b->order[k] = k;
  std::stable_sort(b->order.begin(), b->order.end(), [&](int a, int c) {
    return (long long)b->hch[a].n * b->hch[a].m > (long long)b->hch[c].n * b->hch[c].m;
  });

  // launch shape
  int T = opt->threads;
  bool fit_width = false;   // automatic width for one chain (or cluster) per SM: fitted to the slice below
  if (T == 0) {
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, opt->device);
    T = nchains <= nsm ? 512 : 256;   // one chain per SM: wide CTA; more chains than SMs: two CTAs per SM
    fit_width = nchains <= nsm;
  }
  int optin = 0, nsm = 148;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, opt->device) != cudaSuccess) optin = 232448;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, opt->device);
  // CTAs per chain: a cluster splits each chain's rows over CS SMs when SMs would otherwise idle (or as requested)
  // Automatic choice (measured on B200): the largest cluster of 4..16 CTAs whose clusters are all resident at once,
  // one per chain, when there are SMs to spare and at least 512 rows per CTA; otherwise one CTA per chain.  (Sizes
  // above 8 are non-portable; B200 keeps up to 15 clusters of 7..9 CTAs, 7 of 12..16, resident.)
  std::vector<int> tries;
  if (opt->cluster > 0) tries.push_back(std::min(opt->cluster, 16));
  else {
    for (int c = 16; c >= 4; c--)
      if ((long long)nchains * c <= nsm && n_pad_max / c >= 512) tries.push_back(c);
  }
  tries.push_back(1);
  int CS = 1, rows_in_smem = 1, gmax = 0, maxgrid = 0;
  size_t smem = 0;
  const int T_req = T;
  for (size_t ti = 0; ti < tries.size(); ti++) {
    CS = tries[ti];
    const int cap = 4 * ((n_pad_max / 4 + CS - 1) / CS);   // rows of one CTA's slice
    T = fit_width ? fitted_threads(cap / 4) : T_req;
    rows_in_smem = 1;
    smem = sampler_smem_bytes(T, m_max, cap, 1, CS);
    if (smem > (size_t)optin) { rows_in_smem = 0; smem = sampler_smem_bytes(T, m_max, cap, 0, CS); }
    if (smem > (size_t)optin) { delete b; return fail(FB_ERR_LIMIT, "shared memory %zu exceeds %d", smem, optin); }
    gmax = sampler_gmax(T, cap);
    maxgrid = sampler_max_grid(T, smem, opt->device, gmax, CS);   // CTAs (whole clusters) that can be resident
    const bool all_resident = maxgrid >= nchains * CS;
    if (CS == 1 || (maxgrid > 0 && (opt->cluster > 0 || all_resident))) { b->slice_rows = cap; break; }
  }
  if (maxgrid <= 0) { delete b; return fail(FB_ERR_CUDA, "sampler kernel cannot be resident with %zu bytes of shared memory", smem); }
  b->cluster = CS;
  b->threads = T; b->smem = smem; b->grid = std::min(nchains * CS, maxgrid); b->gmax = gmax;
  b->rows_plain = rows_in_smem; b->smem_model = smem;
  b->spl = opt->sweeps_per_launch > 0 ? opt->sweeps_per_launch : S;
  b->launches = (S + b->spl - 1) / b->spl;

  // device arrays
  DBufs& d = b->d;
  auto A = [&](auto** p, size_t cnt) -> fb_status {
    using T = std::remove_pointer_t<std::remove_pointer_t<decltype(p)>>;
    *p = b->alloc<T>(cnt);
    return *p ? FB_OK : fail(FB_ERR_CUDA, "out of device memory (%zu elements)", cnt);
  };
  DChain* dch; DState* dst; uint8_t* dq; double* dyin; double* dyw; float* dw; int8_t* dyb; float* drs; float* dws;
  uint8_t* dleaf;
  DTree* dtr; long long* ds0; float* dth; double* dtm; double* dsig; double* dyh; unsigned long long* dto; int* dord;
  int* dqueue;
  fb_status s = FB_OK;
  if ((s = A(&dch, nchains)) || (s = A(&dst, nchains)) || (s = A(&dq, b->qbytes)) || (s = A(&dyin, b->rows)) ||
      (s = A(&dyw, b->rows)) || (s = A(&dw, b->rows)) || (s = A(&dyb, b->rows)) || (s = A(&drs, b->rows)) || (s = A(&dws, b->rows)) ||
      (s = A(&dleaf, b->leafbytes)) || (s = A(&dtr, b->ntrees * CS)) ||
      (s = A(&ds0, b->ntrees * CS * LEAF_STAT_WORDS)) || (s = A(&dth, b->ntrees * CS * NODES)) || (s = A(&dtm, b->rows)) || (s = A(&dsig, b->nsig)) ||
      (s = A(&dyh, b->nyhat)) || (s = A(&dto, b->ntout)) || (s = A(&dord, nchains)) || (s = A(&dqueue, 1))) {
    delete b;
    return s;
  }
  CK(cudaStreamSynchronize(0));   // the pool allocations are complete before any stream of the caller uses them
  // inputs, padded rows are zero
  std::vector<uint8_t> hq((size_t)b->qbytes, 0);
  std::vector<double> hy((size_t)b->rows, 0.0);
  std::vector<float> hw((size_t)b->rows, 0.0f);
  std::vector<int8_t> hyb((size_t)b->rows, 0);
  for (int k = 0; k < nchains; k++) {
    const fb_chain& c = chains[k];
    const DChain& D = b->hch[k];
    for (int v = 0; v < c.p; v++) std::memcpy(&hq[(size_t)D.off_q + (size_t)v * D.n_pad], c.q + (size_t)v * c.n, (size_t)c.n);
    for (int i = 0; i < c.n; i++) {
      hy[(size_t)D.off_row + i] = c.probit ? 0.0 : c.y[i];
      hw[(size_t)D.off_row + i] = c.wt ? (float)c.wt[i] : 1.0f;
      hyb[(size_t)D.off_row + i] = c.probit ? (int8_t)(c.ybin[i] != 0) : 0;
    }
  }
  std::vector<DState> hst(nchains);
  std::memset(hst.data(), 0, sizeof(DState) * nchains);
  CK(cudaMemcpy(dch, b->hch.data(), sizeof(DChain) * nchains, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dst, hst.data(), sizeof(DState) * nchains, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dq, hq.data(), hq.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dyin, hy.data(), hy.size() * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dw, hw.data(), hw.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dyb, hyb.data(), hyb.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dord, b->order.data(), sizeof(int) * nchains, cudaMemcpyHostToDevice));
  d.chains = dch; d.states = dst; d.q = dq; d.yin = dyin; d.ywork = dyw; d.win = dw; d.ybin = dyb; d.rsave = drs; d.wsave = dws;
  d.leaf = dleaf; d.trees = dtr; d.s0 = ds0; d.th = dth; d.tm = dtm; d.sigma_out = dsig; d.yhat_out = dyh;
  d.trees_out = dto; d.order = dord; d.queue = dqueue; d.nchains = nchains; d.m_max = m_max;
  d.n_pad_max = b->slice_rows; d.rows_in_smem = rows_in_smem; d.cluster = CS;
  *out = b;
  return FB_OK;
}

fb_status fb_batch_run(fb_batch* b, void* stream) {
  if (!b) return fail(FB_ERR_ARG, "batch is NULL");
  CK(cudaSetDevice(b->device));
  b->stream = reinterpret_cast<cudaStream_t>(stream);
  const int S = b->nskip + b->ndpost;
  if (b->d.train_cap > 0 && cudaMemsetAsync(b->d.train_count, 0, sizeof(int), b->stream) != cudaSuccess)
    return fail(FB_ERR_CUDA, "cannot reset the training-example counter");
  for (int it0 = 0; it0 < S; it0 += b->spl) {
    const int it1 = std::min(S, it0 + b->spl);
    const bool special = b->d.mvar || b->d.cimg || b->d.train_cap > 0;
    if (launch_sampler(b->d, it0, it1, b->threads, b->grid, special ? b->smem_model : b->smem, b->gmax, b->cluster,
                       stream) != 0)
      return fail(FB_ERR_CUDA, "sampler launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  if (!b->done && cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess) {
    b->done = nullptr;
    return fail(FB_ERR_CUDA, "cannot create the batch's completion event");
  }
  CK(cudaEventRecord(b->done, b->stream));
  return FB_OK;
}

fb_status fb_autotune(const fb_chain* chains, int nchains, const fb_options* opt, int trial_sweeps, fb_options* best,
                      double* best_ms) {
  if (!chains || nchains < 1 || !opt || !best) return fail(FB_ERR_ARG, "chains, nchains >= 1, opt and best are required");
  if (trial_sweeps < 2) return fail(FB_ERR_ARG, "trial_sweeps must be >= 2");
  int ndev = 0, nsm = 148;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FB_ERR_CUDA, "no CUDA device is available");
  CK(cudaSetDevice(opt->device));
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, opt->device);
  std::vector<int> clusters{1};
  for (int c = 2; c <= 16; c++)
    if ((long long)nchains * c <= nsm) clusters.push_back(c);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  double bestt = 1e300;
  fb_options keep = *opt;
  for (int T : {256, 384, 416, 448, 512}) {
    for (int c : clusters) {
      fb_options o = *opt;
      o.nskip = trial_sweeps - 1; o.ndpost = 1; o.threads = T; o.cluster = c; o.sweeps_per_launch = 0;
      fb_batch* b = nullptr;
      if (fb_batch_create(chains, nchains, &o, &b) != FB_OK) continue;   // shape not possible here
      // only shapes whose clusters are all resident at once (a second wave is never the fastest)
      if (b->cluster != c || (c > 1 && b->grid < nchains * c)) { fb_batch_destroy(b); continue; }
      float ms = 0.0f;
      const bool ok = fb_batch_run(b, nullptr) == FB_OK && cudaEventRecord(e0) == cudaSuccess &&
                      fb_batch_run(b, nullptr) == FB_OK && cudaEventRecord(e1) == cudaSuccess &&
                      cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
      fb_batch_destroy(b);
      if (!ok) { cudaEventDestroy(e0); cudaEventDestroy(e1); return fail(FB_ERR_CUDA, "trial run failed"); }
      if (ms < bestt) { bestt = ms; keep = *opt; keep.threads = T; keep.cluster = c; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (bestt == 1e300) return fail(FB_ERR_CUDA, "no launch shape could be created");
  *best = keep;
  if (best_ms) *best_ms = bestt;
  return FB_OK;
}

fb_status fb_batch_set_proposal(fb_batch* b, const fb_proposal_model* model) {
  if (!b) return fail(FB_ERR_ARG, "batch is NULL");
  CK(cudaSetDevice(b->device));
  if (!model || model->mix <= 0.0) {
    b->d.mvar = nullptr; b->d.mcorr = nullptr; b->d.mix = 0.0;
    return update_launch(b);
  }
  if (!model->w1 || !model->b1 || !model->w2 || !model->b2 || !model->w3 || !model->b3)
    return fail(FB_ERR_ARG, "every weight and bias array of the model is required");
  if (!(model->mix <= 1.0)) return fail(FB_ERR_ARG, "mix must be in (0, 1]");
  // the sampler's weight image (MIMG_* in fb_internal.h): BF16 pairs row by row, padded rows, then the biases
  std::vector<uint32_t> img(MIMG_WORDS, 0u);
  auto pair = [](const uint16_t* row, int kk) { return (uint32_t)row[2 * kk] | ((uint32_t)row[2 * kk + 1] << 16); };
  for (int o = 0; o < MLP_H; o++)
    for (int kk = 0; kk < MLP_IN / 2; kk++) img[o * MIMG_W1S + kk] = pair(model->w1 + o * MLP_IN, kk);
  for (int o = 0; o < MLP_H; o++)
    for (int kk = 0; kk < MLP_H / 2; kk++) img[MIMG_W2 + o * MIMG_W2S + kk] = pair(model->w2 + o * MLP_H, kk);
  for (int o = 0; o < MLP_OUT; o++)
    for (int kk = 0; kk < MLP_H / 2; kk++) img[MIMG_W3 + o * MIMG_W2S + kk] = pair(model->w3 + o * MLP_H, kk);
  std::memcpy(img.data() + MIMG_B, model->b1, 4 * MLP_H);
  std::memcpy(img.data() + MIMG_B + MLP_H, model->b2, 4 * MLP_H);
  std::memcpy(img.data() + MIMG_B + 2 * MLP_H, model->b3, 4 * MLP_OUT);
  if (!b->model_mem && !(b->model_mem = b->alloc<uint32_t>(img.size()))) return fail(FB_ERR_CUDA, "out of device memory");
  if (!b->mvar) {
    b->mvar = b->alloc<int>((size_t)b->ntrees);
    b->mcorr = b->alloc<double>((size_t)b->ntrees);
    if (!b->mvar || !b->mcorr) { b->mvar = nullptr; return fail(FB_ERR_CUDA, "out of device memory"); }
  }
  CK(cudaStreamSynchronize(0));
  CK(cudaMemcpy(b->model_mem, img.data(), 4 * img.size(), cudaMemcpyHostToDevice));
  b->d.mimg = static_cast<const uint32_t*>(b->model_mem);
  b->d.mix = model->mix;
  b->d.mvar = b->mvar; b->d.mcorr = b->mcorr;
  return update_launch(b);
}

fb_status fb_batch_collect(fb_batch* b, int capacity) {
  if (!b) return fail(FB_ERR_ARG, "batch is NULL");
  if (capacity < 0) return fail(FB_ERR_ARG, "capacity must be >= 0");
  CK(cudaSetDevice(b->device));
  if (capacity > b->collect_cap) {
    float* feat = b->alloc<float>((size_t)MLP_IN * b->ntrees);
    unsigned* fv = b->alloc<unsigned>((size_t)b->ntrees);
    float* tx = b->alloc<float>((size_t)MLP_IN * capacity);
    int* ty = b->alloc<int>((size_t)capacity);
    unsigned* tm = b->alloc<unsigned>((size_t)capacity);
    int* tc = b->alloc<int>(1);
    if (!feat || !fv || !tx || !ty || !tm || !tc) return fail(FB_ERR_CUDA, "out of device memory");
    CK(cudaStreamSynchronize(0));
    b->d.feat = static_cast<float*>(feat); b->d.feat_valid = static_cast<unsigned*>(fv);
    b->d.train_x = static_cast<float*>(tx); b->d.train_y = static_cast<int*>(ty);
    b->d.train_mask = static_cast<unsigned*>(tm); b->d.train_count = static_cast<int*>(tc);
    b->collect_cap = capacity;
  }
  if (capacity > b->cut_cap) {   // the cut examples of the same births
    float* cf = b->alloc<float>((size_t)CUT_IN * b->ntrees);
    int* ci = b->alloc<int>((size_t)3 * b->ntrees);
    float* cx = b->alloc<float>((size_t)CUT_IN * capacity);
    int* cc = b->alloc<int>((size_t)capacity);
    int* clo = b->alloc<int>((size_t)capacity);
    int* chi = b->alloc<int>((size_t)capacity);
    if (!cf || !ci || !cx || !cc || !clo || !chi) return fail(FB_ERR_CUDA, "out of device memory");
    CK(cudaStreamSynchronize(0));
    b->d.cfeat = cf; b->d.cinfo = ci; b->d.train_cx = cx; b->d.train_c = cc; b->d.train_lo = clo; b->d.train_hi = chi;
    b->cut_cap = capacity;
  }
  b->d.train_cap = capacity;
  return update_launch(b);
}

fb_status fb_batch_set_cut_proposal(fb_batch* b, const fb_cut_model* model) {
  if (!b) return fail(FB_ERR_ARG, "batch is NULL");
  CK(cudaSetDevice(b->device));
  if (!model || model->mix <= 0.0) {
    b->d.cimg = nullptr; b->d.cmix = 0.0;
    return update_launch(b);
  }
  if (!model->w1 || !model->b1 || !model->w2 || !model->b2 || !model->w3 || !model->b3 || !model->emb || !model->be)
    return fail(FB_ERR_ARG, "every weight and bias array of the cut model is required");
  if (!(model->mix <= 1.0)) return fail(FB_ERR_ARG, "mix must be in (0, 1]");
  if (b->threads < 256) return fail(FB_ERR_LIMIT, "the cut proposal needs CTAs of at least 256 threads (%d)", b->threads);
  // the sampler's image (CIMG_* in fb_internal.h): BF16 pairs row by row in odd-length rows, then the biases
  std::vector<uint32_t> img(CIMG_WORDS, 0u);
  auto pack = [&](const uint16_t* w, int rows, int cols, int base, int stride) {
    for (int o = 0; o < rows; o++)
      for (int k = 0; k < cols; k++) {
        const uint32_t h = w[o * cols + k];
        img[base + o * stride + k / 2] |= (k & 1) ? (h << 16) : h;
      }
  };
  pack(model->w1, CUT_H, CUT_IN, 0, CIMG_W1S);
  pack(model->w2, CUT_H, CUT_H, CIMG_W2, CIMG_W2S);
  pack(model->w3, CUT_E, CUT_H, CIMG_W3, CIMG_W2S);
  pack(model->emb, CUT_BINS, CUT_E, CIMG_EMB, CIMG_ES);
  std::memcpy(img.data() + CIMG_B, model->b1, 4 * CUT_H);
  std::memcpy(img.data() + CIMG_B + CUT_H, model->b2, 4 * CUT_H);
  std::memcpy(img.data() + CIMG_B + 2 * CUT_H, model->b3, 4 * CUT_E);
  std::memcpy(img.data() + CIMG_B + 2 * CUT_H + CUT_E, model->be, 4 * CUT_BINS);
  if (!b->cut_mem && !(b->cut_mem = b->alloc<uint32_t>(img.size()))) return fail(FB_ERR_CUDA, "out of device memory");
  CK(cudaStreamSynchronize(0));
  CK(cudaMemcpy(b->cut_mem, img.data(), 4 * img.size(), cudaMemcpyHostToDevice));
  b->d.cimg = static_cast<const uint32_t*>(b->cut_mem);
  b->d.cmix = model->mix;
  return update_launch(b);
}

fb_status fb_batch_cut_training_data(fb_batch* b, float* x, int* c, int* lo, int* hi, int cap, int* count) {
  if (!b || !count) return fail(FB_ERR_ARG, "batch and count are required");
  CK(cudaSetDevice(b->device));
  *count = 0;
  if (b->d.train_cap <= 0 || !b->d.train_cx) return FB_OK;
  CK(cudaStreamSynchronize(b->stream));
  int total = 0;
  CK(cudaMemcpy(&total, b->d.train_count, sizeof(int), cudaMemcpyDeviceToHost));
  *count = total;
  const int k = std::min(std::min(total, b->d.train_cap), std::max(cap, 0));
  if (k > 0) {
    if (x) CK(cudaMemcpy(x, b->d.train_cx, sizeof(float) * CUT_IN * (size_t)k, cudaMemcpyDeviceToHost));
    if (c) CK(cudaMemcpy(c, b->d.train_c, sizeof(int) * (size_t)k, cudaMemcpyDeviceToHost));
    if (lo) CK(cudaMemcpy(lo, b->d.train_lo, sizeof(int) * (size_t)k, cudaMemcpyDeviceToHost));
    if (hi) CK(cudaMemcpy(hi, b->d.train_hi, sizeof(int) * (size_t)k, cudaMemcpyDeviceToHost));
  }
  return FB_OK;
}

fb_status fb_batch_training_data(fb_batch* b, float* x, int* y, uint32_t* mask, int cap, int* count) {
  if (!b || !count) return fail(FB_ERR_ARG, "batch and count are required");
  CK(cudaSetDevice(b->device));
  *count = 0;
  if (b->d.train_cap <= 0) return FB_OK;
  CK(cudaStreamSynchronize(b->stream));
  int total = 0;
  CK(cudaMemcpy(&total, b->d.train_count, sizeof(int), cudaMemcpyDeviceToHost));
  *count = total;
  const int k = std::min(std::min(total, b->d.train_cap), std::max(cap, 0));
  if (k > 0) {
    if (x) CK(cudaMemcpy(x, b->d.train_x, sizeof(float) * MLP_IN * (size_t)k, cudaMemcpyDeviceToHost));
    if (y) CK(cudaMemcpy(y, b->d.train_y, sizeof(int) * (size_t)k, cudaMemcpyDeviceToHost));
    if (mask) CK(cudaMemcpy(mask, b->d.train_mask, sizeof(uint32_t) * (size_t)k, cudaMemcpyDeviceToHost));
  }
  return FB_OK;
}

fb_status fb_batch_sync(fb_batch* b) {
  if (!b) return fail(FB_ERR_ARG, "batch is NULL");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaGetLastError());
  return FB_OK;
}

int fb_batch_autotuned(const fb_batch* b) { return b ? b->autotuned : 0; }

fb_status fb_batch_launch_info(const fb_batch* b, int* launches, int* threads, int* grid, size_t* smem_bytes,
                               int* cluster) {
  if (!b) return fail(FB_ERR_ARG, "batch is NULL");
  if (launches) *launches = b->launches;
  if (threads) *threads = b->threads;
  if (grid) *grid = b->grid;
  if (smem_bytes) *smem_bytes = b->smem;
  if (cluster) *cluster = b->cluster;
  return FB_OK;
}

fb_status fb_batch_download(fb_batch* b, fb_chain_out* outs) {
  if (!b || !outs) return fail(FB_ERR_ARG, "batch and outs are required");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  std::vector<DState> st(b->nchains);
  CK(cudaMemcpy(st.data(), b->d.states, sizeof(DState) * b->nchains, cudaMemcpyDeviceToHost));
  for (int k = 0; k < b->nchains; k++)
    if (st[k].status != 0)
      return fail(FB_ERR_CUDA, "chain %d: a bounded wait of the sampler on its own leaf-statistics copy gave up", k);
  const int S = b->nskip + b->ndpost;
  std::vector<double> tm;
  for (int k = 0; k < b->nchains; k++) {
    const DChain& D = b->hch[k];
    fb_chain_out& o = outs[k];
    if (o.sigma) CK(cudaMemcpy(o.sigma, b->d.sigma_out + D.off_sigma, sizeof(double) * S, cudaMemcpyDeviceToHost));
    if (o.yhat)
      CK(cudaMemcpy(o.yhat, b->d.yhat_out + D.off_yhat, sizeof(double) * (size_t)b->ndpost * D.n, cudaMemcpyDeviceToHost));
    if (o.trees)
      CK(cudaMemcpy(o.trees, b->d.trees_out + D.off_tout, sizeof(uint64_t) * (size_t)b->ndpost * D.m * NODES,
                    cudaMemcpyDeviceToHost));
    if (o.yhat_mean) {
      CK(cudaMemcpy(o.yhat_mean, b->d.tm + D.off_row, sizeof(double) * D.n, cudaMemcpyDeviceToHost));
      for (int i = 0; i < D.n; i++) o.yhat_mean[i] = o.yhat_mean[i] / (double)b->ndpost;
    }
    o.moves[0] = st[k].births; o.moves[1] = st[k].deaths; o.moves[2] = st[k].caps;
    o.rtnorm_caps = st[k].rtcaps;
  }
  return FB_OK;
}

void fb_batch_destroy(fb_batch* b) { delete b; }

fb_status fb_release_cached_memory(int device) {
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pools.find(device);
    if (it == g_pools.end()) return FB_OK;
    pool = it->second;
  }
  CK(cudaSetDevice(device));
  CK(cudaStreamSynchronize(0));
  CK(cudaMemPoolTrimTo(pool, 0));
  return FB_OK;
}

fb_status fb_fit_batch(const fb_chain* chains, int nchains, const fb_options* opt, fb_chain_out* outs) {
  fb_batch* b = nullptr;
  fb_status s = fb_batch_create(chains, nchains, opt, &b);
  if (s != FB_OK) return s;
  s = fb_batch_run(b, nullptr);
  if (s == FB_OK) s = fb_batch_sync(b);
  if (s == FB_OK) s = fb_batch_download(b, outs);
  fb_batch_destroy(b);
  return s;
}

// ------------------------------------------------------------------------------------------------ tree text
size_t fb_trees_text(const uint64_t* trees, int ndpost, int ntree, int p, char* buf, size_t cap) {
  std::string s;
  s.reserve((size_t)ndpost * ntree * 64);
  char line[128];
  int k = std::snprintf(line, sizeof line, "%d %d %d\n", ndpost, ntree, p);
  s.append(line, (size_t)k);
  std::vector<std::pair<int, unsigned long long>> stack, order;
  for (int dr = 0; dr < ndpost; dr++)
    for (int j = 0; j < ntree; j++) {
      const uint64_t* T = trees + ((size_t)dr * ntree + j) * NODES;
      auto L = [&](int x) { return (int)((T[x] >> 16) & 255); };
      auto R = [&](int x) { return (int)((T[x] >> 24) & 255); };
      stack.assign(1, {0, 1ull});
      order.clear();
      while (!stack.empty() && order.size() <= (size_t)NODES) {   // pre-order: node, left subtree, right subtree
        auto e = stack.back();
        stack.pop_back();
        order.push_back(e);
        if (L(e.first)) { stack.push_back({R(e.first), 2 * e.second + 1}); stack.push_back({L(e.first), 2 * e.second}); }
      }
      k = std::snprintf(line, sizeof line, "%zu\n", order.size());
      s.append(line, (size_t)k);
      for (auto& e : order) {
        const uint64_t w = T[e.first];
        const bool leaf = L(e.first) == 0;
        float th;
        const uint32_t u = (uint32_t)(w >> 32);
        std::memcpy(&th, &u, 4);
        k = std::snprintf(line, sizeof line, "%llu %d %d %.10g\n", e.second, leaf ? 0 : (int)(w & 255),
                          leaf ? 0 : (int)((w >> 8) & 255), leaf ? (double)th : 0.0);
        s.append(line, (size_t)k);
      }
    }
  if (buf && cap > 0) {
    const size_t c = std::min(cap - 1, s.size());
    std::memcpy(buf, s.data(), c);
    buf[c] = 0;
  }
  return s.size();
}

}  // extern "C"

// Header plus the device-assembled text of ndpost x ntree device trees into buf (the fb_trees_text contract).
static fb_status text_from_device(const uint64_t* d_trees, int ndpost, int ntree, int p, char* buf, size_t cap,
                                  size_t* len) {
  char head[64];
  const int hl = std::snprintf(head, sizeof head, "%d %d %d\n", ndpost, ntree, p);
  unsigned long long body = 0;
  char* d_text = nullptr;
  const bool want = buf && cap > 0;
  if (trees_text_device(d_trees, (long long)ndpost * ntree, want ? &d_text : nullptr, &body, nullptr) != 0)
    return fail(FB_ERR_CUDA, "tree text kernels failed: %s", cudaGetErrorString(cudaGetLastError()));
  const size_t total = (size_t)hl + (size_t)body;
  if (len) *len = total;
  if (!want) return FB_OK;
  const size_t c = std::min(cap - 1, total);
  std::memcpy(buf, head, std::min(c, (size_t)hl));
  fb_status st = FB_OK;
  if (c > (size_t)hl && cudaMemcpy(buf + hl, d_text, c - (size_t)hl, cudaMemcpyDeviceToHost) != cudaSuccess)
    st = fail(FB_ERR_CUDA, "cannot copy the tree text");
  buf[c] = 0;
  cudaFree(d_text);
  return st;
}

extern "C" {

fb_status fb_trees_text_gpu(const uint64_t* trees, int ndpost, int ntree, int p, int device, char* buf, size_t cap,
                            size_t* len) {
  if (!trees || ndpost < 0 || ntree < 0) return fail(FB_ERR_ARG, "trees, ndpost >= 0 and ntree >= 0 are required");
  CK(cudaSetDevice(device));
  const size_t words = (size_t)ndpost * ntree * NODES;
  uint64_t* d = nullptr;
  if (cudaMalloc(&d, sizeof(uint64_t) * (words > 0 ? words : 1)) != cudaSuccess) return fail(FB_ERR_CUDA, "out of device memory");
  fb_status st = FB_OK;
  if (words > 0 && cudaMemcpy(d, trees, sizeof(uint64_t) * words, cudaMemcpyHostToDevice) != cudaSuccess)
    st = fail(FB_ERR_CUDA, "cannot copy the trees to the device");
  if (st == FB_OK) st = text_from_device(d, ndpost, ntree, p, buf, cap, len);
  cudaFree(d);
  return st;
}

fb_status fb_batch_trees_text(fb_batch* b, int chain, char* buf, size_t cap, size_t* len) {
  if (!b) return fail(FB_ERR_ARG, "batch is NULL");
  if (chain < 0 || chain >= b->nchains) return fail(FB_ERR_RANGE, "chain %d is outside 0..%d", chain, b->nchains - 1);
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  const DChain& D = b->hch[chain];
  return text_from_device(reinterpret_cast<const uint64_t*>(b->d.trees_out + D.off_tout), b->ndpost, D.m, D.p, buf,
                          cap, len);
}

fb_status fb_varcount(const uint64_t* trees, int ndpost, int ntree, int p, int* varcount) {
  if (!trees || !varcount) return fail(FB_ERR_ARG, "trees and varcount are required");
  std::memset(varcount, 0, sizeof(int) * (size_t)ndpost * p);
  for (int dr = 0; dr < ndpost; dr++)
    for (int j = 0; j < ntree; j++) {
      const uint64_t* T = trees + ((size_t)dr * ntree + j) * NODES;
      int st[2 * NODES + 2], sp = 0, seen = 0;
      st[sp++] = 0;
      while (sp > 0 && seen <= NODES) {
        const int x = st[--sp];
        seen++;
        const int l = (int)((T[x] >> 16) & 255), r = (int)((T[x] >> 24) & 255), v = (int)(T[x] & 255);
        if (l) {
          if (v < p) varcount[(size_t)dr * p + v] += 1;
          st[sp++] = r; st[sp++] = l;
        }
      }
    }
  return FB_OK;
}

fb_status fb_fbart(const int* q, int n, int p, const double* y, const double* wt, const int* ybin, const int* numcut,
                   const double* pgtab, int ntree, int nskip, int ndpost, double tau, double lambda, double nu,
                   double sigest, uint64_t seed, int probit, double offset, double* sigma, double* yhat_train_mean,
                   double* yhat_train, int* varcount, char* trees_text, size_t text_cap, size_t* text_len, int* moves) {
  if (!q || n < 1 || p < 1) return fail(FB_ERR_ARG, "q, n >= 1 and p >= 1 are required");
  std::vector<uint8_t> qv((size_t)n * p);
  for (size_t k = 0; k < qv.size(); k++) {
    if (q[k] < 0 || q[k] > 255) return fail(FB_ERR_LIMIT, "code %d at %zu is outside 0..255", q[k], k);
    qv[k] = (uint8_t)q[k];
  }
  fb_chain c;
  std::memset(&c, 0, sizeof c);
  c.n = n; c.p = p; c.ntree = ntree; c.q = qv.data(); c.y = y; c.wt = wt; c.ybin = ybin; c.numcut = numcut;
  c.pgtab = pgtab; c.tau = tau; c.lambda = lambda; c.nu = nu; c.sigest = sigest; c.offset = offset; c.seed = seed;
  c.probit = probit;
  fb_options o;
  std::memset(&o, 0, sizeof o);
  o.nskip = nskip; o.ndpost = ndpost;
  std::vector<double> yh((size_t)ndpost * n);
  std::vector<uint64_t> tr((size_t)ndpost * ntree * NODES);
  fb_chain_out out;
  std::memset(&out, 0, sizeof out);
  out.sigma = sigma; out.yhat_mean = yhat_train_mean; out.yhat = yh.data(); out.trees = tr.data();
  fb_batch* b = nullptr;
  fb_status s = fb_batch_create(&c, 1, &o, &b);
  if (s != FB_OK) return s;
  s = fb_batch_run(b, nullptr);
  if (s == FB_OK) s = fb_batch_sync(b);
  if (s == FB_OK) s = fb_batch_download(b, &out);
  size_t len = 0;
  if (s == FB_OK) s = fb_batch_trees_text(b, 0, trees_text, text_cap, &len);   // assembled on the device
  fb_batch_destroy(b);
  if (s != FB_OK) return s;
  if (yhat_train)
    for (int dr = 0; dr < ndpost; dr++)
      for (int i = 0; i < n; i++) yhat_train[(size_t)dr + (size_t)i * ndpost] = yh[(size_t)dr * n + i];
  if (varcount) {
    std::vector<int> vc((size_t)ndpost * p);
    fb_varcount(tr.data(), ndpost, ntree, p, vc.data());
    for (int dr = 0; dr < ndpost; dr++)
      for (int v = 0; v < p; v++) varcount[(size_t)dr + (size_t)v * ndpost] = vc[(size_t)dr * p + v];
  }
  if (text_len) *text_len = len;
  if (moves) { moves[0] = out.moves[0]; moves[1] = out.moves[1]; moves[2] = out.moves[2]; }
  return FB_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------ evaluator
struct fb_compiled {
  int device = 0, ndpost = 0, ntree = 0, p = 0;
  std::vector<int> var, child, root, cidx;
  std::vector<double> cut, theta;
  int* dvar = nullptr; int* dchild = nullptr; int* droot = nullptr;
  double* dcut = nullptr; double* dtheta = nullptr;
  PNode* dnodes = nullptr;
  uint8_t* dgdep = nullptr;
  uint32_t* dn32 = nullptr;     // code-compare layout (null when the cutpoints do not allow it)
  double* dcutflat = nullptr;
  int* dcutoff = nullptr;
  uint32_t* dsame = nullptr;    // trees with the structure of the previous draw's (code-compare layout)
  uint8_t* dtdep = nullptr;
  long long nsame = 0;
  int maxnd = 0;
  ~fb_compiled() {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    cudaFree(dvar); cudaFree(dchild); cudaFree(droot); cudaFree(dcut); cudaFree(dtheta); cudaFree(dnodes); cudaFree(dgdep);
    cudaFree(dn32); cudaFree(dcutflat); cudaFree(dcutoff); cudaFree(dsame); cudaFree(dtdep);
    cudaSetDevice(cur);
  }
  DForest forest() const {
    DForest f;
    f.var = dvar; f.child = dchild; f.cut = dcut; f.theta = dtheta; f.root = droot; f.nodes = dnodes; f.gdepth = dgdep;
    f.n32 = dn32; f.cuts = dcutflat; f.cutoff = dcutoff; f.maxnd = maxnd;
    f.same = dsame; f.tdep = dtdep; f.nsame = nsame;
    f.ntree = ntree; f.ndpost = ndpost; f.p = p; f.nnodes = (int)var.size();
    return f;
  }
};

namespace {

struct Scanner {
  const char* s;
  const char* end;
  bool skip() { while (s < end && (*s == ' ' || *s == '\n' || *s == '\r' || *s == '\t')) s++; return s < end; }
  bool lng(long long* v) {
    if (!skip()) return false;
    char* e;
    *v = std::strtoll(s, &e, 10);
    if (e == s || e > end) return false;
    s = e;
    return true;
  }
  bool ull(unsigned long long* v) {
    if (!skip()) return false;
    char* e;
    *v = std::strtoull(s, &e, 10);
    if (e == s || e > end) return false;
    s = e;
    return true;
  }
  bool dbl(double* v) {
    if (!skip()) return false;
    char* e;
    *v = std::strtod(s, &e);
    if (e == s || e > end) return false;
    s = e;
    return true;
  }
};

}  // namespace

extern "C" {

fb_status fb_compile_trees(const char* text, size_t len, const double* const* cutpoints, const int* ncut, int ncol,
                           int device, fb_compiled** out) {
  if (!out) return fail(FB_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!text || !cutpoints || !ncut) return fail(FB_ERR_ARG, "text, cutpoints and ncut are required");
  std::string owned(text, len);   // NUL-terminated copy so strtod cannot read past the end
  Scanner sc{owned.c_str(), owned.c_str() + owned.size()};
  long long nd, m, p;
  if (!sc.lng(&nd) || !sc.lng(&m) || !sc.lng(&p) || nd < 1 || m < 1 || p < 0)
    return fail(FB_ERR_PARSE, "tree text header must be \"ndpost ntree p\"");
  auto* ct = new fb_compiled();
  ct->device = device; ct->ndpost = (int)nd; ct->ntree = (int)m; ct->p = (int)p;
  ct->root.resize((size_t)(nd * m));
  std::vector<unsigned long long> nid;
  std::vector<int> v, c;
  std::vector<double> th;
  std::unordered_map<unsigned long long, int> pos;
  std::vector<int> qk, slot;
  for (long long t = 0; t < nd * m; t++) {
    long long nn;
    if (!sc.lng(&nn) || nn < 1) { delete ct; return fail(FB_ERR_PARSE, "tree %lld: bad node count", t); }
    nid.resize(nn); v.resize(nn); c.resize(nn); th.resize(nn);
    pos.clear();
    for (long long k = 0; k < nn; k++) {
      long long vv, cc;
      if (!sc.ull(&nid[k]) || !sc.lng(&vv) || !sc.lng(&cc) || !sc.dbl(&th[k])) {
        delete ct;
        return fail(FB_ERR_PARSE, "tree %lld: bad node line %lld", t, k);
      }
      v[k] = (int)vv; c[k] = (int)cc;
      pos[nid[k]] = (int)k;
    }
    // breadth-first from the root (id 1), each node's two children placed next to each other (src/predict.cpp:23-38)
    auto it1 = pos.find(1ull);
    if (it1 == pos.end()) { delete ct; return fail(FB_ERR_PARSE, "tree %lld has no root (id 1)", t); }
    qk.assign(1, it1->second);
    slot.assign(1, (int)ct->var.size());
    ct->root[(size_t)t] = slot[0];
    ct->var.push_back(0); ct->child.push_back(-1); ct->cut.push_back(0.0); ct->theta.push_back(0.0);
    ct->cidx.push_back(0);
    for (size_t h = 0; h < qk.size(); h++) {
      const int k = qk[h], me = slot[h];
      ct->theta[me] = th[k];
      auto L = pos.find(2 * nid[k]);
      if (L != pos.end()) {
        auto R = pos.find(2 * nid[k] + 1);
        if (R == pos.end()) { delete ct; return fail(FB_ERR_PARSE, "tree %lld: node %llu has one child", t, nid[k]); }
        if (v[k] < 0 || v[k] >= ncol || v[k] >= p || c[k] < 0 || c[k] >= ncut[v[k]]) {
          delete ct;
          return fail(FB_ERR_PARSE, "tree %lld: split (v %d, c %d) is not a cutpoint", t, v[k], c[k]);
        }
        const int ch = (int)ct->var.size();
        ct->var[me] = v[k]; ct->cut[me] = cutpoints[v[k]][c[k]]; ct->child[me] = ch; ct->cidx[me] = c[k];
        for (int z = 0; z < 2; z++) {
          ct->var.push_back(0); ct->child.push_back(-1); ct->cut.push_back(0.0); ct->theta.push_back(0.0);
          ct->cidx.push_back(0);
        }
        qk.push_back(L->second); slot.push_back(ch);
        qk.push_back(R->second); slot.push_back(ch + 1);
      }
    }
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { delete ct; return fail(FB_ERR_CUDA, "no CUDA device is available"); }
  if (cudaSetDevice(device) != cudaSuccess) { delete ct; return fail(FB_ERR_CUDA, "cannot use device %d", device); }
  const size_t N = ct->var.size();
  // packed nodes of the tiled evaluator: a leaf points to itself and tests the sentinel column p (all -inf), so a
  // walk may take more steps than its depth; per draw and group of 4 trees, the deepest leaf's depth
  std::vector<PNode> pn(N);
  std::vector<int> dep(N, 0);
  for (size_t k = 0; k < N; k++) {
    const int ch = ct->child[k];
    if (ch >= 0) { dep[ch] = dep[ch + 1] = dep[k] + 1; pn[k] = PNode{ct->cut[k], ch, ct->var[k]}; }
    else pn[k] = PNode{ct->theta[k], (int)k, ct->p};
  }
  const int G = (ct->ntree + 3) / 4;
  std::vector<uint8_t> gd((size_t)nd * G, 0), td((size_t)(nd * m), 0);
  int deepest = 0;
  for (long long t = 0; t < nd * m; t++) {
    const size_t b = (size_t)ct->root[(size_t)t], e = t + 1 < nd * m ? (size_t)ct->root[(size_t)t + 1] : N;
    int mx = 0;
    for (size_t k = b; k < e; k++) mx = std::max(mx, dep[k]);
    deepest = std::max(deepest, mx);
    uint8_t& g = gd[(size_t)(t / m) * G + (size_t)(t % m) / 4];
    g = (uint8_t)std::min(255, std::max<int>(g, mx));
    td[(size_t)t] = (uint8_t)std::min(255, mx);
  }
  const bool tiled = deepest <= 255;   // deeper trees use only the streaming evaluator
  // code-compare layout: x >= cutpoints[v][c]  <=>  code_v(x) > c, with code_v(x) the number of cutpoints of v that
  // are <= x, exact when every cutpoint list is finite and strictly increasing; nodes then pack into 32 bits
  // (child relative to the draw's first node | var << 16 | c << 24; a leaf points to itself with c = 255)
  bool codes = tiled && p <= 255;
  for (int u = 0; codes && u < ncol; u++) {
    if (ncut[u] < 0 || ncut[u] > 255) codes = false;
    for (int k = 0; codes && k < ncut[u]; k++)
      if (!std::isfinite(cutpoints[u][k]) || (k > 0 && !(cutpoints[u][k - 1] < cutpoints[u][k]))) codes = false;
  }
  int maxnd = 0;
  for (long long d = 0; d < nd; d++) {
    const size_t b = (size_t)ct->root[(size_t)(d * m)], e = d + 1 < nd ? (size_t)ct->root[(size_t)((d + 1) * m)] : N;
    maxnd = std::max(maxnd, (int)(e - b));
  }
  if (maxnd > 65535) codes = false;
  std::vector<uint32_t> n32;
  std::vector<double> cutflat;
  std::vector<int> cutoff;
  if (codes) {
    n32.resize(N);
    for (long long d = 0; d < nd; d++) {
      const size_t b = (size_t)ct->root[(size_t)(d * m)], e = d + 1 < nd ? (size_t)ct->root[(size_t)((d + 1) * m)] : N;
      for (size_t k = b; k < e; k++) {
        const int ch = ct->child[k];
        n32[k] = ch >= 0 ? (uint32_t)(ch - b) | (uint32_t)ct->var[k] << 16 | (uint32_t)ct->cidx[k] << 24
                         : (uint32_t)(k - b) | 255u << 24;
      }
    }
    cutoff.assign(1, 0);
    for (int u = 0; u < (int)p; u++) {
      const int nc = u < ncol ? ncut[u] : 0;
      for (int k = 0; k < nc; k++) cutflat.push_back(cutpoints[u][k]);
      cutoff.push_back((int)cutflat.size());
    }
    if (cutflat.empty()) cutflat.push_back(0.0);
    ct->maxnd = maxnd;
  }
  // trees whose structure equals the previous draw's tree of the same index (BART changes few trees per sweep, so
  // consecutive posterior draws share most of theirs): same node count, and every node with the same split (var,
  // cut index) and the same children relative to the tree's root
  const int SW = (m + 31) / 32;
  std::vector<uint32_t> same;
  bool carry = codes && nd > 1;   // leaf offsets are kept in one byte: trees of at most 256 nodes
  for (long long t = 0; carry && t < nd * m; t++)
    carry = (t + 1 < nd * m ? (size_t)ct->root[(size_t)t + 1] : N) - (size_t)ct->root[(size_t)t] <= 256;
  if (carry) {
    same.assign((size_t)nd * SW, 0u);
    for (long long d = 1; d < nd; d++)
      for (int t = 0; t < m; t++) {
        const long long t1 = (d - 1) * m + t, t2 = d * m + t;
        const size_t b1 = (size_t)ct->root[(size_t)t1], e1 = (size_t)ct->root[(size_t)t1 + 1];
        const size_t b2 = (size_t)ct->root[(size_t)t2], e2 = t2 + 1 < nd * m ? (size_t)ct->root[(size_t)t2 + 1] : N;
        bool eq = e1 - b1 == e2 - b2;
        for (size_t k = 0; eq && k < e1 - b1; k++) {
          const int c1 = ct->child[b1 + k], c2 = ct->child[b2 + k];
          eq = (c1 < 0) == (c2 < 0) && (c1 < 0 || (size_t)c1 - b1 == (size_t)c2 - b2) &&
               ct->var[b1 + k] == ct->var[b2 + k] && ct->cidx[b1 + k] == ct->cidx[b2 + k];
        }
        if (eq) { same[(size_t)d * SW + t / 32] |= 1u << (t % 32); ct->nsame++; }
      }
  }
  if (tiled && (cudaMalloc(&ct->dnodes, N * sizeof(PNode)) != cudaSuccess ||
                cudaMemcpy(ct->dnodes, pn.data(), N * sizeof(PNode), cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMalloc(&ct->dgdep, gd.size()) != cudaSuccess ||
                cudaMemcpy(ct->dgdep, gd.data(), gd.size(), cudaMemcpyHostToDevice) != cudaSuccess)) {
    delete ct;
    return fail(FB_ERR_CUDA, "cannot upload the compiled trees");
  }
  if (codes && (cudaMalloc(&ct->dn32, N * 4) != cudaSuccess ||
                cudaMemcpy(ct->dn32, n32.data(), N * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMalloc(&ct->dcutflat, cutflat.size() * 8) != cudaSuccess ||
                cudaMemcpy(ct->dcutflat, cutflat.data(), cutflat.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMalloc(&ct->dcutoff, cutoff.size() * 4) != cudaSuccess ||
                cudaMemcpy(ct->dcutoff, cutoff.data(), cutoff.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)) {
    delete ct;
    return fail(FB_ERR_CUDA, "cannot upload the compiled trees");
  }
  if (carry && (cudaMalloc(&ct->dsame, same.size() * 4) != cudaSuccess ||
                cudaMemcpy(ct->dsame, same.data(), same.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMalloc(&ct->dtdep, td.size()) != cudaSuccess ||
                cudaMemcpy(ct->dtdep, td.data(), td.size(), cudaMemcpyHostToDevice) != cudaSuccess)) {
    delete ct;
    return fail(FB_ERR_CUDA, "cannot upload the compiled trees");
  }
  if (!carry) ct->nsame = 0;
  if (cudaMalloc(&ct->dvar, N * 4) != cudaSuccess || cudaMalloc(&ct->dchild, N * 4) != cudaSuccess ||
      cudaMalloc(&ct->dcut, N * 8) != cudaSuccess || cudaMalloc(&ct->dtheta, N * 8) != cudaSuccess ||
      cudaMalloc(&ct->droot, ct->root.size() * 4) != cudaSuccess ||
      cudaMemcpy(ct->dvar, ct->var.data(), N * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(ct->dchild, ct->child.data(), N * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(ct->dcut, ct->cut.data(), N * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(ct->dtheta, ct->theta.data(), N * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(ct->droot, ct->root.data(), ct->root.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
    delete ct;
    return fail(FB_ERR_CUDA, "cannot upload the compiled trees");
  }
  *out = ct;
  return FB_OK;
}

fb_status fb_compiled_info(const fb_compiled* ct, int* ndpost, int* ntree, int* p, int* nnodes) {
  if (!ct) return fail(FB_ERR_ARG, "compiled trees are NULL");
  if (ndpost) *ndpost = ct->ndpost;
  if (ntree) *ntree = ct->ntree;
  if (p) *p = ct->p;
  if (nnodes) *nnodes = (int)ct->var.size();
  return FB_OK;
}

fb_status fb_predict_evaluator(const fb_compiled* ct, int n, int ndraws, int* evaluator, long long* shared_trees) {
  if (!ct) return fail(FB_ERR_ARG, "compiled trees are NULL");
  if (n < 0 || ndraws < 0) return fail(FB_ERR_ARG, "negative size");
  if (evaluator) *evaluator = predict_evaluator(ct->forest(), n, ndraws);
  if (shared_trees) *shared_trees = ct->nsame;
  return FB_OK;
}

fb_status fb_compiled_arrays(const fb_compiled* ct, int* var, int* child, double* cut, double* theta, int* root) {
  if (!ct) return fail(FB_ERR_ARG, "compiled trees are NULL");
  const size_t N = ct->var.size();
  if (var) std::memcpy(var, ct->var.data(), N * 4);
  if (child) std::memcpy(child, ct->child.data(), N * 4);
  if (cut) std::memcpy(cut, ct->cut.data(), N * 8);
  if (theta) std::memcpy(theta, ct->theta.data(), N * 8);
  if (root) std::memcpy(root, ct->root.data(), ct->root.size() * 4);
  return FB_OK;
}

void fb_compiled_free(fb_compiled* ct) { delete ct; }

fb_status fb_predict_draws_device(const fb_compiled* ct, const double* x_dev, int ncol, int n, int ld, int draw0,
                                  int ndraws, double mu, double* out_dev, int ldo, void* stream) {
  if (!ct) return fail(FB_ERR_ARG, "compiled trees are NULL");
  if (ncol != ct->p) return fail(FB_ERR_SHAPE, "newdata has %d columns, the trees use %d", ncol, ct->p);
  if (draw0 < 1 || ndraws < 0 || draw0 + ndraws - 1 > ct->ndpost)
    return fail(FB_ERR_RANGE, "draw %d out of range 1..%d", draw0 + (draw0 < 1 ? 0 : ndraws - 1), ct->ndpost);
  if (n < 0 || ld < n || ldo < n) return fail(FB_ERR_ARG, "need 0 <= n <= ld and n <= ldo");
  if (n == 0 || ndraws == 0) return FB_OK;
  if ((!x_dev && ncol > 0) || !out_dev) return fail(FB_ERR_ARG, "x_dev and out_dev are required");
  CK(cudaSetDevice(ct->device));
  if (launch_predict(ct->forest(), x_dev, n, ld, draw0 - 1, ndraws, mu, out_dev, ldo, stream) != 0)
    return fail(FB_ERR_CUDA, "predict launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return FB_OK;
}

fb_status fb_predict_draw(const fb_compiled* ct, const double* const* cols, int ncol, int n, int draw, double mu,
                          double* out) {
  if (!ct) return fail(FB_ERR_ARG, "compiled trees are NULL");
  if (ncol != ct->p) return fail(FB_ERR_SHAPE, "newdata has %d columns, the trees use %d", ncol, ct->p);
  if (draw < 1 || draw > ct->ndpost) return fail(FB_ERR_RANGE, "draw %d out of range 1..%d", draw, ct->ndpost);
  if (n <= 0) return FB_OK;
  if (!cols || !out) return fail(FB_ERR_ARG, "cols and out are required");
  CK(cudaSetDevice(ct->device));
  double* dx = nullptr;
  double* dout = nullptr;
  CK(cudaMalloc(&dx, sizeof(double) * (size_t)n * std::max(ncol, 1)));
  if (cudaMalloc(&dout, sizeof(double) * (size_t)n) != cudaSuccess) { cudaFree(dx); return fail(FB_ERR_CUDA, "out of device memory"); }
  fb_status s = FB_OK;
  for (int v = 0; v < ncol && s == FB_OK; v++)
    if (cudaMemcpy(dx + (size_t)v * n, cols[v], sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess)
      s = fail(FB_ERR_CUDA, "copy of column %d failed", v);
  if (s == FB_OK && launch_predict(ct->forest(), dx, n, n, draw - 1, 1, mu, dout, n, nullptr) != 0)
    s = fail(FB_ERR_CUDA, "predict launch failed");
  if (s == FB_OK && cudaMemcpy(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    s = fail(FB_ERR_CUDA, "copy of the result failed: %s", cudaGetErrorString(cudaGetLastError()));
  cudaFree(dx);
  cudaFree(dout);
  return s;
}

fb_status fb_predict_draw_static(const fb_compiled* ct, const double* const* cols, int ncol, int n, int draw,
                                 double mu, double* out) {
  if (!ct) return fail(FB_ERR_ARG, "compiled trees are NULL");
  if (ncol != ct->p) return fail(FB_ERR_SHAPE, "newdata has %d columns, the trees use %d", ncol, ct->p);
  if (draw < 1 || draw > ct->ndpost) return fail(FB_ERR_RANGE, "draw %d out of range 1..%d", draw, ct->ndpost);
  if (n <= 0) return FB_OK;
  if (!cols || !out) return fail(FB_ERR_ARG, "cols and out are required");
  const size_t need = (size_t)n * ((size_t)ncol + 1);
  if (need > PREDICT_SCRATCH_DOUBLES)
    return fail(FB_ERR_LIMIT,
                "n * (ncol + 1) = %zu doubles exceeds the fixed device scratch of %zu doubles; split the rows over "
                "several calls or use fb_predict_draw",
                need, (size_t)PREDICT_SCRATCH_DOUBLES);
  CK(cudaSetDevice(ct->device));
  double* scr = nullptr;
  const int rc = predict_scratch_address(ct->device, &scr);
  if (rc == -2) return fail(FB_ERR_LIMIT, "device %d: the fixed scratch is tracked for devices 0..63", ct->device);
  if (rc != 0)
    return fail(FB_ERR_CUDA, "cannot resolve the fixed predict scratch on device %d: %s", ct->device,
                cudaGetErrorString(cudaGetLastError()));
  double* dx = scr;                        // [ncol][n]
  double* dout = scr + (size_t)n * ncol;   // [n]
  for (int v = 0; v < ncol; v++)
    if (cudaMemcpy(dx + (size_t)v * n, cols[v], sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(FB_ERR_CUDA, "copy of column %d failed", v);
  if (launch_predict(ct->forest(), dx, n, n, draw - 1, 1, mu, dout, n, nullptr) != 0)
    return fail(FB_ERR_CUDA, "predict launch failed");
  if (cudaMemcpy(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return fail(FB_ERR_CUDA, "copy of the result failed: %s", cudaGetErrorString(cudaGetLastError()));
  return FB_OK;
}

// ------------------------------------------------------------------------------------------------ proposal MLP
}  // extern "C"

namespace {
constexpr size_t kN1 = (size_t)MLP_H * MLP_IN, kN2 = (size_t)MLP_H * MLP_H, kN3 = (size_t)MLP_OUT * MLP_H;
constexpr size_t kOffB1 = kN1, kOffW2 = kOffB1 + MLP_H, kOffB2 = kOffW2 + kN2, kOffW3 = kOffB2 + MLP_H,
                 kOffB3 = kOffW3 + kN3;

float bf16_host(uint16_t h) { uint32_t u = (uint32_t)h << 16; float f; std::memcpy(&f, &u, 4); return f; }
uint16_t bf16_round_host(float f) {
  uint32_t u; std::memcpy(&u, &f, 4);
  return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}

// device state of one training or gradient job; frees everything on scope exit
struct MlpJob {
  std::vector<void*> mem;
  ~MlpJob() { for (void* p : mem) cudaFree(p); }
  template <class T> bool alloc(T** p, size_t n) {
    if (cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * (n ? n : 1)) != cudaSuccess) return false;
    mem.push_back(*p);
    return true;
  }
};

// Examples in a canonical order (sorted by their bytes: features, then label and mask), so that training depends on
// its seed only, whatever order the sampler's CTAs collected the examples in.
std::vector<int> canonical_order(const float* x, int width, const int* y, const uint32_t* mask, const int* lo,
                                 const int* hi, int count) {
  std::vector<int> ord(count);
  for (int k = 0; k < count; k++) ord[k] = k;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
    const int c = std::memcmp(x + (size_t)a * width, x + (size_t)b * width, sizeof(float) * (size_t)width);
    if (c != 0) return c < 0;
    if (y[a] != y[b]) return y[a] < y[b];
    if (mask && mask[a] != mask[b]) return mask[a] < mask[b];
    if (lo && lo[a] != lo[b]) return lo[a] < lo[b];
    if (hi && hi[a] != hi[b]) return hi[a] < hi[b];
    return false;
  });
  return ord;
}

fb_status check_cut_examples(const float* x, const int* c, const int* lo, const int* hi, int count) {
  if (!x || !c || !lo || !hi || count < 1) return fail(FB_ERR_ARG, "x, c, lo, hi and count >= 1 are required");
  for (int k = 0; k < count; k++)
    if (lo[k] < 0 || hi[k] >= CUT_BINS || lo[k] > hi[k] || c[k] < lo[k] || c[k] > hi[k])
      return fail(FB_ERR_ARG, "example %d: cut %d is not in its range [%d, %d]", k, c[k], lo[k], hi[k]);
  return FB_OK;
}

fb_status check_examples(const float* x, const int* y, const uint32_t* mask, int count) {
  if (!x || !y || !mask || count < 1) return fail(FB_ERR_ARG, "x, y, mask and count >= 1 are required");
  for (int k = 0; k < count; k++)
    if (y[k] < 0 || y[k] >= MLP_OUT || !((mask[k] >> y[k]) & 1u))
      return fail(FB_ERR_ARG, "example %d: label %d is not one of its valid predictors", k, y[k]);
  return FB_OK;
}
}  // namespace

extern "C" {

fb_status fb_train_proposal(const float* x, const int* y, const uint32_t* mask, int count,
                            const fb_train_options* opt, const fb_proposal_model* init, uint16_t* out_w1,
                            float* out_b1, uint16_t* out_w2, float* out_b2, uint16_t* out_w3, float* out_b3,
                            double* losses) {
  if (!opt || !out_w1 || !out_b1 || !out_w2 || !out_b2 || !out_w3 || !out_b3)
    return fail(FB_ERR_ARG, "options and every output array are required");
  if (opt->epochs < 1 || opt->batch < 1 || !(opt->lr > 0.0)) return fail(FB_ERR_ARG, "epochs, batch and lr must be > 0");
  fb_status st = check_examples(x, y, mask, count);
  if (st != FB_OK) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FB_ERR_CUDA, "no CUDA device is available");
  CK(cudaSetDevice(opt->device));
  // initial parameters (host): the given model, or seeded uniform(-a, a) with a = sqrt(6 / fan_in), zero biases
  std::vector<float> P(MLP_NPARAM, 0.0f);
  if (init) {
    if (!init->w1 || !init->b1 || !init->w2 || !init->b2 || !init->w3 || !init->b3)
      return fail(FB_ERR_ARG, "every weight and bias array of the initial model is required");
    for (size_t k = 0; k < kN1; k++) P[k] = bf16_host(init->w1[k]);
    for (size_t k = 0; k < kN2; k++) P[kOffW2 + k] = bf16_host(init->w2[k]);
    for (size_t k = 0; k < kN3; k++) P[kOffW3 + k] = bf16_host(init->w3[k]);
    for (int k = 0; k < MLP_H; k++) { P[kOffB1 + k] = init->b1[k]; P[kOffB2 + k] = init->b2[k]; }
    for (int k = 0; k < MLP_OUT; k++) P[kOffB3 + k] = init->b3[k];
  } else {
    std::mt19937_64 g(opt->seed);
    std::uniform_real_distribution<float> u(-1.0f, 1.0f);
    const float a1 = std::sqrt(6.0f / MLP_IN), a2 = std::sqrt(6.0f / MLP_H), a3 = 0.1f * std::sqrt(6.0f / MLP_H);
    for (size_t k = 0; k < kN1; k++) P[k] = bf16_host(bf16_round_host(a1 * u(g)));
    for (size_t k = 0; k < kN2; k++) P[kOffW2 + k] = bf16_host(bf16_round_host(a2 * u(g)));
    for (size_t k = 0; k < kN3; k++) P[kOffW3 + k] = bf16_host(bf16_round_host(a3 * u(g)));
  }
  std::vector<uint16_t> W(kN1 + kN2 + kN3);
  for (size_t k = 0; k < kN1; k++) W[k] = bf16_round_host(P[k]);
  for (size_t k = 0; k < kN2; k++) W[kN1 + k] = bf16_round_host(P[kOffW2 + k]);
  for (size_t k = 0; k < kN3; k++) W[kN1 + kN2 + k] = bf16_round_host(P[kOffW3 + k]);
  MlpJob job;
  float *dx = nullptr, *dp = nullptr, *dm1 = nullptr, *dm2 = nullptr, *dg = nullptr, *dl = nullptr;
  int *dy = nullptr, *didx = nullptr;
  unsigned* dmask = nullptr;
  uint16_t* dw = nullptr;
  if (!job.alloc(&dx, (size_t)count * MLP_IN) || !job.alloc(&dy, count) || !job.alloc(&dmask, count) ||
      !job.alloc(&didx, count) || !job.alloc(&dp, MLP_NPARAM) || !job.alloc(&dm1, MLP_NPARAM) ||
      !job.alloc(&dm2, MLP_NPARAM) || !job.alloc(&dg, MLP_NPARAM) || !job.alloc(&dl, 1) || !job.alloc(&dw, W.size()))
    return fail(FB_ERR_CUDA, "out of device memory");
  {   // the examples in canonical order
    const std::vector<int> ord = canonical_order(x, MLP_IN, y, mask, nullptr, nullptr, count);
    std::vector<float> xs((size_t)count * MLP_IN);
    std::vector<int> ys(count);
    std::vector<unsigned> ms(count);
    for (int k = 0; k < count; k++) {
      std::memcpy(xs.data() + (size_t)k * MLP_IN, x + (size_t)ord[k] * MLP_IN, sizeof(float) * MLP_IN);
      ys[k] = y[ord[k]]; ms[k] = mask[ord[k]];
    }
    CK(cudaMemcpy(dx, xs.data(), sizeof(float) * MLP_IN * (size_t)count, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dy, ys.data(), sizeof(int) * (size_t)count, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dmask, ms.data(), sizeof(unsigned) * (size_t)count, cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(dp, P.data(), sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dw, W.data(), sizeof(uint16_t) * W.size(), cudaMemcpyHostToDevice));
  CK(cudaMemset(dm1, 0, sizeof(float) * MLP_NPARAM));
  CK(cudaMemset(dm2, 0, sizeof(float) * MLP_NPARAM));
  MlpParams MP{dw, dw + kN1, dw + kN1 + kN2, dp + kOffB1, dp + kOffB2, dp + kOffB3};
  std::vector<int> perm(count);
  for (int k = 0; k < count; k++) perm[k] = k;
  std::mt19937_64 shuf(opt->seed ^ 0x5851F42D4C957F2Dull);
  int step = 0;
  for (int e = 0; e < opt->epochs; e++) {
    std::shuffle(perm.begin(), perm.end(), shuf);
    CK(cudaMemcpy(didx, perm.data(), sizeof(int) * (size_t)count, cudaMemcpyHostToDevice));
    CK(cudaMemset(dl, 0, sizeof(float)));
    for (int s0 = 0; s0 < count; s0 += opt->batch) {
      const int B = std::min(opt->batch, count - s0);
      CK(cudaMemsetAsync(dg, 0, sizeof(float) * MLP_NPARAM));
      if (mlp_grad_launch(MP, dx, dy, dmask, didx + s0, B, dg, dl, nullptr) != 0)
        return fail(FB_ERR_CUDA, "gradient kernel failed: %s", cudaGetErrorString(cudaGetLastError()));
      if (mlp_adam_launch(dp, dm1, dm2, dg, 1.0f / (float)B, (float)opt->lr, ++step, MP, nullptr) != 0)
        return fail(FB_ERR_CUDA, "update kernel failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    float l = 0.0f;
    CK(cudaMemcpy(&l, dl, sizeof(float), cudaMemcpyDeviceToHost));
    if (losses) losses[e] = (double)l / count;
  }
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(P.data(), dp, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(W.data(), dw, sizeof(uint16_t) * W.size(), cudaMemcpyDeviceToHost));
  std::memcpy(out_w1, W.data(), 2 * kN1);
  std::memcpy(out_w2, W.data() + kN1, 2 * kN2);
  std::memcpy(out_w3, W.data() + kN1 + kN2, 2 * kN3);
  std::memcpy(out_b1, P.data() + kOffB1, 4 * MLP_H);
  std::memcpy(out_b2, P.data() + kOffB2, 4 * MLP_H);
  std::memcpy(out_b3, P.data() + kOffB3, 4 * MLP_OUT);
  return FB_OK;
}

fb_status fb_mlp_loss_grad(const fb_proposal_model* model, const float* x, const int* y, const uint32_t* mask,
                           int count, int device, double* loss, float* gw1, float* gb1, float* gw2, float* gb2,
                           float* gw3, float* gb3) {
  if (!model || !model->w1 || !model->b1 || !model->w2 || !model->b2 || !model->w3 || !model->b3 || !loss)
    return fail(FB_ERR_ARG, "model and loss are required");
  fb_status st = check_examples(x, y, mask, count);
  if (st != FB_OK) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FB_ERR_CUDA, "no CUDA device is available");
  CK(cudaSetDevice(device));
  std::vector<float> P(MLP_NPARAM, 0.0f);
  for (int k = 0; k < MLP_H; k++) { P[kOffB1 + k] = model->b1[k]; P[kOffB2 + k] = model->b2[k]; }
  for (int k = 0; k < MLP_OUT; k++) P[kOffB3 + k] = model->b3[k];
  MlpJob job;
  float *dx = nullptr, *dp = nullptr, *dg = nullptr, *dl = nullptr;
  int* dy = nullptr;
  unsigned* dmask = nullptr;
  uint16_t* dw = nullptr;
  if (!job.alloc(&dx, (size_t)count * MLP_IN) || !job.alloc(&dy, count) || !job.alloc(&dmask, count) ||
      !job.alloc(&dp, MLP_NPARAM) || !job.alloc(&dg, MLP_NPARAM) || !job.alloc(&dl, 1) ||
      !job.alloc(&dw, kN1 + kN2 + kN3))
    return fail(FB_ERR_CUDA, "out of device memory");
  CK(cudaMemcpy(dx, x, sizeof(float) * MLP_IN * (size_t)count, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dy, y, sizeof(int) * (size_t)count, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dmask, mask, sizeof(unsigned) * (size_t)count, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dp, P.data(), sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dw, model->w1, 2 * kN1, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dw + kN1, model->w2, 2 * kN2, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dw + kN1 + kN2, model->w3, 2 * kN3, cudaMemcpyHostToDevice));
  CK(cudaMemset(dg, 0, sizeof(float) * MLP_NPARAM));
  CK(cudaMemset(dl, 0, sizeof(float)));
  MlpParams MP{dw, dw + kN1, dw + kN1 + kN2, dp + kOffB1, dp + kOffB2, dp + kOffB3};
  if (mlp_grad_launch(MP, dx, dy, dmask, nullptr, count, dg, dl, nullptr) != 0)
    return fail(FB_ERR_CUDA, "gradient kernel failed: %s", cudaGetErrorString(cudaGetLastError()));
  CK(cudaDeviceSynchronize());
  std::vector<float> G(MLP_NPARAM);
  float l = 0.0f;
  CK(cudaMemcpy(G.data(), dg, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&l, dl, sizeof(float), cudaMemcpyDeviceToHost));
  const float inv = 1.0f / (float)count;
  *loss = (double)l / count;
  auto put = [&](float* dst, size_t off, size_t n) { if (dst) for (size_t k = 0; k < n; k++) dst[k] = G[off + k] * inv; };
  put(gw1, 0, kN1); put(gb1, kOffB1, MLP_H); put(gw2, kOffW2, kN2); put(gb2, kOffB2, MLP_H);
  put(gw3, kOffW3, kN3); put(gb3, kOffB3, MLP_OUT);
  return FB_OK;
}

namespace {
constexpr size_t cN1 = (size_t)CUT_H * CUT_IN, cN2 = (size_t)CUT_H * CUT_H, cN3 = (size_t)CUT_E * CUT_H,
                 cN4 = (size_t)CUT_BINS * CUT_E;
constexpr size_t cOffB1 = cN1, cOffW2 = cOffB1 + CUT_H, cOffB2 = cOffW2 + cN2, cOffW3 = cOffB2 + CUT_H,
                 cOffB3 = cOffW3 + cN3, cOffE = cOffB3 + CUT_E, cOffBE = cOffE + cN4;
static_assert(cOffBE + CUT_BINS == (size_t)CUT_NPARAM, "cut head parameter layout");
bool cut_model_complete(const fb_cut_model* m) {
  return m && m->w1 && m->b1 && m->w2 && m->b2 && m->w3 && m->b3 && m->emb && m->be;
}
// uploads the examples (canonical order when ordered) of the cut head's training
struct CutData {
  float* x = nullptr; int* c = nullptr; int* lo = nullptr; int* hi = nullptr;
};
bool upload_cut_examples(MlpJob& job, const float* x, const int* c, const int* lo, const int* hi, int count,
                         bool ordered, CutData* d) {
  if (!job.alloc(&d->x, (size_t)count * CUT_IN) || !job.alloc(&d->c, count) || !job.alloc(&d->lo, count) ||
      !job.alloc(&d->hi, count))
    return false;
  std::vector<int> ord(count);
  for (int k = 0; k < count; k++) ord[k] = k;
  if (ordered) ord = canonical_order(x, CUT_IN, c, nullptr, lo, hi, count);
  std::vector<float> xs((size_t)count * CUT_IN);
  std::vector<int> cs(count), ls(count), hs(count);
  for (int k = 0; k < count; k++) {
    std::memcpy(xs.data() + (size_t)k * CUT_IN, x + (size_t)ord[k] * CUT_IN, sizeof(float) * CUT_IN);
    cs[k] = c[ord[k]]; ls[k] = lo[ord[k]]; hs[k] = hi[ord[k]];
  }
  return cudaMemcpy(d->x, xs.data(), sizeof(float) * xs.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(d->c, cs.data(), sizeof(int) * (size_t)count, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(d->lo, ls.data(), sizeof(int) * (size_t)count, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(d->hi, hs.data(), sizeof(int) * (size_t)count, cudaMemcpyHostToDevice) == cudaSuccess;
}
}  // namespace

fb_status fb_train_cut_proposal(const float* x, const int* c, const int* lo, const int* hi, int count,
                                const fb_train_options* opt, const fb_cut_model* init, uint16_t* out_w1, float* out_b1,
                                uint16_t* out_w2, float* out_b2, uint16_t* out_w3, float* out_b3, uint16_t* out_emb,
                                float* out_be, double* losses) {
  if (!opt || !out_w1 || !out_b1 || !out_w2 || !out_b2 || !out_w3 || !out_b3 || !out_emb || !out_be)
    return fail(FB_ERR_ARG, "options and every output array are required");
  if (opt->epochs < 1 || opt->batch < 1 || !(opt->lr > 0.0)) return fail(FB_ERR_ARG, "epochs, batch and lr must be > 0");
  fb_status st = check_cut_examples(x, c, lo, hi, count);
  if (st != FB_OK) return st;
  if (init && !cut_model_complete(init)) return fail(FB_ERR_ARG, "every weight and bias array of the initial model is required");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FB_ERR_CUDA, "no CUDA device is available");
  CK(cudaSetDevice(opt->device));
  // initial parameters: the given model, or seeded uniform(-a, a), a = sqrt(6 / fan_in) (the last two layers scaled
  // down, so that training starts near the uniform cut), zero biases
  std::vector<float> P(CUT_NPARAM, 0.0f);
  if (init) {
    for (size_t k = 0; k < cN1; k++) P[k] = bf16_host(init->w1[k]);
    for (size_t k = 0; k < cN2; k++) P[cOffW2 + k] = bf16_host(init->w2[k]);
    for (size_t k = 0; k < cN3; k++) P[cOffW3 + k] = bf16_host(init->w3[k]);
    for (size_t k = 0; k < cN4; k++) P[cOffE + k] = bf16_host(init->emb[k]);
    for (int k = 0; k < CUT_H; k++) { P[cOffB1 + k] = init->b1[k]; P[cOffB2 + k] = init->b2[k]; }
    for (int k = 0; k < CUT_E; k++) P[cOffB3 + k] = init->b3[k];
    for (int k = 0; k < CUT_BINS; k++) P[cOffBE + k] = init->be[k];
  } else {
    std::mt19937_64 g(opt->seed);
    std::uniform_real_distribution<float> u(-1.0f, 1.0f);
    const float a1 = std::sqrt(6.0f / CUT_IN), a2 = std::sqrt(6.0f / CUT_H), a3 = 0.3f * std::sqrt(6.0f / CUT_H),
                a4 = 0.3f * std::sqrt(6.0f / CUT_E);
    for (size_t k = 0; k < cN1; k++) P[k] = bf16_host(bf16_round_host(a1 * u(g)));
    for (size_t k = 0; k < cN2; k++) P[cOffW2 + k] = bf16_host(bf16_round_host(a2 * u(g)));
    for (size_t k = 0; k < cN3; k++) P[cOffW3 + k] = bf16_host(bf16_round_host(a3 * u(g)));
    for (size_t k = 0; k < cN4; k++) P[cOffE + k] = bf16_host(bf16_round_host(a4 * u(g)));
  }
  std::vector<uint16_t> W(cN1 + cN2 + cN3 + cN4);
  for (size_t k = 0; k < cN1; k++) W[k] = bf16_round_host(P[k]);
  for (size_t k = 0; k < cN2; k++) W[cN1 + k] = bf16_round_host(P[cOffW2 + k]);
  for (size_t k = 0; k < cN3; k++) W[cN1 + cN2 + k] = bf16_round_host(P[cOffW3 + k]);
  for (size_t k = 0; k < cN4; k++) W[cN1 + cN2 + cN3 + k] = bf16_round_host(P[cOffE + k]);
  MlpJob job;
  CutData d;
  float *dp = nullptr, *dm1 = nullptr, *dm2 = nullptr, *dg = nullptr, *dl = nullptr;
  int* didx = nullptr;
  uint16_t* dw = nullptr;
  if (!upload_cut_examples(job, x, c, lo, hi, count, true, &d) || !job.alloc(&didx, count) ||
      !job.alloc(&dp, CUT_NPARAM) || !job.alloc(&dm1, CUT_NPARAM) || !job.alloc(&dm2, CUT_NPARAM) ||
      !job.alloc(&dg, CUT_NPARAM) || !job.alloc(&dl, 1) || !job.alloc(&dw, W.size()))
    return fail(FB_ERR_CUDA, "out of device memory");
  CK(cudaMemcpy(dp, P.data(), sizeof(float) * CUT_NPARAM, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dw, W.data(), sizeof(uint16_t) * W.size(), cudaMemcpyHostToDevice));
  CK(cudaMemset(dm1, 0, sizeof(float) * CUT_NPARAM));
  CK(cudaMemset(dm2, 0, sizeof(float) * CUT_NPARAM));
  CutParams CP{dw, dw + cN1, dw + cN1 + cN2, dw + cN1 + cN2 + cN3, dp + cOffB1, dp + cOffB2, dp + cOffB3, dp + cOffBE};
  std::vector<int> perm(count);
  for (int k = 0; k < count; k++) perm[k] = k;
  std::mt19937_64 shuf(opt->seed ^ 0x5851F42D4C957F2Dull);
  int step = 0;
  for (int e = 0; e < opt->epochs; e++) {
    std::shuffle(perm.begin(), perm.end(), shuf);
    CK(cudaMemcpy(didx, perm.data(), sizeof(int) * (size_t)count, cudaMemcpyHostToDevice));
    CK(cudaMemset(dl, 0, sizeof(float)));
    for (int s0 = 0; s0 < count; s0 += opt->batch) {
      const int B = std::min(opt->batch, count - s0);
      CK(cudaMemsetAsync(dg, 0, sizeof(float) * CUT_NPARAM));
      if (cut_grad_launch(CP, d.x, d.c, d.lo, d.hi, didx + s0, B, dg, dl, nullptr) != 0)
        return fail(FB_ERR_CUDA, "gradient kernel failed: %s", cudaGetErrorString(cudaGetLastError()));
      if (cut_adam_launch(dp, dm1, dm2, dg, 1.0f / (float)B, (float)opt->lr, ++step, CP, nullptr) != 0)
        return fail(FB_ERR_CUDA, "update kernel failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    float l = 0.0f;
    CK(cudaMemcpy(&l, dl, sizeof(float), cudaMemcpyDeviceToHost));
    if (losses) losses[e] = (double)l / count;
  }
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(P.data(), dp, sizeof(float) * CUT_NPARAM, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(W.data(), dw, sizeof(uint16_t) * W.size(), cudaMemcpyDeviceToHost));
  std::memcpy(out_w1, W.data(), 2 * cN1);
  std::memcpy(out_w2, W.data() + cN1, 2 * cN2);
  std::memcpy(out_w3, W.data() + cN1 + cN2, 2 * cN3);
  std::memcpy(out_emb, W.data() + cN1 + cN2 + cN3, 2 * cN4);
  std::memcpy(out_b1, P.data() + cOffB1, 4 * CUT_H);
  std::memcpy(out_b2, P.data() + cOffB2, 4 * CUT_H);
  std::memcpy(out_b3, P.data() + cOffB3, 4 * CUT_E);
  std::memcpy(out_be, P.data() + cOffBE, 4 * CUT_BINS);
  return FB_OK;
}

fb_status fb_cut_loss_grad(const fb_cut_model* model, const float* x, const int* c, const int* lo, const int* hi,
                           int count, int device, double* loss, float* gw1, float* gb1, float* gw2, float* gb2,
                           float* gw3, float* gb3, float* gemb, float* gbe) {
  if (!cut_model_complete(model) || !loss) return fail(FB_ERR_ARG, "model and loss are required");
  fb_status st = check_cut_examples(x, c, lo, hi, count);
  if (st != FB_OK) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FB_ERR_CUDA, "no CUDA device is available");
  CK(cudaSetDevice(device));
  std::vector<float> P(CUT_NPARAM, 0.0f);
  for (int k = 0; k < CUT_H; k++) { P[cOffB1 + k] = model->b1[k]; P[cOffB2 + k] = model->b2[k]; }
  for (int k = 0; k < CUT_E; k++) P[cOffB3 + k] = model->b3[k];
  for (int k = 0; k < CUT_BINS; k++) P[cOffBE + k] = model->be[k];
  MlpJob job;
  CutData d;
  float *dp = nullptr, *dg = nullptr, *dl = nullptr;
  uint16_t* dw = nullptr;
  if (!upload_cut_examples(job, x, c, lo, hi, count, false, &d) || !job.alloc(&dp, CUT_NPARAM) ||
      !job.alloc(&dg, CUT_NPARAM) || !job.alloc(&dl, 1) || !job.alloc(&dw, cN1 + cN2 + cN3 + cN4))
    return fail(FB_ERR_CUDA, "out of device memory");
  CK(cudaMemcpy(dp, P.data(), sizeof(float) * CUT_NPARAM, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dw, model->w1, 2 * cN1, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dw + cN1, model->w2, 2 * cN2, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dw + cN1 + cN2, model->w3, 2 * cN3, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dw + cN1 + cN2 + cN3, model->emb, 2 * cN4, cudaMemcpyHostToDevice));
  CK(cudaMemset(dg, 0, sizeof(float) * CUT_NPARAM));
  CK(cudaMemset(dl, 0, sizeof(float)));
  CutParams CP{dw, dw + cN1, dw + cN1 + cN2, dw + cN1 + cN2 + cN3, dp + cOffB1, dp + cOffB2, dp + cOffB3, dp + cOffBE};
  if (cut_grad_launch(CP, d.x, d.c, d.lo, d.hi, nullptr, count, dg, dl, nullptr) != 0)
    return fail(FB_ERR_CUDA, "gradient kernel failed: %s", cudaGetErrorString(cudaGetLastError()));
  CK(cudaDeviceSynchronize());
  std::vector<float> G(CUT_NPARAM);
  float l = 0.0f;
  CK(cudaMemcpy(G.data(), dg, sizeof(float) * CUT_NPARAM, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&l, dl, sizeof(float), cudaMemcpyDeviceToHost));
  const float inv = 1.0f / (float)count;
  *loss = (double)l / count;
  auto put = [&](float* dst, size_t off, size_t n) { if (dst) for (size_t k = 0; k < n; k++) dst[k] = G[off + k] * inv; };
  put(gw1, 0, cN1); put(gb1, cOffB1, CUT_H); put(gw2, cOffW2, cN2); put(gb2, cOffB2, CUT_H);
  put(gw3, cOffW3, cN3); put(gb3, cOffB3, CUT_E); put(gemb, cOffE, cN4); put(gbe, cOffBE, CUT_BINS);
  return FB_OK;
}

fb_status fb_probit_latent_device(const double* fit_dev, const int* ybin_dev, long long n, double offset,
                                  uint64_t seed, int sweep, double* z_dev, int* capped_dev, void* cuda_stream) {
  if (n < 0) return fail(FB_ERR_ARG, "n must be >= 0");
  if (n > 0xFFFFFFFFll) return fail(FB_ERR_LIMIT, "n %lld exceeds the 2^32 rows a chain's counters address", n);
  if (sweep < -1) return fail(FB_ERR_ARG, "sweep %d: 0-based, or -1 for the initial draw", sweep);
  if (n == 0) return FB_OK;
  if (!fit_dev || !ybin_dev || !z_dev) return fail(FB_ERR_ARG, "fit, ybin and z are required");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FB_ERR_CUDA, "no CUDA device is available");
  if (launch_probit_latent(fit_dev, ybin_dev, n, offset, seed, (uint32_t)sweep, z_dev, capped_dev, cuda_stream) != 0)
    return fail(FB_ERR_CUDA, "latent redraw launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return FB_OK;
}

fb_status fb_sigma_estimate(const double* const* cols, int ncol, int n, const double* y, int device, double* sigest,
                            int* rank) {
  if (ncol < 0 || n < 2) return fail(FB_ERR_ARG, "need ncol >= 0 and n >= 2 (n = %d)", n);
  if (ncol > 32) return fail(FB_ERR_LIMIT, "%d columns (at most 32)", ncol);
  if (!y || !sigest || (ncol > 0 && !cols)) return fail(FB_ERR_ARG, "cols, y and sigest are required");
  for (int v = 0; v < ncol; v++)
    if (!cols[v]) return fail(FB_ERR_ARG, "column %d is missing", v);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FB_ERR_CUDA, "no CUDA device is available");
  if (cudaSetDevice(device) != cudaSuccess) return fail(FB_ERR_CUDA, "cannot use device %d", device);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  const int q = ncol + 2, npairs = q * (q + 1) / 2;
  long long nb = std::min<long long>(((long long)n + 63) / 64, 4ll * nsm);
  const long long chunk = (((long long)n + nb - 1) / nb + 63) / 64 * 64;
  nb = ((long long)n + chunk - 1) / chunk;
  double *dx = nullptr, *dy = nullptr, *dp = nullptr;
  fb_status st = FB_OK;
  if (cudaMalloc(&dx, sizeof(double) * (size_t)std::max(ncol, 1) * n) != cudaSuccess ||
      cudaMalloc(&dy, sizeof(double) * (size_t)n) != cudaSuccess ||
      cudaMalloc(&dp, sizeof(double) * (size_t)nb * npairs) != cudaSuccess)
    st = fail(FB_ERR_CUDA, "cannot allocate %lld rows x %d columns", (long long)n, ncol);
  for (int v = 0; st == FB_OK && v < ncol; v++)
    if (cudaMemcpy(dx + (size_t)v * n, cols[v], sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess)
      st = fail(FB_ERR_CUDA, "column copy failed");
  if (st == FB_OK && cudaMemcpy(dy, y, sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess)
    st = fail(FB_ERR_CUDA, "y copy failed");
  if (st == FB_OK && launch_gram(dx, n, ncol, dy, (int)nb, (int)chunk, dp, nullptr) != 0)
    st = fail(FB_ERR_CUDA, "gram launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  std::vector<double> part((size_t)nb * npairs);
  if (st == FB_OK && cudaMemcpy(part.data(), dp, sizeof(double) * part.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
    st = fail(FB_ERR_CUDA, "gram copy failed: %s", cudaGetErrorString(cudaGetLastError()));
  cudaFree(dx); cudaFree(dy); cudaFree(dp);
  if (st != FB_OK) return st;
  // the blocks' sums in block order, into the symmetric matrix M of [1, x, y]
  std::vector<double> M((size_t)q * q, 0.0);
  for (int t = 0, j = 0, k = 0; t < npairs; t++) {
    double a = 0.0;
    for (long long b = 0; b < nb; b++) a += part[(size_t)b * npairs + t];
    M[(size_t)j * q + k] = M[(size_t)k * q + j] = a;
    if (++k == q) { ++j; k = j; }
  }
  const int yi = q - 1;
  if (ncol >= n) {   // sd(yc) (R/fwbart.R:22 when p >= n)
    const double sy = M[yi], syy = M[(size_t)yi * q + yi];
    *sigest = std::sqrt(std::max(0.0, (syy - sy * sy / n) / (n - 1)));
    if (rank) *rank = 0;
    return FB_OK;
  }
  // lm's residual standard error: eliminate the columns of [1, x] with symmetric pivoting (largest remaining
  // diagonal first, columns whose remaining diagonal falls below 1e-12 of the largest are aliased, as lm drops
  // them); what remains in the y, y entry is the residual sum of squares, with n - rank degrees of freedom
  const int p1 = ncol + 1;
  double dmax = 0.0;
  for (int i = 0; i < p1; i++) dmax = std::max(dmax, M[(size_t)i * q + i]);
  std::vector<int> perm(q);
  for (int i = 0; i < q; i++) perm[i] = i;
  int r = 0;
  for (; r < p1; r++) {
    int piv = r;
    for (int i = r + 1; i < p1; i++)
      if (M[(size_t)perm[i] * q + perm[i]] > M[(size_t)perm[piv] * q + perm[piv]]) piv = i;
    std::swap(perm[r], perm[piv]);
    const int s_ = perm[r];
    const double d = M[(size_t)s_ * q + s_];
    if (!(d > 1e-12 * dmax)) break;
    for (int i = r + 1; i < q; i++) {
      const int a = perm[i];
      const double f = M[(size_t)a * q + s_] / d;
      for (int jj = r + 1; jj < q; jj++) {
        const int b = perm[jj];
        M[(size_t)a * q + b] -= f * M[(size_t)s_ * q + b];
      }
    }
  }
  const double rss = std::max(0.0, M[(size_t)yi * q + yi]);
  *sigest = std::sqrt(rss / (n - r));
  if (rank) *rank = r;
  return FB_OK;
}

fb_status fb_cut_codes(const double* const* cols, int ncol, int n, const double* const* cutpoints, const int* ncut,
                       int device, uint8_t* q) {
  if (ncol < 0 || n < 0) return fail(FB_ERR_ARG, "ncol and n must be >= 0");
  if (ncol == 0 || n == 0) return FB_OK;
  if (!cols || !cutpoints || !ncut || !q) return fail(FB_ERR_ARG, "cols, cutpoints, ncut and q are required");
  std::vector<int> off(ncol + 1, 0);
  for (int v = 0; v < ncol; v++) {
    if (ncut[v] < 0 || ncut[v] > 255) return fail(FB_ERR_LIMIT, "predictor %d has %d cutpoints (0..255 allowed)", v, ncut[v]);
    if (ncut[v] > 0 && !cutpoints[v]) return fail(FB_ERR_ARG, "cutpoints of predictor %d are missing", v);
    for (int k = 1; k < ncut[v]; k++)
      if (!(cutpoints[v][k - 1] < cutpoints[v][k])) return fail(FB_ERR_ARG, "cutpoints of predictor %d are not increasing", v);
    off[v + 1] = off[v] + ncut[v];
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FB_ERR_CUDA, "no CUDA device is available");
  CK(cudaSetDevice(device));
  MlpJob job;
  double *dx = nullptr, *dc = nullptr;
  int* doff = nullptr;
  uint8_t* dq = nullptr;
  const size_t N = (size_t)ncol * n;
  if (!job.alloc(&dx, N) || !job.alloc(&dc, (size_t)std::max(off[ncol], 1)) || !job.alloc(&doff, off.size()) ||
      !job.alloc(&dq, N))
    return fail(FB_ERR_CUDA, "out of device memory");
  for (int v = 0; v < ncol; v++) {
    if (!cols[v]) return fail(FB_ERR_ARG, "column %d is missing", v);
    CK(cudaMemcpy(dx + (size_t)v * n, cols[v], sizeof(double) * n, cudaMemcpyHostToDevice));
    if (ncut[v] > 0) CK(cudaMemcpy(dc + off[v], cutpoints[v], sizeof(double) * ncut[v], cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(doff, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice));
  if (launch_cut_codes(dx, n, ncol, dc, doff, dq, nullptr) != 0)
    return fail(FB_ERR_CUDA, "cut-code launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  CK(cudaMemcpy(q, dq, N, cudaMemcpyDeviceToHost));
  return FB_OK;
}

// ------------------------------------------------------------------------------------------------ diagnostics
fb_status fb_debug_tree_pass(const fb_pass_state* s, int64_t* out) {
  if (!s || !out || !s->r || !s->w || !s->tho || !s->thn || !s->thc) return fail(FB_ERR_ARG, "missing argument");
  if (s->n < 1 || s->n > NMAX) return fail(FB_ERR_LIMIT, "n must be in 1..%d", NMAX);
  const int T = s->threads ? s->threads : 256;
  if (T < MIN_THREADS || T > MAX_THREADS || T % 32)
    return fail(FB_ERR_ARG, "threads must be a multiple of 32 in %d..%d", MIN_THREADS, MAX_THREADS);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(FB_ERR_CUDA, "no CUDA device is available");
  const int n = s->n, n_pad = (int)round_up(n, 16);
  std::vector<uint8_t> lp(n_pad, 0), lc(n_pad, 0), qp(n_pad, 0), qc(n_pad, 0);
  std::vector<float> r(n_pad, 0.0f), w(n_pad, 0.0f);
  if (s->leaf_prev) std::memcpy(lp.data(), s->leaf_prev, n);
  if (s->leaf_cur) std::memcpy(lc.data(), s->leaf_cur, n);
  if (s->qprev) std::memcpy(qp.data(), s->qprev, n);
  if (s->qcur) std::memcpy(qc.data(), s->qcur, n);
  std::memcpy(r.data(), s->r, sizeof(float) * n);
  std::memcpy(w.data(), s->w, sizeof(float) * n);
  uint8_t* dbytes = nullptr;
  float* dfl = nullptr;
  long long* dout = nullptr;
  CK(cudaMalloc(&dbytes, (size_t)n_pad * 4));
  CK(cudaMalloc(&dfl, sizeof(float) * ((size_t)n_pad * 3 + 3 * NODES)));
  CK(cudaMalloc(&dout, sizeof(long long) * 70));
  CK(cudaMemcpy(dbytes, lp.data(), n_pad, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dbytes + n_pad, lc.data(), n_pad, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dbytes + 2 * n_pad, qp.data(), n_pad, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dbytes + 3 * n_pad, qc.data(), n_pad, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dfl, r.data(), sizeof(float) * n_pad, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dfl + n_pad, w.data(), sizeof(float) * n_pad, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dfl + 2 * n_pad, s->tho, sizeof(float) * NODES, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dfl + 2 * n_pad + NODES, s->thn, sizeof(float) * NODES, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dfl + 2 * n_pad + 2 * NODES, s->thc, sizeof(float) * NODES, cudaMemcpyHostToDevice));
  DPassArgs a;
  std::memset(&a, 0, sizeof a);
  a.n = n; a.n_pad = n_pad; a.apply = s->apply; a.stats = s->stats;
  a.pmode = s->pmode; a.pnx = s->pnx; a.pc = s->pc; a.pL = s->pL; a.pR = s->pR; a.pl = s->pl; a.pr = s->pr;
  a.cmode = s->cmode; a.cnx = s->cnx; a.cc = s->cc; a.fx_shift = s->fx_shift; a.leafmask = s->leafmask;
  a.leaf_prev = dbytes; a.leaf_cur = dbytes + n_pad; a.qprev = dbytes + 2 * n_pad; a.qcur = dbytes + 3 * n_pad;
  a.r = dfl; a.w = dfl + n_pad; a.tho = dfl + 2 * n_pad; a.thn = dfl + 2 * n_pad + NODES;
  a.thc = dfl + 2 * n_pad + 2 * NODES; a.wscratch = dfl + 2 * n_pad + 3 * NODES; a.out = dout;
  fb_status st = FB_OK;
  if (launch_debug_pass(a, T, nullptr) != 0) st = fail(FB_ERR_CUDA, "debug pass launch failed");
  if (st == FB_OK && cudaDeviceSynchronize() != cudaSuccess) st = fail(FB_ERR_CUDA, "debug pass failed: %s", cudaGetErrorString(cudaGetLastError()));
  if (st == FB_OK) {
    if (cudaMemcpy(out, dout, sizeof(long long) * 70, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(s->r, dfl, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
        (s->leaf_prev && cudaMemcpy(s->leaf_prev, dbytes, n, cudaMemcpyDeviceToHost) != cudaSuccess))
      st = fail(FB_ERR_CUDA, "copy back failed");
  }
  cudaFree(dbytes); cudaFree(dfl); cudaFree(dout);
  return st;
}

}  // extern "C"
