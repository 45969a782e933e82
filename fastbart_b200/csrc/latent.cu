// latent.cu -- the probit latent redraw of fpbart (src/bart_kernel.cpp:280-292, 543-547) as a streaming kernel.
//
// Inside the sampler the redraw is fused into the end-of-sweep pass, which has just computed every row's fit.  This
// kernel runs the same step on its own over device arrays: for row i with fit f_i (the sum of the trees, without the
// offset) and outcome ybin_i, z_i is N(f_i, 1) truncated to z > -offset when ybin_i = 1 and to z < -offset when
// ybin_i = 0, drawn by fb_rtnorm with the sampler's counters (chain seed, row, sweep), so it equals the value the
// sampler draws for that row and sweep.  One thread per row, grid-stride over the rows: per row it reads the fit
// (8 B) and the outcome (4 B) and writes z (8 B) once.
//
// It also holds the Gram sums behind the least-squares sigest of the preprocessing (R/fwbart.R:22), the one step of
// the R wrapper's preparation that reads every row and column again.
#include <cuda_runtime.h>

#include "fb_internal.h"
#include "fb_math.cuh"

namespace fb {

__global__ void __launch_bounds__(256) probit_latent_kernel(const double* __restrict__ fit, const int* __restrict__ ybin,
                                                            long long n, double offset, uint64_t seed, uint32_t sweep,
                                                            double* __restrict__ z, int* __restrict__ capped) {
  int caps = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double f = fit[i];
    z[i] = ybin[i] == 0 ? -fbm::fb_rtnorm(seed, (uint32_t)i, sweep, -f, offset, &caps)
                        : fbm::fb_rtnorm(seed, (uint32_t)i, sweep, f, -offset, &caps);
  }
  if (capped && caps) atomicAdd(capped, caps);
}

int launch_probit_latent(const double* fit, const int* ybin, long long n, double offset, uint64_t seed, uint32_t sweep,
                         double* z, int* capped, void* stream) {
  if (n <= 0) return 0;
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long blocks = (n + 255) / 256, cap = 8ll * nsm;   // 8 CTAs of 256 per SM, grid-stride beyond
  probit_latent_kernel<<<(unsigned)(blocks < cap ? blocks : cap), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      fit, ybin, n, offset, seed, sweep, z, capped);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace fb

namespace fb {

// Gram sums of the least-squares fit behind sigest (R/fwbart.R:22: summary(lm(yc ~ X))$sigma): for the augmented
// columns a = [1, x_1 .. x_p, y], every sum over rows of a_j a_k (j <= k), in FP64.  CTA r takes rows
// [r chunk, (r + 1) chunk) in tiles of GR_ROWS staged in shared memory; thread t keeps the pairs t, t + 256, ... in
// registers over the CTA's rows and writes them to part[r][pair] (the host adds the CTAs' sums in a fixed order).
constexpr int GR_ROWS = 64, GR_MAXQ = 34, GR_PAIRS = GR_MAXQ * (GR_MAXQ + 1) / 2, GR_PER = (GR_PAIRS + 255) / 256;

__global__ void __launch_bounds__(256) gram_kernel(const double* __restrict__ x, int n, int p,
                                                   const double* __restrict__ y, int chunk, double* __restrict__ part) {
  __shared__ double a_s[GR_MAXQ][GR_ROWS];
  __shared__ uint8_t pj[GR_PAIRS], pk[GR_PAIRS];
  const int q = p + 2, npairs = q * (q + 1) / 2, tid = threadIdx.x;
  for (int t = tid; t < npairs; t += 256) {   // pair index -> (j, k), j <= k
    int j = 0, r = t;
    while (r >= q - j) { r -= q - j; j++; }
    pj[t] = (uint8_t)j; pk[t] = (uint8_t)(j + r);
  }
  double acc[GR_PER];
#pragma unroll
  for (int u = 0; u < GR_PER; u++) acc[u] = 0.0;
  const long long r0 = (long long)blockIdx.x * chunk, r1 = min((long long)n, r0 + chunk);
  for (long long t0 = r0; t0 < r1; t0 += GR_ROWS) {
    __syncthreads();
    for (int k = tid; k < q * GR_ROWS; k += 256) {
      const int c = k / GR_ROWS, i = k % GR_ROWS;
      const long long row = t0 + i;
      double v = 0.0;
      if (row < r1) v = c == 0 ? 1.0 : (c <= p ? x[(long long)(c - 1) * n + row] : y[row]);
      a_s[c][i] = v;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < GR_PER; u++) {
      const int t = tid + 256 * u;
      if (t < npairs) {
        const double* aj = a_s[pj[t]];
        const double* ak = a_s[pk[t]];
        double s = acc[u];
        for (int i = 0; i < GR_ROWS; i++) s = __dadd_rn(s, __dmul_rn(aj[i], ak[i]));
        acc[u] = s;
      }
    }
  }
#pragma unroll
  for (int u = 0; u < GR_PER; u++) {
    const int t = tid + 256 * u;
    if (t < npairs) part[(long long)blockIdx.x * npairs + t] = acc[u];
  }
}

int launch_gram(const double* x, int n, int p, const double* y, int nblocks, int chunk, double* part, void* stream) {
  if (p + 2 > GR_MAXQ) return -2;
  gram_kernel<<<nblocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(x, n, p, y, chunk, part);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace fb
