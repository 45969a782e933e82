// latent.cu -- the probit latent redraw of fpbart (src/bart_kernel.cpp:280-292, 543-547) as a streaming kernel.
//
// Inside the sampler the redraw is fused into the end-of-sweep pass, which has just computed every row's fit.  This
// kernel runs the same step on its own over device arrays: for row i with fit f_i (the sum of the trees, without the
// offset) and outcome ybin_i, z_i is N(f_i, 1) truncated to z > -offset when ybin_i = 1 and to z < -offset when
// ybin_i = 0, drawn by fb_rtnorm with the sampler's counters (chain seed, row, sweep), so it equals the value the
// sampler draws for that row and sweep.  One thread per row, grid-stride over the rows: per row it reads the fit
// (8 B) and the outcome (4 B) and writes z (8 B) once.
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
