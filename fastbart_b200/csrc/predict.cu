// predict.cu -- predict_draw on the device (src/predict.cpp:49-73).
//
// Streaming evaluator: each thread owns one row of one draw and walks the draw's trees in order 1..ntree with the
// branch-free step k = child[k] + (x[var[k]] >= cut[k]) over the breadth-first node arrays (children adjacent), adding
// leaf values to an FP64 accumulator that starts at 0; mu is added last.  That is the reference's summation order, so
// results are bit-identical to predict_draw_cpp / pwbart.  Rows of a warp are consecutive, so the x reads of each
// node visit are coalesced (column-major x); node arrays are read through the read-only cache, where all threads of a
// draw share them.  The grid's y dimension enumerates draws, so a bulk call (many draws) runs in one launch.
#include <cuda_runtime.h>

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

int launch_predict(const DForest& f, const double* x, int n, int ld, int draw0, int ndraws, double mu, double* out,
                   int ldo, void* stream) {
  if (n <= 0 || ndraws <= 0) return 0;
  const int T = 256;
  for (int d0 = 0; d0 < ndraws; d0 += 65535) {
    const int nd = ndraws - d0 < 65535 ? ndraws - d0 : 65535;
    dim3 grid((n + T - 1) / T, nd);
    predict_kernel<<<grid, T, 0, reinterpret_cast<cudaStream_t>(stream)>>>(f, x, n, ld, draw0 + d0, mu,
                                                                            out + (long long)d0 * ldo, ldo);
    if (cudaGetLastError() != cudaSuccess) return -1;
  }
  return 0;
}

}  // namespace fb
