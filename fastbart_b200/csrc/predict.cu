// predict.cu -- predict_draw on the device (src/predict.cpp:49-73).
//
// Streaming evaluator: each thread owns one row of one draw and walks the draw's trees in order 1..ntree with the
// branch-free step k = child[k] + (x[var[k]] >= cut[k]) over the breadth-first node arrays (children adjacent), adding
// leaf values to an FP64 accumulator that starts at 0; mu is added last.  That is the reference's summation order, so
// results are bit-identical to predict_draw_cpp / pwbart.  Rows of a warp are consecutive, so the x reads of each
// node visit are coalesced (column-major x); node arrays are read through the read-only cache, where all threads of a
// draw share them.  The grid's y dimension enumerates draws, so a bulk call (many draws) runs in one launch.
#include <cuda_runtime.h>

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
