// mlp.cu -- training kernels of the learned split-variable proposal (no counterpart in the reference).
//
// The model is the sampler's proposal MLP: MLP_IN node features -> MLP_H -> MLP_H -> MLP_OUT logits (ReLU between),
// BF16 weights and FP32 biases, trained by masked softmax cross-entropy on accepted births (the split variable
// given the node's features, over the predictors with a non-empty cut range at the node).
//
// Parameters live in one flat FP32 vector (the master copy) in the order w1 [H][IN], b1 [H], w2 [H][H], b2 [H],
// w3 [OUT][H], b3 [OUT]; the forward pass reads the BF16-rounded weights, exactly as the sampler does.
//   mlp_grad_kernel   one CTA per tile of MT_TILE examples: forward, softmax, backward for the tile in shared
//                     memory, then one atomic add per parameter and tile into the FP32 gradient vector (and the
//                     tile's summed loss).  Every GEMM of the forward pass, the backward pass and the weight
//                     gradients runs on the tensor cores (warp_gemm below: mma.sync m16n8k8 TF32 tiles with FP32
//                     accumulation, operands split into two TF32 parts so that the products keep FP32 accuracy).
//   cut_grad_kernel   the same for the cutpoint head (40 -> 64 -> 64 -> 16, then 255 cut logits).
//   mlp_adam_kernel   Adam step on the master weights from the summed gradients / batch size, refreshing the BF16
//                     copies of the weights.
#include <cuda_runtime.h>

#include <cstdint>

#include "fb_internal.h"

namespace fb {

constexpr int MT_TILE = 32;
constexpr int MT_THREADS = 256;

__device__ __forceinline__ float bf16_to_f(uint16_t h) { return __uint_as_float((unsigned)h << 16); }

// ---- GEMM tiles on the tensor cores.  A warp computes a 16 x 8 tile of C = A B with mma.sync m16n8k8 (TF32 inputs,
// FP32 accumulation).  TF32 keeps 10 mantissa bits, so each operand is split as x = hi + lo with hi = tf32(x) and
// lo = tf32(x - hi), and the tile accumulates lo*hi + hi*lo + hi*hi (the small terms first): the error of the
// dropped lo*lo term and of the splits is about 2^-21 of the product, as with FP32 arithmetic (the split-TF32 scheme
// of Ootomo and Yokota, 2022).  Fragment layout of m16n8k8 (PTX ISA): lane = 4 g + t; A holds (g, t), (g + 8, t),
// (g, t + 4), (g + 8, t + 4); B holds (t, g), (t + 4, g); C holds (g, 2t), (g, 2t + 1), (g + 8, 2t), (g + 8, 2t + 1).
__device__ __forceinline__ uint32_t tf32_of(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = tf32_of(x);
  lo = tf32_of(__fsub_rn(x, __uint_as_float(hi)));
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
               "{%0, %1, %2, %3};\n"
               : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
// C (M x N, multiples of 16 and 8) = A (M x K) B (K x N), K a multiple of 8: the CTA's warps take the 16 x 8 tiles in
// turn; A(m, k) and B(k, n) return the operands (zero in the padding), E(m, n, value) consumes each result.
template <class FA, class FB, class FE>
__device__ __forceinline__ void warp_gemm(int M, int N, int K, FA A, FB B, FE E) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3, nt = N / 8, tiles = (M / 16) * nt;
  for (int p = warp; p < tiles; p += nw) {
    const int m0 = (p / nt) * 16, n0 = (p % nt) * 8;
    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (int k0 = 0; k0 < K; k0 += 8) {
      uint32_t ah[4], al[4], bh[2], bl[2];
      split_tf32(A(m0 + g, k0 + t), ah[0], al[0]);
      split_tf32(A(m0 + g + 8, k0 + t), ah[1], al[1]);
      split_tf32(A(m0 + g, k0 + t + 4), ah[2], al[2]);
      split_tf32(A(m0 + g + 8, k0 + t + 4), ah[3], al[3]);
      split_tf32(B(k0 + t, n0 + g), bh[0], bl[0]);
      split_tf32(B(k0 + t + 4, n0 + g), bh[1], bl[1]);
      mma_tf32(c, al, bh);
      mma_tf32(c, ah, bl);
      mma_tf32(c, ah, bh);
    }
#pragma unroll
    for (int e = 0; e < 4; e++) E(m0 + g + 8 * (e >> 1), n0 + 2 * t + (e & 1), c[e]);
  }
}
constexpr int pad8(int k) { return (k + 7) / 8 * 8; }
__device__ __forceinline__ uint16_t f_to_bf16(float f) {   // round to nearest even (finite inputs)
  const unsigned u = __float_as_uint(f);
  return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}

__global__ void __launch_bounds__(MT_THREADS) mlp_grad_kernel(MlpParams P, const float* __restrict__ X,
                                                              const int* __restrict__ Y,
                                                              const unsigned* __restrict__ M,
                                                              const int* __restrict__ idx, int B,
                                                              float* __restrict__ grad, float* __restrict__ loss) {
  extern __shared__ float ms[];
  float* w1 = ms;                           // [H][IN]
  float* w2 = w1 + MLP_H * MLP_IN;          // [H][H]
  float* w3 = w2 + MLP_H * MLP_H;           // [OUT][H]
  float* xs = w3 + MLP_OUT * MLP_H;         // [TILE][IN]
  float* h1 = xs + MT_TILE * MLP_IN;        // [TILE][H]
  float* h2 = h1 + MT_TILE * MLP_H;         // [TILE][H]
  float* g3 = h2 + MT_TILE * MLP_H;         // [TILE][OUT]
  float* d2 = g3 + MT_TILE * MLP_OUT;       // [TILE][H]
  float* d1 = d2 + MT_TILE * MLP_H;         // [TILE][H]
  float* lsum = d1 + MT_TILE * MLP_H;       // [1]
  const int tid = threadIdx.x;
  const int b0 = blockIdx.x * MT_TILE;
  const int nb = min(MT_TILE, B - b0);
  for (int k = tid; k < MLP_H * MLP_IN; k += MT_THREADS) w1[k] = bf16_to_f(P.w1[k]);
  for (int k = tid; k < MLP_H * MLP_H; k += MT_THREADS) w2[k] = bf16_to_f(P.w2[k]);
  for (int k = tid; k < MLP_OUT * MLP_H; k += MT_THREADS) w3[k] = bf16_to_f(P.w3[k]);
  for (int k = tid; k < MT_TILE * MLP_IN; k += MT_THREADS) {
    const int b = k / MLP_IN, f = k % MLP_IN;
    xs[k] = b < nb ? X[(long long)(idx ? idx[b0 + b] : b0 + b) * MLP_IN + f] : 0.0f;
  }
  if (tid == 0) *lsum = 0.0f;
  __syncthreads();
  // forward: h1 = relu(x W1^T + b1), h2 = relu(h1 W2^T + b2), logits = h2 W3^T + b3
  warp_gemm(MT_TILE, MLP_H, pad8(MLP_IN),
            [&](int b, int f) { return f < MLP_IN ? xs[b * MLP_IN + f] : 0.0f; },
            [&](int f, int h) { return f < MLP_IN ? w1[h * MLP_IN + f] : 0.0f; },
            [&](int b, int h, float v) { v = __fadd_rn(v, P.b1[h]); h1[b * MLP_H + h] = v > 0.0f ? v : 0.0f; });
  __syncthreads();
  warp_gemm(MT_TILE, MLP_H, MLP_H,
            [&](int b, int f) { return h1[b * MLP_H + f]; },
            [&](int f, int h) { return w2[h * MLP_H + f]; },
            [&](int b, int h, float v) { v = __fadd_rn(v, P.b2[h]); h2[b * MLP_H + h] = v > 0.0f ? v : 0.0f; });
  __syncthreads();
  warp_gemm(MT_TILE, MLP_OUT, MLP_H,
            [&](int b, int f) { return h2[b * MLP_H + f]; },
            [&](int f, int o) { return w3[o * MLP_H + f]; },
            [&](int b, int o, float v) { g3[b * MLP_OUT + o] = __fadd_rn(v, P.b3[o]); });
  __syncthreads();
  // masked softmax and cross-entropy, one thread per example: g3 becomes dLoss/dz (summed, not averaged)
  if (tid < MT_TILE) {
    const int b = tid;
    float* z = g3 + b * MLP_OUT;
    if (b < nb) {
      const long long e = idx ? idx[b0 + b] : b0 + b;
      const unsigned mk = M[e];
      const int y = Y[e];
      float zmax = -3.0e38f;
      for (int o = 0; o < MLP_OUT; o++) if ((mk >> o) & 1u) zmax = fmaxf(zmax, z[o]);
      float S = 0.0f;
      for (int o = 0; o < MLP_OUT; o++) S += ((mk >> o) & 1u) ? __expf(z[o] - zmax) : 0.0f;
      atomicAdd(lsum, -(z[y] - zmax - __logf(S)));
      for (int o = 0; o < MLP_OUT; o++)
        z[o] = (((mk >> o) & 1u) ? __expf(z[o] - zmax) / S : 0.0f) - (o == y ? 1.0f : 0.0f);
    } else {
      for (int o = 0; o < MLP_OUT; o++) z[o] = 0.0f;
    }
  }
  __syncthreads();
  // backward through layer 3 and the second ReLU, then layer 2 and the first ReLU
  warp_gemm(MT_TILE, MLP_H, MLP_OUT,
            [&](int b, int o) { return g3[b * MLP_OUT + o]; },
            [&](int o, int h) { return w3[o * MLP_H + h]; },
            [&](int b, int h, float v) { d2[b * MLP_H + h] = h2[b * MLP_H + h] > 0.0f ? v : 0.0f; });
  __syncthreads();
  warp_gemm(MT_TILE, MLP_H, MLP_H,
            [&](int b, int o) { return d2[b * MLP_H + o]; },
            [&](int o, int h) { return w2[o * MLP_H + h]; },
            [&](int b, int h, float v) { d1[b * MLP_H + h] = h1[b * MLP_H + h] > 0.0f ? v : 0.0f; });
  __syncthreads();
  // parameter gradients of the tile (sums over its examples), one atomic add each
  float* gw1 = grad;
  float* gb1 = gw1 + MLP_H * MLP_IN;
  float* gw2 = gb1 + MLP_H;
  float* gb2 = gw2 + MLP_H * MLP_H;
  float* gw3 = gb2 + MLP_H;
  float* gb3 = gw3 + MLP_OUT * MLP_H;
  warp_gemm(MLP_H, pad8(MLP_IN), MT_TILE,
            [&](int h, int b) { return b < nb ? d1[b * MLP_H + h] : 0.0f; },
            [&](int b, int f) { return f < MLP_IN ? xs[b * MLP_IN + f] : 0.0f; },
            [&](int h, int f, float v) { if (f < MLP_IN) atomicAdd(gw1 + h * MLP_IN + f, v); });
  warp_gemm(MLP_H, MLP_H, MT_TILE,
            [&](int h, int b) { return b < nb ? d2[b * MLP_H + h] : 0.0f; },
            [&](int b, int f) { return h1[b * MLP_H + f]; },
            [&](int h, int f, float v) { atomicAdd(gw2 + h * MLP_H + f, v); });
  warp_gemm(MLP_OUT, MLP_H, MT_TILE,
            [&](int o, int b) { return b < nb ? g3[b * MLP_OUT + o] : 0.0f; },
            [&](int b, int f) { return h2[b * MLP_H + f]; },
            [&](int o, int f, float v) { atomicAdd(gw3 + o * MLP_H + f, v); });
  if (tid < MLP_H) {
    float a = 0.0f, c = 0.0f;
    for (int b = 0; b < nb; b++) { a += d1[b * MLP_H + tid]; c += d2[b * MLP_H + tid]; }
    atomicAdd(gb1 + tid, a);
    atomicAdd(gb2 + tid, c);
  }
  if (tid < MLP_OUT) {
    float a = 0.0f;
    for (int b = 0; b < nb; b++) a += g3[b * MLP_OUT + tid];
    atomicAdd(gb3 + tid, a);
  }
  __syncthreads();
  if (tid == 0) atomicAdd(loss, *lsum);
}

// Adam on the flat parameter vector; weights (not biases) also refresh their BF16 copies.
__global__ void mlp_adam_kernel(float* __restrict__ p, float* __restrict__ m1, float* __restrict__ m2,
                                const float* __restrict__ g, int n, float inv_batch, float lr, float c1, float c2,
                                MlpParams P) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float gk = g[k] * inv_batch;
  const float a = 0.9f * m1[k] + 0.1f * gk;
  const float b = 0.999f * m2[k] + 0.001f * gk * gk;
  m1[k] = a;
  m2[k] = b;
  const float w = p[k] - lr * (a * c1) / (sqrtf(b * c2) + 1e-8f);
  p[k] = w;
  const int o1 = MLP_H * MLP_IN, o2 = o1 + MLP_H, o3 = o2 + MLP_H * MLP_H, o4 = o3 + MLP_H, o5 = o4 + MLP_OUT * MLP_H;
  if (k < o1) P.w1[k] = f_to_bf16(w);
  else if (k >= o2 && k < o3) P.w2[k - o2] = f_to_bf16(w);
  else if (k >= o4 && k < o5) P.w3[k - o4] = f_to_bf16(w);
}

size_t mlp_grad_smem() {
  return sizeof(float) * ((size_t)MLP_H * MLP_IN + MLP_H * MLP_H + MLP_OUT * MLP_H +
                          (size_t)MT_TILE * (MLP_IN + 4 * MLP_H + MLP_OUT) + 1);
}

int mlp_grad_launch(const MlpParams& P, const float* X, const int* Y, const unsigned* M, const int* idx, int B,
                    float* grad, float* loss, void* stream) {
  if (B <= 0) return 0;
  const size_t smem = mlp_grad_smem();
  if (cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return -1;
  mlp_grad_kernel<<<(B + MT_TILE - 1) / MT_TILE, MT_THREADS, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
      P, X, Y, M, idx, B, grad, loss);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int mlp_adam_launch(float* p, float* m1, float* m2, const float* g, float inv_batch, float lr, int step,
                    const MlpParams& P, void* stream) {
  const int n = MLP_NPARAM;
  const float c1 = 1.0f / (1.0f - powf(0.9f, (float)step)), c2 = 1.0f / (1.0f - powf(0.999f, (float)step));
  mlp_adam_kernel<<<(n + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(p, m1, m2, g, n, inv_batch,
                                                                                       lr, c1, c2, P);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// ------------------------------------------------------------------------------------------------ cut head
// Training of the learned cut proposal's head: CUT_IN features -> CUT_H -> CUT_H -> CUT_E -> logits be[c] + emb[c] . e,
// softmax cross-entropy over each example's cut range [lo, hi].  Flat FP32 parameters w1 [H][IN], b1 [H], w2 [H][H],
// b2 [H], w3 [E][H], b3 [E], emb [BINS][E], be [BINS]; the forward pass reads the BF16-rounded weights.
constexpr int CT_ZS = 256;   // logits per example (padded)

__global__ void __launch_bounds__(MT_THREADS) cut_grad_kernel(CutParams P, const float* __restrict__ X,
                                                              const int* __restrict__ Yc, const int* __restrict__ LO,
                                                              const int* __restrict__ HI, const int* __restrict__ idx,
                                                              int B, float* __restrict__ grad,
                                                              float* __restrict__ loss) {
  extern __shared__ float cms[];
  float* w1 = cms;                          // [H][IN]
  float* w2 = w1 + CUT_H * CUT_IN;          // [H][H]
  float* w3 = w2 + CUT_H * CUT_H;           // [E][H]
  float* em = w3 + CUT_E * CUT_H;           // [BINS][E]
  float* xs = em + CUT_BINS * CUT_E;        // [TILE][IN]
  float* h1 = xs + MT_TILE * CUT_IN;        // [TILE][H]
  float* h2 = h1 + MT_TILE * CUT_H;         // [TILE][H]
  float* ev = h2 + MT_TILE * CUT_H;         // [TILE][E]
  float* dz = ev + MT_TILE * CUT_E;         // [TILE][CT_ZS]: logits, then dLoss/dz
  float* de = dz + MT_TILE * CT_ZS;         // [TILE][E]
  float* d2 = de + MT_TILE * CUT_E;         // [TILE][H]
  float* d1 = d2 + MT_TILE * CUT_H;         // [TILE][H]
  float* lsum = d1 + MT_TILE * CUT_H;       // [1]
  int* lo = reinterpret_cast<int*>(lsum + 1);   // [TILE]
  int* hi = lo + MT_TILE;
  int* yc = hi + MT_TILE;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int b0 = blockIdx.x * MT_TILE;
  const int nb = min(MT_TILE, B - b0);
  for (int k = tid; k < CUT_H * CUT_IN; k += MT_THREADS) w1[k] = bf16_to_f(P.w1[k]);
  for (int k = tid; k < CUT_H * CUT_H; k += MT_THREADS) w2[k] = bf16_to_f(P.w2[k]);
  for (int k = tid; k < CUT_E * CUT_H; k += MT_THREADS) w3[k] = bf16_to_f(P.w3[k]);
  for (int k = tid; k < CUT_BINS * CUT_E; k += MT_THREADS) em[k] = bf16_to_f(P.emb[k]);
  for (int k = tid; k < MT_TILE * CUT_IN; k += MT_THREADS) {
    const int b = k / CUT_IN, f = k % CUT_IN;
    xs[k] = b < nb ? X[(long long)(idx ? idx[b0 + b] : b0 + b) * CUT_IN + f] : 0.0f;
  }
  if (tid < MT_TILE) {
    const long long e = tid < nb ? (idx ? idx[b0 + tid] : b0 + tid) : -1;
    lo[tid] = e >= 0 ? LO[e] : 0; hi[tid] = e >= 0 ? HI[e] : -1; yc[tid] = e >= 0 ? Yc[e] : 0;
  }
  if (tid == 0) *lsum = 0.0f;
  __syncthreads();
  // forward: h1, h2 (ReLU), the embedding e = h2 W3^T + b3, and the logits be[c] + emb[c] . e inside [lo, hi]
  warp_gemm(MT_TILE, CUT_H, pad8(CUT_IN),
            [&](int b, int f) { return f < CUT_IN ? xs[b * CUT_IN + f] : 0.0f; },
            [&](int f, int h) { return f < CUT_IN ? w1[h * CUT_IN + f] : 0.0f; },
            [&](int b, int h, float v) { v = __fadd_rn(v, P.b1[h]); h1[b * CUT_H + h] = v > 0.0f ? v : 0.0f; });
  __syncthreads();
  warp_gemm(MT_TILE, CUT_H, CUT_H,
            [&](int b, int f) { return h1[b * CUT_H + f]; },
            [&](int f, int h) { return w2[h * CUT_H + f]; },
            [&](int b, int h, float v) { v = __fadd_rn(v, P.b2[h]); h2[b * CUT_H + h] = v > 0.0f ? v : 0.0f; });
  __syncthreads();
  warp_gemm(MT_TILE, CUT_E, CUT_H,
            [&](int b, int f) { return h2[b * CUT_H + f]; },
            [&](int f, int q) { return w3[q * CUT_H + f]; },
            [&](int b, int q, float v) { ev[b * CUT_E + q] = __fadd_rn(v, P.b3[q]); });
  __syncthreads();
  warp_gemm(MT_TILE, CT_ZS, CUT_E,
            [&](int b, int q) { return ev[b * CUT_E + q]; },
            [&](int q, int c) { return c < CUT_BINS ? em[c * CUT_E + q] : 0.0f; },
            [&](int b, int c, float v) {
              dz[b * CT_ZS + c] = (c >= lo[b] && c <= hi[b]) ? __fadd_rn(v, P.be[c]) : 0.0f;
            });
  __syncthreads();
  // softmax over [lo, hi] and cross-entropy, one warp per example: dz becomes dLoss/dz (summed, not averaged)
  for (int b = warp; b < MT_TILE; b += MT_THREADS / 32) {
    float* z = dz + b * CT_ZS;
    const int L = lo[b], U = hi[b];
    if (b >= nb) {
      for (int c = lane; c < CT_ZS; c += 32) z[c] = 0.0f;
      continue;
    }
    float zm = -3.0e38f;
    for (int c = L + lane; c <= U; c += 32) zm = fmaxf(zm, z[c]);
    for (int o = 16; o > 0; o >>= 1) zm = fmaxf(zm, __shfl_xor_sync(0xffffffffu, zm, o));
    float S = 0.0f;
    for (int c = L + lane; c <= U; c += 32) S += __expf(z[c] - zm);
    for (int o = 16; o > 0; o >>= 1) S += __shfl_xor_sync(0xffffffffu, S, o);
    const float zy = z[yc[b]];
    __syncwarp();
    for (int c = lane; c < CT_ZS; c += 32)
      z[c] = (c >= L && c <= U) ? __expf(z[c] - zm) / S - (c == yc[b] ? 1.0f : 0.0f) : 0.0f;
    if (lane == 0) atomicAdd(lsum, -(zy - zm - __logf(S)));
  }
  __syncthreads();
  // backward: de = dz emb (dz is zero outside [lo, hi]), then the two ReLU layers
  warp_gemm(MT_TILE, CUT_E, CT_ZS,
            [&](int b, int c) { return dz[b * CT_ZS + c]; },
            [&](int c, int q) { return c < CUT_BINS ? em[c * CUT_E + q] : 0.0f; },
            [&](int b, int q, float v) { de[b * CUT_E + q] = v; });
  __syncthreads();
  warp_gemm(MT_TILE, CUT_H, CUT_E,
            [&](int b, int q) { return de[b * CUT_E + q]; },
            [&](int q, int f) { return w3[q * CUT_H + f]; },
            [&](int b, int f, float v) { d2[b * CUT_H + f] = h2[b * CUT_H + f] > 0.0f ? v : 0.0f; });
  __syncthreads();
  warp_gemm(MT_TILE, CUT_H, CUT_H,
            [&](int b, int h) { return d2[b * CUT_H + h]; },
            [&](int h, int f) { return w2[h * CUT_H + f]; },
            [&](int b, int f, float v) { d1[b * CUT_H + f] = h1[b * CUT_H + f] > 0.0f ? v : 0.0f; });
  __syncthreads();
  float* gw1 = grad;
  float* gb1 = gw1 + CUT_H * CUT_IN;
  float* gw2 = gb1 + CUT_H;
  float* gb2 = gw2 + CUT_H * CUT_H;
  float* gw3 = gb2 + CUT_H;
  float* gb3 = gw3 + CUT_E * CUT_H;
  float* gem = gb3 + CUT_E;
  float* gbe = gem + CUT_BINS * CUT_E;
  // parameter gradients of the tile (sums over its examples), one atomic add each
  warp_gemm(CUT_H, pad8(CUT_IN), MT_TILE,
            [&](int h, int b) { return b < nb ? d1[b * CUT_H + h] : 0.0f; },
            [&](int b, int f) { return f < CUT_IN ? xs[b * CUT_IN + f] : 0.0f; },
            [&](int h, int f, float v) { if (f < CUT_IN) atomicAdd(gw1 + h * CUT_IN + f, v); });
  warp_gemm(CUT_H, CUT_H, MT_TILE,
            [&](int h, int b) { return b < nb ? d2[b * CUT_H + h] : 0.0f; },
            [&](int b, int f) { return h1[b * CUT_H + f]; },
            [&](int h, int f, float v) { atomicAdd(gw2 + h * CUT_H + f, v); });
  warp_gemm(CUT_E, CUT_H, MT_TILE,
            [&](int q, int b) { return b < nb ? de[b * CUT_E + q] : 0.0f; },
            [&](int b, int f) { return h2[b * CUT_H + f]; },
            [&](int q, int f, float v) { atomicAdd(gw3 + q * CUT_H + f, v); });
  warp_gemm(CT_ZS, CUT_E, MT_TILE,
            [&](int c, int b) { return b < nb ? dz[b * CT_ZS + c] : 0.0f; },
            [&](int b, int q) { return ev[b * CUT_E + q]; },
            [&](int c, int q, float v) { if (c < CUT_BINS) atomicAdd(gem + c * CUT_E + q, v); });
  if (tid < CUT_H) {
    float a = 0.0f, c = 0.0f;
    for (int b = 0; b < nb; b++) { a += d1[b * CUT_H + tid]; c += d2[b * CUT_H + tid]; }
    atomicAdd(gb1 + tid, a);
    atomicAdd(gb2 + tid, c);
  }
  if (tid < CUT_E) {
    float a = 0.0f;
    for (int b = 0; b < nb; b++) a += de[b * CUT_E + tid];
    atomicAdd(gb3 + tid, a);
  }
  for (int c = tid; c < CUT_BINS; c += MT_THREADS) {
    float a = 0.0f;
    for (int b = 0; b < nb; b++) a += dz[b * CT_ZS + c];
    atomicAdd(gbe + c, a);
  }
  __syncthreads();
  if (tid == 0) atomicAdd(loss, *lsum);
}

// Adam on the cut head's flat parameter vector; the weight matrices also refresh their BF16 copies.
__global__ void cut_adam_kernel(float* __restrict__ p, float* __restrict__ m1, float* __restrict__ m2,
                                const float* __restrict__ g, int n, float inv_batch, float lr, float c1, float c2,
                                CutParams P) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float gk = g[k] * inv_batch;
  const float a = 0.9f * m1[k] + 0.1f * gk;
  const float b = 0.999f * m2[k] + 0.001f * gk * gk;
  m1[k] = a;
  m2[k] = b;
  const float w = p[k] - lr * (a * c1) / (sqrtf(b * c2) + 1e-8f);
  p[k] = w;
  const int o1 = CUT_H * CUT_IN, o2 = o1 + CUT_H, o3 = o2 + CUT_H * CUT_H, o4 = o3 + CUT_H, o5 = o4 + CUT_E * CUT_H,
            o6 = o5 + CUT_E, o7 = o6 + CUT_BINS * CUT_E;
  if (k < o1) P.w1[k] = f_to_bf16(w);
  else if (k >= o2 && k < o3) P.w2[k - o2] = f_to_bf16(w);
  else if (k >= o4 && k < o5) P.w3[k - o4] = f_to_bf16(w);
  else if (k >= o6 && k < o7) P.emb[k - o6] = f_to_bf16(w);
}

size_t cut_grad_smem() {
  return sizeof(float) * ((size_t)CUT_H * CUT_IN + CUT_H * CUT_H + CUT_E * CUT_H + CUT_BINS * CUT_E +
                          (size_t)MT_TILE * (CUT_IN + 4 * CUT_H + 2 * CUT_E + CT_ZS) + 1) +
         sizeof(int) * 3 * MT_TILE;
}

int cut_grad_launch(const CutParams& P, const float* X, const int* Yc, const int* LO, const int* HI, const int* idx,
                    int B, float* grad, float* loss, void* stream) {
  if (B <= 0) return 0;
  const size_t smem = cut_grad_smem();
  if (cudaFuncSetAttribute(cut_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return -1;
  cut_grad_kernel<<<(B + MT_TILE - 1) / MT_TILE, MT_THREADS, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
      P, X, Yc, LO, HI, idx, B, grad, loss);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int cut_adam_launch(float* p, float* m1, float* m2, const float* g, float inv_batch, float lr, int step,
                    const CutParams& P, void* stream) {
  const int n = CUT_NPARAM;
  const float c1 = 1.0f / (1.0f - powf(0.9f, (float)step)), c2 = 1.0f / (1.0f - powf(0.999f, (float)step));
  cut_adam_kernel<<<(n + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(p, m1, m2, g, n, inv_batch,
                                                                                       lr, c1, c2, P);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace fb
