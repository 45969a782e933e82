// text.cu -- BART tree text assembled on the device: the format of src/glue.cpp:29-57 (header "ndpost ntree p", then
// per tree its node count and one line "nid v c theta" per node in pre-order, root 1, children 2 nid and 2 nid + 1,
// theta printed as printf("%.10g") prints the leaf value, 0 for internal nodes), byte for byte what the host writer
// fb_trees_text produces.  One thread per tree: a length pass, an exclusive scan of the lengths, a writing pass.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include "fb_internal.h"

namespace fb {
namespace {

// ---- exact decimal conversion of a float, as printf("%.10g") does it (round to nearest, exact ties to even)
// A float is M 2^E exactly (M < 2^24).  Its 10 significant digits are N = round(M 2^E 10^s) with s = 9 - X, X the
// decimal exponent, computed as P / Q with P, Q integers below 2^192; N comes from a double estimate corrected with
// exact integer arithmetic.
struct U192 { unsigned long long w[3]; };

__device__ __forceinline__ U192 u192(unsigned long long a) { U192 r; r.w[0] = a; r.w[1] = 0; r.w[2] = 0; return r; }
__device__ U192 mul64(const U192& a, unsigned long long m) {   // the product must fit 192 bits
  U192 r;
  unsigned long long carry = 0;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const unsigned long long lo = a.w[i] * m, hi = __umul64hi(a.w[i], m);
    r.w[i] = lo + carry;
    carry = hi + (r.w[i] < lo ? 1ull : 0ull);
  }
  return r;
}
__device__ U192 shl(const U192& a, int s) {   // 0 <= s < 192
  U192 r;
  const int q = s >> 6, b = s & 63;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    unsigned long long v = 0;
    if (i - q >= 0) {
      v = a.w[i - q] << b;
      if (b && i - q - 1 >= 0) v |= a.w[i - q - 1] >> (64 - b);
    }
    r.w[i] = v;
  }
  return r;
}
__device__ int cmp(const U192& a, const U192& b) {
  for (int i = 2; i >= 0; i--)
    if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
  return 0;
}
__device__ U192 sub(const U192& a, const U192& b) {   // a >= b
  U192 r;
  unsigned long long borrow = 0;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const unsigned long long d = a.w[i] - b.w[i];
    const unsigned long long nb = (a.w[i] < b.w[i] ? 1ull : 0ull) | (d < borrow ? 1ull : 0ull);
    r.w[i] = d - borrow;
    borrow = nb;
  }
  return r;
}
__device__ U192 add(const U192& a, const U192& b) {
  U192 r;
  unsigned long long carry = 0;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const unsigned long long s = a.w[i] + b.w[i];
    const unsigned long long c1 = s < a.w[i] ? 1ull : 0ull;
    r.w[i] = s + carry;
    carry = c1 | (r.w[i] < s ? 1ull : 0ull);
  }
  return r;
}
__device__ U192 mul_pow5(U192 a, int k) {   // a 5^k, 0 <= k <= 54
  const unsigned long long P27 = 7450580596923828125ull;   // 5^27
  while (k >= 27) { a = mul64(a, P27); k -= 27; }
  unsigned long long t = 1;
  for (int i = 0; i < k; i++) t *= 5ull;
  return mul64(a, t);
}

__constant__ double kPow10[84] = {1e-29, 1e-28, 1e-27, 1e-26, 1e-25, 1e-24, 1e-23, 1e-22, 1e-21, 1e-20, 1e-19, 1e-18, 1e-17, 1e-16, 1e-15, 1e-14, 1e-13, 1e-12, 1e-11, 1e-10, 1e-9, 1e-8, 1e-7, 1e-6, 1e-5, 1e-4, 1e-3, 1e-2, 1e-1, 1e0, 1e1, 1e2, 1e3, 1e4, 1e5, 1e6, 1e7, 1e8, 1e9, 1e10, 1e11, 1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22, 1e23, 1e24, 1e25, 1e26, 1e27, 1e28, 1e29, 1e30, 1e31, 1e32, 1e33, 1e34, 1e35, 1e36, 1e37, 1e38, 1e39, 1e40, 1e41, 1e42, 1e43, 1e44, 1e45, 1e46, 1e47, 1e48, 1e49, 1e50, 1e51, 1e52, 1e53, 1e54};   // 1e-29 .. 1e54

constexpr unsigned long long TEN9 = 1000000000ull, TEN10 = 10000000000ull;

// floor(M 2^E 10^s) and the rounding of its remainder: *half = sign of (2 r - Q)
__device__ unsigned long long scaled_floor(unsigned M, int E, int s, int* half) {
  const int t = E + s;
  U192 P = u192(M), Q = u192(1);
  if (s >= 0) P = mul_pow5(P, s); else Q = mul_pow5(Q, -s);
  if (t >= 0) P = shl(P, t); else Q = shl(Q, -t);
  double est = ldexp((double)M, E) * kPow10[s + 29];
  long long N = (long long)floor(est);
  if (N < 0) N = 0;
  U192 NQ = mul64(Q, (unsigned long long)N);
  for (int i = 0; i < 4 && N > 0 && cmp(NQ, P) > 0; i++) { N--; NQ = sub(NQ, Q); }   // the estimate is within 1
  U192 R = sub(P, NQ);
  for (int i = 0; i < 4 && cmp(R, Q) >= 0; i++) { N++; R = sub(R, Q); }
  *half = cmp(add(R, R), Q);
  return (unsigned long long)N;
}

// printf("%.10g", (double)f) into o (at most 16 characters); returns the count
__device__ int fmt_g10(float f, char* o) {
  const unsigned u = __float_as_uint(f);
  const unsigned a = u & 0x7fffffffu;
  int n = 0;
  if (u >> 31) o[n++] = '-';
  if (a >= 0x7f800000u) {
    if (a == 0x7f800000u) { o[n++] = 'i'; o[n++] = 'n'; o[n++] = 'f'; }
    else { o[n++] = 'n'; o[n++] = 'a'; o[n++] = 'n'; }
    return n;
  }
  if (a == 0u) { o[n++] = '0'; return n; }
  const unsigned ex = a >> 23;
  const unsigned M = ex ? ((a & 0x7fffffu) | 0x800000u) : (a & 0x7fffffu);
  const int E = ex ? (int)ex - 150 : -149;
  int X = (int)floor(log10(ldexp((double)M, E)));
  X = X < -45 ? -45 : X > 38 ? 38 : X;   // floats lie in [1.4e-45, 3.5e38]
  unsigned long long N = 0;
  int half = -1;
  for (int i = 0; i < 4; i++) {   // the exponent whose 10-digit floor lies in [10^9, 10^10): the estimate is within 1
    N = scaled_floor(M, E, 9 - X, &half);
    if (N >= TEN10 && X < 38) X++;
    else if (N < TEN9 && X > -45) X--;
    else break;
  }
  if (half > 0 || (half == 0 && (N & 1ull))) N++;
  if (N == TEN10) { N = TEN9; X++; }
  char d[10];
  for (int i = 9; i >= 0; i--) { d[i] = (char)('0' + (int)(N % 10ull)); N /= 10ull; }
  int last = 9;
  while (last > 0 && d[last] == '0') last--;
  if (X >= -4 && X < 10) {
    if (X >= 0) {
      for (int i = 0; i <= X; i++) o[n++] = d[i];
      if (last > X) { o[n++] = '.'; for (int i = X + 1; i <= last; i++) o[n++] = d[i]; }
    } else {
      o[n++] = '0'; o[n++] = '.';
      for (int i = 0; i < -X - 1; i++) o[n++] = '0';
      for (int i = 0; i <= last; i++) o[n++] = d[i];
    }
  } else {
    o[n++] = d[0];
    if (last > 0) { o[n++] = '.'; for (int i = 1; i <= last; i++) o[n++] = d[i]; }
    o[n++] = 'e';
    o[n++] = X < 0 ? '-' : '+';
    const int ax = X < 0 ? -X : X;   // |X| <= 45 for a float
    o[n++] = (char)('0' + ax / 10); o[n++] = (char)('0' + ax % 10);
  }
  return n;
}

__device__ int fmt_u64(unsigned long long v, char* o) {
  char t[20];
  int k = 0;
  do { t[k++] = (char)('0' + (int)(v % 10ull)); v /= 10ull; } while (v);
  for (int i = 0; i < k; i++) o[i] = t[k - 1 - i];
  return k;
}

// One tree's text ("count\n" and its node lines); writes to o when W.  The traversal is fb_trees_text's: a stack of
// (slot, nid), the right child pushed before the left, at most NODES + 1 nodes visited.
template <bool W>
__device__ unsigned long long tree_text(const uint64_t* T, char* o) {
  unsigned char ss[2 * NODES + 4];
  unsigned long long sn[2 * NODES + 4];
  char buf[48];
  unsigned long long len = 0;
  // node count first (the header line of the tree)
  int sp = 0, cnt = 0;
  ss[sp] = 0; sn[sp] = 1ull; sp++;
  while (sp > 0 && cnt <= NODES) {
    sp--;
    const int x = ss[sp];
    cnt++;
    const uint64_t w = x < NODES ? T[x] : 0ull;   // slots of a valid tree are below NODES
    const int l = (int)((w >> 16) & 255ull), r = (int)((w >> 24) & 255ull);
    if (l) { ss[sp] = (unsigned char)r; sp++; ss[sp] = (unsigned char)l; sp++; }
  }
  int k = fmt_u64((unsigned long long)cnt, buf);
  buf[k++] = '\n';
  if (W) for (int i = 0; i < k; i++) o[len + i] = buf[i];
  len += (unsigned long long)k;
  sp = 0; cnt = 0;
  ss[sp] = 0; sn[sp] = 1ull; sp++;
  while (sp > 0 && cnt <= NODES) {
    sp--;
    const int x = ss[sp];
    const unsigned long long id = sn[sp];
    cnt++;
    const uint64_t w = x < NODES ? T[x] : 0ull;
    const int l = (int)((w >> 16) & 255ull), r = (int)((w >> 24) & 255ull);
    const bool leaf = l == 0;
    k = fmt_u64(id, buf);
    buf[k++] = ' ';
    k += fmt_u64(leaf ? 0ull : (w & 255ull), buf + k);
    buf[k++] = ' ';
    k += fmt_u64(leaf ? 0ull : ((w >> 8) & 255ull), buf + k);
    buf[k++] = ' ';
    k += fmt_g10(leaf ? __uint_as_float((unsigned)(w >> 32)) : 0.0f, buf + k);
    buf[k++] = '\n';
    if (W) for (int i = 0; i < k; i++) o[len + i] = buf[i];
    len += (unsigned long long)k;
    if (l) {
      ss[sp] = (unsigned char)r; sn[sp] = 2ull * id + 1ull; sp++;
      ss[sp] = (unsigned char)l; sn[sp] = 2ull * id; sp++;
    }
  }
  return len;
}

__global__ void __launch_bounds__(128) tree_text_len_kernel(const uint64_t* trees, long long ntrees,
                                                            unsigned long long* len) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ntrees) len[i] = tree_text<false>(trees + i * NODES, nullptr);
  else if (i == ntrees) len[i] = 0ull;
}

__global__ void __launch_bounds__(128) tree_text_write_kernel(const uint64_t* trees, long long ntrees,
                                                              const unsigned long long* off, char* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ntrees) tree_text<true>(trees + i * NODES, out + off[i]);
}

}  // namespace

int trees_text_device(const uint64_t* d_trees, long long ntrees, char** d_out, unsigned long long* total,
                      void* stream_) {
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  unsigned long long* len = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  const long long n1 = ntrees + 1;
  const unsigned grid = (unsigned)((n1 + 127) / 128);
  int rc = -1;
  if (d_out) *d_out = nullptr;
  if (cudaMalloc(&len, sizeof(unsigned long long) * 2 * (size_t)n1) != cudaSuccess) return -1;
  unsigned long long* off = len + n1;
  tree_text_len_kernel<<<grid, 128, 0, stream>>>(d_trees, ntrees, len);
  if (cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, len, off, (int)n1, stream) != cudaSuccess) goto done;
  if (cudaMalloc(&tmp, tmp_bytes) != cudaSuccess) goto done;
  if (cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, len, off, (int)n1, stream) != cudaSuccess) goto done;
  if (cudaMemcpyAsync(total, off + ntrees, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
    goto done;
  if (cudaStreamSynchronize(stream) != cudaSuccess) goto done;
  if (d_out) {
    if (cudaMalloc(d_out, *total > 0 ? *total : 1) != cudaSuccess) { *d_out = nullptr; goto done; }
    tree_text_write_kernel<<<grid, 128, 0, stream>>>(d_trees, ntrees, off, *d_out);
    if (cudaStreamSynchronize(stream) != cudaSuccess) goto done;
  }
  rc = cudaGetLastError() == cudaSuccess ? 0 : -1;
done:
  cudaFree(tmp);
  cudaFree(len);
  if (rc != 0 && d_out && *d_out) { cudaFree(*d_out); *d_out = nullptr; }
  return rc;
}

}  // namespace fb
