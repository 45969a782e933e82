// fb_math.cuh -- deterministic device arithmetic of the sampler.
//
// The heavy functions are out of line (__noinline__): one copy of each in the kernel keeps the control warp's code
// path short.
//
// Every function here is defined only through IEEE-754 operations that round the same way on any conforming
// machine: + - * / sqrt in double, explicit fma(), conversions with round-to-nearest.  Files including it are compiled
// with -fmad=false so that no a*b+c is contracted behind our back.  A CPU restatement of the same definitions
// (oracle/fb_oracle.c) therefore produces bit-identical values, which is what makes whole-chain parity testable.
//
//   philox4x32_10  counter-based generator of Salmon, Moraes, Dror and Shaw, "Parallel random numbers: as easy as
//                  1, 2, 3" (SC11); 10 rounds, Weyl key schedule.
//   fb_log         x = 2^k f, f in (sqrt(1/2), sqrt(2)]; log f = 2 atanh(s), s = (f-1)/(f+1), Taylor series of atanh
//                  to s^23 in Horner form; k ln 2 added in two parts (Cody-Waite).
//   fb_exp         k = floor(x / ln 2 + 1/2), r = x - k ln 2 (two parts), Taylor series of e^r to r^14, times 2^k.
//   fb_normal      Marsaglia's polar method, at most 64 tries.
//   fb_gamma       Marsaglia-Tsang for shape >= 1, at most 32 tries (the method of src/bart_kernel.cpp:73-83).
//   fb_rtnorm      BART's truncated normal (src/bart_kernel.cpp:280-292), loops capped at 64 tries.
#pragma once
#include <cstdint>

namespace fbm {

enum : uint32_t { TAG_PROP = 1, TAG_MH = 2, TAG_MU = 3, TAG_SIG_N = 4, TAG_SIG_U = 5, TAG_Z_N = 6, TAG_Z_E = 7,
                  TAG_PROP2 = 8, TAG_PROP3 = 9 };
constexpr uint32_t INIT_SWEEP = 0xFFFFFFFFu;

struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t seed) {
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  return U4{c0, c1, c2, c3};
}

// uniform on (0,1) from one word / from a 52-bit integer; both exact in double
__device__ __forceinline__ double u32d(uint32_t x) { return ((double)x + 0.5) * 0x1p-32; }
__device__ __forceinline__ double u52d(uint32_t hi, uint32_t lo) {
  const unsigned long long k = ((unsigned long long)hi << 20) | (unsigned long long)(lo >> 12);
  return ((double)k + 0.5) * 0x1p-52;
}

__device__ __forceinline__ double fb_log_inl(double x);
static __device__ __noinline__ double fb_log(double x) { return fb_log_inl(x); }
// the same logarithm, inlined where its latency is on the critical path (the MH likelihoods)
__device__ __forceinline__ double fb_log_inl(double x) {
  if (x != x) return x;
  if (x <= 0.0) return x == 0.0 ? -__longlong_as_double(0x7FF0000000000000LL) : __longlong_as_double(0x7FF8000000000000LL);
  if (__double_as_longlong(x) == 0x7FF0000000000000LL) return x;
  int k = 0;
  unsigned long long b = (unsigned long long)__double_as_longlong(x);
  if ((b >> 52) == 0) { x = x * 0x1p54; b = (unsigned long long)__double_as_longlong(x); k = -54; }
  k += (int)(b >> 52) - 1023;
  double f = __longlong_as_double((long long)((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull));
  if (f > 0x1.6a09e667f3bcdp+0) { f = f * 0.5; k += 1; }
  const double s = (f - 1.0) / (f + 1.0);
  const double s2 = s * s;
  double p = 0x1.642c8590b2164p-5;
  p = fma(p, s2, 0x1.8618618618618p-5);
  p = fma(p, s2, 0x1.af286bca1af28p-5);
  p = fma(p, s2, 0x1.e1e1e1e1e1e1ep-5);
  p = fma(p, s2, 0x1.1111111111111p-4);
  p = fma(p, s2, 0x1.3b13b13b13b14p-4);
  p = fma(p, s2, 0x1.745d1745d1746p-4);
  p = fma(p, s2, 0x1.c71c71c71c71cp-4);
  p = fma(p, s2, 0x1.2492492492492p-3);
  p = fma(p, s2, 0x1.999999999999ap-3);
  p = fma(p, s2, 0x1.5555555555555p-2);
  const double s2s = 2.0 * s;
  const double lf = fma(s2s, s2 * p, s2s);
  const double kd = (double)k;
  return fma(kd, 0x1.62e42fee00000p-1, fma(kd, 0x1.a39ef35793c76p-33, lf));
}

static __device__ __noinline__ double fb_exp(double x) {
  if (x != x) return x;
  if (x > 709.78) return __longlong_as_double(0x7FF0000000000000LL);
  if (x < -745.2) return 0.0;
  const double kd = floor(x * 0x1.71547652b82fep+0 + 0.5);
  int k = (int)kd;
  double r = fma(-kd, 0x1.62e42fee00000p-1, x);
  r = fma(-kd, 0x1.a39ef35793c76p-33, r);
  double p = 0x1.93974a8c07c9dp-37;
  p = fma(p, r, 0x1.6124613a86d09p-33);
  p = fma(p, r, 0x1.1eed8eff8d898p-29);
  p = fma(p, r, 0x1.ae64567f544e4p-26);
  p = fma(p, r, 0x1.27e4fb7789f5cp-22);
  p = fma(p, r, 0x1.71de3a556c734p-19);
  p = fma(p, r, 0x1.a01a01a01a01ap-16);
  p = fma(p, r, 0x1.a01a01a01a01ap-13);
  p = fma(p, r, 0x1.6c16c16c16c17p-10);
  p = fma(p, r, 0x1.1111111111111p-7);
  p = fma(p, r, 0x1.5555555555555p-5);
  p = fma(p, r, 0x1.5555555555555p-3);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  if (k > 1023) { p = p * 2.0; k -= 1; }
  if (k < -1000) { p = p * 0x1p-200; k += 200; }
  return p * __longlong_as_double((long long)((unsigned long long)(k + 1023) << 52));
}

static __device__ __noinline__ double fb_normal(uint64_t seed, uint32_t c0base, uint32_t c1, uint32_t c2, uint32_t tag) {
  for (uint32_t t = 0; t < 64; t++) {
    const U4 x = philox(c0base + t, c1, c2, tag, seed);
    const double a = 2.0 * u52d(x.x, x.y) - 1.0, b = 2.0 * u52d(x.z, x.w) - 1.0;
    const double s = a * a + b * b;
    if (s < 1.0 && s > 0.0) return a * sqrt(-2.0 * fb_log(s) / s);
  }
  return 0.0;
}

static __device__ __noinline__ double fb_gamma(uint64_t seed, uint32_t it, double a) {
  const double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
  for (uint32_t tt = 0; tt < 32; tt++) {
    const double x = fb_normal(seed, tt << 8, 0u, it, TAG_SIG_N);
    double v = 1.0 + c * x;
    if (v <= 0.0) continue;
    v = v * v * v;
    const U4 w = philox(tt, 0u, it, TAG_SIG_U, seed);
    const double u = u52d(w.x, w.y);
    if (fb_log(u) < 0.5 * x * x + d - d * v + d * fb_log(v)) return d * v;
  }
  return d;
}

// N(mean, 1) truncated to > tau; *capped is incremented when a loop gives up (then tau is returned).
static __device__ __noinline__ double fb_rtnorm(uint64_t seed, uint32_t row, uint32_t it, double mean, double tau, int* capped) {
  tau = tau - mean;
  if (tau <= 0.0) {
    for (uint32_t tt = 0; tt < 64; tt++) {
      const double z = fb_normal(seed, tt << 8, row, it, TAG_Z_N);
      if (!(z < tau)) return z + mean;
    }
  } else {
    const double lambda = 0.5 * (tau + sqrt(tau * tau + 4.0));
    for (uint32_t tt = 0; tt < 64; tt++) {
      const U4 x = philox(tt, row, it, TAG_Z_E, seed);
      const double u1 = u52d(x.x, x.y), u2 = u52d(x.z, x.w);
      const double z = -fb_log(u1) / lambda + tau;
      if (!(u2 > fb_exp(-0.5 * (z - lambda) * (z - lambda)))) return z + mean;
    }
  }
  (*capped)++;
  return tau + mean;
}

}  // namespace fbm
