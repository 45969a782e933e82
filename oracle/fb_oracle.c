/*
 * fb_oracle.c -- CPU oracle for fastbart_b200.  TEST INFRASTRUCTURE ONLY (see fb_oracle.h): the checker that tests,
 * smoke() and bench.py's cpu_baseline leg run on the CPU.  Never part of the product.
 *
 * Build with IEEE semantics (no -ffast-math, -ffp-contract=off): the DEV mode must agree bit for bit with the CUDA
 * kernels, and the REF mode with bart_fit_cpu.
 */
#include "fb_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define BIT(m, i) (((m) >> (i)) & 1ull)

/* ================================================================ DEV arithmetic primitives */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC11). */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n1 = (uint32_t)p1, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1, n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline void philox_seed(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t x[4]) {
  uint32_t ctr[4] = {c0, c1, c2, c3}, key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  orc_philox(ctr, key, x);
}
/* uniform on (0,1) from one 32-bit word, exact in double */
static inline double u32d(uint32_t x) { return ((double)x + 0.5) * 0x1p-32; }
/* uniform on (0,1) from two words: a 52-bit integer plus one half, scaled; exact in double */
static inline double u52d(uint32_t hi, uint32_t lo) {
  uint64_t k = ((uint64_t)hi << 20) | (uint64_t)(lo >> 12);
  return ((double)k + 0.5) * 0x1p-52;
}

static inline uint64_t dbits(double x) { uint64_t b; memcpy(&b, &x, 8); return b; }
static inline double bitsd(uint64_t b) { double x; memcpy(&x, &b, 8); return x; }

#define LN2_HI 0x1.62e42fee00000p-1   /* ln 2 rounded to 32 significant bits (k * LN2_HI exact for |k| < 2^21) */
#define LN2_LO 0x1.a39ef35793c76p-33  /* ln 2 - LN2_HI */
#define INV_LN2 0x1.71547652b82fep+0
#define SQRT2 0x1.6a09e667f3bcdp+0

/* Natural log: x = 2^k f with f in (sqrt(1/2), sqrt(2)], log f = 2 atanh(s), s = (f-1)/(f+1), atanh series to s^23. */
double orc_log(double x) {
  if (x != x) return x;
  if (x <= 0.0) return x == 0.0 ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  int k = 0;
  uint64_t b = dbits(x);
  if ((b >> 52) == 0) { x = x * 0x1p54; b = dbits(x); k = -54; }
  k += (int)(b >> 52) - 1023;
  double f = bitsd((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
  if (f > SQRT2) { f = f * 0.5; k += 1; }
  double s = (f - 1.0) / (f + 1.0);
  double s2 = s * s;
  double p = 0x1.642c8590b2164p-5;          /* 1/23 */
  p = fma(p, s2, 0x1.8618618618618p-5);     /* 1/21 */
  p = fma(p, s2, 0x1.af286bca1af28p-5);     /* 1/19 */
  p = fma(p, s2, 0x1.e1e1e1e1e1e1ep-5);     /* 1/17 */
  p = fma(p, s2, 0x1.1111111111111p-4);     /* 1/15 */
  p = fma(p, s2, 0x1.3b13b13b13b14p-4);     /* 1/13 */
  p = fma(p, s2, 0x1.745d1745d1746p-4);     /* 1/11 */
  p = fma(p, s2, 0x1.c71c71c71c71cp-4);     /* 1/9 */
  p = fma(p, s2, 0x1.2492492492492p-3);     /* 1/7 */
  p = fma(p, s2, 0x1.999999999999ap-3);     /* 1/5 */
  p = fma(p, s2, 0x1.5555555555555p-2);     /* 1/3 */
  double s2s = 2.0 * s;
  double lf = fma(s2s, s2 * p, s2s);
  double kd = (double)k;
  return fma(kd, LN2_HI, fma(kd, LN2_LO, lf));
}

/* exp: k = nearest integer to x/ln2, r = x - k ln2 (two-part ln2), e^r by its Taylor series to r^14, scale by 2^k. */
double orc_exp(double x) {
  if (x != x) return x;
  if (x > 709.78) return INFINITY;
  if (x < -745.2) return 0.0;
  double kd = floor(x * INV_LN2 + 0.5);
  int k = (int)kd;
  double r = fma(-kd, LN2_HI, x);
  r = fma(-kd, LN2_LO, r);
  double p = 0x1.93974a8c07c9dp-37;         /* 1/14! */
  p = fma(p, r, 0x1.6124613a86d09p-33);     /* 1/13! */
  p = fma(p, r, 0x1.1eed8eff8d898p-29);     /* 1/12! */
  p = fma(p, r, 0x1.ae64567f544e4p-26);     /* 1/11! */
  p = fma(p, r, 0x1.27e4fb7789f5cp-22);     /* 1/10! */
  p = fma(p, r, 0x1.71de3a556c734p-19);     /* 1/9! */
  p = fma(p, r, 0x1.a01a01a01a01ap-16);     /* 1/8! */
  p = fma(p, r, 0x1.a01a01a01a01ap-13);     /* 1/7! */
  p = fma(p, r, 0x1.6c16c16c16c17p-10);     /* 1/6! */
  p = fma(p, r, 0x1.1111111111111p-7);      /* 1/5! */
  p = fma(p, r, 0x1.5555555555555p-5);      /* 1/4! */
  p = fma(p, r, 0x1.5555555555555p-3);      /* 1/3! */
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  if (k > 1023) { p = p * 2.0; k -= 1; }
  if (k < -1000) { p = p * 0x1p-200; k += 200; }
  return p * bitsd((uint64_t)(k + 1023) << 52);
}

/* Standard normal, Marsaglia polar method; try t uses Philox counter (c0base + t, c1, c2, tag); at most 64 tries. */
double orc_normal(uint64_t seed, uint32_t c0base, uint32_t c1, uint32_t c2, uint32_t tag) {
  for (uint32_t t = 0; t < 64; t++) {
    uint32_t x[4];
    philox_seed(seed, c0base + t, c1, c2, tag, x);
    double a = 2.0 * u52d(x[0], x[1]) - 1.0, b = 2.0 * u52d(x[2], x[3]) - 1.0;
    double s = a * a + b * b;
    if (s < 1.0 && s > 0.0) return a * sqrt(-2.0 * orc_log(s) / s);
  }
  return 0.0;
}

/* Gamma(a, 1), a >= 1: Marsaglia-Tsang with at most 32 tries (the method of bart_kernel.cpp:73-83). */
double orc_gamma(uint64_t seed, uint32_t it, double a) {
  double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
  for (uint32_t tt = 0; tt < 32; tt++) {
    double x = orc_normal(seed, tt << 8, 0u, it, ORC_TAG_SIG_N);
    double v = 1.0 + c * x;
    if (v <= 0.0) continue;
    v = v * v * v;
    uint32_t w[4];
    philox_seed(seed, tt, 0u, it, ORC_TAG_SIG_U, w);
    double u = u52d(w[0], w[1]);
    if (orc_log(u) < 0.5 * x * x + d - d * v + d * orc_log(v)) return d * v;
  }
  return d;
}

/* N(mean, 1) truncated to > tau: BART's rtnorm (bart_kernel.cpp:280-292) with capped loops (64 tries). */
double orc_rtnorm(uint64_t seed, uint32_t row, uint32_t it, double mean, double tau, int* capped) {
  tau = tau - mean;
  if (tau <= 0.0) {
    for (uint32_t tt = 0; tt < 64; tt++) {
      double z = orc_normal(seed, tt << 8, row, it, ORC_TAG_Z_N);
      if (!(z < tau)) return z + mean;
    }
  } else {
    double lambda = 0.5 * (tau + sqrt(tau * tau + 4.0));
    for (uint32_t tt = 0; tt < 64; tt++) {
      uint32_t x[4];
      philox_seed(seed, tt, row, it, ORC_TAG_Z_E, x);
      double u1 = u52d(x[0], x[1]), u2 = u52d(x[2], x[3]);
      double z = -orc_log(u1) / lambda + tau;
      if (!(u2 > orc_exp(-0.5 * (z - lambda) * (z - lambda)))) return z + mean;
    }
  }
  if (capped) (*capped)++;
  return tau + mean;
}

/* The latent redraw of every row of a probit chain at one sweep (bart_kernel.cpp:543-547): z[i] = -rtnorm(-f, offset)
   for ybin 0, rtnorm(f, -offset) for ybin 1, with the DEV counters (seed, row, sweep). Returns the capped draws. */
int orc_probit_latent(uint64_t seed, uint32_t it, double offset, const double* fit, const int* ybin, long long n,
                      double* z) {
  int caps = 0;
  for (long long i = 0; i < n; i++)
    z[i] = ybin[i] == 0 ? -orc_rtnorm(seed, (uint32_t)i, it, -fit[i], offset, &caps)
                        : orc_rtnorm(seed, (uint32_t)i, it, fit[i], -offset, &caps);
  return caps;
}

/* ================================================================ tree helpers (bart_kernel.cpp:85-109, 220-278) */
typedef struct {
  uint8_t l[ORC_NODES], r[ORC_NODES], par[ORC_NODES], v[ORC_NODES], c[ORC_NODES], d[ORC_NODES], ngv[ORC_NODES];
  float th[ORC_NODES];
  uint64_t used, leaf;
} otree;

static int popc64(uint64_t m) { int c = 0; for (int i = 0; i < ORC_NODES; i++) c += (int)BIT(m, i); return c; }
static int select_kth(uint64_t m, int k) {   /* index of the k-th set bit; 0 if none (bart_kernel.cpp:94-101) */
  int c = 0, r = 0;
  for (int i = 0; i < ORC_NODES; i++) if (BIT(m, i)) { if (c == k) r = i; c++; }
  return r;
}
static int first_free(uint64_t used, int skip) {   /* lowest unused slot >= 1 other than skip (bart_kernel.cpp:102-109) */
  int r = -1;
  for (int i = ORC_NODES - 1; i >= 1; i--) if (!BIT(used, i) && i != skip) r = i;
  return r;
}
static void node_range(const otree* t, int x, int v, int nc, int* L, int* U) {   /* bart_kernel.cpp:238-251 */
  *L = 0; *U = nc - 1;
  int node = x;
  for (int s = 0; s < ORC_MAXDEPTH; s++) {
    if (node == 0) break;
    int pa = t->par[node];
    if ((int)t->v[pa] == v) {
      if ((int)t->l[pa] == node) { if ((int)t->c[pa] - 1 < *U) *U = (int)t->c[pa] - 1; }
      else { if ((int)t->c[pa] + 1 > *L) *L = (int)t->c[pa] + 1; }
    }
    node = pa;
  }
}
static int count_goodvars(const otree* t, int x, const int* nc, int p) {   /* bart_kernel.cpp:253-276 */
  int L[ORC_PMAX], U[ORC_PMAX];
  for (int v = 0; v < ORC_PMAX; v++) { L[v] = 0; U[v] = (v < p ? nc[v] : 0) - 1; }
  int node = x;
  for (int s = 0; s < ORC_MAXDEPTH; s++) {
    if (node == 0) break;
    int pa = t->par[node], v = t->v[pa], c = t->c[pa];
    if ((int)t->l[pa] == node) { if (c - 1 < U[v]) U[v] = c - 1; }
    else { if (c + 1 > L[v]) L[v] = c + 1; }
    node = pa;
  }
  int g = 0;
  for (int v = 0; v < ORC_PMAX; v++) if (v < p && U[v] >= L[v]) g++;
  return g;
}
static void tree_root(otree* t, int root_ngv) {
  memset(t, 0, sizeof *t);
  t->ngv[0] = (uint8_t)root_ngv; t->used = 1; t->leaf = 1;
}

/* Proposal (bart_kernel.cpp:413-464).  `u` yields the uniforms in order: birth?, node, variable, cutpoint. */
typedef double (*unif_fn)(void* ctx);
typedef struct { int mode, nx, v, c; double pr, corr; } oprop;   /* corr: the learned variable's ratio factor (1: none) */
static oprop propose(const otree* t, const double* PG, const int* nc, int p, unif_fn u, void* uctx, int guard_death) {
  const double pb = 0.5;
  uint64_t goodm = 0, nogm = 0;
  for (int s = 0; s < ORC_NODES; s++) {
    int isleaf = (int)BIT(t->leaf, s), isused = (int)BIT(t->used, s);
    if (isused && isleaf && t->ngv[s] > 0) goodm |= 1ull << s;
    if (isused && !isleaf && BIT(t->leaf, (int)t->l[s]) && BIT(t->leaf, (int)t->r[s])) nogm |= 1ull << s;
  }
  int ngood = popc64(goodm), nnogs = popc64(nogm);
  int single = (t->used == 1ull);
  double PBx = ngood == 0 ? 0 : (single ? 1 : pb);
  oprop o = {0, 0, 0, 0, 0.0, 1.0};
  int birth = u(uctx) < PBx;
  if (birth) {
    int nx = select_kth(goodm, (int)(u(uctx) * ngood));
    int v = (int)(u(uctx) * p); if (v >= p) v = p - 1;
    int bL, bU;
    node_range(t, nx, v, nc[v], &bL, &bU);
    if (bU >= bL && (int)t->d[nx] + 1 < ORC_MAXDEPTH) {
      int c = bL + (int)(u(uctx) * (bU - bL + 1)); if (c > bU) c = bU;
      int dnx = t->d[nx];
      double PGnx = PG[dnx], PGly, PGry;
      if (t->ngv[nx] > 1) { PGly = PGry = PG[dnx + 1]; }
      else { PGly = (c - 1 < bL) ? 0 : PG[dnx + 1]; PGry = (bU < c + 1) ? 0 : PG[dnx + 1]; }
      double PDy = (ngood > 1) ? 1 - pb : ((PGry == 0 && PGly == 0) ? 1 : 1 - pb);
      double Pnogy;
      if (nx == 0) Pnogy = 1;
      else {
        int pa = t->par[nx];
        int panog = BIT(t->leaf, (int)t->l[pa]) && BIT(t->leaf, (int)t->r[pa]);
        Pnogy = panog ? (double)1 / nnogs : (double)1 / (nnogs + 1);
      }
      double Pbotx = (double)1 / ngood;
      o.pr = (PGnx * (1 - PGly) * (1 - PGry) * PDy * Pnogy) / ((1 - PGnx) * Pbotx * PBx);
      o.mode = 1; o.nx = nx; o.v = v; o.c = c;
    }
  } else if (!guard_death || nnogs > 0) {
    int nx = select_kth(nogm, (int)(u(uctx) * nnogs));
    int dny = t->d[nx], l = t->l[nx], r = t->r[nx];
    double PGny = PG[dny];
    double PGlx = t->ngv[l] > 0 ? PG[dny + 1] : 0, PGrx = t->ngv[r] > 0 ? PG[dny + 1] : 0;
    double PBy = (nx == 0) ? 1 : pb;
    int ng2 = ngood - (t->ngv[l] > 0) - (t->ngv[r] > 0) + 1;
    double Pboty = (double)1 / ng2, PDx = 1 - PBx, Pnogx = (double)1 / nnogs;
    o.pr = ((1 - PGny) * PBy * Pboty) / (PGny * (1 - PGlx) * (1 - PGrx) * PDx * Pnogx);
    o.mode = 2; o.nx = nx;
  }
  return o;
}

/* ================================================================ learned split-variable proposal (DEV mode) */
static float bf16f(uint16_t h) { uint32_t u = (uint32_t)h << 16; float f; memcpy(&f, &u, 4); return f; }

/* Features of leaf-to-be-split node nx of tree t (depends only on the tree and the node's row count):
 *   x[0] depth / 8;  x[1] floor(log2(cnt + 1)) / 16;
 *   x[2 + v]  min(number of internal nodes splitting on v, 8) / 8 (internal nodes other than `exclude`);
 *   x[34 + v] cut range of v at nx, (U - L + 1) / numcut[v];  x[66 + v] L / numcut[v]  (0 when empty).
 * Returns the mask of variables whose range at nx is non-empty. */
static uint32_t orc_features(const otree* t, int nx, int cnt, int exclude, const int* nc, int p, float* x) {
  for (int k = 0; k < ORC_MLP_IN; k++) x[k] = 0.0f;
  x[0] = (float)t->d[nx] / 8.0f;
  int bl = 0;
  for (unsigned c = (unsigned)cnt + 1u; c > 1u; c >>= 1) bl++;
  x[1] = (float)bl / 16.0f;
  int use[ORC_PMAX];
  for (int v = 0; v < ORC_PMAX; v++) use[v] = 0;
  for (int s = 0; s < ORC_NODES; s++)
    if (BIT(t->used, s) && !BIT(t->leaf, s) && s != exclude) use[t->v[s]]++;
  uint32_t valid = 0;
  for (int v = 0; v < ORC_PMAX; v++) {
    x[2 + v] = (float)(use[v] < 8 ? use[v] : 8) / 8.0f;
    if (v < p && nc[v] > 0) {
      int L, U;
      node_range(t, nx, v, nc[v], &L, &U);
      if (U >= L) {
        x[34 + v] = (float)(U - L + 1) / (float)nc[v];
        x[66 + v] = (float)L / (float)nc[v];
        valid |= 1u << v;
      }
    }
  }
  return valid;
}

void orc_mlp_logits(const orc_model* M, const float* x, float* z) {
  float h1[ORC_MLP_H], h2[ORC_MLP_H];
  for (int h = 0; h < ORC_MLP_H; h++) {
    float a = M->b1[h];
    for (int k = 0; k < ORC_MLP_IN; k++) a = a + bf16f(M->w1[h * ORC_MLP_IN + k]) * x[k];
    h1[h] = a > 0.0f ? a : 0.0f;
  }
  for (int h = 0; h < ORC_MLP_H; h++) {
    float a = M->b2[h];
    for (int k = 0; k < ORC_MLP_H; k++) a = a + bf16f(M->w2[h * ORC_MLP_H + k]) * h1[k];
    h2[h] = a > 0.0f ? a : 0.0f;
  }
  for (int o = 0; o < ORC_MLP_OUT; o++) {
    float a = M->b3[o];
    for (int k = 0; k < ORC_MLP_H; k++) a = a + bf16f(M->w3[o * ORC_MLP_H + k]) * h2[k];
    z[o] = a;
  }
}

void orc_mlp_probs(const float* z, uint32_t valid, double* q) {
  double zmax = 0.0;
  int any = 0;
  for (int v = 0; v < ORC_MLP_OUT; v++)
    if ((valid >> v) & 1u) { if (!any || (double)z[v] > zmax) zmax = (double)z[v]; any = 1; }
  double S = 0.0;
  for (int v = 0; v < ORC_MLP_OUT; v++) { q[v] = ((valid >> v) & 1u) ? orc_exp((double)z[v] - zmax) : 0.0; S = S + q[v]; }
  for (int v = 0; v < ORC_MLP_OUT; v++) q[v] = S > 0.0 ? q[v] / S : 0.0;
}

/* probability that the mixture proposes valid variable v: mix * q[v] + (1 - mix) / p */
static double mix_prob(const orc_model* M, const double* q, int v, int p) {
  return M->mix * q[v] + (1.0 - M->mix) * (1.0 / (double)p);
}

static int count_rows(const uint8_t* lf, int n, int a, int b) {
  int c = 0;
  for (int i = 0; i < n; i++) c += (lf[i] == a || lf[i] == b);
  return c;
}

/* Proposal with the learned model (mirrors the device): BART's proposal (propose()) with the birth variable drawn
 * from the mixture and the proposal-ratio correction folded into pr.  feat/valid/vout receive the birth node's
 * features (for training examples). */
static oprop propose_model(const otree* t, const double* PG, const int* nc, int p, const double* u4, const double* u2,
                           const orc_model* M, const uint8_t* lf, int n, float* feat, uint32_t* valid_out) {
  const double pb = 0.5;
  uint64_t goodm = 0, nogm = 0;
  for (int s = 0; s < ORC_NODES; s++) {
    int isleaf = (int)BIT(t->leaf, s), isused = (int)BIT(t->used, s);
    if (isused && isleaf && t->ngv[s] > 0) goodm |= 1ull << s;
    if (isused && !isleaf && BIT(t->leaf, (int)t->l[s]) && BIT(t->leaf, (int)t->r[s])) nogm |= 1ull << s;
  }
  int ngood = popc64(goodm), nnogs = popc64(nogm);
  int single = (t->used == 1ull);
  double PBx = ngood == 0 ? 0 : (single ? 1 : pb);
  oprop o = {0, 0, 0, 0, 0.0, 1.0};
  *valid_out = 0;
  if (u4[0] < PBx) {
    int nx = select_kth(goodm, (int)(u4[1] * ngood));
    float z[ORC_MLP_OUT];
    double q[ORC_MLP_OUT];
    uint32_t valid = orc_features(t, nx, count_rows(lf, n, nx, nx), -1, nc, p, feat);
    *valid_out = valid;
    orc_mlp_logits(M, feat, z);
    orc_mlp_probs(z, valid, q);
    int v;
    if (u2[0] < M->mix && valid) {
      double c = 0.0;
      v = -1;
      int last = 0;
      for (int k = 0; k < ORC_MLP_OUT; k++)
        if ((valid >> k) & 1u) { c = c + q[k]; last = k; if (v < 0 && u2[1] < c) v = k; }
      if (v < 0) v = last;
    } else {
      v = (int)(u4[2] * p); if (v >= p) v = p - 1;
    }
    int bL, bU;
    node_range(t, nx, v, nc[v], &bL, &bU);
    if (bU >= bL && (int)t->d[nx] + 1 < ORC_MAXDEPTH) {
      int c = bL + (int)(u4[3] * (bU - bL + 1)); if (c > bU) c = bU;
      int dnx = t->d[nx];
      double PGnx = PG[dnx], PGly, PGry;
      if (t->ngv[nx] > 1) { PGly = PGry = PG[dnx + 1]; }
      else { PGly = (c - 1 < bL) ? 0 : PG[dnx + 1]; PGry = (bU < c + 1) ? 0 : PG[dnx + 1]; }
      double PDy = (ngood > 1) ? 1 - pb : ((PGry == 0 && PGly == 0) ? 1 : 1 - pb);
      double Pnogy;
      if (nx == 0) Pnogy = 1;
      else {
        int pa = t->par[nx];
        int panog = BIT(t->leaf, (int)t->l[pa]) && BIT(t->leaf, (int)t->r[pa]);
        Pnogy = panog ? (double)1 / nnogs : (double)1 / (nnogs + 1);
      }
      double Pbotx = (double)1 / ngood;
      o.pr = (PGnx * (1 - PGly) * (1 - PGry) * PDy * Pnogy) / ((1 - PGnx) * Pbotx * PBx);
      o.corr = (1.0 / (double)p) / mix_prob(M, q, v, p);
      o.pr = o.pr * o.corr;
      o.mode = 1; o.nx = nx; o.v = v; o.c = c;
    }
  } else if (nnogs > 0) {
    int nx = select_kth(nogm, (int)(u4[1] * nnogs));
    int dny = t->d[nx], l = t->l[nx], r = t->r[nx];
    double PGny = PG[dny];
    double PGlx = t->ngv[l] > 0 ? PG[dny + 1] : 0, PGrx = t->ngv[r] > 0 ? PG[dny + 1] : 0;
    double PBy = (nx == 0) ? 1 : pb;
    int ng2 = ngood - (t->ngv[l] > 0) - (t->ngv[r] > 0) + 1;
    double Pboty = (double)1 / ng2, PDx = 1 - PBx, Pnogx = (double)1 / nnogs;
    o.pr = ((1 - PGny) * PBy * Pboty) / (PGny * (1 - PGlx) * (1 - PGrx) * PDx * Pnogx);
    /* reverse move: the birth of nx's split in the tree without it */
    float fx[ORC_MLP_IN], z[ORC_MLP_OUT];
    double q[ORC_MLP_OUT];
    uint32_t valid = orc_features(t, nx, count_rows(lf, n, l, r), nx, nc, p, fx);
    orc_mlp_logits(M, fx, z);
    orc_mlp_probs(z, valid, q);
    o.corr = mix_prob(M, q, (int)t->v[nx], p) * (double)p;
    o.pr = o.pr * o.corr;
    o.mode = 2; o.nx = nx;
  }
  return o;
}

/* ================================================================ learned cutpoint proposal (DEV mode) */
void orc_cut_features(int depth, int cnt, int64_t S0, int64_t S1, int64_t Q, int fx_shift, int rss_shift,
                      double sigma, int L, int U, int nc, int uses, int v, float* x) {
  for (int k = 0; k < ORC_CUT_IN; k++) x[k] = 0.0f;
  x[0] = (float)depth / 8.0f;
  int bl = 0;
  for (unsigned c = (unsigned)cnt + 1u; c > 1u; c >>= 1) bl++;
  x[1] = (float)bl / 16.0f;
  double mean = 0.0, sd = 0.0;
  if (S0 > 0) {
    const double w = (double)S0 * ldexp(1.0, -fx_shift);
    mean = (double)S1 / (double)S0;
    const double msq = ((double)Q * ldexp(1.0, -rss_shift)) / w;
    const double var = msq - mean * mean;
    sd = var > 0.0 ? sqrt(var) : 0.0;
  }
  double fm = mean / sigma;
  fm = fm < -4.0 ? -4.0 : (fm > 4.0 ? 4.0 : fm);
  double fs = sd / sigma;
  fs = fs > 4.0 ? 4.0 : fs;
  x[2] = (float)(fm * 0.25);
  x[3] = (float)(fs * 0.25);
  x[4] = (float)(U - L + 1) / (float)nc;
  x[5] = (float)L / (float)nc;
  x[6] = (float)(uses < 8 ? uses : 8) / 8.0f;
  if (v >= 0 && v < 32) x[8 + v] = 1.0f;
}

void orc_cut_logits(const orc_cut_model* M, const float* x, int L, int U, float* z) {
  float h1[ORC_CUT_H], h2[ORC_CUT_H], e[ORC_CUT_E];
  for (int h = 0; h < ORC_CUT_H; h++) {
    float a = M->b1[h];
    for (int k = 0; k < ORC_CUT_IN; k++) a = a + bf16f(M->w1[h * ORC_CUT_IN + k]) * x[k];
    h1[h] = a > 0.0f ? a : 0.0f;
  }
  for (int h = 0; h < ORC_CUT_H; h++) {
    float a = M->b2[h];
    for (int k = 0; k < ORC_CUT_H; k++) a = a + bf16f(M->w2[h * ORC_CUT_H + k]) * h1[k];
    h2[h] = a > 0.0f ? a : 0.0f;
  }
  for (int k = 0; k < ORC_CUT_E; k++) {
    float a = M->b3[k];
    for (int f = 0; f < ORC_CUT_H; f++) a = a + bf16f(M->w3[k * ORC_CUT_H + f]) * h2[f];
    e[k] = a;
  }
  for (int c = L; c <= U; c++) {
    float a = M->be[c];
    for (int k = 0; k < ORC_CUT_E; k++) a = a + bf16f(M->emb[c * ORC_CUT_E + k]) * e[k];
    z[c] = a;
  }
}

double orc_cut_softmax(const float* z, int L, int U, double* ex) {
  double zmax = (double)z[L];
  for (int c = L + 1; c <= U; c++)
    if ((double)z[c] > zmax) zmax = (double)z[c];
  for (int c = L; c <= U; c++) ex[c] = orc_exp((double)z[c] - zmax);
  double S = 0.0;
  for (int b0 = L; b0 <= U; b0 += 8) {
    double bs = 0.0;
    for (int c = b0; c < b0 + 8 && c <= U; c++) bs = bs + ex[c];
    S = S + bs;
  }
  return S;
}

/* Draws the cut of a birth from the mixture (mix: the model's softmax over [L, U], else uniform on [L, U]); *q_out
 * receives the mixture's probability of the drawn cut. */
static int cut_draw(const double* ex, double S, int L, int U, double umix, double uc, double mix, double* q_out) {
  const int range = U - L + 1;
  int c = U;
  if (umix < mix) {
    const double target = uc * S;
    double P = 0.0;
    int found = 0;
    for (int b0 = L; b0 <= U && !found; b0 += 8) {
      double bs = 0.0;
      for (int k = b0; k < b0 + 8 && k <= U; k++) bs = bs + ex[k];
      const double P1 = P + bs;
      if (P1 > target) {
        double run = P;
        c = b0 + 7 < U ? b0 + 7 : U;
        for (int k = b0; k < b0 + 8 && k <= U; k++) {
          run = run + ex[k];
          if (run > target) { c = k; break; }
        }
        found = 1;
      }
      P = P1;
    }
  } else {
    c = L + (int)(uc * range);
    if (c > U) c = U;
  }
  *q_out = mix * (ex[c] / S) + (1.0 - mix) * (1.0 / (double)range);
  return c;
}

/* the mixture's probability of cut c of [L, U] */
static double cut_prob(const double* ex, double S, int L, int U, int c, double mix) {
  return mix * (ex[c] / S) + (1.0 - mix) * (1.0 / (double)(U - L + 1));
}

static int uses_of(const otree* t, int v, int exclude) {
  int u = 0;
  for (int s = 0; s < ORC_NODES; s++)
    if (BIT(t->used, s) && !BIT(t->leaf, s) && s != exclude && (int)t->v[s] == v) u++;
  return u;
}

/* BART's birth ratio of propose() (bart_kernel.cpp:441-451) at node nx for cut c of range [bL, bU] */
static double birth_pr_at(const otree* t, const double* PG, int nx, int c, int bL, int bU) {
  const double pb = 0.5;
  uint64_t goodm = 0, nogm = 0;
  for (int s = 0; s < ORC_NODES; s++) {
    int isleaf = (int)BIT(t->leaf, s), isused = (int)BIT(t->used, s);
    if (isused && isleaf && t->ngv[s] > 0) goodm |= 1ull << s;
    if (isused && !isleaf && BIT(t->leaf, (int)t->l[s]) && BIT(t->leaf, (int)t->r[s])) nogm |= 1ull << s;
  }
  int ngood = popc64(goodm), nnogs = popc64(nogm);
  double PBx = ngood == 0 ? 0 : (t->used == 1ull ? 1 : pb);
  int dnx = t->d[nx];
  double PGnx = PG[dnx], PGly, PGry;
  if (t->ngv[nx] > 1) { PGly = PGry = PG[dnx + 1]; }
  else { PGly = (c - 1 < bL) ? 0 : PG[dnx + 1]; PGry = (bU < c + 1) ? 0 : PG[dnx + 1]; }
  double PDy = (ngood > 1) ? 1 - pb : ((PGry == 0 && PGly == 0) ? 1 : 1 - pb);
  double Pnogy;
  if (nx == 0) Pnogy = 1;
  else {
    int pa = t->par[nx];
    int panog = BIT(t->leaf, (int)t->l[pa]) && BIT(t->leaf, (int)t->r[pa]);
    Pnogy = panog ? (double)1 / nnogs : (double)1 / (nnogs + 1);
  }
  double Pbotx = (double)1 / ngood;
  return (PGnx * (1 - PGly) * (1 - PGry) * PDy * Pnogy) / ((1 - PGnx) * Pbotx * PBx);
}

double orc_cut_loss_grad(const orc_cut_model* M, const float* X, const int* cy, const int* lo, const int* hi, int B,
                         double* gw1, double* gb1, double* gw2, double* gb2, double* gw3, double* gb3, double* gemb,
                         double* gbe) {
  const int I = ORC_CUT_IN, H = ORC_CUT_H, E = ORC_CUT_E, NB = ORC_CUT_BINS;
  memset(gw1, 0, sizeof(double) * H * I); memset(gb1, 0, sizeof(double) * H);
  memset(gw2, 0, sizeof(double) * H * H); memset(gb2, 0, sizeof(double) * H);
  memset(gw3, 0, sizeof(double) * E * H); memset(gb3, 0, sizeof(double) * E);
  memset(gemb, 0, sizeof(double) * NB * E); memset(gbe, 0, sizeof(double) * NB);
  double loss = 0.0;
  for (int b = 0; b < B; b++) {
    const float* x = X + (size_t)b * I;
    double h1[ORC_CUT_H], h2[ORC_CUT_H], e[ORC_CUT_E], z[ORC_CUT_BINS], dz[ORC_CUT_BINS], de[ORC_CUT_E];
    double d2[ORC_CUT_H], d1[ORC_CUT_H];
    for (int h = 0; h < H; h++) {
      double a = M->b1[h];
      for (int k = 0; k < I; k++) a += (double)bf16f(M->w1[h * I + k]) * x[k];
      h1[h] = a > 0 ? a : 0;
    }
    for (int h = 0; h < H; h++) {
      double a = M->b2[h];
      for (int k = 0; k < H; k++) a += (double)bf16f(M->w2[h * H + k]) * h1[k];
      h2[h] = a > 0 ? a : 0;
    }
    for (int k = 0; k < E; k++) {
      double a = M->b3[k];
      for (int f = 0; f < H; f++) a += (double)bf16f(M->w3[k * H + f]) * h2[f];
      e[k] = a;
    }
    const int L = lo[b], U = hi[b];
    double zmax = -1e300;
    for (int c = L; c <= U; c++) {
      double a = M->be[c];
      for (int k = 0; k < E; k++) a += (double)bf16f(M->emb[c * E + k]) * e[k];
      z[c] = a;
      if (a > zmax) zmax = a;
    }
    double S = 0.0;
    for (int c = L; c <= U; c++) S += exp(z[c] - zmax);
    loss += -(z[cy[b]] - zmax - log(S));
    for (int k = 0; k < E; k++) de[k] = 0.0;
    for (int c = L; c <= U; c++) {
      dz[c] = exp(z[c] - zmax) / S - (c == cy[b] ? 1.0 : 0.0);
      gbe[c] += dz[c];
      for (int k = 0; k < E; k++) {
        gemb[c * E + k] += dz[c] * e[k];
        de[k] += dz[c] * (double)bf16f(M->emb[c * E + k]);
      }
    }
    for (int k = 0; k < E; k++) {
      gb3[k] += de[k];
      for (int f = 0; f < H; f++) gw3[k * H + f] += de[k] * h2[f];
    }
    for (int f = 0; f < H; f++) {
      double a = 0.0;
      for (int k = 0; k < E; k++) a += de[k] * (double)bf16f(M->w3[k * H + f]);
      d2[f] = h2[f] > 0 ? a : 0.0;
    }
    for (int h = 0; h < H; h++) {
      gb2[h] += d2[h];
      for (int k = 0; k < H; k++) gw2[h * H + k] += d2[h] * h1[k];
    }
    for (int k = 0; k < H; k++) {
      double a = 0.0;
      for (int h = 0; h < H; h++) a += d2[h] * (double)bf16f(M->w2[h * H + k]);
      d1[k] = h1[k] > 0 ? a : 0.0;
    }
    for (int h = 0; h < H; h++) {
      gb1[h] += d1[h];
      for (int k = 0; k < I; k++) gw1[h * I + k] += d1[h] * x[k];
    }
  }
  const double inv = 1.0 / (double)B;
  for (int k = 0; k < H * I; k++) gw1[k] *= inv;
  for (int k = 0; k < H; k++) { gb1[k] *= inv; gb2[k] *= inv; }
  for (int k = 0; k < H * H; k++) gw2[k] *= inv;
  for (int k = 0; k < E * H; k++) gw3[k] *= inv;
  for (int k = 0; k < E; k++) gb3[k] *= inv;
  for (int k = 0; k < NB * E; k++) gemb[k] *= inv;
  for (int k = 0; k < NB; k++) gbe[k] *= inv;
  return loss * inv;
}

double orc_mlp_loss_grad(const orc_model* M, const float* X, const int* y, const uint32_t* mask, int B,
                         double* gw1, double* gb1, double* gw2, double* gb2, double* gw3, double* gb3) {
  const int I = ORC_MLP_IN, H = ORC_MLP_H, O = ORC_MLP_OUT;
  memset(gw1, 0, sizeof(double) * H * I); memset(gb1, 0, sizeof(double) * H);
  memset(gw2, 0, sizeof(double) * H * H); memset(gb2, 0, sizeof(double) * H);
  memset(gw3, 0, sizeof(double) * O * H); memset(gb3, 0, sizeof(double) * O);
  double loss = 0.0;
  for (int b = 0; b < B; b++) {
    const float* x = X + (size_t)b * I;
    double a1[ORC_MLP_H], h1[ORC_MLP_H], a2[ORC_MLP_H], h2[ORC_MLP_H], z[ORC_MLP_OUT], g[ORC_MLP_OUT];
    for (int h = 0; h < H; h++) {
      double a = M->b1[h];
      for (int k = 0; k < I; k++) a += (double)bf16f(M->w1[h * I + k]) * x[k];
      a1[h] = a; h1[h] = a > 0 ? a : 0;
    }
    for (int h = 0; h < H; h++) {
      double a = M->b2[h];
      for (int k = 0; k < H; k++) a += (double)bf16f(M->w2[h * H + k]) * h1[k];
      a2[h] = a; h2[h] = a > 0 ? a : 0;
    }
    double zmax = -1e300;
    for (int o = 0; o < O; o++) {
      double a = M->b3[o];
      for (int k = 0; k < H; k++) a += (double)bf16f(M->w3[o * H + k]) * h2[k];
      z[o] = a;
      if (((mask[b] >> o) & 1u) && a > zmax) zmax = a;
    }
    double S = 0.0;
    for (int o = 0; o < O; o++) S += ((mask[b] >> o) & 1u) ? exp(z[o] - zmax) : 0.0;
    loss += -(z[y[b]] - zmax - log(S));
    for (int o = 0; o < O; o++) g[o] = (((mask[b] >> o) & 1u) ? exp(z[o] - zmax) / S : 0.0) - (o == y[b] ? 1.0 : 0.0);
    double d2[ORC_MLP_H], d1[ORC_MLP_H];
    for (int k = 0; k < H; k++) d2[k] = 0;
    for (int o = 0; o < O; o++) {
      gb3[o] += g[o];
      for (int k = 0; k < H; k++) { gw3[o * H + k] += g[o] * h2[k]; d2[k] += g[o] * (double)bf16f(M->w3[o * H + k]); }
    }
    for (int k = 0; k < H; k++) d2[k] = a2[k] > 0 ? d2[k] : 0;
    for (int k = 0; k < H; k++) d1[k] = 0;
    for (int h = 0; h < H; h++) {
      gb2[h] += d2[h];
      for (int k = 0; k < H; k++) { gw2[h * H + k] += d2[h] * h1[k]; d1[k] += d2[h] * (double)bf16f(M->w2[h * H + k]); }
    }
    for (int k = 0; k < H; k++) d1[k] = a1[k] > 0 ? d1[k] : 0;
    for (int h = 0; h < H; h++) {
      gb1[h] += d1[h];
      for (int k = 0; k < I; k++) gw1[h * I + k] += d1[h] * x[k];
    }
  }
  const double inv = 1.0 / (B > 0 ? B : 1);
  for (int k = 0; k < H * I; k++) gw1[k] *= inv;
  for (int k = 0; k < H; k++) { gb1[k] *= inv; gb2[k] *= inv; }
  for (int k = 0; k < H * H; k++) gw2[k] *= inv;
  for (int k = 0; k < O * H; k++) gw3[k] *= inv;
  for (int k = 0; k < O; k++) gb3[k] *= inv;
  return loss * inv;
}

/* Birth mutation (bart_kernel.cpp:489-501); returns 0 on node-cap. */
static int do_birth(otree* t, int nx, int v, int c, const int* nc, int p, int* L_out, int* R_out) {
  int L = first_free(t->used, -1), R = first_free(t->used, L);
  if (L < 0 || R < 0) return 0;
  t->v[nx] = (uint8_t)v; t->c[nx] = (uint8_t)c; t->l[nx] = (uint8_t)L; t->r[nx] = (uint8_t)R;
  t->par[L] = (uint8_t)nx; t->par[R] = (uint8_t)nx; t->l[L] = t->r[L] = t->l[R] = t->r[R] = 0;
  t->d[L] = t->d[R] = (uint8_t)(t->d[nx] + 1);
  t->used |= (1ull << L) | (1ull << R);
  t->leaf = (t->leaf & ~(1ull << nx)) | (1ull << L) | (1ull << R);
  t->ngv[L] = (uint8_t)count_goodvars(t, L, nc, p); t->ngv[R] = (uint8_t)count_goodvars(t, R, nc, p);
  *L_out = L; *R_out = R;
  return 1;
}
static void do_death(otree* t, int nx, int l, int r) {   /* bart_kernel.cpp:511-515 */
  t->used &= ~((1ull << l) | (1ull << r));
  t->leaf = (t->leaf & ~((1ull << l) | (1ull << r))) | (1ull << nx);
  t->l[nx] = 0; t->r[nx] = 0; t->v[nx] = 0; t->c[nx] = 0;
}
static uint64_t pack_node(const otree* t, int s) {   /* bart_kernel.cpp:565-569 */
  uint32_t thu; memcpy(&thu, &t->th[s], 4);
  return (uint64_t)(BIT(t->used, s) ? (unsigned)t->v[s] : 255u) | ((uint64_t)t->c[s] << 8) | ((uint64_t)t->l[s] << 16) |
         ((uint64_t)t->r[s] << 24) | ((uint64_t)thu << 32);
}

/* ================================================================ REF mode: bit-exact restatement of bart_fit_cpu */
typedef struct { uint32_t s0, s1, s2, s3; } xrng;
static inline uint32_t rotl32(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }
static inline uint32_t xnext(xrng* r) {   /* xoshiro128** (bart_kernel.cpp:53-58) */
  uint32_t res = rotl32(r->s1 * 5, 7) * 9, t = r->s1 << 9;
  r->s2 ^= r->s0; r->s3 ^= r->s1; r->s1 ^= r->s2; r->s0 ^= r->s3; r->s2 ^= t; r->s3 = rotl32(r->s3, 11);
  return res;
}
static inline float xunif_f(xrng* r) { return ((float)(xnext(r) >> 8) + 0.5f) * (1.0f / 16777216.0f); }   /* :59 */
static inline float xnorm_f(xrng* r) {   /* Box-Muller in float with libm logf/cosf (:60) */
  float u1 = xunif_f(r), u2 = xunif_f(r);
  return sqrtf(-2.f * logf(u1)) * cosf(6.28318531f * u2);
}
static double xunif(xrng* r) { return (double)xunif_f(r); }
static double xnorm(xrng* r) { return (double)xnorm_f(r); }
static double xunif_cb(void* ctx) { return xunif((xrng*)ctx); }
static double xgamma_big(xrng* r, double a) {   /* :73-83 */
  double d = a - 1.0 / 3.0, c = 1.0 / sqrt(9.0 * d);
  for (int it = 0; it < 32; it++) {
    double x = xnorm(r), v = 1.0 + c * x;
    if (v <= 0) continue;
    v = v * v * v;
    double u = xunif(r);
    if (log(u) < 0.5 * x * x + d - d * v + d * log(v)) return d * v;
  }
  return d;
}
static double xrtnorm(double mean, double tau, xrng* r) {   /* :282-292 */
  double z;
  tau = tau - mean;
  if (tau <= 0.) {
    do { z = xnorm(r); } while (z < tau);
  } else {
    double lambda = 0.5 * (tau + sqrt(tau * tau + 4.0));
    do { z = -log((double)xunif(r)) / lambda + tau; } while ((double)xunif(r) > exp(-0.5 * (z - lambda) * (z - lambda)));
  }
  return z + mean;
}
static inline double lh_ref(double b, double M, double t2) { double k = b * t2 + 1; return -0.5 * log(k) + 0.5 * M * M * t2 / k; }

typedef struct { double S0[ORC_NODES], S1[ORC_NODES], sL0, sL1, sR0, sR1, rss; int nL, nR; } rstats;
typedef struct { int mode, nx, v, c, L, R, l, r; double thOld[ORC_NODES], thNew[ORC_NODES]; } rupd;

/* Rows live in KL lanes: row i is lane i % KL, position i / KL (bart_kernel.cpp:348-366). */
typedef struct {
  int n, nper, m;
  double *Y, *AF, *TM, *W;   /* [KL][nper] */
  uint8_t *Q;                /* [KL][p][nper] */
  uint8_t *LF;               /* [KL][m][nper] */
} rrows;
#define RIX(R, k, ii) ((size_t)(k) * (R)->nper + (ii))

static void pass_ref(rrows* R, int p, int jp, int j, const rupd* pu, int apply, int cmode, int cnx, int cv, int cc,
                     const double* thc, int stats, int rss, int keep, rstats* st) {
  double a0[ORC_KL][ORC_NODES], a1[ORC_KL][ORC_NODES], bl0[ORC_KL], bl1[ORC_KL], br0[ORC_KL], br1[ORC_KL], ra[ORC_KL];
  int nl[ORC_KL], nr[ORC_KL];
  for (int k = 0; k < ORC_KL; k++) {
    for (int s = 0; s < ORC_NODES; s++) { a0[k][s] = 0; a1[k][s] = 0; }
    bl0[k] = bl1[k] = br0[k] = br1[k] = ra[k] = 0; nl[k] = nr[k] = 0;
  }
  const int nper = R->nper;
  (void)p;
  for (int ii = 0; ii < nper; ii++) {
    for (int k = 0; k < ORC_KL; k++) {
      int valid = ii * ORC_KL + k < R->n;
      double af = R->AF[RIX(R, k, ii)];
      if (apply) {
        uint8_t* lfp = &R->LF[((size_t)k * R->m + jp) * nper + ii];
        int lf = *lfp, lf2 = lf;
        if (pu->mode == 1 && lf == pu->nx) lf2 = (R->Q[((size_t)k * p + pu->v) * nper + ii] <= pu->c) ? pu->L : pu->R;
        else if (pu->mode == 2 && (lf == pu->l || lf == pu->r)) lf2 = pu->nx;
        af = af - pu->thOld[lf] + pu->thNew[lf2];
        *lfp = (uint8_t)lf2;
        R->AF[RIX(R, k, ii)] = af;
      }
      if (rss) {
        double e = R->Y[RIX(R, k, ii)] - af;
        ra[k] += (double)(R->W[RIX(R, k, ii)] * e) * e;
        if (keep) R->TM[RIX(R, k, ii)] += af;
      }
      if (stats) {
        int lf = R->LF[((size_t)k * R->m + j) * nper + ii];
        double r = R->Y[RIX(R, k, ii)] - af + thc[lf];
        double w = R->W[RIX(R, k, ii)];
        double wr = w * r;
        a0[k][lf] += w; a1[k][lf] += wr;
        if (cmode == 1 && lf == cnx && valid) {
          if (R->Q[((size_t)k * p + cv) * nper + ii] <= cc) { nl[k]++; bl0[k] += w; bl1[k] += wr; }
          else { nr[k]++; br0[k] += w; br1[k] += wr; }
        }
      }
    }
  }
  for (int s = 0; s < ORC_NODES; s++) {
    double x0 = 0, x1 = 0;
    for (int k = 0; k < ORC_KL; k++) { x0 += a0[k][s]; x1 += a1[k][s]; }
    st->S0[s] = x0; st->S1[s] = x1;
  }
  st->sL0 = st->sL1 = st->sR0 = st->sR1 = st->rss = 0; st->nL = st->nR = 0;
  for (int k = 0; k < ORC_KL; k++) {
    st->sL0 += bl0[k]; st->sL1 += bl1[k]; st->sR0 += br0[k]; st->sR1 += br1[k]; st->rss += ra[k];
    st->nL += nl[k]; st->nR += nr[k];
  }
}

static int fit_ref(const orc_chain* C, orc_out* o) {
  const int n = C->n, p = C->p, m = C->m, nskip = C->nskip, ndpost = C->ndpost;
  /* inputs as glue.cpp:14-27 hands them to bart_fit_cpu: float y, w, pgtab and float scalars */
  const float tau = (float)C->tau, lambda = (float)C->lambda, nu = (float)C->nu, sigest = (float)C->sigest,
              offset = (float)C->offset;
  const unsigned seed = (unsigned)C->seed;
  int nc[ORC_PMAX];
  double PG[ORC_NODES];
  for (int v = 0; v < ORC_PMAX; v++) nc[v] = v < p ? C->numcut[v] : 0;
  for (int d = 0; d < ORC_NODES; d++) PG[d] = (double)(float)C->pgtab[d];

  rrows R;
  R.n = n; R.m = m; R.nper = (n + ORC_KL - 1) / ORC_KL;
  const size_t rowsz = (size_t)ORC_KL * R.nper;
  R.Y = calloc(rowsz, sizeof(double)); R.AF = calloc(rowsz, sizeof(double)); R.TM = calloc(rowsz, sizeof(double));
  R.W = calloc(rowsz, sizeof(double)); R.Q = calloc(rowsz * (size_t)p, 1); R.LF = calloc(rowsz * (size_t)m, 1);
  otree* T = calloc((size_t)m, sizeof(otree));
  if (!R.Y || !R.AF || !R.TM || !R.W || !R.Q || !R.LF || !T) return -2;
  for (int i = 0; i < R.nper * ORC_KL; i++) {
    int k = i % ORC_KL, ii = i / ORC_KL, ok = i < n;
    R.Y[RIX(&R, k, ii)] = ok ? (double)(C->probit ? 0.0f : (float)C->y[i]) : 0.0;
    R.W[RIX(&R, k, ii)] = ok ? (double)(C->wt ? (float)C->wt[i] : 1.0f) : 0.0;
  }
  for (int v = 0; v < p; v++)
    for (int i = 0; i < R.nper * ORC_KL; i++)
      R.Q[((size_t)(i % ORC_KL) * p + v) * R.nper + i / ORC_KL] = i < n ? C->q[(size_t)v * n + i] : 0;
  int root_ngv = 0;
  for (int v = 0; v < ORC_PMAX; v++) if (v < p && nc[v] >= 1) root_ngv++;
  for (int j = 0; j < m; j++) tree_root(&T[j], root_ngv);

  xrng rng;
  rng.s0 = seed ^ 0x9E3779B9u; rng.s1 = seed * 2654435761u + 1u; rng.s2 = 0x6A09E667u ^ (seed << 7); rng.s3 = 0xBB67AE85u + seed;
  for (int i = 0; i < 16; i++) xnext(&rng);
  if (C->probit)
    for (int i = 0; i < n; i++)
      R.Y[RIX(&R, i % ORC_KL, i / ORC_KL)] = C->ybin[i] == 0 ? -xrtnorm(0., offset, &rng) : xrtnorm(0., -offset, &rng);

  const double t2 = (double)tau * tau, a_prior = 1 / t2, pb = 0.5;
  (void)pb;
  double sigma = sigest;
  int n_birth = 0, n_death = 0, n_cap = 0;
  rupd pu; memset(&pu, 0, sizeof pu);
  rstats st;
  const int total = nskip + ndpost;
  for (int it = 0; it < total; it++) {
    const double inv_s2 = (double)(1.0 / (sigma * sigma));
    for (int j = 0; j < m; j++) {
      otree* t = &T[j];
      oprop cp = propose(t, PG, nc, p, xunif_cb, &rng, 0);
      double thc[ORC_NODES];
      for (int s = 0; s < ORC_NODES; s++) thc[s] = (double)t->th[s];
      pass_ref(&R, p, j - 1, j, &pu, j > 0, cp.mode, cp.nx, cp.v, cp.c, thc, 1, 0, 0, &st);
      rupd nu_; memset(&nu_, 0, sizeof nu_);
      nu_.nx = cp.nx; nu_.v = cp.v; nu_.c = cp.c;
      for (int s = 0; s < ORC_NODES; s++) nu_.thOld[s] = thc[s];
      double S0[ORC_NODES], S1[ORC_NODES];
      for (int s = 0; s < ORC_NODES; s++) { S0[s] = st.S0[s]; S1[s] = st.S1[s]; }
      double lu = log(xunif(&rng));
      if (cp.mode == 1) {
        if (st.nL >= 5 && st.nR >= 5) {
          double bl = st.sL0 * inv_s2, Ml = st.sL1 * inv_s2, br = st.sR0 * inv_s2, Mr = st.sR1 * inv_s2;
          double lalpha = log(cp.pr) + lh_ref(bl, Ml, t2) + lh_ref(br, Mr, t2) - lh_ref(bl + br, Ml + Mr, t2);
          if (lalpha > 0) lalpha = 0;
          if (lu < lalpha) {
            int L, Rr;
            if (!do_birth(t, cp.nx, cp.v, cp.c, nc, p, &L, &Rr)) n_cap++;
            else {
              S0[L] = st.sL0; S1[L] = st.sL1; S0[Rr] = st.sR0; S1[Rr] = st.sR1;
              nu_.mode = 1; nu_.L = L; nu_.R = Rr;
              n_birth++;
            }
          }
        }
      } else if (cp.mode == 2) {
        int nx = cp.nx, l = t->l[nx], r = t->r[nx];
        double bl = S0[l] * inv_s2, Ml = S1[l] * inv_s2, br = S0[r] * inv_s2, Mr = S1[r] * inv_s2;
        double lalpha = log(cp.pr) + lh_ref(bl + br, Ml + Mr, t2) - lh_ref(bl, Ml, t2) - lh_ref(br, Mr, t2);
        if (lalpha > 0) lalpha = 0;
        if (lu < lalpha) {
          S0[nx] = S0[l] + S0[r]; S1[nx] = S1[l] + S1[r];
          do_death(t, nx, l, r);
          nu_.mode = 2; nu_.l = l; nu_.r = r;
          n_death++;
        }
      }
      for (int s = 0; s < ORC_NODES; s++) {   /* DRMU: one normal per slot, used or not (:520-528) */
        double z = xnorm(&rng);
        if (BIT(t->leaf, s) && BIT(t->used, s)) {
          double b = S0[s] * inv_s2, M = S1[s] * inv_s2;
          t->th[s] = (float)(M / (a_prior + b) + z / sqrt(a_prior + b));
        }
      }
      for (int s = 0; s < ORC_NODES; s++) nu_.thNew[s] = (double)t->th[s];
      pu = nu_;
    }
    int keep = it >= nskip;
    double zero[ORC_NODES] = {0};
    pass_ref(&R, p, m - 1, m, &pu, 1, 0, 0, 0, 0, zero, 0, 1, keep, &st);
    pu.mode = 0;
    if (C->probit) {
      for (int i = 0; i < n; i++) {
        double f = R.AF[RIX(&R, i % ORC_KL, i / ORC_KL)];
        R.Y[RIX(&R, i % ORC_KL, i / ORC_KL)] = C->ybin[i] == 0 ? -xrtnorm(-f, offset, &rng) : xrtnorm(f, -offset, &rng);
      }
    } else {
      double rss = st.rss;
      sigma = sqrt((nu * lambda + rss) / (2.0 * xgamma_big(&rng, (n + nu) / 2.0)));
    }
    if (o->sigma) o->sigma[it] = (double)(float)sigma;
    if (keep && o->trees) {
      size_t base = (size_t)(it - nskip) * m * ORC_NODES;
      for (int j = 0; j < m; j++)
        for (int s = 0; s < ORC_NODES; s++) o->trees[base + (size_t)j * ORC_NODES + s] = pack_node(&T[j], s);
    }
  }
  if (o->fmean)
    for (int i = 0; i < n; i++) o->fmean[i] = (double)((float)R.TM[RIX(&R, i % ORC_KL, i / ORC_KL)] / (float)ndpost);
  if (o->yhat && o->trees) orc_yhat_from_trees(o->trees, ndpost, m, C->q, n, o->yhat);
  o->moves[0] = n_birth; o->moves[1] = n_death; o->moves[2] = n_cap;
  o->rtnorm_caps = 0;
  free(R.Y); free(R.AF); free(R.TM); free(R.W); free(R.Q); free(R.LF); free(T);
  return 0;
}

/* ================================================================ DEV mode: the B200 kernels' arithmetic */

/* Apply-deltas of a tree update: every row moves r -= delta, delta = thn[dest] - tho[src] in FP32.  Non-moving rows of
   leaf s use D[s] = thn[s] - tho[s]; a death moves the rows of l and r to nx, so D[l], D[r] hold thn[nx] - tho[l|r];
   a birth moves the rows of nx to L (code <= c) or R, with deltas *DL / *DR. */
static void apply_deltas(const orc_upd* pu, const float* tho, const float* thn, float* D, float* DL, float* DR) {
  for (int s = 0; s < ORC_NODES; s++) D[s] = thn[s] - tho[s];
  *DL = *DR = 0.0f;
  if (pu->mode == 1) { *DL = thn[pu->L] - tho[pu->nx]; *DR = thn[pu->R] - tho[pu->nx]; }
  else if (pu->mode == 2) { D[pu->l] = thn[pu->nx] - tho[pu->l]; D[pu->r] = thn[pu->nx] - tho[pu->r]; }
}

void orc_pass_dev(int n, uint8_t* leaf_prev, const uint8_t* leaf_cur, float* r, const float* w,
                  const uint8_t* qprev, const uint8_t* qcur, const orc_upd* pu, const float* tho, const float* thn,
                  int apply, const orc_prop* cp, const float* thc, int fx_shift, orc_stats* st) {
  const float scale = ldexpf(1.0f, fx_shift);
  float D[ORC_NODES], DL = 0.0f, DR = 0.0f;
  if (apply) apply_deltas(pu, tho, thn, D, &DL, &DR);
  memset(st, 0, sizeof *st);
  for (int i = 0; i < n; i++) {
    float ri = r[i];
    if (apply) {
      int lf = leaf_prev[i], lf2 = lf;
      float delta = D[lf];
      if (pu->mode == 1 && lf == pu->nx) {
        int left = qprev[i] <= pu->c;
        lf2 = left ? pu->L : pu->R;
        delta = left ? DL : DR;
      } else if (pu->mode == 2 && (lf == pu->l || lf == pu->r)) lf2 = pu->nx;
      ri = ri - delta;
      r[i] = ri;
      leaf_prev[i] = (uint8_t)lf2;
    }
    if (leaf_cur) {
      int lc = leaf_cur[i];
      float ws = w[i] * scale;              /* exact: scaling by a power of two */
      float R = ri + thc[lc];
      int64_t wfx = (int64_t)llrintf(ws), wrfx = (int64_t)llrintf(ws * R);
      st->S0[lc] += wfx; st->S1[lc] += wrfx;
      if (cp && cp->mode == 1 && lc == cp->nx) {
        if (qcur[i] <= cp->c) { st->nL++; st->sL0 += wfx; st->sL1 += wrfx; }
        else { st->nR++; st->sR0 += wfx; st->sR1 += wrfx; }
      }
    }
  }
}

/* Over the rows of tree j's leaves a and b (after the pass applied tree j-1's move to r): Q = sum fx2(w R^2) with R =
   r + theta of the row's leaf; with H0 non-NULL also, per code of qv, sum fx(w), sum fx(w R) and the row count. */
static void node_extras(int n, const uint8_t* lf, int a, int b, const float* r, const float* w, const float* thc,
                        const uint8_t* qv, int fx_shift, int rss_shift, int64_t* Q, int64_t* H0, int64_t* H1,
                        int* Hc) {
  const float scale = ldexpf(1.0f, fx_shift), sqs = ldexpf(1.0f, rss_shift - fx_shift);
  *Q = 0;
  for (int i = 0; i < n; i++) {
    if (lf[i] != a && lf[i] != b) continue;
    const float ws = w[i] * scale, R = r[i] + thc[lf[i]], wr = ws * R;
    *Q += (int64_t)llrintf((wr * R) * sqs);
    if (H0) {
      const int cd = qv[i];
      H0[cd] += (int64_t)llrintf(ws);
      H1[cd] += (int64_t)llrintf(wr);
      Hc[cd]++;
    }
  }
}

typedef struct { double u[4]; int k; } dunif;
static double dunif_cb(void* ctx) { dunif* d = (dunif*)ctx; return d->u[d->k++ & 3]; }
static inline double lh_dev(double b, double M, double t2) { double k = b * t2 + 1.0; return -0.5 * orc_log(k) + 0.5 * M * M * t2 / k; }

static int fit_dev(const orc_chain* C, orc_out* o) {
  const int n = C->n, p = C->p, m = C->m, nskip = C->nskip, ndpost = C->ndpost;
  const uint64_t seed = C->seed;
  int nc[ORC_PMAX];
  for (int v = 0; v < ORC_PMAX; v++) nc[v] = v < p ? C->numcut[v] : 0;
  const double* PG = C->pgtab;
  const double scale_inv = ldexp(1.0, -C->fx_shift), rscale = ldexp(1.0, C->rss_shift), rscale_inv = ldexp(1.0, -C->rss_shift);

  float* r = malloc(sizeof(float) * (size_t)n);
  float* w = malloc(sizeof(float) * (size_t)n);
  double* y = malloc(sizeof(double) * (size_t)n);
  double* TM = calloc((size_t)n, sizeof(double));
  uint8_t* LF = calloc((size_t)n * m, 1);
  otree* T = calloc((size_t)m, sizeof(otree));
  if (!r || !w || !y || !TM || !LF || !T) return -2;
  int root_ngv = 0;
  for (int v = 0; v < ORC_PMAX; v++) if (v < p && nc[v] >= 1) root_ngv++;
  for (int j = 0; j < m; j++) tree_root(&T[j], root_ngv);
  int caps = 0;
  for (int i = 0; i < n; i++) {
    w[i] = C->wt ? (float)C->wt[i] : 1.0f;
    if (C->probit)
      y[i] = C->ybin[i] == 0 ? -orc_rtnorm(seed, (uint32_t)i, ORC_INIT_SWEEP, 0.0, C->offset, &caps)
                             : orc_rtnorm(seed, (uint32_t)i, ORC_INIT_SWEEP, 0.0, -C->offset, &caps);
    else y[i] = C->y[i];
    r[i] = (float)y[i];
  }
  const double t2 = C->tau * C->tau, a_prior = 1.0 / t2;
  double sigma = C->sigest;
  int n_birth = 0, n_death = 0, n_cap = 0;
  orc_upd pu = {0, 0, 0, 0, 0, 0, 0, 0};
  float tho[ORC_NODES], thn[ORC_NODES];
  orc_stats st;
  const int total = nskip + ndpost;
  for (int it = 0; it < total; it++) {
    const double inv_s2 = 1.0 / (sigma * sigma);
    for (int j = 0; j < m; j++) {
      otree* t = &T[j];
      uint32_t x[4];
      philox_seed(seed, 0u, (uint32_t)j, (uint32_t)it, ORC_TAG_PROP, x);
      dunif du = {{u32d(x[0]), u32d(x[1]), u32d(x[2]), u32d(x[3])}, 0};
      oprop cp;
      float feat[ORC_MLP_IN];
      uint32_t fvalid = 0;
      if (C->model && C->model->mix > 0.0) {
        uint32_t x2[4];
        philox_seed(seed, 0u, (uint32_t)j, (uint32_t)it, ORC_TAG_PROP2, x2);
        const double u2[2] = {u32d(x2[0]), u32d(x2[1])};
        cp = propose_model(t, PG, nc, p, du.u, u2, C->model, LF + (size_t)j * n, n, feat, &fvalid);
      } else {
        cp = propose(t, PG, nc, p, dunif_cb, &du, 1);
        if (o->train_cap > 0 && cp.mode == 1) {
          /* the birth node is the one propose() chose */
          fvalid = orc_features(t, cp.nx, count_rows(LF + (size_t)j * n, n, cp.nx, cp.nx), -1, nc, p, feat);
        }
      }
      /* a learned cut proposal draws a birth's cut after the pass: the pass then accumulates no split sums */
      const orc_cut_model* CM = (C->cut && C->cut->mix > 0.0) ? C->cut : NULL;
      const int defer = CM && cp.mode == 1;
      orc_prop cpp = {defer ? 0 : cp.mode, cp.nx, cp.v, cp.c};
      float thc[ORC_NODES];
      for (int s = 0; s < ORC_NODES; s++) thc[s] = t->th[s];
      orc_pass_dev(n, j > 0 ? LF + (size_t)(j - 1) * n : NULL, LF + (size_t)j * n, r, w,
                   pu.mode == 1 ? C->q + (size_t)pu.v * n : NULL, cp.mode == 1 ? C->q + (size_t)cp.v * n : NULL, &pu,
                   tho, thn, j > 0, &cpp, thc, C->fx_shift, &st);
      /* the cut proposal's features (and, for a deferred birth, its cut and split sums) */
      float cx[ORC_CUT_IN];
      int cxL = 0, cxU = 0;
      const int want_cx = o->train_cap > 0 && o->train_cx && cp.mode == 1;
      if (cp.mode == 1 && (defer || want_cx)) {
        static int64_t H0[256], H1[256];
        static int Hc[256];
        memset(H0, 0, sizeof H0); memset(H1, 0, sizeof H1); memset(Hc, 0, sizeof Hc);
        const int nx = cp.nx, v = cp.v;
        node_range(t, nx, v, nc[v], &cxL, &cxU);
        int64_t Q;
        const uint8_t* lfj = LF + (size_t)j * n;
        node_extras(n, lfj, nx, nx, r, w, thc, C->q + (size_t)v * n, C->fx_shift, C->rss_shift, &Q, H0, H1, Hc);
        const int cnt = count_rows(lfj, n, nx, nx);
        orc_cut_features(t->d[nx], cnt, st.S0[nx], st.S1[nx], Q, C->fx_shift, C->rss_shift, sigma, cxL, cxU, nc[v],
                         uses_of(t, v, -1), v, cx);
        if (defer) {
          float z[ORC_CUT_BINS];
          double ex[ORC_CUT_BINS];
          orc_cut_logits(CM, cx, cxL, cxU, z);
          const double S = orc_cut_softmax(z, cxL, cxU, ex);
          uint32_t x3[4];
          philox_seed(seed, 0u, (uint32_t)j, (uint32_t)it, ORC_TAG_PROP3, x3);
          double qc;
          const int c = cut_draw(ex, S, cxL, cxU, u32d(x3[0]), u32d(x3[1]), CM->mix, &qc);
          const double corr_c = (1.0 / (double)(cxU - cxL + 1)) / qc;
          double pr = birth_pr_at(t, PG, nx, c, cxL, cxU);
          pr = pr * cp.corr;
          pr = pr * corr_c;
          cp.pr = pr; cp.c = c;
          int64_t sL0 = 0, sL1 = 0;
          int nL = 0;
          for (int k = 0; k <= c; k++) { sL0 += H0[k]; sL1 += H1[k]; nL += Hc[k]; }
          st.sL0 = sL0; st.sL1 = sL1; st.nL = nL;
          st.sR0 = st.S0[nx] - sL0; st.sR1 = st.S1[nx] - sL1; st.nR = cnt - nL;
        }
      } else if (CM && cp.mode == 2) {   /* the reverse birth's cut probability at the collapsed node */
        const int nx = cp.nx, l = t->l[nx], rr = t->r[nx], v = t->v[nx], cn = t->c[nx];
        int L, U;
        node_range(t, nx, v, nc[v], &L, &U);
        int64_t Q;
        const uint8_t* lfj = LF + (size_t)j * n;
        node_extras(n, lfj, l, rr, r, w, thc, NULL, C->fx_shift, C->rss_shift, &Q, NULL, NULL, NULL);
        float z[ORC_CUT_BINS];
        double ex[ORC_CUT_BINS];
        orc_cut_features(t->d[nx], count_rows(lfj, n, l, rr), st.S0[l] + st.S0[rr], st.S1[l] + st.S1[rr], Q,
                         C->fx_shift, C->rss_shift, sigma, L, U, nc[v], uses_of(t, v, nx), v, cx);
        orc_cut_logits(CM, cx, L, U, z);
        const double S = orc_cut_softmax(z, L, U, ex);
        const double corr_c = cut_prob(ex, S, L, U, cn, CM->mix) * (double)(U - L + 1);
        cp.pr = cp.pr * corr_c;
      }
      orc_upd nu_ = {0, cp.nx, cp.v, cp.c, 0, 0, 0, 0};
      int64_t S0[ORC_NODES], S1[ORC_NODES];
      for (int s = 0; s < ORC_NODES; s++) { S0[s] = st.S0[s]; S1[s] = st.S1[s]; }
      if (cp.mode != 0) {
        philox_seed(seed, 0u, (uint32_t)j, (uint32_t)it, ORC_TAG_MH, x);
        double lu = orc_log(u32d(x[0]));
        double logpr = orc_log(cp.pr);
        if (cp.mode == 1) {
          if (st.nL >= 5 && st.nR >= 5) {
            double bl = (double)st.sL0 * scale_inv * inv_s2, Ml = (double)st.sL1 * scale_inv * inv_s2;
            double br = (double)st.sR0 * scale_inv * inv_s2, Mr = (double)st.sR1 * scale_inv * inv_s2;
            double lalpha = logpr + lh_dev(bl, Ml, t2) + lh_dev(br, Mr, t2) - lh_dev(bl + br, Ml + Mr, t2);
            if (lalpha > 0) lalpha = 0;
            if (lu < lalpha) {
              int L, Rr;
              if (!do_birth(t, cp.nx, cp.v, cp.c, nc, p, &L, &Rr)) n_cap++;
              else {
                S0[L] = st.sL0; S1[L] = st.sL1; S0[Rr] = st.sR0; S1[Rr] = st.sR1;
                nu_.mode = 1; nu_.L = L; nu_.R = Rr;
                n_birth++;
                if (o->train_cap > 0 && o->train_count < o->train_cap) {
                  memcpy(o->train_x + (size_t)o->train_count * ORC_MLP_IN, feat, sizeof feat);
                  o->train_y[o->train_count] = cp.v;
                  o->train_mask[o->train_count] = fvalid;
                  if (o->train_cx) {
                    memcpy(o->train_cx + (size_t)o->train_count * ORC_CUT_IN, cx, sizeof cx);
                    o->train_c[o->train_count] = cp.c;
                    o->train_lo[o->train_count] = cxL;
                    o->train_hi[o->train_count] = cxU;
                  }
                  o->train_count++;
                }
              }
            }
          }
        } else {
          int nx = cp.nx, l = t->l[nx], rr = t->r[nx];
          double bl = (double)S0[l] * scale_inv * inv_s2, Ml = (double)S1[l] * scale_inv * inv_s2;
          double br = (double)S0[rr] * scale_inv * inv_s2, Mr = (double)S1[rr] * scale_inv * inv_s2;
          double lalpha = logpr + lh_dev(bl + br, Ml + Mr, t2) - lh_dev(bl, Ml, t2) - lh_dev(br, Mr, t2);
          if (lalpha > 0) lalpha = 0;
          if (lu < lalpha) {
            S0[nx] = S0[l] + S0[rr]; S1[nx] = S1[l] + S1[rr];
            do_death(t, nx, l, rr);
            nu_.mode = 2; nu_.l = l; nu_.r = rr;
            n_death++;
          }
        }
      }
      for (int s = 0; s < ORC_NODES; s++) tho[s] = t->th[s];
      for (int s = 0; s < ORC_NODES; s++) {
        if (BIT(t->leaf, s) && BIT(t->used, s)) {
          double b = (double)S0[s] * scale_inv * inv_s2, M = (double)S1[s] * scale_inv * inv_s2;
          double z = orc_normal(seed, (uint32_t)s << 8, (uint32_t)j, (uint32_t)it, ORC_TAG_MU);
          t->th[s] = (float)(M / (a_prior + b) + z / sqrt(a_prior + b));
        }
      }
      for (int s = 0; s < ORC_NODES; s++) thn[s] = t->th[s];
      pu = nu_;
    }
    /* end of sweep: apply tree m-1's move to its leaf ids, FP64 tree-order refresh, rss / latent z, kept draws */
    orc_pass_dev(n, LF + (size_t)(m - 1) * n, NULL, r, w, pu.mode == 1 ? C->q + (size_t)pu.v * n : NULL, NULL, &pu,
                 tho, thn, 1, NULL, NULL, C->fx_shift, &st);
    pu.mode = 0;
    const int keep = it >= nskip;
    int64_t rssfx = 0;
    for (int i = 0; i < n; i++) {
      double f = 0.0;
      for (int j = 0; j < m; j++) f += (double)T[j].th[LF[(size_t)j * n + i]];
      if (C->probit)
        y[i] = C->ybin[i] == 0 ? -orc_rtnorm(seed, (uint32_t)i, (uint32_t)it, -f, C->offset, &caps)
                               : orc_rtnorm(seed, (uint32_t)i, (uint32_t)it, f, -C->offset, &caps);
      double e = y[i] - f;
      r[i] = (float)e;
      if (!C->probit) {
        double we = (double)w[i] * e;
        rssfx += (int64_t)llrint(we * e * rscale);
      }
      if (keep) {
        TM[i] += f;
        if (o->yhat) o->yhat[(size_t)(it - nskip) * n + i] = f;
      }
    }
    if (!C->probit) {
      double rss = (double)rssfx * rscale_inv;
      sigma = sqrt((C->nu * C->lambda + rss) / (2.0 * orc_gamma(seed, (uint32_t)it, ((double)n + C->nu) / 2.0)));
    }
    if (o->sigma) o->sigma[it] = sigma;
    if (keep && o->trees) {
      size_t base = (size_t)(it - nskip) * m * ORC_NODES;
      for (int j = 0; j < m; j++)
        for (int s = 0; s < ORC_NODES; s++) o->trees[base + (size_t)j * ORC_NODES + s] = pack_node(&T[j], s);
    }
  }
  if (o->fmean) for (int i = 0; i < n; i++) o->fmean[i] = TM[i] / (double)ndpost;
  o->moves[0] = n_birth; o->moves[1] = n_death; o->moves[2] = n_cap;
  o->rtnorm_caps = caps;
  free(r); free(w); free(y); free(TM); free(LF); free(T);
  return 0;
}

int orc_fit(const orc_chain* c, int mode, orc_out* o) {
  if (c->n < 1 || c->p < 1 || c->p > ORC_PMAX || c->m < 1 || c->m > ORC_MMAX || c->ndpost < 1 || c->nskip < 0) return -1;
  if (c->probit && !c->ybin) return -1;
  if (!c->probit && !c->y) return -1;
  return mode == ORC_MODE_REF ? fit_ref(c, o) : fit_dev(c, o);
}

/* ================================================================ evaluator (src/predict.cpp:11-73) */
typedef struct { int* a; size_t n, cap; } ivec;
typedef struct { double* a; size_t n, cap; } dvec;
static int ipush(ivec* v, int x) {
  if (v->n == v->cap) { size_t c = v->cap ? v->cap * 2 : 1024; int* a = realloc(v->a, c * sizeof(int)); if (!a) return -1; v->a = a; v->cap = c; }
  v->a[v->n++] = x; return 0;
}
static int dpush(dvec* v, double x) {
  if (v->n == v->cap) { size_t c = v->cap ? v->cap * 2 : 1024; double* a = realloc(v->a, c * sizeof(double)); if (!a) return -1; v->a = a; v->cap = c; }
  v->a[v->n++] = x; return 0;
}

int orc_compile_trees(const char* text, const double* const* xi, const int* ncut, int ncol, orc_ct* out) {
  const char* s = text;
  char* e;
  memset(out, 0, sizeof *out);
  long nd = strtol(s, &e, 10); s = e;
  long m = strtol(s, &e, 10); s = e;
  long p = strtol(s, &e, 10); s = e;
  (void)ncol;
  if (nd < 1 || m < 1) return -1;
  ivec var = {0}, child = {0}, root = {0};
  dvec cut = {0}, theta = {0};
  for (long t = 0; t < nd * m; t++) {
    long nn = strtol(s, &e, 10); if (e == s) return -1; s = e;
    size_t* nid = malloc(sizeof(size_t) * (size_t)nn); int* v = malloc(sizeof(int) * (size_t)nn);
    int* c = malloc(sizeof(int) * (size_t)nn); double* th = malloc(sizeof(double) * (size_t)nn);
    for (long k = 0; k < nn; k++) {
      nid[k] = (size_t)strtoull(s, &e, 10); s = e;
      v[k] = (int)strtol(s, &e, 10); s = e;
      c[k] = (int)strtol(s, &e, 10); s = e;
      th[k] = strtod(s, &e); s = e;
    }
    /* position of a node id among this tree's lines (ids are unique per tree); missing ids map to line 0, as
       std::unordered_map::operator[] would insert 0 (src/predict.cpp:26, 38) */
#define POS(id) ({ long _r = -1; for (long _k = 0; _k < nn; _k++) if (nid[_k] == (size_t)(id)) { _r = _k; break; } _r; })
    long* q = malloc(sizeof(long) * (size_t)(nn + 1)); int* slot = malloc(sizeof(int) * (size_t)(nn + 1));
    long qn = 0;
    long r0 = POS(1); if (r0 < 0) r0 = 0;
    q[qn] = r0; slot[qn] = (int)var.n; qn++;
    ipush(&root, (int)var.n);
    ipush(&var, 0); ipush(&child, -1); dpush(&cut, 0); dpush(&theta, 0);
    for (long h = 0; h < qn; h++) {
      long k = q[h]; int me = slot[h];
      long L = POS(2 * nid[k]);
      theta.a[me] = th[k];
      if (L >= 0) {
        int ch = (int)var.n;
        var.a[me] = v[k]; cut.a[me] = xi[v[k]][c[k]]; child.a[me] = ch;
        for (int z = 0; z < 2; z++) { ipush(&var, 0); ipush(&child, -1); dpush(&cut, 0); dpush(&theta, 0); }
        long Rk = POS(2 * nid[k] + 1); if (Rk < 0) Rk = 0;
        q[qn] = L; slot[qn] = ch; qn++;
        q[qn] = Rk; slot[qn] = ch + 1; qn++;
      }
    }
#undef POS
    free(q); free(slot); free(nid); free(v); free(c); free(th);
  }
  (void)ncut;
  out->ndpost = (int)nd; out->ntree = (int)m; out->p = (int)p; out->nnodes = (int)var.n;
  out->var = var.a; out->child = child.a; out->cut = cut.a; out->theta = theta.a; out->root = root.a;
  return 0;
}

void orc_ct_free(orc_ct* ct) {
  free(ct->var); free(ct->child); free(ct->cut); free(ct->theta); free(ct->root);
  memset(ct, 0, sizeof *ct);
}

int orc_predict_draw(const orc_ct* ct, const double* const* cols, int ncol, int n, int draw1, double mu, double* f) {
  if (ncol != ct->p) return -1;                       /* predict.cpp:51 */
  if (draw1 < 1 || draw1 > ct->ndpost) return -2;      /* predict.cpp:52 */
  for (int i = 0; i < n; i++) f[i] = 0.0;
  const int* r0 = ct->root + (size_t)(draw1 - 1) * ct->ntree;
  for (int t = 0; t < ct->ntree; t++) {                /* tree-outer, row-inner (predict.cpp:62-68) */
    const int k0 = r0[t];
    for (int i = 0; i < n; i++) {
      int k = k0;
      while (ct->child[k] >= 0) k = ct->child[k] + (int)(cols[ct->var[k]][i] >= ct->cut[k]);
      f[i] += ct->theta[k];
    }
  }
  for (int i = 0; i < n; i++) f[i] += mu;
  return 0;
}

/* ================================================================ output assembly (src/glue.cpp:29-57) */
#define PK_L(w) ((int)(((w) >> 16) & 255))
#define PK_R(w) ((int)(((w) >> 24) & 255))
#define PK_V(w) ((int)((w) & 255))
#define PK_C(w) ((int)(((w) >> 8) & 255))
static double pk_th(uint64_t w) { uint32_t u = (uint32_t)(w >> 32); float f; memcpy(&f, &u, 4); return (double)f; }

typedef struct { char* buf; size_t cap, len; } sbuf;
static void sput(sbuf* b, const char* s, size_t k) {
  if (b->buf && b->len < b->cap) {
    size_t room = b->cap - b->len, c = k < room ? k : room;
    memcpy(b->buf + b->len, s, c);
  }
  b->len += k;
}

size_t orc_trees_text(const uint64_t* trees, int ndpost, int m, int p, char* buf, size_t cap) {
  sbuf b = {buf, cap, 0};
  char line[128];
  int k = snprintf(line, sizeof line, "%d %d %d\n", ndpost, m, p);
  sput(&b, line, (size_t)k);
  for (int dr = 0; dr < ndpost; dr++)
    for (int j = 0; j < m; j++) {
      const uint64_t* T = &trees[((size_t)dr * m + j) * ORC_NODES];
      int st_s[2 * ORC_NODES + 2], ord_s[ORC_NODES + 1]; size_t st_id[2 * ORC_NODES + 2], ord_id[ORC_NODES + 1];
      int sp = 0, no = 0;
      st_s[sp] = 0; st_id[sp] = 1; sp++;
      while (sp > 0 && no <= ORC_NODES) {   /* pre-order; ids: root 1, children 2id, 2id+1 (glue.cpp:40-44) */
        sp--; int s = st_s[sp]; size_t id = st_id[sp];
        ord_s[no] = s; ord_id[no] = id; no++;
        if (PK_L(T[s])) {
          st_s[sp] = PK_R(T[s]); st_id[sp] = 2 * id + 1; sp++;
          st_s[sp] = PK_L(T[s]); st_id[sp] = 2 * id; sp++;
        }
      }
      k = snprintf(line, sizeof line, "%d\n", no);
      sput(&b, line, (size_t)k);
      for (int q = 0; q < no; q++) {
        int s = ord_s[q], leaf = PK_L(T[s]) == 0;
        int v = leaf ? 0 : PK_V(T[s]), c = leaf ? 0 : PK_C(T[s]);
        k = snprintf(line, sizeof line, "%zu %d %d %.10g\n", ord_id[q], v, c, leaf ? pk_th(T[s]) : 0.0);
        sput(&b, line, (size_t)k);
      }
    }
  if (buf && cap > 0) buf[b.len < cap ? b.len : cap - 1] = 0;
  return b.len;
}

void orc_varcount(const uint64_t* trees, int ndpost, int m, int p, int* varcount) {
  memset(varcount, 0, sizeof(int) * (size_t)ndpost * p);
  for (int dr = 0; dr < ndpost; dr++)
    for (int j = 0; j < m; j++) {
      const uint64_t* T = &trees[((size_t)dr * m + j) * ORC_NODES];
      int st[2 * ORC_NODES + 2], sp = 0, seen = 0;
      st[sp++] = 0;
      while (sp > 0 && seen <= ORC_NODES) {
        int s = st[--sp]; seen++;
        if (PK_L(T[s])) { varcount[(size_t)dr * p + PK_V(T[s])] += 1; st[sp++] = PK_R(T[s]); st[sp++] = PK_L(T[s]); }
      }
    }
}

void orc_yhat_from_trees(const uint64_t* trees, int ndpost, int m, const uint8_t* q, int n, double* yhat) {
  for (int dr = 0; dr < ndpost; dr++) {
    double* y = yhat + (size_t)dr * n;
    for (int i = 0; i < n; i++) y[i] = 0.0;
    for (int j = 0; j < m; j++) {   /* glue.cpp:52-56: tree order, leaf value float -> double */
      const uint64_t* T = &trees[((size_t)dr * m + j) * ORC_NODES];
      for (int i = 0; i < n; i++) {
        int s = 0;
        while (PK_L(T[s])) s = q[(size_t)PK_V(T[s]) * n + i] <= PK_C(T[s]) ? PK_L(T[s]) : PK_R(T[s]);
        y[i] += pk_th(T[s]);
      }
    }
  }
}
