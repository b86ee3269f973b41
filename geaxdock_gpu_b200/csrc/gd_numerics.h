/*
 * gd_numerics.h -- arithmetic that must give the same bits on the host and the device.
 *
 * The Monte Carlo decisions (Metropolis accept, replica exchange) and the proposal moves
 * are written here once, with every rounding step explicit: products and sums go through
 * GD_MUL/GD_ADD (no contraction on either side), multiply-adds through fmaf, and the
 * transcendental functions are our own short polynomial evaluations on a reduced
 * argument (Cody & Waite, "Software Manual for the Elementary Functions", 1980, for the
 * reductions; truncated Taylor / atanh series for the kernels). IEEE division and square
 * root are correctly rounded on both sides. Compiled by gcc with -ffp-contract=off and by
 * nvcc without fast-math, two builds of this header produce identical results from
 * identical inputs, which is what makes accept/exchange decisions replayable bit for bit.
 *
 * Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
 * as easy as 1, 2, 3", SC'11), counter-based, keyed by the run seed.
 */
#ifndef GD_NUMERICS_H
#define GD_NUMERICS_H

#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define GD_HD __host__ __device__ __forceinline__
#define GD_UNROLL _Pragma("unroll")
#else
#define GD_HD static inline
#define GD_UNROLL
#endif

#if defined(__CUDA_ARCH__)
#define GD_MUL(a, b) __fmul_rn((a), (b))
#define GD_ADD(a, b) __fadd_rn((a), (b))
#define GD_SUB(a, b) __fsub_rn((a), (b))
#define GD_FMA(a, b, c) __fmaf_rn((a), (b), (c))
#define GD_RINT(x) rintf(x)
#else
#define GD_MUL(a, b) ((float)(a) * (float)(b))
#define GD_ADD(a, b) ((float)(a) + (float)(b))
#define GD_SUB(a, b) ((float)(a) - (float)(b))
#define GD_FMA(a, b, c) fmaf((a), (b), (c))
#define GD_RINT(x) rintf(x)
#endif

/* ---------------- Philox4x32-10 ---------------- */
typedef struct { uint32_t v[4]; } gd_u32x4;

GD_HD uint32_t gd_mulhi32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

GD_HD gd_u32x4 gd_philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                               uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
GD_UNROLL
  for (int round = 0; round < 10; ++round) {
    const uint32_t hi0 = gd_mulhi32(M0, c0), lo0 = M0 * c0;
    const uint32_t hi1 = gd_mulhi32(M1, c2), lo1 = M1 * c2;
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    k0 += W0; k1 += W1;
  }
  gd_u32x4 r;
  r.v[0] = c0; r.v[1] = c1; r.v[2] = c2; r.v[3] = c3;
  return r;
}

/* Stream purposes (last counter word). */
#define GD_RNG_MOVE 0u      /* word 0..3: move dims 0..3 */
#define GD_RNG_MOVE2 1u     /* word 0..1: move dims 4..5, word 2: accept, word 3: surrogate
                               stage of delayed acceptance */
#define GD_RNG_EXCHANGE 2u  /* word 0: exchange uniform */
#define GD_RNG_INIT 3u
#define GD_RNG_TRAIN 4u     /* surrogate training: batch row picks */

/* [0, 1): 24 random bits, exact in float. */
GD_HD float gd_u01(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-08f; }
/* (0, 1]. */
GD_HD float gd_u01_open0(uint32_t x) { return (float)((x >> 8) + 1u) * 5.9604644775390625e-08f; }
/* (-1, 1), symmetric: odd multiples of 2^-24. */
GD_HD float gd_sym11(uint32_t x) {
  const int j = (int)(x >> 8);
  return (float)(2 * j + 1 - 16777216) * 5.9604644775390625e-08f;
}

/* ---------------- exp ---------------- */
/* exp(x) = 2^k * exp(r), k = rint(x / ln2), r = x - k ln2 (two-part ln2), degree-7 Taylor.
 * Results below FLT_MIN are returned as 0 so that the final scaling is always exact. */
GD_HD float gd_expf(float x) {
  if (!(x == x)) return x;
  if (x > 88.72283172607421875f) return INFINITY;
  if (x < -87.33654475f) return 0.0f;
  const float k = GD_RINT(GD_MUL(x, 1.44269502162933349609375f));
  float r = GD_FMA(-k, 0.693145751953125f, x);
  r = GD_FMA(-k, 1.428606765330187e-06f, r);
  float p = 1.98412698412698e-04f;             /* 1/5040 */
  p = GD_FMA(p, r, 1.38888888888889e-03f);     /* 1/720 */
  p = GD_FMA(p, r, 8.33333333333333e-03f);     /* 1/120 */
  p = GD_FMA(p, r, 4.16666666666667e-02f);     /* 1/24 */
  p = GD_FMA(p, r, 1.66666666666667e-01f);     /* 1/6 */
  p = GD_FMA(p, r, 0.5f);
  p = GD_FMA(p, r, 1.0f);
  p = GD_FMA(p, r, 1.0f);
  return ldexpf(p, (int)k);
}

/* ---------------- log on (0, +inf) ---------------- */
/* log(x) = e ln2 + 2 atanh(s), s = (m-1)/(m+1), m in [sqrt(1/2), sqrt(2)). */
GD_HD float gd_logf(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
  int e;
  float m = frexpf(x, &e); /* x = m 2^e, m in [0.5, 1) */
  if (m < 0.70710678118654752f) { m = GD_MUL(m, 2.0f); e -= 1; }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = GD_MUL(s, s);
  float p = 1.11111111111111e-01f;             /* 1/9 */
  p = GD_FMA(p, s2, 1.42857142857143e-01f);    /* 1/7 */
  p = GD_FMA(p, s2, 2.0e-01f);                 /* 1/5 */
  p = GD_FMA(p, s2, 3.33333333333333e-01f);    /* 1/3 */
  p = GD_FMA(p, s2, 1.0f);
  const float lm = GD_MUL(GD_MUL(2.0f, s), p);
  const float fe = (float)e;
  return GD_FMA(fe, 0.693145751953125f, GD_FMA(fe, 1.428606765330187e-06f, lm));
}

/* ---------------- sin / cos ---------------- */
/* Quadrant reduction by pi/2 in three parts, Taylor kernels on |r| <= pi/4. */
GD_HD void gd_sincosf(float x, float *sp, float *cp) {
  const float k = GD_RINT(GD_MUL(x, 0.636619746685028076171875f));
  float r = GD_FMA(-k, 1.5703125f, x);
  r = GD_FMA(-k, 4.838705062866211e-04f, r);
  r = GD_FMA(-k, -4.371138828673793e-08f, r);
  const float r2 = GD_MUL(r, r);
  float ps = 2.75573192239859e-06f;            /* 1/9! */
  ps = GD_FMA(ps, r2, -1.98412698412698e-04f); /* -1/7! */
  ps = GD_FMA(ps, r2, 8.33333333333333e-03f);  /* 1/5! */
  ps = GD_FMA(ps, r2, -1.66666666666667e-01f); /* -1/3! */
  const float sn = GD_FMA(GD_MUL(ps, r2), r, r);
  float pc = -2.75573192239859e-07f;           /* -1/10! */
  pc = GD_FMA(pc, r2, 2.48015873015873e-05f);  /* 1/8! */
  pc = GD_FMA(pc, r2, -1.38888888888889e-03f); /* -1/6! */
  pc = GD_FMA(pc, r2, 4.16666666666667e-02f);  /* 1/4! */
  pc = GD_FMA(pc, r2, -0.5f);
  const float cs = GD_FMA(pc, r2, 1.0f);
  const int q = ((int)k) & 3;
  float s, c;
  if (q == 0) { s = sn; c = cs; }
  else if (q == 1) { s = cs; c = -sn; }
  else if (q == 2) { s = -sn; c = -cs; }
  else { s = -cs; c = sn; }
  *sp = s; *cp = c;
}

/* ---------------- Gaussian pair (Box-Muller) ---------------- */
GD_HD void gd_box_muller(uint32_t a, uint32_t b, float *z0, float *z1) {
  const float u1 = gd_u01_open0(a);
  const float u2 = gd_u01(b);
  const float rad = sqrtf(GD_MUL(-2.0f, gd_logf(u1)));
  float s, c;
  gd_sincosf(GD_MUL(6.28318548202514648f, u2), &s, &c);
  *z0 = GD_MUL(rad, c);
  *z1 = GD_MUL(rad, s);
}

/* ---------------- proposal for one replica and one step ---------------- */
/* Draws the six move deltas and the accept uniform for (stream, replica, step).
 * stream identifies the complex (so a complex run alone or inside a batch draws the same
 * numbers); replica is the complex-local flat index n_tmp*n_lig*p + n_lig*t + l. */
GD_HD void gd_draw_step(uint64_t seed, uint32_t stream, uint32_t replica, uint32_t step,
                        int move_kind, const float scale[6], float delta[6], float *u_accept) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  const gd_u32x4 a = gd_philox4x32_10(replica, step, stream, GD_RNG_MOVE, k0, k1);
  const gd_u32x4 b = gd_philox4x32_10(replica, step, stream, GD_RNG_MOVE2, k0, k1);
  if (move_kind == 1) {
    float z[6];
    gd_box_muller(a.v[0], a.v[1], &z[0], &z[1]);
    gd_box_muller(a.v[2], a.v[3], &z[2], &z[3]);
    gd_box_muller(b.v[0], b.v[1], &z[4], &z[5]);
    for (int i = 0; i < 6; ++i) delta[i] = GD_MUL(scale[i], z[i]);
  } else {
    const uint32_t w[6] = {a.v[0], a.v[1], a.v[2], a.v[3], b.v[0], b.v[1]};
    for (int i = 0; i < 6; ++i) delta[i] = GD_MUL(scale[i], gd_sym11(w[i]));
  }
  *u_accept = gd_u01(b.v[2]);
}

/* Uniform of the surrogate (first) stage of a delayed-acceptance step: the spare word of the
 * proposal's second Philox block, so the move and the final accept uniform stay those of the
 * plain step. */
GD_HD float gd_draw_stage1(uint64_t seed, uint32_t stream, uint32_t replica, uint32_t step) {
  const gd_u32x4 b = gd_philox4x32_10(replica, step, stream, GD_RNG_MOVE2, (uint32_t)seed,
                                      (uint32_t)(seed >> 32));
  return gd_u01(b.v[3]);
}

/* Exchange uniform for (stream, complex-local group p*n_lig + l, exchange call, pair). */
GD_HD float gd_draw_exchange(uint64_t seed, uint32_t stream, uint32_t group,
                             uint32_t exchange_call, uint32_t pair) {
  const gd_u32x4 a = gd_philox4x32_10(group, exchange_call, stream,
                                      GD_RNG_EXCHANGE | (pair << 8), (uint32_t)seed,
                                      (uint32_t)(seed >> 32));
  return gd_u01(a.v[0]);
}

/* ---------------- rigid-body transform (reference Move_d, src/kernel_cuda_l2_move.cu:21-80) ---------------- */
/* Z-Y-X Euler rotation from movematrix[3..5]. */
GD_HD void gd_rotation(const float mm[6], float rot[9]) {
  float s1, c1, s2, c2, s3, c3;
  gd_sincosf(mm[3], &s1, &c1);
  gd_sincosf(mm[4], &s2, &c2);
  gd_sincosf(mm[5], &s3, &c3);
  rot[0] = GD_MUL(c1, c2);
  rot[1] = GD_SUB(GD_MUL(GD_MUL(c1, s2), s3), GD_MUL(c3, s1));
  rot[2] = GD_ADD(GD_MUL(s1, s3), GD_MUL(GD_MUL(c1, c3), s2));
  rot[3] = GD_MUL(c2, s1);
  rot[4] = GD_ADD(GD_MUL(c1, c3), GD_MUL(GD_MUL(s1, s2), s3));
  rot[5] = GD_SUB(GD_MUL(GD_MUL(c3, s1), s2), GD_MUL(c1, s3));
  rot[6] = -s2;
  rot[7] = GD_MUL(c2, s3);
  rot[8] = GD_MUL(c2, c3);
}

/* x_lab = R x_orig + t + c_orig, with the translation folded first. */
GD_HD void gd_place_atom(const float rot[9], float tx, float ty, float tz, float x, float y,
                         float z, float *ox, float *oy, float *oz) {
  *ox = GD_FMA(rot[0], x, GD_FMA(rot[1], y, GD_FMA(rot[2], z, tx)));
  *oy = GD_FMA(rot[3], x, GD_FMA(rot[4], y, GD_FMA(rot[5], z, ty)));
  *oz = GD_FMA(rot[6], x, GD_FMA(rot[7], y, GD_FMA(rot[8], z, tz)));
}

/* ---------------- decisions ---------------- */
/* Metropolis (reference Accept_d, src/kernel_cuda_l2_accept.cu:13-46):
 * accept iff u < exp((E_new - E_old) * minus_beta). */
GD_HD int gd_metropolis(float e_new, float e_old, float minus_beta, float u) {
  const float d = GD_MUL(GD_SUB(e_new, e_old), minus_beta);
  return u < gd_expf(d);
}

/* Second stage of delayed acceptance (Christen & Fox, J. Comput. Graph. Stat. 14, 2005):
 * accept iff u < exp(((E_new - E_old) - (S_new - S_old)) * minus_beta), S the surrogate
 * energy that admitted the proposal in the first stage. With S_new == S_old the difference is
 * +0 and the decision is bit-identical to gd_metropolis. */
GD_HD int gd_da_stage2(float e_new, float e_old, float s_new, float s_old, float minus_beta,
                       float u) {
  const float d = GD_MUL(GD_SUB(GD_SUB(e_new, e_old), GD_SUB(s_new, s_old)), minus_beta);
  return u < gd_expf(d);
}

/* Temperature swap (reference ExchangeReplicas_d, src/kernel_cuda_l1_exchangereplicas.cu:52-67):
 * accept iff exp((mb1 - mb2) * (E2 - E1)) > u. */
GD_HD int gd_exchange_accept(float e1, float e2, float mb1, float mb2, float u) {
  const float d = GD_MUL(GD_SUB(mb1, mb2), GD_SUB(e2, e1));
  return gd_expf(d) > u;
}

#endif /* GD_NUMERICS_H */
