/*
 * gd_kernels.cu -- sm_100a kernels of the Monte Carlo docking path.
 *
 * gd_mc_kernel: one persistent kernel for MonteCarlo_Init_d, MonteCarlo_d and pose
 * evaluation (reference src/kernel_cuda_l1_montecarlo.cu:12-127). Each CTA pulls tiles from
 * a work queue; a tile is `count` replicas of one protein conformer. Lane (slot j, atom l)
 * owns one ligand atom of one replica for all steps of the launch (a thread holds one lane,
 * or with PACK = 2 the lanes of the same atom in two slots, which share every load):
 *   Move_d        (src/kernel_cuda_l2_move.cu:21-80)       placed in registers from a
 *                                                         Philox draw, no HBM traffic;
 *   CalcEnergy_d  (src/kernel_cuda_l2_calcenergy.cu:19-360) the terms every pair has (vdw,
 *                 ele in its far form, pmf, hdb) in a loop over all protein points staged by
 *                 cp.async.bulk into a shared-memory double buffer, points sorted by type so
 *                 each lane keeps its pair parameters in registers per segment, MUFU rsqrt /
 *                 rcp / ex2, FP32 range sums folded into FP64; the short-range terms
 *                 (contacts, psp, hpc, the ele soft core) from a walk of the conformer's cell
 *                 list over the points within 9 A;
 *   CalcMcc_d     (src/kernel_cuda_l2_calcmcc.cu:148-206) contact count in the cell walk,
 *                 true positives from the sparse reference-contact list;
 *   CalcRmsd_d, KDE, MCS, dst, CombineEnergy_d (src/kernel_cuda_l3_combineenergy.cu:23-37),
 *                 of moved poses (modes 0-3) or of given placed coordinates (mode 4),
 *   Accept_d (src/kernel_cuda_l2_accept.cu:13-46), RecordLigand_d
 *   (src/kernel_cuda_l3_util.cu:74-106) in the per-replica epilogue run by one warp per slot.
 * gd_exchange_kernel: ExchangeReplicas_d (src/kernel_cuda_l1_exchangereplicas.cu:27-77), one
 * thread per (protein conformer, ligand conformer) group instead of one thread for all.
 */
#include <cuda_runtime.h>

#include "gd_device.cuh"
#include "gd_numerics.h"

namespace gd {

/* ---------------- MUFU / PTX helpers ---------------- */
__device__ __forceinline__ float rsqrt_a(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_a(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_a(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ long long gtimer() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
/* Spins on the barrier phase for at most timeout_ns (globaltimer); false on timeout. */
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  long long timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long deadline = gtimer() + timeout_ns;
  while (!mbar_try_wait(bar, parity))
    if (gtimer() > deadline) return false;
  return true;
}

/* Squared distance written the same way everywhere a contact decision is taken. */
__device__ __forceinline__ float dist2(float ax, float ay, float az, float px, float py,
                                       float pz) {
  const float dx = __fsub_rn(ax, px), dy = __fsub_rn(ay, py), dz = __fsub_rn(az, pz);
  return __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
}

/* hpc switching polynomial 1 - (3.5 u/81 - 4.5 u^2/81^2 + 2.5 u^3/81^3 - 0.5 u^4/81^4), u = d^2 */
#define HPC_C1 (3.5f / 81.0f)
#define HPC_C2 (4.5f / 6561.0f)
#define HPC_C3 (2.5f / 531441.0f)
#define HPC_C4 (0.5f / 43046721.0f)
#define LOG2E_F 1.4426950408889634f

struct Acc {
  float2 vdw, ele, pmf, hdb;
};

/* Per-segment pair parameters, splatted over the two lanes of an FP32x2 register pair. */
struct Pair2 {
  float2 p1a, mp2a, p1l, p1ll, b2, c2, hc1, hc0, hs;
};

__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }

/* One pair of protein slots (2m, 2m+1) against the lane's atom: the terms every pair has
 * (vdw, the far form of ele, pmf; hdb on segments whose type has a live hydrogen-bond pair).
 * The short-range terms (contacts, psp, hpc, the electrostatic soft core) come from the cell
 * list pass, short_range(). PAIR = false: only the first slot is a point (the second is
 * segment padding) and nothing of the second is kept. FAR: both points lie beyond the atom's
 * far radius, where the pmf exponent is below -25.5 in base 2 (the host's radius has a margin
 * of 0.5 over the FP32 rounding of tt). There ee < 2^-25, so p4 + p4 ee rounds to p4 and
 * num + num ee to num: the full body's terms are num rcp(p4) and p4 rcp(p4), which the far
 * form computes without tt, ee, pd and vn, bit for bit; where a warp splits a segment into
 * its near and far parts therefore changes no result. */
template <bool HDB, bool PAIR, bool FAR>
__device__ __forceinline__ void pair_body(const float4 A, const float4 B, float2 ax, float2 ay,
                                          float2 az, const Pair2 &q, const GdForceConst &f,
                                          Acc &a) {
  const float2 one = f2(1.0f);
  /* squared distance, per lane exactly dist2(): a + (-p) == a - p */
  const float2 dx = __fadd2_rn(ax, make_float2(A.x, A.y));
  const float2 dy = __fadd2_rn(ay, make_float2(A.z, A.w));
  const float2 dz = __fadd2_rn(az, make_float2(B.x, B.y));
  const float2 d2 = __ffma2_rn(dz, dz, __ffma2_rn(dy, dy, __fmul2_rn(dx, dx)));
  const float2 ri = make_float2(rsqrt_a(d2.x), rsqrt_a(d2.y));
  /* vdw: (p1 - p2) / (p1 lj0 (1 + lj1 d2) + 1), p1 = p1a r^-9, p2 = p2a r^-6; the
   * denominator is (p1l + p1ll d2) r^-9 + 1 with p1l = p1a lj0, p1ll = p1l lj1 */
  const float2 r2i = __fmul2_rn(ri, ri);
  const float2 r3i = __fmul2_rn(r2i, ri);
  const float2 r6i = __fmul2_rn(r3i, r3i);
  const float2 num = __fmul2_rn(r6i, __ffma2_rn(q.p1a, r3i, q.mp2a));
  const float2 p4 = __ffma2_rn(__ffma2_rn(q.p1ll, d2, q.p1l), __fmul2_rn(r6i, r3i), one);
  /* ele: q_l ele_p g(el1 r), q_l applied once per atom. The points hold ele_p / el1, so the
   * far form g = 1 / (el1 r) is one FMA with r^-1; pairs inside r < 1 / el1 get the soft-core
   * difference in short_range() */
  const float2 ep = make_float2(B.z, B.w);
  if constexpr (PAIR) {
    a.ele = __ffma2_rn(ep, ri, a.ele);
  } else {
    a.ele.x = __fmaf_rn(ep.x, ri.x, a.ele.x);
  }
  if constexpr (FAR) {
    const float2 inv = make_float2(rcp_a(p4.x), rcp_a(p4.y));
    if constexpr (PAIR) {
      a.vdw = __ffma2_rn(num, inv, a.vdw);
      a.pmf = __ffma2_rn(p4, inv, a.pmf);
    } else {
      a.vdw.x = __fmaf_rn(num.x, inv.x, a.vdw.x);
      a.pmf.x = __fmaf_rn(p4.x, inv.x, a.pmf.x);
    }
  } else {
  /* pmf: pmf1 / (1 + exp((6 - r/2)(r - pmf0))) as exp2 of the expanded quadratic
   * cA d2 + b2 r + c2 = d2 (b2 r^-1 + cA) + c2 (cA = -log2(e)/2, b2 = log2(e)(6 + pmf0/2),
   * c2 = -6 log2(e) pmf0). Its maximum over r is log2(e) (12 - pmf0)^2 / 8 < 100 for
   * pmf0 > -10 (checked when the force field is loaded), so den stays finite and p4 den does
   * wherever p4 does. */
  const float2 tt = __ffma2_rn(d2, __ffma2_rn(q.b2, ri, f2(-0.5f * LOG2E_F)), q.c2);
  const float2 ee = make_float2(ex2_a(tt.x), ex2_a(tt.y));
  /* one reciprocal for both quotients, den = 1 + ee: num / p4 = num den / (p4 den),
   * 1 / den = p4 / (p4 den), with p4 den = p4 + p4 ee and num den = num + num ee; the
   * segment's pmf1 multiplies the pmf sum when it is folded */
  const float2 pd = __ffma2_rn(p4, ee, p4);
  const float2 inv = make_float2(rcp_a(pd.x), rcp_a(pd.y));
  const float2 vn = __ffma2_rn(num, ee, num);
  if constexpr (PAIR) {
    a.vdw = __ffma2_rn(vn, inv, a.vdw);
    a.pmf = __ffma2_rn(p4, inv, a.pmf);
  } else {
    a.vdw.x = __fmaf_rn(vn.x, inv.x, a.vdw.x);
    a.pmf.x = __fmaf_rn(p4.x, inv.x, a.pmf.x);
  }
  }
  if (HDB) {
    const float2 h = __ffma2_rn(__fmul2_rn(d2, ri), q.hc1, q.hc0);
    const float2 hh = __fmul2_rn(h, h);
    if constexpr (PAIR)
      a.hdb = __ffma2_rn(q.hs, make_float2(ex2_a(-hh.x), ex2_a(-hh.y)), a.hdb);
    else
      a.hdb.x = __fmaf_rn(q.hs.x, ex2_a(-hh.x), a.hdb.x);
  }
}

/* Pair loop over slots [i0, i1) of one point-type segment held in shared memory; i0 is even,
 * an odd i1 leaves one point for a half iteration. HDB: the segment's point type has a live
 * hydrogen-bond pair with some atom type of the ligand (decided per complex on the host, so
 * every warp of the CTA runs the same code). UNROLL: point pairs in flight per lane. */
template <bool HDB, int UNROLL, bool FAR>
__device__ __forceinline__ void pair_range(const float4 *__restrict__ PA,
                                           const float4 *__restrict__ PB, int i0, int i1,
                                           float ax, float ay, float az, const Pair2 &q,
                                           const GdForceConst &f, Acc &a) {
  const float2 ax2 = f2(ax), ay2 = f2(ay), az2 = f2(az);
  const int m0 = i0 >> 1, m1 = i1 >> 1;
#pragma unroll UNROLL
  for (int m = m0; m < m1; ++m)
    pair_body<HDB, true, FAR>(PA[m], PB[m], ax2, ay2, az2, q, f, a);
  if (i1 & 1) pair_body<HDB, false, FAR>(PA[m1], PB[m1], ax2, ay2, az2, q, f, a);
}

/* Pair loop of one of the S lanes of an atom (split sp) over slots [i0, i1) of a segment:
 * every S-th point pair from pair i0 / 2 + sp, the pairs before slot im (even, or i1) in the
 * full form and the rest in the far form; the odd tail point goes to the lane whose turn it
 * is. Each lane's pairs and their order do not depend on im, and the two forms give the same
 * result on far pairs, so neither does its sum. */
template <bool HDB, int UNROLL>
__device__ __forceinline__ void pair_range_split(const float4 *__restrict__ PA,
                                                 const float4 *__restrict__ PB, int i0, int im,
                                                 int i1, int sp, int S, float ax, float ay,
                                                 float az, const Pair2 &q,
                                                 const GdForceConst &f, Acc &a) {
  const float2 ax2 = f2(ax), ay2 = f2(ay), az2 = f2(az);
  const int mm = im >> 1, m1 = i1 >> 1;
  int m = (i0 >> 1) + sp;
#pragma unroll UNROLL
  for (; m < mm; m += S) pair_body<HDB, true, false>(PA[m], PB[m], ax2, ay2, az2, q, f, a);
#pragma unroll UNROLL
  for (; m < m1; m += S) pair_body<HDB, true, true>(PA[m], PB[m], ax2, ay2, az2, q, f, a);
  if ((i1 & 1) && m == m1) {
    if (2 * m1 >= im)
      pair_body<HDB, false, true>(PA[m1], PB[m1], ax2, ay2, az2, q, f, a);
    else
      pair_body<HDB, false, false>(PA[m1], PB[m1], ax2, ay2, az2, q, f, a);
  }
}

/* The same range for the same atom of two replicas (the lane's two slots): one load of each
 * point pair, one loop, the segment's parameters shared; each atom's sums are the operations
 * of pair_range in the same order, so its energies are bit-identical. */
template <bool HDB, int UNROLL, bool FAR>
__device__ __forceinline__ void pair_range2(const float4 *__restrict__ PA,
                                            const float4 *__restrict__ PB, int i0, int i1,
                                            const float *ax, const float *ay, const float *az,
                                            const Pair2 &q, const GdForceConst &f, Acc *a) {
  const float2 ax0 = f2(ax[0]), ay0 = f2(ay[0]), az0 = f2(az[0]);
  const float2 ax1 = f2(ax[1]), ay1 = f2(ay[1]), az1 = f2(az[1]);
  const int m0 = i0 >> 1, m1 = i1 >> 1;
#pragma unroll UNROLL
  for (int m = m0; m < m1; ++m) {
    const float4 A = PA[m], B = PB[m];
    pair_body<HDB, true, FAR>(A, B, ax0, ay0, az0, q, f, a[0]);
    pair_body<HDB, true, FAR>(A, B, ax1, ay1, az1, q, f, a[1]);
  }
  if (i1 & 1) {
    const float4 A = PA[m1], B = PB[m1];
    pair_body<HDB, false, FAR>(A, B, ax0, ay0, az0, q, f, a[0]);
    pair_body<HDB, false, FAR>(A, B, ax1, ay1, az1, q, f, a[1]);
  }
}

/* Sums of the short-range terms of one atom. */
struct ShortSums {
  double hsum;                /* sum of hpp * switch(d^2) over hydrophobic points, d^2 <= 81 */
  float psp;                  /* sum of the PSP entries of class-2 points in contact */
  float ele;                  /* soft-core minus far-form electrostatics, d^2 < (1 / el1)^2 */
  int ncon;                   /* contacts: d^2 <= the pair's contact threshold */
};

/* The terms of CalcEnergy_d that only pairs within a few angstrom have (contacts for mcc and
 * psp, hpc's switching polynomial, the soft core of ele), for one atom at (ax, ay, az), from
 * the conformer's cell list: the rows of cells (fixed y, z) that reach within sr_r of the
 * atom, each over the x range the remaining radius allows, so every point with
 * d^2 <= sr_r2 is visited once and the tests use the same d^2 as the pair loop. The next
 * row's bounds are read while the current row runs. thr: the contact thresholds of the atom's
 * type against every point type (shared memory). */
__device__ __forceinline__ void short_range(const GdDevComplex &cx, int pc,
                                            const float *__restrict__ thr,
                                            const float *__restrict__ psprow,
                                            const GdForceConst &f, float ax, float ay, float az,
                                            int part, int parts, ShortSums &s) {
  s.hsum = 0.0;
  s.psp = 0.0f;
  s.ele = 0.0f;
  s.ncon = 0;
  const int nx = cx.sr_n[0], ny = cx.sr_n[1], nz = cx.sr_n[2];
  const float R = cx.sr_r, R2 = cx.sr_r * cx.sr_r, ic = cx.sr_inv_cell, e = cx.sr_cell;
  const float r2max = cx.sr_r2;
  const float ox = cx.sr_org[0], oy = cx.sr_org[1], oz = cx.sr_org[2];
  const int y0 = max(0, (int)floorf((ay - R - oy) * ic));
  const int y1 = min(ny - 1, (int)floorf((ay + R - oy) * ic));
  const int z0 = max(0, (int)floorf((az - R - oz) * ic));
  const int z1 = min(nz - 1, (int)floorf((az + R - oz) * ic));
  if (y0 > y1 || z0 > z1) return;
  const int *__restrict__ st = cx.sr_start + (size_t)pc * (cx.sr_n[3] + 1);
  const float4 *__restrict__ PA = cx.sr_a + (size_t)pc * cx.pnp;
  const float4 *__restrict__ PB = cx.sr_b + (size_t)pc * cx.pnp;
  /* point range of row (iy, iz) within the remaining radius; empty when out of reach */
  auto bounds = [&](int iy, int iz, int &b0, int &b1) {
    b0 = b1 = 0;
    const float zl = oz + (float)iz * e, yl = oy + (float)iy * e;
    const float gz = fmaxf(0.0f, fmaxf(zl - az, az - (zl + e)));
    const float gy = fmaxf(0.0f, fmaxf(yl - ay, ay - (yl + e)));
    const float rem = R2 - gy * gy - gz * gz;
    if (rem < 0.0f) return;
    const float hx = sqrtf(rem);
    const int x0 = max(0, (int)floorf((ax - hx - ox) * ic));
    const int x1 = min(nx - 1, (int)floorf((ax + hx - ox) * ic));
    if (x0 > x1) return;
    const int row = (iz * ny + iy) * nx;
    b0 = __ldg(st + row + x0);
    b1 = __ldg(st + row + x1 + 1);
  };
  /* rows part, part + parts, ... of the (iy, iz) order: the lanes of a split atom share them */
  const int ny_span = y1 - y0 + 1;
  int iy = y0 + part, iz = z0, n0 = 0, n1 = 0;
  while (iy > y1) {
    iy -= ny_span;
    ++iz;
  }
  bool more = iz <= z1;
  if (more) bounds(iy, iz, n0, n1);
  while (more) {
    const int c0 = n0, c1 = n1;
    iy += parts;
    while (iy > y1) {
      iy -= ny_span;
      ++iz;
    }
    more = iz <= z1;
    if (more) bounds(iy, iz, n0, n1);
    for (int i = c0; i < c1; ++i) {
      const float4 p = __ldg(PA + i);
      const float d2 = dist2(ax, ay, az, p.x, p.y, p.z);
      if (d2 > r2max) continue;
      const int meta = __float_as_int(p.w);
      const bool hpc = (meta & 256) && d2 <= 81.0f;
      const bool con = d2 <= thr[meta & 255];
      const bool cls2 = con && (meta & 512);
      const bool near = d2 < f.near2;
      s.ncon += con ? 1 : 0;
      if (hpc || cls2 || near) {
        const float4 b = __ldg(PB + i);
        if (hpc) {
          float t = __fmaf_rn(d2, HPC_C4, -HPC_C3);
          t = __fmaf_rn(d2, t, HPC_C2);
          t = __fmaf_rn(d2, t, -HPC_C1);
          s.hsum += (double)__fmul_rn(b.x, __fmaf_rn(d2, t, 1.0f));
        }
        if (cls2) s.psp += __ldg(psprow + __float_as_int(b.y));
        if (near) {
          const float ri = rsqrt_a(d2);
          const float s1 = __fmul_rn(f.el1, __fmul_rn(d2, ri));
          const float gn = __fmaf_rn(__fmul_rn(s1, s1), __fmaf_rn(f.b1, s1, f.a1), f.el0);
          /* ep (el1 gn) - ep ri = ele_p gn - ele_p g_far */
          s.ele += __fmaf_rn(b.z * f.el1, gn, -(b.z * ri));
        }
      }
    }
  }
}

/* Per-replica state of the CTA's slots, in shared memory. */
struct Slot {
  int rep, lig_conf, accept, n_acc;
  int rec_next, pad0;
  float mb, u;
  float mm_old[6];
  float mm_new[6];
  float rot[9];
  float tx, ty, tz;
  gd_energy e_old;
  gd_replica replica;
};
static_assert(sizeof(Slot) == GD_SLOT_BYTES, "slot layout");

/* deterministic warp sum of a double */
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

#define NQ 10 /* vdw ele pmf psp hdb hsum->hpc kde rmsd ncon tp */

/* One segment range of the pair loop, dispatched on the segment's flags (bit 2: live
 * hydrogen-bond term). */
template <int UNROLL, int PACK, bool FAR>
__device__ __forceinline__ void pair_dispatch(int flags, const float4 *PA, const float4 *PB,
                                              int i0, int i1, const float *ax, const float *ay,
                                              const float *az, const Pair2 &pq,
                                              const GdForceConst &f, Acc *acc) {
#define GD_PR(H)                                                                             \
  if constexpr (PACK == 2)                                                                   \
    pair_range2<H, UNROLL, FAR>(PA, PB, i0, i1, ax, ay, az, pq, f, acc);                     \
  else                                                                                       \
    pair_range<H, UNROLL, FAR>(PA, PB, i0, i1, ax[0], ay[0], az[0], pq, f, acc[0])
  if (flags & 4) {
    GD_PR(true);
  } else {
    GD_PR(false);
  }
#undef GD_PR
}

/* ExchangeReplicas_d (src/kernel_cuda_l1_exchangereplicas.cu:27-77) for one (protein
 * conformer, ligand conformer) group lg of complex cx: temperature pairs (2 j + mode_t, its
 * successor), accepted by the Metropolis test on their energies with one Philox draw per pair
 * of this exchange call. The group's replica states are read with L2 loads (.cg): inside the
 * Monte Carlo kernel other SMs wrote them in this launch. */
__device__ __forceinline__ void gd_exchange_group(const GdDevComplex &cx, int lg,
                                                  gd_replica *replica, const float *etotal,
                                                  int *acs, uint64_t seed, int call, int mode_t) {
  if (mode_t >= 2) return;
  const int nl = cx.n_lig, nt = cx.n_tmp;
  const int p = lg / nl, l = lg - p * nl;
  int temps[GD_MAXTMP], orders[GD_MAXTMP];
  float en[GD_MAXTMP];
  for (int t = 0; t < nt; ++t) {
    const int f = cx.rep_offset + nt * nl * p + nl * t + l;
    temps[t] = __ldcg(&replica[f].idx_tmp);
    en[t] = __ldcg(etotal + f);
    orders[temps[t]] = t;
  }
  const int maxpair = nt / 2 - (nt % 2 == 0) * (mode_t == 1);
  for (int pair = 0; pair < maxpair; ++pair) {
    const int i1 = (pair << 1) + mode_t, i2 = i1 + 1;
    const int o1 = orders[i1], o2 = orders[i2];
    const int tt = temps[o1];
    const float mb1 = cx.minus_beta[temps[o1]], mb2 = cx.minus_beta[temps[o2]];
    const float u = gd_draw_exchange(seed, (uint32_t)cx.stream, (uint32_t)lg, (uint32_t)call,
                                     (uint32_t)pair);
    if (gd_exchange_accept(en[o1], en[o2], mb1, mb2, u)) {
      temps[o1] = temps[o2];
      temps[o2] = tt;
      acs[cx.rep_offset + nt * nl * p + nl * o1 + l] += 1;
      acs[cx.rep_offset + nt * nl * p + nl * o2 + l] += 1;
    }
  }
  for (int t = 0; t < nt; ++t) replica[cx.rep_offset + nt * nl * p + nl * t + l].idx_tmp = temps[t];
}

/* Delayed acceptance, second stage, for the survivor in pose slot `pos` (mode 3): the
 * corrected Metropolis test u2 < exp(mb ((E_new - E_old) - (S_new - S_cur))) (gd_da_stage2),
 * surrogate-error sums, the collect step's training target, the trace, and on acceptance the
 * state update and the record, as the plain epilogue does them. */
__device__ __forceinline__ void da_decide(const GdMcArgs &a, const GdDevComplex &cx, int ci, int pos,
                                       const gd_energy &en, const float *mm_new, int step) {
  const GdDaEpi &da = *a.da;
  const int r = da.pose_rep[pos];
  const gd_replica rp = a.replica[r];
  const float mb = cx.minus_beta[rp.idx_tmp];
  const float enew = en.e[GD_MAXWEI - 1];
  const float sn = da.s_new[r], so = da.s_cur[r];
  const int acc = gd_da_stage2(enew, a.e_old[r].e[GD_MAXWEI - 1], sn, so, mb, da.u2[r]);
  const bool active = !a.da_collect && da.active[ci];
  if (active) {
    const double e = (double)sn - (double)enew;
    da.err2[r] += e * e;
    da.nerr[r] += 1;
  }
  if (a.da_collect && da.smp_cap > 0)
    da.smp_t[((long long)step * da.n_rep + r) % da.smp_cap] = enew;
  if (da.tr_flag) {
    const int ti = step - da.tr_step0;
    if (ti >= 0 && ti < da.tr_cap) {
      const size_t o = (size_t)r * da.tr_cap + ti;
      da.tr_s[o] = sn;
      da.tr_e[o] = enew;
      da.tr_flag[o] = 1 + acc;
    }
  }
  if (!acc) return;
  a.e_old[r] = en;
  a.etotal[r] = enew;
#pragma unroll
  for (int i = 0; i < 6; ++i) a.mm_old[(size_t)r * 6 + i] = mm_new[i];
  a.n_accept[r] += 1;
  da.s_cur[r] = sn;
  if (active) da.acc[r] += 1; else da.plain_acc[r] += 1;
  if (a.rec) {
    const int kslot = a.rec_next[r];
    if (kslot < a.rec_cap) {
      gd_record_step *q = a.rec + (size_t)r * a.rec_cap + kslot;
      q->replica = rp;
      q->energy = en;
#pragma unroll
      for (int i = 0; i < 6; ++i) q->movematrix[i] = mm_new[i];
      q->step = step;
      a.rec_next[r] = kslot + 1;
    } else {
      atomicOr(a.err, GD_DEV_ERR_RECORD_FULL);
    }
  }
}

/*
 * Shared memory: two mbarriers, two protein buffers of D points (float4 + float2), the
 * placed atoms, NQ FP64 partials per lane, the slots. The protein buffers form a two-stage
 * ring without CTA barriers: every warp waits on the buffer's "full" mbarrier by itself and,
 * when done, bumps the buffer's counter; the last warp to finish refills the buffer with the
 * chunk two ahead. Every wait is bounded (globaltimer); a wait that runs out sets the error
 * word, the CTA leaves at the next step barrier after letting its copies in flight land.
 */
template <int UNROLL, bool SPLIT, bool DA, int PACK>
__global__ void __launch_bounds__(GD_MAX_TPB / PACK, GD_MIN_BLOCKS_PACK(UNROLL, PACK, DA))
    gd_mc_kernel(GdMcArgs a, GdForceConst f) {
  static_assert(PACK == 1 || (PACK == 2 && !SPLIT && !DA),
                "two replicas per lane: plain modes with one lane per atom");
  extern __shared__ __align__(16) unsigned char smem[];
  /* T: lanes of the tile (PACK per thread), the stride of the placed atoms and partials */
  const int NT = blockDim.x, T = NT * PACK, tid = threadIdx.x, D = a.chunk;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
  /* contact thresholds [ligand type][point type], then the ring buffers: buffer b holds D
   * slots as D/2 pairs in two float4 streams */
  float *thr_s = reinterpret_cast<float *>(smem + 16);
  float4 *bpa = reinterpret_cast<float4 *>(smem + 16 + GD_THR_BYTES);
  float4 *bpb = bpa + D;
  float4 *atoms = bpb + D;
  double *part = reinterpret_cast<double *>(atoms + T);
  Slot *slots = reinterpret_cast<Slot *>(part + NQ * T);
  __shared__ int s_tile, s_abort;
  __shared__ int s_done[2];
  __shared__ unsigned s_issued[2];

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
    s_done[0] = s_done[1] = 0;
    s_issued[0] = s_issued[1] = 0;
  }
  for (int i = tid; i < GD_MAXTP2 * GD_MAXTP1; i += NT) thr_s[i] = a.pp[i].thr;
  __syncthreads();
  uint32_t consumed0 = 0, consumed1 = 0; /* completed phases waited for, per buffer */
  const int step_first = a.step0 + (a.step_base ? *a.step_base : 0);
  const int warp = tid >> 5, lane = tid & 31, nwarps = NT >> 5;
  if (DA && a.mode == 3 && blockIdx.x == 0)
    for (int g = a.da_g0 + tid; g < a.da_g1; g += NT) a.da_cnt_next[g] = 0;

  for (;;) {
    if (tid == 0) s_tile = atomicAdd(a.tile_counter, 1);
    __syncthreads();
    const int t = s_tile;
    if (t >= a.n_tiles || s_abort) break;
    const GdTileDesc tile = a.tiles[t];
    int k = tile.count;
    if (DA && a.mode == 3) {
      /* slot (group, capacity): the survivors of the group past this tile's first slot */
      const int g = tile.count >> 8, cap = tile.count & 255;
      k = max(0, min(cap, a.da_cnt[g] - (tile.rep_begin - a.da->group_b0[g])));
    }
    if (k <= 0) {
      /* an empty tile (a delayed-acceptance block with fewer survivors than tiles): no copy
       * issued, nothing to wait for; the barrier keeps s_tile until every thread read it */
      __syncthreads();
      continue;
    }
    const GdDevComplex &cx = a.cx[tile.complex_index];
    /* lane = (slot j, protein split sp, ligand atom l): the S copies of an atom each take
     * every S-th point pair of every protein segment; S = 1 is one lane per atom */
    const int L = cx.lna, S = SPLIT ? a.split : 1, SL = S * L;
    const int kp = (k + PACK - 1) / PACK; /* lane groups */
    const bool active = tid < kp * SL;
    const int jj = active ? tid / SL : 0;
    const int sp = active ? (tid - jj * SL) / L : 0;
    const int l = active ? tid - jj * SL - sp * L : 0;
    /* the thread's lanes: slot jj (PACK 1), or slots 2 jj and 2 jj + 1, the same atom of two
     * replicas (PACK 2); a missing second slot (odd k) repeats the first one's atom and stores
     * nothing. sl_of: each lane's slot; vl: its index in the placed-atom and partial arrays */
    int sl_of[PACK], vl[PACK];
    bool ok[PACK];
#pragma unroll
    for (int h = 0; h < PACK; ++h) {
      const int jh = jj * PACK + h;
      ok[h] = active && jh < k;
      sl_of[h] = ok[h] ? jh : jj * PACK;
      vl[h] = sl_of[h] * SL + sp * L + l;
    }

    /* ---- slot set-up (one thread per replica) ---- */
    if (tid < k) {
      Slot &s = slots[tid];
      const int id = tile.rep_begin + tid;
      s.rep = id;
      s.accept = 0;
      if (a.mode >= 2) {
        s.lig_conf = a.lig_conf_in[id];
      } else {
        s.replica = a.replica[id];
        s.lig_conf = s.replica.idx_lig;
        s.mb = cx.minus_beta[s.replica.idx_tmp];
        if (a.mode == 0) {
          s.e_old = a.e_old[id];
          s.n_acc = a.n_accept[id];
          s.rec_next = a.rec ? a.rec_next[id] : 0;
#pragma unroll
          for (int i = 0; i < 6; ++i) s.mm_old[i] = a.mm_old[(size_t)id * 6 + i];
        } else {
          s.n_acc = 0;
          s.rec_next = 0;
#pragma unroll
          for (int i = 0; i < 6; ++i) s.mm_old[i] = 0.0f;
        }
      }
    }

    /* ---- protein tile pipeline ---- */
    const int pc = tile.prt_conf;
    const size_t pbase = (size_t)pc * (cx.pnp_pad >> 1);
    const float4 *ga = cx.pt_a + pbase, *gb = cx.pt_b + pbase;
    const int P = cx.pnp, pnp_pad = cx.pnp_pad;
    const int nch = (pnp_pad + D - 1) / D;
    const bool resident = nch <= 2;
    const int nsteps = a.mode == 0 ? a.n_steps : 1;
    const int total_q = resident ? nch : nsteps * nch;
    if (tid == 0) {
      s_done[0] = s_done[1] = 0;
      for (int q = 0; q < min(2, total_q); ++q) {
        const int b = q & 1, c0 = q * D, n = min(D, pnp_pad - c0);
        s_issued[b] += 1;
        mbar_expect_tx(&bar[b], (uint32_t)(n * 16));
        bulk_g2s(bpa + b * (D >> 1), ga + (c0 >> 1), (uint32_t)(n * 8), &bar[b]);
        bulk_g2s(bpb + b * (D >> 1), gb + (c0 >> 1), (uint32_t)(n * 8), &bar[b]);
      }
    }
    __syncthreads();

    /* ---- per-lane constants ---- */
    float4 orig[PACK];
#pragma unroll
    for (int h = 0; h < PACK; ++h) orig[h] = cx.lig_pos[slots[sl_of[h]].lig_conf * L + l];
    /* atom types are the same in every conformer of a ligand when PACK is 2 (host-checked) */
    const int tl = cx.lig_meta[slots[sl_of[0]].lig_conf * L + l].x;
    const float *psprow = cx.psp + (size_t)tl * cx.psp_ld;
    const GdPairParam *pprow = a.pp + tl * GD_MAXTP1;
    const int4 *segs = cx.seg + pc * GD_MAX_SEG;
    const int nseg = cx.seg_count[pc];
    bool aborted = false;

    for (int s = 0; s < nsteps; ++s) {
      /* ---- Move_d: one thread per replica draws the move and builds the rotation ---- */
      if (tid < k) {
        Slot &sl = slots[tid];
        float mmn[6], u = 0.0f;
        if (a.mode == 0) {
          float delta[6];
          gd_draw_step(a.seed, (uint32_t)cx.stream, (uint32_t)(sl.rep - cx.rep_offset),
                       (uint32_t)(step_first + s), a.move_kind, a.move_scale, delta, &u);
#pragma unroll
          for (int i = 0; i < 6; ++i) mmn[i] = GD_ADD(sl.mm_old[i], delta[i]);
        } else if (a.mode == 2 || a.mode == 3) {
#pragma unroll
          for (int i = 0; i < 6; ++i) mmn[i] = a.mm_in[(size_t)sl.rep * 6 + i];
        } else {
#pragma unroll
          for (int i = 0; i < 6; ++i) mmn[i] = 0.0f;
        }
        float rot[9];
        gd_rotation(mmn, rot);
#pragma unroll
        for (int i = 0; i < 9; ++i) sl.rot[i] = rot[i];
#pragma unroll
        for (int i = 0; i < 6; ++i) sl.mm_new[i] = mmn[i];
        const float *lc = cx.lig_center + sl.lig_conf * 3;
        sl.tx = GD_ADD(mmn[0], lc[0]);
        sl.ty = GD_ADD(mmn[1], lc[1]);
        sl.tz = GD_ADD(mmn[2], lc[2]);
        if (a.mode == 4) {
          /* given coordinates: the ligand centre comes with them (Ligand.coord_new.center) */
          sl.tx = a.center_in[(size_t)sl.rep * 3];
          sl.ty = a.center_in[(size_t)sl.rep * 3 + 1];
          sl.tz = a.center_in[(size_t)sl.rep * 3 + 2];
        }
        sl.u = u;
      }
      __syncthreads();
      float ax[PACK], ay[PACK], az[PACK];
#pragma unroll
      for (int h = 0; h < PACK; ++h) {
        ax[h] = ay[h] = az[h] = 0.0f;
        if (active) {
          const Slot &sl = slots[sl_of[h]];
          if (a.mode == 4) {
            const float *p = a.xyz_in + ((size_t)sl.rep * L + l) * 3;
            ax[h] = p[0];
            ay[h] = p[1];
            az[h] = p[2];
          } else {
            gd_place_atom(sl.rot, sl.tx, sl.ty, sl.tz, orig[h].x, orig[h].y, orig[h].z, &ax[h],
                          &ay[h], &az[h]);
          }
          if (ok[h]) atoms[vl[h]] = make_float4(ax[h], ay[h], az[h], 0.0f);
        }
      }
      /* each lane clears its own partials (the only ones the epilogue reads) */
#pragma unroll
      for (int h = 0; h < PACK; ++h)
        if (ok[h])
#pragma unroll
          for (int qi = 0; qi < NQ; ++qi) part[qi * T + vl[h]] = 0.0;

      /* ---- short-range terms from the cell list (the S lanes of an atom take every S-th row
       * of its walk), before the pair loop: warps whose walk is short start the loop while
       * the others still walk ---- */
#pragma unroll
      for (int h = 0; h < PACK; ++h) {
        if (!ok[h]) continue;
        ShortSums sr;
        short_range(cx, pc, thr_s + tl * GD_MAXTP1, psprow, f, ax[h], ay[h], az[h], sp, S, sr);
        const int v = vl[h];
        part[1 * T + v] = (double)sr.ele;
        part[3 * T + v] = (double)sr.psp;
        part[5 * T + v] = sr.hsum;
        part[8 * T + v] = (double)sr.ncon;
      }

      /* ---- far-point bin of the warp: a point further from the pocket centre than far_r +
       * the largest distance of the warp's atoms from it is beyond far_r of each of them, and
       * takes the far form of the pair body (the same result, fewer operations) ---- */
      int fbin = 0;
#pragma unroll
      for (int h = 0; h < PACK; ++h) {
        if (!ok[h]) continue;
        const float dx = ax[h] - cx.pocket[0], dy = ay[h] - cx.pocket[1],
                    dz = az[h] - cx.pocket[2];
        const float rho = sqrtf(dx * dx + dy * dy + dz * dz) + cx.far_r;
        fbin = max(fbin, (int)fminf(rho * cx.far_inv_w, (float)(GD_FAR_BINS - 1)));
      }
      fbin = (int)__reduce_max_sync(0xffffffffu, (unsigned)fbin);
      const unsigned short *fcnt = cx.far_cnt + (size_t)pc * GD_MAX_SEG * GD_FAR_BINS + fbin;

      /* ---- CalcEnergy_d pair loop over the protein ring ---- */
      for (int ci = 0; ci < nch; ++ci) {
        const int q = resident ? ci : s * nch + ci;
        const int b = q & 1;
        if (!resident || s == 0) {
          bool ok = !*(volatile int *)&s_abort;
          if (ok) ok = mbar_wait_bounded(&bar[b], b ? (consumed1 & 1u) : (consumed0 & 1u),
                                         a.timeout_ns);
          if (!ok) {
            aborted = true;
            if (lane == 0) { s_abort = 1; atomicOr(a.err, GD_DEV_ERR_TIMEOUT); }
            break;
          }
          if (b) ++consumed1; else ++consumed0;
        }
        if (active) {
          const float4 *PA = bpa + b * (D >> 1); /* local slot = slot - c0 */
          const float4 *PB = bpb + b * (D >> 1);
          const int c0 = ci * D, c1 = min(pnp_pad, c0 + D);
          for (int sg = 0; sg < nseg; ++sg) {
            const int4 g = segs[sg];
            const int i0 = max(g.x, c0) - c0, i1 = min(g.y, c1) - c0;
            if (i0 >= i1) continue;
            const float4 *pr = reinterpret_cast<const float4 *>(pprow + g.z);
            const float4 q0 = __ldg(pr), q1 = __ldg(pr + 1), q2 = __ldg(pr + 2);
            Pair2 pq;
            pq.p1a = f2(q0.x); pq.mp2a = f2(-q0.y); pq.p1l = f2(q0.z);
            pq.p1ll = f2(q0.z * f.lj1); pq.hc1 = f2(q1.z); pq.hc0 = f2(q1.w);
            pq.hs = f2(q2.x); pq.b2 = f2(q2.z); pq.c2 = f2(q2.w);
            const float2 z2 = f2(0.0f);
            Acc acc[PACK];
#pragma unroll
            for (int h = 0; h < PACK; ++h) acc[h] = {z2, z2, z2, z2};
            /* the segment's near points [i0, im) and far points [im, i1); the split slot is
             * even (the segment starts on one), so the near part keeps whole slot pairs */
            const int fs = g.x + ((__ldg(fcnt + sg * GD_FAR_BINS) + 1) & ~1) - c0;
            const int im = min(i1, max(i0, fs));
            if constexpr (SPLIT) {
              /* the S lanes of an atom take every S-th point pair of the range */
              if (g.w & 4)
                pair_range_split<true, UNROLL>(PA, PB, i0, im, i1, sp, S, ax[0], ay[0], az[0],
                                               pq, f, acc[0]);
              else
                pair_range_split<false, UNROLL>(PA, PB, i0, im, i1, sp, S, ax[0], ay[0], az[0],
                                                pq, f, acc[0]);
            } else {
              if (i0 < im)
                pair_dispatch<UNROLL, PACK, false>(g.w, PA, PB, i0, im, ax, ay, az, pq, f, acc);
              if (im < i1)
                pair_dispatch<UNROLL, PACK, true>(g.w, PA, PB, im, i1, ax, ay, az, pq, f, acc);
            }
#pragma unroll
            for (int h = 0; h < PACK; ++h) {
              if (!ok[h]) continue;
              const int v = vl[h];
              part[0 * T + v] += (double)acc[h].vdw.x + (double)acc[h].vdw.y;
              part[1 * T + v] += (double)acc[h].ele.x + (double)acc[h].ele.y;
              part[2 * T + v] += (double)q1.y * ((double)acc[h].pmf.x + (double)acc[h].pmf.y);
              part[4 * T + v] += (double)acc[h].hdb.x + (double)acc[h].hdb.y;
            }
          }
        }
        if (!resident) {
          /* the last warp done with buffer b refills it with chunk q + 2 */
          __syncwarp();
          if (lane == 0) {
            __threadfence_block();
            const int prev = atomicAdd(&s_done[b], 1);
            if (prev == nwarps - 1) {
              s_done[b] = 0;
              if (q + 2 < total_q) {
                const int c0 = ((q + 2) % nch) * D, n = min(D, pnp_pad - c0);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                s_issued[b] += 1;
                mbar_expect_tx(&bar[b], (uint32_t)(n * 16));
                bulk_g2s(bpa + b * (D >> 1), ga + (c0 >> 1), (uint32_t)(n * 8), &bar[b]);
                bulk_g2s(bpb + b * (D >> 1), gb + (c0 >> 1), (uint32_t)(n * 8), &bar[b]);
              }
            }
          }
        }
      }

      /* ---- per-atom tail (split 0 of each atom): hpc, kde, rmsd, reference contacts ---- */
      if (S > 1) {
        /* hpc is nonlinear in the atom's hydrophobic sum: gather the splits' parts first */
        __syncthreads();
        if (ok[0] && sp == 0)
          for (int q = 1; q < S; ++q) {
            part[5 * T + vl[0]] += part[5 * T + vl[0] + q * L];
            part[5 * T + vl[0] + q * L] = 0.0;
          }
      }
#pragma unroll
      for (int h = 0; h < PACK; ++h) {
        if (!ok[h] || aborted) continue;
        const int v = vl[h];
        part[1 * T + v] *= (double)orig[h].w;
        if (sp != 0) continue;
        const double hpc2 = (part[5 * T + v] - (double)f.hpl0[tl]) / (double)f.hpl1[tl];
        part[5 * T + v] = 0.5 * hpc2 * hpc2 - (double)f.hpl2[tl];
        float ks = 0.0f;
        int kn = 0;
        for (int kk = 0; kk < cx.pnk; ++kk) {
          const float4 kd = __ldg(cx.kde + kk);
          if ((int)kd.w == tl) {
            const float dx = ax[h] - kd.x, dy = ay[h] - kd.y, dz = az[h] - kd.z;
            ks += expf(f.kde2 * (dx * dx + dy * dy + dz * dz));
            ++kn;
          }
        }
        part[6 * T + v] = kn ? (double)ks / (double)kn : 0.0;
        const Slot &sl = slots[sl_of[h]];
        const float *lc = cx.lig_center + sl.lig_conf * 3;
        const float rx = ax[h] - (orig[h].x + lc[0]), ry = ay[h] - (orig[h].y + lc[1]),
                    rz = az[h] - (orig[h].z + lc[2]);
        part[7 * T + v] = (double)(rx * rx + ry * ry + rz * rz);
        int tp = 0;
        const int *rs = cx.ref_start + pc * (L + 1);
        for (int i = rs[l]; i < rs[l + 1]; ++i) {
          const float4 rp = __ldg(cx.ref_pts + i);
          tp += dist2(ax[h], ay[h], az[h], rp.x, rp.y, rp.z) <= rp.w ? 1 : 0;
        }
        part[9 * T + v] = (double)tp;
      }
      if (__syncthreads_or(aborted)) {
        aborted = true;
        break;
      }

      /* ---- per-replica epilogue: one warp per slot ---- */
      for (int js = warp; js < k; js += nwarps) {
        Slot &sl = slots[js];
        /* slot totals are written back over the slot's first partial */
        double *tot = part + js * SL;
#pragma unroll 1
        for (int qi = 0; qi < NQ; ++qi) {
          double v = 0.0;
          for (int i = lane; i < SL; i += 32) v += part[qi * T + js * SL + i];
          v = warp_sum(v);
          if (lane == 0) tot[qi * T] = v;
        }
        /* MCS position restraints */
        double elhm = 0.0;
        for (int m = 0; m < cx.pos; ++m) {
          double sm = 0.0;
          int cnt = 0;
          for (int i = lane; i < L; i += 32) {
            const int idx = cx.lig_meta[sl.lig_conf * L + i].y;
            const float mx = cx.mcs_x[(size_t)m * cx.mcs_ld + idx];
            if (mx != GD_MCS_INVALID_COORD) {
              const float4 at = atoms[js * SL + i];
              const float dx = at.x - mx;
              const float dy = at.y - cx.mcs_y[(size_t)m * cx.mcs_ld + idx];
              const float dz = at.z - cx.mcs_z[(size_t)m * cx.mcs_ld + idx];
              sm += (double)(dx * dx + dy * dy + dz * dz);
              ++cnt;
            }
          }
          sm = warp_sum(sm);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
          if (lane == 0 && cnt) elhm += (double)cx.mcs_tcc[m] * sqrt(sm / (double)cnt);
        }
        if (lane == 0) {
          const double Ld = (double)L;
          double e[GD_MAXWEI];
          e[0] = tot[0 * T] / Ld;
          e[1] = tot[1 * T] / Ld;
          e[2] = tot[2 * T] / Ld;
          e[3] = tot[3 * T] / Ld;
          e[4] = tot[4 * T] / Ld;
          e[5] = tot[5 * T] / Ld;
          e[6] = tot[6 * T] / (double)f.kde3 / Ld;
          e[7] = log(elhm / (double)cx.pos);
          {
            const double dx = (double)sl.tx - (double)cx.pocket[0];
            const double dy = (double)sl.ty - (double)cx.pocket[1];
            const double dz = (double)sl.tz - (double)cx.pocket[2];
            e[8] = sqrt(dx * dx + dy * dy + dz * dz);
          }
          double etot = 0.0;
          gd_energy en;
#pragma unroll
          for (int i = 0; i < GD_MAXWEI - 1; ++i) {
            const double v = (double)f.a_para[i] * e[i] + (double)f.b_para[i];
            en.e[i] = (float)v;
            etot += v * (double)f.w[i];
          }
          en.e[GD_MAXWEI - 1] = (float)etot;
          {
            const double tp = tot[9 * T], ncn = tot[8 * T];
            const double fp = ncn - tp, fn = (double)cx.nref_total - tp;
            const double tn = Ld * (double)P - tp - fp - fn;
            const double dv2 = sqrt((tp + fp) * (tp + fn) * (tn + fp) * (tn + fn));
            en.cms = dv2 != 0.0 ? (float)((tp * tn - fp * fn) / dv2) : 0.0f;
          }
          en.rmsd = (float)sqrt(tot[7 * T] / Ld);
          const int rid = sl.rep;
          if (a.mode == 2 || a.mode == 4) {
            a.e_out[rid] = en;
          } else if (DA && a.mode == 3) {
            da_decide(a, cx, tile.complex_index, rid, en, sl.mm_new, step_first + s);
          } else {
            int acc = 1;
            if (a.mode == 0)
              acc = gd_metropolis(en.e[GD_MAXWEI - 1], sl.e_old.e[GD_MAXWEI - 1], sl.mb, sl.u);
            sl.accept = acc;
            if (acc) {
              sl.e_old = en;
#pragma unroll
              for (int i = 0; i < 6; ++i) sl.mm_old[i] = sl.mm_new[i];
              if (a.mode == 0) sl.n_acc += 1;
              if (a.rec) {
                const int kslot = sl.rec_next;
                if (kslot < a.rec_cap) {
                  gd_record_step *r = a.rec + (size_t)rid * a.rec_cap + kslot;
                  r->replica = sl.replica;
                  r->energy = en;
#pragma unroll
                  for (int i = 0; i < 6; ++i) r->movematrix[i] = sl.mm_new[i];
                  r->step = a.mode == 0 ? step_first + s : 0;
                  sl.rec_next = kslot + 1;
                } else {
                  atomicOr(a.err, GD_DEV_ERR_RECORD_FULL);
                }
              }
            }
            if (a.trace_e && a.mode == 0) {
              const int ti = step_first + s - a.trace_step0;
              if (ti >= 0 && ti < a.trace_cap) {
                a.trace_e[(size_t)rid * a.trace_cap + ti] = en.e[GD_MAXWEI - 1];
                a.trace_acc[(size_t)rid * a.trace_cap + ti] = acc;
              }
            }
          }
        }
      }
      __syncthreads();
    }

    if (aborted) {
      /* a bounded wait gave up: let the copies still in flight land (bounded again, with
       * the fixed drain limit) before the CTA leaves, then stop */
      if (tid == 0) {
        const long long drain_ns = 2000000000LL;
        if (s_issued[0]) mbar_wait_bounded(&bar[0], (s_issued[0] - 1u) & 1u, drain_ns);
        if (s_issued[1]) mbar_wait_bounded(&bar[1], (s_issued[1] - 1u) & 1u, drain_ns);
      }
      __syncthreads();
      break;
    }

    /* ---- write back replica state ---- */
    if (a.mode < 2 && tid < k) {
      const Slot &sl = slots[tid];
      a.e_old[sl.rep] = sl.e_old;
      a.etotal[sl.rep] = sl.e_old.e[GD_MAXWEI - 1];
      a.n_accept[sl.rep] = sl.n_acc;
      if (a.rec) a.rec_next[sl.rep] = sl.rec_next;
#pragma unroll
      for (int i = 0; i < 6; ++i) a.mm_old[(size_t)sl.rep * 6 + i] = sl.mm_old[i];
      /* ExchangeReplicas_d fused: the replica that completes its group in this launch (the
       * group's last to be written back, counted with fences on both sides) exchanges the
       * group's temperatures; no CTA waits for another */
      if (a.mode == 0 && a.x_done) {
        const int local = sl.rep - cx.rep_offset, nl = cx.n_lig, nt = cx.n_tmp;
        const int lg = (local / (nt * nl)) * nl + local % nl;
        __threadfence();
        if (atomicAdd(a.x_done + a.x_group_base[tile.complex_index] + lg, 1) == nt - 1) {
          __threadfence();
          const int mode_t = !(((step_first % a.x_spd) / a.x_spe) % 2);
          gd_exchange_group(cx, lg, a.replica, a.etotal, a.x_acs, a.seed,
                            (a.x_call_base ? *a.x_call_base : 0) + a.x_call_off, mode_t);
        }
      }
    }
    __syncthreads();
  }
}

/* the kernel variants the host can launch: point pairs in flight per lane; protein split
 * and the delayed-acceptance exact stage (mode 3) compiled out when false; replicas per
 * thread (two only for the plain modes without split) */
#define GD_INST(U, S, D, P) \
  template __global__ void gd_mc_kernel<U, S, D, P>(GdMcArgs, GdForceConst);
GD_INST(1, false, false, 1) GD_INST(2, false, false, 1) GD_INST(4, false, false, 1)
GD_INST(1, true, false, 1) GD_INST(2, true, false, 1) GD_INST(4, true, false, 1)
GD_INST(1, false, true, 1) GD_INST(2, false, true, 1) GD_INST(4, false, true, 1)
GD_INST(1, true, true, 1) GD_INST(2, true, true, 1) GD_INST(4, true, true, 1)
GD_INST(1, false, false, 2) GD_INST(2, false, false, 2)
#undef GD_INST

/* ExchangeReplicas_d, one thread per (complex, protein conformer, ligand conformer) group of
 * the range [g_begin, g_end). */
__global__ void gd_exchange_kernel(const GdDevComplex *cxs, const int *group_base, int n_complex,
                                   int g_begin, int g_end, gd_replica *replica,
                                   const float *etotal, int *acs, uint64_t seed,
                                   const int *call_base, int call_off, int mode_t) {
  const int g = g_begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= g_end || mode_t >= 2) return;
  int lo = 0, hi = n_complex - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (group_base[mid] <= g) lo = mid; else hi = mid - 1;
  }
  gd_exchange_group(cxs[lo], g - group_base[lo], replica, etotal, acs, seed,
                    (call_base ? *call_base : 0) + call_off, mode_t);
}

/* ResetCounter_d (src/kernel_cuda_l1_resetcounter.cu:12-22). */
__global__ void gd_reset_records_kernel(int *rec_next, int r0, int r1) {
  const int r = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (r <= r1) rec_next[r] = 0;
}

}  // namespace gd
