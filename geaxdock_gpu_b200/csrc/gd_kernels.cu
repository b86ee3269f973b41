/*
 * gd_kernels.cu -- sm_100a kernels of the Monte Carlo docking path.
 *
 * gd_mc_kernel: one persistent kernel for MonteCarlo_Init_d, MonteCarlo_d and pose
 * evaluation (reference src/kernel_cuda_l1_montecarlo.cu:12-127). Each CTA pulls tiles from
 * a work queue; a tile is `count` replicas of one protein conformer. Lane (slot j, atom l)
 * owns one ligand atom of one replica for all steps of the launch:
 *   Move_d        (src/kernel_cuda_l2_move.cu:21-80)       placed in registers from a
 *                                                         Philox draw, no HBM traffic;
 *   CalcEnergy_d  (src/kernel_cuda_l2_calcenergy.cu:19-360) pair loop over protein points
 *                 staged by cp.async.bulk into a shared-memory double buffer, points sorted by
 *                 type so each lane keeps its pair parameters in registers per segment,
 *                 MUFU rsqrt / rcp / ex2 on the FP32 pipe, FP32 range sums folded into FP64;
 *   CalcMcc_d     (src/kernel_cuda_l2_calcmcc.cu:148-206) contact count inside the pair loop,
 *                 true positives from the sparse reference-contact list;
 *   CalcRmsd_d, KDE, MCS, dst, CombineEnergy_d (src/kernel_cuda_l3_combineenergy.cu:23-37),
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
  float vdw, ele, pmf, psp, hdb, hsum;
  int ncon;
};

/* Pair loop over points [i0, i1) of one (type, kind) segment held in shared memory.
 * KIND bit 0: hydrophobic point (hpc), bit 1: class-2 point (psp). HDB: some lane of the
 * warp has a live hydrogen-bond pair for this segment's type. */
template <int KIND, bool HDB>
__device__ __forceinline__ void pair_range(const float4 *__restrict__ P,
                                           const float2 *__restrict__ X, int i0, int i1,
                                           float ax, float ay, float az, const GdPairParam &q,
                                           const float *__restrict__ psprow,
                                           const GdForceConst &f, Acc &a) {
  const float lj1 = f.lj1, el0 = f.el0, el1 = f.el1, a1 = f.a1, b1 = f.b1, iel1 = f.inv_el1;
  const float cA = -0.5f * LOG2E_F, cB = 6.0f * LOG2E_F;
#pragma unroll 2
  for (int i = i0; i < i1; ++i) {
    const float4 p = P[i];
    const float d2 = dist2(ax, ay, az, p.x, p.y, p.z);
    const float ri = rsqrt_a(d2);
    const float r = d2 * ri;
    /* vdw: (p1 - p2) / (p1 lj0 (1 + lj1 d2) + 1), p1 = p1a r^-9, p2 = p2a r^-6 */
    const float r2i = ri * ri;
    const float r3i = r2i * ri;
    const float r6i = r3i * r3i;
    const float num = r6i * __fmaf_rn(q.p1a, r3i, -q.p2a);
    const float p4 = __fmaf_rn(q.p1l * (r6i * r3i), __fmaf_rn(lj1, d2, 1.0f), 1.0f);
    a.vdw = __fmaf_rn(num, rcp_a(p4), a.vdw);
    /* ele: q_l ele_p g(el1 r); q_l applied once per atom */
    const float s1 = el1 * r;
    const float gn = __fmaf_rn(s1 * s1, __fmaf_rn(b1, s1, a1), el0);
    const float gf = ri * iel1;
    a.ele = __fmaf_rn(p.w, (s1 < 1.0f) ? gn : gf, a.ele);
    /* pmf: pmf1 / (1 + exp((6 - r/2)(r - pmf0))) */
    const float ex = ex2_a(__fmaf_rn(cA, r, cB) * (r - q.pmf0));
    a.pmf = __fmaf_rn(q.pmf1, rcp_a(1.0f + ex), a.pmf);
    /* contact (mcc, psp): sqrtf(d2) <= pmf0  <=>  d2 <= thr */
    const bool contact = d2 <= q.thr;
    a.ncon += contact ? 1 : 0;
    if (KIND & 2) {
      const float2 x = X[i];
      if (contact) a.psp += __ldg(psprow + __float_as_int(x.y));
    }
    if (HDB) {
      const float h = __fmaf_rn(r, q.hc1, q.hc0);
      a.hdb = __fmaf_rn(q.hs, ex2_a(-(h * h)), a.hdb);
    }
    if (KIND & 1) {
      const float hp = X[i].x;
      float t = __fmaf_rn(d2, HPC_C4, -HPC_C3);
      t = __fmaf_rn(d2, t, HPC_C2);
      t = __fmaf_rn(d2, t, -HPC_C1);
      const float pl = __fmaf_rn(d2, t, 1.0f);
      if (d2 <= 81.0f) a.hsum = __fmaf_rn(hp, pl, a.hsum);
    }
  }
}

struct Slot {
  int rep, lig_conf, accept, n_acc;
  int rec_next, pad0;
  float mb, u;
  float mm_new[6];
  float pad1[2];
  gd_energy e_old;
  gd_replica replica;
};

/* deterministic warp sum of a double */
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

#define NQ 10 /* vdw ele pmf psp hdb hpc kde rmsd ncon tp */

__global__ void __launch_bounds__(GD_MAX_TPB) gd_mc_kernel(GdMcArgs a, GdForceConst f) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int T = blockDim.x, tid = threadIdx.x, D = a.chunk;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
  float4 *bpos = reinterpret_cast<float4 *>(smem + 16);
  float2 *baux = reinterpret_cast<float2 *>(bpos + 2 * D);
  float4 *atoms = reinterpret_cast<float4 *>(baux + 2 * D);
  double *part = reinterpret_cast<double *>(atoms + T);
  Slot *slots = reinterpret_cast<Slot *>(part + NQ * T);
  __shared__ int s_tile;
  __shared__ int s_abort;

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_abort = 0;
  }
  __syncthreads();
  uint32_t consumed0 = 0, consumed1 = 0; /* completed phases used per buffer */
  uint32_t issued0 = 0, issued1 = 0;     /* copies issued per buffer (thread 0) */
  const int step_first = a.step0 + (a.step_base ? *a.step_base : 0);
  const int warp = tid >> 5, lane = tid & 31, nwarps = T >> 5;

  for (;;) {
    if (tid == 0) s_tile = atomicAdd(a.tile_counter, 1);
    __syncthreads();
    const int t = s_tile;
    if (t >= a.n_tiles || s_abort) break;
    const GdTileDesc tile = a.tiles[t];
    const GdDevComplex &cx = a.cx[tile.complex_index];
    const int L = cx.lna, k = tile.count;
    const bool active = tid < k * L;
    const int j = active ? tid / L : 0;
    const int l = active ? tid - j * L : 0;

    /* ---- slot set-up ---- */
    if (tid < k) {
      Slot &s = slots[tid];
      const int id = tile.rep_begin + tid;
      s.rep = id;
      s.accept = 0;
      if (a.mode == 2) {
        s.lig_conf = a.lig_conf_in[id];
      } else {
        s.replica = a.replica[id];
        s.lig_conf = s.replica.idx_lig;
        s.mb = cx.minus_beta[s.replica.idx_tmp];
        if (a.mode == 0) {
          s.e_old = a.e_old[id];
          s.n_acc = a.n_accept[id];
          s.rec_next = a.rec ? a.rec_next[id] : 0;
        } else {
          s.n_acc = 0;
          s.rec_next = 0;
        }
      }
    }
    __syncthreads();

    /* ---- per-lane constants ---- */
    const int lig_conf = slots[j].lig_conf;
    const int id = tile.rep_begin + j;
    const float4 orig = cx.lig_pos[lig_conf * L + l];
    const int2 meta = cx.lig_meta[lig_conf * L + l];
    const float cxo = cx.lig_center[lig_conf * 3 + 0], cyo = cx.lig_center[lig_conf * 3 + 1],
                czo = cx.lig_center[lig_conf * 3 + 2];
    const int tl = meta.x;
    const float *psprow = cx.psp + (size_t)tl * cx.psp_ld;
    const GdPairParam *pprow = a.pp + tl * GD_MAXTP1;
    float mm[6];
    if (a.mode == 0) {
#pragma unroll
      for (int i = 0; i < 6; ++i) mm[i] = a.mm_old[(size_t)id * 6 + i];
    }
    const unsigned wmask = __ballot_sync(0xffffffffu, active);

    /* ---- protein tile pipeline ---- */
    const int pc = tile.prt_conf;
    const float4 *gpos = cx.pt_pos + (size_t)pc * cx.pnp_pad;
    const float2 *gaux = cx.pt_aux + (size_t)pc * cx.pnp_pad;
    const int4 *segs = cx.seg + pc * GD_MAX_SEG;
    const int nseg = cx.seg_count[pc];
    const int P = cx.pnp;
    const int nch = (P + D - 1) / D;
    const bool resident = nch <= 2;
    const int nsteps = a.mode == 0 ? a.n_steps : 1;
    const int total_q = resident ? nch : nsteps * nch;
    auto issue = [&](int q) {
      const int c = q % nch, b = q & 1;
      const int c0 = c * D;
      const int n = min(D, cx.pnp_pad - c0);
      if (b) ++issued1; else ++issued0;
      mbar_expect_tx(&bar[b], (uint32_t)(n * 24));
      bulk_g2s(bpos + b * D, gpos + c0, (uint32_t)(n * 16), &bar[b]);
      bulk_g2s(baux + b * D, gaux + c0, (uint32_t)(n * 8), &bar[b]);
    };
    if (tid == 0) {
      issue(0);
      if (total_q > 1) issue(1);
    }
    bool aborted = false;

    for (int s = 0; s < nsteps; ++s) {
      /* ---- Move_d: draw, new pose, placed atom ---- */
      float mmn[6], u = 0.0f;
      if (a.mode == 0) {
        float delta[6];
        gd_draw_step(a.seed, (uint32_t)cx.stream, (uint32_t)(id - cx.rep_offset),
                     (uint32_t)(step_first + s), a.move_kind, a.move_scale, delta, &u);
#pragma unroll
        for (int i = 0; i < 6; ++i) mmn[i] = GD_ADD(mm[i], delta[i]);
      } else if (a.mode == 2) {
#pragma unroll
        for (int i = 0; i < 6; ++i) mmn[i] = a.mm_in[(size_t)id * 6 + i];
      } else {
#pragma unroll
        for (int i = 0; i < 6; ++i) mmn[i] = 0.0f;
      }
      float rot[9];
      gd_rotation(mmn, rot);
      const float tx = GD_ADD(mmn[0], cxo), ty = GD_ADD(mmn[1], cyo), tz = GD_ADD(mmn[2], czo);
      float ax, ay, az;
      gd_place_atom(rot, tx, ty, tz, orig.x, orig.y, orig.z, &ax, &ay, &az);

      double dv = 0, de = 0, dp = 0, ds = 0, dh = 0, dhs = 0;
      int ncon = 0;

      for (int ci = 0; ci < nch; ++ci) {
        const int q = resident ? ci : s * nch + ci;
        const int b = q & 1;
        if (!resident || s == 0) {
          const uint32_t par = b ? (consumed1 & 1u) : (consumed0 & 1u);
          const bool ok = mbar_wait_bounded(&bar[b], par, a.timeout_ns);
          if (ok) { if (b) ++consumed1; else ++consumed0; }
          if (__syncthreads_or(!ok)) {
            if (tid == 0) { atomicOr(a.err, GD_DEV_ERR_TIMEOUT); s_abort = 1; }
            aborted = true;
            break;
          }
        }
        if (active) {
          const float4 *P4 = bpos + b * D; /* local index = point index - c0 */
          const float2 *X2 = baux + b * D;
          const int c0 = ci * D, c1 = min(P, c0 + D);
          for (int sg = 0; sg < nseg; ++sg) {
            const int4 g = segs[sg];
            const int i0 = max(g.x, c0) - c0, i1 = min(g.y, c1) - c0;
            if (i0 >= i1) continue;
            const float4 q0 = __ldg(reinterpret_cast<const float4 *>(pprow + g.z));
            const float4 q1 = __ldg(reinterpret_cast<const float4 *>(pprow + g.z) + 1);
            const float4 q2 = __ldg(reinterpret_cast<const float4 *>(pprow + g.z) + 2);
            GdPairParam pq;
            pq.p1a = q0.x; pq.p2a = q0.y; pq.p1l = q0.z; pq.thr = q0.w;
            pq.pmf0 = q1.x; pq.pmf1 = q1.y; pq.hc1 = q1.z; pq.hc0 = q1.w;
            pq.hs = q2.x; pq.hneed = q2.y;
            const bool hdb = __any_sync(wmask, pq.hneed != 0.0f);
            Acc acc = {0, 0, 0, 0, 0, 0, 0};
            const int kind = g.w;
            if (hdb) {
              switch (kind) {
                case 0: pair_range<0, true>(P4, X2, i0, i1, ax, ay, az, pq, psprow, f, acc); break;
                case 1: pair_range<1, true>(P4, X2, i0, i1, ax, ay, az, pq, psprow, f, acc); break;
                case 2: pair_range<2, true>(P4, X2, i0, i1, ax, ay, az, pq, psprow, f, acc); break;
                default: pair_range<3, true>(P4, X2, i0, i1, ax, ay, az, pq, psprow, f, acc); break;
              }
            } else {
              switch (kind) {
                case 0: pair_range<0, false>(P4, X2, i0, i1, ax, ay, az, pq, psprow, f, acc); break;
                case 1: pair_range<1, false>(P4, X2, i0, i1, ax, ay, az, pq, psprow, f, acc); break;
                case 2: pair_range<2, false>(P4, X2, i0, i1, ax, ay, az, pq, psprow, f, acc); break;
                default: pair_range<3, false>(P4, X2, i0, i1, ax, ay, az, pq, psprow, f, acc); break;
              }
            }
            dv += acc.vdw; de += acc.ele; dp += acc.pmf; ds += acc.psp; dh += acc.hdb;
            dhs += acc.hsum;
            ncon += acc.ncon;
          }
        }
        if (!resident) {
          __syncthreads(); /* every lane is done with buffer b */
          if (tid == 0 && q + 2 < total_q) issue(q + 2);
        }
      }
      if (aborted) break;

      /* ---- per-atom tail: hpc, kde, rmsd, reference contacts ---- */
      if (active) {
        const double hpc2 = (dhs - (double)f.hpl0[tl]) / (double)f.hpl1[tl];
        const double vhpc = 0.5 * hpc2 * hpc2 - (double)f.hpl2[tl];
        float ks = 0.0f;
        int kn = 0;
        for (int kk = 0; kk < cx.pnk; ++kk) {
          const float4 kd = __ldg(cx.kde + kk);
          if ((int)kd.w == tl) {
            const float dx = ax - kd.x, dy = ay - kd.y, dz = az - kd.z;
            ks += expf(f.kde2 * (dx * dx + dy * dy + dz * dz));
            ++kn;
          }
        }
        const double vkde = kn ? (double)ks / (double)kn : 0.0;
        const float rx = ax - (orig.x + cxo), ry = ay - (orig.y + cyo), rz = az - (orig.z + czo);
        const double vrms = (double)(rx * rx + ry * ry + rz * rz);
        int tp = 0;
        const int *rs = cx.ref_start + pc * (L + 1);
        for (int i = rs[l]; i < rs[l + 1]; ++i) {
          const float4 rp = __ldg(cx.ref_pts + i);
          tp += dist2(ax, ay, az, rp.x, rp.y, rp.z) <= rp.w ? 1 : 0;
        }
        part[0 * T + tid] = dv;
        part[1 * T + tid] = de * (double)orig.w;
        part[2 * T + tid] = dp;
        part[3 * T + tid] = ds;
        part[4 * T + tid] = dh;
        part[5 * T + tid] = vhpc;
        part[6 * T + tid] = vkde;
        part[7 * T + tid] = vrms;
        part[8 * T + tid] = (double)ncon;
        part[9 * T + tid] = (double)tp;
        atoms[tid] = make_float4(ax, ay, az, 0.0f);
        if (l == 0) {
          Slot &sl = slots[j];
          sl.u = u;
#pragma unroll
          for (int i = 0; i < 6; ++i) sl.mm_new[i] = mmn[i];
        }
      }
      __syncthreads();

      /* ---- per-replica epilogue: one warp per slot ---- */
      for (int js = warp; js < k; js += nwarps) {
        Slot &sl = slots[js];
        double tot[NQ];
#pragma unroll
        for (int qi = 0; qi < NQ; ++qi) {
          double v = 0.0;
          for (int i = lane; i < L; i += 32) v += part[qi * T + js * L + i];
          tot[qi] = warp_sum(v);
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
              const float4 at = atoms[js * L + i];
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
          e[0] = tot[0] / Ld;
          e[1] = tot[1] / Ld;
          e[2] = tot[2] / Ld;
          e[3] = tot[3] / Ld;
          e[4] = tot[4] / Ld;
          e[5] = tot[5] / Ld;
          e[6] = tot[6] / (double)f.kde3 / Ld;
          e[7] = log(elhm / (double)cx.pos);
          {
            const float *lc = cx.lig_center + sl.lig_conf * 3;
            const double dx = (double)GD_ADD(sl.mm_new[0], lc[0]) - (double)cx.pocket[0];
            const double dy = (double)GD_ADD(sl.mm_new[1], lc[1]) - (double)cx.pocket[1];
            const double dz = (double)GD_ADD(sl.mm_new[2], lc[2]) - (double)cx.pocket[2];
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
            const double tp = tot[9], ncn = tot[8];
            const double fp = ncn - tp, fn = (double)cx.nref_total - tp;
            const double tn = Ld * (double)P - tp - fp - fn;
            const double dv2 = sqrt((tp + fp) * (tp + fn) * (tn + fp) * (tn + fn));
            en.cms = dv2 != 0.0 ? (float)((tp * tn - fp * fn) / dv2) : 0.0f;
          }
          en.rmsd = (float)sqrt(tot[7] / Ld);
          const int rid = sl.rep;
          if (a.mode == 2) {
            a.e_out[rid] = en;
          } else {
            int acc = 1;
            if (a.mode == 0)
              acc = gd_metropolis(en.e[GD_MAXWEI - 1], sl.e_old.e[GD_MAXWEI - 1], sl.mb, sl.u);
            sl.accept = acc;
            if (acc) {
              sl.e_old = en;
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
      if (a.mode == 0 && active && slots[j].accept) {
#pragma unroll
        for (int i = 0; i < 6; ++i) mm[i] = mmn[i];
      }
    }

    if (aborted) {
      /* a bounded wait gave up: let the copies still in flight land (bounded again, with
       * the fixed drain limit) before the CTA leaves, then stop */
      if (tid == 0) {
        const long long drain_ns = 2000000000LL;
        if (issued0 > consumed0) mbar_wait_bounded(&bar[0], consumed0 & 1u, drain_ns);
        if (issued1 > consumed1) mbar_wait_bounded(&bar[1], consumed1 & 1u, drain_ns);
      }
      __syncthreads();
      break;
    }

    /* ---- write back replica state ---- */
    if (a.mode != 2) {
      if (tid < k) {
        const Slot &sl = slots[tid];
        a.e_old[sl.rep] = sl.e_old;
        a.etotal[sl.rep] = sl.e_old.e[GD_MAXWEI - 1];
        a.n_accept[sl.rep] = a.mode == 1 ? 0 : sl.n_acc;
        if (a.rec) a.rec_next[sl.rep] = sl.rec_next;
      }
      if (active && l == 0) {
#pragma unroll
        for (int i = 0; i < 6; ++i) a.mm_old[(size_t)id * 6 + i] = a.mode == 1 ? 0.0f : mm[i];
      }
    }
    __syncthreads();
  }
}

/* ExchangeReplicas_d, one thread per (complex, protein conformer, ligand conformer) group. */
__global__ void gd_exchange_kernel(const GdDevComplex *cxs, const int *group_base, int n_complex,
                                   int n_groups, gd_replica *replica, const float *etotal,
                                   int *acs, uint64_t seed, const int *call_base, int call_off,
                                   int mode_t) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_groups || mode_t >= 2) return;
  int lo = 0, hi = n_complex - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (group_base[mid] <= g) lo = mid; else hi = mid - 1;
  }
  const GdDevComplex &cx = cxs[lo];
  const int lg = g - group_base[lo];
  const int nl = cx.n_lig, nt = cx.n_tmp;
  const int p = lg / nl, l = lg - p * nl;
  const int call = (call_base ? *call_base : 0) + call_off;
  int temps[GD_MAXTMP], orders[GD_MAXTMP];
  float en[GD_MAXTMP];
  for (int t = 0; t < nt; ++t) {
    const int f = cx.rep_offset + nt * nl * p + nl * t + l;
    temps[t] = replica[f].idx_tmp;
    en[t] = etotal[f];
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

/* ResetCounter_d (src/kernel_cuda_l1_resetcounter.cu:12-22). */
__global__ void gd_reset_records_kernel(int *rec_next, int r0, int r1) {
  const int r = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (r <= r1) rec_next[r] = 0;
}

}  // namespace gd
