/*
 * gd_da.cu -- delayed-acceptance Monte Carlo steps around the exact energy kernel.
 *
 * One delayed-acceptance step of every replica is two launches on one stream (captured in a
 * CUDA graph by the host):
 *   1. da_front     per CTA of 32 replicas: the plain step's move and accept uniform
 *                   (gd_draw_step, the Philox counters of gd_mc_kernel), the surrogate-stage
 *                   uniform, the feature rows in shared memory, the BF16 tensor-core network
 *                   on them, the surrogate Metropolis test u1 < exp(mb (S_new - S_cur)), and
 *                   the survivors' compaction into their (complex, protein conformer) group's
 *                   pose slots
 *   2. gd_mc_kernel mode 3: exact energies of the survivors only (tiles past a group's
 *                   survivors exit at once) and, in its epilogue, the exact test
 *                   u2 < exp(mb ((E_new - E_old) - (S_new - S_cur))), state update, records
 * The pair is a valid Metropolis-Hastings kernel for the exact distribution (Christen & Fox,
 * "Markov chain Monte Carlo using an approximation", J. Comput. Graph. Stat. 14, 2005) for
 * any fixed surrogate S. With the stage switched off for a complex, S_new = S_cur, every
 * proposal survives and the second test is bit-identical to the plain Metropolis test with
 * the plain step's uniform: the step reproduces gd_mc_kernel's trajectory exactly.
 * Survivors take their slots through an atomic counter per group, so the order of the slots
 * varies between runs; a replica's energy does not depend on its slot (per-lane sums and
 * per-slot reductions in a fixed order), so the chains do not either.
 */
#include <cuda_bf16.h>

#include "gd_mlp.cuh"
#include "gd_mlp_fwd.cuh"
#include "gd_numerics.h"

namespace gd {

namespace {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ int cur_step(const GdDaDev &d, int step0) {
  return step0 + (d.step_base ? *d.step_base : 0);
}

/* Shepperd's method (J. Guidance and Control 1, 1978): quaternion of a rotation matrix
 * (row-major), sign fixed so that w >= 0. */
__device__ void quat_of(const float r[9], float q[4]) {
  const float tr = r[0] + r[4] + r[8];
  float w, x, y, z;
  if (tr > 0.0f) {
    const float S = sqrtf(tr + 1.0f) * 2.0f;
    w = 0.25f * S; x = (r[7] - r[5]) / S; y = (r[2] - r[6]) / S; z = (r[3] - r[1]) / S;
  } else if (r[0] > r[4] && r[0] > r[8]) {
    const float S = sqrtf(1.0f + r[0] - r[4] - r[8]) * 2.0f;
    w = (r[7] - r[5]) / S; x = 0.25f * S; y = (r[1] + r[3]) / S; z = (r[2] + r[6]) / S;
  } else if (r[4] > r[8]) {
    const float S = sqrtf(1.0f + r[4] - r[0] - r[8]) * 2.0f;
    w = (r[2] - r[6]) / S; x = (r[1] + r[3]) / S; y = 0.25f * S; z = (r[5] + r[7]) / S;
  } else {
    const float S = sqrtf(1.0f + r[8] - r[0] - r[4]) * 2.0f;
    w = (r[3] - r[1]) / S; x = (r[2] + r[6]) / S; y = (r[5] + r[7]) / S; z = 0.25f * S;
  }
  const float sg = w < 0.0f ? -1.0f : 1.0f;
  q[0] = sg * w; q[1] = sg * x; q[2] = sg * y; q[3] = sg * z;
}

/* one feature row (layout in gd_mlp.cuh), 16-byte aligned; the embedding columns are written
 * as 0 (the network fills them from its table) */
__device__ void write_features(const GdDaDev &d, int ci, int lc, const float mm[6], bf16 *row) {
  const GdDevComplex &cx = d.cx[ci];
  float rot[9];
  gd_rotation(mm, rot);
  const float *c = cx.lig_center + lc * 3;
  const float tx = c[0] + mm[0] - cx.pocket[0];
  const float ty = c[1] + mm[1] - cx.pocket[1];
  const float tz = c[2] + mm[2] - cx.pocket[2];
  float q[4];
  quat_of(rot, q);
  float f[GD_MLP_IN];
#pragma unroll
  for (int i = 0; i < GD_MLP_IN; ++i) f[i] = 0.0f;
  f[0] = 0.25f * tx; f[1] = 0.25f * ty; f[2] = 0.25f * tz;
  f[3] = q[0]; f[4] = q[1]; f[5] = q[2]; f[6] = q[3];
  const float *pf = d.pocket_feat + ci * GD_MLP_POCKET;
#pragma unroll
  for (int i = 0; i < GD_MLP_POCKET; ++i) f[GD_MLP_POCKET_OFF + i] = pf[i];
  f[55] = rot[0]; f[56] = rot[3]; f[57] = rot[6];
  f[58] = rot[1]; f[59] = rot[4]; f[60] = rot[7];
  f[61] = 0.125f * sqrtf(tx * tx + ty * ty + tz * tz);
  uint4 *dst = reinterpret_cast<uint4 *>(row);
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    __nv_bfloat162 h[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = v * 8 + 2 * e;
      const bool emb0 = i >= GD_MLP_EMB_OFF && i < GD_MLP_EMB_OFF + GD_MLP_EMB;
      const bool emb1 = i + 1 >= GD_MLP_EMB_OFF && i + 1 < GD_MLP_EMB_OFF + GD_MLP_EMB;
      h[e] = __floats2bfloat162_rn(emb0 ? 0.0f : f[i], emb1 ? 0.0f : f[i + 1]);
    }
    dst[v] = *reinterpret_cast<uint4 *>(h);
  }
}

template <int NT>
__global__ void __launch_bounds__(256) front_kernel(GdDaDev d, int mode, int step0, int *cnt,
                                                    int r_begin, int r_end) {
  using D = fwd::Dims<NT>;
  constexpr int FR = fwd::FR;
  extern __shared__ __align__(128) unsigned char fsm[];
  __shared__ int cf[FR];
  __shared__ float ys[FR];
  /* a row's proposal, parked here across the network: pose, u1, u2 / complex, conformer */
  __shared__ float rowf[FR][8];
  __shared__ int rowi[FR][2];
  const fwd::Smem<NT> sm(fsm);
  bf16 *xs = sm.xs;
  const int tid = threadIdx.x;
  if (mode != GD_DA_COLLECT) fwd::stage_params<NT>(sm, d.theta, d.L, tid);
  const int r = r_begin + blockIdx.x * FR + tid; /* the row's replica (threads < FR) */
  const int step = cur_step(d, step0);
  if (tid < FR) {
    bf16 *row = xs + tid * D::LDX;
    float mm[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    float u1 = 0.0f, u2 = 0.0f;
    int ci = 0, lc = 0;
    if (r < r_end) {
      ci = d.rep_cx[r];
      const GdDevComplex &cx = d.cx[ci];
      const gd_replica rp = d.replica[r];
      lc = rp.idx_lig;
#pragma unroll
      for (int i = 0; i < 6; ++i) mm[i] = d.mm_old[(size_t)r * 6 + i];
      if (mode != GD_DA_CURRENT) {
        const uint32_t rl = (uint32_t)(r - cx.rep_offset);
        float delta[6];
        gd_draw_step(d.seed, (uint32_t)cx.stream, rl, (uint32_t)step, d.move_kind, d.move_scale,
                     delta, &u2);
        u1 = gd_draw_stage1(d.seed, (uint32_t)cx.stream, rl, (uint32_t)step);
#pragma unroll
        for (int i = 0; i < 6; ++i) mm[i] = GD_ADD(mm[i], delta[i]);
      }
      write_features(d, ci, lc, mm, row);
      cf[tid] = d.emb_base[ci] >= 0 ? d.emb_base[ci] + rp.idx_prt * cx.n_lig + lc : -1;
    } else {
      uint4 *dst = reinterpret_cast<uint4 *>(row);
#pragma unroll
      for (int v = 0; v < 8; ++v) dst[v] = make_uint4(0u, 0u, 0u, 0u);
      cf[tid] = -1;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) rowf[tid][i] = mm[i];
    rowf[tid][6] = u1;
    rowf[tid][7] = u2;
    rowi[tid][0] = ci;
    rowi[tid][1] = lc;
  }
  /* the first weight fragments are in flight while warp 0 finishes the proposals */
  fwd::Ring<NT> ring;
  if (mode != GD_DA_COLLECT) fwd::prefetch_first<NT>(ring, d.wf, tid);
  __syncthreads();
  if (mode != GD_DA_COLLECT) {
    fwd::fill_embedding<NT>(xs, cf, d.theta, d.L, tid);
    __syncthreads();
    fwd::rows_forward<NT>(sm, ring, d.wf, ys, tid);
  }
  if (tid >= FR || r >= r_end) return;
  if (mode == GD_DA_CURRENT) {
    d.s_cur[r] = __fmaf_rn(ys[tid], d.sigma, d.mu);
    return;
  }
  const int ci = rowi[tid][0], lc = rowi[tid][1];
  const float u1 = rowf[tid][6], u2 = rowf[tid][7];
  const bool act_on = mode == GD_DA_STEP && d.active[ci];
  float sn = d.s_cur[r];
  int pass = 1;
  if (act_on) {
    sn = __fmaf_rn(ys[tid], d.sigma, d.mu);
    const float mb = d.cx[ci].minus_beta[d.replica[r].idx_tmp];
    pass = gd_metropolis(sn, d.s_cur[r], mb, u1);
    d.prop[r] += 1;
    d.pass[r] += pass;
  } else {
    d.plain[r] += 1;
  }
  d.s_new[r] = sn;
  d.u2[r] = u2;
  if (pass) {
    const int g = d.rep_group[r];
    const int pos = d.group_b0[g] + atomicAdd(cnt + g, 1);
    d.pose_rep[pos] = r;
#pragma unroll
    for (int i = 0; i < 6; ++i) d.pose_mm[(size_t)pos * 6 + i] = rowf[tid][i];
    d.pose_lc[pos] = lc;
  } else if (d.tr_flag) {
    const int ti = step - d.tr_step0;
    if (ti >= 0 && ti < d.tr_cap) {
      const size_t o = (size_t)r * d.tr_cap + ti;
      d.tr_s[o] = sn;
      d.tr_e[o] = __int_as_float(0x7fc00000);
      d.tr_flag[o] = 0;
    }
  }
  if (mode == GD_DA_COLLECT && d.smp_cap > 0) {
    const long long idx = ((long long)step * d.n_rep + r) % d.smp_cap;
    const uint4 *src = reinterpret_cast<const uint4 *>(xs + tid * D::LDX);
    uint4 *dst = reinterpret_cast<uint4 *>(d.smp_X + (size_t)idx * GD_MLP_IN);
#pragma unroll
    for (int v = 0; v < 8; ++v) dst[v] = src[v];
    d.smp_conf[idx] = cf[tid];
  }
}

__global__ void pose_features_kernel(GdDaDev d, int ci, int pc, int lc, const float *mm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float m[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) m[k] = mm[(size_t)i * 6 + k];
  write_features(d, ci, lc, m, d.X + (size_t)i * GD_MLP_IN);
  d.conf[i] = d.emb_base[ci] >= 0 ? d.emb_base[ci] + pc * d.cx[ci].n_lig + lc : -1;
}

/* one CTA per complex, fixed-order sums over its replicas */
__global__ void __launch_bounds__(256) stats_kernel(GdDaDev d, GdDaEpi e, const GdDevComplex *cxs,
                                                    unsigned long long *stats, double *err) {
  const GdDevComplex &cx = cxs[blockIdx.x];
  __shared__ unsigned long long sh[5][256];
  __shared__ double she[2][256];
  unsigned long long v[5] = {0, 0, 0, 0, 0};
  double w[2] = {0.0, 0.0};
  for (int i = threadIdx.x; i < cx.n_rep; i += 256) {
    const int r = cx.rep_offset + i;
    v[0] += (unsigned long long)d.prop[r];
    v[1] += (unsigned long long)d.pass[r];
    v[2] += (unsigned long long)e.acc[r];
    v[3] += (unsigned long long)d.plain[r];
    v[4] += (unsigned long long)e.plain_acc[r];
    w[0] += e.err2[r];
    w[1] += (double)e.nerr[r];
  }
  const int t = threadIdx.x;
#pragma unroll
  for (int k = 0; k < 5; ++k) sh[k][t] = v[k];
  she[0][t] = w[0];
  she[1][t] = w[1];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (t < o) {
#pragma unroll
      for (int k = 0; k < 5; ++k) sh[k][t] += sh[k][t + o];
      she[0][t] += she[0][t + o];
      she[1][t] += she[1][t + o];
    }
    __syncthreads();
  }
  if (t == 0) {
    unsigned long long *st = stats + (size_t)blockIdx.x * GD_DA_NSTAT;
    st[GD_DA_PROPOSED] = sh[0][0];
    st[GD_DA_PASSED] = sh[1][0];
    st[GD_DA_ACCEPTED] = sh[2][0];
    st[GD_DA_PLAIN] = sh[3][0];
    st[GD_DA_PLAIN_ACC] = sh[4][0];
    err[(size_t)blockIdx.x * GD_DA_NERR] = she[0][0];
    err[(size_t)blockIdx.x * GD_DA_NERR + 1] = she[1][0];
  }
}

/* 8 threads per row, 16 bytes each */
__global__ void gather_kernel(GdDaDev d, long long start, long long n_valid, int rows,
                              const int *ctr, float *t) {
  const int row = blockIdx.x * (blockDim.x >> 3) + (threadIdx.x >> 3), part = threadIdx.x & 7;
  if (row >= rows) return;
  const int iter = ctr[0];
  const gd_u32x4 h = gd_philox4x32_10((uint32_t)row, (uint32_t)iter, 0u, GD_RNG_TRAIN,
                                      (uint32_t)d.seed, (uint32_t)(d.seed >> 32));
  const unsigned long long rnd = ((unsigned long long)h.v[0] << 32) | h.v[1];
  const long long idx = (start + (long long)(rnd % (unsigned long long)n_valid)) % d.smp_cap;
  reinterpret_cast<uint4 *>(d.X + (size_t)row * GD_MLP_IN)[part] =
      reinterpret_cast<const uint4 *>(d.smp_X + (size_t)idx * GD_MLP_IN)[part];
  if (part == 0) {
    d.conf[row] = d.smp_conf[idx];
    const float z = (d.smp_t[idx] - d.mu) / d.sigma;
    t[row] = fminf(fmaxf(z, -8.0f), 8.0f);
  }
}

__global__ void moments_kernel(GdDaDev d, long long start, long long n_valid, float lo, float hi,
                               double *part) {
  __shared__ double s0[256], s1[256], s2[256];
  double a = 0.0, b = 0.0, c = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_valid;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = d.smp_t[(start + i) % d.smp_cap];
    if (v >= lo && v <= hi) {
      a += v;
      b += (double)v * v;
      c += 1.0;
    }
  }
  const int tid = threadIdx.x;
  s0[tid] = a; s1[tid] = b; s2[tid] = c;
  __syncthreads();
  for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
    if (tid < o) { s0[tid] += s0[tid + o]; s1[tid] += s1[tid + o]; s2[tid] += s2[tid + o]; }
    __syncthreads();
  }
  if (tid == 0) {
    part[blockIdx.x * 3 + 0] = s0[0];
    part[blockIdx.x * 3 + 1] = s1[0];
    part[blockIdx.x * 3 + 2] = s2[0];
  }
}

inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

__global__ void train_tick_kernel(float *hist, const float *loss, int *ctr) {
  hist[ctr[1]] = *loss;
  ctr[0] += 1;
  ctr[1] += 1;
}

}  // namespace

int da_prepare(int hidden) {
  if (hidden == 128)
    return cudaFuncSetAttribute(front_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fwd::Dims<1>::smem) == cudaSuccess ? 0 : -2;
  if (hidden == 256)
    return cudaFuncSetAttribute(front_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fwd::Dims<2>::smem) == cudaSuccess ? 0 : -2;
  return -1;
}

int da_front(const GdDaDev &d, int mode, int step0, int *cnt, int r_begin, int r_end,
             cudaStream_t s) {
  if (r_end <= r_begin) return 0;
  const int grid = nblk(r_end - r_begin, fwd::FR);
  if (d.L.hidden == 128)
    front_kernel<1><<<grid, 256, fwd::Dims<1>::smem, s>>>(d, mode, step0, cnt, r_begin, r_end);
  else if (d.L.hidden == 256)
    front_kernel<2><<<grid, 256, fwd::Dims<2>::smem, s>>>(d, mode, step0, cnt, r_begin, r_end);
  else
    return -1; /* the fused step needs H = 128 or 256 */
  return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

void da_pose_features(const GdDaDev &d, int ci, int pc, int lc, const float *mm, int n,
                      cudaStream_t s) {
  pose_features_kernel<<<nblk(n, 128), 128, 0, s>>>(d, ci, pc, lc, mm, n);
}

void da_stats(const GdDaDev &d, const GdDaEpi &e_host, const GdDevComplex *cx_dev, int n_complex,
              unsigned long long *stats, double *err, cudaStream_t s) {
  stats_kernel<<<n_complex, 256, 0, s>>>(d, e_host, cx_dev, stats, err);
}

void da_gather(const GdDaDev &d, long long start, long long n_valid, int rows, const int *ctr,
               float *t, cudaStream_t s) {
  gather_kernel<<<nblk(rows, 32), 256, 0, s>>>(d, start, n_valid, rows, ctr, t);
}

void da_train_tick(float *hist, const float *loss, int *ctr, cudaStream_t s) {
  train_tick_kernel<<<1, 1, 0, s>>>(hist, loss, ctr);
}

void da_target_moments(const GdDaDev &d, long long start, long long n_valid, float lo, float hi,
                       double *part, cudaStream_t s) {
  moments_kernel<<<GD_DA_MOM_BLOCKS, 256, 0, s>>>(d, start, n_valid, lo, hi, part);
}

}  // namespace gd
