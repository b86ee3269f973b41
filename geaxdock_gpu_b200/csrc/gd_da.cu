/*
 * gd_da.cu -- delayed-acceptance Monte Carlo steps around the exact energy kernel.
 *
 * One delayed-acceptance step of every replica is five launches on one stream (captured in a
 * CUDA graph by the host):
 *   1. da_propose   the plain step's move and accept uniform (gd_draw_step, same Philox
 *                   counters as gd_mc_kernel), the surrogate-stage uniform, feature row
 *   2. mlp_forward  surrogate energy of every proposal (BF16 tensor-core MLP)
 *   3. da_stage1    surrogate Metropolis test u1 < exp(mb (S_new - S_cur)); survivors are
 *                   compacted per (complex, protein conformer) block and cut into tiles
 *   4. gd_mc_kernel mode 2: exact energies of the survivors only
 *   5. da_stage2    exact test u2 < exp(mb ((E_new - E_old) - (S_new - S_cur))), state
 *                   update, records
 * The pair is a valid Metropolis-Hastings kernel for the exact distribution (Christen & Fox,
 * "Markov chain Monte Carlo using an approximation", J. Comput. Graph. Stat. 14, 2005) for
 * any fixed surrogate S. With the stage switched off for a complex, S_new = S_cur, every
 * proposal survives and stage 2 is bit-identical to the plain Metropolis test with the plain
 * step's uniform: the step reproduces gd_mc_kernel's trajectory exactly.
 */
#include <cuda_bf16.h>

#include "gd_mlp.cuh"
#include "gd_numerics.h"

namespace gd {

namespace {

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

/* one feature row (layout in gd_mlp.cuh); the embedding columns are left to mlp_embed */
__device__ void write_features(const GdDaDev &d, int ci, int lc, const float mm[6],
                               __nv_bfloat16 *row) {
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
  /* 8 x 16-byte stores; the embedding columns [7, 39) are written as 0 here */
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

__global__ void propose_kernel(GdDaDev d, int step0, int current) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= d.n_rep) return;
  const int ci = d.rep_cx[r];
  const GdDevComplex &cx = d.cx[ci];
  const gd_replica rp = d.replica[r];
  float mm[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) mm[i] = d.mm_old[(size_t)r * 6 + i];
  if (!current) {
    const int step = cur_step(d, step0);
    const uint32_t rl = (uint32_t)(r - cx.rep_offset);
    float delta[6], u;
    gd_draw_step(d.seed, (uint32_t)cx.stream, rl, (uint32_t)step, d.move_kind, d.move_scale,
                 delta, &u);
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      mm[i] = GD_ADD(mm[i], delta[i]);
      d.mm_prop[(size_t)r * 6 + i] = mm[i];
    }
    d.u2[r] = u;
    d.u1[r] = gd_draw_stage1(d.seed, (uint32_t)cx.stream, rl, (uint32_t)step);
  }
  write_features(d, ci, rp.idx_lig, mm, d.X + (size_t)r * GD_MLP_IN);
  d.conf[r] = d.emb_base[ci] + rp.idx_prt * cx.n_lig + rp.idx_lig;
}

__global__ void pose_features_kernel(GdDaDev d, int ci, int pc, int lc, const float *mm, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float m[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) m[k] = mm[(size_t)i * 6 + k];
  write_features(d, ci, lc, m, d.X + (size_t)i * GD_MLP_IN);
  d.conf[i] = d.emb_base[ci] + pc * d.cx[ci].n_lig + lc;
}

__global__ void set_current_kernel(GdDaDev d) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= d.n_rep) return;
  d.s_cur[r] = __fmaf_rn(d.y[r], d.sigma, d.mu);
}

/* one CTA per group; block-wide stable compaction of the survivors */
__global__ void __launch_bounds__(256) stage1_kernel(GdDaDev d, int step0, int collect) {
  const GdGroup G = d.groups[blockIdx.x];
  const GdDevComplex &cx = d.cx[G.ci];
  const bool act = !collect && d.active[G.ci];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  __shared__ int wsum[8];
  int base = 0;
  const int step = cur_step(d, step0);
  const int ti = step - d.tr_step0;
  const bool trace = d.tr_flag && ti >= 0 && ti < d.tr_cap;
  for (int i0 = 0; i0 < G.n; i0 += blockDim.x) {
    const int i = i0 + tid, r = G.b0 + i;
    int pass = 0;
    if (i < G.n) {
      pass = 1;
      float sn = d.s_cur[r];
      if (act) {
        sn = __fmaf_rn(d.y[r], d.sigma, d.mu);
        const float mb = cx.minus_beta[d.replica[r].idx_tmp];
        pass = gd_metropolis(sn, d.s_cur[r], mb, d.u1[r]);
      }
      d.s_new[r] = sn;
      if (trace && !pass) {
        const size_t o = (size_t)r * d.tr_cap + ti;
        d.tr_s[o] = sn;
        d.tr_e[o] = __int_as_float(0x7fc00000);
        d.tr_flag[o] = 0;
      }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, pass);
    if (lane == 0) wsum[warp] = __popc(bal);
    __syncthreads();
    int pre = 0, tot = 0;
    for (int w = 0; w < nw; ++w) {
      const int v = wsum[w];
      pre += w < warp ? v : 0;
      tot += v;
    }
    if (pass) {
      const int pos = G.b0 + base + pre + __popc(bal & ((1u << lane) - 1u));
      d.pose_rep[pos] = r;
#pragma unroll
      for (int k = 0; k < 6; ++k) d.pose_mm[(size_t)pos * 6 + k] = d.mm_prop[(size_t)r * 6 + k];
      d.pose_lc[pos] = d.replica[r].idx_lig;
    }
    base += tot;
    __syncthreads(); /* wsum is rewritten by the next round */
  }
  for (int i = tid; i < G.n_tiles; i += blockDim.x) {
    GdTileDesc t;
    t.complex_index = G.ci;
    t.prt_conf = G.pc;
    t.rep_begin = G.b0 + i * G.k;
    t.count = max(0, min(G.k, base - i * G.k));
    d.tiles[G.tile_base + i] = t;
  }
  if (tid == 0) {
    d.group_cnt[blockIdx.x] = base;
    unsigned long long *st = d.stats + (size_t)G.ci * GD_DA_NSTAT;
    if (act) {
      atomicAdd(st + GD_DA_PROPOSED, (unsigned long long)G.n);
      atomicAdd(st + GD_DA_PASSED, (unsigned long long)base);
    } else {
      atomicAdd(st + GD_DA_PLAIN, (unsigned long long)G.n);
    }
  }
}

__global__ void __launch_bounds__(256) stage2_kernel(GdDaDev d, int step0, int collect) {
  const GdGroup G = d.groups[blockIdx.x];
  const GdDevComplex &cx = d.cx[G.ci];
  const bool act = !collect && d.active[G.ci];
  const int cnt = d.group_cnt[blockIdx.x];
  const int tid = threadIdx.x;
  const int step = cur_step(d, step0);
  const int ti = step - d.tr_step0;
  const bool trace = d.tr_flag && ti >= 0 && ti < d.tr_cap;
  int nacc = 0;
  double e2 = 0.0;
  for (int i = tid; i < cnt; i += blockDim.x) {
    const int pos = G.b0 + i, r = d.pose_rep[pos];
    const gd_energy en = d.pose_e[pos];
    const float enew = en.e[GD_MAXWEI - 1];
    const float eold = d.e_old[r].e[GD_MAXWEI - 1];
    const gd_replica rp = d.replica[r];
    const float mb = cx.minus_beta[rp.idx_tmp];
    const float sn = d.s_new[r], so = d.s_cur[r];
    const int acc = gd_da_stage2(enew, eold, sn, so, mb, d.u2[r]);
    if (act) {
      const double e = (double)sn - (double)enew;
      e2 += e * e;
    }
    if (collect && d.smp_cap > 0) {
      const long long idx = ((long long)step * d.n_rep + r) % d.smp_cap;
      const uint4 *src = reinterpret_cast<const uint4 *>(d.X + (size_t)r * GD_MLP_IN);
      uint4 *dst = reinterpret_cast<uint4 *>(d.smp_X + (size_t)idx * GD_MLP_IN);
#pragma unroll
      for (int v = 0; v < 8; ++v) dst[v] = src[v];
      d.smp_conf[idx] = d.conf[r];
      d.smp_t[idx] = enew;
    }
    if (trace) {
      const size_t o = (size_t)r * d.tr_cap + ti;
      d.tr_s[o] = sn;
      d.tr_e[o] = enew;
      d.tr_flag[o] = 1 + acc;
    }
    if (acc) {
      ++nacc;
      d.e_old[r] = en;
      d.etotal[r] = enew;
#pragma unroll
      for (int k = 0; k < 6; ++k) d.mm_old[(size_t)r * 6 + k] = d.pose_mm[(size_t)pos * 6 + k];
      d.n_accept[r] += 1;
      d.s_cur[r] = sn;
      if (d.rec) {
        const int kslot = d.rec_next[r];
        if (kslot < d.rec_cap) {
          gd_record_step *q = d.rec + (size_t)r * d.rec_cap + kslot;
          q->replica = rp;
          q->energy = en;
#pragma unroll
          for (int k = 0; k < 6; ++k) q->movematrix[k] = d.pose_mm[(size_t)pos * 6 + k];
          q->step = step;
          d.rec_next[r] = kslot + 1;
        } else {
          atomicOr(d.errw, GD_DEV_ERR_RECORD_FULL);
        }
      }
    }
  }
  /* block totals, fixed order */
  __shared__ int s_acc[256];
  __shared__ double s_e2[256];
  s_acc[tid] = nacc;
  s_e2[tid] = e2;
  __syncthreads();
  for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
    if (tid < o) {
      s_acc[tid] += s_acc[tid + o];
      s_e2[tid] += s_e2[tid + o];
    }
    __syncthreads();
  }
  if (tid == 0) {
    unsigned long long *st = d.stats + (size_t)G.ci * GD_DA_NSTAT;
    atomicAdd(st + (act ? GD_DA_ACCEPTED : GD_DA_PLAIN_ACC), (unsigned long long)s_acc[0]);
    if (act && cnt) {
      atomicAdd(d.err + (size_t)G.ci * GD_DA_NERR, s_e2[0]);
      atomicAdd(d.err + (size_t)G.ci * GD_DA_NERR + 1, (double)cnt);
    }
  }
}

/* 8 threads per row, 16 bytes each */
__global__ void gather_kernel(GdDaDev d, long long start, long long n_valid, int rows, int iter,
                              float *t) {
  const int row = blockIdx.x * (blockDim.x >> 3) + (threadIdx.x >> 3), part = threadIdx.x & 7;
  if (row >= rows) return;
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

}  // namespace

void da_propose(const GdDaDev &d, int step0, bool current, cudaStream_t s) {
  propose_kernel<<<nblk(d.n_rep, 128), 128, 0, s>>>(d, step0, current ? 1 : 0);
}

void da_pose_features(const GdDaDev &d, int ci, int pc, int lc, const float *mm, int n,
                      cudaStream_t s) {
  pose_features_kernel<<<nblk(n, 128), 128, 0, s>>>(d, ci, pc, lc, mm, n);
}

void da_set_current(const GdDaDev &d, cudaStream_t s) {
  set_current_kernel<<<nblk(d.n_rep, 256), 256, 0, s>>>(d);
}

void da_stage1(const GdDaDev &d, int step0, bool collect, cudaStream_t s) {
  stage1_kernel<<<d.n_groups, 256, 0, s>>>(d, step0, collect ? 1 : 0);
}

void da_stage2(const GdDaDev &d, int step0, bool collect, cudaStream_t s) {
  stage2_kernel<<<d.n_groups, 256, 0, s>>>(d, step0, collect ? 1 : 0);
}

void da_gather(const GdDaDev &d, long long start, long long n_valid, int rows, int iter,
               float *t, cudaStream_t s) {
  gather_kernel<<<nblk(rows, 32), 256, 0, s>>>(d, start, n_valid, rows, iter, t);
}

void da_target_moments(const GdDaDev &d, long long start, long long n_valid, float lo, float hi,
                       double *part, cudaStream_t s) {
  moments_kernel<<<GD_DA_MOM_BLOCKS, 256, 0, s>>>(d, start, n_valid, lo, hi, part);
}

}  // namespace gd
