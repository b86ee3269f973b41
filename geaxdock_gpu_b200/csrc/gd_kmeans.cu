/*
 * gd_kmeans.cu -- the k-means of the post-Monte-Carlo clustering on the GPU, many independent
 * problems (segments) per launch.
 *
 * Reference: clusterByKmeans (src/util.C:1801-1880) over seq_kmeans (src/seq_kmeans.c): the
 * records of a segment are shuffled, the first k become the initial centres, then Lloyd
 * iterations (nearest centre by squared Euclidean distance, ties to the lower index; centres
 * = member means) run while more than `threshold` of the objects changed cluster and at most
 * 501 passes; the representative of a cluster is its last member in shuffled order (the
 * reference's medoid loop never updates its running distance, so it keeps the last member).
 *
 * The shuffle here is a seeded pseudorandom permutation of each segment's positions: a
 * 4-round balanced Feistel network on the smallest even power of two covering the segment,
 * with cycle walking (every position is mapped independently, so the permutation needs no
 * sort); round keys come from the seed and the segment index through the lowbias32 integer
 * hash (C. Wellons). The reference shuffles with an unseeded random_shuffle, so only the
 * distribution of orders can be matched, not the order itself.
 *
 * Every float operation is the reference's, in its order: the distance sums the squared
 * coordinate differences dimension by dimension (no fused multiply-add); a centre sums its
 * members' coordinates in shuffled order and divides by the member count. One thread per
 * object assigns. For small segments one thread per cluster walks its segment in order to sum
 * its members; for large ones (the pooled second stage) a stable radix sort of the objects by
 * cluster (CUB) lists each cluster's members in order and one thread per (cluster,
 * coordinate) sums them.
 * A segment stops iterating on its own criterion; the host polls one counter per pass.
 */
#include <cuda_runtime.h>

#include <cstdint>
#include <cub/device/device_radix_sort.cuh>
#include <vector>

#include "gd_kmeans.cuh"

namespace gd {
namespace {

__host__ __device__ inline uint32_t lowbias32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

struct PermKeys {
  uint32_t k[4];
  int half; /* bits per half */
};

__host__ __device__ inline PermKeys perm_keys(uint64_t seed, int seg, int n) {
  PermKeys p;
  int b = 0;
  while ((1u << b) < (uint32_t)n) ++b;
  if (b & 1) ++b;
  p.half = b / 2;
  for (int r = 0; r < 4; ++r)
    p.k[r] = lowbias32((uint32_t)seed ^
                       lowbias32((uint32_t)(seed >> 32) + 0x9E3779B9u * (uint32_t)(seg * 4 + r + 1)));
  return p;
}

/* position i (0 <= i < n) of the shuffled segment holds object perm_index(i) */
__host__ __device__ inline int perm_index(int i, int n, const PermKeys &p) {
  if (n <= 1) return 0;
  const uint32_t mask = (1u << p.half) - 1u;
  uint32_t x = (uint32_t)i;
  do {
    uint32_t l = x >> p.half, r = x & mask;
    for (int k = 0; k < 4; ++k) {
      const uint32_t f = lowbias32(r ^ p.k[k]) & mask;
      const uint32_t nl = r;
      r = l ^ f;
      l = nl;
    }
    x = (l << p.half) | r;
  } while (x >= (uint32_t)n);
  return (int)x;
}

struct Seg {
  int off, n, k, cbase; /* objects [off, off + n), clusters [cbase, cbase + k) */
};

__global__ void gather_kernel(const float *__restrict__ obj, int dim, const Seg *__restrict__ seg,
                              const int *__restrict__ seg_of, int n_obj, uint64_t seed,
                              float *__restrict__ sh, int *__restrict__ perm) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_obj) return;
  const int s = seg_of[p];
  const Seg g = seg[s];
  const PermKeys pk = perm_keys(seed, s, g.n);
  const int src = g.off + perm_index(p - g.off, g.n, pk);
  perm[p] = src;
  for (int j = 0; j < dim; ++j) sh[(size_t)p * dim + j] = obj[(size_t)src * dim + j];
}

__global__ void init_centres(const float *__restrict__ sh, int dim, const Seg *__restrict__ seg,
                             const int *__restrict__ cseg, int n_cl, float *__restrict__ cen) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cl) return;
  const Seg g = seg[cseg[c]];
  for (int j = 0; j < dim; ++j)
    cen[(size_t)c * dim + j] = sh[(size_t)(g.off + (c - g.cbase)) * dim + j];
}

/* Nearest centre of each object. The centres of the clusters of every segment the block's
 * objects belong to (a contiguous range) are staged in shared memory when they fit (SMEM_CL
 * clusters), so that the 9 x k loads per object are shared-memory broadcasts. */
constexpr int SMEM_CL = 1024;

template <int D>
__global__ void __launch_bounds__(256) assign_kernel(
    const float *__restrict__ sh, const Seg *__restrict__ seg, const int *__restrict__ seg_of,
    const unsigned char *__restrict__ act, int n_obj, const float *__restrict__ cen,
    int *__restrict__ mem, int *__restrict__ changed) {
  __shared__ float sc[SMEM_CL * D];
  const int p0 = blockIdx.x * blockDim.x;
  const int pl = min(p0 + (int)blockDim.x, n_obj) - 1;
  const int c0 = seg[seg_of[p0]].cbase;
  const Seg gl = seg[seg_of[pl]];
  const int nc = gl.cbase + gl.k - c0;
  const bool staged = nc <= SMEM_CL;
  if (staged)
    for (int i = threadIdx.x; i < nc * D; i += blockDim.x) sc[i] = cen[(size_t)c0 * D + i];
  __syncthreads();
  const int p = p0 + threadIdx.x;
  if (p >= n_obj) return;
  const int s = seg_of[p];
  if (!act[s]) return;
  const Seg g = seg[s];
  const float *cb = staged ? sc + (size_t)(g.cbase - c0) * D : cen + (size_t)g.cbase * D;
  float o[D];
#pragma unroll
  for (int j = 0; j < D; ++j) o[j] = sh[(size_t)p * D + j];
  int best = 0;
  float best_d = 0.0f;
  for (int c = 0; c < g.k; ++c) {
    const float *q = cb + (size_t)c * D;
    float d = 0.0f;
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const float t = __fsub_rn(o[j], q[j]);
      d = __fadd_rn(d, __fmul_rn(t, t));
    }
    if (c == 0 || d < best_d) {
      best_d = d;
      best = c;
    }
  }
  if (mem[p] != best) atomicAdd(changed + s, 1);
  mem[p] = best;
}

template <int D>
__global__ void update_kernel(const float *__restrict__ sh, const Seg *__restrict__ seg,
                              const int *__restrict__ cseg, const unsigned char *__restrict__ act,
                              int n_cl, const int *__restrict__ mem, float *__restrict__ cen) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cl) return;
  const int s = cseg[c];
  if (!act[s]) return;
  const Seg g = seg[s];
  const int kc = c - g.cbase;
  float sum[D];
#pragma unroll
  for (int j = 0; j < D; ++j) sum[j] = 0.0f;
  int cnt = 0;
  for (int p = g.off; p < g.off + g.n; ++p) {
    if (mem[p] != kc) continue;
    ++cnt;
#pragma unroll
    for (int j = 0; j < D; ++j) sum[j] = __fadd_rn(sum[j], sh[(size_t)p * D + j]);
  }
  if (cnt > 0) {
#pragma unroll
    for (int j = 0; j < D; ++j) cen[(size_t)c * D + j] = __fdiv_rn(sum[j], (float)cnt);
  }
}

__global__ void cluster_key_kernel(const Seg *__restrict__ seg, const int *__restrict__ seg_of,
                                   const int *__restrict__ mem, int n_obj, int *__restrict__ key,
                                   int *__restrict__ pos) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_obj) return;
  const int m = mem[p];
  key[p] = m >= 0 ? seg[seg_of[p]].cbase + m : 0x7fffffff;
  pos[p] = p;
}

/* first / one-past-last index of each cluster in the sorted key array */
__global__ void bounds_kernel(const int *__restrict__ key, int n_obj, int n_cl,
                              int *__restrict__ begin, int *__restrict__ end) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_obj) return;
  const int k = key[i];
  if (k >= n_cl) return;
  if (i == 0 || key[i - 1] != k) begin[k] = i;
  if (i == n_obj - 1 || key[i + 1] != k) end[k] = i + 1;
}

/* centre = in-order sum of its members / count, one thread per (cluster, coordinate) */
__global__ void update_sorted_kernel(const float *__restrict__ sh, int dim,
                                     const int *__restrict__ cseg,
                                     const unsigned char *__restrict__ act, int n_cl,
                                     const int *__restrict__ begin, const int *__restrict__ end,
                                     const int *__restrict__ pos, float *__restrict__ cen) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_cl * dim) return;
  const int c = t / dim, j = t - c * dim;
  if (!act[cseg[c]]) return;
  const int b = begin[c], e = end[c];
  if (e <= b) return;
  float s = 0.0f;
  /* 16 gathers in flight ahead of the (ordered) additions */
  int i = b;
  for (; i + 16 <= e; i += 16) {
    int q[16];
    float v[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) q[u] = pos[i + u];
#pragma unroll
    for (int u = 0; u < 16; ++u) v[u] = sh[(size_t)q[u] * dim + j];
#pragma unroll
    for (int u = 0; u < 16; ++u) s = __fadd_rn(s, v[u]);
  }
  for (; i < e; ++i) s = __fadd_rn(s, sh[(size_t)pos[i] * dim + j]);
  cen[(size_t)c * dim + j] = __fdiv_rn(s, (float)(e - b));
}

/* per segment: delta = changed / n (float); keep iterating while delta > threshold and the
 * pass counter (post-incremented, as `loop++ < 500`) is below max_iter */
__global__ void step_kernel(const Seg *__restrict__ seg, int n_seg, int *__restrict__ changed,
                            int *__restrict__ loops, unsigned char *__restrict__ act,
                            float threshold, int max_iter, int *__restrict__ n_active) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_seg) return;
  if (act[s]) {
    const float delta = __fdiv_rn((float)changed[s], (float)seg[s].n);
    const bool more = delta > threshold && loops[s]++ < max_iter;
    act[s] = more ? 1 : 0;
    if (more) atomicAdd(n_active, 1);
  }
  changed[s] = 0;
}

/* the same from the sorted member lists (last member = the largest position in the list) */
__global__ void medoid_sorted_kernel(int n_cl, const int *__restrict__ begin,
                                     const int *__restrict__ end, const int *__restrict__ pos,
                                     const int *__restrict__ perm, int *__restrict__ medoid,
                                     int *__restrict__ size) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cl) return;
  const int b = begin[c], e = end[c];
  medoid[c] = e > b ? perm[pos[e - 1]] : -1;
  size[c] = e > b ? e - b : 0;
}

__global__ void medoid_kernel(const Seg *__restrict__ seg, const int *__restrict__ cseg, int n_cl,
                              const int *__restrict__ mem, const int *__restrict__ perm,
                              int *__restrict__ medoid, int *__restrict__ size) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n_cl) return;
  const Seg g = seg[cseg[c]];
  const int kc = c - g.cbase;
  int last = -1, cnt = 0;
  for (int p = g.off; p < g.off + g.n; ++p)
    if (mem[p] == kc) {
      last = p;
      ++cnt;
    }
  medoid[c] = last >= 0 ? perm[last] : -1;
  size[c] = cnt;
}

__global__ void unshuffle_kernel(const int *__restrict__ perm, const int *__restrict__ mem,
                                 int n_obj, int *__restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n_obj) out[perm[p]] = mem[p];
}

template <class T>
cudaError_t dmalloc(T **p, size_t n) {
  return cudaMalloc(reinterpret_cast<void **>(p), (n ? n : 1) * sizeof(T));
}

}  // namespace

int kmeans_permutation(uint64_t seed, int seg, int n, int *out) {
  const PermKeys pk = perm_keys(seed, seg, n);
  for (int i = 0; i < n; ++i) out[i] = perm_index(i, n, pk);
  return 0;
}

int kmeans_device(const KmeansJob &job, KmeansResult &res, std::string &err) {
  const int D = job.dim;
  if (D != 9) {
    err = "k-means is built for 9 coordinates (the energy terms)";
    return -1;
  }
  const int n_seg = (int)job.seg_off.size() - 1;
  std::vector<Seg> seg(n_seg);
  std::vector<int> seg_of, cseg;
  int n_obj = job.seg_off.back(), n_cl = 0;
  seg_of.resize(n_obj);
  for (int s = 0; s < n_seg; ++s) {
    Seg &g = seg[s];
    g.off = job.seg_off[s];
    g.n = job.seg_off[s + 1] - g.off;
    /* fewer objects than clusters: not clustered, every object is its own cluster in its
     * original order (clusterByKmeans returns the records as they are) */
    g.k = job.k[s] <= g.n ? job.k[s] : g.n;
    g.cbase = n_cl;
    n_cl += g.k;
    for (int p = g.off; p < g.off + g.n; ++p) seg_of[p] = s;
    for (int c = 0; c < g.k; ++c) cseg.push_back(s);
  }
  res.membership.assign(n_obj, -1);
  res.medoid.assign(n_cl, -1);
  res.size.assign(n_cl, 0);
  res.cluster_base.resize(n_seg);
  for (int s = 0; s < n_seg; ++s) res.cluster_base[s] = seg[s].cbase;
  res.passes.assign(n_seg, 0);
  if (n_obj == 0 || n_cl == 0) return 0;

  float *obj = nullptr, *sh = nullptr, *cen = nullptr;
  Seg *dseg = nullptr;
  int *dseg_of = nullptr, *dcseg = nullptr, *perm = nullptr, *mem = nullptr, *changed = nullptr,
      *loops = nullptr, *n_act = nullptr, *medoid = nullptr, *size = nullptr, *orig = nullptr;
  unsigned char *act = nullptr;
  cudaStream_t st = (cudaStream_t)job.stream;
  cudaError_t e = cudaSuccess;
  auto ok = [&](cudaError_t x) {
    if (e == cudaSuccess) e = x;
    return e == cudaSuccess;
  };
  ok(dmalloc(&obj, (size_t)n_obj * D));
  ok(dmalloc(&sh, (size_t)n_obj * D));
  ok(dmalloc(&cen, (size_t)n_cl * D));
  ok(dmalloc(&dseg, n_seg));
  ok(dmalloc(&dseg_of, n_obj));
  ok(dmalloc(&dcseg, n_cl));
  ok(dmalloc(&perm, n_obj));
  ok(dmalloc(&mem, n_obj));
  ok(dmalloc(&orig, n_obj));
  ok(dmalloc(&changed, n_seg));
  ok(dmalloc(&loops, n_seg));
  ok(dmalloc(&act, n_seg));
  ok(dmalloc(&n_act, 1));
  ok(dmalloc(&medoid, n_cl));
  ok(dmalloc(&size, n_cl));
  int max_n = 0;
  for (const Seg &g : seg) max_n = g.n > max_n ? g.n : max_n;
  const bool sorted = max_n > 8192;
  int *key = nullptr, *key2 = nullptr, *pos = nullptr, *pos2 = nullptr, *cb = nullptr,
      *ce = nullptr;
  void *tmp = nullptr;
  size_t tmp_bytes = 0;
  if (sorted) {
    ok(dmalloc(&key, n_obj));
    ok(dmalloc(&key2, n_obj));
    ok(dmalloc(&pos, n_obj));
    ok(dmalloc(&pos2, n_obj));
    ok(dmalloc(&cb, n_cl));
    ok(dmalloc(&ce, n_cl));
    ok(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key, key2, pos, pos2, n_obj, 0, 31,
                                       st));
    ok(cudaMalloc(&tmp, tmp_bytes ? tmp_bytes : 1));
  }
  if (e == cudaSuccess) {
    std::vector<unsigned char> a0(n_seg);
    for (int s = 0; s < n_seg; ++s) a0[s] = seg[s].k > 0 && job.k[s] <= seg[s].n;
    ok(cudaMemcpyAsync(obj, job.objects, sizeof(float) * (size_t)n_obj * D,
                       cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(dseg, seg.data(), sizeof(Seg) * n_seg, cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(dseg_of, seg_of.data(), sizeof(int) * n_obj, cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(dcseg, cseg.data(), sizeof(int) * n_cl, cudaMemcpyHostToDevice, st));
    ok(cudaMemcpyAsync(act, a0.data(), n_seg, cudaMemcpyHostToDevice, st));
    ok(cudaMemsetAsync(mem, 0xff, sizeof(int) * n_obj, st));
    ok(cudaMemsetAsync(changed, 0, sizeof(int) * n_seg, st));
    ok(cudaMemsetAsync(loops, 0, sizeof(int) * n_seg, st));
    const int T = 256, bo = (n_obj + T - 1) / T, bc = (n_cl + T - 1) / T, bs = (n_seg + T - 1) / T;
    gather_kernel<<<bo, T, 0, st>>>(obj, D, dseg, dseg_of, n_obj, job.seed, sh, perm);
    init_centres<<<bc, T, 0, st>>>(sh, D, dseg, dcseg, n_cl, cen);
    ok(cudaGetLastError());
    for (int pass = 0; e == cudaSuccess; ++pass) {
      assign_kernel<9><<<bo, T, 0, st>>>(sh, dseg, dseg_of, act, n_obj, cen, mem, changed);
      if (sorted) {
        /* stable by key: each cluster's members in shuffled order */
        cluster_key_kernel<<<bo, T, 0, st>>>(dseg, dseg_of, mem, n_obj, key, pos);
        ok(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, key, key2, pos, pos2, n_obj, 0, 31,
                                           st));
        ok(cudaMemsetAsync(cb, 0, sizeof(int) * n_cl, st));
        ok(cudaMemsetAsync(ce, 0, sizeof(int) * n_cl, st));
        bounds_kernel<<<bo, T, 0, st>>>(key2, n_obj, n_cl, cb, ce);
        update_sorted_kernel<<<(n_cl * D + T - 1) / T, T, 0, st>>>(sh, D, dcseg, act, n_cl, cb,
                                                                     ce, pos2, cen);
      } else {
        update_kernel<9><<<bc, T, 0, st>>>(sh, dseg, dcseg, act, n_cl, mem, cen);
      }
      ok(cudaMemsetAsync(n_act, 0, sizeof(int), st));
      step_kernel<<<bs, T, 0, st>>>(dseg, n_seg, changed, loops, act, job.threshold,
                                    job.max_iter, n_act);
      int h_act = 0;
      ok(cudaMemcpyAsync(&h_act, n_act, sizeof(int), cudaMemcpyDeviceToHost, st));
      ok(cudaStreamSynchronize(st));
      if (h_act == 0 || pass > job.max_iter + 1) break;
    }
    if (sorted) {
      /* member lists of the final memberships */
      cluster_key_kernel<<<bo, T, 0, st>>>(dseg, dseg_of, mem, n_obj, key, pos);
      ok(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, key, key2, pos, pos2, n_obj, 0, 31, st));
      ok(cudaMemsetAsync(cb, 0, sizeof(int) * n_cl, st));
      ok(cudaMemsetAsync(ce, 0, sizeof(int) * n_cl, st));
      bounds_kernel<<<bo, T, 0, st>>>(key2, n_obj, n_cl, cb, ce);
      medoid_sorted_kernel<<<bc, T, 0, st>>>(n_cl, cb, ce, pos2, perm, medoid, size);
    } else {
      medoid_kernel<<<bc, T, 0, st>>>(dseg, dcseg, n_cl, mem, perm, medoid, size);
    }
    unshuffle_kernel<<<bo, T, 0, st>>>(perm, mem, n_obj, orig);
    ok(cudaGetLastError());
    ok(cudaMemcpyAsync(res.membership.data(), orig, sizeof(int) * n_obj, cudaMemcpyDeviceToHost,
                       st));
    ok(cudaMemcpyAsync(res.medoid.data(), medoid, sizeof(int) * n_cl, cudaMemcpyDeviceToHost, st));
    ok(cudaMemcpyAsync(res.size.data(), size, sizeof(int) * n_cl, cudaMemcpyDeviceToHost, st));
    ok(cudaMemcpyAsync(res.passes.data(), loops, sizeof(int) * n_seg, cudaMemcpyDeviceToHost,
                       st));
    ok(cudaStreamSynchronize(st));
  }
  void *ps[] = {obj, sh, cen, dseg, dseg_of, dcseg, perm, mem, orig, changed, loops, act, n_act,
                medoid, size, key, key2, pos, pos2, cb, ce, tmp};
  for (void *p : ps)
    if (p) cudaFree(p);
  if (e != cudaSuccess) {
    err = cudaGetErrorString(e);
    return -2;
  }
  /* passes = loop + 1 of the reference (its loop_iterations) */
  for (int s = 0; s < n_seg; ++s) {
    const Seg &g = seg[s];
    if (job.k[s] > g.n) {
      for (int c = 0; c < g.n; ++c) {
        res.medoid[g.cbase + c] = g.off + c;
        res.size[g.cbase + c] = 1;
        res.membership[g.off + c] = c;
      }
      res.passes[s] = 0;
    } else {
      res.passes[s] = g.k > 0 ? res.passes[s] + 1 : 0;
    }
  }
  return 0;
}

}  // namespace gd
