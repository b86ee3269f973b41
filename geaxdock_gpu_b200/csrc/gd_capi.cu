/*
 * gd_capi.cu -- host side of the C ABI declared in include/geauxdock_b200.h.
 *
 * Replaces the reference's Run (src/run.cu:33-288) and its single-GPU launcher loop
 * (src/kernel_cuda_lancher_siglegpu.cu:1-71): instead of ~40 cudaMemcpyToSymbol calls and a
 * synchronous launch per 10 steps, a context owns its device buffers and one stream, turns
 * each complex into the kernel-ready layout once (points sorted by type, segments, folded
 * pair parameters, sparse contact reference), and launches the persistent kernel of
 * gd_kernels.cu, optionally as a captured CUDA graph.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "gd_device.cuh"
#include "gd_kmeans.cuh"
#include "gd_mlp.cuh"
#include "gd_numerics.h"

namespace gd {
template <int UNROLL, bool SPLIT, bool DA, int PACK>
__global__ void gd_mc_kernel(GdMcArgs a, GdForceConst f);
#define GD_EXT(U, S, D, P) \
  extern template __global__ void gd_mc_kernel<U, S, D, P>(GdMcArgs, GdForceConst);
GD_EXT(1, false, false, 1) GD_EXT(2, false, false, 1) GD_EXT(4, false, false, 1)
GD_EXT(1, true, false, 1) GD_EXT(2, true, false, 1) GD_EXT(4, true, false, 1)
GD_EXT(1, false, true, 1) GD_EXT(2, false, true, 1) GD_EXT(4, false, true, 1)
GD_EXT(1, true, true, 1) GD_EXT(2, true, true, 1) GD_EXT(4, true, true, 1)
GD_EXT(1, false, false, 2) GD_EXT(2, false, false, 2)
#undef GD_EXT
__global__ void gd_exchange_kernel(const GdDevComplex *cxs, const int *group_base, int n_complex,
                                   int g_begin, int g_end, gd_replica *replica,
                                   const float *etotal, int *acs, uint64_t seed,
                                   const int *call_base, int call_off, int mode_t);
__global__ void gd_reset_records_kernel(int *rec_next, int r0, int r1);
}  // namespace gd

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return fail(GD_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                               \
  } while (0)

const float kPi = 3.1415926535f; /* reference src/size.h:67 */

/* largest float d2 with sqrtf(d2) <= pmf0, -1 when none */
float contact_threshold(float pmf0) {
  if (!(pmf0 >= 0.0f)) return -1.0f;
  float t = (float)((double)pmf0 * (double)pmf0);
  while (t > 0.0f && sqrtf(t) > pmf0) t = nextafterf(t, -INFINITY);
  while (sqrtf(nextafterf(t, INFINITY)) <= pmf0) t = nextafterf(t, INFINITY);
  return t;
}

float bits_as_float(int v) {
  float f;
  memcpy(&f, &v, sizeof(f));
  return f;
}

float host_dist2(float ax, float ay, float az, float px, float py, float pz) {
  const float dx = ax - px, dy = ay - py, dz = az - pz;
  return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
}

struct ComplexInfo {
  int n_lig, n_prt, n_tmp, lna, pnp, pnp_pad, pnk, pos;
  int rep_offset, n_rep, k;
  int stream;
  int types_uniform; /* every ligand conformer has the same atom types (two replicas per
                        thread share their atom's pair parameters) */
};

/* One chain of the fused loops: a contiguous range of (complex, protein conformer) blocks,
 * their replicas, exchange groups and tiles. Chains share nothing, so the graph runs them on
 * separate streams and one chain's kernels fill the other's tail. */
struct Chain {
  int g0, g1;    /* blocks [g0, g1) in (complex, protein conformer) order */
  int r0, r1;    /* replicas */
  int xg0, xg1;  /* exchange groups */
  int t_off, t_cnt; /* plain tiles in the chain tile list */
};

}  // namespace

struct gd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  gd_mc_params mc{};
  int n_complex = 0, n_rep = 0, n_groups = 0;
  int threads = 256, chunk = 512, unroll = 2, split = 1, num_sms = 148;
  int pack = 1; /* replicas per thread of the plain launches: the tile's lanes (threads) run on
                   threads / pack threads */
  int fill_threads = 0, fill_cap = 0; /* the last gd_set_tile in fill mode (threads > 0) */
  std::vector<ComplexInfo> info;
  std::vector<void *> allocs;
  GdForceConst fc{};
  GdDevComplex *d_cx = nullptr;
  GdPairParam *d_pp = nullptr;
  int *d_group_base = nullptr;
  /* replica state */
  gd_replica *d_replica = nullptr;
  float *d_mm = nullptr;
  gd_energy *d_eold = nullptr;
  float *d_etotal = nullptr;
  int *d_nacc = nullptr, *d_acs = nullptr;
  gd_record_step *d_rec = nullptr;
  int *d_rec_next = nullptr;
  int rec_cap = 0;
  /* work lists */
  GdTileDesc *d_tiles = nullptr;
  int tiles_cap = 0;
  int tiles_r0 = -1, tiles_r1 = -1, tiles_n = 0, tiles_gen = -1, tile_gen = 0;
  std::vector<GdTileDesc> full_tiles;
  int *d_counters = nullptr; /* [counters_cap] persistent-CTA queue heads */
  int counters_cap = 0;
  int *d_cursor = nullptr;   /* [2]: step base, exchange call base (graph replays) */
  int *h_cursor = nullptr;   /* pinned staging */
  unsigned *d_err = nullptr;
  bool initialized = false;
  int exchange_calls = 0;
  /* trace */
  float *d_trace_e = nullptr;
  int *d_trace_acc = nullptr;
  int trace_cap = 0, trace_step0 = 0, trace_steps = 0;
  /* graph cache */
  std::map<long long, cudaGraphExec_t> graphs;
  /* pose evaluation scratch */
  float *d_mm_in = nullptr;
  int *d_lc_in = nullptr;
  gd_energy *d_e_out = nullptr;
  int eval_cap = 0;
  GdTileDesc *d_eval_tiles = nullptr;
  int eval_tiles_cap = 0;
  long long timeout_ns = 2000000000LL;
  /* surrogate and delayed acceptance (gd_sur_create) */
  struct DaState *da = nullptr;
  /* concurrent chains of the fused loops: plain (gd_mc_run_fused) and delayed acceptance */
  int chains = 1, chains_da = 3;
  std::vector<cudaStream_t> aux;             /* streams of chains 1.. */
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
  std::vector<Chain> chain;
  int chain_gen = -1;
  GdTileDesc *d_chain_tiles = nullptr;
  int chain_tiles_cap = 0;
  /* record streaming into host memory (gd_records_stream) */
  struct RecStream *rs = nullptr;
};

/* Copy plan of one record-stream snapshot, one block: for every replica the rows written since
 * the previous snapshot (counters in prev, clamped to the host array's cap) start at start[r]
 * and go to off[r] of the packed buffer; off[n_rep] is the total. prev takes the new counters,
 * cnt keeps them for the host. *overflow is set when the total exceeds the packed buffer's
 * pack_rows (then nothing is gathered). */
__global__ void rs_plan_kernel(const int *__restrict__ cur, int *__restrict__ prev, int n_rep,
                               int cap, long long pack_rows, int *__restrict__ start,
                               int *__restrict__ off, int *__restrict__ cnt, int *overflow) {
  __shared__ int part[1024];
  const int T = blockDim.x, t = threadIdx.x;
  const int per = (n_rep + T - 1) / T, r0 = min(n_rep, t * per), r1 = min(n_rep, r0 + per);
  int sum = 0;
  for (int r = r0; r < r1; ++r)
    sum += max(0, min(cur[r], cap) - min(prev[r], cap));
  part[t] = sum;
  __syncthreads();
  for (int o = 1; o < T; o <<= 1) {
    const int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int base = t ? part[t - 1] : 0;
  for (int r = r0; r < r1; ++r) {
    const int c = cur[r], a = min(prev[r], cap);
    start[r] = a;
    off[r] = base;
    base += max(0, min(c, cap) - a);
    prev[r] = c;
    cnt[r] = c;
  }
  if (t == T - 1) {
    off[n_rep] = part[T - 1];
    *overflow = (long long)part[T - 1] > pack_rows ? 1 : 0;
  }
}

/* rows [start[r], start[r] + off[r+1] - off[r]) of every replica's records packed at off[r],
 * one warp per replica copying 4-byte words */
__global__ void rs_gather_kernel(const gd_record_step *__restrict__ rec, int rec_cap,
                                 const int *__restrict__ start, const int *__restrict__ off,
                                 int n_rep, long long pack_rows, gd_record_step *__restrict__ out) {
  const int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= n_rep || (long long)off[n_rep] > pack_rows) return;
  constexpr int WORDS = sizeof(gd_record_step) / 4;
  const uint32_t *src =
      reinterpret_cast<const uint32_t *>(rec + (size_t)w * rec_cap + start[w]);
  uint32_t *dst = reinterpret_cast<uint32_t *>(out + off[w]);
  const int n = (off[w + 1] - off[w]) * WORDS;
  for (int i = lane; i < n; i += 32) dst[i] = src[i];
}

/* The record stream of gd_records_stream. After each record-writing call the calling thread
 * queues, on the context's stream, the copy plan and the gather of every replica's rows
 * written since the previous snapshot into a packed device buffer of a free snapshot slot
 * (records are appended only, so they are complete); stream order keeps the gather off the
 * SMs while the Monte Carlo kernels run. A worker thread waits for the slot, downloads the plan
 * and the packed rows into page-locked host memory on its own stream (a copy engine, no SMs)
 * and copies them into the caller's array, while the context's stream runs the next work. */
struct RecStream {
  static constexpr int NSNAP = 4;
  gd_record_step *host = nullptr;
  int cap = 0, n_rep = 0, rec_cap = 0, device = 0;
  const gd_record_step *d_rec = nullptr;
  cudaStream_t cs = nullptr;
  int *d_prev = nullptr;                           /* [n_rep] counters of the last snapshot */
  int *d_plan[NSNAP] = {};                         /* start [n_rep], off [n_rep+1], cnt [n_rep],
                                                      overflow [1] */
  gd_record_step *d_pack[NSNAP] = {};
  long long pack_rows[NSNAP] = {};
  cudaEvent_t ev[NSNAP] = {};
  bool busy[NSNAP] = {};
  int *h_plan = nullptr;                           /* page-locked copy of one slot's plan */
  gd_record_step *h_stage = nullptr;               /* page-locked packed rows */
  size_t stage_cap = 0;
  std::deque<int> queue;
  std::mutex mu;
  std::condition_variable cv;
  bool stop = false;
  std::vector<int> snap; /* the counters of the latest snapshot copied */
  cudaError_t err = cudaSuccess;
  bool overflow = false;
  std::thread th;

  size_t plan_ints() const { return 3 * (size_t)n_rep + 2; }

  /* downloads slot k's rows into the caller's array; *ovf: the slot's rows exceeded its
   * packed buffer and nothing was gathered */
  cudaError_t one(int k, bool *ovf) {
    int *start = h_plan, *off = h_plan + n_rep, *cnt = off + n_rep + 1;
    cudaError_t e = cudaMemcpyAsync(h_plan, d_plan[k], sizeof(int) * plan_ints(),
                                    cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    if (e != cudaSuccess) return e;
    *ovf = cnt[n_rep] != 0;
    if (*ovf) return cudaSuccess;
    const size_t total = (size_t)off[n_rep];
    if (total > 0) {
      if (total > stage_cap) {
        if (h_stage) cudaFreeHost(h_stage);
        h_stage = nullptr;
        stage_cap = 0;
        const size_t want = total + total / 4;
        e = cudaHostAlloc(&h_stage, want * sizeof(gd_record_step), cudaHostAllocDefault);
        if (e != cudaSuccess) return e;
        stage_cap = want;
      }
      e = cudaMemcpyAsync(h_stage, d_pack[k], total * sizeof(gd_record_step),
                          cudaMemcpyDeviceToHost, cs);
      if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
      if (e != cudaSuccess) return e;
      for (int r = 0; r < n_rep; ++r)
        if (off[r + 1] > off[r])
          memcpy(host + (size_t)r * cap + start[r], h_stage + off[r],
                 sizeof(gd_record_step) * (size_t)(off[r + 1] - off[r]));
    }
    std::lock_guard<std::mutex> lk(mu);
    snap.assign(cnt, cnt + n_rep);
    return cudaSuccess;
  }

  void worker() {
    cudaSetDevice(device);
    for (;;) {
      int k;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop || !queue.empty(); });
        if (queue.empty()) return;
        k = queue.front();
      }
      bool ovf = false;
      cudaError_t e = cudaEventSynchronize(ev[k]);
      if (e == cudaSuccess) e = one(k, &ovf);
      {
        std::lock_guard<std::mutex> lk(mu);
        if (e != cudaSuccess && err == cudaSuccess) err = e;
        if (ovf) overflow = true;
        queue.pop_front();
        busy[k] = false;
      }
      cv.notify_all();
    }
  }
};

namespace {

/* Device -> host copy of n rows (width bytes each; device pitch dpitch, host pitch hpitch). A
 * large download into freshly allocated pageable memory is bound by the first touch of every
 * host page (one thread faults pages in at about a quarter of the copy rate of resident pages),
 * so above 32 MB the destination rows are first written by up to 8 host threads in parallel,
 * then copied in one call. */
cudaError_t d2h_rows(void *dst, size_t hpitch, const void *src, size_t dpitch, size_t width,
                     int n) {
  if (n < 1 || width == 0) return cudaSuccess;
  int T = (int)std::min(8u, std::max(1u, std::thread::hardware_concurrency()));
  if (width * (size_t)n < ((size_t)32 << 20)) T = 1;
  T = std::min(T, n);
  if (T > 1) {
    auto touch = [&](int t) {
      const int a = (int)((long long)n * t / T), b = (int)((long long)n * (t + 1) / T);
      char *d = static_cast<char *>(dst) + (size_t)a * hpitch;
      if (hpitch == width)
        memset(d, 0, (size_t)(b - a) * width);
      else
        for (int i = a; i < b; ++i, d += hpitch) memset(d, 0, width);
    };
    std::vector<std::thread> th;
    for (int t = 1; t < T; ++t) th.emplace_back(touch, t);
    touch(0);
    for (auto &x : th) x.join();
  }
  return cudaMemcpy2D(dst, hpitch, src, dpitch, width, n, cudaMemcpyDeviceToHost);
}

/* queues a snapshot taken after the work queued on the context's stream so far: the copy plan
 * and the gather of the rows written since the previous snapshot, at most rows_per_rep per
 * replica (the steps of the call that wrote them). No-op without gd_records_stream. */
int rs_enqueue(gd_ctx *c, int rows_per_rep) {
  RecStream *r = c->rs;
  if (!r) return GD_OK;
  int k = -1;
  {
    std::unique_lock<std::mutex> lk(r->mu);
    r->cv.wait(lk, [&] {
      if (r->err != cudaSuccess || r->overflow) return true;
      for (int i = 0; i < RecStream::NSNAP; ++i)
        if (!r->busy[i]) return true;
      return false;
    });
    if (r->err != cudaSuccess)
      return fail(GD_ERR_CUDA, "record stream: %s", cudaGetErrorString(r->err));
    if (r->overflow) return fail(GD_ERR_STATE, "record stream: more rows than the writing calls queued");
    for (int i = 0; i < RecStream::NSNAP && k < 0; ++i)
      if (!r->busy[i]) k = i;
    r->busy[k] = true;
  }
  const long long need = (long long)r->n_rep * std::min(r->cap, std::max(0, rows_per_rep));
  cudaError_t e = cudaSuccess;
  if (need > r->pack_rows[k]) {
    /* the slot is idle: no copy reads its buffer */
    if (r->d_pack[k]) cudaFree(r->d_pack[k]);
    r->d_pack[k] = nullptr;
    r->pack_rows[k] = 0;
    e = cudaMalloc(&r->d_pack[k], (size_t)need * sizeof(gd_record_step));
    if (e == cudaSuccess) r->pack_rows[k] = need;
  }
  int *plan = r->d_plan[k], n = r->n_rep;
  if (e == cudaSuccess) {
    rs_plan_kernel<<<1, 1024, 0, c->stream>>>(c->d_rec_next, r->d_prev, n, r->cap,
                                              r->pack_rows[k], plan, plan + n, plan + 2 * n + 1,
                                              plan + 3 * n + 1);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && r->pack_rows[k] > 0) {
    rs_gather_kernel<<<(unsigned)((n + 7) / 8), 256, 0, c->stream>>>(
        r->d_rec, r->rec_cap, plan, plan + n, n, r->pack_rows[k], r->d_pack[k]);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(r->ev[k], c->stream);
  {
    std::lock_guard<std::mutex> lk(r->mu);
    if (e != cudaSuccess) {
      r->busy[k] = false;
      return fail(GD_ERR_CUDA, "record stream: %s", cudaGetErrorString(e));
    }
    r->queue.push_back(k);
  }
  r->cv.notify_all();
  return GD_OK;
}

/* one more snapshot after everything queued (every record-writing call has queued its own, so
 * it finds no new rows), then wait for every copy: the host array mirrors the device records */
int rs_flush(gd_ctx *c) {
  RecStream *r = c->rs;
  if (!r) return GD_OK;
  int rc = rs_enqueue(c, 0);
  if (rc) return rc;
  std::unique_lock<std::mutex> lk(r->mu);
  r->cv.wait(lk, [&] { return r->queue.empty(); });
  if (r->err != cudaSuccess)
    return fail(GD_ERR_CUDA, "record stream: %s", cudaGetErrorString(r->err));
  if (r->overflow) return fail(GD_ERR_STATE, "record stream: more rows than the writing calls queued");
  return GD_OK;
}

/* after a flush, before the counters of replicas [r0, r1] restart: their next copies start
 * from record 0 */
int rs_restart(gd_ctx *c, int r0, int r1) {
  if (!c->rs) return GD_OK;
  CK(cudaMemsetAsync(c->rs->d_prev + r0, 0, sizeof(int) * (size_t)(r1 - r0 + 1), c->stream));
  return GD_OK;
}

/* stops the worker after the queued copies and frees the stream's resources */
void rs_stop(gd_ctx *c) {
  RecStream *r = c->rs;
  if (!r) return;
  {
    std::lock_guard<std::mutex> lk(r->mu);
    r->stop = true;
  }
  r->cv.notify_all();
  if (r->th.joinable()) r->th.join();
  for (int i = 0; i < RecStream::NSNAP; ++i) {
    if (r->d_plan[i]) cudaFree(r->d_plan[i]);
    if (r->d_pack[i]) cudaFree(r->d_pack[i]);
    if (r->ev[i]) cudaEventDestroy(r->ev[i]);
  }
  if (r->d_prev) cudaFree(r->d_prev);
  if (r->h_plan) cudaFreeHost(r->h_plan);
  if (r->h_stage) cudaFreeHost(r->h_stage);
  if (r->cs) cudaStreamDestroy(r->cs);
  delete r;
  c->rs = nullptr;
}

template <class T>
int dalloc(gd_ctx *c, T **p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, n * sizeof(T));
  if (e != cudaSuccess)
    return fail(GD_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", n * sizeof(T), cudaGetErrorString(e));
  c->allocs.push_back(q);
  *p = (T *)q;
  return GD_OK;
}

template <class T>
int upload(gd_ctx *c, T **p, const std::vector<T> &v) {
  int rc = dalloc(c, p, v.size());
  if (rc) return rc;
  if (!v.empty()) CK(cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice,
                                     c->stream));
  return GD_OK;
}

int check_complex(const gd_complex_desc &d, int idx) {
  if (d.n_lig < 1 || d.n_prt < 1 || d.n_tmp < 1)
    return fail(GD_ERR_INVALID, "complex %d: n_lig/n_prt/n_tmp must be >= 1", idx);
  if (d.lna < 1 || d.lna > GD_MAXLIG)
    return fail(GD_ERR_CAPACITY, "complex %d: lna %d outside 1..%d", idx, d.lna, GD_MAXLIG);
  if (d.pnp < 1 || d.pnp > GD_MAXPRO)
    return fail(GD_ERR_CAPACITY, "complex %d: pnp %d outside 1..%d", idx, d.pnp, GD_MAXPRO);
  if (d.pnk < 0 || d.pnk > GD_MAXKDE)
    return fail(GD_ERR_CAPACITY, "complex %d: pnk %d outside 0..%d", idx, d.pnk, GD_MAXKDE);
  if (d.pos < 1 || d.pos > GD_MAXPOS)
    return fail(GD_ERR_CAPACITY, "complex %d: pos %d outside 1..%d (log(0/0) at pos = 0)", idx,
                d.pos, GD_MAXPOS);
  if (d.n_tmp > GD_MAXTMP)
    return fail(GD_ERR_CAPACITY, "complex %d: n_tmp %d > %d", idx, d.n_tmp, GD_MAXTMP);
  if (!d.lig_x || !d.lig_y || !d.lig_z || !d.lig_center || !d.lig_t || !d.lig_c || !d.lig_n ||
      !d.prt_x || !d.prt_y || !d.prt_z || !d.prt_t || !d.prt_c || !d.prt_ele || !d.prt_seq3r ||
      !d.prt_hflag || !d.prt_hpp || !d.pocket_center || !d.psp || !d.mcs_x || !d.mcs_y ||
      !d.mcs_z || !d.mcs_tcc || !d.temp || (d.pnk > 0 && (!d.kde_x || !d.kde_y || !d.kde_z ||
                                                         !d.kde_t)))
    return fail(GD_ERR_INVALID, "complex %d: null array", idx);
  if (d.psp_ld < 1 || d.mcs_ld < 1)
    return fail(GD_ERR_INVALID, "complex %d: psp_ld / mcs_ld must be >= 1", idx);
  for (int i = 0; i < d.n_lig * d.lna; ++i) {
    if (d.lig_t[i] < 0 || d.lig_t[i] >= GD_MAXTP2)
      return fail(GD_ERR_INVALID, "complex %d: ligand type %d out of range", idx, d.lig_t[i]);
    if (d.lig_n[i] + 1 < 0 || d.lig_n[i] + 1 >= d.mcs_ld)
      return fail(GD_ERR_INVALID, "complex %d: ligand atom number %d outside the MCS row", idx,
                  d.lig_n[i]);
  }
  for (int i = 0; i < d.n_prt * d.pnp; ++i) {
    if (d.prt_t[i] < 0 || d.prt_t[i] >= GD_MAXTP1)
      return fail(GD_ERR_INVALID, "complex %d: point type %d out of range", idx, d.prt_t[i]);
    if (d.prt_c[i] == 2 && (d.prt_seq3r[i] < 0 || d.prt_seq3r[i] >= d.psp_ld))
      return fail(GD_ERR_INVALID, "complex %d: PSP column %d outside 0..%d", idx, d.prt_seq3r[i],
                  d.psp_ld - 1);
  }
  for (int i = 0; i < d.pnk; ++i)
    if (d.kde_t[i] < 0 || d.kde_t[i] >= GD_MAXTP2)
      return fail(GD_ERR_INVALID, "complex %d: KDE type out of range", idx);
  return GD_OK;
}

int pick_threads(const std::vector<ComplexInfo> &info) {
  /* smallest lane waste over the batch, ties to the smaller block */
  int best = 256;
  double best_w = 1e30;
  for (int T = 128; T <= GD_MAX_TPB; T += 32) {
    double used = 0, cap = 0;
    bool ok = true;
    for (const auto &c : info) {
      const int k = std::min(T / c.lna, std::min(GD_MAX_SLOTS, c.n_tmp * c.n_lig));
      if (k < 1) { ok = false; break; }
      const double tiles = (double)c.n_prt * std::ceil((double)(c.n_tmp * c.n_lig) / k);
      used += (double)c.n_rep * c.lna;
      cap += tiles * T;
    }
    if (!ok) continue;
    const double w = 1.0 - used / cap + 1e-4 * T / 32.0;
    if (w < best_w - 1e-9) { best_w = w; best = T; }
  }
  return best;
}

void build_tiles(const gd_ctx *c, int r0, int r1, std::vector<GdTileDesc> &out) {
  out.clear();
  for (int ci = 0; ci < c->n_complex; ++ci) {
    const ComplexInfo &x = c->info[ci];
    const int block = x.n_tmp * x.n_lig;
    for (int p = 0; p < x.n_prt; ++p) {
      const int b0 = x.rep_offset + p * block, b1 = b0 + block; /* [b0, b1) */
      const int lo = std::max(b0, r0), hi = std::min(b1, r1 + 1);
      for (int r = lo; r < hi; r += x.k) {
        GdTileDesc t;
        t.complex_index = ci;
        t.prt_conf = p;
        t.rep_begin = r;
        t.count = std::min(x.k, hi - r);
        out.push_back(t);
      }
    }
  }
  /* longest first: the persistent queue then balances uneven complexes */
  std::stable_sort(out.begin(), out.end(), [&](const GdTileDesc &a, const GdTileDesc &b) {
    const ComplexInfo &x = c->info[a.complex_index], &y = c->info[b.complex_index];
    return (long long)a.count * x.lna * x.pnp > (long long)b.count * y.lna * y.pnp;
  });
}

size_t smem_bytes(const gd_ctx *c) {
  int kmax = 1;
  for (const auto &x : c->info) kmax = std::max(kmax, x.k);
  const size_t slot = GD_SLOT_BYTES;
  return 16 + (size_t)2 * c->chunk * 24 + (size_t)c->threads * 16 + (size_t)10 * c->threads * 8 +
         (size_t)kmax * slot;
}

int ensure_counters(gd_ctx *c, int n) {
  if (n <= c->counters_cap) return GD_OK;
  int *p = nullptr;
  CK(cudaMalloc(&p, sizeof(int) * n));
  if (c->d_counters) cudaFree(c->d_counters);
  c->d_counters = p;
  c->counters_cap = n;
  return GD_OK;
}

typedef void (*McKernel)(GdMcArgs, GdForceConst);

/* the kernel variant for an unroll depth, a protein split and the mode-3 epilogue */
template <bool S, bool D>
McKernel mc_variant(int unroll) {
  if (unroll >= 4) return gd::gd_mc_kernel<4, S, D, 1>;
  if (unroll >= 2) return gd::gd_mc_kernel<2, S, D, 1>;
  return gd::gd_mc_kernel<1, S, D, 1>;
}

McKernel mc_kernel(int unroll, int split, bool da = false, int pack = 1) {
  if (da) return split > 1 ? mc_variant<true, true>(unroll) : mc_variant<false, true>(unroll);
  if (pack == 2 && split <= 1)
    return unroll >= 2 ? gd::gd_mc_kernel<2, false, false, 2> : gd::gd_mc_kernel<1, false, false, 2>;
  return split > 1 ? mc_variant<true, false>(unroll) : mc_variant<false, false>(unroll);
}

/* replicas per thread of a launch: the context's packing for the plain modes without split */
int launch_pack(const gd_ctx *c, int split, bool da) {
  return (!da && (split ? split : c->split) <= 1) ? c->pack : 1;
}

/* threads per CTA of a launch: the tile's lanes over the replicas per thread */
int launch_threads(const gd_ctx *c, int split = 0, bool da = false) {
  return c->threads / launch_pack(c, split, da);
}

McKernel launch_kernel(const gd_ctx *c, int split = 0, bool da = false) {
  const int S = split ? split : c->split;
  return mc_kernel(c->unroll, S, da, launch_pack(c, split, da));
}

int grid_for(gd_ctx *c, int n_tiles, size_t smem, int split = 0, bool da = false) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, launch_kernel(c, split, da),
                                                    launch_threads(c, split, da),
                                                    smem) != cudaSuccess ||
      nb < 1)
    nb = 1;
  return std::max(1, std::min(n_tiles, nb * c->num_sms));
}

GdMcArgs base_args(gd_ctx *c) {
  GdMcArgs a;
  memset(&a, 0, sizeof(a));
  a.cx = c->d_cx;
  a.pp = c->d_pp;
  a.chunk = c->chunk;
  a.split = c->split;
  a.move_kind = c->mc.move_kind;
  a.seed = c->mc.seed;
  for (int i = 0; i < 6; ++i) a.move_scale[i] = c->mc.move_scale[i];
  a.replica = c->d_replica;
  a.mm_old = c->d_mm;
  a.e_old = c->d_eold;
  a.etotal = c->d_etotal;
  a.n_accept = c->d_nacc;
  a.rec = c->mc.record ? c->d_rec : nullptr;
  a.rec_next = c->d_rec_next;
  a.rec_cap = c->rec_cap;
  a.trace_e = c->d_trace_e;
  a.trace_acc = c->d_trace_acc;
  a.trace_cap = c->trace_cap;
  a.trace_step0 = c->trace_step0;
  a.err = c->d_err;
  a.timeout_ns = c->timeout_ns;
  return a;
}

int set_kernel_attrs(const gd_ctx *c, size_t smem, int split = 0, bool da = false) {
  const McKernel k = launch_kernel(c, split, da);
  CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CK(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                          cudaSharedmemCarveoutMaxShared));
  return GD_OK;
}

int launch_mc(gd_ctx *c, GdMcArgs a, const GdTileDesc *d_tiles, int n_tiles, int *counter) {
  if (n_tiles <= 0) return GD_OK;
  const size_t smem = smem_bytes(c);
  int rc = set_kernel_attrs(c, smem);
  if (rc) return rc;
  a.tiles = d_tiles;
  a.n_tiles = n_tiles;
  a.tile_counter = counter;
  CK(cudaMemsetAsync(counter, 0, sizeof(int), c->stream));
  const int grid = grid_for(c, n_tiles, smem);
  launch_kernel(c)<<<grid, launch_threads(c), smem, c->stream>>>(a, c->fc);
  CK(cudaGetLastError());
  return GD_OK;
}

int upload_tiles(gd_ctx *c, int r0, int r1, int *n_out) {
  /* the device list is reused while the range and the tile shape stay the same */
  if (c->tiles_r0 == r0 && c->tiles_r1 == r1 && c->tiles_gen == c->tile_gen) {
    *n_out = c->tiles_n;
    return GD_OK;
  }
  std::vector<GdTileDesc> t;
  const std::vector<GdTileDesc> *src = &c->full_tiles;
  if (!(r0 == 0 && r1 == c->n_rep - 1)) {
    build_tiles(c, r0, r1, t);
    src = &t;
  }
  if ((int)src->size() > c->tiles_cap) return fail(GD_ERR_INVALID, "tile list overflow");
  CK(cudaStreamSynchronize(c->stream));
  if (!src->empty())
    CK(cudaMemcpy(c->d_tiles, src->data(), src->size() * sizeof(GdTileDesc),
                  cudaMemcpyHostToDevice));
  c->tiles_r0 = r0;
  c->tiles_r1 = r1;
  c->tiles_gen = c->tile_gen;
  c->tiles_n = (int)src->size();
  *n_out = c->tiles_n;
  return GD_OK;
}

int check_range(const gd_ctx *c, int r0, int r1) {
  if (r0 < 0 || r1 >= c->n_rep || r0 > r1)
    return fail(GD_ERR_INVALID, "replica range [%d, %d] outside [0, %d]", r0, r1, c->n_rep - 1);
  return GD_OK;
}

/* Partition of the batch into `want` contiguous block ranges of about equal pair work; with
 * `tiles`, each chain's plain tile list (longest first within the chain) appended to it. */
void build_chains(gd_ctx *c, int want, std::vector<Chain> &ch, std::vector<GdTileDesc> *tiles) {
  int n_blocks = 0;
  for (const auto &x : c->info) n_blocks += x.n_prt;
  want = std::max(1, std::min(want, n_blocks));
  struct Blk { int r0, r1, xg0, xg1; double cost; };
  std::vector<Blk> blk;
  int xg = 0;
  double total = 0.0;
  for (int ci = 0; ci < c->n_complex; ++ci) {
    const ComplexInfo &x = c->info[ci];
    const int block = x.n_tmp * x.n_lig;
    for (int p = 0; p < x.n_prt; ++p) {
      Blk b;
      b.r0 = x.rep_offset + p * block;
      b.r1 = b.r0 + block;
      b.xg0 = xg + p * x.n_lig;
      b.xg1 = b.xg0 + x.n_lig;
      b.cost = (double)block * x.lna * x.pnp_pad;
      total += b.cost;
      blk.push_back(b);
    }
    xg += x.n_prt * x.n_lig;
  }
  ch.clear();
  int g = 0;
  double acc = 0.0;
  for (int k = 0; k < want; ++k) {
    Chain cc;
    cc.g0 = g;
    const double target = total * (k + 1) / want;
    /* at least one block, and one left for every later chain */
    do {
      acc += blk[g].cost;
      ++g;
    } while (g < n_blocks - (want - 1 - k) && acc + 0.5 * blk[g].cost <= target);
    if (k == want - 1) g = n_blocks;
    cc.g1 = g;
    cc.r0 = blk[cc.g0].r0;
    cc.r1 = blk[cc.g1 - 1].r1;
    cc.xg0 = blk[cc.g0].xg0;
    cc.xg1 = blk[cc.g1 - 1].xg1;
    cc.t_off = cc.t_cnt = 0;
    if (tiles) {
      std::vector<GdTileDesc> t;
      build_tiles(c, cc.r0, cc.r1 - 1, t);
      cc.t_off = (int)tiles->size();
      cc.t_cnt = (int)t.size();
      tiles->insert(tiles->end(), t.begin(), t.end());
    }
    ch.push_back(cc);
  }
}

/* streams and events for n chains (chain 0 runs on the context's stream) */
int ensure_chain_streams(gd_ctx *c, int n) {
  while ((int)c->aux.size() < n - 1) {
    cudaStream_t st;
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    c->aux.push_back(st);
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    c->ev_join.push_back(ev);
  }
  if (!c->ev_fork) CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  return GD_OK;
}

/* the plain fused loop's chains and their tile lists on the device */
int ensure_chains(gd_ctx *c) {
  if (c->chain_gen == c->tile_gen && !c->chain.empty()) return GD_OK;
  std::vector<Chain> ch;
  std::vector<GdTileDesc> tiles;
  build_chains(c, c->chains, ch, &tiles);
  CK(cudaStreamSynchronize(c->stream));
  if ((int)tiles.size() > c->chain_tiles_cap) {
    if (c->d_chain_tiles) cudaFree(c->d_chain_tiles);
    c->d_chain_tiles = nullptr;
    c->chain_tiles_cap = 0;
    CK(cudaMalloc(&c->d_chain_tiles, sizeof(GdTileDesc) * tiles.size()));
    c->chain_tiles_cap = (int)tiles.size();
  }
  CK(cudaMemcpy(c->d_chain_tiles, tiles.data(), sizeof(GdTileDesc) * tiles.size(),
                cudaMemcpyHostToDevice));
  int rc = ensure_chain_streams(c, (int)ch.size());
  if (rc) return rc;
  c->chain = ch;
  c->chain_gen = c->tile_gen;
  return GD_OK;
}

/* during capture on c->stream: the chains' streams join the capture / rejoin the main stream */
void chains_fork(gd_ctx *c, int n) {
  if (n <= 1) return;
  cudaEventRecord(c->ev_fork, c->stream);
  for (int k = 1; k < n; ++k) cudaStreamWaitEvent(c->aux[k - 1], c->ev_fork, 0);
}
void chains_join(gd_ctx *c, int n) {
  for (int k = 1; k < n; ++k) {
    cudaEventRecord(c->ev_join[k - 1], c->aux[k - 1]);
    cudaStreamWaitEvent(c->stream, c->ev_join[k - 1], 0);
  }
}
cudaStream_t chain_stream(gd_ctx *c, int k) { return k ? c->aux[k - 1] : c->stream; }

void da_free(gd_ctx *c);        /* delayed-acceptance state, defined with its entry points */
void da_drop_graphs(gd_ctx *c);

void drop_graphs(gd_ctx *c) {
  for (auto &g : c->graphs) cudaGraphExecDestroy(g.second);
  c->graphs.clear();
  da_drop_graphs(c);
}

}  // namespace

extern "C" {

const char *gd_last_error_string(void) { return g_err.c_str(); }
const char *gd_version(void) { return "geauxdock-b200 1.0 (sm_100a)"; }

int gd_fold_enepara(const gd_enepara_raw *raw, gd_enepara *o) {
  if (!raw || !o) return fail(GD_ERR_INVALID, "null argument");
  const float sqrt_2_pi = sqrtf(2.0f * kPi);
  memset(o, 0, sizeof(*o));
  for (int i = 0; i < GD_MAXTP2; ++i)
    for (int j = 0; j < GD_MAXTP1; ++j) {
      const float tmp = raw->vdw[j][i][0] * raw->lj[2];
      o->p1a[i][j] = 2.0f * raw->vdw[j][i][1] * powf(tmp, 9.0f);
      o->p2a[i][j] = 3.0f * raw->vdw[j][i][1] * powf(tmp, 6.0f);
    }
  o->lj0 = raw->lj[0];
  o->lj1 = raw->lj[1];
  o->el0 = raw->el[0];
  o->a1 = 4.0f - 3.0f * raw->el[0];
  o->b1 = 2.0f * raw->el[0] - 3.0f;
  o->el1 = raw->el[1];
  for (int i = 0; i < GD_MAXTP3; ++i) o->ele[i] = raw->ele[i];
  for (int i = 0; i < GD_MAXTP2; ++i)
    for (int j = 0; j < GD_MAXTP1; ++j) {
      o->pmf0[i][j] = raw->pmf[j][i][0];
      o->pmf1[i][j] = raw->pmf[j][i][1];
      o->hdb0[i][j] = raw->hdb[j][i][0];
      o->hdb1[i][j] = 1.0f / raw->hdb[j][i][1];
    }
  for (int i = 0; i < GD_MAXTP4; ++i) o->hpp[i] = raw->hpp[i];
  for (int i = 0; i < GD_MAXTP2; ++i) {
    o->hpl0[i] = raw->hpl[i][0];
    o->hpl1[i] = raw->hpl[i][1];
    o->hpl2[i] = logf(1.0f / (o->hpl1[i] * sqrt_2_pi));
  }
  o->kde2 = -0.5f / (raw->kde * raw->kde);
  o->kde3 = powf(raw->kde * sqrt_2_pi, 3.0f);
  for (int i = 0; i < GD_MAXWEI; ++i) {
    o->w[i] = raw->w[i];
    o->a_para[i] = raw->a_para[i];
    o->b_para[i] = raw->b_para[i];
  }
  return GD_OK;
}

int gd_set_temperature(int num_temp, float floor_temp, float ceiling_temp, gd_temp *out) {
  if (!out || num_temp < 1 || num_temp > GD_MAXTMP || !(floor_temp > 0.0f) ||
      !(ceiling_temp > 0.0f))
    return fail(GD_ERR_INVALID, "gd_set_temperature: bad arguments");
  if (num_temp == 1) {
    out[0].t = floor_temp;
    out[0].order = 0;
    out[0].minus_beta = 0.0f - 1.0f / (1.0f * floor_temp);
    return GD_OK;
  }
  const float ratio = (float)exp(log(ceiling_temp / floor_temp) / (float)(num_temp - 1));
  float a = floor_temp;
  for (int i = 0; i < num_temp; ++i) {
    out[i].t = a;
    out[i].order = i;
    out[i].minus_beta = 0.0f - 1.0f / (1.0f * a);
    a *= ratio;
  }
  return GD_OK;
}

int gd_set_replica(int n_prt, int n_tmp, int n_lig, gd_replica *out) {
  if (!out || n_prt < 1 || n_tmp < 1 || n_lig < 1) return fail(GD_ERR_INVALID, "bad arguments");
  for (int p = 0; p < n_prt; ++p)
    for (int t = 0; t < n_tmp; ++t)
      for (int l = 0; l < n_lig; ++l) {
        const int f = n_tmp * n_lig * p + n_lig * t + l;
        out[f].idx_rep = f;
        out[f].idx_prt = p;
        out[f].idx_tmp = t;
        out[f].idx_lig = l;
      }
  return GD_OK;
}

int gd_destroy(gd_ctx *c) {
  if (!c) return GD_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  rs_stop(c);
  drop_graphs(c);
  da_free(c);
  for (void *p : c->allocs) cudaFree(p);
  if (c->d_counters) cudaFree(c->d_counters);
  if (c->d_trace_e) cudaFree(c->d_trace_e);
  if (c->d_trace_acc) cudaFree(c->d_trace_acc);
  if (c->d_mm_in) cudaFree(c->d_mm_in);
  if (c->d_lc_in) cudaFree(c->d_lc_in);
  if (c->d_e_out) cudaFree(c->d_e_out);
  if (c->d_eval_tiles) cudaFree(c->d_eval_tiles);
  if (c->h_cursor) cudaFreeHost(c->h_cursor);
  if (c->d_chain_tiles) cudaFree(c->d_chain_tiles);
  for (cudaStream_t st : c->aux) cudaStreamDestroy(st);
  for (cudaEvent_t ev : c->ev_join) cudaEventDestroy(ev);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return GD_OK;
}

/* set-up of the allocation-free entry point on `device` (defined with it below) */
namespace {
int noalloc_prepare(int device);
}

int gd_create(const gd_enepara *ff, const gd_complex_desc *cxs, int n_complexes,
              const gd_mc_params *mc, int device, gd_ctx **out) {
  if (!out) return fail(GD_ERR_INVALID, "null out");
  *out = nullptr;
  if (!ff || !cxs || !mc || n_complexes < 1) return fail(GD_ERR_INVALID, "null argument");
  if (!(ff->el1 > 0.0f) || !std::isfinite(ff->el1))
    return fail(GD_ERR_INVALID, "electrostatic scale el1 must be finite and > 0");
  for (int i = 0; i < GD_MAXTP2; ++i)
    for (int j = 0; j < GD_MAXTP1; ++j)
      if (!(ff->pmf0[i][j] > -10.0f) || !(ff->pmf0[i][j] < 1e4f))
        return fail(GD_ERR_INVALID,
                    "pmf0[%d][%d] = %g outside (-10, 1e4): the contact-potential exponent "
                    "would leave FP32 range",
                    i, j, (double)ff->pmf0[i][j]);
  if (mc->steps_per_exchange < 1 || mc->steps_per_dump < 1)
    return fail(GD_ERR_INVALID, "steps_per_exchange and steps_per_dump must be >= 1");
  if (mc->move_kind != GD_MOVE_UNIFORM && mc->move_kind != GD_MOVE_GAUSSIAN)
    return fail(GD_ERR_INVALID, "unknown move_kind %d", mc->move_kind);
  for (int i = 0; i < n_complexes; ++i) {
    int rc = check_complex(cxs[i], i);
    if (rc) return rc;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
    return fail(GD_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(GD_ERR_NODEVICE, "device %d absent", device);
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(GD_ERR_NODEVICE, "device %d is sm_%d%d; this library is built for sm_100a",
                device, prop.major, prop.minor);
  CK(cudaSetDevice(device));

  {
    const int rc0 = noalloc_prepare(device);
    if (rc0) return rc0;
  }

  gd_ctx *c = new gd_ctx();
  c->device = device;
  c->mc = *mc;
  c->num_sms = prop.multiProcessorCount;
  c->n_complex = n_complexes;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail(GD_ERR_CUDA, "cudaStreamCreate failed");
  }
  auto bail = [&](int rc) {
    gd_destroy(c);
    return rc;
  };

  /* ---- force-field folds for the kernel ---- */
  GdForceConst &f = c->fc;
  f.lj1 = ff->lj1;
  f.el0 = ff->el0;
  f.el1 = ff->el1;
  f.a1 = ff->a1;
  f.b1 = ff->b1;
  f.inv_el1 = 1.0f / ff->el1;
  f.near2 = f.inv_el1 * f.inv_el1;
  f.kde2 = ff->kde2;
  f.kde3 = ff->kde3;
  for (int i = 0; i < GD_MAXWEI; ++i) {
    f.a_para[i] = ff->a_para[i];
    f.b_para[i] = ff->b_para[i];
    f.w[i] = ff->w[i];
  }
  for (int i = 0; i < GD_MAXTP2; ++i) {
    f.hpl0[i] = ff->hpl0[i];
    f.hpl1[i] = ff->hpl1[i];
    f.hpl2[i] = ff->hpl2[i];
  }
  float thr[GD_MAXTP2][GD_MAXTP1];
  std::vector<GdPairParam> pp(GD_MAXTP2 * GD_MAXTP1);
  {
    const double hsc = std::sqrt(0.5 * 1.4426950408889634);
    const float sqrt_2_pi_m1 = -1.0f / sqrtf(2.0f * kPi);
    for (int i = 0; i < GD_MAXTP2; ++i)
      for (int j = 0; j < GD_MAXTP1; ++j) {
        GdPairParam &q = pp[i * GD_MAXTP1 + j];
        memset(&q, 0, sizeof(q));
        q.p1a = ff->p1a[i][j];
        q.p2a = ff->p2a[i][j];
        q.p1l = ff->p1a[i][j] * ff->lj0;
        thr[i][j] = contact_threshold(ff->pmf0[i][j]);
        q.thr = thr[i][j];
        q.pmf0 = ff->pmf0[i][j];
        q.pmf1 = ff->pmf1[i][j];
        const bool live = ff->hdb0[i][j] > 0.1f;
        /* pairs without an H-bond entry have hdb1 = 1/0: keep their folded argument finite,
         * since they run inside warps where another lane's pair is live (hs = 0 kills them) */
        q.hc1 = live ? (float)((double)ff->hdb1[i][j] * hsc) : 0.0f;
        q.hc0 = live ? (float)(-(double)ff->hdb0[i][j] * (double)ff->hdb1[i][j] * hsc) : 0.0f;
        q.hs = live ? sqrt_2_pi_m1 * ff->hdb1[i][j] : 0.0f;
        q.hneed = live ? 1.0f : 0.0f;
        /* pmf exponent (6 - r/2)(r - pmf0) log2(e) = cA d2 + b2 r + c2 */
        q.b2 = (float)(1.4426950408889634 * (6.0 + 0.5 * (double)ff->pmf0[i][j]));
        q.c2 = (float)(-6.0 * 1.4426950408889634 * (double)ff->pmf0[i][j]);
      }
  }
  int rc = upload(c, &c->d_pp, pp);
  if (rc) return bail(rc);

  /* ---- per complex layout ---- */
  std::vector<GdDevComplex> dcx(n_complexes);
  std::vector<int> group_base(n_complexes);
  int off = 0, goff = 0;
  for (int ci = 0; ci < n_complexes; ++ci) {
    const gd_complex_desc &d = cxs[ci];
    ComplexInfo x;
    x.n_lig = d.n_lig;
    x.n_prt = d.n_prt;
    x.n_tmp = d.n_tmp;
    x.lna = d.lna;
    x.pnp = d.pnp;
    x.pnp_pad = (d.pnp + 3) & ~3;
    x.pnk = d.pnk;
    x.pos = d.pos;
    x.rep_offset = off;
    x.n_rep = d.n_prt * d.n_tmp * d.n_lig;
    x.stream = ci;
    x.k = 1;
    x.types_uniform = 1;
    for (int lc = 1; lc < d.n_lig && x.types_uniform; ++lc)
      for (int i = 0; i < d.lna; ++i)
        if (d.lig_t[lc * d.lna + i] != d.lig_t[i]) {
          x.types_uniform = 0;
          break;
        }
    c->info.push_back(x);
    group_base[ci] = goff;
    goff += d.n_prt * d.n_lig;
    off += x.n_rep;

    GdDevComplex &g = dcx[ci];
    memset(&g, 0, sizeof(g));
    g.n_lig = d.n_lig; g.n_prt = d.n_prt; g.n_tmp = d.n_tmp; g.lna = d.lna;
    g.pnp = d.pnp; g.pnp_pad = x.pnp_pad; g.pnk = d.pnk; g.pos = d.pos;
    g.rep_offset = x.rep_offset; g.n_rep = x.n_rep; g.psp_ld = d.psp_ld; g.mcs_ld = d.mcs_ld;
    g.stream = ci;
    g.pocket[0] = d.pocket_center[0];
    g.pocket[1] = d.pocket_center[1];
    g.pocket[2] = d.pocket_center[2];
    const int L = d.lna, P = d.pnp;

    std::vector<float4> lig_pos((size_t)d.n_lig * L);
    std::vector<int2> lig_meta((size_t)d.n_lig * L);
    for (int i = 0; i < d.n_lig * L; ++i) {
      lig_pos[i] = make_float4(d.lig_x[i], d.lig_y[i], d.lig_z[i], d.lig_c[i]);
      lig_meta[i] = make_int2(d.lig_t[i], d.lig_n[i] + 1);
    }
    std::vector<float> lig_center(d.lig_center, d.lig_center + 3 * d.n_lig);

    /* protein: sort by (type, kind) into segments that start on even slots (one padding
     * slot after an odd-length segment), then write slot pairs */
    std::vector<int4> seg((size_t)d.n_prt * GD_MAX_SEG, make_int4(0, 0, 0, 0));
    std::vector<int> seg_count(d.n_prt, 0);
    std::vector<std::vector<int>> slot_point(d.n_prt); /* point index per slot, -1: padding */
    int max_slots = 4;
    /* the hydrogen-bond term runs for a point type when any atom type of this ligand has a
     * live pair with it: one decision per segment for the whole CTA */
    bool hdb_live[GD_MAXTP1] = {false};
    {
      bool lt_used[GD_MAXTP2] = {false};
      for (int i = 0; i < d.n_lig * L; ++i) lt_used[d.lig_t[i]] = true;
      for (int tp = 0; tp < GD_MAXTP1; ++tp)
        for (int tl = 0; tl < GD_MAXTP2; ++tl)
          if (lt_used[tl] && ff->hdb0[tl][tp] > 0.1f) hdb_live[tp] = true;
    }
    for (int pc = 0; pc < d.n_prt; ++pc) {
      const int o = pc * P;
      std::vector<int> order(P), key(P);
      for (int p = 0; p < P; ++p) {
        const int kind = (d.prt_hflag[o + p] == 1 ? 1 : 0) | (d.prt_c[o + p] == 2 ? 2 : 0);
        key[p] = d.prt_t[o + p] * 4 + kind;
        order[p] = p;
      }
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
      std::vector<int> &sp = slot_point[pc];
      int ns = 0;
      for (int i = 0; i < P; ++i) {
        const int p = order[i];
        if (i == 0 || key[p] != key[order[i - 1]]) {
          if (sp.size() & 1) sp.push_back(-1);
          if (ns == GD_MAX_SEG) return bail(fail(GD_ERR_CAPACITY, "too many point segments"));
          const int s0 = (int)sp.size();
          seg[(size_t)pc * GD_MAX_SEG + ns] = make_int4(
              s0, s0 + 1, d.prt_t[o + p], (key[p] & 3) | (hdb_live[d.prt_t[o + p]] ? 4 : 0));
          ++ns;
        } else {
          seg[(size_t)pc * GD_MAX_SEG + ns - 1].y = (int)sp.size() + 1;
        }
        sp.push_back(p);
      }
      seg_count[pc] = ns;
      max_slots = std::max(max_slots, (int)sp.size());
    }
    const int PP = (max_slots + 3) & ~3;
    c->info[ci].pnp_pad = PP;
    g.pnp_pad = PP;
    const size_t npair = (size_t)PP / 2;
    std::vector<float4> pt_a((size_t)d.n_prt * npair, make_float4(-1e6f, -1e6f, -1e6f, -1e6f));
    std::vector<float4> pt_b((size_t)d.n_prt * npair, make_float4(-1e6f, -1e6f, 0.0f, 0.0f));
    std::vector<float4> pt_x((size_t)d.n_prt * npair,
                             make_float4(0.0f, 0.0f, bits_as_float(-1), bits_as_float(-1)));
    for (int pc = 0; pc < d.n_prt; ++pc) {
      const int o = pc * P;
      const std::vector<int> &sp = slot_point[pc];
      for (size_t sidx = 0; sidx < sp.size(); ++sidx) {
        const int p = sp[sidx];
        if (p < 0) continue;
        const int kind = (d.prt_hflag[o + p] == 1 ? 1 : 0) | (d.prt_c[o + p] == 2 ? 2 : 0);
        float *A = &pt_a[pc * npair + sidx / 2].x;
        float *B = &pt_b[pc * npair + sidx / 2].x;
        float *X = &pt_x[pc * npair + sidx / 2].x;
        const int h = (int)(sidx & 1);
        A[0 + h] = -d.prt_x[o + p];
        A[2 + h] = -d.prt_y[o + p];
        B[0 + h] = -d.prt_z[o + p];
        B[2 + h] = d.prt_ele[o + p] * (1.0f / ff->el1); /* ele_p / el1 */
        X[0 + h] = (kind & 1) ? d.prt_hpp[o + p] : 0.0f;
        X[2 + h] = bits_as_float((kind & 2) ? d.prt_seq3r[o + p] : -1);
      }
    }
    /* contact reference from (protein 0, ligand 0) at movematrix 0 (InitRefMatrix_d) */
    std::vector<int> ref_start((size_t)d.n_prt * (L + 1));
    std::vector<float4> ref_pts;
    {
      float rot[9];
      const float mm0[6] = {0, 0, 0, 0, 0, 0};
      gd_rotation(mm0, rot);
      std::vector<float> ax(L), ay(L), az(L);
      for (int l = 0; l < L; ++l)
        gd_place_atom(rot, 0.0f + d.lig_center[0], 0.0f + d.lig_center[1],
                      0.0f + d.lig_center[2], d.lig_x[l], d.lig_y[l], d.lig_z[l], &ax[l], &ay[l],
                      &az[l]);
      std::vector<std::vector<int>> refp(L);
      int nref = 0;
      for (int l = 0; l < L; ++l) {
        const int tl = d.lig_t[l];
        for (int p = 0; p < P; ++p)
          if (host_dist2(ax[l], ay[l], az[l], d.prt_x[p], d.prt_y[p], d.prt_z[p]) <=
              thr[tl][d.prt_t[p]]) {
            refp[l].push_back(p);
            ++nref;
          }
      }
      g.nref_total = nref;
      for (int pc = 0; pc < d.n_prt; ++pc) {
        const int o = pc * P;
        for (int l = 0; l < L; ++l) {
          ref_start[(size_t)pc * (L + 1) + l] = (int)ref_pts.size();
          for (int p : refp[l])
            ref_pts.push_back(make_float4(d.prt_x[o + p], d.prt_y[o + p], d.prt_z[o + p],
                                          thr[d.lig_t[l]][d.prt_t[o + p]]));
        }
        ref_start[(size_t)pc * (L + 1) + L] = (int)ref_pts.size();
      }
    }
    std::vector<float4> kde(std::max(1, d.pnk));
    for (int i = 0; i < d.pnk; ++i)
      kde[i] = make_float4(d.kde_x[i], d.kde_y[i], d.kde_z[i], (float)d.kde_t[i]);
    const size_t nm = (size_t)d.pos * d.mcs_ld;
    std::vector<float> mx(d.mcs_x, d.mcs_x + nm), my(d.mcs_y, d.mcs_y + nm),
        mz(d.mcs_z, d.mcs_z + nm), mt(d.mcs_tcc, d.mcs_tcc + d.pos);
    std::vector<float> psp(d.psp, d.psp + (size_t)GD_MAXTP2 * d.psp_ld);
    std::vector<float> mb(d.n_tmp);
    for (int t = 0; t < d.n_tmp; ++t) mb[t] = d.temp[t].minus_beta;

    float4 *p_lig_pos; int2 *p_lig_meta; float *p_lig_center; float4 *p_pt_a, *p_pt_b, *p_pt_x;
    int4 *p_seg; int *p_seg_count; float4 *p_kde; float *p_mx, *p_my, *p_mz, *p_mt, *p_psp, *p_mb;
    int *p_ref_start; float4 *p_ref_pts;
    if ((rc = upload(c, &p_lig_pos, lig_pos)) || (rc = upload(c, &p_lig_meta, lig_meta)) ||
        (rc = upload(c, &p_lig_center, lig_center)) || (rc = upload(c, &p_pt_a, pt_a)) ||
        (rc = upload(c, &p_pt_b, pt_b)) || (rc = upload(c, &p_pt_x, pt_x)) ||
        (rc = upload(c, &p_seg, seg)) ||
        (rc = upload(c, &p_seg_count, seg_count)) || (rc = upload(c, &p_kde, kde)) ||
        (rc = upload(c, &p_mx, mx)) || (rc = upload(c, &p_my, my)) ||
        (rc = upload(c, &p_mz, mz)) || (rc = upload(c, &p_mt, mt)) ||
        (rc = upload(c, &p_psp, psp)) || (rc = upload(c, &p_mb, mb)) ||
        (rc = upload(c, &p_ref_start, ref_start)) || (rc = upload(c, &p_ref_pts, ref_pts)))
      return bail(rc);
    /* the host vectors die at the end of this iteration: finish the copies first */
    if (cudaStreamSynchronize(c->stream) != cudaSuccess)
      return bail(fail(GD_ERR_CUDA, "upload failed: %s", cudaGetErrorString(cudaGetLastError())));
    g.lig_pos = p_lig_pos; g.lig_meta = p_lig_meta; g.lig_center = p_lig_center;
    g.pt_a = p_pt_a; g.pt_b = p_pt_b; g.pt_x = p_pt_x; g.seg = p_seg; g.seg_count = p_seg_count;
    g.kde = p_kde; g.mcs_x = p_mx; g.mcs_y = p_my; g.mcs_z = p_mz; g.mcs_tcc = p_mt;
    g.psp = p_psp; g.minus_beta = p_mb; g.ref_start = p_ref_start; g.ref_pts = p_ref_pts;
  }
  c->n_rep = off;
  c->n_groups = goff;
  if ((rc = upload(c, &c->d_cx, dcx)) || (rc = upload(c, &c->d_group_base, group_base)))
    return bail(rc);

  /* ---- replica state ---- */
  const int R = c->n_rep;
  std::vector<gd_replica> rep(R);
  for (int ci = 0; ci < n_complexes; ++ci) {
    const ComplexInfo &x = c->info[ci];
    gd_set_replica(x.n_prt, x.n_tmp, x.n_lig, rep.data() + x.rep_offset);
  }
  if ((rc = upload(c, &c->d_replica, rep)) || (rc = dalloc(c, &c->d_mm, (size_t)R * 6)) ||
      (rc = dalloc(c, &c->d_eold, R)) || (rc = dalloc(c, &c->d_etotal, R)) ||
      (rc = dalloc(c, &c->d_nacc, R)) || (rc = dalloc(c, &c->d_acs, R)) ||
      (rc = dalloc(c, &c->d_rec_next, R)) || (rc = dalloc(c, &c->d_err, 1)))
    return bail(rc);
  CK(cudaMemsetAsync(c->d_mm, 0, sizeof(float) * 6 * R, c->stream));
  CK(cudaMemsetAsync(c->d_nacc, 0, sizeof(int) * R, c->stream));
  CK(cudaMemsetAsync(c->d_acs, 0, sizeof(int) * R, c->stream));
  CK(cudaMemsetAsync(c->d_rec_next, 0, sizeof(int) * R, c->stream));
  CK(cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), c->stream));
  c->rec_cap = mc->steps_per_dump + 1;
  if (mc->record) {
    if ((rc = dalloc(c, &c->d_rec, (size_t)R * c->rec_cap))) return bail(rc);
  }

  /* ---- tiles ---- */
  c->threads = pick_threads(c->info);
  for (auto &x : c->info)
    x.k = std::max(1, std::min(c->threads / x.lna, std::min(GD_MAX_SLOTS, x.n_tmp * x.n_lig)));
  build_tiles(c, 0, R - 1, c->full_tiles);
  c->tiles_cap = (int)c->full_tiles.size() + 16 * n_complexes;
  {
    /* any sub-range adds at most two partial tiles per protein-conformer block */
    int blocks = 0;
    for (auto &x : c->info) blocks += x.n_prt;
    c->tiles_cap = (int)c->full_tiles.size() + 2 * blocks + 16;
  }
  if ((rc = dalloc(c, &c->d_tiles, c->tiles_cap))) return bail(rc);
  if ((rc = ensure_counters(c, 64))) return bail(rc);
  if ((rc = dalloc(c, &c->d_cursor, 2))) return bail(rc);
  CK(cudaMallocHost(&c->h_cursor, 2 * sizeof(int)));
  CK(cudaStreamSynchronize(c->stream));
  *out = c;
  return GD_OK;
}

int gd_num_replicas(const gd_ctx *c, int *n) {
  if (!c || !n) return fail(GD_ERR_INVALID, "null argument");
  *n = c->n_rep;
  return GD_OK;
}

int gd_replica_offset(const gd_ctx *c, int k, int *offset) {
  if (!c || !offset || k < 0 || k >= c->n_complex) return fail(GD_ERR_INVALID, "bad complex");
  *offset = c->info[k].rep_offset;
  return GD_OK;
}

int gd_set_tile(gd_ctx *c, int k, const gd_tile *t) {
  if (!c || !t) return fail(GD_ERR_INVALID, "null argument");
  if (t->unroll != 0 && t->unroll != 1 && t->unroll != 2 && t->unroll != 4)
    return fail(GD_ERR_INVALID, "unroll must be 1, 2 or 4 (0 keeps the current value)");
  if (t->chunk_points < 4 || (t->chunk_points & 3) || t->chunk_points > 4096)
    return fail(GD_ERR_INVALID, "chunk_points must be a multiple of 4 in 4..4096");
  if (t->replicas_per_cta < 0 || t->replicas_per_cta > GD_MAX_SLOTS ||
      (t->replicas_per_cta == 0 && t->threads == 0))
    return fail(GD_ERR_INVALID, "replicas_per_cta outside 1..%d (0 only with threads)",
                GD_MAX_SLOTS);
  if (t->split < 0 || t->split > 16) return fail(GD_ERR_INVALID, "split outside 0..16");
  if (t->threads < 0 || t->threads > GD_MAX_TPB || (t->threads & 31))
    return fail(GD_ERR_INVALID, "threads must be a multiple of 32 in 0..%d", GD_MAX_TPB);
  if (k < -1 || k >= c->n_complex) return fail(GD_ERR_INVALID, "bad complex index");
  if (t->replicas_per_lane < 0 || t->replicas_per_lane > 2)
    return fail(GD_ERR_INVALID, "replicas_per_lane must be 0, 1 or 2");
  const int S = t->split ? t->split : 1;
  const int P = t->replicas_per_lane == 2 ? 2 : 1;
  if ((t->chunk_points / 2) < S)
    return fail(GD_ERR_INVALID, "chunk_points must hold at least two points per split");
  if (P == 2) {
    if (S != 1) return fail(GD_ERR_INVALID, "two replicas per lane need split 1");
    for (int i = 0; i < c->n_complex; ++i)
      if (!c->info[i].types_uniform || c->info[i].lna < 2)
        return fail(GD_ERR_INVALID,
                    "complex %d: two replicas per lane need at least two ligand atoms and the "
                    "same atom types in every ligand conformer",
                    i);
  }
  /* one block size per context: every complex's k must fit the block */
  std::vector<ComplexInfo> info = c->info;
  for (int i = 0; i < c->n_complex; ++i) {
    if (!(k == -1 || k == i)) continue;
    int kk = info[i].n_tmp * info[i].n_lig;
    if (t->replicas_per_cta > 0) kk = std::min(kk, t->replicas_per_cta);
    if (t->threads > 0) {
      if (S * info[i].lna > t->threads)
        return fail(GD_ERR_INVALID, "complex %d: split * lna exceeds threads", i);
      /* two per lane: an even count whose lane pairs fill half the CTA's lanes */
      kk = std::min(kk, P == 2 ? 2 * ((t->threads / 2) / info[i].lna)
                               : t->threads / (S * info[i].lna));
      if (kk < 1)
        return fail(GD_ERR_INVALID, "complex %d: no replica pair fits %d lanes", i, t->threads);
    }
    info[i].k = std::min(kk, GD_MAX_SLOTS);
  }
  /* T: the tile's lanes (a multiple of 32 per pack, so that T / pack threads are whole warps) */
  int T = 32;
  if (P == 2) {
    int Tp = 32;
    for (auto &x : info) Tp = std::max(Tp, (((x.k + 1) / 2 * x.lna + 31) / 32) * 32);
    if (t->threads > 0) Tp = std::max(Tp, ((t->threads / 2 + 31) / 32) * 32);
    T = 2 * Tp; /* Tp, the threads of a launch, is whole warps */
  } else {
    for (auto &x : info) T = std::max(T, ((x.k * S * x.lna + 31) / 32) * 32);
    if (t->threads > 0) T = std::max(T, t->threads);
  }
  if (T > GD_MAX_TPB)
    return fail(GD_ERR_INVALID, "replicas_per_cta * split * lna exceeds %d lanes", GD_MAX_TPB);
  c->info = info;
  c->threads = T;
  c->chunk = t->chunk_points;
  c->split = S;
  c->fill_threads = t->threads;
  c->fill_cap = t->threads > 0 ? t->replicas_per_cta : 0;
  c->pack = P;
  if (t->unroll) c->unroll = t->unroll;
  c->tile_gen += 1;
  build_tiles(c, 0, c->n_rep - 1, c->full_tiles);
  int blocks = 0;
  for (auto &x : c->info) blocks += x.n_prt;
  const int need = (int)c->full_tiles.size() + 2 * blocks + 16;
  if (need > c->tiles_cap) {
    GdTileDesc *p = nullptr;
    CK(cudaMalloc(&p, need * sizeof(GdTileDesc)));
    c->allocs.push_back(p);
    c->d_tiles = p;
    c->tiles_cap = need;
  }
  drop_graphs(c);
  return GD_OK;
}

int gd_autotune(gd_ctx *c, const gd_tile *cand, int n_cand, int repeats, gd_tile *best,
                float *ms_out) {
  if (!c || !cand || n_cand < 1 || repeats < 1 || !best)
    return fail(GD_ERR_INVALID, "gd_autotune: bad arguments");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  /* the probe evaluates pose id == replica id: poses are the chains' mm_old, ligand
   * conformer per pose from the replica table */
  std::vector<gd_replica> rep(c->n_rep);
  CK(cudaMemcpy(rep.data(), c->d_replica, sizeof(gd_replica) * c->n_rep, cudaMemcpyDeviceToHost));
  std::vector<int> lc(c->n_rep);
  for (int r = 0; r < c->n_rep; ++r) lc[r] = rep[r].idx_lig;
  int *d_lc = nullptr;
  gd_energy *d_e = nullptr;
  CK(cudaMalloc(&d_lc, sizeof(int) * c->n_rep));
  if (cudaMalloc(&d_e, sizeof(gd_energy) * c->n_rep) != cudaSuccess) {
    cudaFree(d_lc);
    return fail(GD_ERR_NOMEM, "gd_autotune: no memory for the probe");
  }
  cudaMemcpy(d_lc, lc.data(), sizeof(int) * c->n_rep, cudaMemcpyHostToDevice);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const gd_tile keep_tile = {c->info[0].k, c->chunk, c->unroll, c->split, c->threads, c->pack};
  const int keep_fill_threads = c->fill_threads, keep_fill_cap = c->fill_cap;
  std::vector<int> keep_k;
  for (auto &x : c->info) keep_k.push_back(x.k);
  const int keep_threads = c->threads;
  int best_i = -1, rc = GD_OK;
  float best_ms = 1e30f;
  for (int i = 0; i < n_cand && rc == GD_OK; ++i) {
    if ((rc = gd_set_tile(c, -1, &cand[i])) != GD_OK) {
      /* a candidate that does not fit this batch is skipped */
      if (ms_out) ms_out[i] = -1.0f;
      rc = GD_OK;
      continue;
    }
    int n = 0;
    if ((rc = upload_tiles(c, 0, c->n_rep - 1, &n))) break;
    GdMcArgs a = base_args(c);
    a.mode = 2;
    a.n_steps = 1;
    a.mm_in = c->d_mm;
    a.lig_conf_in = d_lc;
    a.e_out = d_e;
    a.rec = nullptr;
    a.trace_e = nullptr;
    if ((rc = launch_mc(c, a, c->d_tiles, n, c->d_counters))) break; /* warm-up */
    cudaEventRecord(e0, c->stream);
    for (int r = 0; r < repeats && rc == GD_OK; ++r)
      rc = launch_mc(c, a, c->d_tiles, n, c->d_counters);
    cudaEventRecord(e1, c->stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = fail(GD_ERR_CUDA, "gd_autotune: probe failed");
      break;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    ms /= (float)repeats;
    if (ms_out) ms_out[i] = ms;
    if (ms < best_ms) {
      best_ms = ms;
      best_i = i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_lc);
  cudaFree(d_e);
  if (rc == GD_OK && best_i >= 0) {
    rc = gd_set_tile(c, -1, &cand[best_i]);
    *best = cand[best_i];
    best->unroll = c->unroll;
    best->split = c->split;
    best->threads = cand[best_i].threads;
    best->replicas_per_lane = c->pack;
  } else {
    /* restore the tile in use before the probe */
    for (int i = 0; i < c->n_complex; ++i) c->info[i].k = keep_k[i];
    c->threads = keep_threads;
    c->chunk = keep_tile.chunk_points;
    c->unroll = keep_tile.unroll;
    c->split = keep_tile.split;
    c->pack = keep_tile.replicas_per_lane;
    c->fill_threads = keep_fill_threads;
    c->fill_cap = keep_fill_cap;
    c->tile_gen += 1;
    build_tiles(c, 0, c->n_rep - 1, c->full_tiles);
    if (rc == GD_OK) rc = fail(GD_ERR_INVALID, "gd_autotune: no candidate fits this batch");
  }
  return rc;
}

int gd_get_replicas_per_cta(const gd_ctx *c, int k, int *n) {
  if (!c || !n || k < 0 || k >= c->n_complex) return fail(GD_ERR_INVALID, "bad argument");
  *n = c->info[k].k;
  return GD_OK;
}

int gd_set_concurrency(gd_ctx *c, int plain_chains, int da_chains) {
  if (!c || plain_chains < 1 || plain_chains > 16 || da_chains < 1 || da_chains > 16)
    return fail(GD_ERR_INVALID, "chains must be in 1..16");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  c->chains = plain_chains;
  c->chains_da = da_chains;
  c->chain_gen = -1;
  c->chain.clear();
  drop_graphs(c);
  return GD_OK;
}

int gd_set_rng_stream(gd_ctx *c, int k, int stream) {
  if (!c || k < 0 || k >= c->n_complex || stream < 0)
    return fail(GD_ERR_INVALID, "bad complex index or stream");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(reinterpret_cast<char *>(c->d_cx + k) + offsetof(GdDevComplex, stream), &stream,
                sizeof(int), cudaMemcpyHostToDevice));
  c->info[k].stream = stream;
  return GD_OK;
}

int gd_set_wait_timeout(gd_ctx *c, long long ns) {
  if (!c || ns < 0) return fail(GD_ERR_INVALID, "bad timeout");
  c->timeout_ns = ns;
  drop_graphs(c);
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemset(c->d_err, 0, sizeof(unsigned)));
  return GD_OK;
}

int gd_get_tile(const gd_ctx *c, int k, gd_tile *t) {
  if (!c || !t || k < 0 || k >= c->n_complex) return fail(GD_ERR_INVALID, "bad argument");
  /* the tile as set: in fill mode the cap (0: none) and the CTA size, so that gd_set_tile of
   * the result restores it; gd_get_replicas_per_cta gives each complex's count */
  t->replicas_per_cta = c->fill_threads > 0 ? c->fill_cap : c->info[k].k;
  t->chunk_points = c->chunk;
  t->unroll = c->unroll;
  t->split = c->split;
  t->threads = c->fill_threads;
  t->replicas_per_lane = c->pack;
  return GD_OK;
}

int gd_mc_init(gd_ctx *c) {
  if (!c) return fail(GD_ERR_INVALID, "null context");
  CK(cudaSetDevice(c->device));
  int n = 0, rc = upload_tiles(c, 0, c->n_rep - 1, &n);
  if (rc) return rc;
  GdMcArgs a = base_args(c);
  a.mode = 1;
  a.n_steps = 1;
  CK(cudaMemsetAsync(c->d_acs, 0, sizeof(int) * c->n_rep, c->stream));
  CK(cudaMemsetAsync(c->d_err, 0, sizeof(unsigned), c->stream));
  if ((rc = rs_flush(c))) return rc;
  if ((rc = rs_restart(c, 0, c->n_rep - 1))) return rc;
  rc = launch_mc(c, a, c->d_tiles, n, c->d_counters);
  if (rc) return rc;
  c->initialized = true;
  c->exchange_calls = 0;
  return rs_enqueue(c, 1);
}

int gd_reset_records(gd_ctx *c, int r0, int r1) {
  if (!c) return fail(GD_ERR_INVALID, "null context");
  int rc = check_range(c, r0, r1);
  if (rc) return rc;
  const int n = r1 - r0 + 1;
  if ((rc = rs_flush(c))) return rc;
  if ((rc = rs_restart(c, r0, r1))) return rc;
  gd::gd_reset_records_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(c->d_rec_next, r0, r1);
  CK(cudaGetLastError());
  return GD_OK;
}

int gd_mc_run(gd_ctx *c, int r0, int r1, int s1, int s2) {
  if (!c) return fail(GD_ERR_INVALID, "null context");
  if (!c->initialized) return fail(GD_ERR_STATE, "gd_mc_init has not run");
  int rc = check_range(c, r0, r1);
  if (rc) return rc;
  CK(cudaSetDevice(c->device));
  int n = 0;
  if ((rc = upload_tiles(c, r0, r1, &n))) return rc;
  GdMcArgs a = base_args(c);
  a.mode = 0;
  a.n_steps = c->mc.steps_per_exchange;
  a.step0 = s1 + s2;
  if ((rc = launch_mc(c, a, c->d_tiles, n, c->d_counters))) return rc;
  return rs_enqueue(c, c->mc.steps_per_exchange);
}

int gd_exchange(gd_ctx *c, int mode_l, int mode_t) {
  (void)mode_l;
  if (!c) return fail(GD_ERR_INVALID, "null context");
  if (!c->initialized) return fail(GD_ERR_STATE, "gd_mc_init has not run");
  if (mode_t < 0) return fail(GD_ERR_INVALID, "mode_t must be >= 0");
  CK(cudaSetDevice(c->device));
  gd::gd_exchange_kernel<<<(c->n_groups + 127) / 128, 128, 0, c->stream>>>(
      c->d_cx, c->d_group_base, c->n_complex, 0, c->n_groups, c->d_replica, c->d_etotal,
      c->d_acs, c->mc.seed, nullptr, c->exchange_calls, mode_t);
  CK(cudaGetLastError());
  c->exchange_calls += 1;
  return GD_OK;
}

int gd_mc_run_fused(gd_ctx *c, int s1, int n_steps, int exchange) {
  if (!c) return fail(GD_ERR_INVALID, "null context");
  if (!c->initialized) return fail(GD_ERR_STATE, "gd_mc_init has not run");
  const int spe = c->mc.steps_per_exchange;
  if (n_steps < 1 || n_steps % spe)
    return fail(GD_ERR_INVALID, "n_steps must be a positive multiple of steps_per_exchange");
  CK(cudaSetDevice(c->device));
  int rc = ensure_chains(c);
  if (rc) return rc;
  const int nch = (int)c->chain.size();
  const int chunks = n_steps / spe;
  if ((rc = ensure_counters(c, chunks * nch))) return rc;
  const long long key = ((long long)n_steps << 1) | (exchange ? 1 : 0);
  auto it = c->graphs.find(key);
  if (it == c->graphs.end()) {
    CK(cudaStreamSynchronize(c->stream));
    const size_t smem = smem_bytes(c);
    if ((rc = set_kernel_attrs(c, smem))) return rc;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(c->d_counters, 0, sizeof(int) * chunks * nch, c->stream);
    chains_fork(c, nch);
    for (int k = 0; k < nch; ++k) {
      const Chain &ch = c->chain[k];
      cudaStream_t st = chain_stream(c, k);
      const int grid = grid_for(c, ch.t_cnt, smem);
      for (int i = 0; i < chunks; ++i) {
        GdMcArgs a = base_args(c);
        a.mode = 0;
        a.n_steps = spe;
        a.step0 = i * spe;
        a.step_base = c->d_cursor;
        a.tiles = c->d_chain_tiles + ch.t_off;
        a.n_tiles = ch.t_cnt;
        a.tile_counter = c->d_counters + k * chunks + i;
        launch_kernel(c)<<<grid, launch_threads(c), smem, st>>>(a, c->fc);
        if (exchange)
          gd::gd_exchange_kernel<<<(ch.xg1 - ch.xg0 + 127) / 128, 128, 0, st>>>(
              c->d_cx, c->d_group_base, c->n_complex, ch.xg0, ch.xg1, c->d_replica, c->d_etotal,
              c->d_acs, c->mc.seed, c->d_cursor + 1, i, !(i % 2));
      }
    }
    chains_join(c, nch);
    cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    if (ce != cudaSuccess) return fail(GD_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
    cudaGraphExec_t exec;
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return fail(GD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
    it = c->graphs.emplace(key, exec).first;
  }
  /* the graph reads its step and exchange-call bases from the device cursor */
  CK(cudaStreamSynchronize(c->stream));
  c->h_cursor[0] = s1;
  c->h_cursor[1] = c->exchange_calls;
  CK(cudaMemcpyAsync(c->d_cursor, c->h_cursor, 2 * sizeof(int), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaGraphLaunch(it->second, c->stream));
  if (exchange) c->exchange_calls += chunks;
  return rs_enqueue(c, n_steps);
}

int gd_sync(gd_ctx *c) {
  if (!c) return fail(GD_ERR_INVALID, "null context");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  unsigned err = 0;
  CK(cudaMemcpy(&err, c->d_err, sizeof(err), cudaMemcpyDeviceToHost));
  if (err & GD_DEV_ERR_TIMEOUT)
    return fail(GD_ERR_TIMEOUT, "a bounded device wait gave up (protein tile copy)");
  if (err & GD_DEV_ERR_RECORD_FULL)
    return fail(GD_ERR_RECORD_FULL, "a replica's record buffer overflowed; reset records per dump");
  return GD_OK;
}

int gd_get_stream(gd_ctx *c, void **stream) {
  if (!c || !stream) return fail(GD_ERR_INVALID, "null argument");
  *stream = (void *)c->stream;
  return GD_OK;
}

int gd_get_device_error(gd_ctx *c, int *code) {
  if (!c || !code) return fail(GD_ERR_INVALID, "null argument");
  CK(cudaStreamSynchronize(c->stream));
  unsigned err = 0;
  CK(cudaMemcpy(&err, c->d_err, sizeof(err), cudaMemcpyDeviceToHost));
  *code = (int)err;
  return GD_OK;
}

int gd_get_records_raw(gd_ctx *c, gd_record_step *steps, int *next_ptr, int r0, int r1,
                       int cap) {
  if (!c || !steps || !next_ptr) return fail(GD_ERR_INVALID, "null argument");
  if (!c->mc.record || !c->d_rec) return fail(GD_ERR_STATE, "records are disabled");
  int rc = check_range(c, r0, r1);
  if (rc) return rc;
  if (cap < 1 || cap > c->rec_cap)
    return fail(GD_ERR_INVALID, "cap %d outside 1..record capacity %d", cap, c->rec_cap);
  const int n = r1 - r0 + 1;
  CK(cudaStreamSynchronize(c->stream));
  const size_t rs = sizeof(gd_record_step);
  /* the first cap records of each replica */
  CK(d2h_rows(steps, rs * cap, c->d_rec + (size_t)r0 * c->rec_cap, rs * c->rec_cap,
              rs * cap, n));
  CK(cudaMemcpy(next_ptr, c->d_rec_next + r0, sizeof(int) * n, cudaMemcpyDeviceToHost));
  return GD_OK;
}

int gd_get_record_counts(gd_ctx *c, int *next_ptr, int r0, int r1) {
  if (!c || !next_ptr) return fail(GD_ERR_INVALID, "null argument");
  if (!c->mc.record || !c->d_rec) return fail(GD_ERR_STATE, "records are disabled");
  int rc = check_range(c, r0, r1);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(next_ptr, c->d_rec_next + r0, sizeof(int) * (r1 - r0 + 1),
                cudaMemcpyDeviceToHost));
  return GD_OK;
}

int gd_records_stream(gd_ctx *c, gd_record_step *steps, int cap) {
  if (!c) return fail(GD_ERR_INVALID, "null context");
  if (c->rs) {
    const int rc = rs_flush(c);
    rs_stop(c);
    if (rc) return rc;
  }
  if (!steps) return GD_OK;
  if (!c->mc.record || !c->d_rec) return fail(GD_ERR_STATE, "records are disabled");
  if (cap < 1 || cap > c->rec_cap)
    return fail(GD_ERR_INVALID, "cap %d outside 1..record capacity %d", cap, c->rec_cap);
  CK(cudaSetDevice(c->device));
  RecStream *r = new RecStream;
  r->host = steps;
  r->cap = cap;
  r->n_rep = c->n_rep;
  r->rec_cap = c->rec_cap;
  r->device = c->device;
  r->d_rec = c->d_rec;
  r->snap.assign(c->n_rep, 0);
  cudaError_t e = cudaStreamCreateWithFlags(&r->cs, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&r->d_prev, sizeof(int) * (size_t)c->n_rep);
  if (e == cudaSuccess) e = cudaMemsetAsync(r->d_prev, 0, sizeof(int) * (size_t)c->n_rep, c->stream);
  if (e == cudaSuccess) e = cudaHostAlloc(&r->h_plan, sizeof(int) * r->plan_ints(), 0);
  for (int i = 0; i < RecStream::NSNAP && e == cudaSuccess; ++i) {
    e = cudaMalloc(&r->d_plan[i], sizeof(int) * r->plan_ints());
    if (e == cudaSuccess)
      e = cudaEventCreateWithFlags(&r->ev[i], cudaEventDisableTiming | cudaEventBlockingSync);
  }
  c->rs = r;
  if (e != cudaSuccess) {
    rs_stop(c);
    return fail(GD_ERR_CUDA, "gd_records_stream: %s", cudaGetErrorString(e));
  }
  /* the first snapshot copies the rows written before the stream started */
  std::vector<int> cnt(c->n_rep);
  e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy(cnt.data(), c->d_rec_next, sizeof(int) * cnt.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    rs_stop(c);
    return fail(GD_ERR_CUDA, "gd_records_stream: %s", cudaGetErrorString(e));
  }
  int rows = 0;
  for (int v : cnt) rows = std::max(rows, std::min(v, cap));
  r->th = std::thread([r] { r->worker(); });
  return rs_enqueue(c, rows);
}

int gd_records_stream_flush(gd_ctx *c, int *next_ptr) {
  if (!c || !c->rs) return fail(GD_ERR_STATE, "gd_records_stream is not active");
  const int rc = rs_flush(c);
  if (rc) return rc;
  if (next_ptr) {
    std::lock_guard<std::mutex> lk(c->rs->mu);
    std::copy(c->rs->snap.begin(), c->rs->snap.end(), next_ptr);
  }
  return GD_OK;
}

int gd_get_records(gd_ctx *c, gd_lig_record *host, int r0, int r1) {
  if (!c || !host) return fail(GD_ERR_INVALID, "null argument");
  if (c->rec_cap != GD_STEPS_PER_DUMP + 1)
    return fail(GD_ERR_INVALID, "LigRecord layout needs steps_per_dump == %d", GD_STEPS_PER_DUMP);
  if (!c->mc.record || !c->d_rec) return fail(GD_ERR_STATE, "records are disabled");
  int rc = check_range(c, r0, r1);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  const int n = r1 - r0 + 1;
  std::vector<int> nxt(n);
  CK(cudaMemcpy(nxt.data(), c->d_rec_next + r0, sizeof(int) * n, cudaMemcpyDeviceToHost));
  CK(d2h_rows(host[0].step, sizeof(gd_lig_record), c->d_rec + (size_t)r0 * c->rec_cap,
              sizeof(gd_record_step) * c->rec_cap, sizeof(gd_record_step) * c->rec_cap, n));
  for (int i = 0; i < n; ++i) host[i].next_ptr = nxt[i];
  return GD_OK;
}

int gd_get_etotal(gd_ctx *c, float *et, int r0, int r1) {
  if (!c || !et) return fail(GD_ERR_INVALID, "null argument");
  int rc = check_range(c, r0, r1);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(et, c->d_etotal + r0, sizeof(float) * (r1 - r0 + 1), cudaMemcpyDeviceToHost));
  return GD_OK;
}

int gd_get_replicas(gd_ctx *c, gd_replica *rp, int r0, int r1) {
  if (!c || !rp) return fail(GD_ERR_INVALID, "null argument");
  int rc = check_range(c, r0, r1);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(rp, c->d_replica + r0, sizeof(gd_replica) * (r1 - r0 + 1),
                cudaMemcpyDeviceToHost));
  return GD_OK;
}

int gd_get_state(gd_ctx *c, gd_replica_state *st, int r0, int r1) {
  if (!c || !st) return fail(GD_ERR_INVALID, "null argument");
  int rc = check_range(c, r0, r1);
  if (rc) return rc;
  const int n = r1 - r0 + 1;
  std::vector<float> mm((size_t)n * 6);
  std::vector<gd_energy> e(n);
  std::vector<gd_replica> rp(n);
  std::vector<int> na(n), ac(n);
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(mm.data(), c->d_mm + (size_t)r0 * 6, sizeof(float) * 6 * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(e.data(), c->d_eold + r0, sizeof(gd_energy) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(rp.data(), c->d_replica + r0, sizeof(gd_replica) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(na.data(), c->d_nacc + r0, sizeof(int) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ac.data(), c->d_acs + r0, sizeof(int) * n, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; ++i) {
    memcpy(st[i].movematrix_old, &mm[(size_t)i * 6], sizeof(float) * 6);
    st[i].energy_old = e[i];
    st[i].replica = rp[i];
    st[i].n_accept = na[i];
    st[i].n_exchange = ac[i];
  }
  return GD_OK;
}

int gd_set_state(gd_ctx *c, const gd_replica_state *st, int r0, int r1) {
  if (!c || !st) return fail(GD_ERR_INVALID, "null argument");
  int rc = check_range(c, r0, r1);
  if (rc) return rc;
  const int n = r1 - r0 + 1;
  std::vector<float> mm((size_t)n * 6), et(n);
  std::vector<gd_energy> e(n);
  std::vector<gd_replica> rp(n);
  std::vector<int> na(n), ac(n);
  for (int i = 0; i < n; ++i) {
    const gd_replica &want = st[i].replica;
    const int r = r0 + i;
    int ci = 0;
    while (ci + 1 < c->n_complex && c->info[ci + 1].rep_offset <= r) ++ci;
    const ComplexInfo &x = c->info[ci];
    if (want.idx_tmp < 0 || want.idx_tmp >= x.n_tmp)
      return fail(GD_ERR_INVALID, "state %d: idx_tmp %d out of range", i, want.idx_tmp);
    memcpy(&mm[(size_t)i * 6], st[i].movematrix_old, sizeof(float) * 6);
    e[i] = st[i].energy_old;
    et[i] = st[i].energy_old.e[GD_MAXWEI - 1];
    rp[i] = st[i].replica;
    na[i] = st[i].n_accept;
    ac[i] = st[i].n_exchange;
  }
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(c->d_mm + (size_t)r0 * 6, mm.data(), sizeof(float) * 6 * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_eold + r0, e.data(), sizeof(gd_energy) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_etotal + r0, et.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_replica + r0, rp.data(), sizeof(gd_replica) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_nacc + r0, na.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_acs + r0, ac.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  c->initialized = true;
  return GD_OK;
}

int gd_eval_energy(gd_ctx *c, int ci, int prt_conf, int lig_conf, const float *mm, int n,
                   gd_energy *out) {
  if (!c || !mm || !out) return fail(GD_ERR_INVALID, "null argument");
  if (ci < 0 || ci >= c->n_complex) return fail(GD_ERR_INVALID, "bad complex index");
  const ComplexInfo &x = c->info[ci];
  if (prt_conf < 0 || prt_conf >= x.n_prt || lig_conf < 0 || lig_conf >= x.n_lig)
    return fail(GD_ERR_INVALID, "conformer index out of range");
  if (n < 1) return GD_OK;
  CK(cudaSetDevice(c->device));
  if (n > c->eval_cap) {
    if (c->d_mm_in) cudaFree(c->d_mm_in);
    if (c->d_lc_in) cudaFree(c->d_lc_in);
    if (c->d_e_out) cudaFree(c->d_e_out);
    c->d_mm_in = nullptr; c->d_lc_in = nullptr; c->d_e_out = nullptr; c->eval_cap = 0;
    CK(cudaMalloc(&c->d_mm_in, sizeof(float) * 6 * n));
    CK(cudaMalloc(&c->d_lc_in, sizeof(int) * n));
    CK(cudaMalloc(&c->d_e_out, sizeof(gd_energy) * n));
    c->eval_cap = n;
  }
  std::vector<GdTileDesc> tiles;
  for (int i = 0; i < n; i += x.k) {
    GdTileDesc t;
    t.complex_index = ci;
    t.prt_conf = prt_conf;
    t.rep_begin = i;
    t.count = std::min(x.k, n - i);
    tiles.push_back(t);
  }
  if ((int)tiles.size() > c->eval_tiles_cap) {
    if (c->d_eval_tiles) cudaFree(c->d_eval_tiles);
    c->d_eval_tiles = nullptr;
    CK(cudaMalloc(&c->d_eval_tiles, sizeof(GdTileDesc) * tiles.size()));
    c->eval_tiles_cap = (int)tiles.size();
  }
  std::vector<int> lc(n, lig_conf);
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(c->d_mm_in, mm, sizeof(float) * 6 * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_lc_in, lc.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_eval_tiles, tiles.data(), sizeof(GdTileDesc) * tiles.size(),
                cudaMemcpyHostToDevice));
  GdMcArgs a = base_args(c);
  a.mode = 2;
  a.n_steps = 1;
  a.mm_in = c->d_mm_in;
  a.lig_conf_in = c->d_lc_in;
  a.e_out = c->d_e_out;
  a.rec = nullptr;
  a.trace_e = nullptr;
  int rc = launch_mc(c, a, c->d_eval_tiles, (int)tiles.size(), c->d_counters);
  if (rc) return rc;
  if ((rc = gd_sync(c))) return rc;
  CK(cudaMemcpy(out, c->d_e_out, sizeof(gd_energy) * n, cudaMemcpyDeviceToHost));
  return GD_OK;
}

/* One thread per (pose, atom): the rotation of the pose and the placed atom, with the same
 * gd_rotation / gd_place_atom the Monte Carlo kernel places its ligands with. */
__global__ void gd_place_kernel(const GdDevComplex *cxs, int ci, int lig_conf, const float *mm,
                                int n, float *xyz) {
  const GdDevComplex &cx = cxs[ci];
  const int L = cx.lna;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)n * L) return;
  const int pose = (int)(i / L), l = (int)(i % L);
  float m[6], rot[9];
  for (int k = 0; k < 6; ++k) m[k] = mm[pose * 6 + k];
  gd_rotation(m, rot);
  const float *lc = cx.lig_center + lig_conf * 3;
  const float4 o = cx.lig_pos[lig_conf * L + l];
  gd_place_atom(rot, GD_ADD(m[0], lc[0]), GD_ADD(m[1], lc[1]), GD_ADD(m[2], lc[2]), o.x, o.y,
                o.z, &xyz[i * 3], &xyz[i * 3 + 1], &xyz[i * 3 + 2]);
}

int gd_place_ligand(gd_ctx *c, int ci, int lig_conf, const float *mm, int n, float *xyz) {
  if (!c || (n > 0 && (!mm || !xyz))) return fail(GD_ERR_INVALID, "null argument");
  if (ci < 0 || ci >= c->n_complex) return fail(GD_ERR_INVALID, "bad complex index");
  const ComplexInfo &x = c->info[ci];
  if (lig_conf < 0 || lig_conf >= x.n_lig)
    return fail(GD_ERR_INVALID, "ligand conformer %d out of range [0, %d)", lig_conf, x.n_lig);
  if (n < 0) return fail(GD_ERR_INVALID, "negative pose count");
  if (n == 0) return GD_OK;
  CK(cudaSetDevice(c->device));
  const size_t out_bytes = sizeof(float) * 3 * (size_t)x.lna * n;
  float *d_mm = nullptr, *d_xyz = nullptr;
  CK(cudaStreamSynchronize(c->stream));
  cudaError_t e = cudaMalloc(&d_mm, sizeof(float) * 6 * (size_t)n);
  if (e == cudaSuccess) e = cudaMalloc(&d_xyz, out_bytes);
  if (e == cudaSuccess) e = cudaMemcpy(d_mm, mm, sizeof(float) * 6 * (size_t)n,
                                       cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const long long total = (long long)n * x.lna;
    gd_place_kernel<<<(unsigned)((total + 255) / 256), 256, 0, c->stream>>>(c->d_cx, ci, lig_conf,
                                                                           d_mm, n, d_xyz);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) e = cudaMemcpy(xyz, d_xyz, out_bytes, cudaMemcpyDeviceToHost);
  cudaFree(d_mm);
  cudaFree(d_xyz);
  if (e != cudaSuccess) return fail(GD_ERR_CUDA, "gd_place_ligand: %s", cudaGetErrorString(e));
  return GD_OK;
}

int gd_trace_enable(gd_ctx *c, int max_steps) {
  if (!c || max_steps < 0) return fail(GD_ERR_INVALID, "bad argument");
  CK(cudaStreamSynchronize(c->stream));
  if (c->d_trace_e) cudaFree(c->d_trace_e);
  if (c->d_trace_acc) cudaFree(c->d_trace_acc);
  c->d_trace_e = nullptr;
  c->d_trace_acc = nullptr;
  c->trace_cap = 0;
  drop_graphs(c);
  if (max_steps == 0) return GD_OK;
  CK(cudaMalloc(&c->d_trace_e, sizeof(float) * (size_t)c->n_rep * max_steps));
  CK(cudaMalloc(&c->d_trace_acc, sizeof(int) * (size_t)c->n_rep * max_steps));
  CK(cudaMemset(c->d_trace_acc, 0xff, sizeof(int) * (size_t)c->n_rep * max_steps));
  c->trace_cap = max_steps;
  c->trace_step0 = 0;
  return GD_OK;
}

int gd_trace_get(gd_ctx *c, float *e_new, int *acc, int *n_steps) {
  if (!c || !e_new || !acc || !n_steps) return fail(GD_ERR_INVALID, "null argument");
  if (!c->trace_cap) return fail(GD_ERR_STATE, "trace disabled");
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(e_new, c->d_trace_e, sizeof(float) * (size_t)c->n_rep * c->trace_cap,
                cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(acc, c->d_trace_acc, sizeof(int) * (size_t)c->n_rep * c->trace_cap,
                cudaMemcpyDeviceToHost));
  *n_steps = c->trace_cap;
  return GD_OK;
}

}  // extern "C"

/* ---------------- pose evaluation without allocation ----------------
 *
 * Some callers cannot call cudaMalloc at the moment they need energies: code that runs while
 * another framework owns all device memory through its own pool, code inside a real-time or
 * callback context where an allocation (and its implicit synchronisation) is not allowed, or
 * a host that has already placed its poses and result buffer in device memory it manages.
 * gd_eval_energy_noalloc serves them: it reads poses from, and writes energies to, device
 * buffers the caller passes, and keeps the only scratch it needs (the pose work queue, the
 * tile list and the per-pose conformer index) in the fixed device array below. That array
 * holds up to GD_NOALLOC_MAX_POSES poses, is allocated once when the library is loaded on a
 * device and stays there until the process exits, and is shared by every call in the
 * process: each call rewrites the parts it uses (the queue head is cleared by the fill
 * kernel), and calls whose kernels overlap on the GPU would race on it. Its device address
 * is looked up by gd_create (which allocates anyway), once per device, so the entry point
 * itself only reads the cached address. */

namespace {

struct NoallocScratch {
  GdTileDesc tiles[GD_NOALLOC_MAX_POSES];
  int lig_conf[GD_NOALLOC_MAX_POSES];
  int counter;
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoallocScratch)];

/* Writes the tile list, the per-pose conformer index and a cleared queue head into the
 * scratch array for n poses of one (complex, protein conformer, ligand conformer). */
__global__ void gd_noalloc_fill(int complex_index, int prt_conf, int lig_conf, int n, int k) {
  NoallocScratch *s = reinterpret_cast<NoallocScratch *>(g_noalloc_scratch);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) s->counter = 0;
  if (i < n) {
    s->lig_conf[i] = lig_conf;
    if (i % k == 0) {
      GdTileDesc t;
      t.complex_index = complex_index;
      t.prt_conf = prt_conf;
      t.rep_begin = i;
      t.count = min(k, n - i);
      s->tiles[i / k] = t;
    }
  }
}

std::mutex g_noalloc_mu;
void *g_noalloc_addr[64] = {nullptr};

/* Set-up on `device` (the current device), once per device, from gd_create: the device
 * address of the scratch array (host code cannot use the symbol itself as a device address)
 * and the fill kernel's attributes, which load the module's code and data under lazy module
 * loading, so that no later call of the entry point loads anything. */
int noalloc_prepare(int device) {
  if (device < 0 || device >= 64) return fail(GD_ERR_NODEVICE, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_addr[device]) return GD_OK;
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return fail(GD_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
  cudaFuncAttributes fa;
  e = cudaFuncGetAttributes(&fa, gd_noalloc_fill);
  if (e != cudaSuccess)
    return fail(GD_ERR_CUDA, "cudaFuncGetAttributes(fill) failed: %s", cudaGetErrorString(e));
  g_noalloc_addr[device] = p;
  return GD_OK;
}

/* The scratch array's device address cached by noalloc_prepare for `device`. */
int noalloc_scratch(int device, NoallocScratch **out) {
  if (device < 0 || device >= 64) return fail(GD_ERR_NODEVICE, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device])
    return fail(GD_ERR_STATE, "allocation-free scratch not set up on device %d", device);
  *out = reinterpret_cast<NoallocScratch *>(g_noalloc_addr[device]);
  return GD_OK;
}

}  // namespace

extern "C" int gd_eval_energy_noalloc(gd_ctx *c, int ci, int prt_conf, int lig_conf,
                                      const float *d_movematrix, int n, gd_energy *d_out) {
  if (!c || !d_movematrix || !d_out) return fail(GD_ERR_INVALID, "null argument");
  if (ci < 0 || ci >= c->n_complex) return fail(GD_ERR_INVALID, "bad complex index");
  const ComplexInfo &x = c->info[ci];
  if (prt_conf < 0 || prt_conf >= x.n_prt || lig_conf < 0 || lig_conf >= x.n_lig)
    return fail(GD_ERR_INVALID, "conformer index out of range");
  if (n < 0) return fail(GD_ERR_INVALID, "gd_eval_energy_noalloc: negative pose count %d", n);
  if (n > GD_NOALLOC_MAX_POSES)
    return fail(GD_ERR_CAPACITY,
                "gd_eval_energy_noalloc: %d poses; the allocation-free path holds at most %d "
                "(split the batch or use gd_eval_energy)",
                n, GD_NOALLOC_MAX_POSES);
  if (n == 0) return GD_OK;
  CK(cudaSetDevice(c->device));
  NoallocScratch *s = nullptr;
  int rc = noalloc_scratch(c->device, &s);
  if (rc) return rc;
  const int k = x.k, n_tiles = (n + k - 1) / k;
  gd_noalloc_fill<<<(n + 255) / 256, 256, 0, c->stream>>>(ci, prt_conf, lig_conf, n, k);
  CK(cudaGetLastError());
  GdMcArgs a = base_args(c);
  a.mode = 2;
  a.n_steps = 1;
  a.mm_in = d_movematrix;
  a.lig_conf_in = s->lig_conf;
  a.e_out = d_out;
  a.rec = nullptr;
  a.trace_e = nullptr;
  a.tiles = s->tiles;
  a.n_tiles = n_tiles;
  a.tile_counter = &s->counter;
  const size_t smem = smem_bytes(c);
  if ((rc = set_kernel_attrs(c, smem))) return rc;
  const int grid = grid_for(c, n_tiles, smem);
  launch_kernel(c)<<<grid, launch_threads(c), smem, c->stream>>>(a, c->fc);
  CK(cudaGetLastError());
  return GD_OK;
}

/* ======================= surrogate and delayed acceptance ======================= */

struct DaState {
  gd::Mlp net;
  gd_sur_params prm{};
  std::vector<gd::GdGroup> groups;
  int n_tiles = 0, built_gen = -1, built_split = -1;
  int split = 1;                                 /* protein split of the exact stage */
  double last_pass = 1.0;                        /* surrogate-stage pass rate, last window */
  unsigned long long prev_prop = 0, prev_pass = 0;
  std::vector<void *> allocs;
  int *d_rep_cx = nullptr, *d_rep_group = nullptr, *d_group_b0 = nullptr;
  int *d_emb_base = nullptr, *d_active = nullptr;
  float *d_pocket = nullptr;
  float *d_u2 = nullptr, *d_s_cur = nullptr, *d_s_new = nullptr, *d_pose_mm = nullptr;
  int *d_pose_rep = nullptr, *d_pose_lc = nullptr;
  int *d_cnt = nullptr;                          /* [2][n_groups] survivor counters */
  GdTileDesc *d_tiles = nullptr;
  /* per-replica counters */
  int *d_prop = nullptr, *d_pass = nullptr, *d_plain = nullptr, *d_acc = nullptr,
      *d_plain_acc = nullptr, *d_nerr = nullptr;
  double *d_err2 = nullptr;
  GdDaEpi epi{};                                 /* host copy of the device struct */
  GdDaEpi *d_epi = nullptr;
  unsigned long long *d_stats = nullptr;         /* [n_complex][GD_DA_NSTAT] (da_stats) */
  double *d_err = nullptr;                       /* [n_complex][GD_DA_NERR] */
  __nv_bfloat16 *smp_X = nullptr;
  int *smp_conf = nullptr;
  float *smp_t = nullptr;
  long long smp_cap = 0, smp_lo = 0, smp_hi = 0; /* global sample indices written: [lo, hi) */
  long long norm_hi = -1;                        /* sample set the normalisation was made on */
  float *d_t = nullptr;
  double *d_mom = nullptr;
  float *d_loss_hist = nullptr;
  int loss_cap = 0;
  long long train_iter = 0;
  float *d_pred_mm = nullptr;
  int pred_cap = 0;
  float *tr_s = nullptr, *tr_e = nullptr;
  int *tr_flag = nullptr;
  int tr_cap = 0, tr_step0 = 0;
  std::vector<int> active;
  std::vector<unsigned long long> window0; /* counters at the last controller decision */
  std::map<long long, cudaGraphExec_t> graphs;
  int *d_counters = nullptr;               /* persistent-CTA queue heads, one per step */
  int counters_cap = 0;
};

namespace {

template <class T>
int da_alloc(DaState *d, T **p, size_t n) {
  *p = nullptr;
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, std::max<size_t>(1, n) * sizeof(T));
  if (e != cudaSuccess)
    return fail(GD_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", n * sizeof(T), cudaGetErrorString(e));
  d->allocs.push_back(q);
  *p = (T *)q;
  return GD_OK;
}

void da_free_trace(DaState *d) {
  if (d->tr_s) cudaFree(d->tr_s);
  if (d->tr_e) cudaFree(d->tr_e);
  if (d->tr_flag) cudaFree(d->tr_flag);
  d->tr_s = d->tr_e = nullptr;
  d->tr_flag = nullptr;
  d->tr_cap = 0;
}

void da_drop_graphs(gd_ctx *c) {
  if (!c->da) return;
  for (auto &g : c->da->graphs) cudaGraphExecDestroy(g.second);
  c->da->graphs.clear();
}

void da_free(gd_ctx *c) {
  DaState *d = c->da;
  if (!d) return;
  da_drop_graphs(c);
  gd::mlp_destroy(d->net);
  for (void *p : d->allocs) cudaFree(p);
  if (d->d_loss_hist) cudaFree(d->d_loss_hist);
  if (d->d_pred_mm) cudaFree(d->d_pred_mm);
  if (d->d_counters) cudaFree(d->d_counters);
  da_free_trace(d);
  delete d;
  c->da = nullptr;
}

/* the device struct the exact kernel reads in mode 3 (trace pointers included) */
int da_upload_epi(gd_ctx *c) {
  DaState *d = c->da;
  GdDaEpi &e = d->epi;
  e.group_b0 = d->d_group_b0;
  e.n_groups = (int)d->groups.size();
  e.n_rep = c->n_rep;
  e.pose_rep = d->d_pose_rep;
  e.s_new = d->d_s_new;
  e.s_cur = d->d_s_cur;
  e.u2 = d->d_u2;
  e.active = d->d_active;
  e.acc = d->d_acc;
  e.plain_acc = d->d_plain_acc;
  e.err2 = d->d_err2;
  e.nerr = d->d_nerr;
  e.smp_t = d->smp_t;
  e.smp_cap = d->smp_cap;
  e.tr_s = d->tr_s;
  e.tr_e = d->tr_e;
  e.tr_flag = d->tr_flag;
  e.tr_cap = d->tr_cap;
  e.tr_step0 = d->tr_step0;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(d->d_epi, &e, sizeof(e), cudaMemcpyHostToDevice));
  return GD_OK;
}

/* groups and the exact kernel's static tile list for the current tile shapes and the exact
 * stage's split S: tile i of group g covers pose slots [b0 + i k, b0 + i k + cap), k the
 * replicas a CTA holds at split S, and carries (g << 8) | cap */
int da_build_groups(gd_ctx *c, int S) {
  DaState *d = c->da;
  if (d->built_gen == c->tile_gen && d->built_split == S && d->d_tiles) return GD_OK;
  std::vector<gd::GdGroup> g;
  std::vector<GdTileDesc> tiles;
  std::vector<int> rep_group(c->n_rep), b0s;
  for (int ci = 0; ci < c->n_complex; ++ci) {
    const ComplexInfo &x = c->info[ci];
    const int block = x.n_tmp * x.n_lig;
    for (int p = 0; p < x.n_prt; ++p) {
      gd::GdGroup q;
      q.ci = ci;
      q.pc = p;
      q.b0 = x.rep_offset + p * block;
      q.n = block;
      q.k = std::max(1, std::min(x.k, c->threads / (S * x.lna)));
      q.n_tiles = (block + q.k - 1) / q.k;
      q.tile_base = (int)tiles.size();
      q.pad = 0;
      const int gi = (int)g.size();
      for (int i = 0; i < q.n_tiles; ++i) {
        GdTileDesc t;
        t.complex_index = ci;
        t.prt_conf = p;
        t.rep_begin = q.b0 + i * q.k;
        t.count = (gi << 8) | std::min(q.k, block - i * q.k);
        tiles.push_back(t);
      }
      for (int r = 0; r < block; ++r) rep_group[q.b0 + r] = gi;
      b0s.push_back(q.b0);
      g.push_back(q);
    }
  }
  if (g.size() >= (1u << 23)) return fail(GD_ERR_CAPACITY, "too many compaction groups");
  CK(cudaStreamSynchronize(c->stream));
  const bool first = d->d_group_b0 == nullptr;
  if (first) {
    int rc;
    if ((rc = da_alloc(d, &d->d_group_b0, g.size()))) return rc;
    if ((rc = da_alloc(d, &d->d_rep_group, (size_t)c->n_rep))) return rc;
    if ((rc = da_alloc(d, &d->d_cnt, 2 * g.size()))) return rc;
    CK(cudaMemcpy(d->d_group_b0, b0s.data(), sizeof(int) * b0s.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d->d_rep_group, rep_group.data(), sizeof(int) * c->n_rep,
                  cudaMemcpyHostToDevice));
    CK(cudaMemset(d->d_cnt, 0, sizeof(int) * 2 * g.size()));
  }
  if ((int)tiles.size() > d->n_tiles) {
    if (d->d_tiles) {
      cudaFree(d->d_tiles);
      d->allocs.erase(std::remove(d->allocs.begin(), d->allocs.end(), (void *)d->d_tiles),
                      d->allocs.end());
      d->d_tiles = nullptr;
    }
    int rc = da_alloc(d, &d->d_tiles, tiles.size());
    if (rc) return rc;
  }
  CK(cudaMemcpy(d->d_tiles, tiles.data(), sizeof(GdTileDesc) * tiles.size(),
                cudaMemcpyHostToDevice));
  d->groups = g;
  d->n_tiles = (int)tiles.size();
  d->built_gen = c->tile_gen;
  d->built_split = S;
  return GD_OK;
}

/* largest split every complex of the batch fits into the context's CTA */
int da_max_split(const gd_ctx *c) {
  int m = 16;
  for (const auto &x : c->info) m = std::min(m, std::max(1, c->threads / x.lna));
  return m;
}

/* split of the next delayed-acceptance run from the surrogate stage's last pass rate: with
 * few survivors one exact-stage tile per CTA sets the step's latency, and more lanes per atom
 * shorten it, at the price of fewer replicas sharing each staged protein chunk. Thresholds
 * from config-1 sweeps (ms per 10 steps at pass 0.50 / 0.30 / 0.195 / 0.097: split 1 6.9 /
 * 6.1 / 6.0 / 5.8, split 2 8.4 / 5.4 / 4.2 / 4.0, split 3 9.7 / 6.0 / 4.3 / 3.3). */
int da_choose_split(const gd_ctx *c, bool collect) {
  const DaState *d = c->da;
  if (collect) return c->split;
  const int mx = da_max_split(c);
  if (d->prm.split > 0) return std::min(d->prm.split, mx);
  const double p = d->last_pass;
  const int S = p > 0.4 ? 1 : (p > 0.13 ? 2 : (p > 0.05 ? 3 : 4));
  return std::max(c->split, std::min(S, mx));
}

gd::GdDaDev da_args(gd_ctx *c) {
  DaState *d = c->da;
  gd::GdDaDev a;
  memset(&a, 0, sizeof(a));
  a.cx = c->d_cx;
  a.rep_cx = d->d_rep_cx;
  a.rep_group = d->d_rep_group;
  a.group_b0 = d->d_group_b0;
  a.emb_base = d->d_emb_base;
  a.pocket_feat = d->d_pocket;
  a.active = d->d_active;
  a.n_rep = c->n_rep;
  a.replica = c->d_replica;
  a.mm_old = c->d_mm;
  a.u2 = d->d_u2;
  a.s_cur = d->d_s_cur;
  a.s_new = d->d_s_new;
  a.pose_rep = d->d_pose_rep;
  a.pose_mm = d->d_pose_mm;
  a.pose_lc = d->d_pose_lc;
  a.prop = d->d_prop;
  a.pass = d->d_pass;
  a.plain = d->d_plain;
  a.theta = d->net.theta;
  a.wf = d->net.wf;
  a.L = d->net.L;
  a.mu = d->net.mu;
  a.sigma = d->net.sigma;
  a.X = d->net.X;
  a.conf = d->net.conf;
  a.smp_X = d->smp_X;
  a.smp_conf = d->smp_conf;
  a.smp_t = d->smp_t;
  a.smp_cap = d->smp_cap;
  a.tr_s = d->tr_s;
  a.tr_e = d->tr_e;
  a.tr_flag = d->tr_flag;
  a.tr_cap = d->tr_cap;
  a.tr_step0 = d->tr_step0;
  a.seed = c->mc.seed;
  a.move_kind = c->mc.move_kind;
  for (int i = 0; i < 6; ++i) a.move_scale[i] = c->mc.move_scale[i];
  a.step_base = c->d_cursor;
  return a;
}

/* the exact stage of step j of one chain: gd_mc_kernel mode 3 over the chain's part of the
 * static tile list */
void da_launch_exact(gd_ctx *c, const Chain &ch, int k, int n_steps, int j, bool collect,
                     size_t smem, cudaStream_t st, int S) {
  DaState *d = c->da;
  const int ng = (int)d->groups.size();
  const int t0 = d->groups[ch.g0].tile_base;
  const int t1 = d->groups[ch.g1 - 1].tile_base + d->groups[ch.g1 - 1].n_tiles;
  GdMcArgs a = base_args(c);
  a.mode = 3;
  a.n_steps = 1;
  a.step0 = j;
  a.step_base = c->d_cursor;
  a.trace_e = nullptr;
  a.trace_acc = nullptr;
  a.mm_in = d->d_pose_mm;
  a.lig_conf_in = d->d_pose_lc;
  a.tiles = d->d_tiles + t0;
  a.n_tiles = t1 - t0;
  a.tile_counter = d->d_counters + (size_t)k * n_steps + j;
  a.da = d->d_epi;
  a.da_cnt = d->d_cnt + (size_t)(j & 1) * ng;
  a.da_cnt_next = d->d_cnt + (size_t)((j + 1) & 1) * ng;
  a.da_g0 = ch.g0;
  a.da_g1 = ch.g1;
  a.da_collect = collect ? 1 : 0;
  a.split = S;
  mc_kernel(c->unroll, S, true)<<<grid_for(c, t1 - t0, smem, S, true), c->threads, smem, st>>>(
      a, c->fc);
}

/* the graph of n_steps steps (collect: plain steps that store samples), one chain per stream */
int da_graph(gd_ctx *c, int n_steps, int exchange, bool collect, int S, cudaGraphExec_t *out) {
  DaState *d = c->da;
  const long long key =
      ((long long)n_steps << 7) | ((long long)S << 2) | (exchange ? 2 : 0) | (collect ? 1 : 0);
  auto it = d->graphs.find(key);
  if (it != d->graphs.end()) {
    *out = it->second;
    return GD_OK;
  }
  std::vector<Chain> chains;
  build_chains(c, c->chains_da, chains, nullptr);
  int rc = ensure_chain_streams(c, (int)chains.size());
  if (rc) return rc;
  const int nch = (int)chains.size();
  if (n_steps * nch > d->counters_cap) {
    if (d->d_counters) cudaFree(d->d_counters);
    d->d_counters = nullptr;
    d->counters_cap = 0;
    CK(cudaMalloc(&d->d_counters, sizeof(int) * n_steps * nch));
    d->counters_cap = n_steps * nch;
  }
  if ((rc = da_upload_epi(c))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  const size_t smem = smem_bytes(c);
  if ((rc = set_kernel_attrs(c, smem, S, true))) return rc;
  const gd::GdDaDev a = da_args(c);
  const int spe = c->mc.steps_per_exchange;
  const int ng = (int)d->groups.size();
  cudaGraph_t graph;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int frc = 0;
  cudaMemsetAsync(d->d_counters, 0, sizeof(int) * n_steps * nch, c->stream);
  cudaMemsetAsync(d->d_cnt, 0, sizeof(int) * 2 * ng, c->stream);
  chains_fork(c, nch);
  for (int k = 0; k < nch; ++k) {
    const Chain &ch = chains[k];
    cudaStream_t st = chain_stream(c, k);
    if (!collect) frc |= gd::da_front(a, GD_DA_CURRENT, 0, d->d_cnt, ch.r0, ch.r1, st);
    for (int j = 0; j < n_steps; ++j) {
      frc |= gd::da_front(a, collect ? GD_DA_COLLECT : GD_DA_STEP, j,
                          d->d_cnt + (size_t)(j & 1) * ng, ch.r0, ch.r1, st);
      da_launch_exact(c, ch, k, n_steps, j, collect, smem, st, S);
      if (exchange && (j + 1) % spe == 0) {
        const int i = (j + 1) / spe - 1;
        gd::gd_exchange_kernel<<<(ch.xg1 - ch.xg0 + 127) / 128, 128, 0, st>>>(
            c->d_cx, c->d_group_base, c->n_complex, ch.xg0, ch.xg1, c->d_replica, c->d_etotal,
            c->d_acs, c->mc.seed, c->d_cursor + 1, i, !(i % 2));
      }
    }
  }
  chains_join(c, nch);
  cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
  if (ce != cudaSuccess) return fail(GD_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
  if (frc) {
    cudaGraphDestroy(graph);
    return fail(GD_ERR_INVALID, "delayed acceptance needs hidden = 128 or 256");
  }
  cudaGraphExec_t exec;
  ce = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) return fail(GD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
  d->graphs.emplace(key, exec);
  *out = exec;
  return GD_OK;
}

int da_run_steps(gd_ctx *c, int s1, int n_steps, int exchange, bool collect) {
  if (!c) return fail(GD_ERR_INVALID, "null context");
  if (!c->da) return fail(GD_ERR_STATE, "gd_sur_create has not run");
  if (!c->initialized) return fail(GD_ERR_STATE, "gd_mc_init has not run");
  const int spe = c->mc.steps_per_exchange;
  if (n_steps < 1 || (exchange && n_steps % spe))
    return fail(GD_ERR_INVALID, "n_steps must be >= 1 (a multiple of steps_per_exchange "
                                "with exchange)");
  if (s1 < 0) return fail(GD_ERR_INVALID, "s1 must be >= 0");
  CK(cudaSetDevice(c->device));
  const int S = da_choose_split(c, collect);
  if (c->da->built_split != S || c->da->built_gen != c->tile_gen) {
    /* tile lists and graphs of another split or tile shape are stale */
    CK(cudaStreamSynchronize(c->stream));
    da_drop_graphs(c);
  }
  int rc = da_build_groups(c, S);
  if (rc) return rc;
  c->da->split = S;
  cudaGraphExec_t g;
  if ((rc = da_graph(c, n_steps, exchange, collect, S, &g))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  c->h_cursor[0] = s1;
  c->h_cursor[1] = c->exchange_calls;
  CK(cudaMemcpyAsync(c->d_cursor, c->h_cursor, 2 * sizeof(int), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaGraphLaunch(g, c->stream));
  if (exchange) c->exchange_calls += n_steps / spe;
  return GD_OK;
}

int da_read_stats(gd_ctx *c, std::vector<unsigned long long> &st, std::vector<double> &er) {
  DaState *d = c->da;
  st.assign((size_t)c->n_complex * GD_DA_NSTAT, 0);
  er.assign((size_t)c->n_complex * GD_DA_NERR, 0.0);
  gd::da_stats(da_args(c), d->epi, c->d_cx, c->n_complex, d->d_stats, d->d_err, c->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(st.data(), d->d_stats, st.size() * sizeof(unsigned long long),
                cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(er.data(), d->d_err, er.size() * sizeof(double), cudaMemcpyDeviceToHost));
  return GD_OK;
}

int da_upload_active(gd_ctx *c) {
  DaState *d = c->da;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(d->d_active, d->active.data(), sizeof(int) * c->n_complex,
                cudaMemcpyHostToDevice));
  return GD_OK;
}

int da_reset_counters(gd_ctx *c) {
  DaState *d = c->da;
  const size_t R = c->n_rep;
  CK(cudaMemsetAsync(d->d_prop, 0, sizeof(int) * R, c->stream));
  CK(cudaMemsetAsync(d->d_pass, 0, sizeof(int) * R, c->stream));
  CK(cudaMemsetAsync(d->d_plain, 0, sizeof(int) * R, c->stream));
  CK(cudaMemsetAsync(d->d_acc, 0, sizeof(int) * R, c->stream));
  CK(cudaMemsetAsync(d->d_plain_acc, 0, sizeof(int) * R, c->stream));
  CK(cudaMemsetAsync(d->d_nerr, 0, sizeof(int) * R, c->stream));
  CK(cudaMemsetAsync(d->d_err2, 0, sizeof(double) * R, c->stream));
  d->window0.assign((size_t)c->n_complex * GD_DA_NSTAT, 0);
  d->prev_prop = d->prev_pass = 0;
  return GD_OK;
}

/* target normalisation: mean / std of the samples, then again inside mean +- 4 std */
int da_normalise(gd_ctx *c, long long start, long long n_valid) {
  DaState *d = c->da;
  gd::GdDaDev a = da_args(c);
  std::vector<double> part(GD_DA_MOM_BLOCKS * 3);
  double lo = -INFINITY, hi = INFINITY, mean = 0.0, sd = 1.0;
  for (int pass = 0; pass < 2; ++pass) {
    gd::da_target_moments(a, start, n_valid, (float)lo, (float)hi, d->d_mom, c->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaMemcpy(part.data(), d->d_mom, sizeof(double) * part.size(), cudaMemcpyDeviceToHost));
    double s0 = 0, s1 = 0, n = 0;
    for (int b = 0; b < GD_DA_MOM_BLOCKS; ++b) {
      s0 += part[b * 3];
      s1 += part[b * 3 + 1];
      n += part[b * 3 + 2];
    }
    if (n < 1) break;
    mean = s0 / n;
    sd = std::sqrt(std::max(0.0, s1 / n - mean * mean));
    lo = mean - 4.0 * sd;
    hi = mean + 4.0 * sd;
  }
  d->net.mu = (float)mean;
  d->net.sigma = (float)std::max(sd, 1e-3);
  return GD_OK;
}

}  // namespace

struct gd_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  gd::Mlp net;
  float *d_x = nullptr, *d_t = nullptr;
  int *d_conf = nullptr;
  int cap = 0;
};

namespace {

int mlp_stage_rows(gd_mlp *m, const float *x, const int *conf, int rows) {
  if (rows > m->cap) {
    if (m->d_x) cudaFree(m->d_x);
    if (m->d_t) cudaFree(m->d_t);
    if (m->d_conf) cudaFree(m->d_conf);
    m->d_x = m->d_t = nullptr;
    m->d_conf = nullptr;
    m->cap = 0;
    CK(cudaMalloc(&m->d_x, sizeof(float) * GD_MLP_IN * rows));
    CK(cudaMalloc(&m->d_t, sizeof(float) * rows));
    CK(cudaMalloc(&m->d_conf, sizeof(int) * rows));
    m->cap = rows;
  }
  if (gd::mlp_reserve(m->net, rows)) return fail(GD_ERR_NOMEM, "network buffers");
  std::vector<int> cf(rows, -1);
  if (conf) {
    for (int i = 0; i < rows; ++i) {
      if (conf[i] >= m->net.L.n_emb) return fail(GD_ERR_INVALID, "conf %d out of range", conf[i]);
      cf[i] = m->net.L.n_emb ? conf[i] : -1;
    }
  }
  CK(cudaMemcpyAsync(m->d_x, x, sizeof(float) * GD_MLP_IN * rows, cudaMemcpyHostToDevice,
                     m->stream));
  CK(cudaMemcpyAsync(m->d_conf, cf.data(), sizeof(int) * rows, cudaMemcpyHostToDevice,
                     m->stream));
  if (gd::mlp_set_rows(m->net, m->d_x, m->d_conf, rows, m->stream))
    return fail(GD_ERR_CUDA, "row upload failed");
  if (gd::mlp_embed(m->net, rows, m->stream)) return fail(GD_ERR_CUDA, "embedding failed");
  CK(cudaStreamSynchronize(m->stream)); /* cf leaves scope */
  return GD_OK;
}

}  // namespace

extern "C" {

void gd_sur_default_params(gd_sur_params *p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->hidden = 256;
  p->embedding = 1;
  p->lr = 1e-3f;
  p->batch = 8192;
  p->sample_cap = 16LL << 20;
  p->fallback_accept = 0.1f;
  p->fallback_window = 20000;
  p->seed = 7;
}

int gd_sur_create(gd_ctx *c, const gd_sur_params *p) {
  if (!c || !p) return fail(GD_ERR_INVALID, "null argument");
  if (p->hidden < 16 || p->hidden > 1024 || p->hidden % 16)
    return fail(GD_ERR_INVALID, "hidden must be a multiple of 16 in 16..1024");
  if (p->batch < 16 || p->sample_cap < 0 || p->lr <= 0.0f)
    return fail(GD_ERR_INVALID, "bad batch / sample_cap / lr");
  if (p->hidden != 128 && p->hidden != 256)
    return fail(GD_ERR_INVALID, "delayed-acceptance steps run the network fused: hidden must be "
                                "128 or 256");
  CK(cudaSetDevice(c->device));
  if (gd::da_prepare(p->hidden)) return fail(GD_ERR_CUDA, "front kernel attributes");
  CK(cudaStreamSynchronize(c->stream));
  da_free(c);
  DaState *d = new DaState();
  c->da = d;
  d->prm = *p;
  int n_emb = 0;
  std::vector<int> emb_base(c->n_complex), rep_cx(c->n_rep);
  for (int ci = 0; ci < c->n_complex; ++ci) {
    const ComplexInfo &x = c->info[ci];
    emb_base[ci] = n_emb;
    n_emb += x.n_prt * x.n_lig;
    for (int r = 0; r < x.n_rep; ++r) rep_cx[x.rep_offset + r] = ci;
  }
  int rc = 0;
#define DA_TRY(x)        \
  if ((rc = (x))) {      \
    da_free(c);          \
    return rc;           \
  }
  if (gd::mlp_create(d->net, p->hidden, p->embedding ? n_emb : 0, p->seed, c->stream)) {
    da_free(c);
    return fail(GD_ERR_NOMEM, "network allocation failed");
  }
  const int rows = p->batch; /* DA steps keep their rows in shared memory */
  if (gd::mlp_reserve(d->net, rows)) {
    da_free(c);
    return fail(GD_ERR_NOMEM, "network work buffers (%d rows)", rows);
  }
  if (!p->embedding) std::fill(emb_base.begin(), emb_base.end(), -(1 << 30));
  /* pocket features: sizes and the pocket centre, scaled to O(1) */
  std::vector<GdDevComplex> hcx(c->n_complex);
  CK(cudaMemcpy(hcx.data(), c->d_cx, sizeof(GdDevComplex) * c->n_complex,
                cudaMemcpyDeviceToHost));
  std::vector<float> pf((size_t)c->n_complex * GD_MLP_POCKET, 0.0f);
  for (int ci = 0; ci < c->n_complex; ++ci) {
    const ComplexInfo &x = c->info[ci];
    float *f = pf.data() + (size_t)ci * GD_MLP_POCKET;
    f[0] = x.pnp / 1000.0f;
    f[1] = x.pnk / 40.0f;
    f[2] = x.lna / 40.0f;
    f[3] = x.n_lig / 10.0f;
    f[4] = x.n_prt / 10.0f;
    f[5] = x.pos / 8.0f;
    f[6] = x.n_tmp / 20.0f;
    f[7] = hcx[ci].pocket[0] / 10.0f;
    f[8] = hcx[ci].pocket[1] / 10.0f;
    f[9] = hcx[ci].pocket[2] / 10.0f;
    f[10] = 1.0f;
  }
  const size_t R = c->n_rep;
  DA_TRY(da_alloc(d, &d->d_rep_cx, R));
  DA_TRY(da_alloc(d, &d->d_emb_base, c->n_complex));
  DA_TRY(da_alloc(d, &d->d_active, c->n_complex));
  DA_TRY(da_alloc(d, &d->d_pocket, pf.size()));
  DA_TRY(da_alloc(d, &d->d_u2, R));
  DA_TRY(da_alloc(d, &d->d_s_cur, R));
  DA_TRY(da_alloc(d, &d->d_s_new, R));
  DA_TRY(da_alloc(d, &d->d_pose_mm, R * 6));
  DA_TRY(da_alloc(d, &d->d_pose_rep, R));
  DA_TRY(da_alloc(d, &d->d_pose_lc, R));
  DA_TRY(da_alloc(d, &d->d_prop, R));
  DA_TRY(da_alloc(d, &d->d_pass, R));
  DA_TRY(da_alloc(d, &d->d_plain, R));
  DA_TRY(da_alloc(d, &d->d_acc, R));
  DA_TRY(da_alloc(d, &d->d_plain_acc, R));
  DA_TRY(da_alloc(d, &d->d_nerr, R));
  DA_TRY(da_alloc(d, &d->d_err2, R));
  DA_TRY(da_alloc(d, &d->d_epi, 1));
  DA_TRY(da_alloc(d, &d->d_stats, (size_t)c->n_complex * GD_DA_NSTAT));
  DA_TRY(da_alloc(d, &d->d_err, (size_t)c->n_complex * GD_DA_NERR));
  DA_TRY(da_alloc(d, &d->d_t, (size_t)rows));
  DA_TRY(da_alloc(d, &d->d_mom, (size_t)GD_DA_MOM_BLOCKS * 3));
  d->smp_cap = p->sample_cap;
  if (d->smp_cap > 0) {
    DA_TRY(da_alloc(d, &d->smp_X, (size_t)d->smp_cap * GD_MLP_IN));
    DA_TRY(da_alloc(d, &d->smp_conf, (size_t)d->smp_cap));
    DA_TRY(da_alloc(d, &d->smp_t, (size_t)d->smp_cap));
  }
#undef DA_TRY
  d->active.assign(c->n_complex, 0); /* off until trained */
  CK(cudaMemcpy(d->d_rep_cx, rep_cx.data(), sizeof(int) * R, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d->d_emb_base, emb_base.data(), sizeof(int) * c->n_complex,
                cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d->d_pocket, pf.data(), sizeof(float) * pf.size(), cudaMemcpyHostToDevice));
  CK(cudaMemset(d->d_s_cur, 0, sizeof(float) * R));
  CK(cudaMemset(d->d_s_new, 0, sizeof(float) * R));
  rc = da_upload_active(c);
  if (!rc) rc = da_reset_counters(c);
  if (!rc) rc = da_build_groups(c, c->split);
  if (!rc) rc = da_upload_epi(c);
  if (rc) {
    da_free(c);
    return rc;
  }
  CK(cudaStreamSynchronize(c->stream));
  return GD_OK;
}

int gd_sur_collect(gd_ctx *c, int s1, int n_steps, int exchange) {
  if (!c || !c->da) return fail(GD_ERR_STATE, "gd_sur_create has not run");
  DaState *d = c->da;
  if (d->smp_cap <= 0) return fail(GD_ERR_CAPACITY, "sample_cap is 0");
  const long long g0 = (long long)s1 * c->n_rep;
  int rc = da_run_steps(c, s1, n_steps, exchange, true);
  if (rc) return rc;
  if (d->smp_hi != g0) d->smp_lo = g0; /* not contiguous with the earlier samples */
  d->smp_hi = g0 + (long long)n_steps * c->n_rep;
  return rs_enqueue(c, n_steps);
}

int gd_sur_train(gd_ctx *c, int iterations, float *losses) {
  if (!c || !c->da) return fail(GD_ERR_STATE, "gd_sur_create has not run");
  if (iterations < 0) return fail(GD_ERR_INVALID, "iterations < 0");
  DaState *d = c->da;
  const long long vlo = std::max(d->smp_lo, d->smp_hi - d->smp_cap);
  const long long n_valid = d->smp_hi - vlo;
  if (n_valid <= 0) return fail(GD_ERR_STATE, "no samples (gd_sur_collect)");
  CK(cudaSetDevice(c->device));
  const long long start = vlo % d->smp_cap;
  int rc;
  if (d->norm_hi != d->smp_hi) {
    if ((rc = da_normalise(c, start, n_valid))) return rc;
    d->norm_hi = d->smp_hi;
  }
  if (iterations > d->loss_cap) {
    if (d->d_loss_hist) cudaFree(d->d_loss_hist);
    d->d_loss_hist = nullptr;
    d->loss_cap = 0;
    CK(cudaMalloc(&d->d_loss_hist, sizeof(float) * iterations));
    d->loss_cap = iterations;
  }
  gd::GdDaDev a = da_args(c);
  const int B = d->prm.batch;
  for (int it = 0; it < iterations; ++it) {
    gd::da_gather(a, start, n_valid, B, (int)(d->train_iter++), d->d_t, c->stream);
    if (gd::mlp_embed(d->net, B, c->stream) || gd::mlp_loss_backward(d->net, B, d->d_t, c->stream))
      return fail(GD_ERR_CUDA, "training step failed: %s", cudaGetErrorString(cudaGetLastError()));
    CK(cudaMemcpyAsync(d->d_loss_hist + it, d->net.loss, sizeof(float), cudaMemcpyDeviceToDevice,
                       c->stream));
    if (gd::mlp_adam(d->net, d->prm.lr, c->stream))
      return fail(GD_ERR_CUDA, "Adam step failed");
  }
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  if (gd::mlp_status(d->net)) return fail(GD_ERR_CUDA, "tensor-core GEMM wait timed out");
  if (losses && iterations)
    CK(cudaMemcpy(losses, d->d_loss_hist, sizeof(float) * iterations, cudaMemcpyDeviceToHost));
  /* the new network (and normalisation) replaces the old one in every later graph */
  da_drop_graphs(c);
  d->active.assign(c->n_complex, 1);
  if ((rc = da_upload_active(c))) return rc;
  return da_reset_counters(c);
}

int gd_da_run(gd_ctx *c, int s1, int n_steps, int exchange) {
  int rc = da_run_steps(c, s1, n_steps, exchange, false);
  if (rc) return rc;
  if ((rc = rs_enqueue(c, n_steps))) return rc;
  DaState *d = c->da;
  const bool controller = d->prm.fallback_accept > 0.0f;
  if (!controller && d->prm.split > 0) return GD_OK;
  std::vector<unsigned long long> st;
  std::vector<double> er;
  if ((rc = da_read_stats(c, st, er))) return rc;
  /* pass rate of this run (all complexes with the stage on): picks the next run's split */
  unsigned long long prop = 0, pass = 0;
  for (int ci = 0; ci < c->n_complex; ++ci) {
    prop += st[(size_t)ci * GD_DA_NSTAT + GD_DA_PROPOSED];
    pass += st[(size_t)ci * GD_DA_NSTAT + GD_DA_PASSED];
  }
  if (prop > d->prev_prop) d->last_pass = (double)(pass - d->prev_pass) / (double)(prop - d->prev_prop);
  d->prev_prop = prop;
  d->prev_pass = pass;
  if (!controller) return GD_OK;
  bool changed = false;
  for (int ci = 0; ci < c->n_complex; ++ci) {
    if (!d->active[ci]) continue;
    const unsigned long long *s = st.data() + (size_t)ci * GD_DA_NSTAT;
    unsigned long long *w = d->window0.data() + (size_t)ci * GD_DA_NSTAT;
    const unsigned long long passed = s[GD_DA_PASSED] - w[GD_DA_PASSED];
    if ((long long)passed < std::max(1LL, d->prm.fallback_window)) continue;
    const double acc = (double)(s[GD_DA_ACCEPTED] - w[GD_DA_ACCEPTED]) / (double)passed;
    if (acc < d->prm.fallback_accept) {
      d->active[ci] = 0;
      changed = true;
    }
    for (int k = 0; k < GD_DA_NSTAT; ++k) w[k] = s[k];
  }
  if (changed) return da_upload_active(c);
  return GD_OK;
}

int gd_sur_get_stats(gd_ctx *c, gd_sur_stats *out) {
  if (!c || !c->da || !out) return fail(GD_ERR_STATE, "gd_sur_create has not run");
  std::vector<unsigned long long> st;
  std::vector<double> er;
  int rc = da_read_stats(c, st, er);
  if (rc) return rc;
  for (int ci = 0; ci < c->n_complex; ++ci) {
    const unsigned long long *s = st.data() + (size_t)ci * GD_DA_NSTAT;
    gd_sur_stats &o = out[ci];
    memset(&o, 0, sizeof(o));
    o.proposed = (long long)s[GD_DA_PROPOSED];
    o.passed = (long long)s[GD_DA_PASSED];
    o.accepted = (long long)s[GD_DA_ACCEPTED];
    o.plain = (long long)s[GD_DA_PLAIN];
    o.plain_accepted = (long long)s[GD_DA_PLAIN_ACC];
    const double n = er[(size_t)ci * GD_DA_NERR + 1];
    o.n_err = (long long)n;
    o.rmse = n > 0 ? std::sqrt(er[(size_t)ci * GD_DA_NERR] / n) : 0.0;
    o.active = c->da->active[ci];
  }
  return GD_OK;
}

int gd_sur_set_active(gd_ctx *c, int ci, int on) {
  if (!c || !c->da) return fail(GD_ERR_STATE, "gd_sur_create has not run");
  if (ci < 0 || ci >= c->n_complex) return fail(GD_ERR_INVALID, "bad complex index");
  c->da->active[ci] = on ? 1 : 0;
  for (int k = 0; k < GD_DA_NSTAT; ++k) c->da->window0[(size_t)ci * GD_DA_NSTAT + k] = 0;
  /* restart this complex's controller window from the current counters */
  std::vector<unsigned long long> st;
  std::vector<double> er;
  int rc = da_read_stats(c, st, er);
  if (rc) return rc;
  for (int k = 0; k < GD_DA_NSTAT; ++k)
    c->da->window0[(size_t)ci * GD_DA_NSTAT + k] = st[(size_t)ci * GD_DA_NSTAT + k];
  return da_upload_active(c);
}

int gd_sur_predict(gd_ctx *c, int ci, int prt_conf, int lig_conf, const float *mm, int n,
                   float *energy) {
  if (!c || !c->da) return fail(GD_ERR_STATE, "gd_sur_create has not run");
  if (!mm || !energy) return fail(GD_ERR_INVALID, "null argument");
  if (ci < 0 || ci >= c->n_complex) return fail(GD_ERR_INVALID, "bad complex index");
  const ComplexInfo &x = c->info[ci];
  if (prt_conf < 0 || prt_conf >= x.n_prt || lig_conf < 0 || lig_conf >= x.n_lig)
    return fail(GD_ERR_INVALID, "conformer index out of range");
  if (n < 1) return GD_OK;
  DaState *d = c->da;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  if (gd::mlp_reserve(d->net, n)) return fail(GD_ERR_NOMEM, "network work buffers");
  if (n > d->pred_cap) {
    if (d->d_pred_mm) cudaFree(d->d_pred_mm);
    d->d_pred_mm = nullptr;
    d->pred_cap = 0;
    CK(cudaMalloc(&d->d_pred_mm, sizeof(float) * 6 * n));
    d->pred_cap = n;
  }
  /* the work buffers may have moved: graphs that point at them are stale */
  da_drop_graphs(c);
  CK(cudaMemcpy(d->d_pred_mm, mm, sizeof(float) * 6 * n, cudaMemcpyHostToDevice));
  gd::GdDaDev a = da_args(c);
  gd::da_pose_features(a, ci, prt_conf, lig_conf, d->d_pred_mm, n, c->stream);
  if (gd::mlp_forward(d->net, n, c->stream))
    return fail(GD_ERR_CUDA, "forward failed");
  CK(cudaStreamSynchronize(c->stream));
  std::vector<float> y(n);
  CK(cudaMemcpy(y.data(), d->net.y, sizeof(float) * n, cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; ++i) energy[i] = fmaf(y[i], d->net.sigma, d->net.mu);
  return GD_OK;
}

int gd_sur_info(gd_ctx *c, float *mu, float *sigma, long long *n_samples) {
  if (!c || !c->da) return fail(GD_ERR_STATE, "gd_sur_create has not run");
  DaState *d = c->da;
  if (mu) *mu = d->net.mu;
  if (sigma) *sigma = d->net.sigma;
  if (n_samples) *n_samples = d->smp_hi - std::max(d->smp_lo, d->smp_hi - d->smp_cap);
  return GD_OK;
}

int gd_sur_split(gd_ctx *c, int *split) {
  if (!c || !c->da || !split) return fail(GD_ERR_STATE, "gd_sur_create has not run");
  *split = c->da->split;
  return GD_OK;
}

int gd_da_trace_enable(gd_ctx *c, int step0, int max_steps) {
  if (!c || !c->da) return fail(GD_ERR_STATE, "gd_sur_create has not run");
  if (max_steps < 0 || step0 < 0) return fail(GD_ERR_INVALID, "bad argument");
  DaState *d = c->da;
  CK(cudaStreamSynchronize(c->stream));
  da_free_trace(d);
  da_drop_graphs(c);
  d->tr_step0 = step0;
  if (max_steps == 0) return da_upload_epi(c);
  const size_t n = (size_t)c->n_rep * max_steps;
  CK(cudaMalloc(&d->tr_s, sizeof(float) * n));
  CK(cudaMalloc(&d->tr_e, sizeof(float) * n));
  CK(cudaMalloc(&d->tr_flag, sizeof(int) * n));
  CK(cudaMemset(d->tr_flag, 0xff, sizeof(int) * n));
  d->tr_cap = max_steps;
  return da_upload_epi(c);
}

int gd_da_trace_get(gd_ctx *c, float *s_new, float *e_new, int *outcome) {
  if (!c || !c->da) return fail(GD_ERR_STATE, "gd_sur_create has not run");
  DaState *d = c->da;
  if (!d->tr_cap) return fail(GD_ERR_STATE, "trace not enabled");
  CK(cudaStreamSynchronize(c->stream));
  const size_t n = (size_t)c->n_rep * d->tr_cap;
  if (s_new) CK(cudaMemcpy(s_new, d->tr_s, sizeof(float) * n, cudaMemcpyDeviceToHost));
  if (e_new) CK(cudaMemcpy(e_new, d->tr_e, sizeof(float) * n, cudaMemcpyDeviceToHost));
  if (outcome) CK(cudaMemcpy(outcome, d->tr_flag, sizeof(int) * n, cudaMemcpyDeviceToHost));
  return GD_OK;
}

/* ---- the network alone ---- */

int gd_mlp_create(int device, int hidden, int n_emb, uint64_t seed, gd_mlp **out) {
  if (!out) return fail(GD_ERR_INVALID, "null argument");
  *out = nullptr;
  if (hidden < 16 || hidden > 1024 || hidden % 16 || n_emb < 0)
    return fail(GD_ERR_INVALID, "hidden must be a multiple of 16 in 16..1024, n_emb >= 0");
  CK(cudaSetDevice(device));
  gd_mlp *m = new gd_mlp();
  m->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete m;
    return fail(GD_ERR_CUDA, "stream: %s", cudaGetErrorString(e));
  }
  if (gd::mlp_create(m->net, hidden, n_emb, seed, m->stream)) {
    gd::mlp_destroy(m->net);
    cudaStreamDestroy(m->stream);
    delete m;
    return fail(GD_ERR_NOMEM, "network allocation failed");
  }
  *out = m;
  CK(cudaStreamSynchronize(m->stream));
  return GD_OK;
}

int gd_mlp_destroy(gd_mlp *m) {
  if (!m) return GD_OK;
  cudaSetDevice(m->device);
  cudaStreamSynchronize(m->stream);
  gd::mlp_destroy(m->net);
  if (m->d_x) cudaFree(m->d_x);
  if (m->d_t) cudaFree(m->d_t);
  if (m->d_conf) cudaFree(m->d_conf);
  cudaStreamDestroy(m->stream);
  delete m;
  return GD_OK;
}

int gd_mlp_num_params(gd_mlp *m, long long *n) {
  if (!m || !n) return fail(GD_ERR_INVALID, "null argument");
  *n = (long long)m->net.L.total;
  return GD_OK;
}

int gd_mlp_get_params(gd_mlp *m, float *theta, long long n) {
  if (!m || !theta) return fail(GD_ERR_INVALID, "null argument");
  if (n != (long long)m->net.L.total) return fail(GD_ERR_INVALID, "parameter count mismatch");
  CK(cudaSetDevice(m->device));
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(theta, m->net.theta, sizeof(float) * n, cudaMemcpyDeviceToHost));
  return GD_OK;
}

int gd_mlp_set_params(gd_mlp *m, const float *theta, long long n) {
  if (!m || !theta) return fail(GD_ERR_INVALID, "null argument");
  if (n != (long long)m->net.L.total) return fail(GD_ERR_INVALID, "parameter count mismatch");
  CK(cudaSetDevice(m->device));
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(m->net.theta, theta, sizeof(float) * n, cudaMemcpyHostToDevice));
  if (gd::mlp_refresh_bf16(m->net, m->stream)) return fail(GD_ERR_CUDA, "bf16 refresh failed");
  CK(cudaStreamSynchronize(m->stream));
  return GD_OK;
}

int gd_mlp_forward(gd_mlp *m, const float *x, const int *conf, int rows, float *y) {
  if (!m || !x || !y || rows < 0) return fail(GD_ERR_INVALID, "bad argument");
  if (rows == 0) return GD_OK;
  CK(cudaSetDevice(m->device));
  int rc = mlp_stage_rows(m, x, conf, rows);
  if (rc) return rc;
  if (gd::mlp_forward(m->net, rows, m->stream)) return fail(GD_ERR_CUDA, "forward failed");
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(y, m->net.y, sizeof(float) * rows, cudaMemcpyDeviceToHost));
  return GD_OK;
}

int gd_mlp_backward(gd_mlp *m, const float *x, const int *conf, const float *t, int rows,
                    float *loss, float *grad) {
  if (!m || !x || !t || rows < 1) return fail(GD_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(m->device));
  int rc = mlp_stage_rows(m, x, conf, rows);
  if (rc) return rc;
  CK(cudaMemcpyAsync(m->d_t, t, sizeof(float) * rows, cudaMemcpyHostToDevice, m->stream));
  if (gd::mlp_loss_backward(m->net, rows, m->d_t, m->stream))
    return fail(GD_ERR_CUDA, "backward failed");
  CK(cudaStreamSynchronize(m->stream));
  if (gd::mlp_status(m->net)) return fail(GD_ERR_CUDA, "tensor-core GEMM wait timed out");
  if (loss) CK(cudaMemcpy(loss, m->net.loss, sizeof(float), cudaMemcpyDeviceToHost));
  if (grad)
    CK(cudaMemcpy(grad, m->net.grad, sizeof(float) * m->net.L.total, cudaMemcpyDeviceToHost));
  return GD_OK;
}

int gd_mlp_adam(gd_mlp *m, float lr) {
  if (!m || !(lr > 0.0f)) return fail(GD_ERR_INVALID, "bad argument");
  CK(cudaSetDevice(m->device));
  if (gd::mlp_adam(m->net, lr, m->stream)) return fail(GD_ERR_CUDA, "Adam step failed");
  CK(cudaStreamSynchronize(m->stream));
  return GD_OK;
}

int gd_kmeans(int device, const float *objects, int n, int dim, const int *seg_off, int n_seg,
              const int *k, uint64_t seed, float threshold, int max_iter, int *membership,
              int *medoid, int *size, int *passes) {
  if (!objects || !seg_off || !k || n < 0 || n_seg < 1 || max_iter < 0)
    return fail(GD_ERR_INVALID, "gd_kmeans: bad arguments");
  if (dim != GD_MAXWEI - 1) return fail(GD_ERR_INVALID, "gd_kmeans: dim must be %d", GD_MAXWEI - 1);
  if (seg_off[0] != 0 || seg_off[n_seg] != n)
    return fail(GD_ERR_INVALID, "gd_kmeans: segment offsets must run from 0 to n");
  for (int s = 0; s < n_seg; ++s)
    if (seg_off[s + 1] < seg_off[s] || k[s] < 1)
      return fail(GD_ERR_INVALID, "gd_kmeans: segment %d: offsets decrease or k < 1", s);
  CK(cudaSetDevice(device));
  gd::KmeansJob job;
  job.objects = objects;
  job.dim = dim;
  job.seg_off.assign(seg_off, seg_off + n_seg + 1);
  job.k.assign(k, k + n_seg);
  job.seed = seed;
  job.threshold = threshold;
  job.max_iter = max_iter;
  gd::KmeansResult res;
  std::string err;
  if (gd::kmeans_device(job, res, err)) return fail(GD_ERR_CUDA, "gd_kmeans: %s", err.c_str());
  if (membership) std::copy(res.membership.begin(), res.membership.end(), membership);
  if (medoid) std::copy(res.medoid.begin(), res.medoid.end(), medoid);
  if (size) std::copy(res.size.begin(), res.size.end(), size);
  if (passes) std::copy(res.passes.begin(), res.passes.end(), passes);
  return GD_OK;
}

int gd_kmeans_permutation(uint64_t seed, int segment, int n, int *perm) {
  if (!perm || n < 0 || segment < 0) return fail(GD_ERR_INVALID, "gd_kmeans_permutation: bad arguments");
  gd::kmeans_permutation(seed, segment, n, perm);
  return GD_OK;
}

}  // extern "C"
