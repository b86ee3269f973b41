/*
 * gd_capi_stream.cu -- records downloaded while the run proceeds (gd_records_stream,
 * gd_records_stream_flush). The reference copies the whole LigRecord array after each dump
 * window (src/kernel_cuda_lancher_siglegpu.cu:36-46); here a copy plan and a gather kernel
 * queued after each record-writing call pack the new rows, and a worker thread downloads them
 * into the caller's array on its own stream while the next work runs.
 */
#include "gd_capi_internal.cuh"

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

/* One dump window downloaded in the background (gd_get_records_async): the window's rows are
 * snapshotted on the device in the context's stream order (one device-to-device copy, after
 * which the stream may reset and overwrite the records), and a host thread waits for the
 * snapshot and copies it out with the staged multi-threaded copy of d2h_rows. */
struct RecAsync {
  gd_record_step *d_snap = nullptr;                /* [n_rep * cap] */
  int *d_next = nullptr;                           /* [n_rep] */
  size_t snap_rows = 0;
  cudaEvent_t ev = nullptr;
  std::thread th;
  bool busy = false;
  int rows = 0;
  cudaError_t err = cudaSuccess;
};

namespace gdc {

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

/* waits for the background download, if any (the thread's result in *rows) */
int ra_wait(gd_ctx *c, int *rows) {
  RecAsync *a = c->ra;
  if (rows) *rows = 0;
  if (!a || !a->busy) return GD_OK;
  a->th.join();
  a->busy = false;
  if (rows) *rows = a->rows;
  if (a->err != cudaSuccess)
    return fail(GD_ERR_CUDA, "background record download: %s", cudaGetErrorString(a->err));
  return GD_OK;
}

void ra_free(gd_ctx *c) {
  RecAsync *a = c->ra;
  if (!a) return;
  ra_wait(c, nullptr);
  /* the buffers came from the context pool on the context's stream */
  if (a->d_snap) cudaFreeAsync(a->d_snap, c->stream);
  if (a->d_next) cudaFreeAsync(a->d_next, c->stream);
  if (a->d_snap || a->d_next) cudaStreamSynchronize(c->stream);
  if (a->ev) cudaEventDestroy(a->ev);
  delete a;
  c->ra = nullptr;
}

}  // namespace gdc

using namespace gdc;

extern "C" {

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

int gd_get_records_async(gd_ctx *c, gd_record_step *steps, int *next_ptr, int cap) {
  if (!c || !steps || !next_ptr) return fail(GD_ERR_INVALID, "null argument");
  if (!c->mc.record || !c->d_rec) return fail(GD_ERR_STATE, "records are disabled");
  if (cap < 1 || cap > c->rec_cap)
    return fail(GD_ERR_INVALID, "cap %d outside 1..record capacity %d", cap, c->rec_cap);
  CK(cudaSetDevice(c->device));
  if (!c->ra) c->ra = new RecAsync();
  RecAsync *a = c->ra;
  int rc = ra_wait(c, nullptr);
  if (rc) return rc;
  const int n = c->n_rep;
  const size_t rows = (size_t)n * cap, rs = sizeof(gd_record_step);
  /* the snapshot buffers come from the context pool, stream-ordered on the context's stream
   * (the host thread reads them only after the event recorded behind the snapshot) */
  cudaMemPool_t pool = ctx_pool(c->device);
  if (!pool) return fail(GD_ERR_NOMEM, "gd_get_records_async: no memory pool");
  if (a->snap_rows < rows) {
    if (a->d_snap) cudaFreeAsync(a->d_snap, c->stream);
    a->d_snap = nullptr;
    a->snap_rows = 0;
    CK(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&a->d_snap), rows * rs, pool,
                               c->stream));
    a->snap_rows = rows;
  }
  if (!a->d_next)
    CK(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&a->d_next), sizeof(int) * n, pool,
                               c->stream));
  if (!a->ev) CK(cudaEventCreateWithFlags(&a->ev, cudaEventDisableTiming));
  CK(cudaMemcpy2DAsync(a->d_snap, rs * cap, c->d_rec, rs * c->rec_cap, rs * cap, n,
                       cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(a->d_next, c->d_rec_next, sizeof(int) * n, cudaMemcpyDeviceToDevice,
                     c->stream));
  CK(cudaEventRecord(a->ev, c->stream));
  a->busy = true;
  a->err = cudaSuccess;
  a->rows = 0;
  const int dev = c->device;
  a->th = std::thread([a, dev, n, cap, steps, next_ptr, rs] {
    cudaError_t e = cudaSetDevice(dev);
    if (e == cudaSuccess) e = cudaEventSynchronize(a->ev);
    if (e == cudaSuccess)
      e = cudaMemcpy(next_ptr, a->d_next, sizeof(int) * n, cudaMemcpyDeviceToHost);
    int m = 1;
    if (e == cudaSuccess) {
      for (int r = 0; r < n; ++r) m = std::max(m, std::min(next_ptr[r], cap));
      e = d2h_rows(steps, rs * m, a->d_snap, rs * cap, rs * m, n);
    }
    a->rows = m;
    a->err = e;
  });
  return GD_OK;
}

int gd_records_wait(gd_ctx *c, int *rows) {
  if (!c) return fail(GD_ERR_INVALID, "null context");
  return ra_wait(c, rows);
}

}  // extern "C"
