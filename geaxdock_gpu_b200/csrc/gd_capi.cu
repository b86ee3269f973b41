/*
 * gd_capi.cu -- host side of the C ABI declared in include/geauxdock_b200.h: the context.
 *
 * Replaces the reference's Run (src/run.cu:33-288) and its single-GPU launcher loop
 * (src/kernel_cuda_lancher_siglegpu.cu:1-71): instead of ~40 cudaMemcpyToSymbol calls and a
 * synchronous launch per 10 steps, a context owns its device buffers and one stream, turns
 * each complex into the kernel-ready layout once (points sorted by type, segments, folded
 * pair parameters, sparse contact reference), and launches the persistent kernel of
 * gd_kernels.cu, optionally as a captured CUDA graph. The other host units are listed in
 * gd_capi_internal.cuh.
 */
#include "gd_capi_internal.cuh"

namespace gdc {


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





/* largest float d2 with sqrtf(d2) <= pmf0, -1 when none */
float contact_threshold(float pmf0) {
  if (!(pmf0 >= 0.0f)) return -1.0f;
  float t = (float)((double)pmf0 * (double)pmf0);
  while (t > 0.0f && sqrtf(t) > pmf0) t = nextafterf(t, -INFINITY);
  while (sqrtf(nextafterf(t, INFINITY)) <= pmf0) t = nextafterf(t, INFINITY);
  return t;
}

double pmf_far_radius(float pmf0) {
  /* Beyond the larger root r* of (r/2 - 6)(r - pmf0) = 26 / log2(e), which lies past
   * max(12, pmf0), the product only grows, so the pmf exponent in base 2 stays below -26
   * (below -25.5 as the kernel computes it in FP32, whose rounding there is under 0.01) */
  const double k = 26.0 / 1.4426950408889634;
  const double a = 6.0 + 0.5 * (double)pmf0;
  const double r = a + std::sqrt(std::max(0.0, a * a - 2.0 * (6.0 * (double)pmf0 - k)));
  return std::max(r, std::max(12.0, (double)pmf0));
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

/* Device -> host copy of n rows (width bytes each; device pitch dpitch, host pitch hpitch). A
 * large download into freshly allocated pageable memory is bound by the first touch of every
 * host page (one thread faults pages in at about a quarter of the copy rate of resident pages),
 * so above 32 MB the destination rows are first written by up to 8 host threads in parallel,
 * then copied in one call. */
namespace {
/* page-locked staging buffers of the large downloads, one per copy thread, made with the
 * process's first recording context and kept */
constexpr int kStageThreads = 8;
constexpr size_t kStageBytes = (size_t)8 << 20;
std::mutex g_stage_mu;
void *g_stage[kStageThreads] = {};

int stage_threads() {
  return (int)std::min<unsigned>(kStageThreads, std::max(1u, std::thread::hardware_concurrency()));
}

/* with g_stage_mu held: false if a buffer could not be made */
bool stage_ready_locked() {
  for (int t = 0; t < stage_threads(); ++t)
    if (!g_stage[t] && cudaHostAlloc(&g_stage[t], kStageBytes, cudaHostAllocPortable) !=
                           cudaSuccess) {
      g_stage[t] = nullptr;
      cudaGetLastError();
      return false;
    }
  return true;
}
}  // namespace

void stage_prepare() {
  std::lock_guard<std::mutex> lock(g_stage_mu);
  stage_ready_locked();
}

/* n rows of `width` bytes from device memory (row pitch dpitch) into host memory (row pitch
 * hpitch). Into pageable memory, a large copy runs on up to kStageThreads host threads, each
 * taking the next chunk of rows: its own stream copies the chunk into its page-locked staging
 * buffer, then the thread copies it into the destination (touching those pages for the first
 * time), so the DMA engine fills one buffer while other threads empty theirs. The device
 * rows must be complete (the caller synchronised the stream that wrote them). */
cudaError_t d2h_rows(void *dst, size_t hpitch, const void *src, size_t dpitch, size_t width,
                     int n) {
  if (n < 1 || width == 0) return cudaSuccess;
  cudaPointerAttributes at;
  const bool pinned =
      cudaPointerGetAttributes(&at, dst) == cudaSuccess && at.type == cudaMemoryTypeHost;
  cudaGetLastError();
  if (pinned || width * (size_t)n < ((size_t)32 << 20) || width > kStageBytes)
    return cudaMemcpy2D(dst, hpitch, src, dpitch, width, n, cudaMemcpyDeviceToHost);
  std::lock_guard<std::mutex> lock(g_stage_mu);
  const int T = stage_threads();
  if (!stage_ready_locked())
    return cudaMemcpy2D(dst, hpitch, src, dpitch, width, n, cudaMemcpyDeviceToHost);
  int dev = 0;
  cudaError_t e0 = cudaGetDevice(&dev);
  if (e0 != cudaSuccess) return e0;
  const int rows = (int)(kStageBytes / width);
  const int chunks = (n + rows - 1) / rows;
  std::atomic<int> next{0};
  std::atomic<int> err{(int)cudaSuccess};
  auto work = [&](int t) {
    cudaError_t e = cudaSetDevice(dev);
    cudaStream_t st = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    char *stage = static_cast<char *>(g_stage[t]);
    for (int k = next++; e == cudaSuccess && k < chunks && err.load() == (int)cudaSuccess;
         k = next++) {
      const int a = k * rows, b = std::min(n, a + rows);
      e = cudaMemcpy2DAsync(stage, width, static_cast<const char *>(src) + (size_t)a * dpitch,
                            dpitch, width, b - a, cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) break;
      char *d = static_cast<char *>(dst) + (size_t)a * hpitch;
      if (hpitch == width) {
        memcpy(d, stage, (size_t)(b - a) * width);
      } else {
        for (int i = a; i < b; ++i, d += hpitch) memcpy(d, stage + (size_t)(i - a) * width, width);
      }
    }
    if (st) cudaStreamDestroy(st);
    if (e != cudaSuccess) err = (int)e;
  };
  const int nt = std::min(T, chunks);
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
  work(0);
  for (auto &x : th) x.join();
  return (cudaError_t)err.load();
}

namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pool[GD_MAX_DEVICES] = {};
}  // namespace

cudaMemPool_t ctx_pool(int device) {
  if (device < 0 || device >= GD_MAX_DEVICES) return nullptr;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pool[device]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pool[device] = pool;
  }
  return g_pool[device];
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
    /* the short-range cell grid is laid over the points' bounding box */
    if (!std::isfinite(d.prt_x[i]) || !std::isfinite(d.prt_y[i]) || !std::isfinite(d.prt_z[i]))
      return fail(GD_ERR_INVALID, "complex %d: protein point %d has a non-finite coordinate", idx,
                  i);
  }
  /* the pair loop orders each segment's points by distance from the pocket centre */
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(d.pocket_center[a]))
      return fail(GD_ERR_INVALID, "complex %d: the pocket centre has a non-finite coordinate", idx);
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
  return 16 + GD_THR_BYTES + (size_t)2 * c->chunk * 16 + (size_t)c->threads * 16 +
         (size_t)10 * c->threads * 8 +
         (size_t)kmax * slot;
}

int ensure_counters(gd_ctx *c, int n) {
  if (n <= c->counters_cap) return GD_OK;
  if (c->d_counters) {
    /* the captured graphs point at the old counters: finish them and drop them first */
    CK(cudaStreamSynchronize(c->stream));
    for (auto &g : c->graphs) cudaGraphExecDestroy(g.second);
    c->graphs.clear();
  }
  int *p = nullptr;
  cudaMemPool_t pool = ctx_pool(c->device);
  if (pool) {
    CK(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&p), sizeof(int) * n, pool,
                               c->stream));
  } else {
    CK(cudaMalloc(&p, sizeof(int) * n));
  }
  if (c->d_counters) {
    if (c->counters_pooled)
      cudaFreeAsync(c->d_counters, c->stream);
    else
      cudaFree(c->d_counters);
  }
  c->d_counters = p;
  c->counters_cap = n;
  c->counters_pooled = pool != nullptr;
  return GD_OK;
}

int ensure_cursor(gd_ctx *c) {
  if (!c->h_cursor) CK(cudaMallocHost(&c->h_cursor, 2 * sizeof(int)));
  return GD_OK;
}


/* the kernel variant for an unroll depth, a protein split and the mode-3 epilogue */
template <bool S, bool D>
McKernel mc_variant(int unroll) {
  if (unroll >= 4) return gd::gd_mc_kernel<4, S, D, 1>;
  if (unroll >= 2) return gd::gd_mc_kernel<2, S, D, 1>;
  return gd::gd_mc_kernel<1, S, D, 1>;
}

McKernel mc_kernel(int unroll, int split, bool da, int pack) {
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
int launch_threads(const gd_ctx *c, int split, bool da) {
  return c->threads / launch_pack(c, split, da);
}

McKernel launch_kernel(const gd_ctx *c, int split, bool da, int unroll) {
  const int S = split ? split : c->split;
  return mc_kernel(unroll ? unroll : c->unroll, S, da, launch_pack(c, split, da));
}

int grid_for(gd_ctx *c, int n_tiles, size_t smem, int split, bool da, int unroll) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, launch_kernel(c, split, da, unroll),
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

int set_kernel_attrs(const gd_ctx *c, size_t smem, int split, bool da, int unroll) {
  const McKernel k = launch_kernel(c, split, da, unroll);
  CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  /* shared memory for the CTAs an SM can hold and the rest as L1, which caches the cell
   * lists of the short-range pass: the carveout is the share of the SM's maximum shared
   * memory those CTAs take (the driver rounds it up to a supported split) */
  CK(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                          cudaSharedmemCarveoutMaxShared));
  int nb = 0, dev = 0, per_sm = 0, reserved = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  CK(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
  const int threads = launch_threads(c, split, da);
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, threads, smem));
  if (nb >= 1 && per_sm > 0) {
    /* the driver rounds the carveout up to one of the SM's shared-memory sizes; aim at the
     * smallest of them that holds the CTAs (a percentage rounded up could cross into the
     * next size and take the L1 the walk needs) */
    static const int kSizesKB[] = {0, 8, 16, 32, 64, 100, 132, 164, 196, 228};
    const long long need = (long long)nb * (long long)(smem + (size_t)reserved);
    long long size = per_sm;
    for (int kb : kSizesKB)
      if ((long long)kb * 1024 >= need) {
        size = std::min<long long>((long long)kb * 1024, per_sm);
        break;
      }
    const int pct = std::max(1, std::min(100, (int)(100 * size / per_sm)));
    CK(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
    int nb2 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, k, threads, smem) != cudaSuccess ||
        nb2 < nb)
      CK(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                              cudaSharedmemCarveoutMaxShared));
  }
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


void drop_graphs(gd_ctx *c) {
  for (auto &g : c->graphs) cudaGraphExecDestroy(g.second);
  c->graphs.clear();
  da_drop_graphs(c);
}

}  // namespace gdc

using namespace gdc;

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
  ra_free(c);
  drop_graphs(c);
  da_free(c);
  for (void *p : c->pool_allocs) cudaFreeAsync(p, c->stream);
  if (c->d_counters && c->counters_pooled) cudaFreeAsync(c->d_counters, c->stream);
  if (!c->pool_allocs.empty() || c->counters_pooled) cudaStreamSynchronize(c->stream);
  for (void *p : c->allocs) cudaFree(p);
  if (c->d_counters && !c->counters_pooled) cudaFree(c->d_counters);
  if (c->d_trace_e) cudaFree(c->d_trace_e);
  if (c->d_trace_acc) cudaFree(c->d_trace_acc);
  if (c->d_mm_in) cudaFree(c->d_mm_in);
  if (c->d_lc_in) cudaFree(c->d_lc_in);
  if (c->d_e_out) cudaFree(c->d_e_out);
  if (c->d_xyz_in) cudaFree(c->d_xyz_in);
  if (c->d_ctr_in) cudaFree(c->d_ctr_in);
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

int gd_release_memory(int device) {
  if (device < 0 || device >= GD_MAX_DEVICES) return fail(GD_ERR_INVALID, "device %d", device);
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (g_pool[device]) {
    CK(cudaSetDevice(device));
    CK(cudaMemPoolTrimTo(g_pool[device], 0));
  }
  return GD_OK;
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
  int cc_major = 0, cc_minor = 0, n_sms = 0;
  CK(cudaDeviceGetAttribute(&cc_major, cudaDevAttrComputeCapabilityMajor, device));
  CK(cudaDeviceGetAttribute(&cc_minor, cudaDevAttrComputeCapabilityMinor, device));
  CK(cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, device));
  if (cc_major < 10)
    return fail(GD_ERR_NODEVICE, "device %d is sm_%d%d; this library is built for sm_100a",
                device, cc_major, cc_minor);
  CK(cudaSetDevice(device));

  {
    const int rc0 = noalloc_prepare(device);
    if (rc0) return rc0;
  }
  /* the record downloads' staging buffers, once per process */
  if (mc->record) stage_prepare();

  gd_ctx *c = new gd_ctx();
  c->device = device;
  c->mc = *mc;
  c->num_sms = n_sms;
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
    if ((rc = layout_complex(c, ff, thr, d, ci, g))) return bail(rc);
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
    /* cleared: rows past a replica's count read as zeros, not as an earlier context's data */
    if ((rc = dalloc(c, &c->d_rec, (size_t)R * c->rec_cap))) return bail(rc);
    CK(cudaMemsetAsync(c->d_rec, 0, sizeof(gd_record_step) * R * c->rec_cap, c->stream));
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
  /* the persistent-CTA queue heads, then (with the exchange) one count per group and interval */
  const int n_ctr = chunks * nch + (exchange ? chunks * c->n_groups : 0);
  if ((rc = ensure_counters(c, n_ctr))) return rc;
  const long long key = ((long long)n_steps << 1) | (exchange ? 1 : 0);
  auto it = c->graphs.find(key);
  if (it == c->graphs.end()) {
    CK(cudaStreamSynchronize(c->stream));
    const size_t smem = smem_bytes(c);
    if ((rc = set_kernel_attrs(c, smem))) return rc;
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(c->d_counters, 0, sizeof(int) * n_ctr, c->stream);
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
        if (exchange) {
          /* the chain's groups are whole (chains are made of protein-conformer blocks) */
          a.x_done = c->d_counters + chunks * nch + (size_t)i * c->n_groups;
          a.x_group_base = c->d_group_base;
          a.x_acs = c->d_acs;
          a.x_call_base = c->d_cursor + 1;
          a.x_call_off = i;
          a.x_spd = c->mc.steps_per_dump;
          a.x_spe = spe;
        }
        launch_kernel(c)<<<grid, launch_threads(c), smem, st>>>(a, c->fc);
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
  if ((rc = ensure_cursor(c))) return rc;
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

}  // extern "C"
