/*
 * gd_capi_internal.cuh -- what the host-side units of the C ABI share: the context (gd_ctx),
 * the per-complex bookkeeping, the error reporting, and the launch and buffer helpers.
 *
 *   gd_capi.cu          the context, its uploads and tile lists, the Monte Carlo calls,
 *                       records and state (the reference's Run and launcher, src/run.cu:33-288,
 *                       src/kernel_cuda_lancher_siglegpu.cu)
 *   gd_capi_layout.cu   the device layout of one complex
 *   gd_capi_tile.cu     the tile, its autotuning, chains, RNG streams and the wait bound
 *   gd_capi_stream.cu   records downloaded while the run proceeds (gd_records_stream)
 *   gd_capi_eval.cu     pose energies, placed coordinates and the energy trace
 *   gd_capi_noalloc.cu  pose energies without allocation (gd_eval_energy_noalloc)
 *   gd_capi_da.cu       the surrogate, delayed acceptance and its fallback controller, the
 *                       standalone network and k-means entry points
 */
#ifndef GD_CAPI_INTERNAL_CUH
#define GD_CAPI_INTERNAL_CUH

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
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

namespace gdc {

/* the calling thread's last error message (gd_last_error_string) */
extern thread_local std::string g_err;
/* records a formatted message and returns code */
int fail(int code, const char *fmt, ...);

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return fail(GD_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                               \
  } while (0)

constexpr float kPi = 3.1415926535f; /* reference src/size.h:67 */

float contact_threshold(float pmf0);
/* Distance beyond which the pair loop's far form gives its full form's result. */
double pmf_far_radius(float pmf0);
float bits_as_float(int v);
float host_dist2(float ax, float ay, float az, float px, float py, float pz);

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

}  // namespace gdc

struct RecStream;
struct RecAsync;
struct DaState;

struct gd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  gd_mc_params mc{};
  int n_complex = 0, n_rep = 0, n_groups = 0;
  int threads = 256, chunk = 512, unroll = 2, split = 1, num_sms = 148;
  int pack = 1; /* replicas per thread of the plain launches: the tile's lanes (threads) run on
                   threads / pack threads */
  int fill_threads = 0, fill_cap = 0; /* the last gd_set_tile in fill mode (threads > 0) */
  std::vector<gdc::ComplexInfo> info;
  std::vector<void *> allocs;      /* cudaMalloc'd buffers */
  std::vector<void *> pool_allocs; /* buffers from the device's context pool (ctx_pool) */
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
  bool counters_pooled = false; /* d_counters came from ctx_pool */
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
  float *d_xyz_in = nullptr, *d_ctr_in = nullptr; /* given coordinates and centres (mode 4) */
  size_t xyz_cap = 0;                             /* floats of d_xyz_in */
  int ctr_cap = 0;                                /* poses of d_ctr_in */
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
  std::vector<gdc::Chain> chain;
  int chain_gen = -1;
  GdTileDesc *d_chain_tiles = nullptr;
  int chain_tiles_cap = 0;
  /* record streaming into host memory (gd_records_stream) */
  struct RecStream *rs = nullptr;
  /* a dump window downloaded in the background (gd_get_records_async) */
  struct RecAsync *ra = nullptr;
};

#define GD_MAX_DEVICES 64

namespace gdc {

/* ---- the context's helpers (gd_capi.cu) ---- */
cudaError_t d2h_rows(void *dst, size_t hpitch, const void *src, size_t dpitch, size_t width,
                     int n);
/* makes d2h_rows' page-locked staging buffers (once per process) */
void stage_prepare();
/* The device's stream-ordered pool for the buffers gd_create sets up: it keeps freed memory
 * (no release threshold), so gd_destroy returns buffers without unmapping them and the next
 * context of the process reuses them; gd_release_memory trims it. Null if it cannot be made. */
cudaMemPool_t ctx_pool(int device);
/* n elements on the context's device, stream-ordered on its stream (gd_create synchronises
 * the stream before any other stream sees the buffer), freed by gd_destroy */
template <class T>
int dalloc(gd_ctx *c, T **p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  void *q = nullptr;
  cudaMemPool_t pool = ctx_pool(c->device);
  cudaError_t e = pool ? cudaMallocFromPoolAsync(&q, n * sizeof(T), pool, c->stream)
                       : cudaMalloc(&q, n * sizeof(T));
  if (e != cudaSuccess)
    return fail(GD_ERR_NOMEM, "allocation of %zu bytes failed: %s", n * sizeof(T),
                cudaGetErrorString(e));
  (pool ? c->pool_allocs : c->allocs).push_back(q);
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
int check_complex(const gd_complex_desc &d, int idx);
int pick_threads(const std::vector<ComplexInfo> &info);
void build_tiles(const gd_ctx *c, int r0, int r1, std::vector<GdTileDesc> &out);
size_t smem_bytes(const gd_ctx *c);
int ensure_counters(gd_ctx *c, int n);
/* the pinned host cursor of the graph launches (made on first use) */
int ensure_cursor(gd_ctx *c);
typedef void (*McKernel)(GdMcArgs, GdForceConst);
McKernel mc_kernel(int unroll, int split, bool da = false, int pack = 1);
int launch_pack(const gd_ctx *c, int split, bool da);
int launch_threads(const gd_ctx *c, int split = 0, bool da = false);
/* unroll 0: the tile's */
McKernel launch_kernel(const gd_ctx *c, int split = 0, bool da = false, int unroll = 0);
int grid_for(gd_ctx *c, int n_tiles, size_t smem, int split = 0, bool da = false, int unroll = 0);
GdMcArgs base_args(gd_ctx *c);
int set_kernel_attrs(const gd_ctx *c, size_t smem, int split = 0, bool da = false,
                     int unroll = 0);
int launch_mc(gd_ctx *c, GdMcArgs a, const GdTileDesc *d_tiles, int n_tiles, int *counter);
int upload_tiles(gd_ctx *c, int r0, int r1, int *n_out);
int check_range(const gd_ctx *c, int r0, int r1);
void build_chains(gd_ctx *c, int want, std::vector<Chain> &ch, std::vector<GdTileDesc> *tiles);
int ensure_chain_streams(gd_ctx *c, int n);
int ensure_chains(gd_ctx *c);
cudaStream_t chain_stream(gd_ctx *c, int k);
void chains_fork(gd_ctx *c, int n);
void chains_join(gd_ctx *c, int n);
void drop_graphs(gd_ctx *c);

/* ---- the record stream (gd_capi_stream.cu) ---- */
int rs_enqueue(gd_ctx *c, int rows_per_rep);
int rs_flush(gd_ctx *c);
int rs_restart(gd_ctx *c, int r0, int r1);
void rs_stop(gd_ctx *c);
/* waits for, then frees, the background window download */
void ra_free(gd_ctx *c);

/* ---- delayed acceptance (gd_capi_da.cu) ---- */
void da_free(gd_ctx *c);
void da_drop_graphs(gd_ctx *c);

/* ---- the device layout of one complex (gd_capi_layout.cu) ---- */
/* builds complex ci's arrays on the host, uploads them (pool memory, synchronised) and fills g;
 * thr: the contact thresholds [ligand type][point type] */
int layout_complex(gd_ctx *c, const gd_enepara *ff, const float (*thr)[GD_MAXTP1],
                   const gd_complex_desc &d, int ci, GdDevComplex &g);

/* ---- allocation-free pose evaluation (gd_capi_noalloc.cu) ---- */
int noalloc_prepare(int device);

}  // namespace gdc

#endif
