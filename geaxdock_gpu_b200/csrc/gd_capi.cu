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
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "gd_device.cuh"
#include "gd_numerics.h"

namespace gd {
template <int UNROLL>
__global__ void gd_mc_kernel(GdMcArgs a, GdForceConst f);
extern template __global__ void gd_mc_kernel<1>(GdMcArgs, GdForceConst);
extern template __global__ void gd_mc_kernel<2>(GdMcArgs, GdForceConst);
extern template __global__ void gd_mc_kernel<4>(GdMcArgs, GdForceConst);
__global__ void gd_exchange_kernel(const GdDevComplex *cxs, const int *group_base, int n_complex,
                                   int n_groups, gd_replica *replica, const float *etotal,
                                   int *acs, uint64_t seed, const int *call_base, int call_off,
                                   int mode_t);
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
};

}  // namespace

struct gd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  gd_mc_params mc{};
  int n_complex = 0, n_rep = 0, n_groups = 0;
  int threads = 256, chunk = 512, unroll = 2, num_sms = 148;
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
};

namespace {

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

McKernel mc_kernel(int unroll) {
  if (unroll >= 4) return gd::gd_mc_kernel<4>;
  if (unroll >= 2) return gd::gd_mc_kernel<2>;
  return gd::gd_mc_kernel<1>;
}

int grid_for(gd_ctx *c, int n_tiles, size_t smem) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, mc_kernel(c->unroll), c->threads,
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

int set_kernel_attrs(const gd_ctx *c, size_t smem) {
  const McKernel k = mc_kernel(c->unroll);
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
  mc_kernel(c->unroll)<<<grid, c->threads, smem, c->stream>>>(a, c->fc);
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

void drop_graphs(gd_ctx *c) {
  for (auto &g : c->graphs) cudaGraphExecDestroy(g.second);
  c->graphs.clear();
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
  drop_graphs(c);
  for (void *p : c->allocs) cudaFree(p);
  if (c->d_counters) cudaFree(c->d_counters);
  if (c->d_trace_e) cudaFree(c->d_trace_e);
  if (c->d_trace_acc) cudaFree(c->d_trace_acc);
  if (c->d_mm_in) cudaFree(c->d_mm_in);
  if (c->d_lc_in) cudaFree(c->d_lc_in);
  if (c->d_e_out) cudaFree(c->d_e_out);
  if (c->d_eval_tiles) cudaFree(c->d_eval_tiles);
  if (c->h_cursor) cudaFreeHost(c->h_cursor);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
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
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(GD_ERR_NODEVICE, "device %d is sm_%d%d; this library is built for sm_100a",
                device, prop.major, prop.minor);
  CK(cudaSetDevice(device));

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
  if (t->replicas_per_cta < 1 || t->replicas_per_cta > GD_MAX_SLOTS)
    return fail(GD_ERR_INVALID, "replicas_per_cta outside 1..%d", GD_MAX_SLOTS);
  if (k < -1 || k >= c->n_complex) return fail(GD_ERR_INVALID, "bad complex index");
  /* one block size per context: every complex's k must fit the block */
  std::vector<ComplexInfo> info = c->info;
  for (int i = 0; i < c->n_complex; ++i)
    if (k == -1 || k == i) info[i].k = std::min(t->replicas_per_cta, info[i].n_tmp * info[i].n_lig);
  int T = 32;
  for (auto &x : info) T = std::max(T, ((x.k * x.lna + 31) / 32) * 32);
  if (T > GD_MAX_TPB) return fail(GD_ERR_INVALID, "replicas_per_cta * lna exceeds %d", GD_MAX_TPB);
  c->info = info;
  c->threads = T;
  c->chunk = t->chunk_points;
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
  t->replicas_per_cta = c->info[k].k;
  t->chunk_points = c->chunk;
  t->unroll = c->unroll;
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
  rc = launch_mc(c, a, c->d_tiles, n, c->d_counters);
  if (rc) return rc;
  c->initialized = true;
  c->exchange_calls = 0;
  return GD_OK;
}

int gd_reset_records(gd_ctx *c, int r0, int r1) {
  if (!c) return fail(GD_ERR_INVALID, "null context");
  int rc = check_range(c, r0, r1);
  if (rc) return rc;
  const int n = r1 - r0 + 1;
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
  return launch_mc(c, a, c->d_tiles, n, c->d_counters);
}

int gd_exchange(gd_ctx *c, int mode_l, int mode_t) {
  (void)mode_l;
  if (!c) return fail(GD_ERR_INVALID, "null context");
  if (!c->initialized) return fail(GD_ERR_STATE, "gd_mc_init has not run");
  if (mode_t < 0) return fail(GD_ERR_INVALID, "mode_t must be >= 0");
  CK(cudaSetDevice(c->device));
  gd::gd_exchange_kernel<<<(c->n_groups + 127) / 128, 128, 0, c->stream>>>(
      c->d_cx, c->d_group_base, c->n_complex, c->n_groups, c->d_replica, c->d_etotal, c->d_acs,
      c->mc.seed, nullptr, c->exchange_calls, mode_t);
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
  const int chunks = n_steps / spe;
  int rc = ensure_counters(c, chunks);
  if (rc) return rc;
  const long long key = ((long long)n_steps << 1) | (exchange ? 1 : 0);
  auto it = c->graphs.find(key);
  if (it == c->graphs.end()) {
    int n = 0;
    if ((rc = upload_tiles(c, 0, c->n_rep - 1, &n))) return rc;
    CK(cudaStreamSynchronize(c->stream));
    const size_t smem = smem_bytes(c);
    if ((rc = set_kernel_attrs(c, smem))) return rc;
    const int grid = grid_for(c, n, smem);
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(c->d_counters, 0, sizeof(int) * chunks, c->stream);
    for (int i = 0; i < chunks; ++i) {
      GdMcArgs a = base_args(c);
      a.mode = 0;
      a.n_steps = spe;
      a.step0 = i * spe;
      a.step_base = c->d_cursor;
      a.tiles = c->d_tiles;
      a.n_tiles = n;
      a.tile_counter = c->d_counters + i;
      mc_kernel(c->unroll)<<<grid, c->threads, smem, c->stream>>>(a, c->fc);
      if (exchange)
        gd::gd_exchange_kernel<<<(c->n_groups + 127) / 128, 128, 0, c->stream>>>(
            c->d_cx, c->d_group_base, c->n_complex, c->n_groups, c->d_replica, c->d_etotal,
            c->d_acs, c->mc.seed, c->d_cursor + 1, i, !(i % 2));
    }
    cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    if (ce != cudaSuccess) return fail(GD_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
    cudaGraphExec_t exec;
    ce = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return fail(GD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ce));
    it = c->graphs.emplace(key, exec).first;
  }
  /* the graph reads the full-range tile list and its step and exchange-call bases from
   * the device cursor */
  {
    int n = 0;
    if ((rc = upload_tiles(c, 0, c->n_rep - 1, &n))) return rc;
  }
  CK(cudaStreamSynchronize(c->stream));
  c->h_cursor[0] = s1;
  c->h_cursor[1] = c->exchange_calls;
  CK(cudaMemcpyAsync(c->d_cursor, c->h_cursor, 2 * sizeof(int), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaGraphLaunch(it->second, c->stream));
  if (exchange) c->exchange_calls += chunks;
  return GD_OK;
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
  if (cap != c->rec_cap) return fail(GD_ERR_INVALID, "cap %d != record capacity %d", cap, c->rec_cap);
  const int n = r1 - r0 + 1;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(steps, c->d_rec + (size_t)r0 * cap, sizeof(gd_record_step) * (size_t)n * cap,
                cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(next_ptr, c->d_rec_next + r0, sizeof(int) * n, cudaMemcpyDeviceToHost));
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
  for (int i = 0; i < n; ++i) {
    CK(cudaMemcpy(host[i].step, c->d_rec + (size_t)(r0 + i) * c->rec_cap,
                  sizeof(gd_record_step) * c->rec_cap, cudaMemcpyDeviceToHost));
    host[i].next_ptr = nxt[i];
  }
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
 * kernel), and calls whose kernels overlap on the GPU would race on it. */

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

/* Device address of the scratch array on `device` (the current device), looked up once per
 * device: host code cannot use the symbol itself as a device address. */
int noalloc_scratch(int device, NoallocScratch **out) {
  if (device < 0 || device >= 64) return fail(GD_ERR_NODEVICE, "device %d out of range", device);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(GD_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
    g_noalloc_addr[device] = p;
  }
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
  if (n < 0 || n > GD_NOALLOC_MAX_POSES)
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
  mc_kernel(c->unroll)<<<grid, c->threads, smem, c->stream>>>(a, c->fc);
  CK(cudaGetLastError());
  return GD_OK;
}
