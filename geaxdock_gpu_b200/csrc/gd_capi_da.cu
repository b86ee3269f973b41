/*
 * gd_capi_da.cu -- the learned part behind the C ABI: the surrogate's creation, sample
 * collection and training (gd_sur_*), the delayed-acceptance steps and their fallback
 * controller (gd_da_*), the standalone network (gd_mlp_*) and the k-means entry points of
 * post-MC clustering (gd_kmeans*). No counterpart in the reference except k-means
 * (src/util.C:1801-1880).
 */
#include "gd_capi_internal.cuh"

using namespace gdc;

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
  int *d_train_ctr = nullptr; /* [2]: the batch draws' iteration count, this call's loss slot */
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

}  // namespace

namespace gdc {

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

}  // namespace gdc

namespace {

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

/* unroll of the exact stage at split S: with one lane per atom (most proposals surviving:
 * collect steps, or a pass rate above 0.4, da_choose_split) the stage is throughput-bound
 * beside the other chains' front kernels, and the 80-register variant with two point pairs in
 * flight leaves them room on the SMs; split over several lanes (few survivors) one tile's
 * latency sets the step, and the tile's own unroll is kept (four pairs in flight shorten a
 * tile). Config 1, DA / plain at pass 0.96 / 0.50 / 0.20 (splits 1 / 1 / 2): two pairs 1.08 /
 * 1.91 / 3.08, four pairs 1.04 / 1.94 / 3.38. */
int da_unroll(const gd_ctx *c, int S) { return S > 1 ? c->unroll : std::min(c->unroll, 2); }

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
                     size_t smem, cudaStream_t st, int S, int U) {
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
  mc_kernel(U, S, true)<<<grid_for(c, t1 - t0, smem, S, true, U), c->threads, smem, st>>>(
      a, c->fc);
}

/* the graph of n_steps steps (collect: plain steps that store samples), one chain per stream */
int da_graph(gd_ctx *c, int n_steps, int exchange, bool collect, int S, cudaGraphExec_t *out) {
  DaState *d = c->da;
  const int U = da_unroll(c, S);
  const long long key = ((long long)U << 44) | ((long long)n_steps << 7) | ((long long)S << 2) |
                        (exchange ? 2 : 0) | (collect ? 1 : 0);
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
    if (d->d_counters) {
      /* the cached graphs point at the old counters: finish them and drop them first */
      CK(cudaStreamSynchronize(c->stream));
      da_drop_graphs(c);
      cudaFree(d->d_counters);
    }
    d->d_counters = nullptr;
    d->counters_cap = 0;
    CK(cudaMalloc(&d->d_counters, sizeof(int) * n_steps * nch));
    d->counters_cap = n_steps * nch;
  }
  if ((rc = da_upload_epi(c))) return rc;
  CK(cudaStreamSynchronize(c->stream));
  const size_t smem = smem_bytes(c);
  if ((rc = set_kernel_attrs(c, smem, S, true, U))) return rc;
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
      da_launch_exact(c, ch, k, n_steps, j, collect, smem, st, S, U);
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
  if ((rc = ensure_cursor(c))) return rc;
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
  if (!d->d_train_ctr && (rc = da_alloc(d, &d->d_train_ctr, 2))) return rc;
  /* One Adam step: batch draw, forward, loss, backward, Adam, the BF16 weight copies (about 30
   * launches). Its per-step values live on the device (the draw's iteration count and the
   * loss slot in d_train_ctr, Adam's step count in the network), so the step is run once
   * eagerly -- which sets up every allocation and kernel attribute it needs -- then captured in
   * a CUDA graph and replayed for the other steps, each replay one launch. */
  if (iterations > 0) {
    const int ctr[2] = {(int)d->train_iter, 0};
    CK(cudaMemcpyAsync(d->d_train_ctr, ctr, sizeof(ctr), cudaMemcpyHostToDevice, c->stream));
    if (gd::mlp_adam_dev_sync(d->net, c->stream)) return fail(GD_ERR_CUDA, "Adam step count");
    auto step = [&]() -> int {
      gd::da_gather(a, start, n_valid, B, d->d_train_ctr, d->d_t, c->stream);
      if (gd::mlp_embed(d->net, B, c->stream) ||
          gd::mlp_loss_backward(d->net, B, d->d_t, c->stream))
        return fail(GD_ERR_CUDA, "training step failed: %s",
                    cudaGetErrorString(cudaGetLastError()));
      gd::da_train_tick(d->d_loss_hist, d->net.loss, d->d_train_ctr, c->stream);
      if (gd::mlp_adam_dev(d->net, d->prm.lr, c->stream))
        return fail(GD_ERR_CUDA, "Adam step failed");
      return GD_OK;
    };
    if ((rc = step())) return rc;
    if (iterations > 1) {
      CK(cudaStreamSynchronize(c->stream));
      cudaGraph_t graph = nullptr;
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      rc = step();
      const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
      if (rc || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return rc ? rc : fail(GD_ERR_CUDA, "training graph capture: %s", cudaGetErrorString(ce));
      }
      cudaGraphExec_t exec = nullptr;
      const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      if (ie != cudaSuccess)
        return fail(GD_ERR_CUDA, "training graph instantiate: %s", cudaGetErrorString(ie));
      cudaError_t le = cudaSuccess;
      for (int it = 1; it < iterations && le == cudaSuccess; ++it)
        le = cudaGraphLaunch(exec, c->stream);
      const cudaError_t se = cudaStreamSynchronize(c->stream);
      cudaGraphExecDestroy(exec);
      if (le != cudaSuccess || se != cudaSuccess)
        return fail(GD_ERR_CUDA, "training graph: %s",
                    cudaGetErrorString(le != cudaSuccess ? le : se));
    }
    d->train_iter += iterations;
    d->net.adam_t += iterations;
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
