/*
 * gd_capi_tile.cu -- the kernel's tile (gd_set_tile, gd_get_tile, gd_get_replicas_per_cta),
 * its autotuning probe (gd_autotune), the concurrent chains, the RNG stream of a complex and
 * the bound on the kernel's waits.
 */
#include "gd_capi_internal.cuh"

using namespace gdc;

extern "C" {

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
  /* the probe runs Monte Carlo steps of every replica (no records, no trace) from a copy of
   * the chain state, which is put back afterwards: the chains are left as they were */
  const size_t R = (size_t)c->n_rep;
  const size_t bytes = R * (6 * sizeof(float) + sizeof(gd_energy) + sizeof(float) + sizeof(int));
  char *keep = nullptr;
  if (cudaMalloc(&keep, bytes) != cudaSuccess)
    return fail(GD_ERR_NOMEM, "gd_autotune: no memory for the copy of the chain state");
  float *k_mm = reinterpret_cast<float *>(keep);
  gd_energy *k_e = reinterpret_cast<gd_energy *>(k_mm + R * 6);
  float *k_et = reinterpret_cast<float *>(k_e + R);
  int *k_na = reinterpret_cast<int *>(k_et + R);
  cudaMemcpyAsync(k_mm, c->d_mm, R * 6 * sizeof(float), cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(k_e, c->d_eold, R * sizeof(gd_energy), cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(k_et, c->d_etotal, R * sizeof(float), cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(k_na, c->d_nacc, R * sizeof(int), cudaMemcpyDeviceToDevice, c->stream);
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
  /* steps per probe launch: an exchange interval, fewer when one step of the first candidate
   * already takes long (large batches), so that the probe stays short */
  int probe_steps = 0;
  for (int i = 0; i < n_cand && rc == GD_OK; ++i) {
    if ((rc = gd_set_tile(c, -1, &cand[i])) != GD_OK) {
      /* a candidate that does not fit this batch is skipped */
      if (ms_out) ms_out[i] = -1.0f;
      rc = GD_OK;
      continue;
    }
    int n = 0;
    if ((rc = upload_tiles(c, 0, c->n_rep - 1, &n))) break;
    /* every candidate starts from the same chain state (the cost of a step depends on where
     * the ligands are) */
    cudaMemcpyAsync(c->d_mm, k_mm, R * 6 * sizeof(float), cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(c->d_eold, k_e, R * sizeof(gd_energy), cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(c->d_etotal, k_et, R * sizeof(float), cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(c->d_nacc, k_na, R * sizeof(int), cudaMemcpyDeviceToDevice, c->stream);
    GdMcArgs a = base_args(c);
    a.mode = 0;
    a.step0 = 0;
    a.rec = nullptr;
    a.trace_e = nullptr;
    a.trace_acc = nullptr;
    if (probe_steps == 0) {
      a.n_steps = 1;
      if ((rc = launch_mc(c, a, c->d_tiles, n, c->d_counters))) break; /* loads the kernel */
      cudaEventRecord(e0, c->stream);
      if ((rc = launch_mc(c, a, c->d_tiles, n, c->d_counters))) break;
      cudaEventRecord(e1, c->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        rc = fail(GD_ERR_CUDA, "gd_autotune: probe failed");
        break;
      }
      float t1 = 0.0f;
      cudaEventElapsedTime(&t1, e0, e1);
      probe_steps = std::max(1, std::min(c->mc.steps_per_exchange, (int)(20.0f / std::max(t1, 1e-3f))));
    }
    a.n_steps = probe_steps;
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
    ms /= (float)(repeats * probe_steps);
    if (ms_out) ms_out[i] = ms;
    if (ms < best_ms) {
      best_ms = ms;
      best_i = i;
    }
  }
  cudaMemcpyAsync(c->d_mm, k_mm, R * 6 * sizeof(float), cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->d_eold, k_e, R * sizeof(gd_energy), cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->d_etotal, k_et, R * sizeof(float), cudaMemcpyDeviceToDevice, c->stream);
  cudaMemcpyAsync(c->d_nacc, k_na, R * sizeof(int), cudaMemcpyDeviceToDevice, c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess && rc == GD_OK)
    rc = fail(GD_ERR_CUDA, "gd_autotune: restoring the chain state failed");
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(keep);
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

}  // extern "C"
