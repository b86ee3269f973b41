/*
 * gd_capi_eval.cu -- pose energies on demand (gd_eval_energy, gd_eval_energy_xyz): one launch of
 * the Monte Carlo kernel in its evaluation modes over given poses or placed coordinates; placed
 * ligand coordinates of given poses (gd_place_ligand, the reference's PlaceLigand as its trace
 * tool calls it); and the per-step energy trace of replica 0 (gd_trace_enable, gd_trace_get).
 */
#include "gd_capi_internal.cuh"

using namespace gdc;

namespace {

/* Energies of n poses of one (complex, protein conformer, ligand conformer): moved by
 * movematrix rows (mm, kernel mode 2), or given as placed coordinates and centres (xyz and
 * center, mode 4). */
int eval_poses(gd_ctx *c, int ci, int prt_conf, int lig_conf, const float *mm, const float *xyz,
               const float *center, int n, gd_energy *out) {
  if (!c || !out || (!mm && !(xyz && center))) return fail(GD_ERR_INVALID, "null argument");
  if (ci < 0 || ci >= c->n_complex) return fail(GD_ERR_INVALID, "bad complex index");
  const ComplexInfo &x = c->info[ci];
  if (prt_conf < 0 || prt_conf >= x.n_prt || lig_conf < 0 || lig_conf >= x.n_lig)
    return fail(GD_ERR_INVALID, "conformer index out of range");
  if (n < 1) return GD_OK;
  CK(cudaSetDevice(c->device));
  const bool given = mm == nullptr;
  if (given) {
    const size_t need = (size_t)n * x.lna * 3;
    if (need > c->xyz_cap) {
      if (c->d_xyz_in) cudaFree(c->d_xyz_in);
      c->d_xyz_in = nullptr;
      c->xyz_cap = 0;
      CK(cudaMalloc(&c->d_xyz_in, sizeof(float) * need));
      c->xyz_cap = need;
    }
    if (n > c->ctr_cap) {
      if (c->d_ctr_in) cudaFree(c->d_ctr_in);
      c->d_ctr_in = nullptr;
      c->ctr_cap = 0;
      CK(cudaMalloc(&c->d_ctr_in, sizeof(float) * 3 * n));
      c->ctr_cap = n;
    }
  }
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
  if (given) {
    CK(cudaMemcpy(c->d_xyz_in, xyz, sizeof(float) * (size_t)n * x.lna * 3,
                  cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_ctr_in, center, sizeof(float) * 3 * n, cudaMemcpyHostToDevice));
  } else {
    CK(cudaMemcpy(c->d_mm_in, mm, sizeof(float) * 6 * n, cudaMemcpyHostToDevice));
  }
  CK(cudaMemcpy(c->d_lc_in, lc.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_eval_tiles, tiles.data(), sizeof(GdTileDesc) * tiles.size(),
                cudaMemcpyHostToDevice));
  GdMcArgs a = base_args(c);
  a.mode = given ? 4 : 2;
  a.n_steps = 1;
  a.mm_in = given ? nullptr : c->d_mm_in;
  a.xyz_in = given ? c->d_xyz_in : nullptr;
  a.center_in = given ? c->d_ctr_in : nullptr;
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

}  // namespace

extern "C" {

int gd_eval_energy(gd_ctx *c, int ci, int prt_conf, int lig_conf, const float *mm, int n,
                   gd_energy *out) {
  if (!mm) return fail(GD_ERR_INVALID, "null argument");
  return eval_poses(c, ci, prt_conf, lig_conf, mm, nullptr, nullptr, n, out);
}

int gd_eval_energy_xyz(gd_ctx *c, int ci, int prt_conf, int lig_conf, const float *xyz,
                       const float *center, int n, gd_energy *out) {
  if (!xyz || !center) return fail(GD_ERR_INVALID, "null argument");
  return eval_poses(c, ci, prt_conf, lig_conf, nullptr, xyz, center, n, out);
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
