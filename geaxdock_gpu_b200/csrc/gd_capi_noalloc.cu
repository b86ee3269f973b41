/*
 * gd_capi_noalloc.cu -- gd_eval_energy_noalloc, pose energies for callers that cannot
 * allocate device memory when they need them. Its scratch is a file-scope device array of this
 * unit, whose device address gd_create looks up once per device (noalloc_prepare).
 */
#include "gd_capi_internal.cuh"

using namespace gdc;

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

}  // namespace

namespace gdc {

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

}  // namespace gdc

namespace {

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
