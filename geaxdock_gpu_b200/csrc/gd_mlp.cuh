/*
 * gd_mlp.cuh -- the energy surrogate: a 64 -> H -> H -> H -> 1 SiLU MLP with a learned
 * conformer embedding, BF16 weights and activations on the tensor cores, FP32 accumulation,
 * FP32 master parameters and Adam moments. Internal C++ interface shared by gd_mlp.cu (the
 * kernels) and gd_capi_da.cu (delayed acceptance).
 *
 * Input row (64 features): [0,3) ligand centre minus pocket centre / 4 A, [3,7) unit
 * quaternion of the pose rotation (w >= 0), [7,39) conformer embedding (32, learned, one row
 * per (complex, protein conformer, ligand conformer)), [39,55) pocket features (16), [55,61)
 * the first two columns of the rotation matrix (a continuous rotation code), [61] distance
 * to the pocket centre / 8 A, [62,64) zero. The network predicts (E - mu) / sigma; mu, sigma
 * are set from the training samples.
 */
#ifndef GD_MLP_CUH
#define GD_MLP_CUH

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "gd_device.cuh"

#define GD_MLP_IN 64
#define GD_MLP_EMB 32
#define GD_MLP_EMB_OFF 7
#define GD_MLP_POCKET 16
#define GD_MLP_POCKET_OFF 39

namespace gd {

/* the activation and its derivative, written once for every kernel that applies them */
__device__ __forceinline__ float mlp_silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float mlp_silu_grad(float z) {
  const float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

struct MlpLayout {
  int hidden = 256, n_emb = 0;
  size_t w1, b1, w2, b2, w3, b3, w4, b4, emb, total;
  void set(int h, int ne) {
    hidden = h;
    n_emb = ne;
    size_t o = 0;
    w1 = o; o += (size_t)GD_MLP_IN * h;
    b1 = o; o += h;
    w2 = o; o += (size_t)h * h;
    b2 = o; o += h;
    w3 = o; o += (size_t)h * h;
    b3 = o; o += h;
    w4 = o; o += h;
    b4 = o; o += 4; /* keep the embedding 16-byte aligned */
    emb = o; o += (size_t)ne * GD_MLP_EMB;
    total = o;
  }
};

/* One network and its training buffers on one device. */
struct Mlp {
  MlpLayout L;
  float *theta = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr; /* [L.total] */
  __nv_bfloat16 *wh = nullptr;        /* BF16 copies of W1, W2, W3 (same offsets as theta) */
  __nv_bfloat16 *wf = nullptr;        /* W1, W2, W3 in MMA fragment order (H = 128, 256) */
  float mu = 0.0f, sigma = 1.0f;      /* target normalisation */
  int adam_t = 0;
  int *adam_dev = nullptr;            /* [1] Adam step count and [2] its bias corrections (as
                                         floats) on the device, for graph-replayed steps */
  int cap = 0;                        /* rows of the work buffers */
  __nv_bfloat16 *X = nullptr, *A1 = nullptr, *A2 = nullptr, *A3 = nullptr, *D = nullptr;
  __nv_bfloat16 *D2 = nullptr;        /* second buffer of the back-propagated dZ (ping-pong) */
  int *err = nullptr;                 /* [1] nonzero when a tensor-core GEMM's wait ran out */
  float *Z1 = nullptr, *Z2 = nullptr, *Z3 = nullptr, *C = nullptr, *y = nullptr, *dy = nullptr;
  float *loss = nullptr;              /* [1] */
  int *conf = nullptr;                /* [cap] embedding row per input row */
  float *P = nullptr;                 /* per-chunk partials of the batch reductions */
  float *Pb = nullptr;                /* [cap / 128][hidden] per-tile bias-gradient partials */
  size_t p_cap = 0;
};

int mlp_create(Mlp &n, int hidden, int n_emb, uint64_t seed, cudaStream_t s);
void mlp_destroy(Mlp &n);
int mlp_reserve(Mlp &n, int rows);
/* rows of X (bf16, 64 wide) -> y; the embedding columns of rows with conf >= 0 are taken from
 * the table (one fused kernel for H = 128 and 256, layer by layer otherwise) */
int mlp_forward(Mlp &n, int rows, cudaStream_t s);
/* rows of X from device FP32 rows (rounded to BF16) and their conformer ids */
int mlp_set_rows(Mlp &n, const float *x, const int *conf, int rows, cudaStream_t s);
/* fills the embedding columns of X from theta for the rows' conformer ids (n.conf >= 0) */
int mlp_embed(Mlp &n, int rows, cudaStream_t s);
/* forward + MSE loss against t (normalised targets) + backward into n.grad (zeroed first) */
int mlp_loss_backward(Mlp &n, int rows, const float *t, cudaStream_t s);
int mlp_adam(Mlp &n, float lr, cudaStream_t s);
/* the same Adam step with its step count and bias corrections kept on the device (adam_dev,
 * loaded from adam_t by mlp_adam_dev_sync), so that one step can be captured in a CUDA graph and
 * replayed; the host's adam_t is not advanced */
int mlp_adam_dev(Mlp &n, float lr, cudaStream_t s);
int mlp_adam_dev_sync(Mlp &n, cudaStream_t s);
/* BF16 copies of the weight matrices from theta (row-major, and in fragment order) */
int mlp_refresh_bf16(Mlp &n, cudaStream_t s);
/* after a synchronisation: 0, or -6 (and the flag cleared) if a GEMM's bounded wait ran out */
int mlp_status(Mlp &n);

/* ---------------- delayed acceptance (gd_da.cu) ---------------- */

/* One (complex, protein conformer) block of replicas: the unit of survivor compaction. Its
 * tiles occupy the fixed positions [tile_base, tile_base + n_tiles) of the exact kernel's tile
 * list; their counts come from the group's survivor counter at run time. */
struct GdGroup {
  int ci, pc, b0, n;          /* complex, protein conformer, first replica, replicas */
  int tile_base, n_tiles, k, pad;
};

/* per-complex statistics (reduced from per-replica counters by da_stats) */
#define GD_DA_PROPOSED 0      /* proposals seen with the surrogate stage on */
#define GD_DA_PASSED 1        /* ... that passed the surrogate stage */
#define GD_DA_ACCEPTED 2      /* ... that the exact energy then accepted */
#define GD_DA_PLAIN 3         /* proposals handled as plain Metropolis (stage off) */
#define GD_DA_PLAIN_ACC 4     /* ... accepted */
#define GD_DA_NSTAT 8
/* per-complex double sums: squared surrogate error and its count over exact evaluations */
#define GD_DA_NERR 2

/* front kernel modes */
#define GD_DA_STEP 0          /* proposal, surrogate stage, compaction */
#define GD_DA_COLLECT 1       /* proposal, every proposal passes, feature rows to the samples */
#define GD_DA_CURRENT 2       /* surrogate of the current poses -> s_cur */

struct GdDaDev {
  const GdDevComplex *cx;
  const int *rep_cx;          /* [n_rep] complex of each replica */
  const int *rep_group;       /* [n_rep] compaction group of each replica */
  const int *group_b0;        /* [n_groups] first replica (= first pose slot) of each group */
  const int *emb_base;        /* [n_complex] first embedding row of the complex (< 0: none) */
  const float *pocket_feat;   /* [n_complex*16] */
  const int *active;          /* [n_complex] 1: surrogate stage on */
  int n_rep;
  /* replica state (the plain engine's arrays) */
  const gd_replica *replica;
  const float *mm_old;
  /* per step */
  float *u2;                  /* [n_rep] final accept uniform (the plain step's) */
  float *s_cur, *s_new;       /* [n_rep] surrogate energy at the current / proposed pose */
  int *pose_rep;              /* [n_rep] survivors, compacted per group */
  float *pose_mm;             /* [n_rep*6] */
  int *pose_lc;               /* [n_rep] */
  /* per-replica counters */
  int *prop, *pass, *plain;
  /* the network */
  const float *theta;
  const __nv_bfloat16 *wf;    /* fragment-ordered BF16 weights (Mlp::wf) */
  MlpLayout L;
  float mu, sigma;
  __nv_bfloat16 *X;           /* global feature rows (surrogate predictions of given poses) */
  int *conf;
  /* training samples, ring of smp_cap rows */
  __nv_bfloat16 *smp_X;
  int *smp_conf;
  float *smp_t;
  long long smp_cap;
  /* decision trace, [n_rep*tr_cap] or null */
  float *tr_s, *tr_e;
  int *tr_flag;
  int tr_cap, tr_step0;
  /* proposals */
  uint64_t seed;
  int move_kind;
  float move_scale[6];
  const int *step_base;       /* device step cursor */
};

/* Front kernel of one delayed-acceptance step (mode GD_DA_*) for replicas [r_begin, r_end):
 * the plain step's proposal and accept uniform (same Philox counters as gd_mc_kernel), the
 * surrogate-stage uniform, the feature rows, the network on them, the surrogate Metropolis
 * test and the survivors' compaction into their group's pose slots (cnt[group] survivors). */
int da_front(const GdDaDev &d, int mode, int step0, int *cnt, int r_begin, int r_end,
             cudaStream_t s);
/* kernel attributes of da_front for a hidden width (call once per device, outside capture) */
int da_prepare(int hidden);
/* feature rows 0..n-1 of X / conf for n poses of one (complex, protein, ligand conformer) */
void da_pose_features(const GdDaDev &d, int ci, int pc, int lc, const float *mm, int n,
                      cudaStream_t s);
/* per-complex sums of the per-replica counters (one CTA per complex, fixed order):
 * stats[ci*GD_DA_NSTAT + k], err[ci*GD_DA_NERR + k] */
void da_stats(const GdDaDev &d, const GdDaEpi &e_host, const GdDevComplex *cx_dev, int n_complex,
              unsigned long long *stats, double *err, cudaStream_t s);
/* training batch: rows drawn from the sample ring into X / conf / t (normalised, clipped), the
 * draw keyed by the iteration count at ctr[0] (device memory, so that the step replays) */
void da_gather(const GdDaDev &d, long long start, long long n_valid, int rows, const int *ctr,
               float *t, cudaStream_t s);
/* end of a training step: hist[ctr[1]] = *loss, then both counters advance */
void da_train_tick(float *hist, const float *loss, int *ctr, cudaStream_t s);
/* per-block sum, sum of squares and count of the sample targets inside [lo, hi]:
 * GD_DA_MOM_BLOCKS x 3 doubles into part (summed on the host in block order) */
#define GD_DA_MOM_BLOCKS 256
void da_target_moments(const GdDaDev &d, long long start, long long n_valid, float lo, float hi,
                       double *part, cudaStream_t s);

}  // namespace gd

#endif
