/*
 * geauxdock_b200.h -- C ABI of the B200 replica-exchange Monte Carlo docking engine.
 *
 * This is the drop-in boundary for the device half of GeauxDock's docking run
 * (reference: src/run.cu:33-288 `Run`, src/kernel_cuda.cuh:5-13 kernels). Every entry
 * point takes plain pointers and sizes, returns an int status (GD_OK == 0, negative
 * GD_ERR_* on failure), never exits the process, and records a message retrievable
 * with gd_last_error_string(). One context owns one CUDA stream on one device; calls
 * on one context must not race (thread-compatible, not thread-safe).
 *
 * Byte layouts that the reference writes to disk or hands between its host and device
 * halves are reproduced exactly: gd_energy == Energy (src/dock.h:108-128),
 * gd_replica == Replica (src/dock.h:302-309), gd_record_step == LigRecordSingleStep
 * (src/dock.h:361-367), gd_lig_record == LigRecord (src/dock.h:377-381),
 * gd_temp == Temp (src/dock.h:288-293), gd_enepara == EnePara (src/dock_soa.h:99-137),
 * gd_enepara_raw == EnePara0 (src/dock.h:256-272).
 */
#ifndef GEAUXDOCK_B200_H
#define GEAUXDOCK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- capacities (same values as the reference's src/size.h:19-122) ---- */
#define GD_MAXLIG 100          /* ligand heavy atoms */
#define GD_MAXPRO 10000        /* protein effective points */
#define GD_MAXTP1 30           /* protein point types */
#define GD_MAXTP2 24           /* ligand atom types */
#define GD_MAXTP3 50           /* electrostatic point codes */
#define GD_MAXTP4 20           /* residue codes */
#define GD_MAXWEI 10           /* 9 energy terms + total */
#define GD_MAXMCS 256          /* MCS fields per position */
#define GD_MAXTMP 40           /* temperatures */
#define GD_MAXPOS 1000         /* MCS positions */
#define GD_MAXKDE 10000        /* KDE points */
#define GD_STEPS_PER_DUMP 2000 /* reference record capacity (plus one for step 0) */
#define GD_MCS_INVALID_COORD 728492.0f

/* ---- status codes ---- */
#define GD_OK 0
#define GD_ERR_INVALID (-1)    /* bad argument or inconsistent description */
#define GD_ERR_CUDA (-2)       /* a CUDA runtime call failed */
#define GD_ERR_NOMEM (-3)      /* device or host allocation failed */
#define GD_ERR_CAPACITY (-4)   /* a size exceeds a compiled capacity */
#define GD_ERR_TIMEOUT (-5)    /* a bounded device wait gave up */
#define GD_ERR_STATE (-6)      /* call out of order (e.g. run before init) */
#define GD_ERR_NODEVICE (-7)   /* no usable sm_100 device */
#define GD_ERR_RECORD_FULL (-8)/* a replica's record buffer overflowed */

/* move proposal kinds */
#define GD_MOVE_UNIFORM 0      /* m' = m + s*(2u-1): reference Move_d (src/kernel_cuda_l1_montecarlo.cu:100) */
#define GD_MOVE_GAUSSIAN 1     /* m' = m + s*N(0,1) */

/* ---- reference-identical record / state layouts ---- */
typedef struct { float e[GD_MAXWEI]; float cms; float rmsd; } gd_energy;            /* 48 B */
typedef struct { int idx_rep; int idx_prt; int idx_tmp; int idx_lig; } gd_replica;  /* 16 B */
typedef struct {
  gd_replica replica;
  gd_energy energy;
  float movematrix[6];     /* translation x y z, Euler rotation x y z */
  int step;
} gd_record_step;                                                                   /* 92 B */
typedef struct { gd_record_step step[GD_STEPS_PER_DUMP + 1]; int next_ptr; } gd_lig_record;
typedef struct { float t; float minus_beta; int order; } gd_temp;

/* Folded force-field tables, the kernel-ready form produced by OptimizeEnepara
 * (reference src/util.C:717-760). Indices: [ligand type][protein type]. */
typedef struct {
  float p1a[GD_MAXTP2][GD_MAXTP1];
  float p2a[GD_MAXTP2][GD_MAXTP1];
  float lj0, lj1;
  float el0;
  float el1;
  float ele[GD_MAXTP3];
  float a1;
  float b1;
  float pmf0[GD_MAXTP2][GD_MAXTP1];
  float pmf1[GD_MAXTP2][GD_MAXTP1];
  float hdb0[GD_MAXTP2][GD_MAXTP1];
  float hdb1[GD_MAXTP2][GD_MAXTP1];
  float hpp[GD_MAXTP4];
  float hpl0[GD_MAXTP2];
  float hpl1[GD_MAXTP2];
  float hpl2[GD_MAXTP2];
  float kde2;
  float kde3;
  float w[GD_MAXWEI];
  float a_para[GD_MAXWEI];
  float b_para[GD_MAXWEI];
} gd_enepara;

/* Raw force-field parameters as read from the `paras` file (reference EnePara0,
 * src/dock.h:256-272; parsed by loadEnePara, src/load.C:1477-1660).
 * Indices: [protein type][ligand type][k]. */
typedef struct {
  float vdw[GD_MAXTP1][GD_MAXTP2][2];
  float ele[GD_MAXTP3];
  float pmf[GD_MAXTP1][GD_MAXTP2][2];
  float hpp[GD_MAXTP4];
  float hpl[GD_MAXTP2][2];
  float hdb[GD_MAXTP1][GD_MAXTP2][2];
  float lj[3];
  float el[2];
  float kde;
  float w[GD_MAXWEI];
  float a_para[GD_MAXWEI];
  float b_para[GD_MAXWEI];
} gd_enepara_raw;

/* One docking complex: what one reference `Run` call receives
 * (src/run.h:8-19). All arrays are host pointers, copied by gd_create.
 * Conformer-major layouts: element (conformer c, atom/point i) is at [c*count + i]. */
typedef struct {
  int n_lig;  /* ligand conformers (reference ComplexSize.n_lig) */
  int n_prt;  /* protein conformers (n_prt) */
  int n_tmp;  /* temperatures (n_tmp) */
  int lna;    /* ligand atoms */
  int pnp;    /* protein effective points */
  int pnk;    /* KDE points */
  int pos;    /* MCS positions (>= 1; the reference takes log(0/0) otherwise) */
  /* ligand conformers: coord_orig in the ligand-centre frame, per conformer centre (lab frame) */
  const float *lig_x, *lig_y, *lig_z;   /* [n_lig*lna] */
  const float *lig_center;              /* [n_lig*3] */
  const int *lig_t;                     /* [n_lig*lna] atom type 0..GD_MAXTP2-1 */
  const float *lig_c;                   /* [n_lig*lna] charge */
  const int *lig_n;                     /* [n_lig*lna] SDF atom number (MCS field index - 1) */
  /* protein conformers, folded per point as CopyProteinResidue does (src/util.C:574-597) */
  const float *prt_x, *prt_y, *prt_z;   /* [n_prt*pnp] */
  const int *prt_t;                     /* point type 0..GD_MAXTP1-1 */
  const int *prt_c;                     /* point class */
  const float *prt_ele;                 /* ele[t] (t != 0) or ele[d + 30] */
  const int *prt_seq3r;                 /* PSP column (seq3[r]) */
  const int *prt_hflag;                 /* (c == 0 && d == 12) || c == 2 */
  const float *prt_hpp;                 /* hpp[d] */
  const float *pocket_center;           /* [3] */
  /* pocket-specific potential, row-major [GD_MAXTP2][psp_ld], read at [lig type][seq3r] */
  const float *psp;
  int psp_ld;
  /* KDE points */
  const float *kde_x, *kde_y, *kde_z;   /* [pnk] */
  const int *kde_t;                     /* [pnk] */
  /* MCS positions: row-major [pos][mcs_ld] indexed by SDF atom number + 1 */
  const float *mcs_x, *mcs_y, *mcs_z;
  const float *mcs_tcc;                 /* [pos] */
  int mcs_ld;
  const gd_temp *temp;                  /* [n_tmp] */
} gd_complex_desc;

/* Monte Carlo parameters (reference McPara, src/dock.h:335-345, plus the RNG choice). */
typedef struct {
  int steps_per_exchange;   /* steps per gd_mc_run call (reference default 10) */
  int steps_per_dump;       /* record capacity per replica is steps_per_dump + 1 */
  float move_scale[6];      /* translation x y z, rotation x y z */
  int move_kind;            /* GD_MOVE_UNIFORM or GD_MOVE_GAUSSIAN */
  int record;               /* 1: append accepted steps to the per-replica records */
  uint64_t seed;            /* Philox4x32-10 key */
} gd_mc_params;

/* CTA tile of the fused Monte Carlo kernel. */
typedef struct {
  int replicas_per_cta;     /* replicas sharing one protein tile in one CTA */
  int chunk_points;         /* protein points staged per shared-memory buffer */
  int unroll;               /* protein point pairs in flight per lane: 1, 2 or 4 (0: keep) */
  int split;                /* lanes per ligand atom, each walking 1/split of every protein
                               segment (0 or 1: one lane per atom); replicas_per_cta * split *
                               atoms must fit one CTA. The energies' FP32 summation order depends
                               on it (results within the parity tolerance of each other). */
  int threads;              /* CTA size (multiple of 32, <= 256); 0: the smallest that holds
                               replicas_per_cta replicas of every complex. With threads > 0 each
                               complex gets as many replicas as fill the CTA (at most
                               replicas_per_cta when that is > 0): a ragged batch keeps its
                               lanes busy whatever its ligands' sizes. */
  int replicas_per_lane;    /* 0 or 1: a thread holds one lane; 2: a thread holds the same
                               atom of two replicas (the plain Monte Carlo, init and pose
                               evaluation launches; split 1, every ligand conformer with the same
                               atom types), sharing each protein point's loads and pair
                               parameters, on half as many threads. Energies are bit-identical
                               to one replica per lane. */
} gd_tile;

/* Per-replica Monte Carlo state (checkpoint unit). */
typedef struct {
  float movematrix_old[6];
  gd_energy energy_old;
  gd_replica replica;
  int n_accept;             /* accepted MC moves */
  int n_exchange;           /* accepted temperature swaps involving this slot */
} gd_replica_state;

typedef struct gd_ctx gd_ctx;

/* ---- host-side parameter preparation (reference L2, src/util.C) ---- */

/* OptimizeEnepara (src/util.C:717-760). */
int gd_fold_enepara(const gd_enepara_raw *raw, gd_enepara *out);
/* SetTemperature (src/util.C:797-840): geometric ladder, minus_beta = -1/T. */
int gd_set_temperature(int num_temp, float floor_temp, float ceiling_temp, gd_temp *out);
/* SetReplica (src/util.C:842-861): flat index n_tmp*n_lig*p + n_lig*t + l. */
int gd_set_replica(int n_prt, int n_tmp, int n_lig, gd_replica *out);

/* ---- context lifetime ---- */

/* Copies every input to the device. Replaces Run's allocations and cudaMemcpyToSymbol
 * calls (src/run.cu:57-246). Complex k's replicas occupy the global index range
 * [offset_k, offset_k + n_prt*n_tmp*n_lig), offsets in the order given. */
int gd_create(const gd_enepara *ff, const gd_complex_desc *complexes, int n_complexes,
              const gd_mc_params *mc, int device, gd_ctx **out);
/* Frees the context (Run's cudaFree calls, src/run.cu:250-283). The device buffers gd_create
 * made come from one memory pool per device that keeps freed memory for the next context of
 * the process (no unmapping on the way out, no mapping on the way in). */
int gd_destroy(gd_ctx *ctx);
/* Returns the memory the device's context pool holds without a live context to the driver
 * (no reference counterpart). */
int gd_release_memory(int device);
int gd_num_replicas(const gd_ctx *ctx, int *n_rep);
int gd_replica_offset(const gd_ctx *ctx, int complex_index, int *offset);
/* Tile of the fused kernel for one complex (-1: all); one CTA size per context. */
int gd_set_tile(gd_ctx *ctx, int complex_index, const gd_tile *tile);
int gd_get_tile(const gd_ctx *ctx, int complex_index, gd_tile *tile);
/* replicas per CTA the tile gives complex k (differs between complexes in fill mode) */
int gd_get_replicas_per_cta(const gd_ctx *ctx, int complex_index, int *replicas);
/* Autotuner: times each candidate tile by Monte Carlo steps of every replica (gd_mc_run
 * without records or trace; an exchange interval per launch, fewer for batches where one step
 * takes over 2 ms), `repeats` launches each, from a copy of the chain state that is put back
 * afterwards (the chains are left as they were); applies the fastest to every complex and
 * returns it with its mean time per step (ms) in ms_out[i] per candidate (may be null). */
int gd_autotune(gd_ctx *ctx, const gd_tile *candidates, int n_candidates, int repeats,
                gd_tile *best, float *ms_out);
/* Independent replica chains that gd_mc_run_fused (default 1) and the delayed-acceptance loops
 * (default 3) run concurrently on separate streams of one CUDA graph: a chain is a contiguous
 * range of (complex, protein conformer) blocks, so chains share no replica or exchange group,
 * and one chain's kernels fill the other's last wave and launch gaps. Results do not depend on
 * the numbers. */
int gd_set_concurrency(gd_ctx *ctx, int plain_chains, int da_chains);
/* RNG stream id of a complex (default: its index in the batch). Draws depend only on
 * (seed, stream, complex-local replica, step), so a complex run alone with the stream id it
 * has in a batch reproduces its batched trajectory. */
int gd_set_rng_stream(gd_ctx *ctx, int complex_index, int stream);
/* Limit (ns) of every bounded device wait; a wait that runs out ends the kernel with
 * GD_ERR_TIMEOUT from gd_sync. Default 2 s. */
int gd_set_wait_timeout(gd_ctx *ctx, long long timeout_ns);

/* ---- the Monte Carlo path ---- */

/* MonteCarlo_Init_d + ResetCounter_d + InitAcs_d (src/kernel_cuda_l1_montecarlo.cu:12-67,
 * src/kernel_cuda_l1_resetcounter.cu:12-22, src/kernel_cuda_l3_util.cu:16-23): energy of
 * the initial pose, contact reference map from each complex's first replica, step-0 record. */
int gd_mc_init(gd_ctx *ctx);
/* ResetCounter_d (src/kernel_cuda_l1_resetcounter.cu:12-22). */
int gd_reset_records(gd_ctx *ctx, int rep_begin, int rep_end);
/* MonteCarlo_d (src/kernel_cuda_l1_montecarlo.cu:72-127): steps_per_exchange steps for
 * replicas rep_begin..rep_end (inclusive); record step numbers are s1 + s2 + s3. */
int gd_mc_run(gd_ctx *ctx, int rep_begin, int rep_end, int s1, int s2);
/* ExchangeReplicas_d (src/kernel_cuda_l1_exchangereplicas.cu:7-137); mode_l is accepted
 * for signature parity and ignored (the reference only implements mode_l = 4). */
int gd_exchange(gd_ctx *ctx, int mode_l, int mode_t);
/* The reference's per-dump loop body (src/kernel_cuda_lancher_siglegpu.cu:25-32) over
 * n_steps steps from step s1, captured once into a CUDA graph and replayed:
 * gd_mc_run + (if exchange) gd_exchange with mode_t = !((s2 / steps_per_exchange) % 2), s2 the
 * interval's first step within its dump window (s mod steps_per_dump), so a window may be run
 * in several calls. The exchange runs inside the Monte Carlo kernel (the last replica of each
 * group to finish the interval exchanges the group), one launch per interval. */
int gd_mc_run_fused(gd_ctx *ctx, int s1, int n_steps, int exchange);
int gd_sync(gd_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order or time work on it. */
int gd_get_stream(gd_ctx *ctx, void **stream);

/* ---- results ---- */

/* Copies LigRecord-identical records (capacity steps_per_dump + 1 must equal
 * GD_STEPS_PER_DUMP + 1) for rep_begin..rep_end into host[0..]. */
int gd_get_records(gd_ctx *ctx, gd_lig_record *host, int rep_begin, int rep_end);
/* Same data for any record capacity: the first `cap` (1..steps_per_dump + 1) records of each
 * replica, steps[(r - rep_begin) * cap + i], and next_ptr[r - rep_begin]; a cap just above the
 * largest gd_get_record_counts value copies only the filled rows. */
int gd_get_records_raw(gd_ctx *ctx, gd_record_step *steps, int *next_ptr, int rep_begin,
                       int rep_end, int cap);
/* Records held per replica (next_ptr) for rep_begin..rep_end. */
int gd_get_record_counts(gd_ctx *ctx, int *next_ptr, int rep_begin, int rep_end);
/* The records downloaded while the run proceeds, instead of all at the end (the reference
 * copies the whole LigRecord array after each dump window, src/kernel_cuda_lancher_siglegpu.cu:
 * 36-46). From this call on, every call that writes records (gd_mc_init, gd_mc_run,
 * gd_mc_run_fused, gd_sur_collect, gd_da_run) also has a host worker thread copy, on its own
 * CUDA stream and while the next work runs, the record rows written so far into
 * steps[r * cap + i] (all replicas, the first `cap` records each; pageable or pinned memory,
 * which must stay valid until streaming stops). gd_records_stream_flush waits for the copies
 * of everything queued so far and returns the counts (next_ptr[n_rep]); the buffer then holds
 * what gd_get_records_raw with the same cap would return. gd_reset_records and gd_mc_init
 * flush first (read the window before resetting it). steps = NULL flushes and stops. */
int gd_records_stream(gd_ctx *ctx, gd_record_step *steps, int cap);
int gd_records_stream_flush(gd_ctx *ctx, int *next_ptr);
/* One dump window's records copied out while the next window runs (the reference copies its
 * LigRecord array after each dump window and waits, src/kernel_cuda_lancher_siglegpu.cu:36-46):
 * the first `cap` rows of every replica are snapshotted on the device in stream order (calls
 * that follow, gd_reset_records included, may overwrite them), and a host thread copies the
 * filled rows into steps[r * m + i] (m = min(cap, the largest count); any host memory of at
 * least n_rep * cap rows) and the counts into next_ptr[n_rep]. Returns at once;
 * gd_records_wait returns m in *rows once the copy is done, and neither array may be read or
 * freed before. A second call first waits for the first. */
int gd_get_records_async(gd_ctx *ctx, gd_record_step *steps, int *next_ptr, int cap);
int gd_records_wait(gd_ctx *ctx, int *rows);
int gd_get_etotal(gd_ctx *ctx, float *etotal, int rep_begin, int rep_end);
int gd_get_replicas(gd_ctx *ctx, gd_replica *replicas, int rep_begin, int rep_end);
int gd_get_state(gd_ctx *ctx, gd_replica_state *state, int rep_begin, int rep_end);
int gd_set_state(gd_ctx *ctx, const gd_replica_state *state, int rep_begin, int rep_end);
/* Device-side error word of the last kernels (0 when clean). */
int gd_get_device_error(gd_ctx *ctx, int *code);

/* Energy (9 normalized terms, weighted total, cms, rmsd) of n_poses poses given as
 * movematrix[6] each, for one (complex, protein conformer, ligand conformer).
 * cms is measured against the complex's contact reference (built by gd_mc_init). */
int gd_eval_energy(gd_ctx *ctx, int complex_index, int prt_conf, int lig_conf,
                   const float *movematrix, int n_poses, gd_energy *out);
/* CalcEnergy_d + CalcMcc_d + CalcRmsd_d (src/kernel_cuda_l2_calcenergy.cu:19-360,
 * src/kernel_cuda_l2_calcmcc.cu:148-206, src/kernel_cuda_l2_calcrmsd.cu:1-36) on given placed
 * coordinates, as the reference's kernels read them from Ligand.coord_new: pose i's atoms at
 * xyz[(i * lna + atom) * 3 + {0, 1, 2}] and its centre (coord_new.center, which gives dst) at
 * center[i * 3 + {0, 1, 2}], lab frame; rmsd is taken against conformer lig_conf's reference
 * pose. Same output as gd_eval_energy; placing movematrix poses with gd_place_ligand and their
 * centres movematrix[0..2] + the conformer's centre gives gd_eval_energy's results bit for bit. */
int gd_eval_energy_xyz(gd_ctx *ctx, int complex_index, int prt_conf, int lig_conf,
                       const float *xyz, const float *center, int n_poses, gd_energy *out);

/* Pose energies like gd_eval_energy, for callers that cannot allocate device memory when
 * they need the result (a framework that owns the whole device pool, a callback or
 * real-time context where cudaMalloc and its implicit synchronisation are not allowed).
 * No counterpart in the reference. d_movematrix (n_poses x 6 floats) and d_out (n_poses
 * gd_energy) are DEVICE pointers the caller owns; the call allocates nothing: its work queue
 * and tile list live in one fixed device array of the library, sized for at most
 * GD_NOALLOC_MAX_POSES poses (larger n_poses returns GD_ERR_CAPACITY, a negative one
 * GD_ERR_INVALID). The call only enqueues work on the context's stream; gd_sync (or a stream
 * sync) makes d_out ready. gd_create looks up that array's device address once per device,
 * so the call itself loads and allocates nothing. Every call in the process shares the
 * array, so calls whose kernels overlap on the GPU (two contexts on different streams) race:
 * serialise them. */
#define GD_NOALLOC_MAX_POSES 16384
int gd_eval_energy_noalloc(gd_ctx *ctx, int complex_index, int prt_conf, int lig_conf,
                           const float *d_movematrix, int n_poses, gd_energy *d_out);

/* Laboratory-frame ligand coordinates of n_poses poses (movematrix[6] each) of one ligand
 * conformer: xyz[(pose * lna + atom) * 3 + {0, 1, 2}], placed on the device by the transform
 * the Monte Carlo kernel applies. Replaces PlaceLigand (src/util.C:457-502) as the trace tool
 * calls it (src/trace.C:104-105); n_poses = 0 is a no-op. */
int gd_place_ligand(gd_ctx *ctx, int complex_index, int lig_conf, const float *movematrix,
                    int n_poses, float *xyz);

/* Per-step trace for bit-exact replay: when enabled, gd_mc_run logs for each replica and
 * step the proposal's total energy and the accept flag; trace[(r * max_steps) + s]. */
int gd_trace_enable(gd_ctx *ctx, int max_steps);
int gd_trace_get(gd_ctx *ctx, float *e_new_total, int *accepted, int *n_steps);

/* ---- learned energy surrogate and delayed acceptance (no reference counterpart) ----
 *
 * A 64 -> H -> H -> H -> 1 SiLU MLP of the total energy (pose translation and rotation, a
 * learned embedding per (complex, protein conformer, ligand conformer), per-pocket features)
 * with BF16 weights/activations on the tensor cores and FP32 accumulation, FP32 master
 * weights and Adam. It is the first stage of a delayed-acceptance Metropolis step; the exact
 * energy decides on every surviving proposal with the corrected ratio, so the stationary
 * distribution is the plain method's. */

typedef struct {
  int hidden;               /* hidden width, multiple of 16 (default 256) */
  int embedding;            /* 1: learned conformer embedding (32 wide) */
  float lr;                 /* Adam learning rate (default 1e-3) */
  int batch;                /* training rows per Adam step (default 8192) */
  long long sample_cap;     /* training samples kept (ring; default 16M) */
  float fallback_accept;    /* a complex whose stage-2 acceptance over the last window falls
                               below this reverts to plain MC (0: never) */
  long long fallback_window;/* surviving proposals per complex between decisions */
  uint64_t seed;            /* weight init and batch draws */
  int split;                /* protein split of the exact stage (gd_tile.split); 0: chosen per
                               gd_da_run from the surrogate stage's pass rate (1 when every
                               proposal survives, up to the CTA's limit when few do) */
  int pad;
} gd_sur_params;

/* per-complex counters since gd_sur_create / the last gd_sur_train */
typedef struct {
  long long proposed;       /* proposals with the surrogate stage on */
  long long passed;         /* ... surviving the surrogate stage (exact evaluations) */
  long long accepted;       /* ... accepted by the exact stage */
  long long plain;          /* proposals handled as plain Metropolis (stage off) */
  long long plain_accepted;
  double rmse;              /* surrogate error against the exact energy over evaluations */
  long long n_err;
  int active;               /* surrogate stage currently on */
  int pad;
} gd_sur_stats;

void gd_sur_default_params(gd_sur_params *p);
int gd_sur_create(gd_ctx *ctx, const gd_sur_params *p);
/* n_steps plain Monte Carlo steps from step s1 (the trajectory of gd_mc_run_fused with the
 * same arguments), each proposal's features and exact energy appended to the sample ring */
int gd_sur_collect(gd_ctx *ctx, int s1, int n_steps, int exchange);
/* iterations Adam steps on batches drawn from the samples; losses[i] (normalised MSE) when
 * not null; re-activates the surrogate stage of every complex */
int gd_sur_train(gd_ctx *ctx, int iterations, float *losses);
/* delayed-acceptance steps (the loop of gd_mc_run_fused, graph-captured); afterwards the
 * fallback controller switches off the stage of complexes below fallback_accept */
int gd_da_run(gd_ctx *ctx, int s1, int n_steps, int exchange);
int gd_sur_get_stats(gd_ctx *ctx, gd_sur_stats *per_complex);
int gd_sur_set_active(gd_ctx *ctx, int complex_index, int active);
/* surrogate energies of n poses (movematrix[6] each) of one conformer pair */
int gd_sur_predict(gd_ctx *ctx, int complex_index, int prt_conf, int lig_conf,
                   const float *movematrix, int n_poses, float *energy);
/* normalisation of the targets (E = mu + sigma * network output), valid samples */
int gd_sur_info(gd_ctx *ctx, float *mu, float *sigma, long long *n_samples);
/* protein split the last gd_da_run's exact stage ran with (gd_sur_params.split) */
int gd_sur_split(gd_ctx *ctx, int *split);
/* decision trace of gd_da_run: per replica and step the surrogate energy of the proposal,
 * its exact energy (NaN when the surrogate stage rejected it) and the outcome
 * (0 stage-1 reject, 1 stage-2 reject, 2 accept); index r * max_steps + (step - step0) */
int gd_da_trace_enable(gd_ctx *ctx, int step0, int max_steps);
int gd_da_trace_get(gd_ctx *ctx, float *s_new, float *e_new, int *outcome);

/* The network alone (gradient checks, offline training). x: rows x 64 features (row-major;
 * the embedding columns 7..38 are taken from the table for rows with conf >= 0). */
typedef struct gd_mlp gd_mlp;
int gd_mlp_create(int device, int hidden, int n_embedding, uint64_t seed, gd_mlp **out);
int gd_mlp_destroy(gd_mlp *net);
int gd_mlp_num_params(gd_mlp *net, long long *n);
/* flat parameter vector: W1 [64][H], b1, W2 [H][H], b2, W3 [H][H], b3, w4 [H], b4 (+3 pad),
 * embedding [n_embedding][32] */
int gd_mlp_get_params(gd_mlp *net, float *theta, long long n);
int gd_mlp_set_params(gd_mlp *net, const float *theta, long long n);
int gd_mlp_forward(gd_mlp *net, const float *x, const int *conf, int rows, float *y);
/* forward + mean squared error against t + backward; loss and the gradient (may be null) */
int gd_mlp_backward(gd_mlp *net, const float *x, const int *conf, const float *t, int rows,
                    float *loss, float *grad);
int gd_mlp_adam(gd_mlp *net, float lr);

const char *gd_last_error_string(void);
const char *gd_version(void);

/* Measured FP32 FMA throughput of `device` in TFLOP/s (2 FLOP per FMA, best of `repeats`):
 * the roofline denominator for the FP32-bound pair-energy kernel. No reference counterpart. */
int gd_probe_fp32_peak(int device, int repeats, double *tflops);

/* ---------------------------------------------------------------------------------------
 * Post-Monte-Carlo clustering (post_mc, src/post_mc.C:40-101): k-means over the 9 energy
 * terms of the records, clusterByKmeans (src/util.C:1801-1880) over seq_kmeans
 * (src/seq_kmeans.c), for n_seg independent segments at once on the device.
 * Segment s is objects[seg_off[s] .. seg_off[s+1]-1] (each `dim` = 9 floats) with k[s]
 * clusters; a segment with fewer objects than k[s] is not clustered (each object is its own
 * cluster, in order, as the reference returns them). Each segment is shuffled by the seeded
 * permutation of gd_kmeans_permutation (the reference shuffles without a seed), its first k
 * shuffled objects seed the centres, Lloyd passes run while more than `threshold` of its
 * objects change cluster and at most max_iter + 1 passes, and the representative of each
 * cluster is its last member in shuffled order. Clusters are numbered per segment from
 * cluster base = sum over earlier segments of min(k, n):
 *   membership[n]   cluster of each object within its segment (original object order)
 *   medoid[total]   object index of each cluster's representative, -1 if it ended empty
 *   size[total]     members of each cluster
 *   passes[n_seg]   Lloyd passes per segment (the reference's loop_iterations)
 * Any output may be NULL. */
int gd_kmeans(int device, const float *objects, int n, int dim, const int *seg_off, int n_seg,
              const int *k, uint64_t seed, float threshold, int max_iter, int *membership,
              int *medoid, int *size, int *passes);
/* The shuffle of segment `segment` of n objects: perm[i] = the object at shuffled position i
 * (a 4-round Feistel permutation with cycle walking, keys from seed and segment). */
int gd_kmeans_permutation(uint64_t seed, int segment, int n, int *perm);

#ifdef __cplusplus
}
#endif

#endif /* GEAUXDOCK_B200_H */
