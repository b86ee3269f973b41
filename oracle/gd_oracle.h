/*
 * gd_oracle.h -- CPU restatement of GeauxDock's Monte Carlo docking path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product (the geaxdock_gpu_b200 package or
 * its CUDA library) may link, load or call this code; only tests/, the smoke check and
 * the CPU-baseline leg of bench.py use it, as the checker and the reported baseline.
 *
 * What it restates (all paths relative to the reference project root):
 *   energy     src/kernel_cuda_l2_calcenergy.cu:19-360 (CalcEnergy_d), FP64 and FP32
 *   combine    src/kernel_cuda_l3_combineenergy.cu:23-37 (CombineEnergy_d, IS_OPT=0)
 *   move       src/kernel_cuda_l2_move.cu:21-80 (Move_d), src/util.C:457-500 (PlaceLigand)
 *   accept     src/kernel_cuda_l2_accept.cu:13-46 (Accept_d)
 *   exchange   src/kernel_cuda_l1_exchangereplicas.cu:27-77 (ExchangeReplicas_d)
 *   mcc        src/kernel_cuda_l2_calcmcc.cu:57-82,148-206 (InitRefMatrix_d, CalcMcc_d)
 *   rmsd       src/kernel_cuda_l2_calcrmsd.cu:1-36 (CalcRmsd_d, without its shared-memory overrun)
 *   records    src/kernel_cuda_l3_util.cu:74-106 (RecordLigand_d)
 *   init       src/kernel_cuda_l1_montecarlo.cu:12-67 (MonteCarlo_Init_d)
 *   step loop  src/kernel_cuda_l1_montecarlo.cu:72-127 (MonteCarlo_d), OpenMP over replicas
 *              as in src/unused/cpu_mic/montecarlo_cpu.C:29-44
 *   host folds src/util.C:717-760 (OptimizeEnepara), :797-840 (SetTemperature),
 *              :842-861 (SetReplica)
 *
 * Parity pin: tests compare this code with the reference's own kernel source compiled for
 * the CPU (oracle/refpin) on the reference's real 1a07C1 complex; the committed fixtures
 * under tests/golden/ come from that run.
 */
#ifndef GD_ORACLE_H
#define GD_ORACLE_H

#include <stdint.h>
#include "../include/geauxdock_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  double e[GD_MAXWEI];   /* normalized terms 0..8, weighted total at 9 */
  double raw[9];         /* per-term value before a*x+b (vdw..kde divided by lna, lhm, dst) */
  double mag[7];         /* sum of |contribution| / lna for terms 0..6 (conditioning scale) */
  double cms, rmsd;
  int64_t tp, fn, fp, tn;
  int64_t hits_hpc, hits_hdb, hits_psp, hits_kde, hits_mcs;  /* conditional-work counters */
} gdo_energy;

/* contact threshold: largest float d2 with sqrtf(d2) <= pmf0 (-1 when none) */
float gdo_contact_threshold(float pmf0);

/* Energy of the ligand atoms at FP32 lab coordinates x,y,z (lna each) and ligand centre
 * `center`, for protein conformer prt_conf of complex cx. refmap is [lna*pnp] contact
 * reference (or NULL: cms reported as 0). precision: 64 or 32. */
int gdo_energy_eval(const gd_enepara *ff, const gd_complex_desc *cx, int prt_conf,
                    int lig_conf, const float *x, const float *y, const float *z,
                    const float center[3], const uint8_t *refmap, int precision,
                    gdo_energy *out);

/* FP32 placement shared with the device (x = R x_orig + t + c_orig). */
void gdo_place_f32(const gd_complex_desc *cx, int lig_conf, const float mm[6], float *x,
                   float *y, float *z, float center[3]);
/* FP64 restatement of Move_d / PlaceLigand with libm sin/cos. */
void gdo_place_f64(const gd_complex_desc *cx, int lig_conf, const float mm[6], double *x,
                   double *y, double *z, double center[3]);
/* InitRefMatrix_d from the pose at movematrix 0 of (prt 0, lig 0). */
void gdo_ref_map(const gd_enepara *ff, const gd_complex_desc *cx, uint8_t *refmap);

/* Host folds. */
void gdo_fold_enepara(const gd_enepara_raw *raw, gd_enepara *out);
void gdo_set_temperature(int num_temp, float floor_temp, float ceiling_temp, gd_temp *out);

/* RNG / decision primitives (the shared Philox stream). */
void gdo_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                uint32_t out[4]);
float gdo_expf(float x);
float gdo_logf(float x);
void gdo_sincosf(float x, float *s, float *c);
void gdo_draw_steps(uint64_t seed, uint32_t stream, int move_kind, const float scale[6], int n,
                    const uint32_t *replica, const uint32_t *step, float *delta6, float *u);
void gdo_metropolis_batch(int n, const float *e_new, const float *e_old, const float *mb,
                          const float *u, int32_t *out);
float gdo_draw_exchange(uint64_t seed, uint32_t stream, uint32_t group, uint32_t call,
                        uint32_t pair);

/* ---- one complex's Monte Carlo chain set (MonteCarlo_Init_d / MonteCarlo_d /
 *      ExchangeReplicas_d restated) ---- */
typedef struct gdo_mc gdo_mc;
/* stream: the complex's RNG stream id (its index in a batch; 0 for a single complex). */
gdo_mc *gdo_mc_create(const gd_enepara *ff, const gd_complex_desc *cx, const gd_mc_params *mc,
                      int stream, int precision);
void gdo_mc_destroy(gdo_mc *m);
int gdo_mc_num_replicas(const gdo_mc *m);
void gdo_mc_init(gdo_mc *m);
/* n_steps steps from step s1 + s2 for every replica, OpenMP with nthreads (0: default). */
void gdo_mc_run(gdo_mc *m, int s1, int s2, int n_steps, int nthreads);
/* Same for replicas [r0, r1) only (bounded CPU-baseline samples). */
void gdo_mc_run_range(gdo_mc *m, int r0, int r1, int s1, int s2, int n_steps, int nthreads);
void gdo_mc_exchange(gdo_mc *m, int mode_t);
void gdo_mc_reset_records(gdo_mc *m);
void gdo_mc_get(const gdo_mc *m, gd_replica *replica, float *mm_old, gd_energy *e_old,
                float *etotal, int32_t *n_accept, int32_t *acs_exchange);
void gdo_mc_set(gdo_mc *m, const gd_replica *replica, const float *mm_old,
                const gd_energy *e_old, const float *etotal);
int gdo_mc_get_records(const gdo_mc *m, gd_record_step *steps, int32_t *next_ptr);
const uint8_t *gdo_mc_refmap(const gdo_mc *m);
int gdo_mc_exchange_calls(const gdo_mc *m);
void gdo_mc_set_exchange_calls(gdo_mc *m, int n);
/* Exchange restated over caller-owned arrays (for replaying device results). */
void gdo_exchange_apply(const gd_complex_desc *cx, uint64_t seed, int stream,
                        int exchange_call, int mode_t, gd_replica *replica, const float *etotal,
                        int32_t *acs_exchange);

int gdo_max_threads(void);

#ifdef __cplusplus
}
#endif

#endif
