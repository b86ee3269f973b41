/*
 * run_gpu.cpp -- the reference's host entry point `Run` (src/run.h:8-19, src/run.cu:33-288)
 * on top of the B200 engine's C ABI (include/geauxdock_b200.h).
 *
 * A maintainer of the reference links this file and libgeauxdock_b200.so in place of
 * src/run.cu: src/dock.C and everything it calls (loaders, folds, post_mc, printStates) stay
 * as they are. It is compiled against the reference's own headers (dock.h, run.h, size.h,
 * toggle.h), so the struct layouts it reads are the reference's.
 *
 * What Run does here, in the reference's order:
 *   - the reference's SoA structs (after OptimizeLigand/Protein/Psp/Kde/Mcs/Enepara,
 *     InitLigCoord, SetTemperature, SetReplica) become one gd_complex_desc; gd_create copies
 *     them to the device (src/run.cu:57-246: the cudaMalloc + cudaMemcpyToSymbol block);
 *   - gd_mc_init = ResetCounter_d + MonteCarlo_Init_d (src/kernel_cuda_lancher_siglegpu.cu:
 *     7-8);
 *   - dump windows of steps_per_dump steps until the gathered records reach
 *     steps_per_dump * n_rep (the launcher's while loop, :15-58): gd_reset_records after the
 *     first window, the window's MonteCarlo_d calls -- and ExchangeReplicas_d when the
 *     reference's IS_EXCHANGE toggle is on -- as one graph-captured gd_mc_run_fused call,
 *     then every replica's filled record rows appended to multi_reps_records[replica];
 *   - McLog: compute time t0, wall time t1, steps_total, acceptance ratio ar (:35, 60-69), and
 *     the per-temperature-slot exchange counts acs_temp_exchg that ExchangeReplicas_d keeps
 *     (src/kernel_cuda_l1_exchangereplicas.cu:65-66).
 *
 * Differences, all deliberate: the RNG is Philox4x32-10 keyed by GD_SEED (environment;
 * unset: the time, as the reference seeds curand from time(NULL), src/run.cu:64), so a run
 * can be repeated; the device is GD_DEVICE (default 0; the reference uses NGPU devices from
 * 0). Moves are the reference's uniform form (Move_d). Records are always kept (the
 * reference's IS_OUTPUT == 0 setting would stop RecordLigand_d and loop forever); with
 * IS_OUTPUT == 0 and a non-empty hdf_path, each window's LigRecord array is also written as
 * raw bytes to <hdf_path>.bin (no HDF5 library is linked). Errors print the library's message
 * and exit(1), as the reference's CUDA checks do (src/include/yeah/cudautil.h:81-97).
 */
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <map>
#include <vector>

#include "dock.h"
#include "run.h"
#include "size.h"
#include "toggle.h"

#include "geauxdock_b200.h"

static_assert(sizeof(EnePara) == sizeof(gd_enepara), "EnePara layout");
static_assert(sizeof(Energy) == sizeof(gd_energy), "Energy layout");
static_assert(sizeof(Replica) == sizeof(gd_replica), "Replica layout");
static_assert(sizeof(LigRecordSingleStep) == sizeof(gd_record_step), "record layout");
static_assert(sizeof(LigRecord) == sizeof(gd_lig_record), "LigRecord layout");
static_assert(sizeof(Temp) == sizeof(gd_temp), "Temp layout");

namespace {

void check(int rc, const char *what) {
  if (rc != GD_OK) {
    fprintf(stderr, "Run: %s failed: %s\n", what, gd_last_error_string());
    exit(1);
  }
}

double now_s() {
  using clk = std::chrono::steady_clock;
  return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

uint64_t seed_from_env() {
  const char *s = getenv("GD_SEED");
  if (s && *s) return strtoull(s, nullptr, 10);
  return (uint64_t)time(nullptr);
}

int device_from_env() {
  const char *s = getenv("GD_DEVICE");
  return (s && *s) ? atoi(s) : 0;
}

/* Host copies of one complex in the C ABI's conformer-major layout. Ligand conformer k is
 * lig[k]: SetReplica (src/util.C:842-861) fills lig[flat] from lig[idx_lig], and the first
 * n_lig flat indices (protein 0, temperature 0) are the conformers themselves. */
struct Complex {
  std::vector<float> lx, ly, lz, lc, lq, px, py, pz, pe, ph, mx, my, mz, mt;
  std::vector<int> lt, ln, pt, pc, ps, pf;
  gd_complex_desc d{};

  Complex(const Ligand *lig, const Protein *prt, const Psp *psp, const Kde *kde,
          const Mcs *mcs, const Temp *temp, const ComplexSize &cs) {
    const int L = cs.lna, P = cs.pnp, NL = cs.n_lig, NP = cs.n_prt, M = cs.pos;
    lx.resize(NL * L); ly.resize(NL * L); lz.resize(NL * L); lq.resize(NL * L);
    lt.resize(NL * L); ln.resize(NL * L); lc.resize(NL * 3);
    for (int k = 0; k < NL; ++k) {
      for (int i = 0; i < L; ++i) {
        lx[k * L + i] = lig[k].coord_orig.x[i];
        ly[k * L + i] = lig[k].coord_orig.y[i];
        lz[k * L + i] = lig[k].coord_orig.z[i];
        lt[k * L + i] = lig[k].t[i];
        lq[k * L + i] = lig[k].c[i];
        ln[k * L + i] = lig[k].n[i];
      }
      for (int a = 0; a < 3; ++a) lc[k * 3 + a] = lig[k].coord_orig.center[a];
    }
    px.resize(NP * P); py.resize(NP * P); pz.resize(NP * P); pe.resize(NP * P);
    ph.resize(NP * P); pt.resize(NP * P); pc.resize(NP * P); ps.resize(NP * P);
    pf.resize(NP * P);
    for (int p = 0; p < NP; ++p)
      for (int i = 0; i < P; ++i) {
        const int o = p * P + i;
        px[o] = prt[p].x[i];
        py[o] = prt[p].y[i];
        pz[o] = prt[p].z[i];
        pt[o] = prt[p].t[i];
        pc[o] = prt[p].c[i];
        pe[o] = prt[p].ele[i];
        ps[o] = prt[p].seq3r[i];
        pf[o] = prt[p].c0_and_d12_or_c2[i];
        ph[o] = prt[p].hpp[i];
      }
    mx.resize(M * MAXMCS); my.resize(M * MAXMCS); mz.resize(M * MAXMCS); mt.resize(M);
    for (int m = 0; m < M; ++m) {
      std::copy(mcs[m].x, mcs[m].x + MAXMCS, &mx[m * MAXMCS]);
      std::copy(mcs[m].y, mcs[m].y + MAXMCS, &my[m * MAXMCS]);
      std::copy(mcs[m].z, mcs[m].z + MAXMCS, &mz[m * MAXMCS]);
      mt[m] = mcs[m].tcc;
    }
    d.n_lig = NL; d.n_prt = NP; d.n_tmp = cs.n_tmp; d.lna = L; d.pnp = P;
    d.pnk = kde->pnk; d.pos = M;
    d.lig_x = lx.data(); d.lig_y = ly.data(); d.lig_z = lz.data(); d.lig_center = lc.data();
    d.lig_t = lt.data(); d.lig_c = lq.data(); d.lig_n = ln.data();
    d.prt_x = px.data(); d.prt_y = py.data(); d.prt_z = pz.data(); d.prt_t = pt.data();
    d.prt_c = pc.data(); d.prt_ele = pe.data(); d.prt_seq3r = ps.data();
    d.prt_hflag = pf.data(); d.prt_hpp = ph.data();
    d.pocket_center = prt[0].pocket_center;
    d.psp = &psp->psp[0][0];   /* Psp.psp[MAXLIG][MAXPRO], read at [ligand type][seq3r] */
    d.psp_ld = MAXPRO;
    d.kde_x = kde->x; d.kde_y = kde->y; d.kde_z = kde->z; d.kde_t = kde->t;
    d.mcs_x = mx.data(); d.mcs_y = my.data(); d.mcs_z = mz.data(); d.mcs_tcc = mt.data();
    d.mcs_ld = MAXMCS;
    d.temp = reinterpret_cast<const gd_temp *>(temp);
  }
};

}  // namespace

void Run(const Ligand *lig, const Protein *prt, const Psp *psp, const Kde *kde, const Mcs *mcs,
         const EnePara *enepara, const Temp *temp, const Replica *replica, const McPara *mcpara,
         McLog *mclog, map<int, vector<LigRecordSingleStep> > &multi_reps_records,
         const ComplexSize complexsize) {
  (void)replica; /* the replica layout is SetReplica's, which gd_create rebuilds the same way */
  const double t_start = now_s();
  const int n_rep = complexsize.n_rep;
  Complex cx(lig, prt, psp, kde, mcs, temp, complexsize);

  gd_mc_params mc{};
  mc.steps_per_exchange = mcpara->steps_per_exchange;
  mc.steps_per_dump = mcpara->steps_per_dump;
  for (int i = 0; i < 6; ++i) mc.move_scale[i] = mcpara->move_scale[i];
  mc.move_kind = GD_MOVE_UNIFORM;
  mc.record = 1;
  mc.seed = seed_from_env();

  gd_ctx *ctx = nullptr;
  check(gd_create(reinterpret_cast<const gd_enepara *>(enepara), &cx.d, 1, &mc,
                  device_from_env(), &ctx),
        "gd_create");
  check(gd_mc_init(ctx), "gd_mc_init");

  const long est_tot_rec = (long)mcpara->steps_per_dump * n_rep;
  printf("estimated total records: %ld\n", est_tot_rec);
  long have = 0;
  int s1 = 0;
  std::vector<int> nxt(n_rep);
  std::vector<gd_record_step> rows;
  while (have < est_tot_rec) {
    if (s1 != 0) check(gd_reset_records(ctx, 0, n_rep - 1), "gd_reset_records");
    const double t0 = now_s();
    check(gd_mc_run_fused(ctx, s1, mcpara->steps_per_dump, IS_EXCHANGE == 1 ? 1 : 0),
          "gd_mc_run_fused");
    check(gd_sync(ctx), "gd_sync");
    mclog->t0 += now_s() - t0;

    /* the filled record rows only (the reference copies the whole LigRecord array) */
    check(gd_get_record_counts(ctx, nxt.data(), 0, n_rep - 1), "gd_get_record_counts");
    const int cap = std::max(1, *std::max_element(nxt.begin(), nxt.end()));
    rows.resize((size_t)n_rep * cap);
    check(gd_get_records_raw(ctx, rows.data(), nxt.data(), 0, n_rep - 1, cap),
          "gd_get_records_raw");
    for (int r = 0; r < n_rep; ++r) {
      vector<LigRecordSingleStep> &v = multi_reps_records[r];
      const LigRecordSingleStep *src =
          reinterpret_cast<const LigRecordSingleStep *>(&rows[(size_t)r * cap]);
      v.insert(v.end(), src, src + nxt[r]);
      have += nxt[r];
    }
    printf("# points\t\t\t%ld\n", have);
    fflush(stdout);

#if IS_OUTPUT == 0
    if (mcpara->hdf_path[0] && mcpara->steps_per_dump == STEPS_PER_DUMP) {
      std::vector<gd_lig_record> dump(n_rep);
      check(gd_get_records(ctx, dump.data(), 0, n_rep - 1), "gd_get_records");
      char path[MAXSTRINGLENG + 8];
      snprintf(path, sizeof(path), "%s.bin", mcpara->hdf_path);
      FILE *f = fopen(path, "wb");
      if (!f || fwrite(dump.data(), sizeof(gd_lig_record), n_rep, f) != (size_t)n_rep) {
        fprintf(stderr, "Run: cannot write %s\n", path);
        exit(1);
      }
      fclose(f);
    }
#endif
    s1 += mcpara->steps_per_dump;
  }

  std::vector<gd_replica_state> st(n_rep);
  check(gd_get_state(ctx, st.data(), 0, n_rep - 1), "gd_get_state");
  check(gd_destroy(ctx), "gd_destroy");

  /* exchange counts per temperature slot, folded over (protein, ligand) conformers: the
   * counter ExchangeReplicas_d increments at acs_temp_exchg_dc[slot] */
  const int nt = complexsize.n_tmp, nl = complexsize.n_lig;
  long swaps = 0, accepted = 0;
  for (int t = 0; t < nt && t < MAXREP; ++t) mclog->acs_temp_exchg[t] = 0;
  for (int r = 0; r < n_rep; ++r) {
    const int t = (r % (nt * nl)) / nl;
    if (t < MAXREP) mclog->acs_temp_exchg[t] += st[r].n_exchange;
    swaps += st[r].n_exchange;
    accepted += st[r].n_accept;
  }
  mclog->ac_temp_exchg = (int)(swaps / 2);
  mclog->ac_mc = (int)accepted;
  mclog->t1 += now_s() - t_start;
  mclog->steps_total = s1;
  mclog->ar = (float)have / (float)((double)n_rep * s1);
}
