/*
 * refpin_main.cpp -- runs the reference's own code on the CPU to pin the oracle.
 * TEST INFRASTRUCTURE ONLY; built by oracle/refpin/Makefile into oracle/_ref/refpin from the
 * reference sources where they lie (nothing of the reference is copied into this tree).
 *
 * Input: a real complex (PDB, SDF, .ff, paras) read by the reference's loaders
 * (src/load.C:157,931,1355,1477) and folded by its host prep (src/util.C:264-861).
 * Output (one .gdfx container, named arrays):
 *   - the folded complex as the product's gd_complex_desc arrays + gd_enepara / raw params;
 *   - energies of random poses computed by the reference's Move_d + CalcEnergy_d +
 *     CalcMcc_d (src/kernel_cuda_l2_*.cu);
 *   - a Monte Carlo trajectory driven step by step through the reference's device
 *     functions in MonteCarlo_d's order (src/kernel_cuda_l1_montecarlo.cu:95-117) with
 *     ExchangeReplicas_d (src/kernel_cuda_l1_exchangereplicas.cu) between intervals, fed
 *     with the product's Philox stream (uniform moves, reference style).
 */
#include "refpin_shim.h"

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <ctime>
#include <list>
#include <map>
#include <string>
#include <vector>

#include "dock.h"
#include "load.h"
#include "util.h"
#include "kernel_cuda.cuh"
#include "kernel_cuda.cu"

#include "bench_complex.h"

#include "../../include/geauxdock_b200.h"
#include "../../geaxdock_gpu_b200/csrc/gd_numerics.h"

static_assert(sizeof(EnePara) == sizeof(gd_enepara), "EnePara layout");
static_assert(sizeof(EnePara0) == sizeof(gd_enepara_raw), "EnePara0 layout");
static_assert(sizeof(Energy) == sizeof(gd_energy), "Energy layout");
static_assert(sizeof(LigRecordSingleStep) == sizeof(gd_record_step), "record layout");
static_assert(sizeof(LigRecord) == sizeof(gd_lig_record), "LigRecord layout");
static_assert(sizeof(Temp) == sizeof(gd_temp), "Temp layout");
/* field by field: the record structs that the reference's dumps and readers use */
#define GD_SAME_OFFSET(R, G, f) static_assert(offsetof(R, f) == offsetof(G, f), #R "." #f)
GD_SAME_OFFSET(Replica, gd_replica, idx_rep);
GD_SAME_OFFSET(Replica, gd_replica, idx_prt);
GD_SAME_OFFSET(Replica, gd_replica, idx_tmp);
GD_SAME_OFFSET(Replica, gd_replica, idx_lig);
GD_SAME_OFFSET(Energy, gd_energy, e);
GD_SAME_OFFSET(Energy, gd_energy, cms);
GD_SAME_OFFSET(Energy, gd_energy, rmsd);
GD_SAME_OFFSET(LigRecordSingleStep, gd_record_step, replica);
GD_SAME_OFFSET(LigRecordSingleStep, gd_record_step, energy);
GD_SAME_OFFSET(LigRecordSingleStep, gd_record_step, movematrix);
GD_SAME_OFFSET(LigRecordSingleStep, gd_record_step, step);
GD_SAME_OFFSET(LigRecord, gd_lig_record, step);
GD_SAME_OFFSET(LigRecord, gd_lig_record, next_ptr);
static_assert(sizeof(((LigRecord *)0)->step) == sizeof(((gd_lig_record *)0)->step),
              "LigRecord steps per dump");
#undef GD_SAME_OFFSET

/* ---------------- named-array container ---------------- */
struct Writer {
  FILE *f;
  explicit Writer(const char *path) {
    f = fopen(path, "wb");
    if (!f) { perror(path); exit(2); }
    fwrite("GDFX1\n", 1, 6, f);
  }
  ~Writer() { fclose(f); }
  void put(const char *name, char dtype, std::vector<uint64_t> dims, const void *data,
           size_t elem) {
    uint32_t n = (uint32_t)strlen(name);
    fwrite(&n, 4, 1, f);
    fwrite(name, 1, n, f);
    fwrite(&dtype, 1, 1, f);
    uint32_t nd = (uint32_t)dims.size();
    fwrite(&nd, 4, 1, f);
    uint64_t count = 1;
    for (auto d : dims) { fwrite(&d, 8, 1, f); count *= d; }
    fwrite(data, elem, count, f);
  }
  void f32(const char *n, std::vector<uint64_t> d, const float *p) { put(n, 'f', d, p, 4); }
  void i32(const char *n, std::vector<uint64_t> d, const int *p) { put(n, 'i', d, p, 4); }
};

static const char *arg(int argc, char **argv, const char *key, const char *def) {
  for (int i = 1; i + 1 < argc; ++i)
    if (!strcmp(argv[i], key)) return argv[i + 1];
  return def;
}

/* Move_d emulation: threads 5..1 write their dims, thread 0 writes dim 0, builds the
 * rotation and places every atom (TperB = 1). */
static void move_all(Ligand *lig, const float p[6]) {
  for (int b = 5; b >= 0; --b) Move_d(b, lig, p[b]);
}

/* Accept_d emulation: thread 0 draws and copies the energy, threads 1..5 copy their dims. */
static void accept_all(Ligand *lig, float mybeta, int rep) {
  for (int b = 0; b < 6; ++b) Accept_d(b, lig, mybeta, rep);
}

/* Timing mode: the reference's own MonteCarlo_d step functions (Move_d, CalcEnergy_d,
 * CalcMcc_d, Accept_d, RecordLigand_d, src/kernel_cuda_l1_montecarlo.cu:95-117) on a complex
 * given as product arrays (--bench file.gdfx), replicas [--r0, --r1), --steps steps each, one
 * thread; prints "replica_steps seconds accepted". Moves: the container's move kind drawn from
 * the product's Philox stream (stream 0, replica r, step) and handed to Move_d as its p, which
 * the reference scales by move_scale (src/kernel_cuda_l2_move.cu:27): uniform p = 2u - 1 as
 * MonteCarlo_d draws it, or Gaussian p = z (Box-Muller), the configured N(0, scale) moves. */
static int bench_main(int argc, char **argv) {
  Reader rd(arg(argc, argv, "--bench", ""));
  BenchComplex bc;
  if (!read_bench_complex(rd, &bc)) {
    fprintf(stderr, "cannot read the --bench container\n");
    return 2;
  }
  const ComplexSize cs = bc.cs;
  const int r0 = atoi(arg(argc, argv, "--r0", "0"));
  const int r1 = std::min(cs.n_rep, atoi(arg(argc, argv, "--r1", "1")));
  const int steps = atoi(arg(argc, argv, "--steps", "10"));
  const uint64_t seed = strtoull(arg(argc, argv, "--seed", "42"), 0, 10);
  const int move_kind = bc.move_kind;
  float move_scale[6];
  for (int k = 0; k < 6; ++k) move_scale[k] = bc.move_scale[k];
  Ligand *lig = bc.lig;
  Protein *prt = bc.prt;
  Psp *psp = bc.psp;
  Kde *kde = bc.kde;
  Mcs *mcs = bc.mcs;
  EnePara *ep = bc.ep;
  Temp *temp = bc.temp;
  Replica *replica = bc.replica;
  ConfusionMatrix *ref = (ConfusionMatrix *)calloc(1, sizeof(ConfusionMatrix));
  LigRecord *rec = (LigRecord *)calloc(cs.n_rep, sizeof(LigRecord)); /* pages of r0..r1 only */
  float *etotal = (float *)calloc(cs.n_rep, sizeof(float));
  LigMoveVector *lmv = (LigMoveVector *)calloc(cs.n_rep, sizeof(LigMoveVector));
  int *acs = (int *)calloc(cs.n_rep, sizeof(int));
  curandState rng_state[1];
  prt_dc = prt; psp_dc = psp; kde_dc = kde; mcs_dc = mcs; enepara_dc = ep; temp_dc = temp;
  lig_dc = lig; replica_dc = replica; etotal_dc = etotal; ligmovevector_dc = lmv;
  ligrecord_dc = rec; acs_temp_exchg_dc = acs; ref_matrix_dc = ref; curandstate_dc = rng_state;
  steps_per_exchange_dc = steps; steps_per_dump_dc = STEPS_PER_DUMP;
  steps_total_dc = STEPS_PER_DUMP;
  move_scale_dc = move_scale;
  enepara_lj0_dc = ep->lj0; enepara_lj1_dc = ep->lj1; enepara_el0_dc = ep->el0;
  enepara_el1_dc = ep->el1; enepara_a1_dc = ep->a1; enepara_b1_dc = ep->b1;
  enepara_kde2_dc = ep->kde2; enepara_kde3_dc = ep->kde3;
  n_lig_dc = cs.n_lig; n_prt_dc = cs.n_prt; n_tmp_dc = cs.n_tmp; n_rep_dc = cs.n_rep;
  lna_dc = cs.lna; pnp_dc = cs.pnp; pnk_dc = cs.pnk; pos_dc = cs.pos;
  /* contact reference from replica 0 (as MonteCarlo_Init_d), then the initial energies */
  InitRefMatrix_d(0, &lig[replica[0].idx_rep], &prt[replica[0].idx_prt]);
  for (int r = r0; r < r1; ++r) {
    Ligand *ml = &lig[replica[r].idx_rep];
    const Protein *mp = &prt[replica[r].idx_prt];
    CalcEnergy_d(0, ml, mp);
    CalcMcc_d(0, ml, mp);
    ml->energy_old = ml->energy_new;
    rec[r].next_ptr = 0;
  }
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  long acc = 0;
  for (int r = r0; r < r1; ++r) {
    Ligand *ml = &lig[replica[r].idx_rep];
    const Protein *mp = &prt[replica[r].idx_prt];
    const float mybeta = temp[replica[r].idx_tmp].minus_beta;
    for (int step = 0; step < steps; ++step) {
      const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
      const gd_u32x4 a = gd_philox4x32_10((uint32_t)r, (uint32_t)step, 0u, GD_RNG_MOVE, k0, k1);
      const gd_u32x4 b = gd_philox4x32_10((uint32_t)r, (uint32_t)step, 0u, GD_RNG_MOVE2, k0, k1);
      float pm[6];
      if (move_kind == GD_MOVE_GAUSSIAN) {
        gd_box_muller(a.v[0], a.v[1], &pm[0], &pm[1]);
        gd_box_muller(a.v[2], a.v[3], &pm[2], &pm[3]);
        gd_box_muller(b.v[0], b.v[1], &pm[4], &pm[5]);
      } else {
        const uint32_t wd[6] = {a.v[0], a.v[1], a.v[2], a.v[3], b.v[0], b.v[1]};
        for (int k = 0; k < 6; ++k) pm[k] = gd_sym11(wd[k]);
      }
      move_all(ml, pm);
      CalcEnergy_d(0, ml, mp);
      CalcMcc_d(0, ml, mp);
      g_shim_uniforms.push_back(gd_u01(b.v[2]));
      accept_all(ml, mybeta, r);
      if (rec[r].next_ptr >= STEPS_PER_DUMP) rec[r].next_ptr = 0; /* keep appending in place */
      RecordLigand_d(0, 0, step, r, 0, ml);
      acc += ml->is_move_accepted;
    }
  }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  const double sec = (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
  printf("%ld %.6f %ld\n", (long)(r1 - r0) * steps, sec, acc);
  return 0;
}

/* the reference's k-means module (src/kmeans.h:68,71) */
extern "C" float **seq_kmeans(float **, int, int, int, float, int *, int *);
extern "C" float **file_read(int, char *, int *, int *);

/* --kmeans file --k N --out f.gdfx: the run of cluster_test (src/cluster_test.C:23-66) --
 * the reference's file_read of a text data file (an id, then the coordinates, per line) and
 * its seq_kmeans with threshold 0.001 -- written as objects, membership, centres, loops. */
static int kmeans_main(int argc, char **argv) {
  char path[4096];
  snprintf(path, sizeof(path), "%s", arg(argc, argv, "--kmeans", ""));
  const int k = atoi(arg(argc, argv, "--k", "10"));
  int n = 0, d = 0;
  float **obj = file_read(0, path, &n, &d);
  if (!obj || n < k || k < 1) { fprintf(stderr, "cannot read %s\n", path); return 2; }
  std::vector<float> objects(obj[0], obj[0] + (size_t)n * d);
  std::vector<int> mem(n);
  int loops = 0;
  float **cen = seq_kmeans(obj, d, n, k, 0.001f, mem.data(), &loops);
  {
    Writer w(arg(argc, argv, "--out", "kmeans.gdfx"));
    w.put("objects", 'f', {(uint64_t)n, (uint64_t)d}, objects.data(), 4);
    w.put("membership", 'i', {(uint64_t)n}, mem.data(), 4);
    w.put("centres", 'f', {(uint64_t)k, (uint64_t)d}, cen[0], 4);
    w.put("loops", 'i', {1}, &loops, 4);
  }
  free(obj[0]);
  free(obj);
  free(cen[0]);
  free(cen);
  return 0;
}

/* --states records.bin --out table.txt: the reference's printStates (src/util.C:1504-1545) on
 * the LigRecordSingleStep array of a raw file (the product's gd_record_step layout). */
static int states_main(int argc, char **argv) {
  const char *in = arg(argc, argv, "--states", "");
  FILE *f = fopen(in, "rb");
  if (!f) { perror(in); return 2; }
  std::vector<LigRecordSingleStep> steps;
  LigRecordSingleStep s;
  while (fread(&s, sizeof(s), 1, f) == 1) steps.push_back(s);
  fclose(f);
  std::string out = arg(argc, argv, "--out", "states.txt");
  printStates(steps, out);
  return 0;
}

int main(int argc, char **argv) {
  if (strcmp(arg(argc, argv, "--bench", ""), "")) return bench_main(argc, argv);
  if (strcmp(arg(argc, argv, "--kmeans", ""), "")) return kmeans_main(argc, argv);
  if (strcmp(arg(argc, argv, "--states", ""), "")) return states_main(argc, argv);
  InputFiles in = InputFiles();
  in.prt_file.path = arg(argc, argv, "--pdb", "");
  in.lig_file.path = arg(argc, argv, "--sdf", "");
  in.lhm_file.path = arg(argc, argv, "--ff", "");
  in.enepara_file.path = arg(argc, argv, "--paras", "");
  in.lhm_file.ligand_id = arg(argc, argv, "--id", "");
  in.lig_file.molid = "MOLID";
  const char *out = arg(argc, argv, "--out", "refpin.gdfx");
  const int nt = atoi(arg(argc, argv, "--nt", "4"));
  const float floor_t = (float)atof(arg(argc, argv, "--floor", "0.5"));
  const float ceil_t = (float)atof(arg(argc, argv, "--ceil", "2.0"));
  const int nc = atoi(arg(argc, argv, "--nc", "10"));
  const int nex = atoi(arg(argc, argv, "--nex", "3"));
  const uint64_t seed = strtoull(arg(argc, argv, "--seed", "42"), 0, 10);
  const float ts = (float)atof(arg(argc, argv, "--ts", "0.02"));
  const float rs = (float)atof(arg(argc, argv, "--rs", "0.08"));
  const int n_poses = atoi(arg(argc, argv, "--poses", "64"));

  /* ---- load and fold (dock.C:97-181) ---- */
  Ligand0 *lig0 = new Ligand0[MAXEN2];
  Protein0 *prt0 = new Protein0[MAXEN1];
  Psp0 *psp0 = (Psp0 *)calloc(1, sizeof(Psp0));
  Kde0 *kde0 = new Kde0;
  Mcs0 *mcs0 = new Mcs0[MAXPOS];
  EnePara0 *ep0 = (EnePara0 *)calloc(1, sizeof(EnePara0));
  loadLigand(&in, lig0);
  loadProtein(&in.prt_file, prt0);
  loadLHM(&in.lhm_file, psp0, kde0, mcs0);
  loadEnePara(&in.enepara_file, ep0);

  ComplexSize cs;
  cs.n_prt = in.prt_file.conf_total;
  cs.n_tmp = nt;
  cs.n_lig = in.lig_file.conf_total;
  cs.n_rep = cs.n_lig * cs.n_prt * cs.n_tmp;
  cs.lna = in.lig_file.lna;
  cs.pnp = in.prt_file.pnp;
  cs.pnk = kde0->pnk;
  cs.pos = in.lhm_file.pos;
  fprintf(stderr, "n_lig %d n_prt %d n_tmp %d lna %d pnp %d pnk %d pos %d\n", cs.n_lig,
          cs.n_prt, cs.n_tmp, cs.lna, cs.pnp, cs.pnk, cs.pos);

  Ligand *lig = (Ligand *)calloc(cs.n_rep, sizeof(Ligand));
  Protein *prt = (Protein *)calloc(cs.n_prt, sizeof(Protein));
  Psp *psp = (Psp *)calloc(1, sizeof(Psp));
  Kde *kde = (Kde *)calloc(1, sizeof(Kde));
  Mcs *mcs = (Mcs *)calloc(cs.pos, sizeof(Mcs));
  EnePara *ep = (EnePara *)calloc(1, sizeof(EnePara));
  Temp *temp = (Temp *)calloc(cs.n_tmp, sizeof(Temp));
  Replica *replica = (Replica *)calloc(cs.n_rep, sizeof(Replica));
  OptimizeLigand(lig0, lig, cs);
  OptimizeProtein(prt0, prt, ep0, lig0, cs);
  OptimizePsp(psp0, psp, lig, prt);
  OptimizeKde(kde0, kde);
  OptimizeMcs(mcs0, mcs, cs);
  OptimizeEnepara(ep0, ep);
  InitLigCoord(lig, cs);
  ExchgPara xp;
  xp.floor_temp = floor_t;
  xp.ceiling_temp = ceil_t;
  xp.num_temp = nt;
  SetTemperature(temp, &xp);
  SetReplica(replica, lig, cs);

  /* --trace rows.txt: the trace program's loop (src/trace.C:90-122) -- the rows of a
   * trajectory file as its read2D reads them (src/load.C:80-105), each placed by PlaceLigand
   * (conformer int(row[1]), move vector row[2..7]) and written by replaceLigandCoords
   * (src/util.C:457-545) -- every row's SDF text into `out`, each after a line ">>>> row k". */
  const char *trace_rows = arg(argc, argv, "--trace", "");
  if (trace_rows[0]) {
    TraceFile tf;
    tf.path = trace_rows;
    std::vector<std::vector<float> > rows = read2D(&tf);
    FILE *fo = fopen(out, "w");
    if (!fo) { perror(out); return 2; }
    int k = 0;
    for (auto &row : rows) {
      if (row.size() < 8 || (int)row[1] < 0 || (int)row[1] >= cs.n_lig) break;
      float mv[6];
      for (int i = 0; i < 6; ++i) mv[i] = row[2 + i];
      Ligand *my = &lig[(int)row[1]];
      PlaceLigand(my, mv);
      std::list<std::string> sdf = replaceLigandCoords(&in.lig_file, my);
      fprintf(fo, ">>>> row %d\n", k++);
      for (auto &line : sdf) fprintf(fo, "%s\n", line.c_str());
    }
    fclose(fo);
    return 0;
  }

  Writer w(out);
  {
    const int L = cs.lna, P = cs.pnp, NL = cs.n_lig, NP = cs.n_prt;
    int sizes[8] = {cs.n_lig, cs.n_prt, cs.n_tmp, cs.lna, cs.pnp, cs.pnk, cs.pos, 0};
    w.i32("sizes", {8}, sizes);
    std::vector<float> lx(NL * L), ly(NL * L), lz(NL * L), lc(NL * L), lcen(NL * 3);
    std::vector<int> lt(NL * L), ln(NL * L);
    for (int c = 0; c < NL; ++c) {
      for (int a = 0; a < L; ++a) {
        lx[c * L + a] = lig[c].coord_orig.x[a];
        ly[c * L + a] = lig[c].coord_orig.y[a];
        lz[c * L + a] = lig[c].coord_orig.z[a];
        lt[c * L + a] = lig[c].t[a];
        lc[c * L + a] = lig[c].c[a];
        ln[c * L + a] = lig[c].n[a];
      }
      for (int k = 0; k < 3; ++k) lcen[c * 3 + k] = lig[c].coord_orig.center[k];
    }
    w.f32("lig_x", {(uint64_t)NL, (uint64_t)L}, lx.data());
    w.f32("lig_y", {(uint64_t)NL, (uint64_t)L}, ly.data());
    w.f32("lig_z", {(uint64_t)NL, (uint64_t)L}, lz.data());
    w.f32("lig_center", {(uint64_t)NL, 3}, lcen.data());
    w.i32("lig_t", {(uint64_t)NL, (uint64_t)L}, lt.data());
    w.f32("lig_c", {(uint64_t)NL, (uint64_t)L}, lc.data());
    w.i32("lig_n", {(uint64_t)NL, (uint64_t)L}, ln.data());
    std::vector<float> px(NP * P), py(NP * P), pz(NP * P), pe(NP * P), ph(NP * P);
    std::vector<int> pt(NP * P), pc(NP * P), ps(NP * P), pf(NP * P);
    int max_s = 0;
    for (int c = 0; c < NP; ++c)
      for (int p = 0; p < P; ++p) {
        px[c * P + p] = prt[c].x[p];
        py[c * P + p] = prt[c].y[p];
        pz[c * P + p] = prt[c].z[p];
        pt[c * P + p] = prt[c].t[p];
        pc[c * P + p] = prt[c].c[p];
        pe[c * P + p] = prt[c].ele[p];
        ps[c * P + p] = prt[c].seq3r[p];
        pf[c * P + p] = prt[c].c0_and_d12_or_c2[p];
        ph[c * P + p] = prt[c].hpp[p];
        if (prt[c].seq3r[p] > max_s) max_s = prt[c].seq3r[p];
      }
    w.f32("prt_x", {(uint64_t)NP, (uint64_t)P}, px.data());
    w.f32("prt_y", {(uint64_t)NP, (uint64_t)P}, py.data());
    w.f32("prt_z", {(uint64_t)NP, (uint64_t)P}, pz.data());
    w.i32("prt_t", {(uint64_t)NP, (uint64_t)P}, pt.data());
    w.i32("prt_c", {(uint64_t)NP, (uint64_t)P}, pc.data());
    w.f32("prt_ele", {(uint64_t)NP, (uint64_t)P}, pe.data());
    w.i32("prt_seq3r", {(uint64_t)NP, (uint64_t)P}, ps.data());
    w.i32("prt_hflag", {(uint64_t)NP, (uint64_t)P}, pf.data());
    w.f32("prt_hpp", {(uint64_t)NP, (uint64_t)P}, ph.data());
    w.f32("pocket_center", {3}, prt[0].pocket_center);
    const int ld = max_s + 1;
    std::vector<float> pspv((size_t)MAXTP2 * ld);
    for (int i = 0; i < MAXTP2; ++i)
      for (int j = 0; j < ld; ++j) pspv[(size_t)i * ld + j] = psp->psp[i][j];
    w.f32("psp", {MAXTP2, (uint64_t)ld}, pspv.data());
    w.f32("kde_x", {(uint64_t)cs.pnk}, kde->x);
    w.f32("kde_y", {(uint64_t)cs.pnk}, kde->y);
    w.f32("kde_z", {(uint64_t)cs.pnk}, kde->z);
    w.i32("kde_t", {(uint64_t)cs.pnk}, kde->t);
    std::vector<float> mx(cs.pos * MAXMCS), my(cs.pos * MAXMCS), mz(cs.pos * MAXMCS), mt(cs.pos);
    for (int m = 0; m < cs.pos; ++m) {
      for (int j = 0; j < MAXMCS; ++j) {
        mx[m * MAXMCS + j] = mcs[m].x[j];
        my[m * MAXMCS + j] = mcs[m].y[j];
        mz[m * MAXMCS + j] = mcs[m].z[j];
      }
      mt[m] = mcs[m].tcc;
    }
    w.f32("mcs_x", {(uint64_t)cs.pos, MAXMCS}, mx.data());
    w.f32("mcs_y", {(uint64_t)cs.pos, MAXMCS}, my.data());
    w.f32("mcs_z", {(uint64_t)cs.pos, MAXMCS}, mz.data());
    w.f32("mcs_tcc", {(uint64_t)cs.pos}, mt.data());
    w.f32("temp", {(uint64_t)cs.n_tmp, 3}, (const float *)temp); /* order is an int */
    w.f32("enepara", {sizeof(EnePara) / 4}, (const float *)ep);
    w.f32("enepara_raw", {sizeof(EnePara0) / 4}, (const float *)ep0);
  }

  /* ---- device-side globals (run.cu:110-242) ---- */
  const float zero6[6] = {0, 0, 0, 0, 0, 0};
  float move_scale[6] = {ts, ts, ts, rs, rs, rs};
  ConfusionMatrix *ref = (ConfusionMatrix *)calloc(1, sizeof(ConfusionMatrix));
  LigRecord *rec = (LigRecord *)calloc(cs.n_rep, sizeof(LigRecord));
  float *etotal = (float *)calloc(cs.n_rep, sizeof(float));
  LigMoveVector *lmv = (LigMoveVector *)calloc(cs.n_rep, sizeof(LigMoveVector));
  int *acs = (int *)calloc(cs.n_rep, sizeof(int));
  curandState rng_state[1];
  prt_dc = prt; psp_dc = psp; kde_dc = kde; mcs_dc = mcs; enepara_dc = ep; temp_dc = temp;
  lig_dc = lig; replica_dc = replica; etotal_dc = etotal; ligmovevector_dc = lmv;
  ligrecord_dc = rec; acs_temp_exchg_dc = acs; ref_matrix_dc = ref; curandstate_dc = rng_state;
  steps_per_exchange_dc = nc; steps_per_dump_dc = STEPS_PER_DUMP; steps_total_dc = STEPS_PER_DUMP;
  move_scale_dc = move_scale;
  enepara_lj0_dc = ep->lj0; enepara_lj1_dc = ep->lj1; enepara_el0_dc = ep->el0;
  enepara_el1_dc = ep->el1; enepara_a1_dc = ep->a1; enepara_b1_dc = ep->b1;
  enepara_kde2_dc = ep->kde2; enepara_kde3_dc = ep->kde3;
  n_lig_dc = cs.n_lig; n_prt_dc = cs.n_prt; n_tmp_dc = cs.n_tmp; n_rep_dc = cs.n_rep;
  lna_dc = cs.lna; pnp_dc = cs.pnp; pnk_dc = cs.pnk; pos_dc = cs.pos;

  /* ---- MonteCarlo_Init_d, emulated (src/kernel_cuda_l1_montecarlo.cu:12-67) ---- */
  for (int r = 0; r < cs.n_rep; ++r) rec[r].next_ptr = 0;
  std::vector<float> init_e((size_t)cs.n_rep * 12);
  for (int r = 0; r < cs.n_rep; ++r) {
    Ligand *ml = &lig[replica[r].idx_rep];
    const Protein *mp = &prt[replica[r].idx_prt];
    if (r == 0) InitRefMatrix_d(0, ml, mp);
    CalcEnergy_d(0, ml, mp);
    CalcMcc_d(0, ml, mp);
    ml->energy_new.rmsd = 0.0f; /* CalcRmsd_d is not emulated (its value is 0 at the start) */
    ml->energy_old = ml->energy_new;
    ml->is_move_accepted = 1;
    RecordLigand_d(0, 0, 0, r, 0, ml);
    memcpy(&init_e[(size_t)r * 12], &ml->energy_old, 48);
  }
  w.f32("init_energy", {(uint64_t)cs.n_rep, 12}, init_e.data());
  {
    std::vector<int> rm((size_t)cs.lna * cs.pnp);
    for (int l = 0; l < cs.lna; ++l)
      for (int p = 0; p < cs.pnp; ++p) rm[(size_t)l * cs.pnp + p] = ref->matrix[l][p];
    w.i32("ref_matrix", {(uint64_t)cs.lna, (uint64_t)cs.pnp}, rm.data());
  }

  /* ---- random poses through Move_d + CalcMcc_d + CalcEnergy_d ---- */
  {
    std::vector<float> pose((size_t)n_poses * 6), pe((size_t)n_poses * 12);
    std::vector<float> pxyz((size_t)n_poses * 3 * cs.lna), pcen((size_t)n_poses * 3);
    std::vector<int> pidx((size_t)n_poses * 2);
    float saved_scale[6];
    memcpy(saved_scale, move_scale, sizeof(saved_scale));
    memcpy(move_scale, zero6, sizeof(saved_scale));
    Ligand scratch;
    for (int i = 0; i < n_poses; ++i) {
      const gd_u32x4 a = gd_philox4x32_10((uint32_t)i, 7u, 0u, 99u, 12345u, 678u);
      const gd_u32x4 b = gd_philox4x32_10((uint32_t)i, 7u, 1u, 99u, 12345u, 678u);
      const int ip = (int)(a.v[0] % (uint32_t)cs.n_prt), il = (int)(a.v[1] % (uint32_t)cs.n_lig);
      float mm[6];
      mm[0] = 2.0f * gd_sym11(a.v[2]);
      mm[1] = 2.0f * gd_sym11(a.v[3]);
      mm[2] = 2.0f * gd_sym11(b.v[0]);
      mm[3] = 3.14159265f * gd_sym11(b.v[1]);
      mm[4] = 3.14159265f * gd_sym11(b.v[2]);
      mm[5] = 3.14159265f * gd_sym11(b.v[3]);
      scratch = lig[il];
      memcpy(scratch.movematrix_old, mm, sizeof(mm));
      const float p0[6] = {0, 0, 0, 0, 0, 0};
      move_all(&scratch, p0);
      /* CalcEnergy_d stores an uninitialised Energy over energy_new (its cms/rmsd are never
       * set, src/kernel_cuda_l2_calcenergy.cu:331,353), so CalcMcc_d runs after it here. */
      CalcEnergy_d(0, &scratch, &prt[ip]);
      CalcMcc_d(0, &scratch, &prt[ip]);
      scratch.energy_new.rmsd = 0.0f;
      memcpy(&pose[(size_t)i * 6], mm, sizeof(mm));
      memcpy(&pxyz[((size_t)i * 3 + 0) * cs.lna], scratch.coord_new.x, 4 * cs.lna);
      memcpy(&pxyz[((size_t)i * 3 + 1) * cs.lna], scratch.coord_new.y, 4 * cs.lna);
      memcpy(&pxyz[((size_t)i * 3 + 2) * cs.lna], scratch.coord_new.z, 4 * cs.lna);
      memcpy(&pcen[(size_t)i * 3], scratch.coord_new.center, 12);
      memcpy(&pe[(size_t)i * 12], &scratch.energy_new, 48);
      pidx[i * 2 + 0] = ip;
      pidx[i * 2 + 1] = il;
    }
    memcpy(move_scale, saved_scale, sizeof(saved_scale));
    w.f32("pose_mm", {(uint64_t)n_poses, 6}, pose.data());
    w.i32("pose_idx", {(uint64_t)n_poses, 2}, pidx.data());
    w.f32("pose_energy", {(uint64_t)n_poses, 12}, pe.data());
    w.f32("pose_xyz", {(uint64_t)n_poses, 3, (uint64_t)cs.lna}, pxyz.data());
    w.f32("pose_center", {(uint64_t)n_poses, 3}, pcen.data());
  }

  /* ---- trajectory: MonteCarlo_d order, then ExchangeReplicas_d ---- */
  const int n_rep = cs.n_rep, n_steps = nex * nc;
  std::vector<float> t_mm_old((size_t)n_rep * n_steps * 6), t_mm_new((size_t)n_rep * n_steps * 6);
  std::vector<float> t_u((size_t)n_rep * n_steps), t_e((size_t)n_rep * n_steps * 12);
  std::vector<int> t_acc((size_t)n_rep * n_steps);
  std::vector<float> x_etotal((size_t)nex * n_rep);
  std::vector<int> x_before((size_t)nex * n_rep), x_after((size_t)nex * n_rep);
  std::vector<int> x_acs((size_t)nex * n_rep);
  for (int e = 0; e < nex; ++e) {
    const int s2 = e * nc;
    for (int r = 0; r < n_rep; ++r) {
      Ligand *ml = &lig[replica[r].idx_rep];
      const Protein *mp = &prt[replica[r].idx_prt];
      const float mybeta = temp[replica[r].idx_tmp].minus_beta;
      for (int s3 = 0; s3 < nc; ++s3) {
        const int step = s2 + s3;
        const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
        const gd_u32x4 a = gd_philox4x32_10((uint32_t)r, (uint32_t)step, 0u, GD_RNG_MOVE, k0, k1);
        const gd_u32x4 b = gd_philox4x32_10((uint32_t)r, (uint32_t)step, 0u, GD_RNG_MOVE2, k0, k1);
        const float p[6] = {gd_sym11(a.v[0]), gd_sym11(a.v[1]), gd_sym11(a.v[2]),
                            gd_sym11(a.v[3]), gd_sym11(b.v[0]), gd_sym11(b.v[1])};
        const float u = gd_u01(b.v[2]);
        const size_t ti = (size_t)r * n_steps + step;
        memcpy(&t_mm_old[ti * 6], ml->movematrix_old, 24);
        move_all(ml, p);
        CalcEnergy_d(0, ml, mp);
        CalcMcc_d(0, ml, mp);
        ml->energy_new.rmsd = 0.0f;
        g_shim_uniforms.push_back(u);
        accept_all(ml, mybeta, r);
        RecordLigand_d(0, 0, step, r, 0, ml);
        memcpy(&t_mm_new[ti * 6], ml->movematrix_new, 24);
        memcpy(&t_e[ti * 12], &ml->energy_new, 48);
        t_u[ti] = u;
        t_acc[ti] = ml->is_move_accepted;
      }
      etotal[r] = ml->energy_old.e[MAXWEI - 1];
    }
    for (int r = 0; r < n_rep; ++r) {
      x_etotal[(size_t)e * n_rep + r] = etotal[r];
      x_before[(size_t)e * n_rep + r] = replica[r].idx_tmp;
    }
    const int mode_t = !((s2 / nc) % 2);
    for (int pp = 0; pp < cs.n_prt; ++pp)
      for (int l = 0; l < cs.n_lig; ++l) {
        const int maxpair = nt / 2 - (nt % 2 == 0) * (mode_t == 1);
        for (int pair = 0; pair < maxpair; ++pair)
          g_shim_uniforms.push_back(
              gd_draw_exchange(seed, 0u, (uint32_t)(pp * cs.n_lig + l), (uint32_t)e, (uint32_t)pair));
      }
    ExchangeReplicas_d(4, mode_t);
    for (int r = 0; r < n_rep; ++r) {
      x_after[(size_t)e * n_rep + r] = replica[r].idx_tmp;
      x_acs[(size_t)e * n_rep + r] = acs[r];
    }
  }
  w.f32("traj_mm_old", {(uint64_t)n_rep, (uint64_t)n_steps, 6}, t_mm_old.data());
  w.f32("traj_mm_new", {(uint64_t)n_rep, (uint64_t)n_steps, 6}, t_mm_new.data());
  w.f32("traj_u", {(uint64_t)n_rep, (uint64_t)n_steps}, t_u.data());
  w.f32("traj_energy", {(uint64_t)n_rep, (uint64_t)n_steps, 12}, t_e.data());
  w.i32("traj_accept", {(uint64_t)n_rep, (uint64_t)n_steps}, t_acc.data());
  w.f32("xch_etotal", {(uint64_t)nex, (uint64_t)n_rep}, x_etotal.data());
  w.i32("xch_before", {(uint64_t)nex, (uint64_t)n_rep}, x_before.data());
  w.i32("xch_after", {(uint64_t)nex, (uint64_t)n_rep}, x_after.data());
  w.i32("xch_acs_ref", {(uint64_t)nex, (uint64_t)n_rep}, x_acs.data());
  {
    std::vector<int> np(n_rep);
    for (int r = 0; r < n_rep; ++r) np[r] = rec[r].next_ptr;
    w.i32("rec_next_ptr", {(uint64_t)n_rep}, np.data());
    int params[6] = {nc, nex, (int)seed, 0, 0, 0};
    w.i32("run_params", {6}, params);
    w.f32("move_scale", {6}, move_scale);
  }
  if (g_shim_underflow || !g_shim_uniforms.empty()) {
    fprintf(stderr, "uniform stream mismatch: underflow %ld leftover %zu\n", g_shim_underflow,
            g_shim_uniforms.size());
    return 3;
  }
  fprintf(stderr, "wrote %s\n", out);
  return 0;
}
