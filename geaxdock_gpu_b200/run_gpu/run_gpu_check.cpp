/*
 * run_gpu_check.cpp -- the reference's docking flow up to its Run call (src/dock.C:97-191),
 * linked with run_gpu.cpp, for checking the drop-in from the reference's side.
 *
 * It loads a complex with the reference's own loaders (loadLigand, loadProtein, loadLHM,
 * loadEnePara; src/load.C), folds it with the reference's host preparation
 * (OptimizeLigand/Protein/Psp/Kde/Mcs/Enepara, InitLigCoord, SetTemperature, SetReplica,
 * SetMcLog; src/util.C), calls Run exactly as src/dock.C:191 does, and writes what Run
 * returned: the per-replica record lists and the McLog figures.
 *
 * The reference's main parses its options with Boost (absent here); this driver takes the
 * same ones by name: --pdb --sdf --ff --para --id --nt --floor_temp --ceiling_temp --nc -t -r
 * (defaults of src/dock.C:32-43), and --out for the records file:
 *   int32 n_rep, int32 count[n_rep], then every replica's LigRecordSingleStep rows in order.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "dock.h"
#include "load.h"
#include "run.h"
#include "size.h"
#include "util.h"

static const char *arg(int argc, char **argv, const char *key, const char *def) {
  for (int i = 1; i + 1 < argc; ++i)
    if (!strcmp(argv[i], key)) return argv[i + 1];
  return def;
}

int main(int argc, char **argv) {
  McPara mcpara = McPara();
  ExchgPara exchgpara = ExchgPara();
  InputFiles inputfiles = InputFiles();
  mcpara.steps_total = STEPS_PER_DUMP;
  mcpara.steps_per_dump = STEPS_PER_DUMP;
  mcpara.steps_per_exchange = atoi(arg(argc, argv, "--nc", "10"));
  exchgpara.floor_temp = (float)atof(arg(argc, argv, "--floor_temp", "0.3"));
  exchgpara.ceiling_temp = (float)atof(arg(argc, argv, "--ceiling_temp", "0.3"));
  exchgpara.num_temp = atoi(arg(argc, argv, "--nt", "1"));
  const float ts = (float)atof(arg(argc, argv, "-t", "0.02"));
  const float rs = (float)atof(arg(argc, argv, "-r", "0.08"));
  for (int i = 0; i < 3; ++i) {
    mcpara.move_scale[i] = ts;
    mcpara.move_scale[i + 3] = rs;
  }
  inputfiles.prt_file.path = arg(argc, argv, "--pdb", "");
  inputfiles.lig_file.path = arg(argc, argv, "--sdf", "");
  inputfiles.lhm_file.path = arg(argc, argv, "--ff", "");
  inputfiles.enepara_file.path = arg(argc, argv, "--para", "");
  inputfiles.lhm_file.ligand_id = arg(argc, argv, "--id", "");
  inputfiles.lig_file.molid = "MOLID";
  const char *out = arg(argc, argv, "--out", "records.bin");

  McLog *mclog = new McLog();
  Ligand0 *lig0 = new Ligand0[MAXEN2];
  Protein0 *prt0 = new Protein0[MAXEN1];
  Psp0 *psp0 = new Psp0();
  Kde0 *kde0 = new Kde0();
  Mcs0 *mcs0 = new Mcs0[MAXPOS];
  EnePara0 *enepara0 = new EnePara0();
  loadLigand(&inputfiles, lig0);
  loadProtein(&inputfiles.prt_file, prt0);
  loadLHM(&inputfiles.lhm_file, psp0, kde0, mcs0);
  loadEnePara(&inputfiles.enepara_file, enepara0);

  ComplexSize cs;
  cs.n_prt = inputfiles.prt_file.conf_total;
  cs.n_tmp = exchgpara.num_temp;
  cs.n_lig = inputfiles.lig_file.conf_total;
  cs.n_rep = cs.n_lig * cs.n_prt * cs.n_tmp;
  cs.lna = inputfiles.lig_file.lna;
  cs.pnp = inputfiles.prt_file.pnp;
  cs.pnk = kde0->pnk;
  cs.pos = inputfiles.lhm_file.pos;

  Ligand *lig = new Ligand[cs.n_rep];
  Protein *prt = new Protein[cs.n_prt];
  Psp *psp = new Psp();
  Kde *kde = new Kde();
  Mcs *mcs = new Mcs[cs.pos];
  EnePara *enepara = new EnePara();
  Temp *temp = new Temp[cs.n_tmp];
  Replica *replica = new Replica[cs.n_rep];
  OptimizeLigand(lig0, lig, cs);
  OptimizeProtein(prt0, prt, enepara0, lig0, cs);
  OptimizePsp(psp0, psp, lig, prt);
  OptimizeKde(kde0, kde);
  OptimizeMcs(mcs0, mcs, cs);
  OptimizeEnepara(enepara0, enepara);
  InitLigCoord(lig, cs);
  SetTemperature(temp, &exchgpara);
  SetReplica(replica, lig, cs);
  SetMcLog(mclog);

  std::map<int, std::vector<LigRecordSingleStep> > multi_reps_records;
  Run(lig, prt, psp, kde, mcs, enepara, temp, replica, &mcpara, mclog, multi_reps_records, cs);

  FILE *f = fopen(out, "wb");
  if (!f) {
    perror(out);
    return 2;
  }
  std::vector<int> count(cs.n_rep, 0);
  for (int r = 0; r < cs.n_rep; ++r)
    if (multi_reps_records.count(r)) count[r] = (int)multi_reps_records[r].size();
  fwrite(&cs.n_rep, sizeof(int), 1, f);
  fwrite(count.data(), sizeof(int), cs.n_rep, f);
  for (int r = 0; r < cs.n_rep; ++r)
    if (count[r])
      fwrite(multi_reps_records[r].data(), sizeof(LigRecordSingleStep), count[r], f);
  fclose(f);
  printf("{\"n_rep\": %d, \"steps_total\": %d, \"ar\": %.6f, \"ac_mc\": %d, "
         "\"ac_temp_exchg\": %d, \"t0\": %.6f, \"t1\": %.6f}\n",
         cs.n_rep, mclog->steps_total, mclog->ar, mclog->ac_mc, mclog->ac_temp_exchg,
         mclog->t0, mclog->t1);
  return 0;
}
