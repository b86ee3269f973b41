/*
 * refgpu_main.cu -- the reference's own GPU implementation timed on this machine's GPU (a
 * witness for the benchmark, not part of the product).
 * BENCHMARK INFRASTRUCTURE ONLY; built by oracle/refgpu/Makefile into oracle/_ref/refgpu_gd<GD>
 * from the reference's sources where they lie: its Run (src/run.cu:33-288) with every kernel it
 * includes (src/kernel_cuda.cu) compiled for sm_100a, linked with this driver and the
 * reference's host code.
 *
 * Input: a complex as the product's arrays (--bench file.gdfx, written by oracle/refbench.py),
 * turned into the reference's structs by bench_complex.h; then McPara (steps_per_exchange 10,
 * --dump steps per dump window, the container's move scales; the reference's moves are its
 * uniform U(-1, 1) times the scale, src/kernel_cuda_l1_montecarlo.cu:100), SetMcLog, and Run,
 * which loops over dump windows until the records reach steps_per_dump x n_rep
 * (src/kernel_cuda_lancher_siglegpu.cu:15-58) and times its kernel launches itself (McLog t0,
 * src/kernel_cuda_lancher_siglegpu.cu:35). Prints one JSON line with the reference's own
 * figures.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "dock.h"
#include "run.h"
#include "size.h"
#include "util.h"

#include "../refpin/bench_complex.h"

static const char *arg(int argc, char **argv, const char *key, const char *def) {
  for (int i = 1; i + 1 < argc; ++i)
    if (!strcmp(argv[i], key)) return argv[i + 1];
  return def;
}

int main(int argc, char **argv) {
  Reader rd(arg(argc, argv, "--bench", ""));
  BenchComplex b;
  if (!read_bench_complex(rd, &b)) {
    fprintf(stderr, "cannot read the --bench container\n");
    return 2;
  }
  McPara mcpara = McPara();
  mcpara.steps_per_exchange = 10;
  mcpara.steps_per_dump = atoi(arg(argc, argv, "--dump", "100"));
  mcpara.steps_total = mcpara.steps_per_dump;
  if (mcpara.steps_per_dump < 10 || mcpara.steps_per_dump > STEPS_PER_DUMP) return 2;
  for (int k = 0; k < 6; ++k) mcpara.move_scale[k] = b.move_scale[k];
  McLog *mclog = new McLog();
  SetMcLog(mclog);
  std::map<int, std::vector<LigRecordSingleStep> > records;
  Run(b.lig, b.prt, b.psp, b.kde, b.mcs, b.ep, b.temp, b.replica, &mcpara, mclog, records, b.cs);
  long n_rec = 0;
  for (auto &kv : records) n_rec += (long)kv.second.size();
  printf("{\"n_rep\": %d, \"steps_total\": %d, \"t0\": %.6f, \"t1\": %.6f, \"ar\": %.6f, "
         "\"records\": %ld, \"replica_steps_per_s\": %.3f, \"GD\": %d, \"BDx\": %d, "
         "\"BDy\": %d}\n",
         b.cs.n_rep, mclog->steps_total, mclog->t0, mclog->t1, mclog->ar, n_rec,
         (double)mclog->steps_total * b.cs.n_rep / mclog->t0, GD, BDx, BDy);
  return 0;
}
