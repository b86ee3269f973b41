"""The reference's `dock` program on this library:

    python -m geaxdock_gpu_b200.dock -p prt.pdb -l lig.sdf -s pocket.ff --para paras \\
        -i <complex id> -o out.csv [--nc 10] [--nt 1] [--floor_temp 0.3] [--ceiling_temp 0.3] \\
        [-t 0.02] [-r 0.08]

Same options, defaults and pipeline as src/dock.C:25-240: load and fold the inputs
(loaders.py), then the single-GPU run loop (src/kernel_cuda_lancher_siglegpu.cu:1-70): records
reset, MonteCarlo_Init, and dump windows of steps_per_dump steps (Monte Carlo steps with a
replica exchange every `nc` steps, temperature mode alternating) until the accepted-step
records of all replicas reach steps_per_dump x n_rep; then post_mc clustering (postmc.py) and
the table of the 500 representatives (printStates) in the --csv file, and a run summary.
Options of this implementation: --device, --seed (Monte Carlo and clustering), --dump-dir
(write every dump window's LigRecord array, records.py), --gaussian (Gaussian moves instead
of the reference's uniform ones), --surrogate (delayed acceptance with the learned surrogate,
trained on the first window's plain steps).
"""
from __future__ import annotations

import argparse
import sys
import time

import numpy as np

from . import abi, engine, loaders, postmc, records


def parse(argv=None):
    ap = argparse.ArgumentParser(prog="geaxdock_gpu_b200.dock", description="GeauxDock on B200")
    ap.add_argument("-p", "--pdb", required=True, help="protein path (PDB)")
    ap.add_argument("-l", "--sdf", required=True, help="ligand path (SDF)")
    ap.add_argument("-s", "--ff", required=True, help="force field path")
    ap.add_argument("--para", required=True, help="parameter file path")
    ap.add_argument("-i", "--id", required=True, help="complex id")
    ap.add_argument("-o", "--csv", required=True, help="trajectories")
    ap.add_argument("--nc", type=int, default=10, help="steps per exchange")
    ap.add_argument("--nt", type=int, default=1, help="number of temperatures")
    ap.add_argument("--ceiling_temp", type=float, default=0.3, help="ceiling temperature")
    ap.add_argument("--floor_temp", type=float, default=0.3, help="floor temperature")
    ap.add_argument("-t", type=float, default=0.02, help="translational scale")
    ap.add_argument("-r", type=float, default=0.08, help="rotational scale")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--seed", type=int, default=None, help="default: from the clock, as the "
                    "reference seeds its generators")
    ap.add_argument("--dump-dir", default="", help="write each dump window's records here")
    ap.add_argument("--gaussian", action="store_true")
    ap.add_argument("--surrogate", action="store_true",
                    help="delayed acceptance with the learned energy surrogate: the first dump "
                         "window's plain steps train it (one pass of Adam over their proposals), "
                         "later windows run delayed-acceptance steps")
    ap.add_argument("--train-iterations", type=int, default=0,
                    help="--surrogate: Adam steps (default: one pass over the samples)")
    ap.add_argument("--max-dumps", type=int, default=1000,
                    help="stop after this many dump windows even if records are short")
    return ap.parse_args(argv)


def run(a) -> int:
    t_start = time.perf_counter()
    seed = a.seed if a.seed is not None else time.time_ns() & ((1 << 63) - 1)
    cx, ff, _ = loaders.load_complex(a.pdb, a.sdf, a.ff, a.para, a.id, a.nt, a.floor_temp,
                                     a.ceiling_temp)
    spd = abi.STEPS_PER_DUMP
    params = abi.mc_params(steps_per_exchange=a.nc, steps_per_dump=spd,
                           move_scale=(a.t, a.t, a.t, a.r, a.r, a.r),
                           move_kind=abi.MOVE_GAUSSIAN if a.gaussian else abi.MOVE_UNIFORM,
                           record=1, seed=seed)
    n_rep = cx.n_rep
    print("n_lig %d n_prt %d n_tmp %d n_rep %d lna %d pnp %d pnk %d pos %d" %
          (cx.n_lig, cx.n_prt, cx.n_tmp, n_rep, cx.lna, cx.pnp, cx.pnk, cx.pos))
    per_rep = [[] for _ in range(n_rep)]
    est = spd * n_rep
    print("estimated total records: %d" % est)
    have = 0
    s1 = 0
    t_mc = 0.0
    t_train = 0.0
    with engine.Engine(ff, [cx], params, device=a.device) as e:
        e.mc_init()
        sur = engine.Surrogate(e, sample_cap=n_rep * spd) if a.surrogate else None
        dump = 0
        while have < est and dump < a.max_dumps:
            if s1 != 0:
                e.reset_records()
            t0 = time.perf_counter()
            if sur is None:
                e.run_fused(s1, spd, exchange=True)
            elif dump == 0:
                sur.collect(s1, spd, exchange=True)  # plain steps; their proposals are samples
            else:
                sur.run(s1, spd, exchange=True)
            e.sync()
            t_mc += time.perf_counter() - t0
            if sur is not None and dump == 0:
                t0 = time.perf_counter()
                iters = a.train_iterations or max(1, n_rep * spd // 8192)
                sur.train(iters)
                t_train = time.perf_counter() - t0
            steps, nxt = e.records()
            for i in range(n_rep):
                per_rep[i].append(steps[i, :nxt[i]])
            have += int(nxt.sum())
            print("# points\t\t\t%d" % have, flush=True)
            if a.dump_dir:
                records.write_dump(e, a.dump_dir, a.id, s1 // spd)
            s1 += spd
            dump += 1
        sur_stats = sur.stats() if sur is not None else None
    recs = [np.concatenate(r) if r else np.zeros(0, abi.RECORD_DTYPE) for r in per_rep]
    t0 = time.perf_counter()
    medoids, sizes = postmc.post_mc(recs, seed=seed & 0xFFFFFFFF, device=a.device)
    t_post = time.perf_counter() - t0
    print("Final output")
    postmc.write_states(medoids, a.csv)
    trials = n_rep * s1
    print("=" * 80)
    print("ligand file\t\t\t%s\nprotein file\t\t\t%s\nlhm file\t\t\t%s\nenepara file\t\t\t%s"
          % (a.sdf, a.pdb, a.ff, a.para))
    print("out file (csv)\t\t\t%s" % a.csv)
    print("steps_total\t\t\t%d\nsteps_per_dump\t\t\t%d\nsteps_per_exchange\t\t%d" %
          (s1, spd, a.nc))
    print("translational scale\t\t%.8f %.8f %.8f" % (a.t, a.t, a.t))
    print("rotational scale\t\t%.8f %.8f %.8f" % (a.r, a.r, a.r))
    print("temperatures\t\t\t%d (%.4f .. %.4f)" % (a.nt, a.floor_temp, a.ceiling_temp))
    print("acceptance ratio\t\t%.5f" % (have / trials if trials else 0.0))
    if a.surrogate:
        st = sur_stats[0] if sur_stats else {}
        print("surrogate\t\t\tproposed %d passed %d accepted %d rmse %.4f (training %.3f s)"
              % (st.get("proposed", 0), st.get("passed", 0), st.get("accepted", 0),
                 st.get("rmse", 0.0), t_train))
    print("representatives\t\t\t%d" % medoids.shape[0])
    print("Monte Carlo time (s)\t\t%.3f\npost-processing time (s)\t%.3f\ntotal time (s)\t\t\t%.3f"
          % (t_mc, t_post, time.perf_counter() - t_start))
    print("=" * 80)
    return 0


def main(argv=None) -> int:
    try:
        return run(parse(argv))
    except loaders.LoadError as ex:
        print("GeauxDock: %s" % ex, file=sys.stderr)
        return 2


if __name__ == "__main__":
    sys.exit(main())
