"""Check the CPU baseline's extrapolation against fully converged solves.

bench.py times the oracle (the C restatement of the reference, test
infrastructure) on a bounded sample -- setup, one assembly and two PCG
runs -- and extrapolates it to a converged solve with the solve's Picard
and PCG iteration counts.  This script times a whole converged oracle solve
of a workload (one thread) and the bench's sample extrapolated with that
solve's own counts, and prints both as one JSON line per workload.

    python oracle/validate_cpu_baseline.py c0 c1 c4 [--resid 0|4]

c4 is the bench's first marine domain (256 x 256 cells, dx = 2 km, the
column preconditioner), built by bench.make_models as the bench builds it.
"""
import argparse
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[0] = ROOT  # the repository root, not this folder (whose oracle.py would shadow the package)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workloads", nargs="+")
    ap.add_argument("--resid", type=int, default=4)
    a = ap.parse_args()
    import bench
    from oracle import oracle

    picard = {v: k for k, v in bench.PICARD.items()}[a.resid]
    for w in a.workloads:
        m = bench.make_models(bench.parse_args(["--workload", w, "--batch", "1", "--picard", picard]))[0]
        t0 = time.perf_counter()
        _, _, _, _, st = oracle.velo_higher_solve(m)
        full = time.perf_counter() - t0
        cs = bench.cpu_sample(m, (st["picard_iters"], st["pcg_iters_total"]))
        print(json.dumps({"workload": w, "which_resid": a.resid, "picard_iters": st["picard_iters"],
                          "pcg_iters_total": st["pcg_iters_total"], "full_solve_s": round(full, 2),
                          "extrapolated_s": round(cs["t_solve_est"], 2),
                          "ratio_extrapolated_over_full": round(cs["t_solve_est"] / full, 4),
                          "sample_s": round(cs["sample_seconds"], 2), "cpu": os.cpu_count()}), flush=True)


if __name__ == "__main__":
    main()
