"""Check the CPU baseline's extrapolation against fully converged solves.

bench.py times the oracle (the C restatement of the reference, test
infrastructure) on a bounded sample -- setup, one assembly and two PCG
runs -- and extrapolates it to a converged solve with the solve's Picard
and PCG iteration counts.  This script times a whole converged oracle solve
of a workload (one thread) and the bench's sample extrapolated with that
solve's own counts, and prints both as one JSON line per workload.

    python oracle/validate_cpu_baseline.py c0 c1 [--resid 0|4]
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
    from cism_b200 import configs
    from oracle import oracle

    for w in a.workloads:
        m = configs.workload(w).copy(pcg_maxiters=5000, which_resid=a.resid)
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
