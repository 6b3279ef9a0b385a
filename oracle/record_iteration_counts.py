"""Record the oracle's Picard / PCG iteration counts of converged solves of a
bench workload's domains into profiles/iteration_counts.json.

The bench's CPU baseline and its reference arm time a bounded sample of the
oracle (the C restatement of the reference's solver, test infrastructure)
and extrapolate it to a converged solve with these counts.  Each domain is
solved to convergence by the oracle in its own process (one thread each),
with the bench's own model of that domain (bench.make_models).

    python oracle/record_iteration_counts.py c4 --batch 4 [--picard l2rel]
"""
import argparse
import json
import multiprocessing as mp
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[0] = ROOT  # the repository root, not this folder (whose oracle.py would shadow the package)
OUT = os.path.join(ROOT, "profiles", "iteration_counts.json")


def _solve(job):
    workload, batch, picard, i = job
    os.environ["OMP_NUM_THREADS"] = "1"
    import bench
    from oracle import oracle

    m = bench.make_models(bench.parse_args(["--workload", workload, "--batch", str(batch), "--picard", picard]))[i]
    t0 = time.perf_counter()
    _, _, _, _, st = oracle.velo_higher_solve(m)
    return {"domain": i, "picard_iters": int(st["picard_iters"]), "pcg_iters_total": int(st["pcg_iters_total"]),
            "status": int(st.get("status", 0)), "oracle_seconds": round(time.perf_counter() - t0, 1)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload")
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--picard", default="l2rel")
    a = ap.parse_args()
    n = a.batch if a.workload in ("c4", "c3") else 1
    with mp.get_context("spawn").Pool(n) as pool:
        res = pool.map(_solve, [(a.workload, a.batch, a.picard, i) for i in range(n)])
    d = json.load(open(OUT)) if os.path.exists(OUT) else {}
    d[f"{a.workload}/{a.picard}"] = {
        "per_domain": res,
        "source": f"oracle converged solves (oracle/record_iteration_counts.py {a.workload} --batch {a.batch} "
                  f"--picard {a.picard}), one thread per domain",
    }
    with open(OUT, "w") as f:
        json.dump(d, f, indent=1)
    print(json.dumps(d[f"{a.workload}/{a.picard}"]))


if __name__ == "__main__":
    main()
