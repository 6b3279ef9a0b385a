#!/usr/bin/env python
"""Converged Blatter-Pattyn velocity solves per second on B200.

Default workload (c4): the learned-guess evaluation set -- held-out marine
ice sheets drawn as the large marine configuration (seeded Gaussian-random
bed with a trough, parabolic 3000 m sheet with a calving front, log-normal
beta, zero under the shelf) at 256 x 256 cells, dx = 2 km, 11 sigma
levels, Glen n = 3; `--batch` domains (default 4).  Every linear solve to
a relative residual of 1e-8; the Picard loop to the reference's relative
nonlinear residual criterion (which_ho_resid = 4: |A(u)u - b| / |b| < 1e-7
before the last linear solve), whose answer does not depend on the start
(two starts agree to ~1e-10), so every path can be held to 1e-6 of the
plain FP64 answer.  A "step" solves every domain of the workload once.
Synthetic seeded inputs; no dataset is used.

Paths: the plain FP64 path (P: FP64, zero start, one domain at a time,
with the workload's solver -- for the marine workloads the reference's
default SIA column preconditioner and Chronopoulos-Gear PCG) and the
additions: mixed precision (FP32-inner / FP64-refined), batching (all
domains in one resident problem) and the learned guess (the U-Net behind
the C ABI); the marine workloads also time the mixed batched solve from
the shallow-ice velocity (sia_mixed_batched), the classical start.  The headline `value` is learned + mixed + batched; `paths`
lists every path with its iterations and its distance to P's answer.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload c4|c2|c1|c0|c3] [--batch B]

With N > 1 (torchrun) every rank solves its own replica (the solve does
not shard across GPUs); value = all ranks' solves / max rank time.
`--impl reference` times the CPU oracle (a C restatement of the
reference's Fortran, which cannot be compiled here) single-threaded on
one host core, on bounded samples of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged velocity solves/sec @1e-8 rel resid: learned+mixed vs plain FP64, 1 B200"
UNIT = "solves/s"
WORKLOAD_DESC = {
    "c4": "held-out marine ice sheets 256x256 cells x 11 levels, dx=2 km, grounding line + shelf + calving front "
          "(drawn as the 400x400 marine configuration); learned guess + mixed + batched vs plain FP64",
    "c2": "marine ice sheet 400x400 cells x 11 levels, dx=4 km, grounding line + shelf + calving front",
    "c1": "periodic slab 160x160 cells x 11 levels, dx=0.5 km, sinusoidal beta, Glen n=3",
    "c0": "parabolic dome 31x31 cells x 10 levels, dx=2 km, no-slip bed",
    "c3": "ensemble of domes and slabs, 32-192 cells per side x 11 levels, dx=2 km, log-normal beta",
}
PICARD = {"l2rel": 4, "maxu": 0}
PICARD_DESC = {4: "relative nonlinear residual |A(u)u-b|/|b| < 1e-7 (which_ho_resid = 4)",
               0: "max relative speed change < 1e-4 (which_ho_resid = 0)"}
# per-domain Picard / PCG iteration counts of the plain FP64 path, by
# workload, used to extrapolate the bounded CPU samples to whole solves
ITERATION_COUNTS = os.path.join(ROOT, "profiles", "iteration_counts.json")
# the marine network also serves the c3 ensemble (domes and slabs it never
# saw in training: its features are the solve's own fields)
WEIGHTS = {"c4": "unet_marine", "c2": "unet_marine", "c3": "unet_marine"}
HELDOUT_SEED = 70000  # past every training seed of the marine network
ASM_FLOP_PER_ELEMENT = 18.1e3  # 8 quadrature points x ~2.2k + scatter (FP64)


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c4", choices=sorted(WORKLOAD_DESC))
    ap.add_argument("--batch", type=int, default=4, help="c4 / c3: domains of the workload")
    ap.add_argument("--picard", default="l2rel", choices=sorted(PICARD))
    ap.add_argument("--paths", default="all", help="comma-separated path names, or all")
    ap.add_argument("--other-steps", type=int, default=1, help="timed steps of the non-headline paths")
    ap.add_argument("--pcg-maxiters", type=int, default=5000)
    ap.add_argument("--refine-eta", type=float, default=1e-4,
                    help="mixed path: residual reduction of one FP32 refinement cycle")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-run", action="store_true",
                    help="one untimed run of --paths (first path) (for ncu launch lists / captures)")
    ap.add_argument("--weights", default=None,
                    help="U-Net weights (.bin) for the learned paths of any 3-D workload (default: the "
                         "workload's own network, where it has one)")
    ap.add_argument("--picard-cap", type=int, default=0,
                    help="with --profile-run: stop after this many Picard iterations")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
# workloads and paths
# ---------------------------------------------------------------------------
def make_models(args):
    from cism_b200 import configs

    w = args.workload
    if w == "c4":
        ms = [configs.marine(n=256, dx=2000.0, seed=HELDOUT_SEED + i) for i in range(args.batch)]
    elif w == "c3":
        ms = configs.ensemble(count=args.batch)
    else:
        ms = [configs.workload(w)]
    if w in ("c4", "c2"):  # the reference's default preconditioner (glide_types.F90:698)
        ms = [m.copy(which_precond=configs.PRECOND_SIA) for m in ms]
    # the reference hard-codes maxiters = 200 (glissade_velo_higher_pcg.F90:67-69),
    # which does not reach 1e-8 on these systems; the metric needs converged solves
    return [m.copy(pcg_maxiters=args.pcg_maxiters, which_resid=PICARD[args.picard]) for m in ms]


class Path:
    """One way of solving the workload: start (zero | sia: the shallow-ice
    velocity, guess.sia_guess | learned), precision,
    preconditioner (None: the workload's; "diag" | "sia" to override), PCG
    variant (the workload's | Chronopoulos-Gear), batched (all domains in
    one resident problem) or one domain at a time."""

    def __init__(self, name, start, mixed, precond, cg, batched):
        self.name, self.start, self.mixed, self.precond, self.cg, self.batched = (name, start, mixed, precond,
                                                                                 cg, batched)

    def model(self, m):
        from cism_b200 import configs

        if self.precond == "sia":
            m = m.copy(which_precond=configs.PRECOND_SIA)
        elif self.precond == "diag":
            m = m.copy(which_precond=configs.PRECOND_DIAG)
        if self.cg:
            m = m.copy(which_sparse=configs.SPARSE_PCG_CHRONGEAR)
        return m

    def describe(self, m):
        from cism_b200 import configs

        mm = self.model(m)
        return {"start": self.start, "precision": "fp32-inner/fp64-refined" if self.mixed else "fp64",
                "preconditioner": "sia_column" if mm.which_precond == configs.PRECOND_SIA else "diagonal",
                "pcg": "chronopoulos_gear" if mm.which_sparse == configs.SPARSE_PCG_CHRONGEAR else "standard",
                "domains": "batched in one problem" if self.batched else "one at a time"}


def paths_for(args, have_net):
    """The marine workloads (c4, c2) solve with the reference's default
    preconditioner (the SIA column one, which_ho_precond = 2) and the
    Chronopoulos-Gear PCG every reference higher-order test uses, so P and
    the additions share the preconditioner; plain_fp64_diag (by --paths)
    is P with the diagonal one.  c0 and c1 specify the diagonal
    preconditioner and the standard PCG; their additions also swap in the
    column preconditioner and Chronopoulos-Gear (fp64_colpc isolates that)."""
    multi = args.workload in ("c4", "c3")
    sfx = "_batched" if multi else ""
    if args.workload in ("c4", "c2"):
        P = [Path("plain_fp64", "zero", False, None, False, False),
             Path("mixed" + sfx, "zero", True, None, False, multi)]
        P.append(Path("sia_mixed" + sfx, "sia", True, None, False, multi))
        if have_net:
            P += [Path("learned_fp64" + sfx, "learned", False, None, False, multi),
                  Path("learned_mixed" + sfx, "learned", True, None, False, multi)]
        extra = [Path("plain_fp64_diag", "zero", False, "diag", False, False)]
    else:
        P = [Path("plain_fp64", "zero", False, None, False, False),
             Path("fp64_colpc", "zero", False, "sia", False, False),
             Path("mixed_colpc_cg" + sfx, "zero", True, "sia", True, multi)]
        if have_net:
            P += [Path("learned_fp64_colpc" + sfx, "learned", False, "sia", False, multi),
                  Path("learned_mixed_colpc_cg" + sfx, "learned", True, "sia", True, multi)]
        extra = []
    if args.paths != "all":
        want = args.paths.split(",")
        P = [p for p in P + extra if p.name in want]
    return P


def headline_name(paths):
    names = [p.name for p in paths]
    for n in names[::-1]:
        if n.startswith("learned_mixed"):
            return n
    return names[-1]


def weights_path(workload, override=None):
    if override:
        return override if os.path.exists(override) else None
    name = WEIGHTS.get(workload)
    if not name:
        return None
    p = os.path.join(ROOT, "cism_b200", "weights", name + ".bin")
    return p if os.path.exists(p) else None


def workload_stats(models):
    """Columns and nodes of the workload (host setup only)."""
    import numpy as np

    from cism_b200 import solver

    cols = 0
    for m in models:
        prep, _, _ = solver.prepare(m)
        js, is_ = m.owned_vertex_slices()
        cols += int(np.count_nonzero(np.asarray(prep.arrays["active_vertex"])[js, is_]))
    return cols, cols * models[0].nz


def config_dict(args, models, cols, nodes, world=1):
    return {"workload": WORKLOAD_DESC[args.workload], "name": args.workload, "domains": len(models),
            "columns": cols, "nodes": nodes, "pcg_maxiters": args.pcg_maxiters, "pcg_tol": 1e-8,
            "picard_criterion": PICARD_DESC[PICARD[args.picard]],
            "l2": "inputs larger than L2 (FP64 matrix %.0f MB > 126 MB)" % (nodes * 448 / 1e6),
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


# ---------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------
class Dist:
    """One process per GPU (replicas): NCCL with a GPU, gloo without (the
    CPU tests); only a barrier and the max over ranks of the timed region."""

    def __init__(self, gpus, backend=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.cuda = False
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            self.cuda = backend != "gloo" and torch.cuda.is_available()
            if self.cuda:
                torch.cuda.set_device(self.local)
            dist.init_process_group("nccl" if self.cuda else "gloo", timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            if self.cuda:
                import torch

                self.pg.barrier(device_ids=[self.local])
                torch.cuda.synchronize()
            else:
                self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch

        dev = f"cuda:{self.local}" if self.cuda else "cpu"
        t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index=0):
        self.proc = None
        self.path = None
        self.uuid = None
        try:
            import torch

            u = torch.cuda.get_device_properties(device_index).uuid
            self.uuid = "GPU-" + str(u)
        except Exception:
            pass

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader",
                                          "-lms", "200"], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            if self.uuid and f[0] != self.uuid:
                continue
            try:
                rows.append((float(f[1].split()[0]), float(f[2].split()[0]), f[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for _, _, r in rows for n, v in zip(names, r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def committed_traffic(precision):
    """DRAM bytes per node of the dominant kernel from the committed ncu
    summary (profiles/ncu_traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    k = d.get("fp32_inner" if precision == "mixed" else "fp64_pcg")
    return k if k else None


# ---------------------------------------------------------------------------
# CPU baseline: bounded sample of the oracle, extrapolated to whole solves
# ---------------------------------------------------------------------------
def cpu_sample(m, counts, iters=(20, 60)):
    """Setup, one assembly and two PCG runs of the oracle (the checker, a C
    restatement of the reference) on domain m, 1 thread; the per-iteration
    time and the fixed costs extrapolated to `counts` (Picard, PCG)
    iterations of a converged solve."""
    import numpy as np

    from oracle import oracle  # the checker

    t0 = time.perf_counter()
    su = oracle.setup(m)
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    A, bu, bv, _, _ = oracle.assemble_system(m, su, su["uvel"], su["vvel"])
    t_asm = time.perf_counter() - t0
    z = np.zeros(m.vshape3)
    ts = []
    for it in iters:
        t0 = time.perf_counter()
        oracle.pcg(m, su["active_vertex"], A, bu, bv, z, z, precond=m.which_precond,
                   variant=m.which_sparse if m.which_sparse in (2, 3) else 2, maxiters=it, tol=0.0)
        ts.append(time.perf_counter() - t0)
    t_iter = (ts[1] - ts[0]) / (iters[1] - iters[0])
    t_pcg_fixed = max(ts[0] - iters[0] * t_iter, 0.0)  # preconditioner setup + initial residual
    Pc, I = counts
    t_solve = t_setup + Pc * (t_asm + t_pcg_fixed) + I * t_iter
    return {"t_solve_est": t_solve, "t_setup": t_setup, "t_assembly": t_asm, "t_pcg_iter": t_iter,
            "sample_seconds": t_setup + t_asm + sum(ts)}


def load_counts(workload):
    if os.path.exists(ITERATION_COUNTS):
        d = json.load(open(ITERATION_COUNTS))
        return d.get(workload)
    return None


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_path(ctx, path, models, args, D, steps, warmup, weights, clocks=None):
    """Time `steps` steps of one path (each solves every domain once);
    returns timings, stats, solutions and, for batched paths, the problem."""
    import numpy as np

    from cism_b200 import solver

    prec = solver.MIXED if path.mixed else solver.FP64
    mode = solver.GUESS_LEARNED if path.start == "learned" else solver.GUESS_GIVEN
    ms_ = [path.model(m) for m in models]
    preps = [solver.prepare(m, precision=prec, inner_tol=args.refine_eta, guess_mode=mode)[0] for m in ms_]
    if path.start == "sia":  # the shallow-ice velocity (host arrays, copied in every step)
        from cism_b200 import guess

        starts = [guess.sia_guess(m) for m in ms_]
    else:
        starts = [(np.zeros(m.vshape3), np.zeros(m.vshape3)) for m in ms_]
    probs = [ctx.problem(preps)] if path.batched else [ctx.problem([p]) for p in preps]
    first = [0]
    for pb in probs[:-1]:
        first.append(first[-1] + pb.n)

    def step():
        sts = []
        for pb, f0 in zip(probs, first):
            if mode == solver.GUESS_LEARNED:  # the network runs on the device here
                pb.set_guess([None] * pb.n, [None] * pb.n)
            else:
                pb.set_guess([u for u, _ in starts[f0:f0 + pb.n]], [v for _, v in starts[f0:f0 + pb.n]])
            sts += pb.run()
        return sts

    for _ in range(warmup):
        step()
    D.barrier()
    g0 = ctx.guess_launches()
    if clocks:
        clocks.start()
    ctx.timer_start()
    t0 = time.perf_counter()
    sts = [step() for _ in range(steps)][-1]
    wall = (time.perf_counter() - t0) * 1000.0
    ms = ctx.timer_stop()
    ck = clocks.stop() if clocks else None
    D.barrier()
    guess_launches = (ctx.guess_launches() - g0) // max(1, steps)
    ms = D.max(max(ms, wall))
    sols = []
    for pb in probs:
        us, vs, _ = pb.get()
        sols += list(zip(us, vs))
    return {"ms": ms, "ms_per_step": ms / steps, "steps": steps, "stats": sts, "sols": sols, "probs": probs,
            "preps": preps, "clocks": ck, "guess_launches_per_step": guess_launches}


def kernel_profile(res, models):
    """One timing run (CUDA events around every launch, graphs off) of a
    path's problems: Krylov matvec time and bytes, assembly time, launches."""
    import numpy as np

    t_mv = n_mv = t_asm = n_asm = 0.0
    n64 = n32 = 0.0
    launches = 0
    info = None
    for pb in res["probs"]:
        pb.timing(True)
        g = [None if p.inputs.guess_mode else np.zeros(p.model.vshape3) for p in pb.preps]
        pb.set_guess(g, g)
        pb.run()
        kt = pb.kernel_times()
        a, b, minb, grid = pb.mv_nodes()
        n64 += a
        n32 += b
        t_mv += kt["pcg_matvec_fp64"][0]
        n_mv += kt["pcg_matvec_fp64"][1]
        t_asm += kt["assembly_qp"][0] + kt["assembly_rows"][0]
        n_asm += kt["assembly_rows"][1]
        launches += sum(n for _, n in kt.values())
        pb.timing(False)
        inf = pb.info()
        if info is None:
            info = dict(inf)
        else:
            for k in ("nodes", "columns", "elements", "matvec_bytes_fp64", "matvec_bytes_fp32"):
                info[k] += inf[k]
    return {"t_mv_ms": t_mv, "n_mv": n_mv, "n64": n64, "n32": n32, "t_asm_ms": t_asm, "n_asm": n_asm,
            "launches": launches, "info": info}


def rel_l2(a, b):
    import numpy as np

    num = math.sqrt(float(np.sum((a[0] - b[0]) ** 2 + (a[1] - b[1]) ** 2)))
    den = math.sqrt(float(np.sum(b[0] ** 2 + b[1] ** 2)))
    return num / den if den > 0 else num


def run_ours(args, D):
    import numpy as np

    from cism_b200 import solver

    ctx = solver.Context(D.local)
    models = make_models(args)
    weights = weights_path(args.workload, args.weights)
    if weights:
        ctx.load_guess(weights)
    paths = paths_for(args, weights is not None)
    head = headline_name(paths)
    res = {}
    for p in paths:
        is_head = p.name == head
        res[p.name] = run_path(ctx, p, models, args, D, args.steps if is_head else args.other_steps,
                               args.warmup if is_head else 1, weights,
                               clocks=Clocks(D.local) if is_head else None)
    H = res[head]
    ref_sol = res["plain_fp64"]["sols"] if "plain_fp64" in res else H["sols"]
    nd = len(models)
    out_paths = {}
    for p in paths:
        r = res[p.name]
        sts = r["stats"]
        errs = [rel_l2(a, b) for a, b in zip(r["sols"], ref_sol)]
        out_paths[p.name] = p.describe(models[0]) | {
            "value": round(nd * D.world / (r["ms_per_step"] / 1000.0), 4),
            "ms_per_step": round(r["ms_per_step"], 2), "steps": r["steps"],
            "status": sorted({int(s["status"]) for s in sts}),
            "picard_iters_mean": round(float(np.mean([s["picard_iters"] for s in sts])), 2),
            "pcg_iters_mean": round(float(np.mean([s["pcg_iters_total"] for s in sts])), 1),
            "final_rel_resid_max": float("%.3e" % max(s["pcg_err_last"] for s in sts)),
            "rel_l2_vs_plain_fp64_max": float("%.3e" % max(errs)),
            "per_domain": [{"picard_iters": int(s["picard_iters"]), "pcg_iters_total": int(s["pcg_iters_total"])}
                           for s in sts]}
    # accepted: every domain converged (status 0, last linear solve < 1e-8)
    # and within 1e-6 relative L2 of the plain FP64 answer
    hd = out_paths[head]
    ok = hd["status"] == [0] and hd["final_rel_resid_max"] < 1e-8 and hd["rel_l2_vs_plain_fp64_max"] <= 1e-6
    # e2e: the C-ABI call a user makes (bp_batch_solve on host arrays: the
    # guess, H2D, the solve and D2H inside every step)
    hp = [p for p in paths if p.name == head][0]
    preps = H["preps"]
    zeros = [np.zeros(p.model.vshape3) for p in preps]
    groups = [list(range(len(preps)))] if hp.batched else [[i] for i in range(len(preps))]

    def e2e_step():
        st = []
        for g in groups:  # uvel/vvel: the start (unless learned) in, the solution out
            st += ctx.batch_solve([preps[i] for i in g], [zeros[i] for i in g], [zeros[i] for i in g])[3]
        return st

    e2e_steps = min(args.steps, 3)  # the same work as the timed steps, fewer of them
    e2e_step()
    D.barrier()
    ctx.timer_start()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        st_e = e2e_step()
    ms_e = max(ctx.timer_stop(), (time.perf_counter() - t0) * 1000.0)
    D.barrier()
    ms_e = D.max(ms_e)
    e2e = {"value": round(nd * D.world * e2e_steps / (ms_e / 1000.0), 4), "unit": UNIT, "steps": e2e_steps,
           "h2d_bytes_per_step": int(sum(s["h2d_bytes"] for s in st_e)),
           "d2h_bytes_per_step": int(sum(s["d2h_bytes"] for s in st_e)),
           "call": "bp_batch_solve (C ABI) on host arrays, learned guess formed on the device inside the call"
                   if hp.start == "learned" else "bp_batch_solve (C ABI) on host arrays"}
    # roofline of the dominant kernel and assembly FLOP/s (timing run)
    kp = kernel_profile(H, models)
    info = kp["info"]
    N = info["nodes"]
    b64, b32 = info["matvec_bytes_fp64"] / N, info["matvec_bytes_fp32"] / N
    total_bytes = kp["n64"] * b64 + kp["n32"] * b32
    peak, peak_src = measured_peaks()
    achieved = total_bytes / (kp["t_mv_ms"] / 1000.0) / 1e9 if kp["n_mv"] else 0.0
    tr = committed_traffic("mixed" if hp.mixed else "fp64")
    roof = {"bound": "hbm",
            "kernel": "%s (Krylov matvec, thread per node, %s)" % (
                "k_cg_mv" if hp.describe(models[0])["pcg"] == "chronopoulos_gear" else "k_std_mv",
                "FP32 half storage + compensated FP64 diagonal" if hp.mixed else "FP64 half storage"),
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4) if peak else None,
            "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)",
            "traffic": round(tr["dram_bytes_per_node"] * N) if tr else None,
            "traffic_source": (tr["source"] + "; bytes per node scaled to this workload's nodes") if tr else None,
            "algorithmic_bytes_per_launch": round(total_bytes / max(kp["n_mv"], 1)),
            "algorithmic_bytes_per_node": {"fp32": b32, "fp64": b64},
            "avg_launch_us": round(kp["t_mv_ms"] / max(kp["n_mv"], 1) * 1e3, 2),
            "launches_timed": int(kp["n_mv"]),
            "fp32_share": round(kp["n32"] / max(1.0, kp["n32"] + kp["n64"]), 3)}
    asm_flop = info["elements"] * ASM_FLOP_PER_ELEMENT
    asm = {"flop_per_assembly": asm_flop, "ms_per_assembly": round(kp["t_asm_ms"] / max(kp["n_asm"], 1), 3),
           "achieved_tflops": round(asm_flop / (kp["t_asm_ms"] / max(kp["n_asm"], 1) / 1000.0) / 1e12, 3)
           if kp["n_asm"] else None,
           "peak_tflops": 37.0, "peak_source": "nominal FP64 (no measured FP64 peak on this pool)",
           "flop_count": "18.1k FP64 flops per element (8 quadrature points x Jacobian, inverse, strain, "
                         "viscosity and 64 block pairs x 28, plus the row gather)"}
    if asm["achieved_tflops"] is not None:
        asm["frac"] = round(asm["achieved_tflops"] / asm["peak_tflops"], 4)
    cols, nodes = info["columns"], info["nodes"]
    out = {
        "metric": METRIC, "value": out_paths[head]["value"], "unit": UNIT, "n_gpus": D.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": out_paths[head]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": ("f32+f64" if hp.mixed else "f64") + ("+bf16" if hp.start == "learned" else ""),
        "data": "synthetic (seeded geometry generator, no dataset)",
        "config": config_dict(args, models, cols, nodes, D.world), "path": head,
        "accepted": bool(ok),
        "e2e": e2e, "roofline": roof, "assembly": asm,
        "gpu_launches": (kp["launches"] + H["guess_launches_per_step"]) * args.steps,
        "clocks": H["clocks"], "paths": out_paths,
    }
    if "plain_fp64" in res:
        out["speedup_vs_plain_fp64"] = round(out_paths[head]["value"] / out_paths["plain_fp64"]["value"], 3)
    if "fp64_colpc" in res:  # c0, c1: the plain path with the additions' preconditioner
        out["speedup_vs_plain_fp64_same_preconditioner"] = round(
            out_paths[head]["value"] / out_paths["fp64_colpc"]["value"], 3)
    if D.rank == 0 and D.world == 1 and not args.no_cpu_baseline and "plain_fp64" in res:
        # the oracle's own counts for domain 0 where recorded, else the GPU FP64 path's
        rec = load_counts(f"{args.workload}/{args.picard}")
        if rec:
            c0 = rec["per_domain"][0]
            counts, src = (c0["picard_iters"], c0["pcg_iters_total"]), "the oracle's converged-solve counts"
        else:
            st0 = res["plain_fp64"]["stats"][0]
            counts, src = (st0["picard_iters"], st0["pcg_iters_total"]), "the GPU FP64 path's counts"
        cs = cpu_sample(models[0], counts)
        out["cpu_baseline"] = {
            "value": round(1.0 / cs["t_solve_est"], 8), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": (f"oracle (C restatement of the reference, 1 thread): setup, one assembly and 20 / 60 PCG "
                       f"iterations of domain 0, extrapolated to {src} ({counts[0]} Picard, {counts[1]} PCG); "
                       f"profiles/cpu_oracle_validation.md checks the extrapolation against fully converged "
                       f"oracle solves"),
            "sample_seconds": round(cs["sample_seconds"], 1)}
    for r in res.values():
        for pb in r["probs"]:
            pb.close()
    ctx.close()
    return out


# ---------------------------------------------------------------------------
# reference arm: the oracle (restatement of the reference Fortran) on one
# host core, bounded samples extrapolated with the recorded iteration counts
# ---------------------------------------------------------------------------
def run_reference(args, D):
    if D.rank != 0:
        return None
    models = make_models(args)
    counts = load_counts(f"{args.workload}/{args.picard}")
    if counts is None:
        return {"impl": "reference", "unavailable": "no recorded iteration counts for this workload"}
    vals, walls = [], []
    for step in range(args.warmup + args.steps):
        i = step % len(models)
        c = counts["per_domain"][i % len(counts["per_domain"])]
        t0 = time.perf_counter()
        cs = cpu_sample(models[i], (c["picard_iters"], c["pcg_iters_total"]))
        if step >= args.warmup:
            vals.append(cs["t_solve_est"])
            walls.append(time.perf_counter() - t0)
    v = len(vals) / sum(vals)
    cols, nodes = workload_stats(models)
    sample = (f"oracle (C restatement of the reference's Fortran, which cannot be compiled here), 1 process, "
              f"1 thread on {os.cpu_count()} host cores: per step setup, one assembly and 20 / 60 PCG iterations "
              f"of one domain, extrapolated to that domain's recorded plain-FP64 Picard / PCG counts "
              f"({counts['source']})")
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": D.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(statistics.mean(walls) * 1000.0, 1),
            "value_basis": "extrapolated: value = domains / sum of the extrapolated solve times; ms_per_step is "
                           "the sample's own wall time",
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(args, models, cols, nodes, D.world), "path": "plain_fp64 (oracle, CPU)",
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def profile_run(args):
    """One untimed run of the first selected path (for ncu)."""
    from cism_b200 import solver

    models = make_models(args)
    if args.picard_cap > 0:
        models = [m.copy(maxiter_nonlinear=args.picard_cap) for m in models]
    ctx = solver.Context(0)
    w = weights_path(args.workload, args.weights)
    if w:
        ctx.load_guess(w)
    p = paths_for(args, w is not None)[0]

    class _D:
        world, rank = 1, 0

        def barrier(self):
            pass

        def max(self, x):
            return x

    r = run_path(ctx, p, models, args, _D(), 1, 0, w)
    sts = r["stats"]
    print(json.dumps({"profile_run": args.workload, "path": p.name, "status": sorted({s["status"] for s in sts}),
                      "picard_iters": [s["picard_iters"] for s in sts],
                      "pcg_iters_total": [s["pcg_iters_total"] for s in sts]}), flush=True)
    for pb in r["probs"]:
        pb.close()
    ctx.close()


def main(argv=None):
    args = parse_args(argv)
    if args.profile_run:
        profile_run(args)
        return
    D = Dist(args.gpus)
    try:
        out = run_reference(args, D) if args.impl == "reference" else run_ours(args, D)
        if D.rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        D.close()


if __name__ == "__main__":
    main()
