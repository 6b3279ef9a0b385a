"""Training of the learned initial guess on solutions of this solver.

    python -m cism_b200.train_guess --family marine --out cism_b200/weights/unet_marine.npz
    python -m cism_b200.train_guess --family slab --out cism_b200/weights/unet_slab.npz

draws seeded members of a domain family, solves them with this solver from
a zero start (several domains per resident multi-instance problem), trains
the U-Net on (fields -> velocity) with the project's BF16 kernels and Adam,
saves the weights with their input and output normalisation, and evaluates
held-out domains: the guess's error and the Picard and PCG iterations and
solve time from zero and learned starts.  Runs on one GPU.

Families: ``marine`` -- marine ice sheets around the large marine workload
(``configs.random_marine``, 128-256 cells per side at dx = 2 km), trained
on the features of ``net.input_features`` (built from bp_setup's outputs,
as the C-ABI guess builds them) and evaluated on held-out members drawn
exactly as the marine workload at 256 x 256 cells, dx = 2 km; ``slab`` --
the periodic-slab family of ``configs.random_slab`` (the first network).
Marine targets are converged to the relative nonlinear residual criterion
(which_ho_resid = 4), whose answer does not depend on the start.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time
from typing import Dict, List

import numpy as np

from . import configs, guess, net, solver


def solve_models(ctx, models: List[configs.BPModel], precision=solver.FP64, guesses=None, batch: int = 8,
                 keep_arrays: bool = False):
    """Solve domains (same size) in resident multi-instance problems; returns
    velocities, stats and the device time per problem (and with keep_arrays
    each domain's bp_setup arrays)."""
    us, vs, sts, ms, arrs = [], [], [], [], []
    for i in range(0, len(models), batch):
        group = models[i:i + batch]
        preps = [solver.prepare(m, precision=precision) for m in group]
        if keep_arrays:
            arrs += [p[0].arrays for p in preps]
        prob = ctx.problem([p[0] for p in preps])
        if guesses is None:
            prob.set_guess([p[1] for p in preps], [p[2] for p in preps])
        else:
            prob.set_guess([g[0] for g in guesses[i:i + batch]], [g[1] for g in guesses[i:i + batch]])
        ctx.timer_start()
        st = prob.run()
        ms.append(ctx.timer_stop())
        u, v, _ = prob.get()
        us += u
        vs += v
        sts += st
        prob.close()
    if keep_arrays:
        return us, vs, sts, ms, arrs
    return us, vs, sts, ms


def make_set(ctx, count: int, n: int, seed: int, batch: int):
    rng = np.random.default_rng(seed)
    models = [configs.random_slab(rng, n=n) for _ in range(count)]
    # targets from the column-preconditioned solver (the same answers to the
    # solver's tolerances, in a third of the iterations)
    models = [m.copy(pcg_maxiters=3000, which_precond=configs.PRECOND_SIA) for m in models]
    us, vs, sts, _ = solve_models(ctx, models, batch=batch)
    ok = [i for i, s in enumerate(sts) if s["status"] == 0]
    feats = np.stack([net.features(models[i]) for i in ok])
    targs = np.stack([net.velocity_targets(models[i], us[i], vs[i]) for i in ok])
    return [models[i] for i in ok], feats, targs, [(us[i], vs[i]) for i in ok]


# marine family: the solver settings of its targets and evaluations
MARINE_SOLVE = dict(which_resid=configs.RESID_L2NORM_RELATIVE, pcg_maxiters=5000,
                    which_precond=configs.PRECOND_SIA, which_sparse=configs.SPARSE_PCG_CHRONGEAR)


def make_marine_set(ctx, sizes, count: int, seed: int, batch: int, log=None, deadline=None, n_in: int = net.N_IN):
    """`count` members of the marine family, sizes drawn from `sizes`,
    solved (mixed precision, column preconditioner, Chronopoulos-Gear, the
    relative-residual Picard criterion) in problems of `batch` same-size
    domains, the sizes taken in turn so that a deadline cuts every size
    alike.  Returns per size: (models, padded features, padded targets,
    padded masks of the active vertices)."""
    rng = np.random.default_rng(seed)
    plan = [int(rng.choice(sizes)) for _ in range(count)]
    per_size = {n: [configs.random_marine(rng, n=n).copy(**MARINE_SOLVE) for _ in range(plan.count(n))]
                for n in sorted(set(plan))}
    chunks = {n: [ms[i:i + batch] for i in range(0, len(ms), batch)] for n, ms in per_size.items()}
    order = []  # round robin over the sizes
    for r in range(max(len(c) for c in chunks.values())):
        order += [(n, c[r]) for n, c in chunks.items() if r < len(c)]
    out = {}
    t0 = time.time()
    for n, grp in order:
        if deadline is not None and time.time() > deadline:
            break
        us, vs, sts, _, arrs = solve_models(ctx, grp, precision=solver.MIXED, batch=batch, keep_arrays=True)
        M, F, T, K = out.setdefault(n, ([], [], [], []))
        for m, u, v, st, a in zip(grp, us, vs, sts, arrs):
            if st["status"] != 0:
                continue
            M.append(m)
            F.append(net.pad_grid(net.input_features(m, a, n_in)).astype(np.float32))
            T.append(net.pad_grid(net.velocity_targets(m, u, v)).astype(np.float32))
            js, is_ = m.owned_vertex_slices()
            K.append(net.pad_grid((np.asarray(a["active_vertex"])[js, is_] != 0).astype(np.float32)[..., None])[..., 0])
        if log:
            log(f"  {n}x{n}: {len(M)} solved ({time.time() - t0:.0f} s)")
    return {n: (M, np.stack(F), np.stack(T), np.stack(K)) for n, (M, F, T, K) in out.items() if M}


def step_size(lr: float, frac: float, warm: float = 0.03) -> float:
    """Adam's step size at the fraction `frac` of the schedule: a linear
    ramp to `lr` over the first `warm` of it, then a cosine decay to zero."""
    if frac < warm:
        return lr * frac / warm
    return lr * 0.5 * (1.0 + math.cos(math.pi * min((frac - warm) / (1.0 - warm), 1.0)))


def train(model: net.UNet, groups, epochs: int, lr: float, batch: int, seed: int, log=None, periodic: int = 1,
          deadline=None):
    """groups: list of (features [N,H,W,n_in], targets [N,H,W,C][, masks
    [N,H,W]]) of one size each, already normalised.  Adam; the step size
    ramps up linearly over the first 3% of the schedule, then decays as a
    cosine; stops at the deadline (time.time()) if given."""
    import torch

    rng = np.random.default_rng(seed)
    dev = [(torch.tensor(g[0], dtype=torch.float32, device="cuda").to(torch.bfloat16),
            torch.tensor(g[1], dtype=torch.float32, device="cuda"),
            torch.tensor(g[2], dtype=torch.float32, device="cuda") if len(g) > 2 else None) for g in groups]
    steps_per_epoch = sum(math.ceil(len(g[0]) / batch) for g in groups)
    total = epochs * steps_per_epoch
    t = 0
    hist = []
    t_start = time.time()
    for ep in range(epochs):
        if deadline is not None and time.time() > deadline:
            if log:
                log(f"stopped at the time limit after {ep} epochs")
            break
        order = [(g, idx) for g, gr in enumerate(groups)
                 for idx in np.array_split(rng.permutation(len(gr[0])), math.ceil(len(gr[0]) / batch))]
        rng.shuffle(order)
        el = 0.0
        for g, idx in order:
            x, y, mk = dev[g]
            it = torch.tensor(idx, device="cuda")
            xb = x.index_select(0, it).contiguous()
            yb = y.index_select(0, it).contiguous()
            if mk is None:
                mask = torch.ones(xb.shape[:3], dtype=torch.float32, device="cuda")
            else:
                mask = mk.index_select(0, it).contiguous()
            out = model.forward(xb, periodic, train=True)
            loss, dy = net.mse(out, yb, mask)
            model.backward(dy)
            t += 1
            frac = t / total
            if deadline is not None:  # the schedule also follows the time left
                frac = max(frac, (time.time() - t_start) / max(deadline - t_start, 1.0))
            model.adam(step_size(lr, frac), t)
            el += loss
        hist.append(el / len(order))
        if log and (ep % 10 == 0 or ep == epochs - 1):
            log(f"epoch {ep} loss {hist[-1]:.4e}")
    return hist


def evaluate(ctx, model: net.UNet, models, refs) -> Dict:
    """Held-out domains: guess error and iterations/time from each start."""
    out = {}
    starts = {"zero": [guess.zero_guess(m) for m in models], "learned": guess.learned_guesses(model, models)}
    for name, gs in starts.items():
        errs = []
        for (gu, gv), (u, v), m in zip(gs, refs, models):
            js, is_ = m.owned_vertex_slices()
            num = np.linalg.norm(np.concatenate([(gu - u)[js, is_].ravel(), (gv - v)[js, is_].ravel()]))
            den = np.linalg.norm(np.concatenate([u[js, is_].ravel(), v[js, is_].ravel()]))
            errs.append(num / den)
        for prec_name, prec, extra in (("fp64_colpc", solver.FP64, {}),
                                       ("mixed_colpc_cg", solver.MIXED,
                                        {"which_sparse": configs.SPARSE_PCG_CHRONGEAR})):
            ms_ = [m.copy(**extra) for m in models]
            us, vs, sts, ms = solve_models(ctx, ms_, precision=prec, guesses=gs, batch=len(models))
            sol_err = [float(np.linalg.norm(np.concatenate([(a - u).ravel(), (b - v).ravel()])) /
                             np.linalg.norm(np.concatenate([u.ravel(), v.ravel()])))
                       for a, b, (u, v) in zip(us, vs, refs)]
            out[f"{name}/{prec_name}"] = {
                "guess_rel_err": float(np.mean(errs)),
                "picard_iters": float(np.mean([s["picard_iters"] for s in sts])),
                "pcg_iters": float(np.mean([s["pcg_iters_total"] for s in sts])),
                "status": sorted({int(s["status"]) for s in sts}),
                "ms_total": float(sum(ms)),
                "solution_rel_err_vs_fp64_zero": float(np.max(sol_err)),
            }
    return out


def marine_heldout(count: int, seed: int = 70000):
    """Held-out members drawn exactly as the marine workload (configs.marine
    with its parameters) at 256 x 256 cells, dx = 2 km, seeds past every
    training seed."""
    return [configs.marine(n=256, dx=2000.0, seed=seed + i).copy(**MARINE_SOLVE) for i in range(count)]


def learned_marine(model: net.UNet, models, arrays):
    """The network's guesses for same-size non-periodic domains."""
    import torch

    F = np.stack([net.normalized_input(model, net.pad_grid(net.input_features(m, a, model.n_in)))
                  for m, a in zip(models, arrays)])
    x = torch.tensor(F, dtype=torch.float32, device="cuda").to(torch.bfloat16)
    out = model.forward(x.contiguous(), int(models[0].periodic), train=False).cpu().numpy() * model.out_scale
    return [net.guess_from_grid(m, o, a["active_vertex"]) for m, o, a in zip(models, out, arrays)]


def evaluate_marine(ctx, model: net.UNet, models) -> Dict:
    """Held-out marine domains, all in one resident problem per path: the
    plain path (FP64, diagonal preconditioner, the workload's
    Chronopoulos-Gear PCG) from zero, and FP64 / mixed with the column
    preconditioner from zero and from the learned guess; iterations, time,
    the guess's error and each answer's distance to the plain one."""
    arrays = [solver.prepare(m)[0].arrays for m in models]
    learned = learned_marine(model, models, arrays)
    zero = [guess.zero_guess(m) for m in models]
    paths = (("plain_fp64_diag", solver.FP64, dict(which_precond=configs.PRECOND_DIAG), zero),
             ("fp64_colpc", solver.FP64, {}, zero), ("mixed_colpc", solver.MIXED, {}, zero),
             ("learned_fp64_colpc", solver.FP64, {}, learned), ("learned_mixed_colpc", solver.MIXED, {}, learned))
    out, ref = {}, None
    for name, prec, extra, gs in paths:
        ms_ = [m.copy(**extra) for m in models]
        us, vs, sts, ms = solve_models(ctx, ms_, precision=prec, guesses=gs, batch=len(models))
        if ref is None:
            ref = list(zip(us, vs))
        rel = [float(np.linalg.norm(np.concatenate([(a - u).ravel(), (b - v).ravel()])) /
                     np.linalg.norm(np.concatenate([u.ravel(), v.ravel()]))) for a, b, (u, v) in zip(us, vs, ref)]
        gerr = [float(np.linalg.norm(np.concatenate([(g[0] - u).ravel(), (g[1] - v).ravel()])) /
                      np.linalg.norm(np.concatenate([u.ravel(), v.ravel()]))) for g, (u, v) in zip(gs, ref)]
        out[name] = {"picard_iters": float(np.mean([s["picard_iters"] for s in sts])),
                     "pcg_iters": float(np.mean([s["pcg_iters_total"] for s in sts])),
                     "status": sorted({int(s["status"]) for s in sts}), "ms_total": float(sum(ms)),
                     "guess_rel_err": float(np.mean(gerr)), "max_rel_l2_vs_plain": float(np.max(rel))}
    return out


def main_marine(a, log):
    ctx = solver.Context(0)
    t0 = time.time()
    sizes = [int(x) for x in a.sizes.split(",")]
    sets = make_marine_set(ctx, sizes, a.count, a.seed, a.solve_batch, log=log,
                           deadline=t0 + 60.0 * a.data_minutes)
    t_data = time.time() - t0
    ntrain = sum(len(v[0]) for v in sets.values())
    log(f"solved {ntrain} training domains in {t_data:.0f} s")
    model = net.UNet(n_out=24, seed=a.seed)
    act = np.concatenate([v[3].reshape(-1) for v in sets.values()]) > 0
    allf = np.concatenate([v[1].reshape(-1, model.n_in) for v in sets.values()])[act]
    allt = np.concatenate([v[2].reshape(-1, 24) for v in sets.values()])[act]
    shift = allf.mean(axis=0)
    scale = 1.0 / np.maximum(allf.std(axis=0), 1e-6)
    shift[4], scale[4] = 0.0, 1.0  # the mask stays -1/0/1
    model.in_shift, model.in_scale = shift.astype(np.float32), scale.astype(np.float32)
    model.out_scale = float(np.sqrt(np.mean(allt[:, :22] ** 2)))
    del allf, allt
    groups = [(net.normalized_input(model, v[1]), v[2] / model.out_scale, v[3]) for v in sets.values()]
    log(f"U-Net parameters: {model.params()}")
    t1 = time.time()
    # the family's domains are doubly periodic (the ice sheet sits inside
    # an ocean that reaches every edge), as the marine workload is
    hist = train(model, groups, a.epochs, a.lr, a.batch, a.seed, log=log, periodic=1,
                 deadline=t1 + 60.0 * a.train_minutes)
    t_train = time.time() - t1
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    model.save(a.out)
    ev = evaluate_marine(ctx, model, marine_heldout(a.heldout))
    report = {"family": "marine", "params": model.params(),
              "train_domains": {str(n): len(v[0]) for n, v in sets.items()}, "data_seconds": t_data,
              "epochs_run": len(hist), "final_loss": hist[-1] if hist else None, "train_seconds": t_train,
              "heldout": a.heldout, "eval": ev}
    log(json.dumps(report, indent=1))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)
    ctx.close()


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--family", default="marine", choices=["marine", "slab"])
    ap.add_argument("--out", default=None)
    ap.add_argument("--count", type=int, default=2000, help="marine: training domains")
    ap.add_argument("--sizes", default="128,160,192,224,256", help="marine: cells per side")
    ap.add_argument("--solve-batch", type=int, default=16, help="marine: domains per resident problem")
    ap.add_argument("--data-minutes", type=float, default=20.0, help="marine: time limit of the data generation")
    ap.add_argument("--train-minutes", type=float, default=15.0, help="marine: time limit of the training")
    ap.add_argument("--train96", type=int, default=640)
    ap.add_argument("--train160", type=int, default=128)
    ap.add_argument("--heldout", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--lr", type=float, default=6e-4)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)

    def log(s):
        print(s, flush=True)

    if a.family == "marine":
        a.out = a.out or os.path.join(os.path.dirname(__file__), "weights", "unet_marine.npz")
        main_marine(a, log)
        return
    a.out = a.out or os.path.join(os.path.dirname(__file__), "weights", "unet_slab.npz")
    ctx = solver.Context(0)
    t0 = time.time()
    sets = []
    for n, count, sd in ((96, a.train96, a.seed), (160, a.train160, a.seed + 1)):
        if count > 0:
            sets.append(make_set(ctx, count, n, sd, batch=16 if n == 96 else 8))
            log(f"solved {len(sets[-1][0])} training domains of {n}x{n} ({time.time() - t0:.0f} s)")
    model = net.UNet(n_out=24, seed=a.seed, n_in=5)  # the slab family's five features (net.features)
    allf = np.concatenate([s[1].reshape(-1, 5) for s in sets])
    allt = np.concatenate([s[2].reshape(-1, 24) for s in sets])
    shift = allf.mean(axis=0)
    scale = 1.0 / np.maximum(allf.std(axis=0), 1e-6)
    shift[4], scale[4] = 0.0, 1.0  # the mask stays 0/1
    model.in_shift, model.in_scale = shift.astype(np.float32), scale.astype(np.float32)
    model.out_scale = float(np.sqrt(np.mean(allt[:, :2 * 11] ** 2)))
    groups = [((s[1] - shift) * scale, s[2] / model.out_scale) for s in sets]
    log(f"U-Net parameters: {model.params()}")
    t1 = time.time()
    hist = train(model, groups, a.epochs, a.lr, a.batch, a.seed, log=log)
    t_train = time.time() - t1
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    model.save(a.out)
    held = make_set(ctx, a.heldout, 160, a.seed + 1000, batch=8)
    ev = evaluate(ctx, model, held[0], held[3])
    report = {"params": model.params(), "train_domains": [len(s[0]) for s in sets], "epochs": a.epochs,
              "final_loss": hist[-1], "train_seconds": t_train, "heldout": len(held[0]), "eval": ev}
    log(json.dumps(report, indent=1))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)
    ctx.close()


if __name__ == "__main__":
    main()
