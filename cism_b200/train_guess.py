"""Training of the learned initial guess on solutions of this solver.

    python -m cism_b200.train_guess --out cism_b200/weights/unet_slab.npz

draws seeded members of the periodic-slab family (``configs.random_slab``),
solves them with the FP64 solver from a zero start (several domains per
resident multi-instance problem), trains the U-Net on (fields -> velocity)
with the project's BF16 kernels and Adam, saves the weights with their input
and output normalisation, and evaluates held-out domains: the guess's error
and the Picard and PCG iterations and solve time from zero, shallow-ice and
learned starts.  Runs on one GPU.
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


def solve_models(ctx, models: List[configs.BPModel], precision=solver.FP64, guesses=None, batch: int = 8):
    """Solve domains (same size) in resident multi-instance problems; returns
    velocities, stats and the device time per problem."""
    us, vs, sts, ms = [], [], [], []
    for i in range(0, len(models), batch):
        group = models[i:i + batch]
        preps = [solver.prepare(m, precision=precision) for m in group]
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


def train(model: net.UNet, groups, epochs: int, lr: float, batch: int, seed: int, log=None):
    """groups: list of (features [N,H,W,5], targets [N,H,W,C]) of one size
    each, already normalised.  Adam with cosine decay of the step size."""
    import torch

    rng = np.random.default_rng(seed)
    dev = [(torch.tensor(f, dtype=torch.float32, device="cuda").to(torch.bfloat16),
            torch.tensor(t, dtype=torch.float32, device="cuda")) for f, t in groups]
    steps_per_epoch = sum(math.ceil(len(f) / batch) for f, _ in groups)
    total = epochs * steps_per_epoch
    t = 0
    hist = []
    for ep in range(epochs):
        order = [(g, idx) for g, (f, _) in enumerate(groups)
                 for idx in np.array_split(rng.permutation(len(f)), math.ceil(len(f) / batch))]
        rng.shuffle(order)
        el = 0.0
        for g, idx in order:
            x, y = dev[g]
            it = torch.tensor(idx, device="cuda")
            xb = x.index_select(0, it).contiguous()
            yb = y.index_select(0, it).contiguous()
            mask = torch.ones(xb.shape[:3], dtype=torch.float32, device="cuda")
            out = model.forward(xb, 1, train=True)
            loss, dy = net.mse(out, yb, mask)
            model.backward(dy)
            t += 1
            step = lr * 0.5 * (1.0 + math.cos(math.pi * t / total))
            model.adam(step, t)
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


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "weights", "unet_slab.npz"))
    ap.add_argument("--train96", type=int, default=640)
    ap.add_argument("--train160", type=int, default=128)
    ap.add_argument("--heldout", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--report", default=None)
    a = ap.parse_args(argv)

    def log(s):
        print(s, flush=True)

    ctx = solver.Context(0)
    t0 = time.time()
    sets = []
    for n, count, sd in ((96, a.train96, a.seed), (160, a.train160, a.seed + 1)):
        if count > 0:
            sets.append(make_set(ctx, count, n, sd, batch=16 if n == 96 else 8))
            log(f"solved {len(sets[-1][0])} training domains of {n}x{n} ({time.time() - t0:.0f} s)")
    model = net.UNet(n_out=24, seed=a.seed)
    allf = np.concatenate([s[1].reshape(-1, net.N_IN) for s in sets])
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
