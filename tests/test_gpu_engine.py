"""GPU tests of the engine's execution paths: the device-resident Picard
loop against the host-driven one, and the learned guess behind the C ABI
against the network's Python forward.

Tolerances: device loop vs host loop, bitwise (the same kernels in the
same order); the C-ABI guess vs the Python forward of the same weights,
1e-6 relative
(identical arithmetic and BF16 rounding points; a last-bit difference of
log10 can move one BF16 input by one unit).
"""
import os

import numpy as np
import pytest

from cism_b200 import configs, solver

from helpers import rel_l2, small_models

pytestmark = pytest.mark.gpu

MODELS = {m.name: m for m in small_models()}


class _Env:
    """Set environment switches the engine reads when it builds a problem or
    starts a run, and restore them."""

    def __init__(self, **kw):
        self.kw = kw
        self.old = {}

    def __enter__(self):
        for k, v in self.kw.items():
            self.old[k] = os.environ.get(k)
            os.environ[k] = v

    def __exit__(self, *a):
        for k, v in self.old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


@pytest.mark.parametrize("precision", [solver.FP64, solver.MIXED])
def test_device_loop_equals_host_loop(ctx, precision):
    m = configs.marine(n=40, dx=4000.0).copy(pcg_maxiters=2000, which_resid=configs.RESID_L2NORM_RELATIVE,
                                             which_precond=configs.PRECOND_SIA)
    prep, u0, v0 = solver.prepare(m, precision=precision)
    out = {}
    for loop in ("0", "1"):
        with _Env(BP_DEVICE_LOOP=loop):
            prob = ctx.problem([prep])
            prob.set_guess([u0], [v0])
            prob.run()  # first run: the autotuner, then the device loop takes over
            prob.set_guess([u0], [v0])
            st = prob.run()[0]  # a whole run in the device loop
            u, v, _ = prob.get()
            prob.close()
        out[loop] = (u[0], v[0], st)
    (ua, va, sa), (ub, vb, sb) = out["0"], out["1"]
    assert sa["status"] == sb["status"] == 0
    assert (sa["picard_iters"], sa["pcg_iters_total"]) == (sb["picard_iters"], sb["pcg_iters_total"])
    assert np.array_equal(ua, ub) and np.array_equal(va, vb)


def _random_network(seed=3, n_in=6):
    from cism_b200 import net

    model = net.UNet(n_out=24, seed=seed, n_in=n_in)
    model.in_shift = np.array([1.0, 0.1, -0.1, 2.5, 0.0, 4.0][:n_in], np.float32)
    model.in_scale = np.array([0.8, 0.5, 0.5, 1.2, 1.0, 2.0][:n_in], np.float32)
    model.out_scale = 35.0
    return model


@pytest.mark.parametrize("n_in", [5, 6])
def test_learned_guess_c_abi_matches_python(ctx, tmp_path, n_in):
    """Five inputs, or six with the flow-law factor channel."""
    torch = pytest.importorskip("torch")
    from cism_b200 import net

    model = _random_network(n_in=n_in)
    path = str(tmp_path / "net.npz")
    model.save(path)
    ctx.load_guess(path)
    ms = [configs.marine(n=40, dx=4000.0, seed=s) for s in (11, 12)]
    preps = [solver.prepare(m, guess_mode=solver.GUESS_LEARNED)[0] for m in ms]
    prob = ctx.problem(preps)
    n0 = ctx.guess_launches()
    prob.set_guess([None, None], [None, None])
    assert ctx.guess_launches() > n0
    gu, gv = prob.get_guess()
    prob.close()
    # the Python forward of the same weights on the same features
    F = np.stack([net.normalized_input(model, net.pad_grid(net.input_features(m, p.arrays, n_in)))
                  for m, p in zip(ms, preps)])
    x = torch.tensor(F, dtype=torch.float32, device="cuda").to(torch.bfloat16).contiguous()
    out = model.forward(x, int(ms[0].periodic), train=False).cpu().numpy() * model.out_scale
    for m, p, o, u, v in zip(ms, preps, out, gu, gv):
        pu, pv = net.guess_from_grid(m, o, p.arrays["active_vertex"])
        av = p.arrays["active_vertex"].astype(bool)
        assert np.abs(pu).max() > 0.0
        assert rel_l2([u[av], v[av]], [pu[av], pv[av]]) < 1e-6


def test_learned_start_converges_to_the_plain_answer(ctx, tmp_path):
    pytest.importorskip("torch")
    model = _random_network(seed=4)
    path = str(tmp_path / "net.npz")
    model.save(path)
    ctx.load_guess(path)
    m = configs.marine(n=40, dx=4000.0, seed=7).copy(pcg_maxiters=2000, which_resid=configs.RESID_L2NORM_RELATIVE)
    prep, u0, v0 = solver.prepare(m)
    u, v, _, st = ctx.solve_prepared(prep, u0, v0, want_efvs=False)
    prep_l, _, _ = solver.prepare(m, precision=solver.MIXED, guess_mode=solver.GUESS_LEARNED)
    ul, vl, _, stl = ctx.solve_prepared(prep_l, np.zeros_like(u0), np.zeros_like(v0), want_efvs=False)
    assert st["status"] == stl["status"] == 0
    # the relative-residual criterion ends both at the same point
    assert rel_l2([ul, vl], [u, v]) < 1e-6


def test_learned_guess_needs_a_network():
    c = solver.Context(0)
    try:
        m = configs.marine(n=40, dx=4000.0)
        prep, u0, v0 = solver.prepare(m, guess_mode=solver.GUESS_LEARNED)
        with pytest.raises(solver.BPError) as e:
            c.solve_prepared(prep, u0, v0)
        assert e.value.code == 10
        with pytest.raises(solver.BPError):
            c.load_guess("/nonexistent/weights.bin")
    finally:
        c.close()


@pytest.mark.parametrize("name", ["marine", "slab"])
def test_element_centric_assembly_equals_row_form(ctx, name):
    """k_asm_elem + the gathering row kernel against the row-integrating
    kernel (BP_ASM_ELEM=0) on the same state: bitwise the same matrix,
    right-hand side and viscosity."""
    m = (configs.marine(n=40, dx=4000.0) if name == "marine" else configs.slab(n=24))
    prep, u0, v0 = solver.prepare(m)
    rng = np.random.default_rng(5)
    u = u0 + 50.0 * rng.standard_normal(u0.shape)
    v = v0 + 50.0 * rng.standard_normal(v0.shape)
    outs = []
    for flag in ("0", "1"):
        with _Env(BP_ASM_ELEM=flag):
            A, bu, bv, efvs = ctx.assemble(prep, u, v)
        outs.append(A + [bu, bv, efvs])
    assert np.count_nonzero(outs[0][0]) > 0
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
