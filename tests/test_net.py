"""Learned-guess network: the CPU restatement (its gradients against finite
differences) and the device BF16 kernels against it.

Tolerances: the device GEMM against an FP64 product of the same BF16
operands 1e-5 relative (FP32 accumulation); network outputs and gradients
against the restatement with the same BF16 rounding points 2e-2 relative
in the L2 norm (a BF16 rounding that flips on FP32-vs-FP64 accumulation
propagates one BF16 ulp, 2^-8, through the layers that follow).
"""
import numpy as np
import pytest

from oracle import unet_oracle as uo

from helpers import rel_l2


def _tiny(rng, channels=(4, 4, 6, 6), n_in=5, n_out=3):
    convs = []
    cin = n_in
    for ch in channels:
        convs.append((rng.standard_normal((ch, 9 * cin)) * 0.3, rng.standard_normal(ch) * 0.1, True, True))
        convs.append((rng.standard_normal((ch, 9 * ch)) * 0.3, rng.standard_normal(ch) * 0.1, True, True))
        cin = ch
    for lv in range(len(channels) - 2, -1, -1):
        cin = channels[lv + 1] + channels[lv]
        convs.append((rng.standard_normal((channels[lv], 9 * cin)) * 0.3, rng.standard_normal(channels[lv]) * 0.1,
                      True, True))
        convs.append((rng.standard_normal((channels[lv], 9 * channels[lv])) * 0.3,
                      rng.standard_normal(channels[lv]) * 0.1, True, True))
    convs.append((rng.standard_normal((n_out, channels[0])) * 0.3, rng.standard_normal(n_out) * 0.1, False, False))
    return convs


@pytest.mark.parametrize("periodic", [0, 1])
def test_oracle_gradients_match_finite_differences(periodic):
    rng = np.random.default_rng(5)
    channels = (4, 4, 6, 6)
    convs = _tiny(rng, channels)
    x = rng.standard_normal((1, 8, 8, 5))
    net = uo.OracleUNet(convs, channels, bf16_points=False)
    dout = rng.standard_normal(net.forward(x, periodic).shape)
    grads = net.backward(dout, periodic)

    def loss():
        return float(np.sum(uo.OracleUNet(convs, channels, bf16_points=False).forward(x, periodic) * dout))

    h = 1e-6
    for i in (0, 3, 7, len(convs) - 2, len(convs) - 1):
        w, b, k3, act = convs[i]
        for (r, c) in ((0, 0), (w.shape[0] - 1, w.shape[1] - 1), (w.shape[0] // 2, w.shape[1] // 3)):
            old = w[r, c]
            w[r, c] = old + h
            lp = loss()
            w[r, c] = old - h
            lm = loss()
            w[r, c] = old
            fd = (lp - lm) / (2 * h)
            assert abs(fd - grads[i][0][r, c]) <= 1e-6 * max(1.0, abs(fd)), (i, r, c)
        old = b[0]
        b[0] = old + h
        lp = loss()
        b[0] = old - h
        lm = loss()
        b[0] = old
        assert abs((lp - lm) / (2 * h) - grads[i][1][0]) <= 1e-6 * max(1.0, abs(grads[i][1][0]))


def test_bf16_rounding_is_nearest_even():
    torch = pytest.importorskip("torch")
    x = np.random.default_rng(1).standard_normal(10000) * np.logspace(-8, 8, 10000)
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(uo.bf16(x), ref)


# ---------------------------------------------------------------------
# device kernels
# ---------------------------------------------------------------------
def _net_from_oracle(convs, channels, n_out):
    import torch
    from cism_b200 import net as netmod

    w0, _, k30, _ = convs[0]
    n_in = w0.shape[1] // 9 if k30 else w0.shape[1]  # the restatement's input channels
    dev = netmod.UNet(n_out=n_out, channels=channels, n_in=n_in)
    for cv, (w, b, k3, act) in zip(dev.convs(), convs):
        cv.w.copy_(torch.tensor(w, dtype=torch.float32))
        cv.b.copy_(torch.tensor(b, dtype=torch.float32))
        cv.refresh()
    return dev


def _device_setup(periodic, B=2, H=16, W=24, channels=(8, 8, 16, 16), n_out=8, seed=7):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(seed)
    convs = _tiny(rng, channels, n_out=n_out)
    # the device keeps FP32 master weights; both sides see them rounded to BF16
    convs = [(uo.bf16(w).astype(np.float32).astype(np.float64), b.astype(np.float32).astype(np.float64), k3, a)
             for (w, b, k3, a) in convs]
    x = uo.bf16(rng.standard_normal((B, H, W, 5)))
    dev = _net_from_oracle(convs, channels, n_out)
    xt = torch.tensor(x, dtype=torch.float32, device="cuda").to(torch.bfloat16).contiguous()
    return torch, rng, convs, x, dev, xt


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["tma", "tc", "mma"])
@pytest.mark.parametrize("shape", [(64, 64, 64), (100, 40, 72), (7, 130, 8), (256, 96, 1160), (300, 24, 48),
                                   (96, 1440, 64), (130, 64, 1000), (200, 128, 640), (32, 288, 8192),
                                   (64, 200, 4104)])
def test_gemm_matches_bf16_product(shape, kernel):
    # the tcgen05 kernels -- operands by TMA boxes into a four-stage ring
    # ("tma", the default) or by register-staged loads in two stages ("tc");
    # 128 x 64, 128 x 32 (at most 32 columns) and 128 x 128 tiles (N = 96,
    # 128, 200); the last two shapes split K, the weight-gradient form -- and
    # the mma.sync one against the
    # FP64 product of the same BF16 operands
    torch = pytest.importorskip("torch")
    from cism_b200 import net as netmod

    M, N, K = shape
    rng = np.random.default_rng(3)
    a = uo.bf16(rng.standard_normal((M, K)))
    b = uo.bf16(rng.standard_normal((N, K)))
    bias = rng.standard_normal(N).astype(np.float32)
    at = torch.tensor(a, dtype=torch.float32, device="cuda").to(torch.bfloat16).contiguous()
    bt = torch.tensor(b, dtype=torch.float32, device="cuda").to(torch.bfloat16).contiguous()
    out = torch.empty((M, N), dtype=torch.float32, device="cuda")
    biast = torch.tensor(bias, device="cuda")
    netmod.gemm_tn(at, bt, out, biast, M, N, K, K, K, N, kernel=kernel)
    ref = a @ b.T + bias
    assert rel_l2(out.cpu().numpy(), ref) < 1e-5
    netmod.gemm_tn(at, bt, out, None, M, N, K, K, K, N, accum=True, kernel=kernel)
    assert rel_l2(out.cpu().numpy(), 2 * (a @ b.T) + bias) < 1e-5
    assert netmod.gemm_status() == 0  # no bounded wait of the tcgen05 kernel ran out


@pytest.mark.gpu
@pytest.mark.parametrize("periodic", [0, 1])
def test_unet_forward_and_gradients_match_oracle(periodic):
    torch, rng, convs, x, dev, xt = _device_setup(periodic)
    channels = (8, 8, 16, 16)
    ref = uo.OracleUNet(convs, channels, bf16_points=True)
    yo = ref.forward(x, periodic)
    yd = dev.forward(xt, periodic, train=True)
    torch.cuda.synchronize()
    assert rel_l2(yd.cpu().numpy(), yo) < 2e-2
    dout = rng.standard_normal(yo.shape)
    go = ref.backward(dout, periodic)
    dev.backward(torch.tensor(dout, dtype=torch.float32, device="cuda"))
    torch.cuda.synchronize()
    for cv, (gw, gb) in zip(dev.convs(), go):
        assert rel_l2(cv.gw.cpu().numpy(), gw) < 2e-2
        assert rel_l2(cv.gb.cpu().numpy(), gb) < 2e-2


@pytest.mark.gpu
def test_training_steps_reduce_the_loss():
    torch, rng, convs, x, dev, xt = _device_setup(1)
    from cism_b200 import net as netmod

    target = torch.tensor(np.tanh(x[..., :1].repeat(8, axis=-1)), dtype=torch.float32, device="cuda")
    mask = torch.ones(x.shape[:3], dtype=torch.float32, device="cuda")
    losses = []
    for t in range(1, 41):
        y = dev.forward(xt, 1, train=True)
        loss, dy = netmod.mse(y, target, mask)
        dev.backward(dy)
        dev.adam(3e-3, t)
        losses.append(loss)
    assert losses[-1] < 0.5 * losses[0]


def test_bindings_match_the_c_declarations():
    """Every ctypes signature of net.py has the parameter count of its
    extern "C" definition in net_kernels.cu (the library loads without a GPU)."""
    import os
    import re

    from cism_b200 import net as netmod

    src = open(os.path.join(os.path.dirname(netmod.__file__), "csrc", "net_kernels.cu")).read()
    body = src[src.index('extern "C" {'):]
    decl = {m.group(1): len([a for a in m.group(2).split(",") if a.strip()])
            for m in re.finditer(r"\bint\s+(bpnet_\w+)\s*\(([^)]*)\)", body)}
    L = netmod.lib()
    assert decl
    for name, n in decl.items():
        assert len(getattr(L, name).argtypes) == n, name


@pytest.mark.gpu
def test_shipped_network_reduces_iterations_on_held_out_slab(ctx):
    """The trained weights shipped in cism_b200/weights: on a slab drawn from
    the family with a seed outside the training seeds, the learned start
    needs fewer Picard and PCG iterations than the zero start, and both meet
    the same convergence criteria (Picard max speed change 1e-4, PCG 1e-8),
    so the answers agree to the Picard tolerance's scale."""
    import os

    from cism_b200 import configs, guess, net as netmod, solver

    path = os.path.join(os.path.dirname(netmod.__file__), "weights", "unet_slab.npz")
    model = netmod.UNet.load(path)
    m = configs.random_slab(np.random.default_rng(424242), n=96).copy(pcg_maxiters=3000)
    u0, v0, _, st0 = ctx.velo_higher_solve(m)
    gu, gv = guess.learned_guesses(model, [m])[0]
    prep, _, _ = solver.prepare(m)
    u1, v1, _, st1 = ctx.solve_prepared(prep, gu, gv)
    assert st0["status"] == 0 and st1["status"] == 0
    js, is_ = m.owned_vertex_slices()
    guess_err = rel_l2([gu[js, is_], gv[js, is_]], [u0[js, is_], v0[js, is_]])
    assert guess_err < 0.2
    assert st1["picard_iters"] < st0["picard_iters"]
    assert st1["pcg_iters_total"] < 0.8 * st0["pcg_iters_total"]
    assert rel_l2([u1, v1], [u0, v0]) < 1e-3
