"""The learned guess's host-side pieces on the CPU: the input features of
the marine network (net.input_features, which the device's
k_guess_features restates and a GPU test compares bitwise in effect), and
bench.py's choice of paths and models for the workloads.

The sixth channel is checked against a direct computation from the
setup's own arrays: log10 of the mean flow-law factor over the layers of
the active cells around each owned vertex."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from cism_b200 import configs, net, solver  # noqa: E402


@pytest.mark.parametrize("seed", [11, 12])
def test_flow_factor_channel_is_the_mean_over_active_cells(seed):
    rng = np.random.default_rng(seed)
    m = configs.random_marine(rng, n=48, dx=4000.0)
    a = solver.prepare(m)[0].arrays
    f6 = net.input_features(m, a)
    f5 = net.input_features(m, a, 5)
    assert f6.shape[-1] == 6 and f5.shape[-1] == 5
    assert np.array_equal(f6[..., :5], f5)  # the five channels are unchanged
    js, is_ = m.owned_vertex_slices()
    fl = np.asarray(a["flwafact"])
    ac = np.asarray(a["active_cell"]) != 0
    act = f6[..., 4] != 0
    for jj, j in enumerate(range(js.start, js.stop)):
        for ii, i in enumerate(range(is_.start, is_.stop)):
            if not act[jj, ii]:
                assert f6[jj, ii, 5] == 0.0
                continue
            vals = [fl[j + dj, i + di, k] for dj, di in ((0, 0), (0, 1), (1, 0), (1, 1))
                    if ac[j + dj, i + di] for k in range(fl.shape[-1])]
            assert vals
            assert f6[jj, ii, 5] == pytest.approx(np.log10(np.mean(vals)), rel=1e-12, abs=1e-12)


def test_flow_factor_channel_follows_the_rate_factor():
    # flwafact = 0.5 A^(-1/3): a fourfold rate factor lowers the channel by log10(4)/3
    m1 = configs.marine(n=32, dx=8000.0, seed=3, flwa=1.0e-16)
    m4 = configs.marine(n=32, dx=8000.0, seed=3, flwa=4.0e-16)
    f1 = net.input_features(m1, solver.prepare(m1)[0].arrays)
    f4 = net.input_features(m4, solver.prepare(m4)[0].arrays)
    act = f1[..., 4] != 0
    assert np.allclose(f1[..., 5][act] - f4[..., 5][act], np.log10(4.0) / 3.0, atol=1e-12)


def _args(*argv):
    return bench.parse_args(list(argv))


def test_bench_paths_of_the_marine_workload():
    names = [p.name for p in bench.paths_for(_args("--workload", "c4"), True)]
    assert names == ["plain_fp64", "mixed_batched", "sia_mixed_batched", "learned_fp64_batched",
                     "learned_mixed_batched"]
    assert bench.headline_name(bench.paths_for(_args("--workload", "c4"), True)) == "learned_mixed_batched"
    # without a network the learned paths are absent and the headline is the last path
    names = [p.name for p in bench.paths_for(_args("--workload", "c4"), False)]
    assert names == ["plain_fp64", "mixed_batched", "sia_mixed_batched"]
    # a single marine domain (c2) is solved one at a time
    names = [p.name for p in bench.paths_for(_args("--workload", "c2"), True)]
    assert names == ["plain_fp64", "mixed", "sia_mixed", "learned_fp64", "learned_mixed"]
    # --paths picks by name, the diagonal-preconditioner P included
    names = [p.name for p in bench.paths_for(_args("--workload", "c4", "--paths", "plain_fp64_diag,mixed_batched"),
                                             True)]
    assert names == ["mixed_batched", "plain_fp64_diag"]


def test_bench_models_and_networks():
    ms = bench.make_models(_args("--workload", "c4", "--batch", "3"))
    assert len(ms) == 3
    assert all(m.which_precond == configs.PRECOND_SIA for m in ms)  # the reference's default
    assert all(m.which_resid == configs.RESID_L2NORM_RELATIVE and m.pcg_maxiters == 5000 for m in ms)
    assert len({float(np.sum(m.topg)) for m in ms}) == 3  # three different held-out domains
    assert bench.make_models(_args("--workload", "c4", "--picard", "maxu"))[0].which_resid == 0
    # the marine network serves c4, c2 and the c3 ensemble; a given file overrides
    for w in ("c4", "c2", "c3"):
        assert bench.weights_path(w) and bench.weights_path(w).endswith("unet_marine.bin")
    assert bench.weights_path("c1") is None
    assert bench.weights_path("c1", os.path.join(ROOT, "cism_b200", "weights", "unet_marine.bin"))
    assert bench.weights_path("c4", "/nonexistent.bin") is None


def test_training_step_size_schedule():
    from cism_b200.train_guess import step_size

    lr = 6e-4
    assert step_size(lr, 0.0) == 0.0
    assert step_size(lr, 0.015) == pytest.approx(lr / 2)  # halfway up the ramp
    assert step_size(lr, 0.03) == pytest.approx(lr)  # the peak
    assert step_size(lr, 0.03 + 0.97 / 2) == pytest.approx(lr / 2)  # halfway down the cosine
    assert step_size(lr, 1.0) == pytest.approx(0.0, abs=1e-18)
    assert step_size(lr, 1.5) == pytest.approx(0.0, abs=1e-18)  # past the deadline: stays at zero
    xs = np.linspace(0.03, 1.0, 50)
    ys = [step_size(lr, x) for x in xs]
    assert all(a >= b for a, b in zip(ys, ys[1:]))  # monotone decay after the ramp
