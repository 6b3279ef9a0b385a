"""Shallow-shelf (SSA) branch of glissade_velo_higher_solve (solve_2d with
whichapprox = HO_APPROX_SSA): the oracle's restatement
(oracle/bp_oracle.c, orc_velo_ssa_solve) pinned by the closed-form SSA
solution of a periodic slab whose surface carries one Fourier mode.

With constant viscosity eta, thickness H and friction beta, v = 0 and
d/dy = 0, the SSA balance d/dx(4 eta H du/dx) - beta u = rho g H ds/dx with
s = -x tan(theta) + A sin(kx) has the solution
u = rho g H tan(theta) / beta - rho g H A k cos(kx) / (4 eta H k^2 + beta):
the uniform part exactly (no strain), the Fourier mode to the bilinear
elements' second order.
"""
import math

import numpy as np
import pytest

from cism_b200 import configs
from oracle import oracle

RHO_G = 910.0 * 9.81


def _fourier_slab(n, length=32.0e3, amp=10.0, H=1000.0, beta=1000.0, eta=2.0e6, theta=0.1, **kw):
    dx = length / n
    m = configs.slab(n=n, dx=dx, theta_deg=theta)
    k = 2.0 * math.pi / length
    t = math.tan(math.radians(theta))
    xc = (np.arange(n) + 0.5) * dx
    s_owned = np.tile(-xc * t + amp * np.sin(k * xc), (n, 1))
    usrf = configs.halo_fill_cells(configs._embed(s_owned), offset_ew=length * t)
    thck = configs.halo_fill_cells(configs._embed(np.full((n, n), H)))
    opts = dict(usrf=usrf, thck=thck, topg=usrf - thck, which_babc=configs.BABC_BETA_CONSTANT,
                beta_const=beta, which_efvs=configs.EFVS_CONSTANT, efvs_constant=eta, pcg_maxiters=5000)
    m = m.copy(**(opts | kw))
    u0 = RHO_G * H * t / beta
    U = -RHO_G * H * amp * k / (4.0 * eta * H * k * k + beta)
    return m, k, u0, U


def _modes(m, u, k):
    js, is_ = m.owned_vertex_slices()
    n = m.nx - 4
    row = u[js, is_, 0][n // 2]
    xv = (np.arange(n) + 1) * m.dx
    return np.mean(row), 2.0 / n * np.sum(row * np.cos(k * xv))


def test_ssa_matches_the_fourier_solution():
    m, k, u0, U = _fourier_slab(32)
    u, v, efvs, beta, st = oracle.velo_ssa_solve(m)
    assert st["status"] == 0 and st["picard_iters"] == 2  # linear: the second pass changes nothing
    mean, amp = _modes(m, u, k)
    assert mean == pytest.approx(u0, rel=1e-12)
    assert amp == pytest.approx(U, rel=2e-3)
    assert np.max(np.abs(v)) <= 1e-12 * np.max(np.abs(u))
    js, is_ = m.owned_vertex_slices()
    assert np.ptp(u[js, is_, 0], axis=0).max() <= 1e-10 * np.max(np.abs(u))  # uniform in y
    # the 2-D solution on every level
    assert np.all(u == u[..., :1])


def test_ssa_converges_at_second_order():
    errs = []
    for n in (8, 16, 32):
        m, k, u0, U = _fourier_slab(n)
        u, _, _, _, st = oracle.velo_ssa_solve(m)
        assert st["status"] == 0
        errs.append(abs(_modes(m, u, k)[1] - U) / abs(U))
    assert 3.8 < errs[0] / errs[1] < 4.2
    assert 3.8 < errs[1] / errs[2] < 4.2


def test_ssa_with_glen_law_keeps_the_plug_flow():
    """A uniform slope on a sliding bed is pure plug flow in the SSA: no
    strain, so Glen's viscosity (with its strain-rate floor) does not enter
    and u = rho g H tan(theta) / beta exactly."""
    m, k, u0, U = _fourier_slab(16, amp=0.0, which_efvs=configs.EFVS_NONLINEAR)
    u, _, _, _, st = oracle.velo_ssa_solve(m)
    assert st["status"] == 0
    js, is_ = m.owned_vertex_slices()
    assert np.allclose(u[js, is_, :], u0, rtol=1e-10)


def test_ssa_on_a_frozen_bed_is_zero():
    """The reference sets the SSA velocity to zero on a no-slip bed
    (glissade_velo_higher.F90:3227-3240)."""
    m = configs.dome()
    u, v, _, _, st = oracle.velo_ssa_solve(m)
    assert st["picard_iters"] == 1
    assert np.all(u == 0.0) and np.all(v == 0.0)
