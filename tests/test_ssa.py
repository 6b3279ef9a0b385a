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
import ctypes as C
import math
import os

import numpy as np
import pytest

from cism_b200 import configs, solver
from oracle import oracle

from helpers import owned_active_rows, random_state

EMU = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "hostemu",
                   "libhostemu.so")
_dp = C.POINTER(C.c_double)

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


def _p(a):
    return a.ctypes.data_as(_dp)


def _ssa_models():
    m1, _, _, _ = _fourier_slab(24, which_efvs=configs.EFVS_NONLINEAR)
    m1.name = "fourier_slab_glen"
    m2 = configs.dome().copy(which_babc=configs.BABC_BETA_EXTERNAL)
    m2.beta_external = np.full_like(m2.beta_external, 400.0)
    m2.name = "dome_sliding"
    m3 = configs.marine(n=32, dx=4000.0).copy(periodic=0, which_assemble_beta=configs.ASSEMBLE_STANDARD)
    m3.name = "marine_outflow_standard_beta"
    m4 = configs.dome(n=20).copy(which_babc=configs.BABC_BETA_EXTERNAL, which_efvs=configs.EFVS_FLOWFACT)
    m4.beta_external = np.full_like(m4.beta_external, 200.0)
    m4.kinbcmask = np.zeros((m4.ny - 1, m4.nx - 1), np.int32)
    m4.kinbcmask[9:11, 9:11] = 1
    m4.name = "dome_kinematic_flowfact"
    return [m.copy(approx_2d=configs.APPROX_SSA) for m in (m1, m2, m3, m4)]


@pytest.mark.parametrize("m", _ssa_models(), ids=lambda m: m.name)
def test_device_ssa_bodies_match_oracle(m):
    """The device's 2-D assembly bodies (pass 1 per cell and point, the
    9-point rows with the basal and Dirichlet terms) on the host plan,
    compiled for the CPU, against the oracle's assembled shallow-shelf
    system at a random velocity: 1e-13 relative."""
    emu = C.CDLL(EMU)
    prep, _, _ = solver.prepare(m)
    su = oracle.setup(m)
    u, v = random_state(m, su, seed=5, scale=30.0)
    A, bu, bv, efvs, nnz = oracle.assemble_ssa_system(m, su, su["beta_internal"], u[..., -1], v[..., -1])
    shp = (m.ny - 1, m.nx - 1, 1, 27)
    E = [np.zeros(shp) for _ in range(4)]
    ebu, ebv = np.zeros((m.ny - 1, m.nx - 1)), np.zeros((m.ny - 1, m.nx - 1))
    eef = np.zeros((m.ny, m.nx, m.nz - 1))
    rc = emu.emu_assemble_2d(C.byref(prep.inputs), _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(v)),
                              *[_p(a) for a in E], _p(ebu), _p(ebv), _p(eef))
    assert rc == 0
    rows = owned_active_rows(m, su["active_vertex"])
    for a, e in zip(A, E):
        assert np.max(np.abs(a[rows] - e[rows])) <= 1e-13 * np.max(np.abs(a[rows]))
    scale = max(np.max(np.abs(bu[rows])), np.max(np.abs(bv[rows])))
    assert np.max(np.abs(ebu[rows] - bu[rows])) <= 1e-13 * scale
    assert np.max(np.abs(ebv[rows] - bv[rows])) <= 1e-13 * scale
    assert np.max(np.abs(eef - efvs)) <= 1e-13 * np.max(np.abs(efvs))
    # only the horizontal (kA = 0) entries are set: a 9-point operator
    for e in E:
        assert not np.any(e[..., :9]) and not np.any(e[..., 18:])


def test_ssa_refuses_the_column_preconditioner():
    """The reference's 2-D preconditioner setup knows the diagonal only
    (setup_preconditioner_2d, glissade_velo_higher_pcg.F90:2269-2329); the
    plan refuses which_precond = 2 for the shallow-shelf solve."""
    emu = C.CDLL(EMU)
    m = _ssa_models()[1]
    prep, _, _ = solver.prepare(m.copy(which_precond=configs.PRECOND_SIA))
    out = np.zeros((m.ny - 1, m.nx - 1))
    u = np.zeros(m.vshape3)
    assert emu.emu_slide_beta(C.byref(prep.inputs), _p(u), _p(u), _p(out)) == 10


# ---------------------------------------------------------------------------
# GPU: the shallow-shelf Picard solve against the oracle
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("m", _ssa_models(), ids=lambda m: m.name)
def test_device_ssa_picard_matches_oracle(ctx, m):
    from helpers import rel_l2

    m = m.copy(pcg_maxiters=3000)
    u, v, efvs, st = ctx.velo_higher_solve(m)
    uo, vo, eo, _, sto = oracle.velo_ssa_solve(m)
    assert st["status"] == sto["status"] == 0, (st, sto)
    assert st["picard_iters"] == sto["picard_iters"]
    assert rel_l2([u, v], [uo, vo]) < 1e-8
    assert np.abs(efvs - eo).max() <= 1e-6 * np.abs(eo).max()


@pytest.mark.gpu
def test_device_ssa_on_a_frozen_bed_is_zero(ctx):
    m = configs.dome().copy(approx_2d=configs.APPROX_SSA)
    u, v, _, st = ctx.velo_higher_solve(m)
    assert st["status"] == 0 and st["picard_iters"] == 1
    assert np.all(u == 0.0) and np.all(v == 0.0)


def test_ssa_plan_takes_the_bed_velocity_and_fills_every_level():
    """The shallow-shelf plan starts from uvel(nz,:,:) (:1179-1180) and
    hands the 2-D solution back on every level (:3745-3750), halo-updated;
    vertices without a column keep what the caller's arrays held."""
    emu = C.CDLL(EMU)
    m = _ssa_models()[1]
    prep, u, v = solver.prepare(m)
    su = oracle.setup(m)
    u, v = random_state(m, su, seed=8, scale=20.0)
    uo, vo = np.zeros(m.vshape3), np.zeros(m.vshape3)
    assert emu.emu_velocity_roundtrip(C.byref(prep.inputs), _p(np.ascontiguousarray(u)),
                                      _p(np.ascontiguousarray(v)), _p(uo), _p(vo)) == 0
    cols = owned_active_rows(m, su["active_vertex"])
    for a, b in ((uo, u), (vo, v)):
        assert np.array_equal(a[cols], np.repeat(b[cols][:, -1:], m.nz, axis=1))
        assert np.array_equal(a, oracle.halo_stag(a, m.periodic))


@pytest.mark.parametrize("m", _ssa_models(), ids=lambda m: m.name)
def test_emulated_ssa_picard_loop_matches_oracle(m):
    """The device's shallow-shelf steps in the engine's order (the oracle's
    PCG as the linear solver) against the oracle's solve: the same Picard
    count and velocity to 1e-9."""
    from helpers import rel_l2
    from test_velocity_l1l2 import emulated_picard

    m = m.copy(pcg_maxiters=3000)
    u, v, ef, it, _ = emulated_picard(m)
    uo, vo, eo, _, sto = oracle.velo_ssa_solve(m)
    assert sto["status"] == 0 and it == sto["picard_iters"]
    assert rel_l2([u, v], [uo, vo]) < 1e-9
    # 1e-6 as on the GPU: where the flow is nearly plug flow the strain rate
    # is a small difference of large speeds, so velocities equal to 1e-9
    # give viscosities equal to about 1e-8 there
    assert np.abs(ef - eo).max() <= 1e-6 * np.abs(eo).max()
