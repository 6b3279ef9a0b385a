"""L1L2 branch of glissade_velo_higher_solve (solve_2d with whichapprox =
HO_APPROX_L1L2): the 2-D solve of the basal velocity with the layer
viscosities of compute_effective_viscosity_L1L2
(glissade_velo_higher.F90:7382-7618), then the 3-D velocity of
compute_3d_velocity_L1L2 (:5834-6356).

The oracle's restatement (oracle/bp_oracle.c: effective_viscosity_l1l2,
assemble_2d, velocity_3d_l1l2, orc_velo_2d_solve) is pinned by closed forms
of the discrete equations:

* a uniform slab sliding on a uniform bed has no strain, so the basal
  velocity is the plug flow rho g H tan(theta) / beta and each layer adds
  the shallow-ice increment 2 A tau^3 (sigma(k+1) - sigma(k)) H with tau =
  rho g d tan(theta), d the depth of the layer midpoint (this sum tends to
  the shallow-ice surface speed A/2 (rho g tan(theta))^3 H^4 at second
  order in the layer thickness);
* with a constant viscosity eta the basal velocity is the shallow-shelf
  one, and on a slab with one Fourier mode in x the vertex equation
  4 eta H D2(u) - beta u = rho g H ds/dx of the 2-D solve turns the
  reconstruction's shear stress into tau_xz(k) = -rho g d_k ds/dx +
  sigma(k+1) (rho g H ds/dx + beta u): the membrane-stress gradient term,
  its factor 2 and the depth integral of the viscosity are fixed by it;
* a no-slip bed holds every level of a column at the (zero) basal value:
  the reference's Dirichlet branch (:6320-6329) applies at every level.
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

from cism_b200 import configs, solver
from oracle import oracle

from helpers import owned_active_rows, random_state
from test_ssa import _fourier_slab

EMU = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "hostemu",
                   "libhostemu.so")
_dp = C.POINTER(C.c_double)

RHO_G = 910.0 * 9.81


def _p(a):
    return a.ctypes.data_as(_dp)


def _shear_profile(sigma, H, A, tau_of, ub):
    """u(k) = u(k+1) + 2 A tau_eff^2 (sigma(k+1) - sigma(k)) H tau(k), the
    column integral of the reconstruction with tau_eff^2 = tau(k)^2 +
    tp^2 supplied by tau_of(k, d) -> (tau, tp)."""
    nz = len(sigma)
    u = np.zeros(np.shape(ub) + (nz,))
    u[..., -1] = ub
    for k in range(nz - 2, -1, -1):
        d = 0.5 * (sigma[k] + sigma[k + 1]) * H
        tau, tp = tau_of(k, d)
        u[..., k] = u[..., k + 1] + 2.0 * A * (tp ** 2 + tau ** 2) * (sigma[k + 1] - sigma[k]) * H * tau
    return u


@pytest.mark.parametrize("beta", [1000.0, 1.0e8])
def test_uniform_slab_is_plug_flow_plus_shallow_ice_shear(beta):
    theta, H, A = 0.5, 1000.0, 1.0e-16
    t = math.tan(math.radians(theta))
    m = configs.slab(n=12, nz=11, theta_deg=theta, beta0=beta, beta1=0.0).copy(approx_2d=configs.APPROX_L1L2)
    u, v, efvs, _, st = oracle.velo_l1l2_solve(m)
    assert st["status"] == 0
    ub = RHO_G * H * t / beta
    e = _shear_profile(configs.sigma_glide(m.nz), H, A, lambda k, d: (RHO_G * d * t, 0.0), ub)
    js, is_ = m.owned_vertex_slices()
    assert np.abs(u[js, is_, :] - e).max() <= 1e-12 * np.abs(e).max()
    assert np.abs(v).max() <= 1e-12 * np.abs(u).max()
    assert np.all(efvs[2:-2, 2:-2] > 0.0)


def test_shallow_ice_sum_converges_at_second_order():
    """The closed form above against the continuous shallow-ice surface
    speed: the midpoint sum converges at second order in the layers."""
    theta, H, A = 0.5, 1000.0, 1.0e-16
    t = math.tan(math.radians(theta))
    exact = 0.5 * A * (RHO_G * t) ** 3 * H ** 4
    errs = []
    for nz in (11, 21, 41):
        e = _shear_profile(configs.sigma_glide(nz), H, A, lambda k, d: (RHO_G * d * t, 0.0), 0.0)
        errs.append(abs(e[0] - exact) / exact)
    assert 3.8 < errs[0] / errs[1] < 4.2 and 3.8 < errs[1] / errs[2] < 4.2


def test_constant_viscosity_matches_the_shallow_shelf_and_the_membrane_identity():
    n = 32
    m, k, u0, U = _fourier_slab(n)
    uS, _, _, _, stS = oracle.velo_ssa_solve(m)
    uL, vL, _, _, stL = oracle.velo_l1l2_solve(m)
    assert stS["status"] == stL["status"] == 0 and stS["picard_iters"] == stL["picard_iters"]
    assert np.abs(uL[..., -1] - uS[..., -1]).max() <= 1e-12 * np.abs(uS).max()
    su = oracle.setup(m)
    js, is_ = m.owned_vertex_slices()
    row = uL[js, is_, :][n // 2]  # owned vertices x = i dx, i = 1..n
    ub = row[:, -1]
    sx = su["dusrf_dx"][js, is_][n // 2]
    H, eta, A, beta = 1000.0, m.efvs_constant, 1.0e-16, m.beta_const
    ux = (ub - np.roll(ub, 1)) / m.dx  # the cell west of each vertex
    tp = eta * (np.abs(ux) + np.abs(np.roll(ux, -1)))  # 2 eta |ux| staggered over the W and E cells
    s = su["sigma"]
    e = _shear_profile(s, H, A, lambda kk, d: (-RHO_G * d * sx + s[kk + 1] * (RHO_G * H * sx + beta * ub), tp), ub)
    assert np.abs(row - e).max() <= 1e-12 * np.abs(row).max()
    assert np.ptp(row[:, 0] - row[:, -1]) > 0.1  # the shear varies along the mode
    assert np.abs(vL).max() <= 1e-12 * np.abs(uL).max()


def test_no_slip_bed_holds_every_level():
    m = configs.slab(n=12, nz=11, theta_deg=0.5).copy(which_babc=configs.BABC_NO_SLIP,
                                                      approx_2d=configs.APPROX_L1L2)
    u, v, _, _, st = oracle.velo_l1l2_solve(m)
    assert st["status"] == 0 and st["picard_iters"] == 1
    assert np.all(u == 0.0) and np.all(v == 0.0)


def _l1l2_models():
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
    return [m.copy(approx_2d=configs.APPROX_L1L2) for m in (m1, m2, m3, m4)]


@pytest.mark.parametrize("m", _l1l2_models(), ids=lambda m: m.name)
def test_device_l1l2_assembly_bodies_match_oracle(m):
    """The device's 2-D assembly bodies with the L1L2 layer viscosities
    (l1l2_point_efvs in qp2_element_point, the per-layer point mean of
    k_asm2_qp) on the host plan, compiled for the CPU, against the oracle's
    assembled L1L2 system at a random velocity: 1e-13 relative."""
    emu = C.CDLL(EMU)
    prep, _, _ = solver.prepare(m)
    su = oracle.setup(m)
    u, v = random_state(m, su, seed=5, scale=30.0)
    A, bu, bv, efvs, nnz = oracle.assemble_2d_system(m, su, su["beta_internal"], u[..., -1], v[..., -1],
                                                     oracle.APPROX_L1L2)
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
    # a viscosity per layer (not the shallow-shelf copy).  1e-11: near the
    # switch to its first-order form (a^3/27 = 1e-6 b^2/4) the second
    # Cardano root is b/2 + c with c = |b|/2 (1 + O(1e-6)), so a last-bit
    # difference in the strain rate (the device contracts products into
    # fused multiply-adds) grows by up to 1e6 there; the column average in
    # the matrix damps it again
    assert np.max(np.abs(eef - efvs)) <= 1e-11 * np.max(np.abs(efvs))
    if m.which_efvs == configs.EFVS_NONLINEAR:
        ac = su["active_cell"].astype(bool)
        assert np.ptp(efvs[ac], axis=1).max() > 0.0


@pytest.mark.parametrize("m", _l1l2_models(), ids=lambda m: m.name)
def test_device_l1l2_reconstruction_bodies_match_oracle(m):
    """l1l2_cell and l1l2_column (the device's compute_3d_velocity_L1L2)
    with the host scatter, compiled for the CPU, against the oracle on a
    random basal velocity and the layer viscosities of the oracle's
    assembly there: 1e-12 relative to the largest speed."""
    emu = C.CDLL(EMU)
    prep, _, _ = solver.prepare(m)
    su = oracle.setup(m)
    u, v = random_state(m, su, seed=9, scale=30.0)
    _, _, _, efvs, _ = oracle.assemble_2d_system(m, su, su["beta_internal"], u[..., -1], v[..., -1],
                                                 oracle.APPROX_L1L2)
    uo, vo = oracle.velocity_3d_l1l2(m, su, efvs, u, v)
    ue, ve = np.ascontiguousarray(u.copy()), np.ascontiguousarray(v.copy())
    rc = emu.emu_velocity_3d_l1l2(C.byref(prep.inputs), _p(np.ascontiguousarray(u)),
                                  _p(np.ascontiguousarray(v)), _p(np.ascontiguousarray(efvs)), _p(ue), _p(ve))
    assert rc == 0
    scale = max(np.abs(uo).max(), np.abs(vo).max())
    assert np.abs(ue - uo).max() <= 1e-12 * scale
    assert np.abs(ve - vo).max() <= 1e-12 * scale
    # the reconstruction changes the column (levels above the bed differ from it)
    rows = owned_active_rows(m, su["active_vertex"])
    assert np.abs(uo[rows][:, 0] - uo[rows][:, -1]).max() > 1e-6 * scale


def test_l1l2_plan_options():
    """The plan refuses the column preconditioner for the L1L2 solve and an
    L1L2 problem without its fields; the setup hands over the surface
    gradient it computed."""
    emu = C.CDLL(EMU)
    m = _l1l2_models()[1]
    prep, _, _ = solver.prepare(m.copy(which_precond=configs.PRECOND_SIA))
    out = np.zeros((m.ny - 1, m.nx - 1))
    u = np.zeros(m.vshape3)
    assert emu.emu_slide_beta(C.byref(prep.inputs), _p(u), _p(u), _p(out)) == 10
    prep, _, _ = solver.prepare(m)
    su = oracle.setup(m)
    assert np.array_equal(prep.arrays["dusrf_dx"], su["dusrf_dx"])
    assert np.array_equal(prep.arrays["dusrf_dy"], su["dusrf_dy"])
    prep.inputs.l1l2 = C.cast(None, C.POINTER(solver.L1L2))
    assert emu.emu_slide_beta(C.byref(prep.inputs), _p(u), _p(u), _p(out)) == 10


# ---------------------------------------------------------------------------
# GPU: the L1L2 Picard solve and 3-D velocity against the oracle
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("m", _l1l2_models(), ids=lambda m: m.name)
def test_device_l1l2_picard_matches_oracle(ctx, m):
    from helpers import rel_l2

    m = m.copy(pcg_maxiters=3000)
    u, v, efvs, st = ctx.velo_higher_solve(m)
    uo, vo, eo, _, sto = oracle.velo_l1l2_solve(m)
    assert st["status"] == sto["status"] == 0, (st, sto)
    assert st["picard_iters"] == sto["picard_iters"]
    assert rel_l2([u, v], [uo, vo]) < 1e-8
    assert np.abs(efvs - eo).max() <= 1e-6 * np.abs(eo).max()


@pytest.mark.gpu
def test_device_l1l2_uniform_slab_profile(ctx):
    theta, H, A, beta = 0.5, 1000.0, 1.0e-16, 1000.0
    t = math.tan(math.radians(theta))
    m = configs.slab(n=12, nz=11, theta_deg=theta, beta0=beta, beta1=0.0).copy(approx_2d=configs.APPROX_L1L2)
    u, v, _, st = ctx.velo_higher_solve(m)
    assert st["status"] == 0
    e = _shear_profile(configs.sigma_glide(m.nz), H, A, lambda k, d: (RHO_G * d * t, 0.0), RHO_G * H * t / beta)
    js, is_ = m.owned_vertex_slices()
    assert np.abs(u[js, is_, :] - e).max() <= 1e-9 * np.abs(e).max()


@pytest.mark.gpu
def test_device_l1l2_no_slip_bed_is_zero(ctx):
    m = configs.dome().copy(approx_2d=configs.APPROX_L1L2)
    u, v, _, st = ctx.velo_higher_solve(m)
    assert st["status"] == 0 and st["picard_iters"] == 1
    assert np.all(u == 0.0) and np.all(v == 0.0)


def emulated_picard(m, uvel=None, vvel=None):
    """The 2-D Picard loop through the device bodies in the engine's launch
    order, the oracle's PCG as its linear solver (tests/hostemu
    emu_picard): (uvel, vvel, efvs, picard iterations, prepared)."""
    emu = C.CDLL(EMU)
    prep, u, v = solver.prepare(m, uvel, vvel)
    uo, vo = np.ascontiguousarray(u.copy()), np.ascontiguousarray(v.copy())
    ef = np.zeros((m.ny, m.nx, m.nz - 1))
    it = C.c_int(0)
    rc = emu.emu_picard(C.byref(prep.inputs), _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(v)),
                           _p(uo), _p(vo), _p(ef), C.byref(it))
    assert rc == 0
    return uo, vo, ef, it.value, prep


@pytest.mark.parametrize("m", _l1l2_models(), ids=lambda m: m.name)
def test_emulated_l1l2_picard_loop_matches_oracle(m):
    """The composition of the device's L1L2 steps (the loop order, the
    layer viscosities, the reconstruction after the loop) against the
    oracle's solve: the same Picard count and the 3-D velocity to 1e-9."""
    from helpers import rel_l2

    m = m.copy(pcg_maxiters=3000)
    u, v, ef, it, _ = emulated_picard(m)
    uo, vo, eo, _, sto = oracle.velo_l1l2_solve(m)
    assert sto["status"] == 0 and it == sto["picard_iters"]
    assert rel_l2([u, v], [uo, vo]) < 1e-9
    # 1e-6 as on the GPU: the Cardano switch amplifies last-bit strain-rate
    # differences up to 1e6 (see the assembly test above)
    assert np.abs(ef - eo).max() <= 1e-6 * np.abs(eo).max()


@pytest.mark.parametrize("resid", [0, 1, 2])
@pytest.mark.parametrize("approx", [0, configs.APPROX_L1L2], ids=["bp", "l1l2"])
def test_emulated_picard_criteria_match_oracle(approx, resid):
    """The Picard criteria (which_ho_resid 0 max, 1 max without the bed
    level, 2 mean; the 2-D solves have no bed level to leave out) with the
    Chronopoulos-Gear PCG, through the emulated device loop."""
    from helpers import rel_l2

    m = configs.dome(n=15, nz=6, radius=12.0e3, hmax=1000.0).copy(
        which_babc=configs.BABC_BETA_EXTERNAL, which_resid=resid, approx_2d=approx,
        which_sparse=configs.SPARSE_PCG_CHRONGEAR, pcg_maxiters=2000)
    m.beta_external = np.full_like(m.beta_external, 400.0)
    u, v, _, it, _ = emulated_picard(m)
    if approx:
        uo, vo, _, _, sto = oracle.velo_l1l2_solve(m)
    else:
        uo, vo, _, _, sto = oracle.velo_higher_solve(m)
    assert sto["status"] == 0 and it == sto["picard_iters"]
    assert rel_l2([u, v], [uo, vo]) < 1e-9
