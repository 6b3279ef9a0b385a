"""DIVA branch of glissade_velo_higher_solve (whichapprox = HO_APPROX_DIVA,
after Goldberg 2011): the 2-D solve of the depth-mean velocity with
beta_eff = beta / (1 + beta omega), the layer viscosities of
compute_effective_viscosity_diva (glissade_velo_higher.F90:7622-7864), the
integrals of compute_integrals_diva (:5601-5726) and the 3-D velocity of
compute_3d_velocity_diva (:5730-5830) after every iteration.

The oracle's restatement (oracle/bp_oracle.c: effective_viscosity_diva,
integrals_diva, orc_assemble_diva_system, orc_velocity_3d_diva,
orc_velo_diva_solve) is pinned by closed forms of the discrete equations:

* a uniform slab with a constant viscosity eta has no strain: the basal
  traction is the driving stress tau_b = rho g H tan(theta), omega_k(k) is
  the midpoint sum of depth / eta over the layers below level k, the basal
  velocity tau_b / beta, the velocity u(k) = tau_b / beta + tau_b omega_k(k)
  and the mean velocity tau_b (1 / beta + omega), all exactly;
* with Glen's law the same slab converges to the shallow-ice profile of the
  layer midpoints (the viscosity's fixed point is 1 / (2 A tau^2)), the
  profile the L1L2 reconstruction gives in closed form;
* on a no-slip bed beta_eff = 1 / omega makes the basal velocity zero;
* on the Fourier slab with constant viscosity the mean velocity solves the
  shallow-shelf equation with beta_eff: the uniform part exactly, the mode
  at the elements' second order.
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

from cism_b200 import configs, solver
from oracle import oracle

from helpers import owned_active_rows, random_state
from test_ssa import _fourier_slab, _modes

EMU = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "hostemu",
                   "libhostemu.so")
_dp = C.POINTER(C.c_double)

RHO_G = 910.0 * 9.81


def _p(a):
    return a.ctypes.data_as(_dp)


def _omega_k(sigma, H, visc):
    """omega_k(k): sum over the layers below level k of depth / efvs dz."""
    nz = len(sigma)
    om = np.zeros(nz)
    for k in range(nz - 2, -1, -1):
        d = 0.5 * (sigma[k] + sigma[k + 1])
        om[k] = om[k + 1] + d / visc(k, d) * (sigma[k + 1] - sigma[k]) * H
    return om


def _slab(beta=1000.0, **kw):
    return configs.slab(n=12, nz=11, theta_deg=0.5, beta0=beta, beta1=0.0).copy(
        approx_2d=configs.APPROX_DIVA, **kw)


def test_uniform_slab_with_constant_viscosity_is_exact():
    eta, H, beta = 2.0e6, 1000.0, 1000.0
    m = _slab(beta, which_efvs=configs.EFVS_CONSTANT, efvs_constant=eta)
    u, v, efvs, _, st, ex = oracle.velo_diva_solve(m)
    assert st["status"] == 0
    s = configs.sigma_glide(m.nz)
    tb = RHO_G * H * math.tan(math.radians(0.5))
    omk = _omega_k(s, H, lambda k, d: eta)
    om = sum(0.5 * (omk[k] + omk[k + 1]) * (s[k + 1] - s[k]) for k in range(m.nz - 1))
    js, is_ = m.owned_vertex_slices()
    e = tb / beta + tb * omk
    assert np.abs(u[js, is_, :] - e).max() <= 1e-12 * e.max()
    assert np.abs(ex["btractx"][js, is_] - tb).max() <= 1e-12 * tb
    assert np.abs(ex["uvel_2d"][js, is_] - tb * (1.0 / beta + om)).max() <= 1e-12 * e.max()
    assert np.abs(v).max() <= 1e-12 * e.max()
    assert np.all(efvs[2:-2, 2:-2] == eta)


def test_uniform_slab_with_glen_law_reaches_the_shallow_ice_profile():
    H, A, beta = 1000.0, 1.0e-16, 1000.0
    m = _slab(beta)
    u, v, _, _, st, ex = oracle.velo_diva_solve(m)
    assert st["status"] == 0 and st["picard_iters"] > 5
    s = configs.sigma_glide(m.nz)
    tb = RHO_G * H * math.tan(math.radians(0.5))
    e = tb / beta + tb * _omega_k(s, H, lambda k, d: 1.0 / (2.0 * A * (tb * d) ** 2))
    js, is_ = m.owned_vertex_slices()
    assert np.abs(u[js, is_, :] - e).max() <= 1e-3 * e.max()  # the Picard tolerance, 1e-4 per step


def test_no_slip_bed_has_zero_basal_velocity():
    eta, H = 2.0e6, 1000.0
    m = _slab(which_efvs=configs.EFVS_CONSTANT, efvs_constant=eta, which_babc=configs.BABC_NO_SLIP)
    u, v, _, _, st, ex = oracle.velo_diva_solve(m)
    assert st["status"] == 0
    s = configs.sigma_glide(m.nz)
    tb = RHO_G * H * math.tan(math.radians(0.5))
    js, is_ = m.owned_vertex_slices()
    us = u[js, is_, :]
    assert np.abs(us[..., -1]).max() <= 1e-10 * us.max()
    assert np.abs(us - tb * _omega_k(s, H, lambda k, d: eta)).max() <= 1e-10 * us.max()


def test_fourier_slab_mean_velocity_is_the_shallow_shelf_with_beta_eff():
    errs = []
    for n in (8, 16, 32):
        m, k, _, _ = _fourier_slab(n)
        m = m.copy(approx_2d=configs.APPROX_DIVA)
        _, _, _, _, st, ex = oracle.velo_diva_solve(m)
        assert st["status"] == 0
        H, eta, beta = 1000.0, m.efvs_constant, m.beta_const
        s = configs.sigma_glide(m.nz)
        omk = _omega_k(s, H, lambda kk, d: eta)
        om = sum(0.5 * (omk[kk] + omk[kk + 1]) * (s[kk + 1] - s[kk]) for kk in range(m.nz - 1))
        be = beta / (1.0 + beta * om)
        t = math.tan(math.radians(0.1))
        U = -RHO_G * H * 10.0 * k / (4.0 * eta * H * k * k + be)
        mean, amp = _modes(m, np.repeat(ex["uvel_2d"][..., None], m.nz, axis=2), k)
        assert mean == pytest.approx(RHO_G * H * t / be, rel=1e-12)
        errs.append(abs(amp - U) / abs(U))
    assert 3.8 < errs[0] / errs[1] < 4.2 and 3.8 < errs[1] / errs[2] < 4.2


def test_state_carries_over_between_solves():
    """A second solve from the first one's velocity, traction and
    viscosities starts at the fixed point: one Picard iteration."""
    m = _slab()
    u, v, efvs, _, st, ex = oracle.velo_diva_solve(m)
    u2, v2, _, _, st2, ex2 = oracle.velo_diva_solve(m, u, v, efvs=efvs, **ex)
    assert st["picard_iters"] > 5 and st2["picard_iters"] <= 2
    assert np.abs(u2 - u).max() <= 1e-3 * np.abs(u).max()


def _diva_models():
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
    m5 = configs.dome().copy(which_assemble_beta=configs.ASSEMBLE_STANDARD)
    m5.name = "dome_no_slip_standard"
    return [m.copy(approx_2d=configs.APPROX_DIVA) for m in (m1, m2, m3, m4, m5)]


def _random_diva_state(m, su, seed):
    rng = np.random.default_rng(seed)
    u, v = random_state(m, su, seed=seed, scale=30.0)
    av = su["active_vertex"].astype(bool)
    bx = configs.halo_fill_stag(rng.uniform(-5e4, 5e4, (m.ny - 1, m.nx - 1)) * av, m.periodic)
    by = configs.halo_fill_stag(rng.uniform(-5e4, 5e4, (m.ny - 1, m.nx - 1)) * av, m.periodic)
    ef = rng.uniform(1e5, 1e7, (m.ny, m.nx, m.nz - 1))
    for k in range(m.nz - 1):  # halo-updated, as the reference's caller leaves efvs
        ef[..., k] = configs.halo_fill_cells(np.ascontiguousarray(ef[..., k]), m.periodic)
    if seed % 2:  # no viscosity yet: the strain-rate floor's value starts the iteration
        ef[:] = 0.0
    return u, v, dict(uvel_2d=u[..., 0].copy(), vvel_2d=v[..., 0].copy(), btractx=bx, btracty=by, efvs=ef)


@pytest.mark.parametrize("seed", [1, 2])
@pytest.mark.parametrize("m", _diva_models(), ids=lambda m: m.name)
def test_device_diva_bodies_match_oracle(m, seed):
    """One DIVA iteration's device bodies (the point viscosities, the omega
    integrals, beta_eff, the rows with the basal and Dirichlet terms, the
    traction and the 3-D velocity) on the host plan, compiled for the CPU,
    against the oracle: 1e-13 relative for the system, 1e-12 for the
    viscosities, integrals and velocities."""
    emu = C.CDLL(EMU)
    su = oracle.setup(m)
    u, v, st0 = _random_diva_state(m, su, seed)
    m = m.copy(diva_state=st0)
    prep, pu, pv = solver.prepare(m, u, v)
    A_ = prep.arrays
    nx, ny, nz = m.nx, m.ny, m.nz
    # the oracle's setup masks, with a DIVA no-slip bed carrying no bed mask
    if m.which_babc == configs.BABC_NO_SLIP:
        kin = np.zeros((ny - 1, nx - 1), bool) if m.kinbcmask is None else m.kinbcmask == 1
        su["umask_dirichlet"][..., -1] = kin
        su["vmask_dirichlet"][..., -1] = kin
    eq3 = np.ascontiguousarray(np.repeat(st0["efvs"][:, :, None, :], 4, axis=2))
    A, bu, bv, efvs, omk, omg, be, nnz = oracle.assemble_diva_system(
        m, su, su["beta_internal"], A_["uvel_2d"], A_["vvel_2d"], st0["btractx"], st0["btracty"], eq3)
    bxo, byo, uo, vo = oracle.velocity_3d_diva(m, su, be, omk, omg, A_["uvel_2d"], A_["vvel_2d"], pu, pv)
    shp = (ny - 1, nx - 1, 1, 27)
    E = [np.zeros(shp) for _ in range(4)]
    ebu, ebv = np.zeros((ny - 1, nx - 1)), np.zeros((ny - 1, nx - 1))
    eef = np.zeros((ny, nx, nz - 1))
    eeq = np.zeros((ny, nx, 4, nz - 1))
    eomk, eom, ebe = np.zeros((ny, nx, nz)), np.zeros((ny, nx)), np.zeros((ny - 1, nx - 1))
    ue, ve = np.ascontiguousarray(pu.copy()), np.ascontiguousarray(pv.copy())
    rc = emu.emu_diva_step(C.byref(prep.inputs), *[_p(a) for a in E], _p(ebu), _p(ebv), _p(eef), _p(eeq),
                           _p(eomk), _p(eom), _p(ebe), _p(ue), _p(ve))
    assert rc == 0
    rows = owned_active_rows(m, su["active_vertex"])
    for a, e in zip(A, E):
        assert np.max(np.abs(a[rows] - e[rows])) <= 1e-13 * np.max(np.abs(a[rows]))
    scale = max(np.max(np.abs(bu[rows])), np.max(np.abs(bv[rows])))
    assert np.max(np.abs(ebu[rows] - bu[rows])) <= 1e-13 * scale
    assert np.max(np.abs(ebv[rows] - bv[rows])) <= 1e-13 * scale
    ac = su["active_cell"].astype(bool)
    assert np.max(np.abs(eef - efvs)) <= 1e-12 * np.max(np.abs(efvs))
    assert np.max(np.abs(eeq[ac] - eq3[ac])) <= 1e-12 * np.max(np.abs(eq3[ac]))
    assert np.max(np.abs(eomk[ac] - omk[ac])) <= 1e-12 * np.max(np.abs(omk[ac]))
    assert np.max(np.abs(eom[ac] - omg[ac])) <= 1e-12 * np.max(np.abs(omg[ac]))
    assert np.max(np.abs(ebe[rows] - be[rows])) <= 1e-12 * np.max(np.abs(be[rows]))
    vs = max(np.abs(uo).max(), np.abs(vo).max())
    assert np.abs(ue - uo).max() <= 1e-12 * vs and np.abs(ve - vo).max() <= 1e-12 * vs
    bs = max(np.abs(bxo).max(), np.abs(byo).max())
    assert np.abs(A_["btractx"] - bxo).max() <= 1e-12 * bs and np.abs(A_["btracty"] - byo).max() <= 1e-12 * bs
    assert np.array_equal(A_["ice_plus_land_mask"] == 1, (su["ice_mask"] == 1) | (su["land_mask"] == 1))


def test_diva_setup_and_plan_options():
    """bp_setup starts a Dirichlet column's mean velocity from its bed
    velocity and zeroes it at owned inactive vertices, sets no bed mask
    for a no-slip DIVA solve; the plan refuses the column preconditioner
    and a DIVA problem without its state."""
    emu = C.CDLL(EMU)
    m = _diva_models()[3]
    su = oracle.setup(m)
    u, v, st0 = _random_diva_state(m, su, 4)
    prep, pu, pv = solver.prepare(m.copy(diva_state=st0), u, v)
    kin = m.kinbcmask == 1
    assert np.array_equal(prep.arrays["uvel_2d"][kin], u[..., -1][kin])
    js, is_ = m.owned_vertex_slices()
    own = np.zeros(kin.shape, bool)
    own[js, is_] = True
    dead = own & (su["active_vertex"] == 0)
    assert np.all(prep.arrays["uvel_2d"][dead] == 0.0) and np.all(prep.arrays["vvel_2d"][dead] == 0.0)
    prep2, _, _ = solver.prepare(_diva_models()[4])
    assert not prep2.arrays["umask_dirichlet"].any()
    out = np.zeros((m.ny - 1, m.nx - 1))
    z = np.zeros(m.vshape3)
    prep3, _, _ = solver.prepare(m.copy(which_precond=configs.PRECOND_SIA))
    assert emu.emu_slide_beta(C.byref(prep3.inputs), _p(z), _p(z), _p(out)) == 10
    prep.inputs.diva = C.cast(None, C.POINTER(solver.Diva))
    assert emu.emu_slide_beta(C.byref(prep.inputs), _p(z), _p(z), _p(out)) == 10


# ---------------------------------------------------------------------------
# GPU: the DIVA Picard solve against the oracle
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("m", _diva_models(), ids=lambda m: m.name)
def test_device_diva_picard_matches_oracle(ctx, m):
    from helpers import rel_l2

    m = m.copy(pcg_maxiters=3000)
    u, v, efvs, st = ctx.velo_higher_solve(m)
    uo, vo, eo, _, sto, ex = oracle.velo_diva_solve(m)
    assert st["status"] == sto["status"] == 0, (st, sto)
    assert st["picard_iters"] == sto["picard_iters"]
    assert rel_l2([u, v], [uo, vo]) < 1e-8
    d = st["diva"]
    assert rel_l2([d["uvel_2d"], d["vvel_2d"]], [ex["uvel_2d"], ex["vvel_2d"]]) < 1e-8
    assert rel_l2([d["btractx"], d["btracty"]], [ex["btractx"], ex["btracty"]]) < 1e-8
    assert np.abs(efvs - eo).max() <= 1e-6 * np.abs(eo).max()


@pytest.mark.gpu
def test_device_diva_uniform_slab_profile(ctx):
    eta, H, beta = 2.0e6, 1000.0, 1000.0
    m = _slab(beta, which_efvs=configs.EFVS_CONSTANT, efvs_constant=eta)
    u, v, _, st = ctx.velo_higher_solve(m)
    assert st["status"] == 0
    s = configs.sigma_glide(m.nz)
    tb = RHO_G * H * math.tan(math.radians(0.5))
    e = tb / beta + tb * _omega_k(s, H, lambda k, d: eta)
    js, is_ = m.owned_vertex_slices()
    assert np.abs(u[js, is_, :] - e).max() <= 1e-10 * e.max()


@pytest.mark.parametrize("m", _diva_models(), ids=lambda m: m.name)
def test_emulated_diva_picard_loop_matches_oracle(m):
    """The composition of the device's DIVA steps (the point viscosities
    carried between iterations, beta_eff before the rows, the traction and
    3-D velocity after each solve, the sliding law reading the 3-D basal
    velocity) in the engine's order, the oracle's PCG as the linear solver,
    against the oracle's solve from the same carried-over state: the same
    Picard count; the 3-D velocity, mean velocity and traction to 1e-9."""
    from helpers import rel_l2
    from test_velocity_l1l2 import emulated_picard

    m = m.copy(pcg_maxiters=3000)
    su = oracle.setup(m)
    _, _, st0 = _random_diva_state(m, su, 2)
    st0 = {k: a * 0.1 for k, a in st0.items()}  # a nearby start, as the last solve's would be
    m = m.copy(diva_state=st0)
    u, v, ef, it, prep = emulated_picard(m)
    uo, vo, eo, _, sto, ex = oracle.velo_diva_solve(m, **st0)
    assert sto["status"] == 0 and it == sto["picard_iters"]
    assert rel_l2([u, v], [uo, vo]) < 1e-9
    A_ = prep.arrays
    assert rel_l2([A_["uvel_2d"], A_["vvel_2d"]], [ex["uvel_2d"], ex["vvel_2d"]]) < 1e-9
    assert rel_l2([A_["btractx"], A_["btracty"]], [ex["btractx"], ex["btracty"]]) < 1e-9
    assert np.abs(ef - eo).max() <= 1e-6 * np.abs(eo).max()


def test_emulated_diva_with_a_sliding_law_matches_oracle():
    """A power-law bed under DIVA: the law reads the 3-D basal velocity of
    the previous iteration."""
    from helpers import rel_l2
    from test_velocity_l1l2 import emulated_picard

    m = configs.with_sliding(configs.slab(n=16), configs.BABC_POWERLAW, seed=3).copy(
        approx_2d=configs.APPROX_DIVA, pcg_maxiters=3000)
    u, v, ef, it, prep = emulated_picard(m)
    uo, vo, eo, _, sto, ex = oracle.velo_diva_solve(m)
    assert sto["status"] == 0 and it == sto["picard_iters"] and it > 2
    assert rel_l2([u, v], [uo, vo]) < 1e-9


@pytest.mark.gpu
def test_device_diva_state_carries_over(ctx):
    """A second device solve from the state the first one wrote back starts
    at the fixed point, as the oracle's does."""
    from helpers import rel_l2

    m = _slab().copy(pcg_maxiters=3000)
    u, v, efvs, st = ctx.velo_higher_solve(m)
    assert st["status"] == 0 and st["picard_iters"] > 5
    m2 = m.copy(diva_state=dict(st["diva"], efvs=efvs))
    u2, v2, _, st2 = ctx.velo_higher_solve(m2, uvel=u, vvel=v)
    uo, vo, eo, _, sto, ex = oracle.velo_diva_solve(m)
    uo2, vo2, _, _, sto2, _ = oracle.velo_diva_solve(m, uo, vo, efvs=eo, **ex)
    assert st2["status"] == 0 and st2["picard_iters"] == sto2["picard_iters"] <= 2
    assert rel_l2([u2, v2], [uo2, vo2]) < 1e-8


def test_emulated_diva_state_carries_over():
    """The emulated device loop from the state its first solve wrote back
    (through the plan's scatters and the binding) needs the oracle's
    iteration count, at most two."""
    from helpers import rel_l2
    from test_velocity_l1l2 import emulated_picard

    m = _slab().copy(pcg_maxiters=3000)
    u, v, ef, it, prep = emulated_picard(m)
    st = {k: prep.arrays[k].copy() for k in ("uvel_2d", "vvel_2d", "btractx", "btracty")}
    u2, v2, _, it2, _ = emulated_picard(m.copy(diva_state=dict(st, efvs=ef)), u, v)
    uo, vo, eo, _, sto, ex = oracle.velo_diva_solve(m)
    uo2, vo2, _, _, sto2, _ = oracle.velo_diva_solve(m, uo, vo, efvs=eo, **ex)
    assert it == sto["picard_iters"] and it2 == sto2["picard_iters"] <= 2
    assert rel_l2([u2, v2], [uo2, vo2]) < 1e-9
