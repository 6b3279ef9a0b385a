"""Post-solve diagnostics of glissade_velo_higher_solve
(glissade_velo_higher.F90:3847-3872): compute_internal_stress (:6968-7195)
and compute_basal_friction_heatflx (:6755-6964), both bfric methods.

CPU: the device's per-element and per-cell/column bodies with the
engine's scatters (compiled for the CPU by tests/hostemu) against the
oracle's restatement at random halo-consistent velocities, relative 1e-12
(the bodies form the basis-function derivatives with fused multiply-adds,
the restatement without), for the 3-D solve and for the 3-D elements of
the 2-D solves (shallow-shelf, L1L2, DIVA).  GPU: bp_problem_diagnostics at
a converged solution against the oracle at that solution, relative 1e-10.
"""
import ctypes as C
import os

import numpy as np
import pytest

from cism_b200 import configs, solver
from oracle import oracle

from helpers import random_state

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU = os.path.join(ROOT, "tests", "hostemu", "libhostemu.so")
_dp = C.POINTER(C.c_double)
NAMES = ("tau_xz", "tau_yz", "tau_xx", "tau_yy", "tau_xy", "tau_eff")


def _p(a):
    return a.ctypes.data_as(_dp)


def _models():
    out = []
    m = configs.dome()
    m = m.copy(which_babc=configs.BABC_BETA_EXTERNAL, beta_external=np.full_like(m.beta_external, 300.0))
    m.name = "dome_sliding"
    out.append(m)
    out.append(configs.slab(n=24))
    out.append(configs.marine(n=40, dx=4000.0))
    m = configs.dome(n=20).copy(periodic=0, which_babc=configs.BABC_BETA_EXTERNAL)
    m.beta_external = np.full_like(m.beta_external, 500.0)
    m.name = "dome_outflow"
    out.append(m)
    m = configs.dome().copy(which_efvs=configs.EFVS_FLOWFACT)
    m.name = "dome_flowfact"
    out.append(m)
    return out


MODELS = _models()


def _close(a, b, tol):
    scale = max(np.max(np.abs(b)), 1e-300)
    return np.max(np.abs(a - b)) <= tol * scale


def _emu(m, prep, u, v, beta, which):
    emu = C.CDLL(EMU)
    tau = {k: np.full((m.ny, m.nx, m.nz - 1), np.nan) for k in NAMES}
    bf = np.full((m.ny, m.nx), np.nan)
    rc = emu.emu_diagnostics(C.byref(prep.inputs), _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(v)),
                             _p(np.ascontiguousarray(beta)) if beta is not None else C.cast(None, _dp),
                             which, *[_p(tau[k]) for k in NAMES], _p(bf))
    assert rc == 0
    return tau, bf


@pytest.mark.parametrize("which", [0, 1])
@pytest.mark.parametrize("m", MODELS, ids=lambda m: m.name)
def test_diagnostic_bodies_match_oracle(m, which):
    prep, _, _ = solver.prepare(m)
    su = oracle.setup(m)
    u, v = random_state(m, su, seed=3, scale=50.0)
    tau, bf = _emu(m, prep, u, v, None, which)
    ref = oracle.internal_stress(m, su, u, v)
    for k in NAMES:
        assert np.all(np.isfinite(tau[k])), k
        assert _close(tau[k], ref[k], 1e-12), k
    rbf = oracle.basal_friction_heatflx(m, su, u, v, su["beta_internal"], which)
    assert np.all(np.isfinite(bf))
    assert _close(bf, rbf, 1e-12)
    if m.which_babc != configs.BABC_NO_SLIP:
        assert np.max(rbf) > 0.0


@pytest.mark.parametrize("which", [0, 1])
def test_heat_flux_with_a_sliding_law_uses_the_given_beta(which):
    m = configs.with_sliding(configs.slab(n=24), configs.BABC_POWERLAW, seed=1)
    prep, _, _ = solver.prepare(m)
    su = oracle.setup(m)
    u, v = random_state(m, su, seed=4, scale=30.0)
    beta = oracle.setup(m, u, v)["beta_internal"]
    _, bf = _emu(m, prep, u, v, beta, which)
    assert _close(bf, oracle.basal_friction_heatflx(m, su, u, v, beta, which), 1e-12)


def test_stress_of_a_uniform_shear_is_exact():
    """u = a z on a flat slab (all other gradients zero): tau_xz = efvs a,
    tau_eff = |tau_xz|, every other component zero -- an analytic check of
    the restatement independent of its arithmetic."""
    m = configs.slab(n=12, theta_deg=0.0).copy(which_efvs=configs.EFVS_CONSTANT)
    su = oracle.setup(m)
    sigma, H = su["sigma"], 1000.0
    a = 1.0e-3  # 1/a
    u = np.zeros(m.vshape3)
    u[...] = -a * sigma * H  # z = s - sigma H: du/dz = a
    ref = oracle.internal_stress(m, su, u, np.zeros(m.vshape3))
    act = su["active_cell"].astype(bool)
    assert np.allclose(ref["tau_xz"][act], m.efvs_constant * a, rtol=1e-12)
    assert np.allclose(ref["tau_eff"][act], m.efvs_constant * a, rtol=1e-12)
    for k in ("tau_yz", "tau_xx", "tau_yy", "tau_xy"):
        assert np.max(np.abs(ref[k])) <= 1e-12 * m.efvs_constant * a


def _models_2d():
    out = []
    for approx, name in ((configs.APPROX_SSA, "ssa"), (configs.APPROX_L1L2, "l1l2"),
                         (configs.APPROX_DIVA, "diva")):
        m = MODELS[0].copy(approx_2d=approx)
        m.name = f"dome_sliding_{name}"
        out.append(m)
        m = configs.marine(n=32, dx=4000.0).copy(periodic=0, approx_2d=approx,
                                                 which_assemble_beta=configs.ASSEMBLE_STANDARD)
        m.name = f"marine_outflow_{name}"
        out.append(m)
    return out


@pytest.mark.parametrize("which", [0, 1])
@pytest.mark.parametrize("m", _models_2d(), ids=lambda m: m.name)
def test_diagnostic_bodies_of_2d_solves_match_oracle(m, which):
    """compute_internal_stress's shallow-shelf branch (horizontal gradients
    and viscosity only), its L1L2 branch (the layer viscosity efvs(k,i,j)
    at every point) and the 3-D branch for DIVA, on the 3-D elements of a
    2-D solve through the engine's diagnostics view, against the oracle at
    a random 3-D velocity; the heat flux from its basal level."""
    emu = C.CDLL(EMU)
    prep, _, _ = solver.prepare(m)
    su = oracle.setup(m)
    u, v = random_state(m, su, seed=6, scale=50.0)
    rng = np.random.default_rng(7)
    efvs = rng.uniform(1e5, 1e7, (m.ny, m.nx, m.nz - 1))
    for k in range(m.nz - 1):
        efvs[..., k] = configs.halo_fill_cells(np.ascontiguousarray(efvs[..., k]), m.periodic)
    tau = {k: np.full((m.ny, m.nx, m.nz - 1), np.nan) for k in NAMES}
    bf = np.full((m.ny, m.nx), np.nan)
    rc = emu.emu_diagnostics_2d(C.byref(prep.inputs), _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(v)),
                                _p(efvs), which, *[_p(tau[k]) for k in NAMES], _p(bf))
    assert rc == 0
    ref = oracle.internal_stress(m, su, u, v, approx=m.approx_2d, efvs=efvs)
    for k in NAMES:
        assert np.all(np.isfinite(tau[k])), k
        assert _close(tau[k], ref[k], 1e-12), k
    if m.approx_2d == configs.APPROX_SSA:
        assert not ref["tau_xz"].any() and not ref["tau_yz"].any()
    else:
        assert np.max(np.abs(ref["tau_xz"])) > 0.0
    rbf = oracle.basal_friction_heatflx(m, su, u, v, su["beta_internal"], which)
    assert _close(bf, rbf, 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("which", [0, 1])
def test_device_diagnostics_at_solution_match_oracle(ctx, which):
    for m in (configs.slab(n=24), MODELS[0]):
        m = m.copy(pcg_maxiters=2000)
        prep, u0, v0 = solver.prepare(m)
        prob = ctx.problem([prep])
        prob.set_guess([u0], [v0])
        st = prob.run()[0]
        assert st["status"] == 0, st
        us, vs, _ = prob.get()
        d = prob.diagnostics(which)[0]
        prob.close()
        su = oracle.setup(m)
        ref = oracle.internal_stress(m, su, us[0], vs[0])
        for k in NAMES:
            assert _close(d[k], ref[k], 1e-10), k
        rbf = oracle.basal_friction_heatflx(m, su, us[0], vs[0], su["beta_internal"], which)
        assert _close(d["bfricflx"], rbf, 1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("m", _models_2d()[::2], ids=lambda m: m.name)
def test_device_diagnostics_of_2d_solves_match_oracle(ctx, m):
    """bp_problem_diagnostics after a shallow-shelf, L1L2 or DIVA solve: the
    3-D elements with the solve's 3-D velocity (and L1L2's layer
    viscosities) against the oracle at that solution, relative 1e-10."""
    m = m.copy(pcg_maxiters=3000)
    prep, u0, v0 = solver.prepare(m)
    prob = ctx.problem([prep])
    prob.set_guess([u0], [v0])
    st = prob.run()[0]
    assert st["status"] == 0, st
    us, vs, es = prob.get(want_efvs=True)
    su = oracle.setup(m)
    for which in (0, 1):
        d = prob.diagnostics(which)[0]
        ref = oracle.internal_stress(m, su, us[0], vs[0], approx=m.approx_2d, efvs=es[0])
        for k in NAMES:
            assert _close(d[k], ref[k], 1e-10), k
        rbf = oracle.basal_friction_heatflx(m, su, us[0], vs[0], su["beta_internal"], which)
        assert _close(d["bfricflx"], rbf, 1e-10)
    prob.close()
