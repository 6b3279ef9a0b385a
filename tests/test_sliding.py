"""Velocity-dependent sliding laws: calcbeta
(libglissade/glissade_basal_traction.F90:67-598) evaluated from the basal
velocity at the start of every Picard iteration
(glissade_velo_higher.F90:2502-2517).

The reference ships no fixture for these laws, so the oracle's laws are
pinned by the limits the published laws have by construction (linear and
plastic ends of the power and pseudo-plastic laws, the Coulomb bounds of
the Schoof and Tsai laws, the yield stress of the Picard yield law) and
by a second restatement of the formulas in numpy.  CPU: those checks, the
setup mirror's sliding fields bitwise, and the device's per-column body
(compiled for the CPU by tests/hostemu) bitwise against the oracle.  GPU:
Picard solves with every law against the oracle (relative L2 1e-8, the
Picard-converged parity bar of the plain path).
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

from cism_b200 import configs, solver
from oracle import oracle

from helpers import rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU = os.path.join(ROOT, "tests", "hostemu", "libhostemu.so")
_dp = C.POINTER(C.c_double)
LAWS = list(configs.SLIDING_LAWS)
SMALLNUM = 1.0e-2


def _p(a):
    return a.ctypes.data_as(_dp)


def _model(law, base="slab", **params):
    if base == "slab":
        m = configs.slab(n=24)
    else:  # dome on a flat bed at sea level: pseudo-plastic phi in its ramp
        m = configs.dome(n=21, radius=15e3, nz=8).copy(eus=0.0)
    # near-flotation effective pressure for the Schoof and Tsai laws, so that
    # both of their regimes occur at the slab's speeds
    n_scale = 0.005 if law in (11, 12) else 0.8
    return configs.with_sliding(m, law, seed=law, n_scale=n_scale, **params)


def _velocity(m, seed, scale=60.0):
    rng = np.random.default_rng(seed)
    return rng.uniform(-scale, scale, m.vshape3), rng.uniform(-scale, scale, m.vshape3)


def _numpy_calcbeta(m, su, u, v):
    """The laws once more, in numpy, at every vertex, before the halo update."""
    sl = m.sliding
    ub, vb = u[..., -1], v[..., -1]
    s0 = np.sqrt(ub ** 2 + vb ** 2 + SMALLNUM ** 2)
    speed = np.minimum(s0, sl.beta_powerlaw_umax) if sl.beta_powerlaw_umax > 0 else s0
    N = sl.effecpress_stag
    law = sl.law
    if law == 2:
        b = sl.yield_stress / s0
    elif law == 3:
        bed = m.topg[:-1, :-1] - m.eus
        ramp = sl.pseudo_plastic_phimin + ((bed - sl.pseudo_plastic_bedmin) /
                                           (sl.pseudo_plastic_bedmax - sl.pseudo_plastic_bedmin)) * \
            (sl.pseudo_plastic_phimax - sl.pseudo_plastic_phimin)
        phi = np.where(bed <= sl.pseudo_plastic_bedmin, sl.pseudo_plastic_phimin,
                       np.where(bed >= sl.pseudo_plastic_bedmax, sl.pseudo_plastic_phimax, ramp))
        b = np.tan(phi * 3.14159265358979 / 180.0) * N / (
            sl.pseudo_plastic_u0 ** sl.pseudo_plastic_q * speed ** (1.0 - sl.pseudo_plastic_q))
    elif law == 9:
        b = sl.powerlaw_c * speed ** (1.0 / sl.powerlaw_m - 1.0)
    elif law == 10:
        imask = (m.thck > 0.0).astype(np.float64)
        fl = m.flwa[..., -1]
        num = imask[1:, :-1] * fl[1:, :-1] + imask[1:, 1:] * fl[1:, 1:] + imask[:-1, :-1] * fl[:-1, :-1] + \
            imask[:-1, 1:] * fl[:-1, 1:]
        cnt = imask[1:, :-1] + imask[1:, 1:] + imask[:-1, :-1] + imask[:-1, 1:]
        flst = np.where(cnt > 0, num / np.maximum(cnt, 1.0), 0.0)
        lam = (sl.coulomb_bump_wavelength / sl.coulomb_bump_max_slope) * flst
        b = sl.coulomb_c * sl.c_space_factor_stag * N * speed ** (1.0 / 3 - 1.0) * \
            (speed + N * N * N * lam) ** (-1.0 / 3)
        b = np.minimum(b, 1.0e8)
    elif law == 11:
        mm = sl.powerlaw_m
        b = (sl.powerlaw_c * sl.coulomb_c * N /
             (sl.powerlaw_c ** mm * speed + (sl.coulomb_c * N) ** mm) ** (1.0 / mm)) * speed ** (1.0 / mm - 1.0)
        b = np.minimum(b, 1.0e8)
    elif law == 12:
        tp = sl.powerlaw_c * speed ** (1.0 / sl.powerlaw_m)
        tc = sl.coulomb_c * N
        b = np.where(tc <= tp, tc, tp) / speed
    else:  # 13
        b = sl.friction_powerlaw_k ** (-1.0 / 3.0) * N ** (1.0 / 3.0) * speed ** (1.0 / 3.0 - 1.0)
    fg = su["f_ground"]
    b = b * fg
    return np.where((fg > 0.0) & (b < m.beta_grounded_min), m.beta_grounded_min, b)


@pytest.mark.parametrize("law", LAWS)
@pytest.mark.parametrize("base", ["slab", "dome"])
def test_oracle_laws_match_numpy_restatement(law, base):
    m = _model(law, base, beta_powerlaw_umax=40.0 if law == 9 else 0.0)
    u, v = _velocity(m, seed=law)
    su = oracle.setup(m, u, v)
    ref = oracle.halo_stag(_numpy_calcbeta(m, su, su["uvel"], su["vvel"]), m.periodic)
    got = su["beta_internal"]
    assert np.all(np.isfinite(got)) and np.all(got >= 0.0)
    assert np.max(np.abs(got - ref)) <= 1e-14 * np.max(np.abs(ref))


def _oracle_beta_at(law, speed, **params):
    """Oracle beta for a uniform grounded slab at basal speed ``speed``
    (u = speed, v = 0) with N and the other fields uniform."""
    m = configs.slab(n=8)
    m = configs.with_sliding(m, law, seed=0, **params)
    m.sliding.effecpress_stag = np.full_like(m.sliding.effecpress_stag, 1.0e6)
    if m.sliding.yield_stress is not None:
        m.sliding.yield_stress = np.full_like(m.sliding.yield_stress, 3.0e4)
    if m.sliding.c_space_factor_stag is not None:
        m.sliding.c_space_factor_stag = np.ones_like(m.sliding.c_space_factor_stag)
    u = np.zeros(m.vshape3)
    u[..., -1] = speed
    su = oracle.setup(m.copy(beta_grounded_min=0.0), u, np.zeros(m.vshape3))
    js, is_ = m.owned_vertex_slices()
    b = su["beta_internal"][js, is_]
    assert np.ptp(b) == 0.0
    return float(b.flat[0]), math.sqrt(speed ** 2 + SMALLNUM ** 2)


def test_oracle_law_limits():
    """Limits that define each law (its published form), independent of the
    restated arithmetic."""
    N = 1.0e6
    # power law: linear for m = 1 (beta = C), tau = C s^(1/m) otherwise
    b, s = _oracle_beta_at(9, 37.0, powerlaw_c=2.0e3, powerlaw_m=1.0)
    assert b == pytest.approx(2.0e3, rel=1e-14)
    b, s = _oracle_beta_at(9, 37.0, powerlaw_c=2.0e3, powerlaw_m=3.0)
    assert b * s == pytest.approx(2.0e3 * s ** (1.0 / 3.0), rel=1e-13)
    # speed cap: beyond umax beta no longer falls
    b1, _ = _oracle_beta_at(9, 80.0, powerlaw_c=2.0e3, beta_powerlaw_umax=50.0)
    b2, _ = _oracle_beta_at(9, 500.0, powerlaw_c=2.0e3, beta_powerlaw_umax=50.0)
    assert b1 == b2 == pytest.approx(2.0e3 * 50.0 ** (-2.0 / 3.0), rel=1e-13)
    # yield-stress law: tau = tau_y
    b, s = _oracle_beta_at(2, 12.0)
    assert b * s == pytest.approx(3.0e4, rel=1e-14)
    # pseudo-plastic: q = 1 linear (tau_c / u0), q = 0 plastic (tau = tau_c);
    # the slab's bed is far above bedmax, so phi = phimax
    tau_c = math.tan(math.radians(40.0)) * N
    b, s = _oracle_beta_at(3, 25.0, pseudo_plastic_q=1.0)
    assert b == pytest.approx(tau_c / 100.0, rel=1e-12)
    b, s = _oracle_beta_at(3, 25.0, pseudo_plastic_q=0.0)
    assert b * s == pytest.approx(tau_c, rel=1e-12)
    # Tsai: tau = min(c N, C s^(1/m)), both branches
    for sp in (0.5, 5.0e4):
        b, s = _oracle_beta_at(12, sp, powerlaw_c=1.0e4, coulomb_c=0.42)
        assert b * s == pytest.approx(min(0.42 * N, 1.0e4 * s ** (1.0 / 3.0)), rel=1e-13)
    # Schoof: tau = c N (C^m s / (C^m s + (c N)^m))^(1/m): the power law
    # when slow, bounded by c N when fast
    for sp in (1.0e-3, 3.0, 1.0e7):
        b, s = _oracle_beta_at(11, sp, powerlaw_c=1.0e4, coulomb_c=0.42)
        assert b * s == pytest.approx(0.42 * N * (1.0e12 * s / (1.0e12 * s + (0.42 * N) ** 3)) ** (1.0 / 3.0),
                                      rel=1e-12)
        assert b * s < 0.42 * N
    b, s = _oracle_beta_at(11, 1.0e-3, powerlaw_c=1.0e4, coulomb_c=0.42)
    assert b * s == pytest.approx(1.0e4 * s ** (1.0 / 3.0), rel=1e-6)
    # Coulomb friction (Schoof 2005): tau = c N (s / (s + N^n lambda))^(1/n), below c N
    lam = (2.0 / 0.5) * 1.0e-16
    b, s = _oracle_beta_at(10, 40.0, coulomb_c=0.42)
    assert b * s == pytest.approx(0.42 * N * (s / (s + N ** 3 * lam)) ** (1.0 / 3.0), rel=1e-13)
    assert b * s < 0.42 * N
    # effective-pressure power law (p = 3, q = 1): tau = (N / k)^(1/3) s^(1/3)
    b, s = _oracle_beta_at(13, 9.0, friction_powerlaw_k=8.4e-9)
    assert b * s == pytest.approx((N / 8.4e-9) ** (1.0 / 3.0) * s ** (1.0 / 3.0), rel=1e-13)


@pytest.mark.parametrize("law", [9, 10])
def test_setup_mirror_sliding_fields_bitwise(law):
    """bp_setup's f_ground and basal-layer staggered flow factor equal the
    oracle's."""
    m = _model(law, "dome")
    prep, _, _ = solver.prepare(m)
    su = oracle.setup(m)
    assert np.array_equal(prep.arrays["f_ground"], su["f_ground"])
    if law == 10:
        imask = np.ascontiguousarray(m.thck > 0.0, dtype=np.int32)
        fl = np.ascontiguousarray(m.flwa[..., -1])
        out = np.zeros((m.ny - 1, m.nx - 1))
        L = oracle.lib()
        L.orc_stagger(m.nx, m.ny, _p(fl), _p(out), imask.ctypes.data_as(C.POINTER(C.c_int)), 1)
        assert np.array_equal(prep.arrays["flwa_basal_stag"], out)


@pytest.mark.parametrize("law", LAWS)
@pytest.mark.parametrize("base", ["slab", "dome"])
def test_device_body_matches_oracle(law, base):
    """The per-column body of k_slide_beta on the host plan, compiled for
    the CPU, against the oracle at every column's vertex: bitwise."""
    emu = C.CDLL(EMU)
    m = _model(law, base, beta_powerlaw_umax=40.0 if law == 9 else 0.0)
    u, v = _velocity(m, seed=100 + law)
    prep, pu, pv = solver.prepare(m, u, v)
    su = oracle.setup(m, u, v)
    got = np.full((m.ny - 1, m.nx - 1), np.nan)
    rc = emu.emu_slide_beta(C.byref(prep.inputs), _p(np.ascontiguousarray(pu)), _p(np.ascontiguousarray(pv)),
                            _p(got))
    assert rc == 0
    cols = np.isfinite(got)
    assert cols.sum() == int(np.sum(su["active_vertex"][m.owned_vertex_slices()]))
    assert np.array_equal(got[cols], su["beta_internal"][cols])


def test_plan_rejects_incomplete_laws():
    emu = C.CDLL(EMU)
    m = _model(12, "slab")
    m.sliding.effecpress_stag = None
    prep, u, v = solver.prepare(m)
    out = np.zeros((m.ny - 1, m.nx - 1))
    assert emu.emu_slide_beta(C.byref(prep.inputs), _p(u), _p(v), _p(out)) == 10
    with pytest.raises(ValueError):
        solver.prepare(_model(9, "slab").copy(which_babc=5))


# ---------------------------------------------------------------------------
# GPU: Picard solves with each law
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("law", LAWS)
def test_picard_with_sliding_law_matches_oracle(ctx, law):
    m = _model(law, "slab").copy(pcg_maxiters=2000)
    u, v, efvs, st = ctx.velo_higher_solve(m)
    uo, vo, eo, bo, sto = oracle.velo_higher_solve(m)
    assert st["status"] == sto["status"] == 0, (st, sto)
    assert st["picard_iters"] == sto["picard_iters"]
    assert rel_l2([u, v], [uo, vo]) < 1e-8


@pytest.mark.gpu
def test_sliding_law_with_standard_basal_assembly(ctx):
    """Face-quadrature basal term: the corner betas are regathered from the
    columns after every beta update."""
    m = _model(9, "dome").copy(which_assemble_beta=configs.ASSEMBLE_STANDARD, pcg_maxiters=2000)
    u, v, _, st = ctx.velo_higher_solve(m)
    uo, vo, _, _, sto = oracle.velo_higher_solve(m)
    assert st["status"] == sto["status"] == 0, (st, sto)
    assert st["picard_iters"] == sto["picard_iters"]
    assert rel_l2([u, v], [uo, vo]) < 1e-8


@pytest.mark.gpu
def test_batch_mixes_sliding_and_fixed_beta(ctx):
    """A batch (one nz for all instances) of two laws and a fixed beta
    equals the single solves."""
    dome11 = configs.with_sliding(configs.dome(n=21, radius=15e3, nz=11).copy(eus=0.0), 9, seed=9)
    ms = [_model(11, "slab"), configs.slab(n=20), dome11]
    ms = [m.copy(pcg_maxiters=2000) for m in ms]
    preps = [solver.prepare(m) for m in ms]
    us, vs, _, sts = ctx.batch_solve([p[0] for p in preps], [p[1] for p in preps], [p[2] for p in preps])
    for m, u, v, st in zip(ms, us, vs, sts):
        ui, vi, _, sti = ctx.velo_higher_solve(m)
        assert st["picard_iters"] == sti["picard_iters"]
        assert rel_l2([u, v], [ui, vi]) < 1e-12


def _nan_beta_model():
    """A NaN beta (a negative effective pressure under the cube root of the
    effective-pressure power law); a negative beta cannot reach the check
    where ice is grounded, since the grounded minimum raises it first
    (glissade_basal_traction.F90:560-566)."""
    m = _model(13, "slab")
    m.sliding.effecpress_stag = -np.abs(m.sliding.effecpress_stag)
    return m


def test_oracle_reports_nan_beta():
    _, _, _, _, sto = oracle.velo_higher_solve(_nan_beta_model())
    assert sto["status"] == 9


@pytest.mark.gpu
def test_nan_beta_from_sliding_law_is_reported(ctx):
    with pytest.raises(solver.BPError) as e:
        ctx.velo_higher_solve(_nan_beta_model())
    assert e.value.code == 9


@pytest.mark.parametrize("law", configs.SLIDING_LAWS)
def test_emulated_picard_loop_with_a_sliding_law_matches_oracle(law):
    """The 3-D Picard loop through the device bodies in the engine's order
    (k_slide_beta from the bed nodes, k_cell_beta, assembly, the rows), the
    oracle's PCG as the linear solver, against the oracle's solve: the same
    Picard count and the velocity to 1e-9."""
    from helpers import rel_l2
    from test_velocity_l1l2 import emulated_picard

    m = configs.with_sliding(configs.slab(n=16), law, seed=2).copy(pcg_maxiters=2000)
    u, v, ef, it, _ = emulated_picard(m)
    uo, vo, eo, _, sto = oracle.velo_higher_solve(m)
    assert sto["status"] == 0 and it == sto["picard_iters"], (it, sto)
    assert rel_l2([u, v], [uo, vo]) < 1e-9


@pytest.mark.parametrize("law", [configs.BABC_POWERLAW, configs.BABC_COULOMB_POWERLAW_SCHOOF,
                                 configs.BABC_PSEUDO_PLASTIC])
@pytest.mark.parametrize("approx", [configs.APPROX_SSA, configs.APPROX_L1L2, configs.APPROX_DIVA],
                         ids=["ssa", "l1l2", "diva"])
def test_emulated_2d_picard_loop_with_a_sliding_law_matches_oracle(approx, law):
    """The sliding laws inside the 2-D solves: the shallow-shelf and L1L2
    laws read the 2-D (basal) velocity, DIVA's the 3-D basal velocity of the
    previous iteration; the device bodies in the engine's order against the
    oracle's solve."""
    from helpers import rel_l2
    from test_velocity_l1l2 import emulated_picard

    m = configs.with_sliding(configs.slab(n=16), law, seed=5).copy(approx_2d=approx, pcg_maxiters=2000)
    u, v, ef, it, _ = emulated_picard(m)
    if approx == configs.APPROX_DIVA:
        uo, vo, eo, _, sto, _ = oracle.velo_diva_solve(m)
    else:
        uo, vo, eo, _, sto = oracle.velo_2d_solve(m, approx)
    assert sto["status"] == 0 and it == sto["picard_iters"] and it > 2, (it, sto)
    assert rel_l2([u, v], [uo, vo]) < 1e-8
