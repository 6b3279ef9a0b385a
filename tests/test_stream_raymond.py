"""The reference's idealised ice stream (tests/stream/runStream.py,
stream.config) against Raymond's (2000) analytic profile.

A 1000 m slab on a bed sloping at 1e-3 has a till yield stress (the
yield-stress sliding law, which_ho_babc = 2) of 5.2 kPa inside a 50 km
stream and 70 kPa (above the 8.9 kPa driving stress) outside it.  Raymond's
solution, u = 2A/(n+1) ((tau_d - tau_0)/H)^n (w^(n+1) - |y|^(n+1)), is the
depth-integrated lateral-shear balance: the shallow-shelf solve follows it
to 0.4 % of the centre-line speed at the reference's resolution (2 km, 25
cells across the stream, 2 levels), the Blatter-Pattyn solve, which also
resolves the vertical shear at the margins, to 1.8 %.  Both pin the oracle
on the reference's own test case; the device bodies, run as the engine
runs them (the host emulator, the oracle's PCG as the linear solver), give
the oracle's Picard count and velocity.
"""
import numpy as np
import pytest

from cism_b200 import configs
from oracle import oracle

from helpers import rel_l2
from test_velocity_l1l2 import emulated_picard


def _profile(m, u):
    """The surface speed across the stream (mean along flow) and the
    vertex rows' y."""
    js, is_ = m.owned_vertex_slices()
    gy = m.ny - 4
    y0 = m.dy * (np.arange(gy) + 1) - m.dy * gy / 2.0
    return y0, u[js, is_, 0].mean(axis=1), np.ptp(u[js, is_, 0], axis=1).max()


@pytest.mark.parametrize("approx,tol", [(configs.APPROX_SSA, 0.006), (0, 0.025)], ids=["ssa", "bp"])
def test_stream_follows_raymond(approx, tol):
    m = configs.raymond_stream().copy(approx_2d=approx)
    assert (m.nx - 4, m.ny - 4) == (15, 31)  # stream.config's ewn, nsn
    solve = oracle.velo_ssa_solve if approx == configs.APPROX_SSA else oracle.velo_higher_solve
    u, v, _, _, st = solve(m)
    assert st["status"] == 0
    y0, us, spread = _profile(m, u)
    ua = configs.raymond_uvel(y0)
    assert np.abs(us - ua).max() <= tol * ua.max()
    assert spread <= 1e-6 * ua.max()  # uniform along flow
    # symmetric about the centre line: rows y0 and -y0 (the last row, at
    # the periodic seam, has no partner)
    assert np.abs(us[:-1] - us[-2::-1]).max() <= 1e-6 * ua.max()


@pytest.mark.parametrize("approx", [configs.APPROX_SSA, 0], ids=["ssa", "bp"])
def test_emulated_stream_matches_oracle(approx):
    m = configs.raymond_stream().copy(approx_2d=approx)
    u, v, _, it, _ = emulated_picard(m)
    solve = oracle.velo_ssa_solve if approx == configs.APPROX_SSA else oracle.velo_higher_solve
    uo, vo, _, _, st = solve(m)
    assert it == st["picard_iters"]
    # the plastic bed's regularised beta (tau_y / |u|) at near-zero speeds
    # makes the shallow-shelf system the less well conditioned one
    assert rel_l2([u, v], [uo, vo]) < (1e-6 if approx else 1e-8)


@pytest.mark.gpu
@pytest.mark.parametrize("approx", [configs.APPROX_SSA, 0], ids=["ssa", "bp"])
def test_device_stream_matches_oracle(ctx, approx):
    m = configs.raymond_stream().copy(approx_2d=approx, pcg_maxiters=3000)
    u, v, _, st = ctx.velo_higher_solve(m)
    solve = oracle.velo_ssa_solve if approx == configs.APPROX_SSA else oracle.velo_higher_solve
    uo, vo, _, _, sto = solve(m)
    assert st["status"] == 0 and abs(st["picard_iters"] - sto["picard_iters"]) <= 1
    # the plastic bed amplifies the PCG's summation-order differences (1e-7
    # between two solves that share the oracle's PCG, shallow-shelf)
    assert rel_l2([u, v], [uo, vo]) < (1e-5 if approx else 1e-7)
    y0, us, _ = _profile(m, u)
    ua = configs.raymond_uvel(y0)
    assert np.abs(us - ua).max() <= (0.006 if approx else 0.025) * ua.max()
