"""GPU parity at the workloads' full sizes.

* The periodic slab (160 x 160 x 11) and the large marine sheet
  (400 x 400 x 11): one Picard pass from the shallow-ice velocity with
  exactly 40 PCG iterations (tolerance 0) -- setup, assembly at that
  velocity (element-centric), the Krylov matvec and both PCG variants --
  against the oracle doing the same, to 1e-10 relative L2 (the same
  algorithm for a fixed iteration count: roundoff differences only).
* The periodic slab solved to convergence against the oracle's converged
  solve frozen in tests/golden/c1_picard_oracle.npz (made by
  tests/golden/make_golden.py --c1): the same Picard count, the velocity
  at every 4th owned vertex to 1e-8 and whole-field checksums to 1e-8.
"""
import os

import numpy as np
import pytest

from cism_b200 import configs, guess, solver
from oracle import oracle

from helpers import rel_l2

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name,variant", [("c1", configs.SPARSE_PCG_STANDARD), ("c1", configs.SPARSE_PCG_CHRONGEAR),
                                          ("c2", configs.SPARSE_PCG_CHRONGEAR)])
def test_fullsize_fixed_pcg_matches_oracle(ctx, name, variant):
    m = configs.workload(name).copy(which_sparse=variant, maxiter_nonlinear=1, pcg_maxiters=40, pcg_tol=0.0)
    u0, v0 = guess.sia_guess(m)
    u, v, _, st = ctx.velo_higher_solve(m, uvel=u0, vvel=v0)
    uo, vo, _, _, sto = oracle.velo_higher_solve(m, u0, v0)
    assert st["pcg_iters_total"] == sto["pcg_iters_total"] == 40
    js, is_ = m.owned_vertex_slices()
    assert rel_l2([u[js, is_], v[js, is_]], [uo[js, is_], vo[js, is_]]) < 1e-10


def test_c1_converged_matches_oracle_fixture(ctx):
    g = np.load(os.path.join(HERE, "golden", "c1_picard_oracle.npz"))
    m = configs.workload("c1").copy(pcg_maxiters=3000)
    u, v, _, st = ctx.velo_higher_solve(m)
    assert st["status"] == 0
    assert st["picard_iters"] == int(g["picard_iters"])
    js, is_ = m.owned_vertex_slices()
    uo, vo = u[js, is_], v[js, is_]
    k = int(g["sub"])
    assert rel_l2([uo[::k, ::k], vo[::k, ::k]], [g["u_sub"], g["v_sub"]]) < 1e-8
    sums = np.array([uo.sum(), vo.sum(), (uo ** 2).sum(), (vo ** 2).sum()])
    scale = np.array([np.abs(uo).sum(), np.abs(vo).sum(), (uo ** 2).sum(), (vo ** 2).sum()])
    assert np.all(np.abs(sums - g["sums"]) <= 1e-8 * scale)
