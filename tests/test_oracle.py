"""Pins of the CPU oracle (runs without a GPU).

The reference has no golden vectors and cannot be compiled here (no Fortran
compiler), so the oracle is pinned by: the reference's own slab test and its
analytic first-order solution (tests/slab/runSlab.py, plotSlab.py:143-157);
the reference's invariants (exactly symmetric element and assembled
matrices, the symmetry repair of check_symmetry_assembled_matrix_3d being
a no-op, positive diagonal); standard vs Chronopoulos-Gear agreement on the
same system; and frozen fixtures in tests/golden (regression).
"""
import math
import os

import numpy as np
import pytest

from cism_b200 import configs
from oracle import oracle

from helpers import oracle_system, owned_active_rows, rel_l2

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_sigma_levels():
    s = configs.sigma_glide(10)
    assert s[0] == 0.0 and abs(s[-1] - 1.0) < 1e-15
    su = oracle.setup(configs.dome())
    assert np.array_equal(su["sigma"], s)


@pytest.mark.parametrize("periodic", [1, 0])
def test_halo_fill_matches_oracle(periodic):
    rng = np.random.default_rng(0)
    a = rng.standard_normal((14, 17))
    ours = configs.halo_fill_cells(a.copy(), periodic, offset_ew=3.5 if periodic else 0.0,
                                   offset_ns=-1.25 if periodic else 0.0)
    ref = oracle.halo_cell(a, periodic, 3.5 if periodic else 0.0, -1.25 if periodic else 0.0)
    assert np.array_equal(ours, ref)
    b = rng.standard_normal((13, 16, 3))
    assert np.array_equal(configs.halo_fill_stag(b.copy(), periodic), oracle.halo_stag(b, periodic))


def test_slab_matches_analytic_first_order_solution():
    """The reference's slab test: n = 1 (constant viscosity), theta = 18 deg,
    eta = 10.  The model column equals the analytic first-order profile of
    plotSlab.py plus the basal slip expressed per unit horizontal area
    (analytic slip / cos(theta), the coordinate difference the script notes)."""
    m = configs.analytic_slab()
    u, v, _, _, st = oracle.velo_higher_solve(m)
    assert st["status"] == 0 and st["converged"] == 1
    ua = configs.analytic_slab_profile(m)
    col = u[12, 17, :]
    ub = ua[-1]
    expected = ua + ub * (1.0 / math.cos(math.radians(18.0)) - 1.0)
    assert np.max(np.abs(col - expected)) / np.max(np.abs(expected)) < 2e-5
    # the slab is uniform: every owned column carries the same profile
    js, is_ = m.owned_vertex_slices()
    owned = u[js, is_, :]
    assert np.max(np.abs(owned - col)) < 1e-9 * np.max(np.abs(col))
    assert np.max(np.abs(v)) < 1e-9 * np.max(np.abs(col))


@pytest.mark.parametrize("model", [configs.dome(), configs.slab(n=16), configs.marine(n=30, dx=4000.0)],
                         ids=lambda m: m.name)
def test_assembled_matrix_is_symmetric(model):
    m = model
    su, u, v, A, bu, bv, _ = oracle_system(m, seed=4)
    Auu, Auv, Avu, Avv = A
    rows = owned_active_rows(m, su["active_vertex"])
    diag = Auu[..., 13]
    assert np.all(diag[rows] > 0.0) and np.all(Avv[..., 13][rows] > 0.0)
    # A(row, col) vs A(col, row) through the stencil for interior neighbours
    W, V = m.ny - 1, m.nx - 1
    worst = 0.0
    for j in range(3, W - 2):
        for i in range(3, V - 2):
            if not rows[j, i]:
                continue
            for k in range(m.nz):
                for kA in (-1, 0, 1):
                    if not 0 <= k + kA < m.nz:
                        continue
                    for jA in (-1, 0, 1):
                        for iA in (-1, 0, 1):
                            mm = (iA + 1) + 3 * (jA + 1) + 9 * (kA + 1)
                            mt = 26 - mm
                            a = Auu[j, i, k, mm]
                            b = Auu[j + jA, i + iA, k + kA, mt]
                            c = Auv[j, i, k, mm]
                            d = Avu[j + jA, i + iA, k + kA, mt]
                            worst = max(worst, abs(a - b), abs(c - d))
    assert worst == 0.0


def test_standard_and_chrongear_agree():
    m = configs.dome()
    su, u, v, A, bu, bv, _ = oracle_system(m, seed=5, scale=10.0)
    z = np.zeros(m.vshape3)
    s = oracle.pcg(m, su["active_vertex"], A, bu, bv, z, z, precond=1, variant=2, maxiters=4000, tol=1e-12)
    c = oracle.pcg(m, su["active_vertex"], A, bu, bv, z, z, precond=1, variant=3, maxiters=4000, tol=1e-12)
    assert s[4] == 0 and c[4] == 0
    assert rel_l2(s[:2], c[:2]) < 1e-10


def test_golden_dome_solve():
    g = np.load(os.path.join(GOLDEN, "dome15_solve.npz"))
    m = configs.dome(n=15, dx=2000.0, nz=6, radius=12.0e3, hmax=1000.0)
    u, v, efvs, _, st = oracle.velo_higher_solve(m)
    assert st["picard_iters"] == int(g["picard_iters"])
    assert rel_l2([u, v], [g["uvel"], g["vvel"]]) < 1e-12


def test_golden_slab_system():
    g = np.load(os.path.join(GOLDEN, "slab12_system.npz"))
    m = configs.slab(n=12, nz=6).copy(pcg_maxiters=1000)
    su = oracle.setup(m)
    A, bu, bv, _, _ = oracle.assemble_system(m, su, su["uvel"], su["vvel"])
    for a, k in zip(A, ("Auu", "Auv", "Avu", "Avv")):
        assert np.max(np.abs(a - g[k])) <= 1e-13 * np.max(np.abs(g[k]))
    assert rel_l2([bu, bv], [g["bu"], g["bv"]]) < 1e-13
