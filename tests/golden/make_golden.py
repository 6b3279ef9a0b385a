"""Regenerates the golden fixtures of tests/golden from the CPU oracle.

The reference ships no numeric golden vectors and its Fortran cannot be
built here, so these fixtures freeze the oracle's outputs on small seeded
cases (regression pins); the oracle itself is pinned to the reference by
the analytic slab test and the reference invariants (tests/test_oracle.py).

Usage: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cism_b200 import configs  # noqa: E402
from oracle import oracle  # noqa: E402


def main():
    m = configs.dome(n=15, dx=2000.0, nz=6, radius=12.0e3, hmax=1000.0)
    u, v, efvs, beta, st = oracle.velo_higher_solve(m)
    np.savez_compressed(os.path.join(HERE, "dome15_solve.npz"), uvel=u, vvel=v, efvs=efvs,
                        picard_iters=st["picard_iters"], pcg_iters_total=st["pcg_iters_total"])
    m = configs.slab(n=12, nz=6).copy(pcg_maxiters=1000)
    su = oracle.setup(m)
    A, bu, bv, _, _ = oracle.assemble_system(m, su, su["uvel"], su["vvel"])
    np.savez_compressed(os.path.join(HERE, "slab12_system.npz"), Auu=A[0], Auv=A[1], Avu=A[2],
                        Avv=A[3], bu=bu, bv=bv, active_vertex=su["active_vertex"])
    print("wrote", os.listdir(HERE))


# every SUB-th owned vertex in each direction, all levels
SUB = 4


def c1_fixture():
    """The full-size periodic slab (160 x 160 x 11) solved by the oracle
    (about 14 CPU-minutes): its Picard and PCG counts, the velocity at every
    SUB-th owned vertex in each direction and whole-field checksums (sum and
    sum of squares of u and v over the owned vertices)."""
    m = configs.workload("c1").copy(pcg_maxiters=3000)
    u, v, efvs, beta, st = oracle.velo_higher_solve(m)
    js, is_ = m.owned_vertex_slices()
    uo, vo = u[js, is_], v[js, is_]
    np.savez_compressed(os.path.join(HERE, "c1_picard_oracle.npz"), sub=SUB,
                        u_sub=uo[::SUB, ::SUB], v_sub=vo[::SUB, ::SUB],
                        sums=np.array([uo.sum(), vo.sum(), (uo ** 2).sum(), (vo ** 2).sum()]),
                        picard_iters=st["picard_iters"], pcg_iters_total=st["pcg_iters_total"])
    print("wrote c1_picard_oracle.npz", st)


if __name__ == "__main__":
    if "--c1" in sys.argv:
        c1_fixture()
    else:
        main()
