"""Shared helpers of the test suite (checker side: may use the oracle)."""
import numpy as np

from cism_b200 import configs
from oracle import oracle


def rel_l2(a_pairs, b_pairs):
    num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(a_pairs, b_pairs))
    den = sum(float(np.sum(b ** 2)) for b in b_pairs)
    return np.sqrt(num / den) if den > 0 else np.sqrt(num)


def owned_active_rows(m, active_vertex):
    js, is_ = m.owned_vertex_slices()
    own = np.zeros((m.ny - 1, m.nx - 1), bool)
    own[js, is_] = True
    return own & active_vertex.astype(bool)


def random_state(m, su, seed=0, scale=100.0):
    """Random velocity on active vertices, halo-consistent."""
    rng = np.random.default_rng(seed)
    av = su["active_vertex"].astype(bool)
    u = rng.standard_normal(m.vshape3) * scale * av[..., None]
    v = rng.standard_normal(m.vshape3) * scale * av[..., None]
    return configs.halo_fill_stag(u, m.periodic), configs.halo_fill_stag(v, m.periodic)


def oracle_system(m, seed=0, scale=100.0):
    """An assembled oracle system (A, b) at a random velocity."""
    su = oracle.setup(m)
    u, v = random_state(m, su, seed, scale)
    A, bu, bv, efvs, nnz = oracle.assemble_system(m, su, u, v)
    return su, u, v, A, bu, bv, efvs


def small_models():
    return [configs.dome(), configs.slab(n=24), configs.marine(n=40, dx=4000.0)]
