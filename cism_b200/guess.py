"""Initial guesses for the Picard loop: zero, shallow ice, learned.

The reference starts the higher-order solve from the previous time step's
velocity (zero on the first step).  Two alternatives feed the same
unchanged solver: a local shallow-ice-plus-sliding estimate, and the
learned U-Net (``net.py``).  The solver then converges to the same
tolerance from any of them.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

from . import configs


def zero_guess(m: configs.BPModel):
    return np.zeros(m.vshape3), np.zeros(m.vshape3)


def sia_guess(m: configs.BPModel):
    """Shallow-ice velocity with local sliding balance, per vertex column:
    u(sigma) = u_b - 2 A / (n + 1) (rho g)^n |grad s|^(n-1) grad s H^(n+1)
    (1 - sigma^(n+1)), n = 3, and u_b = -rho g H grad s / beta where the bed
    slides (external beta), 0 for a no-slip bed.  sigma = 0 at the surface,
    1 at the bed; A is the column's mean rate factor."""
    n = 3
    def stag(a):
        return 0.25 * (a[:-1, :-1] + a[1:, :-1] + a[:-1, 1:] + a[1:, 1:])
    H = stag(m.thck)
    s = m.usrf
    sx = (s[:-1, 1:] + s[1:, 1:] - s[:-1, :-1] - s[1:, :-1]) / (2.0 * m.dx)
    sy = (s[1:, :-1] + s[1:, 1:] - s[:-1, :-1] - s[:-1, 1:]) / (2.0 * m.dy)
    A = stag(np.asarray(m.flwa).mean(axis=-1))
    rg = m.rhoi * m.grav
    slope = np.sqrt(sx * sx + sy * sy)
    coef = 2.0 * A / (n + 1) * rg ** n * slope ** (n - 1) * H ** (n + 1)
    if m.which_babc == configs.BABC_BETA_EXTERNAL and m.beta_external is not None:
        beta = np.maximum(np.asarray(m.beta_external, np.float64), 1.0)
        ubx, uby = -rg * H * sx / beta, -rg * H * sy / beta
    else:
        ubx = uby = np.zeros_like(H)
    sigma = configs.sigma_glide(m.nz)
    shape = 1.0 - sigma ** (n + 1)
    u = ubx[..., None] - (coef * sx)[..., None] * shape
    v = uby[..., None] - (coef * sy)[..., None] * shape
    act = (H > m.thklim)[..., None]
    u, v = np.where(act, u, 0.0), np.where(act, v, 0.0)
    return configs.halo_fill_stag(u, m.periodic), configs.halo_fill_stag(v, m.periodic)


def learned_guesses(net, models: Sequence[configs.BPModel]):
    """U-Net guesses for domains of one size and border type."""
    from . import net as netmod

    return netmod.predict(net, models)
