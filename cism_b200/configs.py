"""Synthetic model states for the Blatter-Pattyn solve.

Each generator returns a :class:`BPModel`: the fields that CISM's
``glissade_velo_higher_solve`` reads from ``model`` (thickness, surface,
bed, flow factor, external beta) on the reference's local grid, i.e. with a
2-cell halo on every side, already halo-updated the way
``libglimmer/parallel_slap.F90`` does it (periodic global boundary, with the
optional ``periodic_offset_ew`` of ``libglissade/glissade.F90:336-348``).

Array convention: a Fortran array ``a(nx, ny)`` (i fastest) is the numpy
C-order array of shape ``(ny, nx)``; ``a(nz, nx-1, ny-1)`` is shape
``(ny-1, nx-1, nz)``.  Units are the solver's internal ones: m, m/a,
Pa^-3 a^-1, Pa a/m.

No public dataset is used: every field is a seeded synthetic restatement of
the workload's stated shapes and distributions.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

NHALO = 2

# option values, libglide/glide_types.F90:198-263
EFVS_CONSTANT, EFVS_FLOWFACT, EFVS_NONLINEAR = 0, 1, 2
BABC_BETA_CONSTANT, BABC_BETA_EXTERNAL, BABC_NO_SLIP = 0, 5, 6
RESID_MAXU, RESID_MAXU_NO_UBAS, RESID_MEANU, RESID_L2NORM, RESID_L2NORM_RELATIVE = 0, 1, 2, 3, 4
SPARSE_PCG_STANDARD, SPARSE_PCG_CHRONGEAR = 2, 3
# New which_ho_sparse value selecting the B200 solver (one past Trilinos = 4).
SPARSE_B200 = 5
PRECOND_NONE, PRECOND_DIAG, PRECOND_SIA = 0, 1, 2
ASSEMBLE_STANDARD, ASSEMBLE_LOCAL = 0, 1
# velocity-dependent sliding laws (glide_types.F90:211-225)
(BABC_YIELD_PICARD, BABC_PSEUDO_PLASTIC, BABC_POWERLAW, BABC_COULOMB_FRICTION,
 BABC_COULOMB_POWERLAW_SCHOOF, BABC_COULOMB_POWERLAW_TSAI, BABC_POWERLAW_EFFECPRESS) = 2, 3, 9, 10, 11, 12, 13
SLIDING_LAWS = (2, 3, 9, 10, 11, 12, 13)
# the 2-D solves (whichapprox, glide_types.F90:255-259); 0 = the 3-D Blatter-Pattyn solve
APPROX_SSA, APPROX_L1L2, APPROX_DIVA = 1, 3, 4


@dataclasses.dataclass
class SlidingLaw:
    """A velocity-dependent sliding law of calcbeta
    (libglissade/glissade_basal_traction.F90:67-598), evaluated from the
    basal velocity at every Picard iteration.  ``law`` is the which_ho_babc
    value; the parameters default to libglide/glide_types.F90:1300-1370.
    Vertex fields have shape (ny-1, nx-1)."""

    law: int
    effecpress_stag: Optional[np.ndarray] = None      # N, Pa (laws 3, 10-13)
    c_space_factor_stag: Optional[np.ndarray] = None  # law 10 (None: 1)
    yield_stress: Optional[np.ndarray] = None          # mintauf * tau0, Pa (law 2)
    beta_powerlaw_umax: float = 0.0
    powerlaw_c: float = 1.0e4
    powerlaw_m: float = 3.0
    coulomb_c: float = 0.42
    coulomb_bump_max_slope: float = 0.5
    coulomb_bump_wavelength: float = 2.0
    friction_powerlaw_k: float = 8.4e-9
    pseudo_plastic_q: float = 0.5
    pseudo_plastic_u0: float = 100.0
    pseudo_plastic_phimin: float = 5.0
    pseudo_plastic_phimax: float = 40.0
    pseudo_plastic_bedmin: float = -700.0
    pseudo_plastic_bedmax: float = 700.0


@dataclasses.dataclass
class BPModel:
    """Inputs of one velocity solve on the halo'd local grid."""

    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    thck: np.ndarray          # (ny, nx)
    usrf: np.ndarray          # (ny, nx)
    topg: np.ndarray          # (ny, nx)
    flwa: np.ndarray          # (ny, nx, nz-1)
    beta_external: np.ndarray  # (ny-1, nx-1)
    periodic: int = 1
    kinbcmask: Optional[np.ndarray] = None
    eus: float = 0.0
    thklim: float = 100.0
    max_slope: float = 1.0
    thck_gradient_ramp: float = 0.0
    rhoi: float = 910.0
    rhoo: float = 1028.0
    grav: float = 9.81
    beta_const: float = 10.0
    beta_grounded_min: float = 1.0
    efvs_constant: float = 2336041.0
    which_babc: int = BABC_NO_SLIP
    which_efvs: int = EFVS_NONLINEAR
    which_resid: int = RESID_MAXU
    which_sparse: int = SPARSE_PCG_STANDARD
    which_precond: int = PRECOND_DIAG
    which_gradient: int = 0
    which_gradient_margin: int = 1
    which_assemble_beta: int = ASSEMBLE_LOCAL
    which_assemble_taud: int = ASSEMBLE_LOCAL
    which_ground: int = 0
    maxiter_nonlinear: int = 100
    pcg_maxiters: int = 200
    pcg_tol: float = 1.0e-8
    pcg_ncheck: int = 5
    sliding: Optional[SlidingLaw] = None  # velocity-dependent law (which_babc = sliding.law)
    approx_2d: int = 0  # 2-D solve: APPROX_SSA (1), APPROX_L1L2 (3) or APPROX_DIVA (4); 0 = 3-D Blatter-Pattyn
    # DIVA: the state of the last solve (uvel_2d, vvel_2d, btractx, btracty
    # (ny-1, nx-1); efvs (ny, nx, nz-1)); None or a missing key = zero
    diva_state: Optional[dict] = None
    name: str = ""

    @property
    def vshape3(self):
        return (self.ny - 1, self.nx - 1, self.nz)

    def zeros3(self):
        return np.zeros(self.vshape3, dtype=np.float64)

    def owned_vertex_slices(self):
        """(j, i) slices of the locally owned vertices, parallel_slap.F90:655-673."""
        lo = 2 if self.periodic else 1
        return slice(lo, self.ny - 2), slice(lo, self.nx - 2)

    def copy(self, **kw):
        return dataclasses.replace(self, **kw)


def halo_fill_cells(a: np.ndarray, periodic: int = 1, offset_ew: float = 0.0,
                    offset_ns: float = 0.0) -> np.ndarray:
    """parallel_halo for a cell field (parallel_slap.F90:1790-1860), in place.

    ``a`` has shape (ny, nx) including 2 halo cells on each side.
    """
    ny, nx = a.shape
    if not periodic:
        a[2:ny - 2, 0:2] = 0
        a[2:ny - 2, nx - 2:] = 0
        a[0:2, :] = 0
        a[ny - 2:, :] = 0
        return a
    rows = slice(2, ny - 2)
    e = a[rows, nx - 4:nx - 2].copy()
    w = a[rows, 2:4].copy()
    a[rows, 0:2] = e + offset_ew
    a[rows, nx - 2:] = w - offset_ew
    n = a[ny - 4:ny - 2, :].copy()
    s = a[2:4, :].copy()
    a[0:2, :] = n + offset_ns
    a[ny - 2:, :] = s - offset_ns
    return a


def halo_fill_stag(a: np.ndarray, periodic: int = 1) -> np.ndarray:
    """staggered_parallel_halo for an array shaped (ny-1, nx-1, ...), in place."""
    W, V = a.shape[0], a.shape[1]
    if not periodic:
        a[:, 0] = 0
        a[:, V - 1] = 0
        a[0, :] = 0
        a[W - 1, :] = 0
        return a
    rows = slice(2, W - 1)
    wcp = a[rows, 2].copy()
    ecp = a[rows, V - 3:V - 1].copy()
    a[rows, V - 1] = wcp
    a[rows, 0:2] = ecp
    scp = a[2].copy()
    ncp = a[W - 3:W - 1].copy()
    a[W - 1] = scp
    a[0:2] = ncp
    return a


def _embed(owned: np.ndarray) -> np.ndarray:
    """Place an owned (gy, gx) cell field into a halo'd (gy+4, gx+4) array."""
    gy, gx = owned.shape
    out = np.zeros((gy + 2 * NHALO, gx + 2 * NHALO), dtype=np.float64)
    out[NHALO:NHALO + gy, NHALO:NHALO + gx] = owned
    return out


def _vertex_from_owned(owned_v: np.ndarray, periodic: int = 1) -> np.ndarray:
    """Owned vertices (gy, gx) -> halo'd vertex array (gy+3, gx+3)."""
    gy, gx = owned_v.shape
    out = np.zeros((gy + 3, gx + 3), dtype=np.float64)
    out[2:2 + gy, 2:2 + gx] = owned_v
    return halo_fill_stag(out, periodic)


def calc_lsrf_usrf(thck, topg, eus, rhoi, rhoo):
    """Upper surface from flotation (glide_calclsrf + usrf = lsrf + thck)."""
    lsrf = np.where(topg - eus < -(rhoi / rhoo) * thck, -(rhoi / rhoo) * thck + eus, topg)
    return lsrf + thck


def _cell_centres(g: int, d: float) -> np.ndarray:
    return (np.arange(g) + 0.5) * d


def dome(n: int = 31, dx: float = 2000.0, nz: int = 10, radius: float = 25.0e3,
         hmax: float = 2000.0, flwa: float = 1.0e-16) -> BPModel:
    """Parabolic dome, no-slip bed (workload: 31x31, dx = 2 km, 10 levels).

    H = hmax * sqrt(1 - r^2/R^2) centred on the grid, flat bed at 0 m,
    uniform A, Dirichlet no-slip bed (which_ho_babc = 6), standard PCG with
    diagonal preconditioner, Picard on max relative speed change.
    """
    xc = _cell_centres(n, dx)
    X, Y = np.meshgrid(xc, xc)
    c = n * dx / 2.0
    r2 = (X - c) ** 2 + (Y - c) ** 2
    H = np.where(r2 < radius ** 2, hmax * np.sqrt(np.maximum(0.0, 1.0 - r2 / radius ** 2)), 0.0)
    thck = halo_fill_cells(_embed(H))
    topg = np.zeros_like(thck)
    usrf = topg + thck
    ny, nx = thck.shape
    return BPModel(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, thck=thck, usrf=usrf, topg=topg,
                   flwa=np.full((ny, nx, nz - 1), flwa), beta_external=np.zeros((ny - 1, nx - 1)),
                   thklim=1.0, which_babc=BABC_NO_SLIP, which_sparse=SPARSE_PCG_STANDARD,
                   which_precond=PRECOND_DIAG, which_resid=RESID_MAXU, name=f"dome{n}x{n}x{nz}")


def slab(n: int = 160, dx: float = 500.0, nz: int = 11, theta_deg: float = 0.1,
         thickness: float = 1000.0, flwa: float = 1.0e-16, beta0: float = 1000.0,
         beta1: float = 1000.0, ny_cells: Optional[int] = None) -> BPModel:
    """Periodic slab on a sliding bed (workload: 160x160, dx = 0.5 km, 11 levels).

    s = -x tan(theta), H uniform, b = s - H, doubly periodic with the E-W
    periodic offset L tan(theta) so the surface is continuous across the
    seam.  beta = beta0 + beta1 sin(2 pi x/L) sin(2 pi y/L) at vertices,
    applied as external beta (which_ho_babc = 5) with LOCAL assembly.  Sea
    level is placed far below the bed so the whole slab is grounded land.
    """
    gy = n if ny_cells is None else ny_cells
    gx = n
    L = gx * dx
    Ly = gy * dx
    t = math.tan(math.radians(theta_deg))
    xc = _cell_centres(gx, dx)
    s_owned = np.tile(-xc * t, (gy, 1))
    offset = L * t
    usrf = halo_fill_cells(_embed(s_owned), offset_ew=offset)
    thck = halo_fill_cells(_embed(np.full((gy, gx), thickness)))
    topg = usrf - thck
    ny, nx = thck.shape
    # vertex (i,j) sits at the NE corner of cell (i,j): x = i*dx (owned i = 1..gx)
    xv = (np.arange(gx) + 1) * dx
    yv = (np.arange(gy) + 1) * dx
    XV, YV = np.meshgrid(xv, yv)
    beta_v = beta0 + beta1 * np.sin(2 * np.pi * XV / L) * np.sin(2 * np.pi * YV / Ly)
    beta_ext = _vertex_from_owned(beta_v)
    return BPModel(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, thck=thck, usrf=usrf, topg=topg,
                   flwa=np.full((ny, nx, nz - 1), flwa), beta_external=beta_ext,
                   eus=-1.0e5, thklim=1.0, which_babc=BABC_BETA_EXTERNAL,
                   which_sparse=SPARSE_PCG_STANDARD, which_precond=PRECOND_DIAG,
                   which_resid=RESID_MAXU, name=f"slab{gx}x{gy}x{nz}")


def analytic_slab(nx_cells: int = 30, ny_cells: int = 20, nz: int = 50, dx: float = 50.0,
                  theta_deg: float = 18.0, thickness: float = 1000.0, eta: float = 10.0,
                  efvs: float = 2336041.42829, rhoi: float = 910.0, grav: float = 9.81) -> BPModel:
    """The reference's own slab test (tests/slab/runSlab.py:115-136, 180-260).

    Constant viscosity (which_ho_efvs = 0, so n = 1), external beta chosen
    from the dimensionless slip parameter eta, bed inclined at theta, vertical
    thickness thickness/cos(theta), periodic offset nx*dx*tan(theta).
    """
    t = math.tan(math.radians(theta_deg))
    beta = eta / thickness * efvs  # n = 1: beta = eta / H / efvs**-1
    x = dx * np.arange(nx_cells)
    xmax = x.max()
    topg_o = np.tile((xmax - x) * t + 1000.0, (ny_cells, 1))
    thk_o = np.full((ny_cells, nx_cells), thickness / math.cos(math.radians(theta_deg)))
    offset = nx_cells * dx * t
    topg = halo_fill_cells(_embed(topg_o), offset_ew=offset)
    thck = halo_fill_cells(_embed(thk_o))
    usrf = topg + thck
    ny, nx = thck.shape
    beta_ext = _vertex_from_owned(np.full((ny_cells, nx_cells), beta))
    return BPModel(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, thck=thck, usrf=usrf, topg=topg,
                   flwa=np.full((ny, nx, nz - 1), 1.0e-16), beta_external=beta_ext,
                   eus=-1.0e5, thklim=1.0, rhoi=rhoi, grav=grav, efvs_constant=efvs,
                   which_efvs=EFVS_CONSTANT, which_babc=BABC_BETA_EXTERNAL,
                   which_sparse=SPARSE_PCG_CHRONGEAR, which_precond=PRECOND_DIAG,
                   which_resid=RESID_MAXU, pcg_maxiters=4000, pcg_tol=1.0e-11,
                   name=f"analytic_slab{nx_cells}x{ny_cells}x{nz}")


def analytic_slab_profile(model: BPModel, theta_deg: float = 18.0, thickness: float = 1000.0,
                          eta: float = 10.0) -> np.ndarray:
    """First-order (BP) analytic u(sigma) for the slab test, n = 1.

    Restates tests/slab/plotSlab.py:55-57 and :143-157 (the "FO" solution,
    Dukowicz), transformed to the model's column at the domain centre
    exactly as plotSlab.py does (x' = 0 there).
    """
    n = 1
    efvs = model.efvs_constant
    rhoi, grav = model.rhoi, model.grav
    thetar = math.radians(theta_deg)
    velscale = (rhoi * grav * thickness / efvs) ** n * thickness
    sigma = sigma_glide(model.nz)
    z = (1.0 - sigma)  # thk[col]/thickness scaling cancels (thk = H/cos) -> handled below
    z = z * (thickness / math.cos(thetar)) / thickness
    zprime = z * math.cos(thetar)
    u = ((-1) ** n * 2 ** ((1.0 - n) / 2.0) * math.tan(thetar) ** n
         / ((n + 1) * (1.0 + 3.0 * math.sin(thetar) ** 2) ** ((n + 1.0) / 2.0))
         * ((zprime - 1.0) ** (n + 1) - (-1.0) ** (n + 1)) + math.tan(thetar) / eta)
    return u * velscale


def sigma_glide(nz: int) -> np.ndarray:
    """Glide sigma levels, libglide/glide_setup.F90:281-290, 375-382."""
    level = np.arange(nz, dtype=np.float64) / (nz - 1)
    return (1.0 - (level + 1.0) ** (-2.0)) / (1.0 - 2.0 ** (-2.0))


def gaussian_random_field(rng: np.random.Generator, shape, dx: float, corr_len: float) -> np.ndarray:
    """Zero-mean unit-variance field with squared-exponential covariance
    exp(-r^2 / (2 corr_len^2)), by FFT filtering of white noise."""
    gy, gx = shape
    noise = rng.standard_normal((gy, gx))
    kx = np.fft.fftfreq(gx, d=dx) * 2 * np.pi
    ky = np.fft.fftfreq(gy, d=dx) * 2 * np.pi
    KX, KY = np.meshgrid(kx, ky)
    spec = np.exp(-0.25 * (KX ** 2 + KY ** 2) * corr_len ** 2)  # sqrt of the SE spectrum
    f = np.real(np.fft.ifft2(np.fft.fft2(noise) * spec))
    f -= f.mean()
    sd = f.std()
    return f / sd if sd > 0 else f


def marine(n: int = 400, dx: float = 4000.0, nz: int = 11, seed: int = 2, peak: float = 3000.0,
           radius_frac: float = 0.45, front_thickness: float = 200.0, flwa: float = 1.0e-16,
           rhoi: float = 917.0, rhoo: float = 1028.0, beta_median: float = 1.0e3,
           beta_sigma_ln: float = 1.0, bed_mean: float = -200.0, bed_std: float = 600.0,
           bed_corr: float = 40.0e3, trough_depth: float = 1500.0, trough_dir: int = 0,
           trough_width: float = 60.0e3, beta_corr: float = 20.0e3, ny_cells: Optional[int] = None,
           rng: Optional[np.random.Generator] = None) -> BPModel:
    """Marine ice sheet with grounding line and floating shelf (workload:
    400x400, dx = 4 km, 11 levels).

    Bed: seeded Gaussian random field (mean -200 m, std 600 m, correlation
    length 40 km) plus a 1500 m deep radial trough from the centre to the
    east edge (Gaussian cross-section of 60 km half-width, depth ramping
    linearly from 0 at the centre to 1500 m at the edge).  Thickness
    H = peak (1 - r^2/R^2), R = radius_frac * L, cut to zero where it falls
    below front_thickness, so a calving front sits at the margin; ice floats
    where rhoi H < -rhoo (b - eus).  beta is log-normal (median beta_median,
    sigma_ln, correlation length 20 km) and calcbeta zeroes it under the
    shelf through f_ground.  Chronopoulos-Gear PCG.

    The keyword arguments past beta_sigma_ln vary the family for the
    learned guess's training set (random_marine); their defaults are the
    workload's.  trough_dir turns the trough toward the east (0), north (1),
    west (2) or south (3) edge; ny_cells makes the domain non-square (the
    radius then follows the shorter side).
    """
    rng = np.random.default_rng(seed) if rng is None else rng
    gx, gy = n, (n if ny_cells is None else ny_cells)
    xc = _cell_centres(gx, dx)
    yc = _cell_centres(gy, dx)
    X, Y = np.meshgrid(xc, yc)
    cx, cy = gx * dx / 2.0, gy * dx / 2.0
    bed = bed_mean + bed_std * gaussian_random_field(rng, (gy, gx), dx, bed_corr)
    along, across, half = [((X - cx), (Y - cy), cx), ((Y - cy), (X - cx), cy),
                           ((cx - X), (Y - cy), cx), ((cy - Y), (X - cx), cy)][trough_dir % 4]
    ramp = np.clip(along / half, 0.0, 1.0)
    bed -= trough_depth * ramp * np.exp(-(across ** 2) / (2 * trough_width ** 2))
    R = radius_frac * min(gx, gy) * dx
    r2 = (X - cx) ** 2 + (Y - cy) ** 2
    H = peak * np.maximum(0.0, 1.0 - r2 / R ** 2)
    H = np.where(H >= front_thickness, H, 0.0)
    topg = halo_fill_cells(_embed(bed))
    thck = halo_fill_cells(_embed(H))
    usrf = calc_lsrf_usrf(thck, topg, 0.0, rhoi, rhoo)
    ny, nx = thck.shape
    lnb = gaussian_random_field(rng, (gy, gx), dx, beta_corr)
    beta_v = beta_median * np.exp(beta_sigma_ln * lnb)
    beta_ext = _vertex_from_owned(beta_v)
    return BPModel(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, thck=thck, usrf=usrf, topg=topg,
                   flwa=np.full((ny, nx, nz - 1), flwa), beta_external=beta_ext,
                   eus=0.0, thklim=1.0, rhoi=rhoi, rhoo=rhoo, which_babc=BABC_BETA_EXTERNAL,
                   which_sparse=SPARSE_PCG_CHRONGEAR, which_precond=PRECOND_DIAG,
                   which_resid=RESID_MAXU, pcg_maxiters=5000, name=f"marine{gx}x{gy}x{nz}")


def random_marine(rng: np.random.Generator, n: int = 256, dx: float = 2000.0, nz: int = 11,
                  ny_cells: Optional[int] = None) -> BPModel:
    """A member of the learned guess's training family around the marine
    workload: the same generator with random peak thickness (2000-3500 m),
    radius (0.35-0.48 of the domain), bed mean (-400-0 m), standard
    deviation (300-800 m) and correlation length (20-60 km), trough depth
    (0-1500 m) and direction, median beta (10^2.5-10^3.5 Pa a/m), its log
    spread (0.5-1.5) and correlation length (10-40 km), and rate factor
    (0.5-2 x 1e-16)."""
    kw = dict(peak=rng.uniform(2000.0, 3500.0), radius_frac=rng.uniform(0.35, 0.48),
              bed_mean=rng.uniform(-400.0, 0.0), bed_std=rng.uniform(300.0, 800.0),
              bed_corr=rng.uniform(20.0e3, 60.0e3), trough_depth=rng.uniform(0.0, 1500.0),
              trough_dir=int(rng.integers(0, 4)), beta_median=10.0 ** rng.uniform(2.5, 3.5),
              beta_sigma_ln=rng.uniform(0.5, 1.5), beta_corr=rng.uniform(10.0e3, 40.0e3),
              flwa=1.0e-16 * np.exp(rng.uniform(np.log(0.5), np.log(2.0))))
    m = marine(n=n, dx=dx, nz=nz, ny_cells=ny_cells, rng=rng, **kw)
    return m.copy(name=f"rmarine{m.nx - 4}x{m.ny - 4}")


def ensemble(count: int = 256, seed: int = 3, lo: int = 32, hi: int = 192, dx: float = 2000.0,
             nz: int = 11, beta_sigma_ln: float = 0.5) -> list:
    """Batched ensemble: `count` independent domains, side lengths uniform in
    [lo, hi] cells independently in x and y, dome or slab per instance, each
    with its own log-normal beta perturbation (sigma_ln = beta_sigma_ln)."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(count):
        gx = int(rng.integers(lo, hi + 1))
        gy = int(rng.integers(lo, hi + 1))
        kind = int(rng.integers(0, 2))
        pert = np.exp(beta_sigma_ln * gaussian_random_field(rng, (gy, gx), dx, 20.0e3))
        if kind == 0:
            m = _sliding_dome(gx, gy, dx, nz, rng)
        else:
            m = slab(n=gx, ny_cells=gy, dx=dx, nz=nz, theta_deg=float(rng.uniform(0.05, 0.2)))
        owned = m.beta_external[2:2 + gy, 2:2 + gx] if kind == 1 else np.full((gy, gx), 1000.0)
        m.beta_external = _vertex_from_owned(owned * pert)
        m.which_babc = BABC_BETA_EXTERNAL
        m.name = f"ens{b}_{'dome' if kind == 0 else 'slab'}{gx}x{gy}x{nz}"
        out.append(m)
    return out


def _sliding_dome(gx: int, gy: int, dx: float, nz: int, rng: np.random.Generator) -> BPModel:
    """Elliptic dome on a sliding bed that fills 80% of a gx x gy domain."""
    xc = _cell_centres(gx, dx)
    yc = _cell_centres(gy, dx)
    X, Y = np.meshgrid(xc, yc)
    a, b = 0.4 * gx * dx, 0.4 * gy * dx
    q = ((X - gx * dx / 2) / a) ** 2 + ((Y - gy * dx / 2) / b) ** 2
    hmax = float(rng.uniform(1000.0, 3000.0))
    H = np.where(q < 1.0, hmax * np.sqrt(np.maximum(0.0, 1.0 - q)), 0.0)
    thck = halo_fill_cells(_embed(H))
    topg = np.zeros_like(thck)
    ny, nx = thck.shape
    return BPModel(nx=nx, ny=ny, nz=nz, dx=dx, dy=dx, thck=thck, usrf=topg + thck, topg=topg,
                   flwa=np.full((ny, nx, nz - 1), 1.0e-16), beta_external=np.zeros((ny - 1, nx - 1)),
                   thklim=1.0, which_babc=BABC_BETA_EXTERNAL, which_sparse=SPARSE_PCG_STANDARD,
                   which_precond=PRECOND_DIAG, which_resid=RESID_MAXU, name=f"dome{gx}x{gy}")


def with_sliding(m: BPModel, law: int, seed: int = 0, n_scale: float = 0.8, **params) -> BPModel:
    """``m`` with a velocity-dependent sliding law (which_babc = law).

    Synthetic basal fields on the (ny-1, nx-1) vertex grid: effective
    pressure N = n_scale * rho_i g H (H averaged over the four cells of the
    vertex) times a seeded smooth factor in [0.7, 1.3]; for law 2 a yield
    stress of 40 kPa times such a factor; for law 10 a C_space factor in
    [0.8, 1.2].  ``params`` override SlidingLaw's defaults.
    """
    rng = np.random.default_rng(seed)
    ny, nx = m.thck.shape
    hv = 0.25 * (m.thck[:-1, :-1] + m.thck[:-1, 1:] + m.thck[1:, :-1] + m.thck[1:, 1:])
    jj, ii = np.meshgrid(np.arange(ny - 1), np.arange(nx - 1), indexing="ij")

    def factor(amp):
        ph = rng.uniform(0.0, 2.0 * np.pi, 2)
        return 1.0 + amp * np.sin(2.0 * np.pi * ii / max(nx - 5, 1) + ph[0]) * \
            np.cos(2.0 * np.pi * jj / max(ny - 5, 1) + ph[1])

    sl = SlidingLaw(law=law, effecpress_stag=n_scale * m.rhoi * m.grav * hv * factor(0.3), **params)
    if law == BABC_YIELD_PICARD:
        sl.yield_stress = 4.0e4 * factor(0.3)
    if law == BABC_COULOMB_FRICTION:
        sl.c_space_factor_stag = factor(0.2)
    return m.copy(which_babc=law, sliding=sl, name=f"{m.name}_law{law}")


def raymond_stream(n_stream: int = 25, nz: int = 2, half_width: float = 25.0e3, along: float = 30.0e3,
                   thickness: float = 1000.0, dsdx: float = -1.0e-3, flwa: float = 1.0e-16,
                   tau_stream: float = 5.2e3, tau_strong: float = 0.7e5) -> BPModel:
    """The reference's idealised ice stream (tests/stream/runStream.py:124-360,
    its doubly periodic form, kinflag = 0): a slab of thickness H on a bed
    sloping at dsdx along x, a till yield stress (which_ho_babc = 2) of
    tau_stream inside |y| < half_width and tau_strong (above the driving
    stress) outside, uniform along flow, 5 H of strong bed on each side,
    Glen's law with a uniform rate factor, Chronopoulos-Gear PCG with the
    diagonal preconditioner, local basal assembly, no grounded minimum of
    beta (stream.config).  The stream edges fall on vertex rows.  Raymond's
    (2000) solution :func:`raymond_uvel` is its analytic profile.
    """
    dy = 2.0 * half_width / n_stream
    dx = dy
    n_strong = int(np.floor(5.0 * thickness / dy + 0.5))  # the script's round(), halves away from zero
    gy = n_stream + 2 * n_strong
    gx = int(round(along / dx))
    L = gx * dx
    x1 = dx * np.arange(gx)
    topg_owned = np.tile(1000.0 + dsdx * x1, (gy, 1))
    usrf = halo_fill_cells(_embed(topg_owned + thickness), offset_ew=-dsdx * L)
    thck = halo_fill_cells(_embed(np.full((gy, gx), thickness)))
    topg = usrf - thck
    ny, nx = thck.shape
    # vertex row j (the NE corner of cell row j) sits at y0 = dy (j + 1) - dy gy / 2
    y0 = dy * (np.arange(gy) + 1) - dy * gy / 2.0
    tau = np.where(np.abs(y0) >= half_width, tau_strong, tau_stream)
    yield_stress = _vertex_from_owned(np.tile(tau[:, None], (1, gx)))
    sl = SlidingLaw(law=BABC_YIELD_PICARD, yield_stress=yield_stress)
    return BPModel(nx=nx, ny=ny, nz=nz, dx=dx, dy=dy, thck=thck, usrf=usrf, topg=topg,
                   flwa=np.full((ny, nx, nz - 1), flwa), beta_external=np.zeros((ny - 1, nx - 1)),
                   eus=0.0, thklim=1.0, beta_grounded_min=0.0, which_babc=BABC_YIELD_PICARD, sliding=sl,
                   which_efvs=EFVS_NONLINEAR, which_sparse=SPARSE_PCG_CHRONGEAR, which_precond=PRECOND_DIAG,
                   which_assemble_beta=ASSEMBLE_LOCAL, maxiter_nonlinear=300,
                   name=f"raymond_stream{gx}x{gy}x{nz}")


def raymond_uvel(y: np.ndarray, half_width: float = 25.0e3, thickness: float = 1000.0,
                 dsdx: float = -1.0e-3, flwa: float = 1.0e-16, tau_stream: float = 5.2e3,
                 tau_strong: float = 0.7e5, rhoi: float = 910.0, grav: float = 9.81) -> np.ndarray:
    """Raymond's (2000) ice-stream velocity across the stream (the
    reference's raymond_uvel, tests/stream/runStream.py:166-172): u =
    2 A / (n+1) ((tau_d - tau_0) / H)^n (w^(n+1) - |y|^(n+1)), n = 3, zero
    where the bed is stronger than the driving stress tau_d."""
    n = 3.0
    taud = -rhoi * grav * thickness * dsdx
    tau0 = np.where(np.abs(y) >= half_width, tau_strong, tau_stream)
    tau0 = np.minimum(tau0, taud)
    u = 2.0 * flwa / (n + 1.0) * ((taud - tau0) / thickness) ** n * (half_width ** (n + 1) - np.abs(y) ** (n + 1))
    return np.maximum(u, 0.0)


def random_slab(rng: np.random.Generator, n: int = 96, dx: float = 500.0, nz: int = 11) -> BPModel:
    """A member of the periodic-slab family of the learned guess's training
    and held-out sets: the slab above with a random slope (0.05-0.2 deg),
    thickness (700-1300 m), rate factor (0.5-2 x 1e-16) and basal friction
    beta = beta0 (1 + a sin(2 pi kx x / L + px) sin(2 pi ky y / L + py))
    exp(s g - s^2 / 2), g a periodic unit Gaussian field (correlation 2-8
    km), beta0 500-2000 Pa a/m, a 0-1, kx, ky in {1, 2}, s 0-0.4."""
    theta = rng.uniform(0.05, 0.2)
    H = rng.uniform(700.0, 1300.0)
    flwa = 1.0e-16 * np.exp(rng.uniform(np.log(0.5), np.log(2.0)))
    m = slab(n=n, dx=dx, nz=nz, theta_deg=theta, thickness=H, flwa=flwa)
    L = n * dx
    xv = (np.arange(n) + 1) * dx
    XV, YV = np.meshgrid(xv, xv)
    kx, ky = rng.integers(1, 3, size=2)
    px, py = rng.uniform(0.0, 2 * np.pi, size=2)
    beta0 = rng.uniform(500.0, 2000.0)
    amp = rng.uniform(0.0, 1.0)
    sig = rng.uniform(0.0, 0.4)
    g = gaussian_random_field(rng, (n, n), dx, rng.uniform(2.0e3, 8.0e3))
    beta_v = beta0 * (1.0 + amp * np.sin(2 * np.pi * kx * XV / L + px) * np.sin(2 * np.pi * ky * YV / L + py))
    beta_v = beta_v * np.exp(sig * g - 0.5 * sig * sig)
    return m.copy(beta_external=_vertex_from_owned(beta_v), name=f"rslab{n}")


def workload(name: str) -> BPModel:
    """The named synthetic workloads."""
    if name == "c0":
        return dome()
    if name == "c1":
        return slab()
    if name == "c2":
        return marine()
    raise KeyError(name)
