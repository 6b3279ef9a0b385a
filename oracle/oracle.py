"""ctypes front end of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product never imports it.

Arrays follow cism_b200.configs: Fortran a(nx,ny) <-> numpy (ny,nx) C-order.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OrcBasalPhysics(C.Structure):
    _fields_ = [("effecpress_stag", _dp), ("c_space_factor_stag", _dp), ("mintauf_tau0", _dp)] + \
        [(n, C.c_double) for n in (
            "beta_powerlaw_umax", "powerlaw_c", "powerlaw_m", "coulomb_c", "coulomb_bump_max_slope",
            "coulomb_bump_wavelength", "friction_powerlaw_k", "pseudo_plastic_q", "pseudo_plastic_u0",
            "pseudo_plastic_phimin", "pseudo_plastic_phimax", "pseudo_plastic_bedmin",
            "pseudo_plastic_bedmax")]


class OrcModel(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nhalo", C.c_int),
        ("periodic", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
        ("thck", _dp), ("usrf", _dp), ("topg", _dp), ("flwa", _dp),
        ("beta_external", _dp), ("kinbcmask", _ip),
        ("eus", C.c_double), ("thklim", C.c_double), ("max_slope", C.c_double),
        ("thck_gradient_ramp", C.c_double), ("rhoi", C.c_double), ("rhoo", C.c_double),
        ("grav", C.c_double), ("beta_const", C.c_double), ("beta_grounded_min", C.c_double),
        ("efvs_constant", C.c_double),
        ("which_babc", C.c_int), ("which_efvs", C.c_int), ("which_resid", C.c_int),
        ("which_sparse", C.c_int), ("which_precond", C.c_int), ("which_gradient", C.c_int),
        ("which_gradient_margin", C.c_int), ("which_assemble_beta", C.c_int),
        ("which_assemble_taud", C.c_int), ("which_ground", C.c_int),
        ("maxiter_nonlinear", C.c_int), ("pcg_maxiters", C.c_int), ("pcg_tol", C.c_double),
        ("pcg_ncheck", C.c_int), ("basal", C.POINTER(OrcBasalPhysics)),
    ]


class OrcStats(C.Structure):
    _fields_ = [
        ("picard_iters", C.c_int), ("pcg_iters_total", C.c_int), ("pcg_iters_last", C.c_int),
        ("pcg_err_last", C.c_double), ("resid_velo", C.c_double), ("L2_norm", C.c_double),
        ("L2_norm_relative", C.c_double), ("converged", C.c_int), ("status", C.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class OrcSetup(C.Structure):
    _fields_ = [(n, _dp) for n in (
        "sigma", "stagwbndsigma", "stagusrf", "stagthck", "dusrf_dx", "dusrf_dy",
        "xVertex", "yVertex", "f_ground", "flwafact", "loadu", "loadv")] + \
        [(n, _ip) for n in ("active_cell", "active_vertex", "umask_dirichlet", "vmask_dirichlet",
                            "ice_mask", "floating_mask", "ocean_mask", "land_mask")]


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = C.CDLL(_LIB)
        _lib.orc_velo_higher_solve.restype = C.c_int
        _lib.orc_setup_solve.restype = C.c_int
    return _lib


def _p(a, typ=_dp):
    return a.ctypes.data_as(typ)


class _Keep:
    """Holds numpy buffers referenced by a ctypes struct."""

    def __init__(self):
        self.items = []

    def f64(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.items.append(a)
        return _p(a)

    def i32(self, a):
        a = np.ascontiguousarray(a, dtype=np.int32)
        self.items.append(a)
        return _p(a, _ip)


def make_model(m, keep: _Keep) -> OrcModel:
    om = OrcModel()
    om.nx, om.ny, om.nz, om.nhalo, om.periodic = m.nx, m.ny, m.nz, 2, m.periodic
    om.dx, om.dy = m.dx, m.dy
    om.thck = keep.f64(m.thck)
    om.usrf = keep.f64(m.usrf)
    om.topg = keep.f64(m.topg)
    om.flwa = keep.f64(m.flwa)
    om.beta_external = keep.f64(m.beta_external)
    om.kinbcmask = keep.i32(m.kinbcmask) if m.kinbcmask is not None else C.cast(None, _ip)
    for f in ("eus", "thklim", "max_slope", "thck_gradient_ramp", "rhoi", "rhoo", "grav",
              "beta_const", "beta_grounded_min", "efvs_constant", "which_babc", "which_efvs",
              "which_resid", "which_sparse", "which_precond", "which_gradient",
              "which_gradient_margin", "which_assemble_beta", "which_assemble_taud",
              "which_ground", "maxiter_nonlinear", "pcg_maxiters", "pcg_tol", "pcg_ncheck"):
        setattr(om, f, getattr(m, f))
    if om.which_sparse not in (2, 3):
        om.which_sparse = 2
    om.basal = C.cast(None, C.POINTER(OrcBasalPhysics))
    if m.sliding is not None:
        sl = m.sliding
        bp = OrcBasalPhysics()
        null = C.cast(None, _dp)
        bp.effecpress_stag = keep.f64(sl.effecpress_stag) if sl.effecpress_stag is not None else null
        bp.c_space_factor_stag = (keep.f64(sl.c_space_factor_stag) if sl.c_space_factor_stag is not None
                                  else null)
        bp.mintauf_tau0 = keep.f64(sl.yield_stress) if sl.yield_stress is not None else null
        for n, _ in OrcBasalPhysics._fields_[3:]:
            setattr(bp, n, getattr(sl, n))
        keep.items.append(bp)
        om.basal = C.pointer(bp)
    return om


def velo_higher_solve(m, uvel=None, vvel=None):
    """Whole Picard solve; returns (uvel, vvel, efvs, beta_internal, stats)."""
    keep = _Keep()
    om = make_model(m, keep)
    u = np.zeros(m.vshape3) if uvel is None else np.array(uvel, dtype=np.float64, copy=True)
    v = np.zeros(m.vshape3) if vvel is None else np.array(vvel, dtype=np.float64, copy=True)
    efvs = np.zeros((m.ny, m.nx, m.nz - 1))
    beta = np.zeros((m.ny - 1, m.nx - 1))
    st = OrcStats()
    lib().orc_velo_higher_solve(C.byref(om), _p(u), _p(v), _p(efvs), _p(beta), C.byref(st))
    return u, v, efvs, beta, st.as_dict()


APPROX_SSA, APPROX_L1L2 = 1, 3  # whichapprox, libglide/glide_types.F90:255-259


def velo_2d_solve(m, approx, uvel=None, vvel=None):
    """A 2-D branch of the solve (approx = APPROX_SSA or APPROX_L1L2);
    returns (uvel, vvel, efvs, beta_internal, stats): the SSA velocity on
    every level, or the L1L2 basal velocity with the 3-D velocity
    reconstructed above it."""
    keep = _Keep()
    om = make_model(m, keep)
    u = np.zeros(m.vshape3) if uvel is None else np.array(uvel, dtype=np.float64, copy=True)
    v = np.zeros(m.vshape3) if vvel is None else np.array(vvel, dtype=np.float64, copy=True)
    efvs = np.zeros((m.ny, m.nx, m.nz - 1))
    beta = np.zeros((m.ny - 1, m.nx - 1))
    st = OrcStats()
    rc = lib().orc_velo_2d_solve(C.byref(om), approx, _p(u), _p(v), _p(efvs), _p(beta), C.byref(st))
    if rc == 10:
        raise RuntimeError("orc_velo_2d_solve: bad arguments")
    return u, v, efvs, beta, st.as_dict()


def velo_ssa_solve(m, uvel=None, vvel=None):
    """Shallow-shelf (SSA) branch of the solve."""
    return velo_2d_solve(m, APPROX_SSA, uvel, vvel)


def velo_l1l2_solve(m, uvel=None, vvel=None):
    """L1L2 branch of the solve."""
    return velo_2d_solve(m, APPROX_L1L2, uvel, vvel)


def velo_diva_solve(m, uvel=None, vvel=None, uvel_2d=None, vvel_2d=None, btractx=None, btracty=None,
                    efvs=None):
    """DIVA branch of the solve.  The mean velocity (uvel_2d, vvel_2d), the
    basal traction (btractx, btracty) and efvs are the last solve's (zero
    by default) on entry; returns (uvel, vvel, efvs, beta_internal, stats,
    extra) with extra = dict(uvel_2d, vvel_2d, btractx, btracty)."""
    keep = _Keep()
    om = make_model(m, keep)
    vs = (m.ny - 1, m.nx - 1)

    def arr(a, shape):
        return np.zeros(shape) if a is None else np.array(a, dtype=np.float64, copy=True)

    u, v = arr(uvel, m.vshape3), arr(vvel, m.vshape3)
    u2, v2, bx, by = arr(uvel_2d, vs), arr(vvel_2d, vs), arr(btractx, vs), arr(btracty, vs)
    ef = arr(efvs, (m.ny, m.nx, m.nz - 1))
    beta = np.zeros(vs)
    st = OrcStats()
    rc = lib().orc_velo_diva_solve(C.byref(om), _p(u), _p(v), _p(u2), _p(v2), _p(bx), _p(by), _p(ef),
                                   _p(beta), C.byref(st))
    if rc == 10:
        raise RuntimeError("orc_velo_diva_solve: bad arguments")
    return u, v, ef, beta, st.as_dict(), dict(uvel_2d=u2, vvel_2d=v2, btractx=bx, btracty=by)


def setup(m, uvel=None, vvel=None):
    """Setup of glissade_velo_higher_solve: returns dict of boundary inputs."""
    keep = _Keep()
    om = make_model(m, keep)
    nx, ny, nz = m.nx, m.ny, m.nz
    arrs = {
        "sigma": np.zeros(nz), "stagwbndsigma": np.zeros(nz + 1),
        "stagusrf": np.zeros((ny - 1, nx - 1)), "stagthck": np.zeros((ny - 1, nx - 1)),
        "dusrf_dx": np.zeros((ny - 1, nx - 1)), "dusrf_dy": np.zeros((ny - 1, nx - 1)),
        "xVertex": np.zeros((ny - 1, nx - 1)), "yVertex": np.zeros((ny - 1, nx - 1)),
        "f_ground": np.zeros((ny - 1, nx - 1)), "flwafact": np.zeros((ny, nx, nz - 1)),
        "loadu": np.zeros((ny - 1, nx - 1, nz)), "loadv": np.zeros((ny - 1, nx - 1, nz)),
        "active_cell": np.zeros((ny, nx), np.int32), "active_vertex": np.zeros((ny - 1, nx - 1), np.int32),
        "umask_dirichlet": np.zeros((ny - 1, nx - 1, nz), np.int32),
        "vmask_dirichlet": np.zeros((ny - 1, nx - 1, nz), np.int32),
        "ice_mask": np.zeros((ny, nx), np.int32), "floating_mask": np.zeros((ny, nx), np.int32),
        "ocean_mask": np.zeros((ny, nx), np.int32), "land_mask": np.zeros((ny, nx), np.int32),
    }
    s = OrcSetup()
    for k, a in arrs.items():
        setattr(s, k, _p(a, _ip if a.dtype == np.int32 else _dp))
    u = np.zeros(m.vshape3) if uvel is None else np.array(uvel, dtype=np.float64, copy=True)
    v = np.zeros(m.vshape3) if vvel is None else np.array(vvel, dtype=np.float64, copy=True)
    rc = lib().orc_setup_solve(C.byref(om), C.byref(s), _p(u), _p(v))
    if rc != 0:
        raise RuntimeError(f"orc_setup_solve failed: {rc}")
    beta = np.zeros((ny - 1, nx - 1))
    rc = lib().orc_calcbeta(C.byref(om), C.byref(s), _p(u), _p(v), _p(beta))
    if rc != 0:
        raise RuntimeError(f"orc_calcbeta failed: {rc}")
    arrs["beta_internal"] = beta
    arrs["uvel"], arrs["vvel"] = u, v
    arrs["_keep"] = (keep, om, s)
    return arrs


def assemble_system(m, su, uvel, vvel):
    """A and b of one Picard iteration at velocity (uvel, vvel)."""
    keep, om, s = su["_keep"]
    nx, ny, nz = m.nx, m.ny, m.nz
    shp = (ny - 1, nx - 1, nz, 27)
    A = [np.zeros(shp) for _ in range(4)]
    bu, bv = np.zeros((ny - 1, nx - 1, nz)), np.zeros((ny - 1, nx - 1, nz))
    efvs = np.zeros((ny, nx, nz - 1))
    nnz = C.c_long(0)
    u = np.ascontiguousarray(uvel, np.float64)
    v = np.ascontiguousarray(vvel, np.float64)
    rc = lib().orc_assemble_system(C.byref(om), C.byref(s), _p(su["beta_internal"]), _p(u), _p(v),
                                   _p(efvs), *[_p(a) for a in A], _p(bu), _p(bv), C.byref(nnz))
    if rc != 0:
        raise RuntimeError(f"orc_assemble_system failed: {rc}")
    return A, bu, bv, efvs, nnz.value


def internal_stress(m, su, uvel, vvel, approx=2, efvs=None):
    """compute_internal_stress at velocity (uvel, vvel) for approximation
    approx (2 Blatter-Pattyn; APPROX_SSA, APPROX_L1L2 with the layer
    viscosities efvs, 4 DIVA): dict of the six stresses, each (ny, nx, nz-1)."""
    nx, ny, nz = m.nx, m.ny, m.nz
    names = ("tau_xz", "tau_yz", "tau_xx", "tau_yy", "tau_xy", "tau_eff")
    outs = {k: np.zeros((ny, nx, nz - 1)) for k in names}
    fn = lib().orc_internal_stress_approx
    fn.argtypes = ([C.c_int] * 4 + [_dp, _ip, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, C.c_double, C.c_int,
                                    _dp, _dp] + [_dp] * 6)
    ef = np.zeros((ny, nx, nz - 1)) if efvs is None else np.ascontiguousarray(efvs, np.float64)
    rc = fn(nx, ny, nz, 2, _p(su["sigma"]), _p(su["active_cell"], _ip), _p(su["xVertex"]), _p(su["yVertex"]),
            _p(su["stagusrf"]), _p(su["stagthck"]), _p(su["flwafact"]), _p(ef), m.which_efvs, m.efvs_constant,
            approx, _p(np.ascontiguousarray(uvel, np.float64)), _p(np.ascontiguousarray(vvel, np.float64)),
            *[_p(outs[k]) for k in names])
    if rc != 0:
        raise RuntimeError(f"orc_internal_stress failed: {rc}")
    return outs


def basal_friction_heatflx(m, su, uvel, vvel, beta, which=1):
    """compute_basal_friction_heatflx from the bed layer of (uvel, vvel):
    (ny, nx), W/m^2."""
    nx, ny, nz = m.nx, m.ny, m.nz
    out = np.zeros((ny, nx))
    fn = lib().orc_basal_friction_heatflx
    fn.argtypes = [C.c_int] * 5 + [_ip, _ip, _dp, _dp, _dp, C.c_int, _dp]
    fn.restype = None
    fn(nx, ny, nz, 2, m.periodic, _p(su["active_cell"], _ip), _p(su["active_vertex"], _ip),
       _p(np.ascontiguousarray(uvel, np.float64)), _p(np.ascontiguousarray(vvel, np.float64)),
       _p(np.ascontiguousarray(beta, np.float64)), which, _p(out))
    return out


def assemble_2d_system(m, su, beta, u2, v2, approx=APPROX_SSA):
    """One assembled 2-D system (SSA or L1L2) at the 2-D velocity (u2, v2)
    (ny-1, nx-1): A as four (ny-1, nx-1, 1, 27) arrays, b, efvs, nonzeros."""
    keep, om, s = su["_keep"]
    nx, ny, nz = m.nx, m.ny, m.nz
    A = [np.zeros((ny - 1, nx - 1, 1, 27)) for _ in range(4)]
    bu, bv = np.zeros((ny - 1, nx - 1)), np.zeros((ny - 1, nx - 1))
    efvs = np.zeros((ny, nx, nz - 1))
    nnz = C.c_long(0)
    rc = lib().orc_assemble_2d_system(C.byref(om), C.byref(s), approx,
                                      _p(np.ascontiguousarray(beta, np.float64)),
                                      _p(np.ascontiguousarray(u2, np.float64)),
                                      _p(np.ascontiguousarray(v2, np.float64)), _p(efvs),
                                      *[_p(a) for a in A], _p(bu), _p(bv), C.byref(nnz))
    if rc != 0:
        raise RuntimeError(f"orc_assemble_2d_system failed: {rc}")
    return A, bu, bv, efvs, nnz.value


def assemble_ssa_system(m, su, beta, u2, v2):
    return assemble_2d_system(m, su, beta, u2, v2, APPROX_SSA)


def velocity_3d_l1l2(m, su, efvs, uvel, vvel):
    """compute_3d_velocity_L1L2 (+ halo update): levels 1..nz-1 of copies
    of (uvel, vvel) from their basal level and the layer viscosities."""
    keep, om, s = su["_keep"]
    u = np.array(uvel, dtype=np.float64, copy=True)
    v = np.array(vvel, dtype=np.float64, copy=True)
    lib().orc_velocity_3d_l1l2(C.byref(om), C.byref(s), _p(np.ascontiguousarray(efvs, np.float64)),
                               _p(u), _p(v))
    return u, v


def assemble_diva_system(m, su, beta, u2, v2, btx, bty, eq3):
    """One assembled DIVA system at the mean velocity (u2, v2) with the
    traction (btx, bty); eq3 (ny, nx, 4, nz-1) is efvs_qp_3d, updated in
    place.  Returns A, bu, bv, efvs, omega_k (ny, nx, nz), omega (ny, nx),
    beta_eff (ny-1, nx-1), nonzeros."""
    keep, om, s = su["_keep"]
    nx, ny, nz = m.nx, m.ny, m.nz
    A = [np.zeros((ny - 1, nx - 1, 1, 27)) for _ in range(4)]
    bu, bv = np.zeros((ny - 1, nx - 1)), np.zeros((ny - 1, nx - 1))
    efvs = np.zeros((ny, nx, nz - 1))
    omk, omg, be = np.zeros((ny, nx, nz)), np.zeros((ny, nx)), np.zeros((ny - 1, nx - 1))
    assert eq3.dtype == np.float64 and eq3.flags["C_CONTIGUOUS"] and eq3.shape == (ny, nx, 4, nz - 1)
    nnz = C.c_long(0)
    c = np.ascontiguousarray
    rc = lib().orc_assemble_diva_system(C.byref(om), C.byref(s), _p(c(beta, np.float64)), _p(c(u2, np.float64)),
                                        _p(c(v2, np.float64)), _p(c(btx, np.float64)), _p(c(bty, np.float64)),
                                        _p(eq3), _p(efvs), _p(omk), _p(omg), _p(be), *[_p(a) for a in A],
                                        _p(bu), _p(bv), C.byref(nnz))
    if rc != 0:
        raise RuntimeError(f"orc_assemble_diva_system failed: {rc}")
    return A, bu, bv, efvs, omk, omg, be, nnz.value


def velocity_3d_diva(m, su, beta_eff, omega_k, omega, u2, v2, uvel, vvel):
    """The step after a DIVA linear solve: returns (btx, bty, uvel, vvel)."""
    keep, om, s = su["_keep"]
    c = np.ascontiguousarray
    bx, by = np.zeros((m.ny - 1, m.nx - 1)), np.zeros((m.ny - 1, m.nx - 1))
    u = np.array(uvel, dtype=np.float64, copy=True)
    v = np.array(vvel, dtype=np.float64, copy=True)
    lib().orc_velocity_3d_diva(C.byref(om), C.byref(s), _p(c(beta_eff, np.float64)), _p(c(omega_k, np.float64)),
                               _p(c(omega, np.float64)), _p(c(u2, np.float64)), _p(c(v2, np.float64)),
                               _p(bx), _p(by), _p(u), _p(v))
    return bx, by, u, v


def matvec(m, active_vertex, A, xu, xv):
    nx, ny, nz = m.nx, m.ny, m.nz
    yu, yv = np.zeros((ny - 1, nx - 1, nz)), np.zeros((ny - 1, nx - 1, nz))
    av = np.ascontiguousarray(active_vertex, np.int32)
    lib().orc_matvec_3d(nx, ny, nz, m.periodic, _p(av, _ip), *[_p(np.ascontiguousarray(a)) for a in A],
                        _p(np.ascontiguousarray(xu)), _p(np.ascontiguousarray(xv)), _p(yu), _p(yv))
    return yu, yv


def pcg(m, active_vertex, A, bu, bv, xu, xv, precond=1, variant=2, maxiters=200, tol=1e-8, ncheck=5):
    nx, ny, nz = m.nx, m.ny, m.nz
    xu = np.array(xu, np.float64, copy=True)
    xv = np.array(xv, np.float64, copy=True)
    av = np.ascontiguousarray(active_vertex, np.int32)
    err = C.c_double(0)
    nit = C.c_int(0)
    fn = lib().orc_pcg_chrongear_3d if variant == 3 else lib().orc_pcg_standard_3d
    fn.argtypes = [C.c_int] * 4 + [_ip] + [_dp] * 8 + [C.c_int, C.c_int, C.c_double, C.c_int,
                                                       _dp, _ip]
    rc = fn(nx, ny, nz, m.periodic, _p(av, _ip), *[_p(np.ascontiguousarray(a)) for a in A],
            _p(np.ascontiguousarray(bu)), _p(np.ascontiguousarray(bv)), _p(xu), _p(xv),
            precond, maxiters, tol, ncheck, C.byref(err), C.byref(nit))
    return xu, xv, err.value, nit.value, rc


def halo_cell(a, periodic=1, offset_ew=0.0, offset_ns=0.0):
    a = np.array(a, np.float64, copy=True)
    ny, nx = a.shape
    lib().orc_halo_cell_real.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_double, C.c_double]
    lib().orc_halo_cell_real(nx, ny, periodic, _p(a), offset_ew, offset_ns)
    return a


def halo_stag(a, periodic=1):
    a = np.array(a, np.float64, copy=True)
    W, V = a.shape[0], a.shape[1]
    nlead = int(np.prod(a.shape[2:])) if a.ndim > 2 else 1
    lib().orc_halo_stag(V + 1, W + 1, nlead, periodic, _p(a))
    return a
