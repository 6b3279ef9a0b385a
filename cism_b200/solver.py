"""Python front end of the B200 Blatter-Pattyn solver (ctypes over libbpgpu.so).

Mirrors the reference interface for the path it replaces:

* :func:`velo_higher_solve` -- ``glissade_velo_higher_solve`` with
  ``which_ho_sparse = 5``: setup on the host (C++), Picard loop on the GPU;
* :func:`pcg_solve` -- ``pcg_solver_standard_3d`` / ``pcg_solver_chrongear_3d``
  on an assembled system;
* :func:`matvec` -- ``matvec_multiply_structured_3d``;
* :func:`assemble` -- one assembled system (assembly + basal + Dirichlet BCs);
* :func:`batch_solve` -- many independent solves in one set of launches.

Every call goes through the C ABI declared in include/bp_b200.h.  There is
no CPU fallback: if the library or a CUDA device is missing, the context
constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

from . import configs

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbpgpu.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

STATUS = {0: "ok", 1: "NaN in PCG", 2: "singular Jacobian", 3: "PCG not converged",
          4: "Picard not converged", 5: "all-zero matrix", 6: "CUDA error",
          7: "iteration budget exhausted", 9: "invalid beta", 10: "bad arguments",
          11: "no CUDA device"}
FP64, MIXED = 0, 1


class BPError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"bp status {code} ({STATUS.get(code, '?')}) {msg}".strip())
        self.code = code


class Sliding(C.Structure):
    """bp_sliding: a velocity-dependent sliding law."""
    _fields_ = [
        ("law", C.c_int), ("f_ground", _dp), ("effecpress_stag", _dp), ("c_space_factor_stag", _dp),
        ("flwa_basal_stag", _dp), ("yield_stress", _dp), ("topg", _dp), ("eus", C.c_double),
        ("beta_grounded_min", C.c_double), ("beta_powerlaw_umax", C.c_double),
        ("powerlaw_c", C.c_double), ("powerlaw_m", C.c_double), ("coulomb_c", C.c_double),
        ("coulomb_bump_max_slope", C.c_double), ("coulomb_bump_wavelength", C.c_double),
        ("friction_powerlaw_k", C.c_double), ("pseudo_plastic_q", C.c_double),
        ("pseudo_plastic_u0", C.c_double), ("pseudo_plastic_phimin", C.c_double),
        ("pseudo_plastic_phimax", C.c_double), ("pseudo_plastic_bedmin", C.c_double),
        ("pseudo_plastic_bedmax", C.c_double),
    ]


class L1L2(C.Structure):
    """bp_l1l2: the fields of the L1L2 solve beyond the shallow-shelf ones."""
    _fields_ = [("thck", _dp), ("flwa", _dp), ("dusrf_dx", _dp), ("dusrf_dy", _dp),
                ("rhoi", C.c_double), ("grav", C.c_double)]


class Diva(C.Structure):
    """bp_diva: the state a DIVA solve carries from one solve to the next."""
    _fields_ = [("uvel_2d", _dp), ("vvel_2d", _dp), ("btractx", _dp), ("btracty", _dp), ("efvs", _dp),
                ("thck", _dp), ("ice_plus_land_mask", _ip)]


class Inputs(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nhalo", C.c_int),
        ("periodic", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
        ("sigma", _dp), ("stagusrf", _dp), ("stagthck", _dp), ("beta_internal", _dp),
        ("flwafact", _dp), ("active_cell", _ip), ("active_vertex", _ip),
        ("loadu", _dp), ("loadv", _dp), ("umask_dirichlet", _ip), ("vmask_dirichlet", _ip),
        ("which_babc", C.c_int), ("which_efvs", C.c_int), ("efvs_constant", C.c_double),
        ("which_assemble_beta", C.c_int), ("which_resid", C.c_int), ("pcg_variant", C.c_int),
        ("which_precond", C.c_int), ("maxiter_nonlinear", C.c_int), ("pcg_maxiters", C.c_int),
        ("pcg_ncheck", C.c_int), ("pcg_tol", C.c_double), ("precision", C.c_int),
        ("inner_tol", C.c_double), ("sliding", C.POINTER(Sliding)), ("approx_2d", C.c_int),
        ("l1l2", C.POINTER(L1L2)), ("diva", C.POINTER(Diva)), ("guess_mode", C.c_int),
    ]


GUESS_GIVEN, GUESS_LEARNED = 0, 1  # bp_guess_mode


class Stats(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("picard_iters", C.c_int), ("pcg_iters_total", C.c_int),
        ("pcg_iters_last", C.c_int), ("refine_steps_total", C.c_int), ("converged", C.c_int),
        ("pcg_err_last", C.c_double), ("resid_velo", C.c_double), ("L2_norm", C.c_double),
        ("L2_norm_relative", C.c_double), ("ms_upload", C.c_float), ("ms_assemble", C.c_float),
        ("ms_pcg", C.c_float), ("ms_total", C.c_float), ("h2d_bytes", C.c_double),
        ("d2h_bytes", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Model(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("nhalo", C.c_int), ("periodic", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double),
        ("thck", _dp), ("usrf", _dp), ("topg", _dp), ("flwa", _dp), ("beta_external", _dp),
        ("kinbcmask", _ip),
        ("eus", C.c_double), ("thklim", C.c_double), ("max_slope", C.c_double),
        ("thck_gradient_ramp", C.c_double), ("rhoi", C.c_double), ("rhoo", C.c_double),
        ("grav", C.c_double), ("beta_const", C.c_double), ("beta_grounded_min", C.c_double),
        ("efvs_constant", C.c_double),
        ("which_babc", C.c_int), ("which_efvs", C.c_int), ("which_resid", C.c_int),
        ("which_sparse", C.c_int), ("which_precond", C.c_int), ("which_gradient", C.c_int),
        ("which_gradient_margin", C.c_int), ("which_assemble_beta", C.c_int),
        ("which_assemble_taud", C.c_int), ("which_ground", C.c_int),
        ("maxiter_nonlinear", C.c_int), ("pcg_maxiters", C.c_int), ("pcg_ncheck", C.c_int),
        ("pcg_tol", C.c_double), ("precision", C.c_int), ("inner_tol", C.c_double),
        ("sliding", C.POINTER(Sliding)), ("approx_2d", C.c_int), ("diva", C.POINTER(Diva)),
    ]


class SetupArrays(C.Structure):
    _fields_ = [("sigma", _dp), ("stagusrf", _dp), ("stagthck", _dp), ("beta_internal", _dp),
                ("flwafact", _dp), ("active_cell", _ip), ("active_vertex", _ip),
                ("loadu", _dp), ("loadv", _dp), ("umask_dirichlet", _ip), ("vmask_dirichlet", _ip),
                ("f_ground", _dp), ("flwa_basal_stag", _dp), ("sliding", Sliding),
                ("dusrf_dx", _dp), ("dusrf_dy", _dp), ("l1l2", L1L2),
                ("ice_plus_land_mask", _ip), ("diva", Diva)]


SETUP_ARRAYS = [k for k, _ in SetupArrays._fields_[:11]]


_lib = None


def lib():
    """Load libbpgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() (make -C cism_b200/csrc)")
        L = C.CDLL(LIB_PATH)
        L.bp_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
        L.bp_destroy.argtypes = [C.c_void_p]
        L.bp_last_error.argtypes = [C.c_void_p]
        L.bp_last_error.restype = C.c_char_p
        L.bp_solve.argtypes = [C.c_void_p, C.POINTER(Inputs), _dp, _dp, _dp, C.POINTER(Stats)]
        L.bp_batch_solve.argtypes = [C.c_void_p, C.c_int, C.POINTER(Inputs), C.POINTER(_dp),
                                     C.POINTER(_dp), C.POINTER(_dp), C.POINTER(Stats)]
        L.bp_pcg.argtypes = ([C.c_void_p] + [C.c_int] * 4 + [_ip] + [_dp] * 8 +
                             [C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, _dp, _ip])
        L.bp_matvec.argtypes = [C.c_void_p] + [C.c_int] * 4 + [_ip] + [_dp] * 8
        L.bp_assemble.argtypes = [C.c_void_p, C.POINTER(Inputs)] + [_dp] * 9
        L.bp_setup.argtypes = [C.POINTER(Model), C.POINTER(SetupArrays), _dp, _dp, C.POINTER(Inputs)]
        L.bp_velo_higher_solve.argtypes = [C.c_void_p, C.POINTER(Model), _dp, _dp, _dp, C.POINTER(Stats)]
        L.bp_problem_create.argtypes = [C.c_void_p, C.c_int, C.POINTER(Inputs), C.POINTER(C.c_void_p)]
        L.bp_problem_set_guess.argtypes = [C.c_void_p, C.POINTER(_dp), C.POINTER(_dp)]
        L.bp_problem_run.argtypes = [C.c_void_p, C.POINTER(Stats)]
        L.bp_problem_get.argtypes = [C.c_void_p, C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp)]
        L.bp_problem_destroy.argtypes = [C.c_void_p]
        L.bp_problem_timing.argtypes = [C.c_void_p, C.c_int]
        L.bp_problem_kernel_times.argtypes = [C.c_void_p, _dp, _ip]
        L.bp_problem_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_long)] * 3 + [_dp, _dp]
        L.bp_problem_tune_mv.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.POINTER(C.c_float)]
        L.bp_problem_mv_nodes.argtypes = [C.c_void_p, _dp, _dp, _ip, _ip]
        L.bp_problem_diagnostics.argtypes = [C.c_void_p, C.c_int] + [C.POINTER(_dp)] * 7
        L.bp_timer_start.argtypes = [C.c_void_p]
        L.bp_timer_stop.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
        L.bp_guess_load.argtypes = [C.c_void_p, C.c_char_p]
        L.bp_guess_launches.argtypes = [C.c_void_p]
        L.bp_problem_get_guess.argtypes = [C.c_void_p, C.POINTER(_dp), C.POINTER(_dp)]
        _lib = L
    return _lib


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _p(a):
    return a.ctypes.data_as(_ip if a.dtype == np.int32 else _dp)


class Prepared:
    """Boundary inputs of one solve (host arrays kept alive with the struct)."""

    def __init__(self, model: configs.BPModel, arrays: dict, inputs: Inputs, keep):
        self.model = model
        self.arrays = arrays
        self.inputs = inputs
        self._keep = keep


def make_model_struct(m: configs.BPModel, precision: int = FP64, inner_tol: float = 1e-4):
    keep = []

    def f(a):
        a = _f64(a)
        keep.append(a)
        return _p(a)

    s = Model()
    s.nx, s.ny, s.nz, s.nhalo, s.periodic = m.nx, m.ny, m.nz, 2, m.periodic
    s.dx, s.dy = m.dx, m.dy
    s.thck, s.usrf, s.topg, s.flwa = f(m.thck), f(m.usrf), f(m.topg), f(m.flwa)
    s.beta_external = f(m.beta_external)
    if m.kinbcmask is not None:
        k = _i32(m.kinbcmask)
        keep.append(k)
        s.kinbcmask = _p(k)
    else:
        s.kinbcmask = C.cast(None, _ip)
    for name in ("eus", "thklim", "max_slope", "thck_gradient_ramp", "rhoi", "rhoo", "grav",
                 "beta_const", "beta_grounded_min", "efvs_constant", "which_babc", "which_efvs",
                 "which_resid", "which_sparse", "which_precond", "which_gradient",
                 "which_gradient_margin", "which_assemble_beta", "which_assemble_taud",
                 "which_ground", "maxiter_nonlinear", "pcg_maxiters", "pcg_ncheck", "pcg_tol"):
        setattr(s, name, getattr(m, name))
    s.precision = precision
    s.inner_tol = inner_tol
    s.approx_2d = m.approx_2d
    s.sliding = C.cast(None, C.POINTER(Sliding))
    if m.sliding is not None:
        if m.which_babc != m.sliding.law:
            raise ValueError("which_babc must equal sliding.law")
        sl = sliding_struct(m.sliding, f)
        keep.append(sl)
        s.sliding = C.pointer(sl)
    return s, keep


def sliding_struct(law: "configs.SlidingLaw", f) -> Sliding:
    """bp_sliding of a model's sliding law (vertex fields through f; the
    setup fills f_ground, flwa_basal_stag, topg and eus)."""
    sl = Sliding()
    sl.law = law.law
    null = C.cast(None, _dp)
    for name in ("effecpress_stag", "c_space_factor_stag", "yield_stress"):
        a = getattr(law, name)
        setattr(sl, name, f(a) if a is not None else null)
    sl.f_ground = sl.flwa_basal_stag = sl.topg = null
    for name in ("beta_powerlaw_umax", "powerlaw_c", "powerlaw_m", "coulomb_c",
                 "coulomb_bump_max_slope", "coulomb_bump_wavelength", "friction_powerlaw_k",
                 "pseudo_plastic_q", "pseudo_plastic_u0", "pseudo_plastic_phimin",
                 "pseudo_plastic_phimax", "pseudo_plastic_bedmin", "pseudo_plastic_bedmax"):
        setattr(sl, name, getattr(law, name))
    return sl


def prepare(m: configs.BPModel, uvel=None, vvel=None, precision: int = FP64,
            inner_tol: float = 1e-4, guess_mode: int = GUESS_GIVEN) -> tuple:
    """Host setup (bp_setup): returns (Prepared, uvel, vvel).  guess_mode =
    GUESS_LEARNED makes the solve start from the network loaded into the
    context (Context.load_guess) instead of (uvel, vvel)."""
    nx, ny, nz = m.nx, m.ny, m.nz
    arrays = {
        "sigma": np.zeros(nz), "stagusrf": np.zeros((ny - 1, nx - 1)),
        "stagthck": np.zeros((ny - 1, nx - 1)), "beta_internal": np.zeros((ny - 1, nx - 1)),
        "flwafact": np.zeros((ny, nx, nz - 1)), "active_cell": np.zeros((ny, nx), np.int32),
        "active_vertex": np.zeros((ny - 1, nx - 1), np.int32),
        "loadu": np.zeros((ny - 1, nx - 1, nz)), "loadv": np.zeros((ny - 1, nx - 1, nz)),
        "umask_dirichlet": np.zeros((ny - 1, nx - 1, nz), np.int32),
        "vmask_dirichlet": np.zeros((ny - 1, nx - 1, nz), np.int32),
    }
    sa = SetupArrays(*[_p(arrays[k]) for k in SETUP_ARRAYS])
    if m.sliding is not None:
        arrays["f_ground"] = np.zeros((ny - 1, nx - 1))
        arrays["flwa_basal_stag"] = np.zeros((ny - 1, nx - 1))
        sa.f_ground, sa.flwa_basal_stag = _p(arrays["f_ground"]), _p(arrays["flwa_basal_stag"])
    if m.approx_2d == configs.APPROX_L1L2:
        arrays["dusrf_dx"] = np.zeros((ny - 1, nx - 1))
        arrays["dusrf_dy"] = np.zeros((ny - 1, nx - 1))
        sa.dusrf_dx, sa.dusrf_dy = _p(arrays["dusrf_dx"]), _p(arrays["dusrf_dy"])
    ms, keep = make_model_struct(m, precision, inner_tol)
    if m.approx_2d == configs.APPROX_DIVA:
        # the carried-over state (copies: the setup and the solve write them)
        st0 = m.diva_state or {}
        vs = (ny - 1, nx - 1)
        for name, shape in (("uvel_2d", vs), ("vvel_2d", vs), ("btractx", vs), ("btracty", vs),
                            ("efvs_in", (ny, nx, nz - 1))):
            a = st0.get(name[:-3] if name == "efvs_in" else name)
            arrays[name] = np.zeros(shape) if a is None else np.array(a, np.float64, copy=True)
        arrays["ice_plus_land_mask"] = np.zeros((ny, nx), np.int32)
        sa.ice_plus_land_mask = _p(arrays["ice_plus_land_mask"])
        dv = Diva(_p(arrays["uvel_2d"]), _p(arrays["vvel_2d"]), _p(arrays["btractx"]), _p(arrays["btracty"]),
                  _p(arrays["efvs_in"]), C.cast(None, _dp), C.cast(None, _ip))
        keep.append(dv)
        ms.diva = C.pointer(dv)
    u = np.zeros(m.vshape3) if uvel is None else np.array(uvel, np.float64, copy=True)
    v = np.zeros(m.vshape3) if vvel is None else np.array(vvel, np.float64, copy=True)
    inp = Inputs()
    rc = lib().bp_setup(C.byref(ms), C.byref(sa), _p(u), _p(v), C.byref(inp))
    if rc != 0:
        raise BPError(rc, "in bp_setup")
    inp.guess_mode = guess_mode
    return Prepared(m, arrays, inp, (keep, ms, sa)), u, v


class Context:
    """One CUDA device + stream + persistent device buffers (bp_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        rc = lib().bp_create(device, C.byref(h))
        if rc != 0:
            raise BPError(rc, "bp_create failed (a CUDA device is required)")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().bp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, allow=(0, 3, 4, 5)):
        if rc not in allow:
            msg = lib().bp_last_error(self.h)
            raise BPError(rc, msg.decode() if msg else "")
        return rc

    # -- learned initial guess (bp_guess_load) -------------------------------
    def load_guess(self, path: str):
        """Load the U-Net weights (.bin; a .npz path means the .bin beside it)
        into the context; inputs with guess_mode = GUESS_LEARNED then start
        from the network's guess, formed on the device."""
        if path.endswith(".npz"):
            path = path[:-4] + ".bin"
        self._check(lib().bp_guess_load(self.h, path.encode()), allow=(0,))

    def guess_launches(self) -> int:
        return int(lib().bp_guess_launches(self.h))

    # -- whole solve --------------------------------------------------------
    def solve_prepared(self, prep: Prepared, uvel, vvel, want_efvs=True):
        m = prep.model
        u = np.array(uvel, np.float64, copy=True)
        v = np.array(vvel, np.float64, copy=True)
        efvs = np.zeros((m.ny, m.nx, m.nz - 1)) if want_efvs else None
        st = Stats()
        rc = lib().bp_solve(self.h, C.byref(prep.inputs), _p(u), _p(v),
                            _p(efvs) if efvs is not None else C.cast(None, _dp), C.byref(st))
        self._check(rc)
        out = st.as_dict()
        if m.approx_2d == configs.APPROX_DIVA:  # the state written back for the next solve
            out["diva"] = {k: prep.arrays[k].copy() for k in ("uvel_2d", "vvel_2d", "btractx", "btracty")}
        return u, v, efvs, out

    def velo_higher_solve(self, m: configs.BPModel, uvel=None, vvel=None, precision: int = FP64,
                          inner_tol: float = 1e-4):
        """glissade_velo_higher_solve: host setup + device Picard loop."""
        prep, u, v = prepare(m, uvel, vvel, precision, inner_tol)
        return self.solve_prepared(prep, u, v)

    def batch_solve(self, preps: Sequence[Prepared], uvels, vvels, want_efvs=False):
        n = len(preps)
        arr = (Inputs * n)(*[p.inputs for p in preps])
        us = [np.array(u, np.float64, copy=True) for u in uvels]
        vs = [np.array(v, np.float64, copy=True) for v in vvels]
        es = [np.zeros((p.model.ny, p.model.nx, p.model.nz - 1)) for p in preps] if want_efvs else None
        up = (_dp * n)(*[_p(a) for a in us])
        vp = (_dp * n)(*[_p(a) for a in vs])
        ep = (_dp * n)(*[_p(a) for a in es]) if es else C.cast(None, C.POINTER(_dp))
        st = (Stats * n)()
        rc = lib().bp_batch_solve(self.h, n, arr, up, vp, ep, st)
        self._check(rc)
        return us, vs, es, [s.as_dict() for s in st]

    def problem(self, preps: Sequence[Prepared]) -> "Problem":
        return Problem(self, preps)

    def timer_start(self):
        lib().bp_timer_start(self.h)

    def timer_stop(self) -> float:
        ms = C.c_float()
        lib().bp_timer_stop(self.h, C.byref(ms))
        return ms.value

    # -- matrix-level entry points -------------------------------------------
    def pcg_solve(self, m: configs.BPModel, active_vertex, A, bu, bv, xu, xv, precond=1,
                  variant=2, tol=1e-8, maxiters=200, ncheck=5, precision=FP64):
        xu = np.array(xu, np.float64, copy=True)
        xv = np.array(xv, np.float64, copy=True)
        av = _i32(active_vertex)
        A = [_f64(a) for a in A]
        bu, bv = _f64(bu), _f64(bv)
        err = C.c_double(0)
        nit = C.c_int(0)
        rc = lib().bp_pcg(self.h, m.nx, m.ny, m.nz, m.periodic, _p(av), *[_p(a) for a in A],
                          _p(bu), _p(bv), _p(xu), _p(xv), precond, variant, tol, maxiters, ncheck,
                          precision, C.byref(err), C.byref(nit))
        self._check(rc)
        return xu, xv, err.value, nit.value, rc

    def matvec(self, m: configs.BPModel, active_vertex, A, xu, xv):
        av = _i32(active_vertex)
        A = [_f64(a) for a in A]
        xu, xv = _f64(xu), _f64(xv)
        yu = np.zeros(m.vshape3)
        yv = np.zeros(m.vshape3)
        rc = lib().bp_matvec(self.h, m.nx, m.ny, m.nz, m.periodic, _p(av), *[_p(a) for a in A],
                             _p(xu), _p(xv), _p(yu), _p(yv))
        self._check(rc, allow=(0,))
        return yu, yv

    def assemble(self, prep: Prepared, uvel, vvel):
        m = prep.model
        shp = (m.ny - 1, m.nx - 1, m.nz, 27)
        A = [np.zeros(shp) for _ in range(4)]
        bu, bv = np.zeros(m.vshape3), np.zeros(m.vshape3)
        efvs = np.zeros((m.ny, m.nx, m.nz - 1))
        u, v = _f64(uvel), _f64(vvel)
        rc = lib().bp_assemble(self.h, C.byref(prep.inputs), _p(u), _p(v), *[_p(a) for a in A],
                               _p(bu), _p(bv), _p(efvs))
        self._check(rc, allow=(0, 5))
        return A, bu, bv, efvs


KERNEL_CATEGORIES = ("pcg_matvec_fp64", "pcg_update_fp64", "residual_check_fp64", "inner_matvec_fp32",
                     "inner_update_fp32", "assembly_qp", "assembly_rows", "rhs", "other")


class Problem:
    """A compiled solve (or batch) resident in device memory (bp_problem)."""

    def __init__(self, ctx: "Context", preps: Sequence[Prepared]):
        self.ctx = ctx
        self.preps = list(preps)
        self.n = len(self.preps)
        self._arr = (Inputs * self.n)(*[p.inputs for p in self.preps])
        h = C.c_void_p()
        rc = lib().bp_problem_create(ctx.h, self.n, self._arr, C.byref(h))
        ctx._check(rc, allow=(0,))
        self.h = h

    def set_guess(self, uvels, vvels):
        """Initial guesses per instance; None for an instance whose inputs ask
        for the learned guess (guess_mode = GUESS_LEARNED)."""
        us = [None if u is None else _f64(u) for u in uvels]
        vs = [None if v is None else _f64(v) for v in vvels]
        ptr = lambda a: C.cast(None, _dp) if a is None else _p(a)
        rc = lib().bp_problem_set_guess(self.h, (_dp * self.n)(*[ptr(a) for a in us]),
                                        (_dp * self.n)(*[ptr(a) for a in vs]))
        self.ctx._check(rc, allow=(0,))

    def get_guess(self):
        """The stored initial guess of each instance (3-D solves)."""
        us = [np.zeros(p.model.vshape3) for p in self.preps]
        vs = [np.zeros(p.model.vshape3) for p in self.preps]
        rc = lib().bp_problem_get_guess(self.h, (_dp * self.n)(*[_p(a) for a in us]),
                                        (_dp * self.n)(*[_p(a) for a in vs]))
        self.ctx._check(rc, allow=(0,))
        return us, vs

    def run(self):
        st = (Stats * self.n)()
        rc = lib().bp_problem_run(self.h, st)
        self.ctx._check(rc)
        return [s.as_dict() for s in st]

    def get(self, want_efvs=False):
        us = [np.zeros(p.model.vshape3) for p in self.preps]
        vs = [np.zeros(p.model.vshape3) for p in self.preps]
        es = [np.zeros((p.model.ny, p.model.nx, p.model.nz - 1)) for p in self.preps] if want_efvs else None
        rc = lib().bp_problem_get(self.h, (_dp * self.n)(*[_p(a) for a in us]),
                                  (_dp * self.n)(*[_p(a) for a in vs]),
                                  (_dp * self.n)(*[_p(a) for a in es]) if es else C.cast(None, C.POINTER(_dp)))
        self.ctx._check(rc, allow=(0,))
        return us, vs, es

    def diagnostics(self, which_bfric: int = 1):
        """Post-solve diagnostics at the last run's solution, per instance:
        the six element stresses (ny, nx, nz-1) and bfricflx (ny, nx)."""
        names = ("tau_xz", "tau_yz", "tau_xx", "tau_yy", "tau_xy", "tau_eff")
        out = [{k: np.zeros((p.model.ny, p.model.nx, p.model.nz - 1)) for k in names} |
               {"bfricflx": np.zeros((p.model.ny, p.model.nx))} for p in self.preps]
        arrs = [(_dp * self.n)(*[_p(o[k]) for o in out]) for k in names + ("bfricflx",)]
        rc = lib().bp_problem_diagnostics(self.h, which_bfric, *arrs)
        self.ctx._check(rc, allow=(0,))
        return out

    def tune_mv(self, store: int, minb: int = 0, grid: int = 0, reps: int = 50):
        """Mean ms of a plain y = A x launch (store 0 full, 1 sym FP64, 2 sym FP32)."""
        ms = C.c_float()
        rc = lib().bp_problem_tune_mv(self.h, store, minb, grid, reps, C.byref(ms))
        return ms.value if rc == 0 else None

    def timing(self, enable: bool):
        lib().bp_problem_timing(self.h, 1 if enable else 0)

    def kernel_times(self):
        ms = (C.c_double * len(KERNEL_CATEGORIES))()
        n = (C.c_int * len(KERNEL_CATEGORIES))()
        lib().bp_problem_kernel_times(self.h, ms, n)
        return {k: (ms[i], n[i]) for i, k in enumerate(KERNEL_CATEGORIES)}

    def mv_nodes(self):
        """(FP64 nodes, FP32 nodes) of the last timing run's Krylov matvecs and
        the autotuner's (minb, grid)."""
        a, b = C.c_double(), C.c_double()
        mb, g = C.c_int(), C.c_int()
        lib().bp_problem_mv_nodes(self.h, C.byref(a), C.byref(b), C.byref(mb), C.byref(g))
        return a.value, b.value, mb.value, g.value

    def info(self):
        nodes, cols, elems = C.c_long(), C.c_long(), C.c_long()
        b64, b32 = C.c_double(), C.c_double()
        lib().bp_problem_info(self.h, C.byref(nodes), C.byref(cols), C.byref(elems), C.byref(b64),
                              C.byref(b32))
        return {"nodes": nodes.value, "columns": cols.value, "elements": elems.value,
                "matvec_bytes_fp64": b64.value, "matvec_bytes_fp32": b32.value}

    def close(self):
        if getattr(self, "h", None):
            lib().bp_problem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def velo_higher_solve(m: configs.BPModel, uvel=None, vvel=None, precision: int = FP64,
                      inner_tol: float = 1e-4):
    return default_context().velo_higher_solve(m, uvel, vvel, precision, inner_tol)
