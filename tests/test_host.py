"""CPU tests of the product's host side: the setup mirror (C++), the host
plan (compaction, periodic images) and the device kernels' per-thread
bodies (compiled for the CPU by tests/hostemu), all against the oracle, and
the C-ABI library's exported symbols."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from cism_b200 import configs, solver
from oracle import oracle

from helpers import oracle_system, owned_active_rows, random_state, rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU = os.path.join(ROOT, "tests", "hostemu", "libhostemu.so")
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _p(a):
    return a.ctypes.data_as(_ip if a.dtype == np.int32 else _dp)


def _models():
    out = [configs.dome(), configs.slab(n=24), configs.marine(n=40, dx=4000.0),
           configs.analytic_slab(nz=8)]
    m = configs.marine(n=32, dx=4000.0)
    m.which_assemble_beta = 0
    m.name = "marine_standard_beta"
    out.append(m)
    m = configs.dome()
    m.kinbcmask = np.zeros((m.ny - 1, m.nx - 1), np.int32)
    m.kinbcmask[15:18, 14:16] = 1
    m.which_babc = 5
    m.beta_external[:] = 500.0
    m.name = "dome_kinematic_bc"
    out.append(m)
    m = configs.dome(n=20).copy(periodic=0)
    m.name = "dome_outflow"
    out.append(m)
    # standard (finite-element) gravity assembly, :4436-4528
    m = configs.slab(n=24).copy(which_assemble_taud=configs.ASSEMBLE_STANDARD)
    m.name = "slab_standard_taud"
    out.append(m)
    m = configs.marine(n=32, dx=4000.0).copy(which_assemble_taud=configs.ASSEMBLE_STANDARD, periodic=0)
    m.name = "marine_outflow_standard_taud"
    out.append(m)
    # first- and second-order upstream surface gradients
    # (glissade_grid_operators.F90:1028-1093)
    for g in (1, 2):
        m = configs.marine(n=32, dx=4000.0).copy(which_gradient=g)
        m.name = f"marine_upstream{g}_gradient"
        out.append(m)
    return out


MODELS = _models()


@pytest.mark.parametrize("m", MODELS, ids=lambda m: m.name)
def test_setup_mirror_bitwise(m):
    prep, u, v = solver.prepare(m)
    su = oracle.setup(m)
    for k, a in prep.arrays.items():
        assert np.array_equal(a, su[k]), k


@pytest.mark.parametrize("m", MODELS, ids=lambda m: m.name)
def test_kernel_bodies_match_oracle(m):
    emu = C.CDLL(EMU)
    prep, _, _ = solver.prepare(m)
    su, u, v, A, bu, bv, efvs = oracle_system(m, seed=0, scale=10.0)
    shp = (m.ny - 1, m.nx - 1, m.nz, 27)
    E = [np.zeros(shp) for _ in range(4)]
    ebu, ebv = np.zeros(m.vshape3), np.zeros(m.vshape3)
    eef = np.zeros((m.ny, m.nx, m.nz - 1))
    rc = emu.emu_assemble(C.byref(prep.inputs), _p(np.ascontiguousarray(u)), _p(np.ascontiguousarray(v)),
                          *[_p(a) for a in E], _p(ebu), _p(ebv), _p(eef))
    assert rc == 0
    rows = owned_active_rows(m, su["active_vertex"])
    for a, e in zip(A, E):
        assert np.max(np.abs(a[rows] - e[rows])) <= 1e-13 * np.max(np.abs(a[rows]))
    assert rel_l2([ebu[rows], ebv[rows]], [bu[rows], bv[rows]]) < 1e-13
    assert np.max(np.abs(eef - efvs)) <= 1e-13 * np.max(np.abs(efvs))
    xu, xv = random_state(m, su, seed=9, scale=1.0)
    yu, yv = oracle.matvec(m, su["active_vertex"], A, xu, xv)
    eyu, eyv = np.zeros(m.vshape3), np.zeros(m.vshape3)
    av = np.ascontiguousarray(su["active_vertex"], np.int32)
    rc = emu.emu_matvec(m.nx, m.ny, m.nz, m.periodic, _p(av), *[_p(np.ascontiguousarray(a)) for a in A],
                        _p(xu), _p(xv), _p(eyu), _p(eyv))
    assert rc == 0
    assert rel_l2([eyu, eyv], [yu, yv]) < 1e-14


@pytest.mark.parametrize("m", MODELS, ids=lambda m: m.name)
def test_element_centric_assembly_is_bitwise_the_row_form(m):
    """Pass 2 of the assembly in its element-centric form (each element's
    four blocks formed once, k_asm_elem, then summed per row in the
    reference's element order) gives the matrix, the right-hand side and
    the viscosity of the row-integrating form bit for bit."""
    emu = C.CDLL(EMU)
    prep, _, _ = solver.prepare(m)
    su, u, v, A, bu, bv, efvs = oracle_system(m, seed=4, scale=10.0)
    outs = []
    for gather in (0, 1):
        E = [np.zeros((m.ny - 1, m.nx - 1, m.nz, 27)) for _ in range(4)]
        ebu, ebv = np.zeros(m.vshape3), np.zeros(m.vshape3)
        eef = np.zeros((m.ny, m.nx, m.nz - 1))
        rc = emu.emu_assemble_form(C.byref(prep.inputs), _p(np.ascontiguousarray(u)),
                                   _p(np.ascontiguousarray(v)), *[_p(a) for a in E], _p(ebu), _p(ebv),
                                   _p(eef), C.c_int(gather))
        assert rc == 0
        outs.append(E + [ebu, ebv, eef])
    assert np.count_nonzero(outs[0][0]) > 0
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("m", MODELS[:4], ids=lambda m: m.name)
def test_symmetric_storage_matvec_bodies(m):
    """The device's half-storage matvec (lower stencil half read from the
    neighbours' rows), FP64 and FP32, against the oracle's full-row matvec."""
    emu = C.CDLL(EMU)
    su, u, v, A, bu, bv, efvs = oracle_system(m, seed=2, scale=10.0)
    xu, xv = random_state(m, su, seed=3, scale=1.0)
    yu, yv = oracle.matvec(m, su["active_vertex"], A, xu, xv)
    av = np.ascontiguousarray(su["active_vertex"], np.int32)
    for fp32, tol in ((0, 1e-13), (1, 1e-6)):
        eyu, eyv = np.zeros(m.vshape3), np.zeros(m.vshape3)
        rc = emu.emu_matvec_sym(m.nx, m.ny, m.nz, m.periodic, _p(av),
                                *[_p(np.ascontiguousarray(a)) for a in A], _p(xu), _p(xv),
                                _p(eyu), _p(eyv), fp32)
        assert rc == 0
        assert rel_l2([eyu, eyv], [yu, yv]) < tol, fp32


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "bp_b200.h")).read()
    names = set(re.findall(r"^\s*(?:int|const char \*)\s*\**\s*(bp_\w+)\s*\(", hdr, re.M))
    assert {"bp_create", "bp_solve", "bp_pcg", "bp_matvec", "bp_assemble", "bp_batch_solve"} <= names
    lib = C.CDLL(solver.LIB_PATH)
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert lib.bp_abi_version() == int(re.search(r"#define BP_ABI_VERSION (\d+)", hdr).group(1))


def test_context_needs_a_device():
    """No CPU fallback: without a CUDA device bp_create fails loudly."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(solver.BPError) as e:
        solver.Context(0)
    assert e.value.code == 11


@pytest.mark.parametrize("m", MODELS[:4], ids=lambda m: m.name)
def test_fp32_copy_keeps_row_sums(m):
    """The FP32 matrix of the mixed path carries the rounding of each row in
    its FP64 diagonal block: on the translation fields (u = 1, v = 0 and
    u = 0, v = 1) it gives the FP64 product to summation rounding, where an
    entry-wise FP32 copy is off by about eps32 times the row's entries."""
    emu = C.CDLL(EMU)
    su, u, v, A, bu, bv, efvs = oracle_system(m, seed=4, scale=10.0)
    av = np.ascontiguousarray(su["active_vertex"], np.int32)
    one = configs.halo_fill_stag(np.ones(m.vshape3) * av[..., None], m.periodic)
    zero = np.zeros(m.vshape3)
    scale = max(np.abs(a).max() for a in A)
    for xu, xv in ((one, zero), (zero, one)):
        out = []
        for fp32 in (0, 1):
            eyu, eyv = np.zeros(m.vshape3), np.zeros(m.vshape3)
            rc = emu.emu_matvec_sym(m.nx, m.ny, m.nz, m.periodic, _p(av),
                                    *[_p(np.ascontiguousarray(a)) for a in A], _p(xu), _p(xv),
                                    _p(eyu), _p(eyv), fp32)
            assert rc == 0
            out.append((eyu, eyv))
        diff = max(np.abs(out[0][0] - out[1][0]).max(), np.abs(out[0][1] - out[1][1]).max())
        assert diff <= 1e-13 * scale


@pytest.mark.parametrize("m", MODELS[:4], ids=lambda m: m.name)
def test_sia_preconditioner_bodies(m):
    """The device's SIA column preconditioner (coefficients from half or full
    storage, Thomas solve) against a banded solve of each owned column's
    vertical uu and vv tridiagonals (offsets 4, 13, 22) of the oracle's
    matrix."""
    from scipy.linalg import solve_banded

    emu = C.CDLL(EMU)
    su, u, v, A, bu, bv, efvs = oracle_system(m, seed=6, scale=10.0)
    ru, rv = random_state(m, su, seed=7, scale=1.0)
    av = np.ascontiguousarray(su["active_vertex"], np.int32)
    js, is_ = m.owned_vertex_slices()
    ref = []
    for Ab, r in ((A[0], ru), (A[3], rv)):
        z = np.zeros(m.vshape3)
        for j in range(js.start, js.stop):
            for i in range(is_.start, is_.stop):
                if not av[j, i]:
                    continue
                ab = np.zeros((3, m.nz))
                ab[0, 1:] = Ab[j, i, :-1, 22]
                ab[1, :] = Ab[j, i, :, 13]
                ab[2, :-1] = Ab[j, i, 1:, 4]
                z[j, i] = solve_banded((1, 1), ab, r[j, i])
        ref.append(z)
    rows = owned_active_rows(m, su["active_vertex"])
    for sym in (1, 0):
        zu, zv = np.zeros(m.vshape3), np.zeros(m.vshape3)
        rc = emu.emu_sia_apply(m.nx, m.ny, m.nz, m.periodic, _p(av), *[_p(np.ascontiguousarray(a)) for a in A],
                               _p(ru), _p(rv), _p(zu), _p(zv), sym)
        assert rc == 0
        assert rel_l2([zu[rows], zv[rows]], [ref[0][rows], ref[1][rows]]) < 1e-12, sym


def test_singular_jacobian_is_reported_by_body_and_oracle():
    """The reference stops unless |detJ| > 0 (glissade_velo_higher.F90:
    6458-6473), which a NaN corner thickness fails (a geometrically flat
    element rarely gives detJ exactly 0 in floating point).  The device body
    (assembly pass 1) reports it, as the oracle does."""
    emu = C.CDLL(EMU)
    m = configs.slab(n=12)
    prep, u, v = solver.prepare(m)
    su = oracle.setup(m)
    j, i = 6, 6  # vertex (7, 7) in 1-based indices, a corner of four active cells
    for a in (prep.arrays["stagthck"], su["stagthck"]):
        a[j, i] = np.nan
    assert prep.arrays["active_vertex"][j, i] == 1
    shp = (m.ny - 1, m.nx - 1, m.nz, 27)
    E = [np.zeros(shp) for _ in range(4)]
    ebu, ebv = np.zeros(m.vshape3), np.zeros(m.vshape3)
    eef = np.zeros((m.ny, m.nx, m.nz - 1))
    rc = emu.emu_assemble(C.byref(prep.inputs), _p(u), _p(v), *[_p(a) for a in E], _p(ebu), _p(ebv), _p(eef))
    assert rc == 2
    with pytest.raises(RuntimeError, match="failed: 2"):
        oracle.assemble_system(m, su, u, v)


@pytest.mark.parametrize("opt", [dict(which_gradient=3), dict(which_ground=1), dict(which_gradient_margin=3),
                                 dict(which_assemble_taud=2), dict(which_babc=1), dict(which_babc=9)])
def test_setup_rejects_options_it_does_not_restate(opt):
    """The grounding-line parameterisation (which the reference does not
    support either, glissade_grounding_line.F90:73), calcbeta options the
    mirror does not evaluate (BPMP; a velocity-dependent law without its
    parameters) and unknown option values are refused by the host mirror
    instead of computing something else."""
    with pytest.raises(solver.BPError) as e:
        solver.prepare(configs.slab(n=12).copy(**opt))
    assert e.value.code == 10


@pytest.mark.parametrize("field,value", [("which_efvs", 3), ("which_resid", 5), ("pcg_variant", 4),
                                         ("which_precond", 3), ("precision", 2), ("maxiter_nonlinear", 0)])
def test_plan_rejects_out_of_range_options(field, value):
    """The host plan refuses option values the device does not implement
    (the library returns BP_ERR_ARGS before any device work)."""
    emu = C.CDLL(EMU)
    m = configs.slab(n=12)
    prep, u, v = solver.prepare(m)
    setattr(prep.inputs, field, value)
    out = np.zeros((m.ny - 1, m.nx - 1))
    assert emu.emu_slide_beta(C.byref(prep.inputs), _p(u), _p(v), _p(out)) == 10


def test_upstream_gradient_takes_the_higher_edge():
    """First-order upstream: each vertex takes the edge gradient of the
    higher pair of cells; on a plane tilted in x that is the plane's slope
    at every vertex."""
    m = configs.slab(n=16, theta_deg=0.5).copy(which_gradient=1, max_slope=1.0)
    su = oracle.setup(m)
    js, is_ = m.owned_vertex_slices()
    slope = -np.tan(np.radians(0.5))
    assert np.allclose(su["dusrf_dx"][js, is_], slope, rtol=1e-12)
    assert np.all(su["dusrf_dy"][js, is_] == 0.0)


def _c_struct_fields(hdr, name):
    """Field names, in order, of the typedef struct `name` in the header."""
    end = re.search(r"\}\s*" + name + r";", hdr).start()
    body = hdr[hdr.rindex("typedef struct {", 0, end) + len("typedef struct {"):end]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        decl = re.sub(r"^(const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*", "", decl)  # drop the type
        for part in decl.split(","):
            names.append(part.strip().lstrip("*").strip())
    return names


@pytest.mark.parametrize("cname,pystruct", [("bp_inputs", solver.Inputs), ("bp_stats", solver.Stats),
                                            ("bp_model", solver.Model), ("bp_setup_arrays", solver.SetupArrays),
                                            ("bp_sliding", solver.Sliding), ("bp_l1l2", solver.L1L2),
                                            ("bp_diva", solver.Diva)])
def test_ctypes_structs_follow_the_header(cname, pystruct):
    """The Python binding's structs list the C ABI structs' fields in the
    header's order (a drift would shift every later field)."""
    hdr = open(os.path.join(ROOT, "include", "bp_b200.h")).read()
    assert _c_struct_fields(hdr, cname) == [n for n, _ in pystruct._fields_]
    # and the same size as the C compiler lays it out (a field of the wrong
    # type would shift the ones after it)
    emu = C.CDLL(os.path.join(ROOT, "tests", "hostemu", "libhostemu.so"))
    emu.emu_sizeof.restype = C.c_long
    emu.emu_sizeof.argtypes = [C.c_char_p]
    assert emu.emu_sizeof(cname.encode()) == C.sizeof(pystruct)
