"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and rejects bad arguments on the host before any launch."""
import ctypes
import os
import re


import similie_b200 as sil
from similie_b200 import _native

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "sil_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sil_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_functions():
    names = declared_functions()
    assert "sil_deriv" in names and "sil_laplacian_run" in names and "sil_mag2d_solve_batch" in names


def test_every_declared_symbol_is_exported():
    L = ctypes.CDLL(_native.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    bound = {name for name, _, _ in _native.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_status_strings():
    L = sil.lib()
    for code, name in _native.STATUS_NAMES.items():
        assert L.sil_status_string(code).decode() == name


def test_null_arguments_rejected_on_host():
    L = sil.lib()
    assert L.sil_deriv(None, 1, 0, None, None) == 1
    assert b"NULL" in L.sil_last_error()
    f = _native.SilField()
    f.ndims = 0
    assert L.sil_deriv(None, 1, 0, ctypes.byref(f), ctypes.byref(f)) == 1
    assert L.sil_laplacian_run(None, None, None, None) == 1
    assert L.sil_mag2d_solve_batch(None, 0, None, None, None) == 1
    assert L.sil_geometry_create(None, 2, None, None, None) == 1


def test_mag3d_arguments_checked_on_host():
    import numpy as np
    L = sil.lib()
    x = np.linspace(0.0, 1.0, 4)
    p = _native.SilMag3dProblem()
    p.nx = p.ny = p.nz = 4
    p.x = p.y = p.z = x.ctypes.data
    p.node_mu = p.rhs = p.solution = 256  # never dereferenced: the checks fail first
    p.gauge_penalty = 0.0
    assert L.sil_mag3d_apply(None, ctypes.byref(p), 256, 256) == 1
    assert b"gauge_penalty" in L.sil_last_error()
    p.gauge_penalty = 20.0
    p.nz = 2
    assert L.sil_mag3d_apply(None, ctypes.byref(p), 256, 256) == 1
    assert b"3x3x3" in L.sil_last_error()
    p.nz = 4
    bad = np.array([0.0, 0.5, 0.5, 1.0])
    p.y = bad.ctypes.data
    st = _native.SilSolveSettings()
    diag = (_native.SilSolveDiagnostics * 1)()
    assert L.sil_mag3d_solve_batch(ctypes.byref(p), 1, ctypes.byref(st), diag, None) == 1
    assert b"increase" in L.sil_last_error()
    assert L.sil_mag3d_apply(None, None, None, None) == 1
    assert L.sil_mag3d_solve_batch(None, 0, None, None, None) == 1


def test_gauge_and_nonlinear_arguments_checked_on_host():
    import numpy as np
    L = sil.lib()
    # 3D gauge kind and sign rules
    x = np.linspace(0.0, 1.0, 4)
    p = _native.SilMag3dProblem()
    p.nx = p.ny = p.nz = 4
    p.x = p.y = p.z = x.ctypes.data
    p.node_mu = p.rhs = p.solution = 256
    p.gauge_penalty = 20.0
    p.gauge = 2
    assert L.sil_mag3d_apply(None, ctypes.byref(p), 256, 256) == 1
    assert b"gauge must be 0 or 1" in L.sil_last_error()
    p.gauge = 0
    p.gauge_penalty = -20.0                # a negative penalty: only the divergence gauge takes a sign
    assert L.sil_mag3d_apply(None, ctypes.byref(p), 256, 256) == 1
    p.gauge = 1
    p.gauge_penalty = 0.0
    assert L.sil_mag3d_apply(None, ctypes.byref(p), 256, 256) == 1
    assert b"nonzero" in L.sil_last_error()
    # nonlinear problem: geometry, material arrays and the B-H curve are checked before any launch
    b = np.array([0.0, 1.0, 2.0])
    h = np.array([0.0, 1.0, 3.0])
    q = _native.SilMag2dNlProblem()
    q.nx, q.ny = 2, 8
    q.node_mu = q.node_ferro = 256
    q.curve = _native.SilBHCurve(3, b.ctypes.data, h.ctypes.data)
    assert L.sil_mag2d_nl_apply(None, ctypes.byref(q), 256, 256) == 1
    assert b"3x3" in L.sil_last_error()
    q.nx = 8
    q.node_ferro = None
    assert L.sil_mag2d_nl_apply(None, ctypes.byref(q), 256, 256) == 1
    assert b"NULL" in L.sil_last_error()
    q.node_ferro = 256
    bad = np.array([0.0, 1.0, 1.0])
    q.curve = _native.SilBHCurve(3, bad.ctypes.data, h.ctypes.data)
    assert L.sil_mag2d_nl_apply_jacobian(None, ctypes.byref(q), 256, 256, 256) == 1
    assert b"increase" in L.sil_last_error()
    q.curve = _native.SilBHCurve(65, b.ctypes.data, h.ctypes.data)
    assert L.sil_mag2d_nl_apply(None, ctypes.byref(q), 256, 256) == 1
    assert b"64" in L.sil_last_error()
    neg = np.array([-1.0, 1.0, 2.0])
    q.curve = _native.SilBHCurve(3, neg.ctypes.data, h.ctypes.data)
    assert L.sil_mag2d_nl_apply(None, ctypes.byref(q), 256, 256) == 1
    q.curve = _native.SilBHCurve(3, b.ctypes.data, h.ctypes.data)
    st = _native.SilSolveSettings()
    diag = (_native.SilSolveDiagnostics * 1)()
    q.rhs = None
    assert L.sil_mag2d_nl_solve_batch(ctypes.byref(q), 1, ctypes.byref(st), diag, None) == 1
    assert b"NULL" in L.sil_last_error()
    assert L.sil_mag2d_nl_solve_batch(None, 0, None, None, None) == 1
    # 3D nonlinear problem: grid, coordinates, gauge penalty, material arrays, curve, fields
    r = _native.SilMag3dNlProblem()
    r.nx, r.ny, r.nz = 4, 4, 2
    r.x = r.y = r.z = x.ctypes.data
    r.node_mu = r.node_ferro = 256
    r.curve = _native.SilBHCurve(3, b.ctypes.data, h.ctypes.data)
    r.gauge_penalty = 20.0
    assert L.sil_mag3d_nl_apply(None, ctypes.byref(r), 256, 256) == 1
    assert b"3x3x3" in L.sil_last_error()
    r.nz = 4
    r.gauge_penalty = 0.0
    assert L.sil_mag3d_nl_apply(None, ctypes.byref(r), 256, 256) == 1
    assert b"gauge_penalty" in L.sil_last_error()
    r.gauge_penalty = 20.0
    down = np.array([0.0, 0.5, 0.4, 1.0])
    r.z = down.ctypes.data
    assert L.sil_mag3d_nl_apply_jacobian(None, ctypes.byref(r), 256, 256, 256) == 1
    assert b"increase strictly" in L.sil_last_error()
    r.z = x.ctypes.data
    r.node_ferro = None
    assert L.sil_mag3d_nl_apply(None, ctypes.byref(r), 256, 256) == 1
    assert b"NULL material" in L.sil_last_error()
    r.node_ferro = 256
    r.curve = _native.SilBHCurve(3, bad.ctypes.data, h.ctypes.data)
    assert L.sil_mag3d_nl_apply(None, ctypes.byref(r), 256, 256) == 1
    assert b"increase" in L.sil_last_error()
    r.curve = _native.SilBHCurve(3, b.ctypes.data, h.ctypes.data)
    r.rhs = None
    assert L.sil_mag3d_nl_solve_batch(ctypes.byref(r), 1, ctypes.byref(st), diag, None) == 1
    assert b"NULL field" in L.sil_last_error()
    assert L.sil_mag3d_nl_solve_batch(None, 0, None, None, None) == 1


def test_assembled_path_arguments_checked_on_host():
    L = sil.lib()
    h = ctypes.c_void_p()
    assert L.sil_mag2d_assemble(None, 8, 8, None, ctypes.byref(h)) == 1
    assert L.sil_mag2d_assemble(None, 2, 8, 256, ctypes.byref(h)) == 1
    assert b"3x3" in L.sil_last_error()
    p = _native.SilMag3dProblem()
    p.nx, p.ny, p.nz = 4, 4, 2
    assert L.sil_mag3d_assemble(None, ctypes.byref(p), ctypes.byref(h)) == 1
    assert b"3x3x3" in L.sil_last_error()
    assert L.sil_csr_get(None, None, None, None, None, None) == 1
    assert L.sil_csr_spmv(None, None, 256, 256) == 1
    assert L.sil_csr_copy(None, None, 256, 256, 256) == 1
    cfg = _native.SilMenuSettings()
    assert L.sil_csr_precond_create(None, None, ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert L.sil_csr_precond_apply(None, None, 256, 256) == 1
    st = _native.SilSolveSettings()
    d = _native.SilSolveDiagnostics()
    assert L.sil_csr_solve(None, None, None, 256, 256, ctypes.byref(st), ctypes.byref(d)) == 1
    assert L.sil_csr_krylov_solve(None, None, None, 3, 0, 256, 256, ctypes.byref(st), ctypes.byref(d)) == 1
    q = _native.SilMag2dNlProblem()
    q.nx, q.ny = 2, 8
    assert L.sil_mag2d_nl_assemble_jacobian(None, ctypes.byref(q), 256, ctypes.byref(h)) == 1
    assert b"3x3" in L.sil_last_error()
    assert L.sil_mag2d_nl_assemble_jacobian(None, ctypes.byref(q), None, ctypes.byref(h)) == 1
    r = _native.SilMag3dNlProblem()
    r.nx, r.ny, r.nz = 4, 2, 4
    assert L.sil_mag3d_nl_assemble_jacobian(None, ctypes.byref(r), 256, ctypes.byref(h)) == 1
    assert b"3x3x3" in L.sil_last_error()
    L.sil_csr_destroy(None)
    L.sil_csr_precond_destroy(None)
    import similie_b200.assembled as asm
    assert asm.kind_of("SSOR") == 4 and asm.kind_of("isai") == 7 and asm.kind_of("spd_isai") == 2


def test_rank_and_component_checks_on_host():
    L = sil.lib()
    fi = _native.SilField()
    fi.data = 16
    fi.dtype = _native.SIL_F64
    fi.ndims = 2
    fi.ncomp = 3  # wrong: a 2D 1-form has 2 components
    for d in range(2):
        fi.extent[d] = 4
        fi.stride[d] = 1
    fo = _native.SilField.from_buffer_copy(fi)
    fo.ncomp = 1
    assert L.sil_deriv(None, 3, 1, ctypes.byref(fi), ctypes.byref(fo)) == 1
    assert b"components" in L.sil_last_error()
    fi.ncomp = 2
    # d of a top-rank form is rejected
    fo.ncomp = 1
    fi2 = _native.SilField.from_buffer_copy(fi)
    fi2.ncomp = 1
    assert L.sil_deriv(None, 3, 2, ctypes.byref(fi2), ctypes.byref(fo)) == 1
    # four form dims are fine for d, the Hodge-star operators stop at three
    assert L.sil_laplacian(None, None, 3, 0, ctypes.byref(fi2), ctypes.byref(fi2)) == 1


def test_field_struct_layout_matches_header():
    # data, dtype, ndims, ncomp, reserved, front[6], extent[6], stride[6], comp_stride
    assert ctypes.sizeof(_native.SilField) == 8 + 4 * 4 + 3 * 6 * 8 + 8
