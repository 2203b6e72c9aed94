"""ctypes wrapper of the plain-C oracle (oracle/_build/libcfdx_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker used by tests/, __graft_entry__.smoke()
and the CPU legs of bench.py.  The product (cfdx_dev_b200) never imports it.
The library is the C restatement in cfdx_oracle.c (reference citations in
cfdx_oracle.h); it needs no reference tree and is built with
``make -C oracle oracle`` (gcc only), or on first use by :func:`lib`.

The functions mirror ``oracle.ref`` (the reference compiled from its own
sources) so the two can be compared call for call.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libcfdx_oracle.so"

_c_i64p = C.POINTER(C.c_int64)
_c_i32p = C.POINTER(C.c_int32)
_c_f64p = C.POINTER(C.c_double)


class CoMesh(C.Structure):
    _fields_ = [
        ("n_points", C.c_int64), ("n_faces", C.c_int64), ("n_cells", C.c_int64),
        ("px", _c_f64p), ("py", _c_f64p), ("pz", _c_f64p),
        ("face_offsets", _c_i64p), ("face_vertices", _c_i64p),
        ("owner", _c_i64p), ("neighbour", _c_i64p),
        ("cell_offsets", _c_i64p), ("cell_faces", _c_i64p),
        ("n_patches", C.c_int32), ("patch_of_face", _c_i32p), ("patch_types", _c_i32p),
    ]


class CoReport(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int64), ("residual", C.c_double),
                ("residual_relative", C.c_double), ("residual_replacements", C.c_int64),
                ("preconditioner_applications", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class CoHierarchy(C.Structure):
    _fields_ = [("n_levels", C.c_int32), ("n_rows", _c_i64p),
                ("row_offsets", C.POINTER(_c_i64p)), ("columns", C.POINTER(_c_i64p)),
                ("values", C.POINTER(_c_f64p)), ("inv_diag", C.POINTER(_c_f64p)),
                ("p_offsets", C.POINTER(_c_i64p)), ("p_columns", C.POINTER(_c_i64p)),
                ("p_values", C.POINTER(_c_f64p)), ("omega", C.c_double),
                ("pre_sweeps", C.c_int32), ("post_sweeps", C.c_int32),
                ("constant_null_space", C.c_int32)]


_lib = None
_lock = threading.Lock()


def available() -> bool:
    return LIB_PATH.exists() or (HERE / "cfdx_oracle.c").exists()


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
            L = C.CDLL(str(LIB_PATH))
            L.co_last_error.restype = C.c_char_p
            L.co_fv_geometry.argtypes = [C.c_void_p] * 5
            L.co_gauss_gradient.argtypes = [C.c_void_p] * 5
            L.co_pressure_assemble.restype = C.c_int64
            L.co_pressure_assemble.argtypes = [C.c_void_p] * 4 + [C.c_double] + [C.c_void_p] * 8
            L.co_rhie_chow_flux.argtypes = [C.c_void_p] * 4 + [C.c_double] + [C.c_void_p] * 3
            L.co_build_hbya.argtypes = [C.c_int64] + [C.c_void_p] * 9
            L.co_assemble_diffusion.restype = C.c_int64
            L.co_assemble_diffusion.argtypes = [C.c_void_p] * 3 + [C.c_double] + [C.c_void_p] * 5
            L.co_spmv.argtypes = [C.c_int64] + [C.c_void_p] * 5
            L.co_vcycle.argtypes = [C.c_void_p] * 3
            L.co_solve_gmres.argtypes = [C.c_int64] + [C.c_void_p] * 6 + [C.c_int32, C.c_int64, C.c_double,
                                                                          C.c_void_p]
            L.co_solve_cg.argtypes = [C.c_int64] + [C.c_void_p] * 3 + [C.c_int32] + [C.c_void_p] * 3 + [
                C.c_int64, C.c_double, C.c_void_p]
            L.co_solve_cg_ns.argtypes = [C.c_int64] + [C.c_void_p] * 3 + [C.c_int32] + [C.c_void_p] * 3 + [
                C.c_int64, C.c_double, C.c_int32, C.c_void_p]
            L.co_solve_projected_gmres.argtypes = [C.c_int64] + [C.c_void_p] * 6 + [C.c_int32, C.c_int64,
                                                                                    C.c_double, C.c_void_p]
            L.co_null_space_entry.restype = C.c_double
            L.co_null_space_entry.argtypes = [C.c_int64]
            L.co_null_space_checks.argtypes = [C.c_int64] + [C.c_void_p] * 5
            _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc, what):
    if rc < 0:
        raise RuntimeError(f"oracle {what} failed: {lib().co_last_error().decode()}")
    return rc


class _MeshHolder:
    def __init__(self, m):
        self.m = m
        s = self.s = CoMesh()
        s.n_points, s.n_faces, s.n_cells = m.px.size, m.owner.size, m.cell_offsets.size - 1
        for k in ("px", "py", "pz"):
            setattr(s, k, getattr(m, k).ctypes.data_as(_c_f64p))
        for k in ("face_offsets", "face_vertices", "owner", "neighbour", "cell_offsets", "cell_faces"):
            setattr(s, k, getattr(m, k).ctypes.data_as(_c_i64p))
        s.n_patches = m.patch_types.size
        s.patch_of_face = m.patch_of_face.ctypes.data_as(_c_i32p)
        s.patch_types = m.patch_types.ctypes.data_as(_c_i32p)

    @property
    def ptr(self):
        return C.byref(self.s)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def geometry(mesh) -> dict:
    h = _MeshHolder(mesh)
    nf, nc = mesh.owner.size, mesh.cell_offsets.size - 1
    out = dict(face_centres=np.empty(3 * nf), face_Sf=np.empty(3 * nf), cell_centres=np.empty(3 * nc),
               cell_volumes=np.empty(nc))
    _check(lib().co_fv_geometry(h.ptr, *(_p(out[k]) for k in ("face_centres", "face_Sf", "cell_centres",
                                                              "cell_volumes"))), "geometry")
    return out


def gauss_gradient(mesh, p, fixed, value):
    h = _MeshHolder(mesh)
    g = np.empty(3 * (mesh.cell_offsets.size - 1))
    pp, fx, va = _f64(p), np.ascontiguousarray(fixed, np.int32), _f64(value)
    _check(lib().co_gauss_gradient(h.ptr, _p(pp), _p(fx), _p(va), _p(g)), "gauss_gradient")
    return g


def simple_assemble(mesh, HbyA, rAU, p, rho, fixed, value):
    h = _MeshHolder(mesh)
    nc, nf = mesh.cell_offsets.size - 1, mesh.owner.size
    ro = np.empty(nc + 1, np.int64)
    co = np.empty(nc + 2 * nf, np.int64)
    va = np.empty(nc + 2 * nf)
    b, phi, grad = np.empty(nc), np.empty(nf), np.empty(3 * nc)
    U, R, P = _f64(HbyA), _f64(rAU), _f64(p)
    fx, vv = np.ascontiguousarray(fixed, np.int32), _f64(value)
    nnz = _check(lib().co_pressure_assemble(h.ptr, _p(U), _p(R), _p(P), float(rho), _p(fx), _p(vv), _p(phi),
                                            _p(grad), _p(ro), _p(co), _p(va), _p(b)), "pressure assembly")
    return dict(row_offsets=ro, columns=co[:nnz].copy(), values=va[:nnz].copy(), b=b, phiHbyA=phi, grad_p=grad)


def rhie_chow_flux(mesh, HbyA, rAU, p, rho, fixed, value):
    h = _MeshHolder(mesh)
    flux = np.empty(mesh.owner.size)
    U, R, P = _f64(HbyA), _f64(rAU), _f64(p)
    fx, vv = np.ascontiguousarray(fixed, np.int32), _f64(value)
    _check(lib().co_rhie_chow_flux(h.ptr, _p(U), _p(R), _p(P), float(rho), _p(fx), _p(vv), _p(flux)),
           "rhie_chow_flux")
    return flux


def assemble_diffusion(mesh, bc_values, diffusivity, source, bc_types=None):
    h = _MeshHolder(mesh)
    nc, nf = mesh.cell_offsets.size - 1, mesh.owner.size
    ro = np.empty(nc + 1, np.int64)
    co = np.empty(nc + 2 * nf, np.int64)
    va = np.empty(nc + 2 * nf)
    rhs = np.empty(nc)
    bc, src = _f64(bc_values), _f64(source)
    bt = None if bc_types is None else np.ascontiguousarray(bc_types, np.int32)
    nnz = _check(lib().co_assemble_diffusion(h.ptr, _p(bc), _p(bt), float(diffusivity), _p(src), _p(ro), _p(co),
                                             _p(va), _p(rhs)), "assemble_diffusion")
    return ro, co[:nnz].copy(), va[:nnz].copy(), rhs


def spmv(ro, co, va, x):
    ro, co, va, x = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64), _f64(va), _f64(x))
    y = np.empty(ro.size - 1)
    lib().co_spmv(ro.size - 1, _p(ro), _p(co), _p(va), _p(x), _p(y))
    return y


class Hierarchy:
    """An AMG hierarchy (list of level dicts: row_offsets, columns, values,
    inv_diag and, on all but the last level, p_offsets, p_columns, p_values)
    with the reference's V(pre, post) damped-Jacobi cycle."""

    def __init__(self, levels, omega, pre_sweeps=6, post_sweeps=6, constant_null_space=False):
        L = len(levels)
        self.levels = [{k: (None if v is None else np.ascontiguousarray(v)) for k, v in lv.items()} for lv in levels]
        lv = self.levels

        def arr(t, key):
            ptrs = []
            for l in range(L):
                v = lv[l].get(key)
                if v is None or (key.startswith("p_") and l + 1 == L):
                    ptrs.append(t())
                else:
                    ptrs.append(v.ctypes.data_as(t))
            return (t * L)(*ptrs)

        self.n_rows = np.array([x["inv_diag"].size for x in lv], np.int64)
        h = self.h = CoHierarchy()
        h.n_levels = L
        h.n_rows = self.n_rows.ctypes.data_as(_c_i64p)
        self._arrays = [arr(_c_i64p, "row_offsets"), arr(_c_i64p, "columns"), arr(_c_f64p, "values"),
                        arr(_c_f64p, "inv_diag"), arr(_c_i64p, "p_offsets"), arr(_c_i64p, "p_columns"),
                        arr(_c_f64p, "p_values")]
        (h.row_offsets, h.columns, h.values, h.inv_diag, h.p_offsets, h.p_columns, h.p_values) = self._arrays
        h.omega = float(omega)
        h.pre_sweeps, h.post_sweeps = int(pre_sweeps), int(post_sweeps)
        h.constant_null_space = int(bool(constant_null_space))

    @property
    def ptr(self):
        return C.byref(self.h)

    def apply(self, r):
        r = _f64(r)
        z = np.empty_like(r)
        _check(lib().co_vcycle(self.ptr, _p(r), _p(z)), "V-cycle")
        return z


def solve_gmres(ro, co, va, b, hierarchy=None, x0=None, restart=30, max_iterations=1000, tolerance=1e-8):
    ro, co, va, b = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64), _f64(va), _f64(b))
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    rep = CoReport()
    _check(lib().co_solve_gmres(b.size, _p(ro), _p(co), _p(va), hierarchy.ptr if hierarchy else None, _p(b), _p(x),
                                int(restart), int(max_iterations), float(tolerance), C.byref(rep)), "GMRES")
    return x, rep.as_dict()


CG_PRECONDITIONERS = {"internal_jacobi": 0, "none": 1, "jacobi": 2, "native_amg": 6}


def solve_cg(ro, co, va, b, preconditioner="native_amg", hierarchy=None, x0=None, max_iterations=1000,
             tolerance=1e-8, null_space=False):
    """co_solve_cg_ns: the reference's CG (cg_solver.h:45-560) with the solver's
    own diagonal ("internal_jacobi") or the dispatch's identity / Jacobi /
    native-AMG preconditioner object (the AMG one applies ``hierarchy``);
    null_space: the constant NullSpaceProjector of the solve."""
    ro, co, va, b = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64), _f64(va), _f64(b))
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    rep = CoReport()
    _check(lib().co_solve_cg_ns(b.size, _p(ro), _p(co), _p(va), CG_PRECONDITIONERS[preconditioner],
                                hierarchy.ptr if hierarchy else None, _p(b), _p(x), int(max_iterations),
                                float(tolerance), int(bool(null_space)), C.byref(rep)), "CG")
    return x, rep.as_dict()


def solve_projected_gmres(ro, co, va, b, hierarchy=None, x0=None, restart=30, max_iterations=1000,
                          tolerance=1e-8):
    """co_solve_projected_gmres: solve_projected_gmres (projected_gmres.h:84-150),
    FGMRES on P A P preconditioned by P M P; status 3 with x unchanged when the
    right-hand side or the operator does not fit the constant null space."""
    ro, co, va, b = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64), _f64(va), _f64(b))
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    rep = CoReport()
    _check(lib().co_solve_projected_gmres(b.size, _p(ro), _p(co), _p(va), hierarchy.ptr if hierarchy else None,
                                          _p(b), _p(x), int(restart), int(max_iterations), float(tolerance),
                                          C.byref(rep)), "projected GMRES")
    return x, rep.as_dict()


def null_space_entry(n):
    """Every entry of NullSpaceProjector::constant(n)'s normalised basis vector."""
    return lib().co_null_space_entry(int(n))


def null_space_checks(ro, co, va, b):
    """(is_compatible(b), is_null_space(A), is_bilateral_null_space(A)) of the constant null space."""
    ro, co, va, b = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64), _f64(va), _f64(b))
    out = np.zeros(3, np.int32)
    _check(lib().co_null_space_checks(b.size, _p(ro), _p(co), _p(va), _p(b), _p(out)), "null-space checks")
    return tuple(bool(v) for v in out)


def gauge_eliminate(ro, co, va, b, ref):
    """co_gauge_eliminate: (row_offsets, columns, values, b) of the system without cell ref."""
    ro, co, va, b = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64), _f64(va), _f64(b))
    n = b.size
    f = lib().co_gauge_eliminate
    f.restype = C.c_int64
    f.argtypes = [C.c_int64] + [C.c_void_p] * 4 + [C.c_int64] + [C.c_void_p] * 4
    ro_o, co_o, va_o, b_o = np.empty(n, np.int64), np.empty(co.size, np.int64), np.empty(va.size), np.empty(n - 1)
    nnz = _check(f(n, _p(ro), _p(co), _p(va), _p(b), int(ref), _p(ro_o), _p(co_o), _p(va_o), _p(b_o)), "gauge")
    return ro_o, co_o[:nnz].copy(), va_o[:nnz].copy(), b_o


def gauge_expand(x_reduced, ref):
    xr = _f64(x_reduced)
    x = np.empty(xr.size + 1)
    f = lib().co_gauge_expand
    f.argtypes = [C.c_int64, C.c_void_p, C.c_int64, C.c_void_p]
    f(x.size, _p(xr), int(ref), _p(x))
    return x


def gauge_identity_row(ro, co, va, b, ref, value=0.0):
    """co_gauge_identity_row: apply_reference_cell_gauge (scalar_diffusion.h:177-210)."""
    ro, co, va, b = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64), _f64(va), _f64(b))
    n = b.size
    f = lib().co_gauge_identity_row
    f.restype = C.c_int64
    f.argtypes = [C.c_int64] + [C.c_void_p] * 4 + [C.c_int64, C.c_double] + [C.c_void_p] * 4
    ro_o, co_o, va_o, b_o = (np.empty(n + 1, np.int64), np.empty(co.size + 1, np.int64), np.empty(va.size + 1),
                             np.empty(n))
    nnz = _check(f(n, _p(ro), _p(co), _p(va), _p(b), int(ref), float(value), _p(ro_o), _p(co_o), _p(va_o),
                   _p(b_o)), "gauge")
    return ro_o, co_o[:nnz].copy(), va_o[:nnz].copy(), b_o


def build_hbya(row_offsets, columns, values3, rhs, U, gradp, volumes, rAU):
    """physics/steady_incompressible_solver.h:6430-6465 (build_hbya): values3 is
    the three components' momentum values (3 x nnz, one pattern)."""
    ro = np.ascontiguousarray(row_offsets, np.int64)
    co = np.ascontiguousarray(columns, np.int64)
    n = ro.size - 1
    va = np.ascontiguousarray(values3, np.float64).reshape(-1)
    out = np.empty(3 * n)
    args = [_f64(a) for a in (rhs, U, gradp, volumes, rAU)]
    _check(lib().co_build_hbya(n, _p(ro), _p(co), _p(va), *(_p(a) for a in args), _p(out)), "build_hbya")
    return out
