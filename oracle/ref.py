"""ctypes wrapper of the reference-built oracle (oracle/_ref/libcfdx_ref.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker / reference timing.  The product
(cfdx_dev_b200) never imports it.  Build it with ``make -C oracle ref`` (needs
the reference source tree); the built .so then works without that tree.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libcfdx_ref.so"

_c_i64p = C.POINTER(C.c_int64)
_c_i32p = C.POINTER(C.c_int32)
_c_f64p = C.POINTER(C.c_double)


class RefMesh(C.Structure):
    _fields_ = [
        ("n_points", C.c_int64), ("n_faces", C.c_int64), ("n_cells", C.c_int64),
        ("px", _c_f64p), ("py", _c_f64p), ("pz", _c_f64p),
        ("face_offsets", _c_i64p), ("face_vertices", _c_i64p),
        ("owner", _c_i64p), ("neighbour", _c_i64p),
        ("cell_offsets", _c_i64p), ("cell_faces", _c_i64p),
        ("n_patches", C.c_int32), ("patch_of_face", _c_i32p), ("patch_types", _c_i32p),
    ]


class RefReport(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int64), ("residual", C.c_double),
                ("residual_relative", C.c_double), ("physical_residual_relative", C.c_double),
                ("setup_seconds", C.c_double), ("solve_seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle ref`")
        _lib = C.CDLL(str(LIB_PATH))
        _lib.ref_last_error.restype = C.c_char_p
        _lib.ref_amg_create.restype = C.c_void_p
        _lib.ref_amg_create.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
        _lib.ref_amg_destroy.argtypes = [C.c_void_p]
        _lib.ref_amg_num_levels.argtypes = [C.c_void_p]
        _lib.ref_amg_omega.argtypes = [C.c_void_p]
        _lib.ref_amg_omega.restype = C.c_double
        _lib.ref_amg_level_sizes.argtypes = [C.c_void_p, C.c_int32, _c_i64p, _c_i64p, _c_i64p]
        _lib.ref_amg_level_matrix.argtypes = [C.c_void_p, C.c_int32] + [C.c_void_p] * 4
        _lib.ref_amg_level_prolongation.argtypes = [C.c_void_p, C.c_int32] + [C.c_void_p] * 4
        _lib.ref_amg_apply.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.ref_solve_gmres_prepared.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_double,
                                                  C.c_void_p]
        _lib.ref_solve_linear_system.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int64,
                                                 C.c_double, C.c_void_p]
        _lib.ref_assemble_diffusion.restype = C.c_int64
        _lib.ref_assemble_diffusion.argtypes = [C.c_void_p, C.c_void_p, C.c_double] + [C.c_void_p] * 6
        _lib.ref_simple_assemble.restype = C.c_int64
        _lib.ref_simple_assemble.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double] + \
            [C.c_void_p] * 9
        _lib.ref_rhie_chow_flux.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double] + \
            [C.c_void_p] * 3
        _lib.ref_gauss_gradient.argtypes = [C.c_void_p] * 5
        _lib.ref_fixture_tet_v52_sizes.argtypes = [C.c_int64, C.c_void_p]
        _lib.ref_fixture_tet_v52.argtypes = [C.c_int64] + [C.c_void_p] * 9
        _lib.ref_geometry_cache.argtypes = [C.c_void_p] * 5
        _lib.ref_fv_geometry.argtypes = [C.c_void_p] * 5
        _lib.ref_spmv.argtypes = [C.c_int64] + [C.c_void_p] * 5
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc, what):
    if rc < 0:
        raise RuntimeError(f"reference {what} failed: {lib().ref_last_error().decode()}")
    return rc


class _MeshHolder:
    def __init__(self, m):
        self.m = m  # keep arrays alive
        self.s = RefMesh()
        s = self.s
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


def fixture_tet_v52(n: int) -> dict:
    sizes = np.zeros(5, np.int64)
    _check(lib().ref_fixture_tet_v52_sizes(n, _p(sizes)), "tet fixture")
    npnt, nf, nfv, nc, ncf = (int(v) for v in sizes)
    out = dict(px=np.empty(npnt), py=np.empty(npnt), pz=np.empty(npnt), face_offsets=np.empty(nf + 1, np.int64),
               face_vertices=np.empty(nfv, np.int64), owner=np.empty(nf, np.int64),
               neighbour=np.empty(nf, np.int64), cell_offsets=np.empty(nc + 1, np.int64),
               cell_faces=np.empty(ncf, np.int64))
    _check(lib().ref_fixture_tet_v52(n, *(_p(out[k]) for k in (
        "px", "py", "pz", "face_offsets", "face_vertices", "owner", "neighbour", "cell_offsets", "cell_faces"))),
        "tet fixture")
    return out


def geometry(mesh, kind: str = "fv") -> dict:
    h = _MeshHolder(mesh)
    nf, nc = mesh.owner.size, mesh.cell_offsets.size - 1
    out = dict(face_centres=np.empty(3 * nf), face_Sf=np.empty(3 * nf), cell_centres=np.empty(3 * nc),
               cell_volumes=np.empty(nc))
    fn = lib().ref_fv_geometry if kind == "fv" else lib().ref_geometry_cache
    _check(fn(h.ptr, *(_p(out[k]) for k in ("face_centres", "face_Sf", "cell_centres", "cell_volumes"))), "geometry")
    return out


def assemble_diffusion(mesh, bc_values, diffusivity, source):
    h = _MeshHolder(mesh)
    nc, nf = mesh.cell_offsets.size - 1, mesh.owner.size
    ro = np.empty(nc + 1, np.int64)
    co = np.empty(nc + 2 * nf, np.int64)
    va = np.empty(nc + 2 * nf)
    rhs = np.empty(nc)
    sec = C.c_double()
    bc = np.ascontiguousarray(bc_values, dtype=np.float64)
    src = np.ascontiguousarray(source, dtype=np.float64)
    nnz = _check(lib().ref_assemble_diffusion(h.ptr, _p(bc), float(diffusivity), _p(src), _p(ro), _p(co), _p(va),
                                              _p(rhs), C.byref(sec)), "assemble_cell_diffusion_matrix")
    return ro, co[:nnz].copy(), va[:nnz].copy(), rhs, sec.value


def simple_assemble(mesh, HbyA, rAU, p, rho, p_bc_fixed, p_bc_value):
    h = _MeshHolder(mesh)
    nc, nf = mesh.cell_offsets.size - 1, mesh.owner.size
    ro = np.empty(nc + 1, np.int64)
    co = np.empty(nc + 2 * nf, np.int64)
    va = np.empty(nc + 2 * nf)
    b = np.empty(nc)
    phi = np.empty(nf)
    grad = np.empty(3 * nc)
    sec = C.c_double()
    args = [np.ascontiguousarray(a, dtype=np.float64) for a in (HbyA, rAU, p)]
    fixed = np.ascontiguousarray(p_bc_fixed, dtype=np.int32)
    value = np.ascontiguousarray(p_bc_value, dtype=np.float64)
    nnz = _check(lib().ref_simple_assemble(h.ptr, *(_p(a) for a in args), float(rho), _p(fixed), _p(value), _p(phi),
                                           _p(grad), _p(ro), _p(co), _p(va), _p(b), C.byref(sec)),
                 "pressure-corrector assembly")
    return dict(row_offsets=ro, columns=co[:nnz].copy(), values=va[:nnz].copy(), b=b, phiHbyA=phi, grad_p=grad,
                seconds=sec.value)


def rhie_chow_flux(mesh, HbyA, rAU, p, rho, p_bc_fixed, p_bc_value):
    h = _MeshHolder(mesh)
    flux = np.empty(mesh.owner.size)
    args = [np.ascontiguousarray(a, dtype=np.float64) for a in (HbyA, rAU, p)]
    fixed = np.ascontiguousarray(p_bc_fixed, dtype=np.int32)
    value = np.ascontiguousarray(p_bc_value, dtype=np.float64)
    _check(lib().ref_rhie_chow_flux(h.ptr, *(_p(a) for a in args), float(rho), _p(fixed), _p(value), _p(flux)),
           "make_rhie_chow_mass_flux")
    return flux


def gauss_gradient(mesh, p, p_bc_fixed, p_bc_value):
    h = _MeshHolder(mesh)
    g = np.empty(3 * (mesh.cell_offsets.size - 1))
    pp = np.ascontiguousarray(p, dtype=np.float64)
    fixed = np.ascontiguousarray(p_bc_fixed, dtype=np.int32)
    value = np.ascontiguousarray(p_bc_value, dtype=np.float64)
    _check(lib().ref_gauss_gradient(h.ptr, _p(pp), _p(fixed), _p(value), _p(g)), "gauss_gradient")
    return g


def spmv(ro, co, va, x):
    y = np.empty(ro.size - 1)
    _check(lib().ref_spmv(ro.size - 1, _p(ro), _p(co), _p(va), _p(np.ascontiguousarray(x, dtype=np.float64)), _p(y)),
           "spmv")
    return y


class Amg:
    """The reference's native Boomer-style AMG, Balanced policy."""

    def __init__(self, ro, co, va, require_smoother_certificate=False, constant_null_space=False):
        self.ro, self.co, self.va = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64),
                                     np.ascontiguousarray(va, np.float64))
        sec = C.c_double()
        f = lib().ref_amg_create_ns
        f.restype = C.c_void_p
        f.argtypes = [C.c_int64] + [C.c_void_p] * 3 + [C.c_int32, C.c_int32, C.c_void_p]
        self.h = f(self.ro.size - 1, _p(self.ro), _p(self.co), _p(self.va), int(require_smoother_certificate),
                   int(bool(constant_null_space)), C.byref(sec))
        if not self.h:
            raise RuntimeError(f"reference AMG setup failed: {lib().ref_last_error().decode()}")
        self.setup_seconds = sec.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_amg_destroy(self.h)
            self.h = None

    @property
    def omega(self):
        return lib().ref_amg_omega(self.h)

    def num_levels(self):
        return lib().ref_amg_num_levels(self.h)

    def level(self, l: int) -> dict:
        n, nnz, pn = C.c_int64(), C.c_int64(), C.c_int64()
        lib().ref_amg_level_sizes(self.h, l, C.byref(n), C.byref(nnz), C.byref(pn))
        n, nnz, pn = n.value, nnz.value, pn.value
        out = dict(row_offsets=np.empty(n + 1, np.int64), columns=np.empty(nnz, np.int64), values=np.empty(nnz),
                   inv_diag=np.empty(n))
        lib().ref_amg_level_matrix(self.h, l, _p(out["row_offsets"]), _p(out["columns"]), _p(out["values"]),
                                   _p(out["inv_diag"]))
        if pn:
            out.update(p_offsets=np.empty(n + 1, np.int64), p_columns=np.empty(pn, np.int64),
                       p_values=np.empty(pn), aggregate=np.empty(n, np.int64))
            lib().ref_amg_level_prolongation(self.h, l, _p(out["p_offsets"]), _p(out["p_columns"]),
                                             _p(out["p_values"]), _p(out["aggregate"]))
        else:
            out.update(p_offsets=None, p_columns=np.empty(0, np.int64), p_values=np.empty(0), aggregate=None)
        return out

    def update_values(self, ro, co, va) -> bool:
        ro, co, va = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64),
                      np.ascontiguousarray(va, np.float64))
        f = lib().ref_amg_update_values
        f.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        rc = _check(f(self.h, ro.size - 1, _p(ro), _p(co), _p(va)), "update_values")
        if rc == 0:
            self.ro, self.co, self.va = ro, co, va
        return rc == 0

    def apply(self, r):
        r = np.ascontiguousarray(r, np.float64)
        z = np.empty_like(r)
        rc = lib().ref_amg_apply(self.h, _p(r), _p(z))
        if rc != 0:
            raise RuntimeError("reference V-cycle failed")
        return z

    def solve_gmres(self, rhs, x0=None, restart=30, max_iterations=1000, tolerance=1e-8):
        b = np.ascontiguousarray(rhs, np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
        rep = RefReport()
        _check(lib().ref_solve_gmres_prepared(self.h, b.size, _p(self.ro), _p(self.co), _p(self.va), _p(b), _p(x),
                                              restart, max_iterations, tolerance, C.byref(rep)), "solve_gmres")
        return x, rep.as_dict()


class AmgFromLevels(Amg):
    """The reference's V-cycle/GMRES around a supplied hierarchy (list of level dicts with
    row_offsets, columns, values, inv_diag, p_offsets, p_columns, p_values) and damping."""

    def __init__(self, levels, omega, constant_null_space=False):
        L = len(levels)
        self._keep = levels
        self.ro, self.co, self.va = levels[0]["row_offsets"], levels[0]["columns"], levels[0]["values"]
        P64 = C.POINTER(C.c_int64)
        PD = C.POINTER(C.c_double)
        arr = lambda t, key: (t * L)(*[(levels[l][key].ctypes.data_as(t) if levels[l].get(key) is not None
                                        else t()) for l in range(L)])
        n_rows = np.array([lv["inv_diag"].size for lv in levels], np.int64)
        f = lib().ref_amg_create_from_levels
        f.restype = C.c_void_p
        f.argtypes = [C.c_int32, C.c_void_p] + [C.c_void_p] * 7 + [C.c_double]
        self._ptrs = [arr(P64, "row_offsets"), arr(P64, "columns"), arr(PD, "values"), arr(PD, "inv_diag"),
                      arr(P64, "p_offsets"), arr(P64, "p_columns"), arr(PD, "p_values")]
        self.h = f(L, n_rows.ctypes.data_as(C.c_void_p), *[C.cast(p, C.c_void_p) for p in self._ptrs], float(omega))
        if not self.h:
            raise RuntimeError(f"reference AMG from levels failed: {lib().ref_last_error().decode()}")
        self.setup_seconds = float("nan")
        g = lib().ref_amg_set_constant_null_space
        g.argtypes = [C.c_void_p, C.c_int32]
        g(self.h, int(bool(constant_null_space)))


class AmgFromTransfers(Amg):
    """The reference's setup() with each level's C/F interpolation read from a
    complete earlier run of that setup (``transfers``: p_offsets_l, p_columns_l,
    p_values_l, aggregate_l per level l, as ``Amg.level`` exports them) and
    every other step -- Galerkin products, diagonals, damping -- run by the
    reference's own code (ref_amg_create_from_transfers)."""

    def __init__(self, ro, co, va, transfers, level_rows):
        self.ro, self.co, self.va = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64),
                                     np.ascontiguousarray(va, np.float64))
        L = len(level_rows)
        self._keep = {k: np.ascontiguousarray(v, np.float64 if k.startswith("p_values") else np.int64)
                      for k, v in transfers.items()}
        P64 = C.POINTER(C.c_int64)
        PD = C.POINTER(C.c_double)

        def arr(t, key):
            return (t * max(1, L - 1))(*[self._keep[f"{key}_{l}"].ctypes.data_as(t) for l in range(L - 1)])

        self._ptrs = [arr(P64, "p_offsets"), arr(P64, "p_columns"), arr(PD, "p_values"), arr(P64, "aggregate")]
        rows = np.ascontiguousarray(level_rows, np.int64)
        f = lib().ref_amg_create_from_transfers
        f.restype = C.c_void_p
        f.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p] + [C.c_void_p] * 5
        sec = C.c_double()
        self.h = f(self.ro.size - 1, _p(self.ro), _p(self.co), _p(self.va), L, _p(rows),
                   *[C.cast(p, C.c_void_p) for p in self._ptrs], C.byref(sec))
        if not self.h:
            raise RuntimeError(f"reference AMG rebuild failed: {lib().ref_last_error().decode()}")
        self.setup_seconds = sec.value


def fingerprint_levels(levels) -> list[dict]:
    """Per level (dicts as ``Amg.level`` or the library's ``export_level`` give
    them), the SHA-256 of each array as int64 indices / FP64 values -- the
    fingerprint used to compare hierarchies too large to store."""
    import hashlib
    out = []
    for lv in levels:
        e = {"n_rows": int(lv["inv_diag"].size), "nnz": int(lv["columns"].size)}
        for k in ("row_offsets", "columns", "values", "inv_diag", "p_offsets", "p_columns", "p_values", "aggregate"):
            a = lv.get(k)
            if a is not None and (k not in ("p_columns", "p_values") or lv.get("p_offsets") is not None):
                a = np.ascontiguousarray(a, np.float64 if k in ("values", "inv_diag", "p_values") else np.int64)
                e[k] = hashlib.sha256(a.tobytes()).hexdigest()
        out.append(e)
    return out


def hierarchy_sha256(amg) -> list[dict]:
    """fingerprint_levels of a reference hierarchy, one level in memory at a time."""
    out = []
    for l in range(amg.num_levels()):
        out += fingerprint_levels([amg.level(l)])
    return out


def solve_linear_system(ro, co, va, rhs, x0=None, krylov=3, preconditioner=6, restart=30, max_iterations=1000,
                        tolerance=1e-8):
    ro, co, va = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64),
                  np.ascontiguousarray(va, np.float64))
    b = np.ascontiguousarray(rhs, np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    rep = RefReport()
    _check(lib().ref_solve_linear_system(b.size, _p(ro), _p(co), _p(va), _p(b), _p(x), krylov, preconditioner,
                                         restart, max_iterations, tolerance, C.byref(rep)), "solve_linear_system")
    return x, rep.as_dict()


def solve_linear_system_null_space(ro, co, va, rhs, x0=None, krylov=3, preconditioner=6, restart=30,
                                   max_iterations=1000, tolerance=1e-8, null_space=1):
    """solve_linear_system with LinearSolverRequest::null_space (1: NullSpaceModel::Constant)."""
    f = lib().ref_solve_linear_system_ns
    f.argtypes = [C.c_int64] + [C.c_void_p] * 5 + [C.c_int32] * 3 + [C.c_int64, C.c_double, C.c_int32, C.c_void_p]
    ro, co, va = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64),
                  np.ascontiguousarray(va, np.float64))
    b = np.ascontiguousarray(rhs, np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    rep = RefReport()
    _check(f(b.size, _p(ro), _p(co), _p(va), _p(b), _p(x), krylov, preconditioner, restart, max_iterations,
             tolerance, null_space, C.byref(rep)), "solve_linear_system (null space)")
    return x, rep.as_dict()


def write_capture(path, ro, co, va, rhs, guess, problem=1, null_space=0, scaling=0, max_iterations=1000,
                  tolerance=1e-8):
    """The reference's write_linear_system_capture (linear_system_capture.h:170)."""
    f = lib().ref_write_capture
    f.argtypes = [C.c_char_p, C.c_int64] + [C.c_void_p] * 5 + [C.c_int32] * 3 + [C.c_int64, C.c_double]
    ro, co = np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64)
    va, b, x = (np.ascontiguousarray(a, np.float64) for a in (va, rhs, guess))
    _check(f(str(path).encode(), b.size, _p(ro), _p(co), _p(va), _p(b), _p(x), problem, null_space, scaling,
             max_iterations, tolerance), "write_linear_system_capture")


def read_capture(path) -> dict:
    """The reference's read_linear_system_capture (linear_system_capture.h:233)."""
    f = lib().ref_read_capture
    f.argtypes = [C.c_char_p] + [C.c_void_p] * 7
    meta = np.zeros(6, np.int64)
    tol = C.c_double()
    _check(f(str(path).encode(), _p(meta), C.byref(tol), None, None, None, None, None),
           "read_linear_system_capture")
    n, nnz = int(meta[0]), int(meta[1])
    out = dict(row_offsets=np.empty(n + 1, np.int64), columns=np.empty(nnz, np.int64), values=np.empty(nnz),
               rhs=np.empty(n), initial_solution=np.empty(n))
    _check(f(str(path).encode(), _p(meta), C.byref(tol), *(_p(out[k]) for k in (
        "row_offsets", "columns", "values", "rhs", "initial_solution"))), "read_linear_system_capture")
    out.update(problem=int(meta[2]), null_space=int(meta[3]), scaling=int(meta[4]), max_iterations=int(meta[5]),
               tolerance=tol.value)
    return out


def solve_cg_internal(ro, co, va, rhs, x0=None, max_iterations=1000, tolerance=1e-8):
    """The reference's solve_cg without a preconditioner object (cg_solver.h:591)."""
    f = lib().ref_solve_cg_internal
    f.argtypes = [C.c_int64] + [C.c_void_p] * 5 + [C.c_int64, C.c_double, C.c_void_p]
    ro, co = np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64)
    va, b = np.ascontiguousarray(va, np.float64), np.ascontiguousarray(rhs, np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    rep = RefReport()
    _check(f(b.size, _p(ro), _p(co), _p(va), _p(b), _p(x), max_iterations, tolerance, C.byref(rep)), "solve_cg")
    return x, rep.as_dict()


def apply_reference_cell_gauge(ro, co, va, rhs, ref, value=0.0):
    """The reference's apply_reference_cell_gauge (scalar_diffusion.h:177-210)."""
    f = lib().ref_apply_reference_cell_gauge
    f.restype = C.c_int64
    f.argtypes = [C.c_int64] + [C.c_void_p] * 4 + [C.c_int64, C.c_double] + [C.c_void_p] * 4
    ro, co = np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64)
    va, b = np.ascontiguousarray(va, np.float64), np.ascontiguousarray(rhs, np.float64)
    n = b.size
    ro_o, co_o, va_o, b_o = (np.empty(n + 1, np.int64), np.empty(co.size + 1, np.int64), np.empty(va.size + 1),
                             np.empty(n))
    nnz = _check(f(n, _p(ro), _p(co), _p(va), _p(b), int(ref), float(value), _p(ro_o), _p(co_o), _p(va_o), _p(b_o)),
                 "apply_reference_cell_gauge")
    return ro_o, co_o[:nnz].copy(), va_o[:nnz].copy(), b_o


def solve_poisson_mixed(mesh, bc_values, source, bc_types=None, diffusivity=1.0, max_iterations=2000,
                        tolerance=1e-10, reference_cell=0, reference_value=0.0):
    """The reference's solve_poisson_mixed (scalar_diffusion.h:294-340) -> (x, report)."""
    f = lib().ref_solve_poisson_mixed
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_int64, C.c_double, C.c_int64,
                  C.c_double, C.c_void_p, C.c_void_p]
    h = _MeshHolder(mesh)
    nc = mesh.cell_offsets.size - 1
    bc = np.ascontiguousarray(bc_values, np.float64)
    ty = None if bc_types is None else np.ascontiguousarray(bc_types, np.int32)
    src = np.ascontiguousarray(source, np.float64)
    x = np.empty(nc)
    rep = RefReport()
    _check(f(h.ptr, _p(bc), _p(ty), float(diffusivity), _p(src), int(max_iterations), float(tolerance),
             int(reference_cell), float(reference_value), _p(x), C.byref(rep)), "solve_poisson_mixed")
    return x, rep.as_dict()


_FLAG_NAMES = ("square", "numerically_symmetric", "diagonally_dominant", "strongly_scaled",
               "large_diagonal_dynamic_range", "strongly_directional_coupling", "positive_diagonal", "saddle_point")


def measure_characteristics(ro, co, va, saddle_point=False, symmetry_tolerance=1e-12) -> dict:
    """core/linalg/matrix_diagnostics.h:285 measure_matrix_characteristics."""
    ro, co, va = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64),
                  np.ascontiguousarray(va, np.float64))
    d = np.empty(3)
    f = np.empty(8, np.int32)
    L = lib()
    L.ref_measure_characteristics.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                              C.c_double, C.c_void_p, C.c_void_p]
    _check(L.ref_measure_characteristics(ro.size - 1, _p(ro), _p(co), _p(va), int(bool(saddle_point)),
                                         float(symmetry_tolerance), _p(d), _p(f)), "characteristics")
    out = dict(equations=int(d[0]), average_nnz_per_row=float(d[1]), coefficient_range=float(d[2]))
    out.update({k: int(v) for k, v in zip(_FLAG_NAMES, f)})
    return out


def select_linear_solver(problem: int, characteristics: dict, krylov=0, preconditioner=0, gmres_restart=40,
                         null_space=0, scaling=0, braess_sarazin_alpha=1.0):
    """core/linalg/linear_solver_models.h:228 select_linear_solver -> (krylov, preconditioner,
    null_space, automatic_krylov, automatic_preconditioner), or None where it throws."""
    c = characteristics
    flags = np.array([c[k] for k in _FLAG_NAMES], np.int32)
    req = np.array([krylov, preconditioner, gmres_restart, null_space, scaling], np.int32)
    plan = np.zeros(5, np.int32)
    L = lib()
    L.ref_select_linear_solver.argtypes = [C.c_int32, C.c_int64, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                           C.c_double, C.c_void_p]
    rc = L.ref_select_linear_solver(int(problem), int(c["equations"]), float(c["average_nnz_per_row"]),
                                    float(c["coefficient_range"]), _p(flags), _p(req), float(braess_sarazin_alpha),
                                    _p(plan))
    return None if rc != 0 else tuple(int(v) for v in plan)


def scale_matrix(ro, co, va, scaling, zero_tolerance=0.0):
    """core/linalg/matrix_diagnostics.h:410 scale_matrix -> (row_scale, column_scale,
    scaled values, zero rows, zero columns)."""
    ro, co, va = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64),
                  np.ascontiguousarray(va, np.float64))
    n = ro.size - 1
    rs, cs, sv = np.empty(n), np.empty(n), np.empty(va.size)
    zc = np.zeros(2, np.int64)
    nnz = C.c_int64()
    L = lib()
    L.ref_scale_matrix.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_double] + \
        [C.c_void_p] * 5
    _check(L.ref_scale_matrix(n, _p(ro), _p(co), _p(va), int(scaling), float(zero_tolerance), _p(rs), _p(cs),
                              _p(sv), _p(zc), C.byref(nnz)), "scale_matrix")
    assert nnz.value == va.size
    return rs, cs, sv, int(zc[0]), int(zc[1])


_DIAG_COUNTS = ("rows", "columns", "nnz", "finite", "structurally_consistent", "empty_rows", "empty_columns",
                "missing_diagonal", "near_zero_diagonal", "isolated_dofs", "duplicate_entries", "connected_components")
_DIAG_VALUES = ("max_abs_value", "min_nonzero_abs_value", "max_row_sum", "min_nonzero_row_sum", "max_column_sum",
                "min_nonzero_column_sum", "max_abs_diagonal", "min_nonzero_abs_diagonal", "diagonal_dynamic_range",
                "row_sum_dynamic_range", "column_sum_dynamic_range", "minimum_gershgorin_margin")


def diagnose_matrix(ro, co, va, n_cols=None, tolerance=1e-14, topology=True) -> dict:
    """core/linalg/matrix_diagnostics.h:126 diagnose_matrix."""
    ro, co, va = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co, np.int64),
                  np.ascontiguousarray(va, np.float64))
    n = ro.size - 1
    c, v = np.zeros(12, np.int64), np.zeros(12)
    L = lib()
    L.ref_diagnose_matrix.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                      C.c_int32, C.c_void_p, C.c_void_p]
    _check(L.ref_diagnose_matrix(n, n if n_cols is None else int(n_cols), _p(ro), _p(co), _p(va), float(tolerance),
                                 int(bool(topology)), _p(c), _p(v)), "diagnose_matrix")
    out = {k: int(x) for k, x in zip(_DIAG_COUNTS, c)}
    out.update({k: float(x) for k, x in zip(_DIAG_VALUES, v)})
    return out
