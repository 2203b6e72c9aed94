"""Python mirror of the reference's pressure-path API over the C ABI.

Names and argument meanings follow the reference (stevendaix/cfdx_dev):

* ``assemble_cell_diffusion_matrix``  -- core/solvers/scalar_diffusion.h:39
* ``assemble_pressure_correction``    -- physics/steady_incompressible_solver.h:8048-8181
* ``make_rhie_chow_mass_flux``        -- physics/steady_incompressible_solver.h:2064
* ``gauss_gradient_with_boundary``    -- physics/steady_incompressible_solver.h:1634
* ``NativeBoomerAMGPreconditioner``   -- core/linalg/hypre_amg.h:106 (setup / update_values /
                                         apply / name / last_error)
* ``solve_linear_system``             -- core/linalg/linear_solver_dispatch.h:227
* ``solve_gmres`` / ``solve_fgmres``  -- core/linalg/gmres_solver.h:28, 612
* ``solve_cg``                        -- core/linalg/cg_solver.h:605
* ``read_linear_system_capture`` /
  ``write_linear_system_capture``     -- core/linalg/linear_system_capture.h:170, 233

Errors surface as :class:`CfdxgError` (bad requests raise, like the
reference's ``std::invalid_argument``); solver outcomes are reported through
``report["status_name"]`` as the reference's ``SolverStatus``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N


class CfdxgError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{N.ERRORS.get(code, code)}: {message}")
        self.code = code


def _f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Context:
    """A CUDA device + stream owned by the library (cfdxg_context)."""

    def __init__(self, device: int = 0):
        self.lib = N.load()
        h = C.c_void_p()
        rc = self.lib.cfdxg_context_create(device, C.byref(h))
        if rc != 0:
            raise CfdxgError(rc, f"cannot create a context on device {device}")
        self.handle = h

    def check(self, rc: int, what: str = "") -> int:
        if rc < 0:
            msg = self.lib.cfdxg_last_error(self.handle).decode()
            raise CfdxgError(rc, f"{what}: {msg}" if what else msg)
        return rc

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.cfdxg_kernel_launches(self.handle))

    def synchronize(self):
        self.check(self.lib.cfdxg_synchronize(self.handle))

    @property
    def stream(self) -> int:
        """The library's CUDA stream handle (cudaStream_t as an integer)."""
        return int(self.lib.cfdxg_context_stream(self.handle) or 0)

    def profile(self, on: bool = True):
        """Enable (and reset) / disable live kernel timing."""
        self.check(self.lib.cfdxg_profile_enable(self.handle, int(on)))

    def profile_read(self) -> list[dict]:
        """Per kernel class: launches, device ms and algorithmic bytes since profile(True)."""
        buf = (N.KernelProfile * 64)()
        cnt = C.c_int32()
        self.check(self.lib.cfdxg_profile_read(self.handle, buf, 64, C.byref(cnt)))
        return [dict(name=buf[k].name.decode(), launches=buf[k].launches, total_ms=buf[k].total_ms,
                     bytes=buf[k].bytes) for k in range(min(cnt.value, 64))]

    def close(self):
        if getattr(self, "handle", None):
            self.lib.cfdxg_context_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- meshes
@dataclass
class HostMesh:
    """A mesh as flat host arrays (the reference's Mesh contents, core/mesh/mesh.h:51)."""
    px: np.ndarray
    py: np.ndarray
    pz: np.ndarray
    face_offsets: np.ndarray
    face_vertices: np.ndarray
    owner: np.ndarray
    neighbour: np.ndarray
    cell_offsets: np.ndarray
    cell_faces: np.ndarray
    patch_of_face: np.ndarray
    patch_types: np.ndarray

    @property
    def n_points(self):
        return self.px.size

    @property
    def n_faces(self):
        return self.owner.size

    @property
    def n_cells(self):
        return self.cell_offsets.size - 1

    @property
    def n_patches(self):
        return self.patch_types.size

    def desc(self) -> N.MeshDesc:
        d = N.MeshDesc()
        d.n_points, d.n_faces, d.n_cells = self.n_points, self.n_faces, self.n_cells
        for name in ("px", "py", "pz"):
            setattr(d, name, getattr(self, name).ctypes.data_as(N.c_double_p))
        for name in ("face_offsets", "face_vertices", "owner", "neighbour", "cell_offsets", "cell_faces"):
            setattr(d, name, getattr(self, name).ctypes.data_as(N.c_int64_p))
        d.n_patches = self.n_patches
        d.patch_of_face = self.patch_of_face.ctypes.data_as(N.c_int32_p)
        d.patch_types = self.patch_types.ctypes.data_as(N.c_int32_p)
        return d


def _case_to_mesh(lib, h) -> HostMesh:
    sizes = np.zeros(6, dtype=np.int64)
    lib.cfdxg_case_sizes(h, sizes.ctypes.data_as(N.c_int64_p))
    npnt, nf, nfv, nc, ncf, npat = (int(v) for v in sizes)
    m = HostMesh(
        px=np.empty(npnt), py=np.empty(npnt), pz=np.empty(npnt),
        face_offsets=np.empty(nf + 1, np.int64), face_vertices=np.empty(nfv, np.int64),
        owner=np.empty(nf, np.int64), neighbour=np.empty(nf, np.int64),
        cell_offsets=np.empty(nc + 1, np.int64), cell_faces=np.empty(ncf, np.int64),
        patch_of_face=np.empty(nf, np.int32), patch_types=np.empty(npat, np.int32))
    lib.cfdxg_case_export(h, *(N.ptr(getattr(m, f)) for f in (
        "px", "py", "pz", "face_offsets", "face_vertices", "owner", "neighbour", "cell_offsets",
        "cell_faces", "patch_of_face", "patch_types")))
    lib.cfdxg_case_destroy(h)
    return m


def hex_case(nx: int, ny: int | None = None, nz: int | None = None) -> HostMesh:
    """Hex lattice on the unit cube (reference hex-fixture numbering)."""
    lib = N.load()
    h = C.c_void_p()
    rc = lib.cfdxg_case_hex(nx, ny or nx, nz or nx, C.byref(h))
    if rc != 0:
        raise CfdxgError(rc, "hex case")
    return _case_to_mesh(lib, h)


def tet_case(n: int, jitter: float = 0.0, seed: int = 0) -> HostMesh:
    """Kuhn 6-tet split of an n^3 lattice (reference tet-fixture numbering), jittered."""
    lib = N.load()
    h = C.c_void_p()
    rc = lib.cfdxg_case_tet(n, jitter, seed, C.byref(h))
    if rc != 0:
        raise CfdxgError(rc, "tet case")
    return _case_to_mesh(lib, h)


def boundary_layer_case(nx, ny, nz, lx=10.0, lz=1.0, dy0=1e-4, growth=1.08, jitter=0.05, seed=0) -> HostMesh:
    lib = N.load()
    h = C.c_void_p()
    rc = lib.cfdxg_case_boundary_layer(nx, ny, nz, lx, lz, dy0, growth, jitter, seed, C.byref(h))
    if rc != 0:
        raise CfdxgError(rc, "boundary-layer case")
    return _case_to_mesh(lib, h)


def fourier_field(centres: np.ndarray, n_modes: int = 8, perturbation: float = 0.01, seed: int = 0):
    lib = N.load()
    centres = _f64(centres)
    n = centres.size // 3
    u = np.empty(3 * n)
    rc = lib.cfdxg_field_fourier(n, N.ptr(centres), n_modes, perturbation, seed, N.ptr(u))
    if rc != 0:
        raise CfdxgError(rc, "fourier field")
    return u


def random_field(n: int, kind: str, lo: float, hi: float, seed: int):
    lib = N.load()
    v = np.empty(n)
    rc = lib.cfdxg_field_random(n, 0 if kind == "loguniform" else 1, lo, hi, seed, N.ptr(v))
    if rc != 0:
        raise CfdxgError(rc, "random field")
    return v


class Mesh:
    """A mesh resident on the device (cfdxg_mesh) with its GPU-built geometry."""

    def __init__(self, ctx: Context, host: HostMesh, build_geometry: bool = True):
        self.ctx, self.host = ctx, host
        h = C.c_void_p()
        d = host.desc()
        ctx.check(ctx.lib.cfdxg_mesh_upload(ctx.handle, C.byref(d), C.byref(h)), "mesh upload")
        self.handle = h
        if build_geometry:
            self.build_geometry()

    def build_geometry(self):
        self.ctx.check(self.ctx.lib.cfdxg_geometry_build(self.ctx.handle, self.handle), "geometry")

    def geometry(self) -> dict:
        nf, nc = self.host.n_faces, self.host.n_cells
        out = dict(face_centres=np.empty(3 * nf), face_Sf=np.empty(3 * nf),
                   cell_centres=np.empty(3 * nc), cell_volumes=np.empty(nc))
        self.ctx.check(self.ctx.lib.cfdxg_geometry_download(
            self.ctx.handle, self.handle, *(N.ptr(out[k]) for k in
                                            ("face_centres", "face_Sf", "cell_centres", "cell_volumes"))))
        return out

    def __del__(self):  # pragma: no cover
        try:
            if self.handle:
                self.ctx.lib.cfdxg_mesh_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class SparseMatrix:
    """Device CSR (cfdxg_matrix), the reference's SparseMatrix (core/linalg/sparse_matrix.h:27)."""

    def __init__(self, ctx: Context, handle):
        self.ctx, self.handle = ctx, handle
        n, nnz = C.c_int64(), C.c_int64()
        ctx.lib.cfdxg_matrix_size(handle, C.byref(n), C.byref(nnz))
        self.n, self.nnz = n.value, nnz.value

    @classmethod
    def from_csr(cls, ctx: Context, row_offsets, columns, values):
        ro, co, va = _i64(row_offsets), _i64(columns), _f64(values)
        h = C.c_void_p()
        ctx.check(ctx.lib.cfdxg_matrix_create(ctx.handle, ro.size - 1, N.ptr(ro), N.ptr(co), N.ptr(va),
                                              N.CFDXG_MEM_HOST, C.byref(h)), "matrix")
        return cls(ctx, h)

    def to_csr(self):
        ro = np.empty(self.n + 1, np.int64)
        co = np.empty(self.nnz, np.int64)
        va = np.empty(self.nnz)
        self.ctx.check(self.ctx.lib.cfdxg_matrix_download(self.ctx.handle, self.handle, N.ptr(ro), N.ptr(co),
                                                          N.ptr(va)))
        return ro, co, va

    def matvec(self, x):
        x = _f64(x, self.n)
        y = np.empty(self.n)
        self.ctx.check(self.ctx.lib.cfdxg_matrix_spmv(self.ctx.handle, self.handle, N.ptr(x), N.ptr(y),
                                                      N.CFDXG_MEM_HOST))
        return y

    def __del__(self):  # pragma: no cover
        try:
            if self.handle:
                self.ctx.lib.cfdxg_matrix_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def _bc_arrays(mesh_host: HostMesh, fixed, value):
    npat = mesh_host.n_patches
    f = np.zeros(npat, np.int32) if fixed is None else _i32(fixed)
    v = np.zeros(npat) if value is None else _f64(value)
    return f, v


def assemble_cell_diffusion_matrix(mesh: Mesh, bc_face_values, diffusivity, source, bc_face_types=None):
    """core/solvers/scalar_diffusion.h:39-163 -> (SparseMatrix, rhs)."""
    ctx = mesh.ctx
    bcv = _f64(bc_face_values, mesh.host.n_faces)
    bct = None if bc_face_types is None else _i32(bc_face_types)
    src = _f64(source, mesh.host.n_cells)
    rhs = np.empty(mesh.host.n_cells)
    h = C.c_void_p()
    ctx.check(ctx.lib.cfdxg_assemble_cell_diffusion(ctx.handle, mesh.handle, N.ptr(bcv), N.ptr(bct),
                                                    float(diffusivity), N.ptr(src), N.CFDXG_MEM_HOST,
                                                    C.byref(h), N.ptr(rhs)), "assemble_cell_diffusion_matrix")
    return SparseMatrix(ctx, h), rhs


def solve_poisson_mixed(mesh: Mesh, bc_face_values, source, bc_face_types=None, diffusivity=1.0,
                        max_iterations=2000, tolerance=1e-10, reference_cell=0, reference_value=0.0,
                        compatibility_tolerance=1e-12) -> dict:
    """solve_poisson_mixed (core/solvers/scalar_diffusion.h:294-340), the
    Poisson driver of the reference's apps/poisson: cell-centred diffusion
    assembly; without a Dirichlet face the pure-Neumann compatibility check
    (:306-325) and the reference-cell identity-row gauge (:326-333); then CG
    with the solver's own diagonal scaling, from zero (the reference value at
    the reference cell).  bc_face_types: 0 Dirichlet (default), 1 Neumann
    (prescribed flux).  Returns dict(solution, report, matrix, rhs); ValueError
    on incompatible pure-Neumann data."""
    A, rhs = assemble_cell_diffusion_matrix(mesh, bc_face_values, diffusivity, source, bc_face_types)
    bcv = _f64(bc_face_values, mesh.host.n_faces)
    types = np.zeros(bcv.size, np.int32) if bc_face_types is None else _i32(bc_face_types)
    x0 = np.zeros(A.n)
    finite = np.isfinite(bcv)
    if not np.any(finite & (types == 0)):
        # scalar_diffusion.h:223-238 pure_neumann_compatibility_residual and the scale of :309-317
        g = mesh.geometry()
        vol = g["cell_volumes"]
        area = np.linalg.norm(g["face_Sf"].reshape(3, -1), axis=0)
        src = _f64(source, A.n)
        neumann = finite & (types == 1)
        balance = 0.0
        for c in range(A.n):
            balance += src[c] * vol[c]
        for f in np.flatnonzero(neumann):
            balance += bcv[f] * area[f]
        scale = 1.0 + float(np.sum(np.abs(src) * vol)) + float(np.sum(np.abs(bcv[neumann]) * area[neumann]))
        if not np.isfinite(balance) or not (compatibility_tolerance >= 0.0) or \
                abs(balance) > compatibility_tolerance * scale:
            raise ValueError("solve_poisson_mixed: incompatible pure-Neumann data; "
                             "integral(S dV) + integral(q_n dA) must be zero")
        gauge = ReferenceCellGauge(A.ctx, A, ref=reference_cell, mode="identity_row", value=reference_value)
        A, rhs = gauge.apply(A, rhs)
        x0[reference_cell] = reference_value
    x, report = solve_linear_system(A, rhs, x0, krylov="cg", preconditioner="own_diagonal",
                                    max_iterations=max_iterations, tolerance=tolerance)
    return dict(solution=x, report=report, matrix=A, rhs=rhs)


def assemble_pressure_correction(mesh: Mesh, HbyA, rAU, p, rho=1.0, p_bc_fixed=None, p_bc_value=None,
                                 matrix: SparseMatrix | None = None):
    """Pressure-corrector assembly (steady_incompressible_solver.h:8048-8181).

    Returns (A, b, phiHbyA, grad_p)."""
    ctx, hm = mesh.ctx, mesh.host
    U, r, pp = _f64(HbyA, 3 * hm.n_cells), _f64(rAU, 3 * hm.n_cells), _f64(p, hm.n_cells)
    f, v = _bc_arrays(hm, p_bc_fixed, p_bc_value)
    b = np.empty(hm.n_cells)
    phi = np.empty(hm.n_faces)
    grad = np.empty(3 * hm.n_cells)
    h = C.c_void_p(matrix.handle.value if matrix is not None else None)
    ctx.check(ctx.lib.cfdxg_assemble_pressure_correction(
        ctx.handle, mesh.handle, N.ptr(U), N.ptr(r), N.ptr(pp), float(rho), N.ptr(f), N.ptr(v),
        N.CFDXG_MEM_HOST, C.byref(h), N.ptr(b), N.ptr(phi), N.ptr(grad)), "pressure-correction assembly")
    A = matrix if matrix is not None else SparseMatrix(ctx, h)
    return A, b, phi, grad


def make_rhie_chow_mass_flux(mesh: Mesh, HbyA, rAU, p, rho=1.0, p_bc_fixed=None, p_bc_value=None):
    """physics/steady_incompressible_solver.h:2064-2217 (HBYA_PREDICTOR contract)."""
    ctx, hm = mesh.ctx, mesh.host
    U, r, pp = _f64(HbyA, 3 * hm.n_cells), _f64(rAU, 3 * hm.n_cells), _f64(p, hm.n_cells)
    f, v = _bc_arrays(hm, p_bc_fixed, p_bc_value)
    flux = np.empty(hm.n_faces)
    ctx.check(ctx.lib.cfdxg_rhie_chow_flux(ctx.handle, mesh.handle, N.ptr(U), N.ptr(r), N.ptr(pp), float(rho),
                                           N.ptr(f), N.ptr(v), N.CFDXG_MEM_HOST, N.ptr(flux)),
              "make_rhie_chow_mass_flux")
    return flux


def build_hbya(mesh: Mesh, momentum, rhs, U, gradp, rAU):
    """physics/steady_incompressible_solver.h:6430-6465 (build_hbya) -> HbyA (3*n_cells).

    ``momentum``: one SparseMatrix, or three (one per component) sharing a pattern."""
    ctx, hm = mesh.ctx, mesh.host
    mats = list(momentum) if isinstance(momentum, (list, tuple)) else [momentum] * 3
    handles = (C.c_void_p * 3)(*[M.handle.value for M in mats])
    n3 = 3 * hm.n_cells
    b, u, g, r = (_f64(a, n3) for a in (rhs, U, gradp, rAU))
    out = np.empty(n3)
    ctx.check(ctx.lib.cfdxg_build_hbya(ctx.handle, mesh.handle, handles, N.ptr(b), N.ptr(u), N.ptr(g), N.ptr(r),
                                       N.CFDXG_MEM_HOST, N.ptr(out)), "build_hbya")
    return out


def gauss_gradient_with_boundary(mesh: Mesh, p, p_bc_fixed=None, p_bc_value=None):
    ctx, hm = mesh.ctx, mesh.host
    pp = _f64(p, hm.n_cells)
    f, v = _bc_arrays(hm, p_bc_fixed, p_bc_value)
    g = np.empty(3 * hm.n_cells)
    ctx.check(ctx.lib.cfdxg_gauss_gradient(ctx.handle, mesh.handle, N.ptr(pp), N.ptr(f), N.ptr(v),
                                           N.CFDXG_MEM_HOST, N.ptr(g)), "gauss_gradient_with_boundary")
    return g


# ---------------------------------------------------------------- AMG
class NativeBoomerAMGPreconditioner:
    """Native classical RS AMG (core/linalg/hypre_amg.h:106), GPU V-cycle.

    ``precision="fp32_vcycle"`` runs the V-cycle in FP32 with a dense coarse
    inverse formed in FP64 (the hierarchy itself is identical); between the
    fine and the coarsest level it smooths with sparsified copies of the
    Galerkin operators (``coarse_drop_tolerance``, default 0.02: each row's
    diagonal and its entries of at least that fraction of the row's largest
    off-diagonal magnitude, the rest added to the diagonal; 0 smooths with
    the Galerkin operators).  Other keyword options are the fields of
    ``cfdxg_amg_options`` (include/cfdxg.h)."""

    def __init__(self, ctx: Context | None = None, precision: str = "fp64", require_smoother_certificate=False,
                 **options):
        self.ctx = ctx
        self.lib = N.load()
        o = N.AmgOptions()
        self.lib.cfdxg_amg_options_default(C.byref(o))
        o.precision = N.PRECISION[precision]
        o.require_smoother_certificate = int(bool(require_smoother_certificate))
        if "coarse_sweeps" in options:   # shorthand: the same count before and after
            o.coarse_pre_sweeps = o.coarse_post_sweeps = options.pop("coarse_sweeps")
        for k, v in options.items():
            setattr(o, k, v)
        h = C.c_void_p()
        rc = self.lib.cfdxg_amg_create(ctx.handle if ctx else None, C.byref(o), C.byref(h))
        if rc != 0:
            raise CfdxgError(rc, "AMG options")
        self.handle = h

    def setup(self, A: SparseMatrix) -> bool:
        rc = self.lib.cfdxg_amg_setup(self.ctx.handle, self.handle, A.handle)
        if rc == -3:
            return False
        self.ctx.check(rc, "AMG setup")
        return True

    def setup_host(self, row_offsets, columns, values) -> bool:
        ro, co, va = _i64(row_offsets), _i64(columns), _f64(values)
        rc = self.lib.cfdxg_amg_setup_host(self.handle, ro.size - 1, N.ptr(ro), N.ptr(co), N.ptr(va))
        if rc == -3:
            return False
        if rc != 0:
            raise CfdxgError(rc, self.last_error())
        return True

    def update_values(self, A: SparseMatrix) -> bool:
        """Numeric refresh on an unchanged pattern, computed on the device."""
        rc = self.lib.cfdxg_amg_update_values(self.ctx.handle, self.handle, A.handle)
        if rc == -3:
            return False
        self.ctx.check(rc, "AMG update_values")
        return True

    def update_values_host(self, row_offsets, columns, values) -> bool:
        """Numeric refresh of a setup_host hierarchy on the host."""
        ro, co, va = _i64(row_offsets), _i64(columns), _f64(values)
        rc = self.lib.cfdxg_amg_update_values_host(self.handle, ro.size - 1, N.ptr(ro), N.ptr(co), N.ptr(va))
        if rc == -3:
            return False
        if rc != 0:
            raise CfdxgError(rc, self.last_error())
        return True

    def apply(self, r) -> np.ndarray:
        r = _f64(r)
        z = np.empty_like(r)
        self.ctx.check(self.lib.cfdxg_amg_apply(self.ctx.handle, self.handle, N.ptr(r), N.ptr(z), N.CFDXG_MEM_HOST),
                       "AMG apply")
        return z

    def name(self) -> str:
        return self.lib.cfdxg_amg_name(self.handle).decode()

    def last_error(self) -> str:
        return self.lib.cfdxg_amg_last_error(self.handle).decode()

    @property
    def omega(self) -> float:
        return float(self.lib.cfdxg_amg_omega(self.handle))

    @property
    def setup_seconds(self) -> float:
        return float(self.lib.cfdxg_amg_setup_seconds(self.handle))

    def hierarchy_level_sizes(self):
        return [self._info(l)[0] for l in range(self.lib.cfdxg_amg_num_levels(self.handle))]

    def hierarchy_level_nnz(self):
        return [self._info(l)[1] for l in range(self.lib.cfdxg_amg_num_levels(self.handle))]

    def operator_complexity(self) -> float:
        nnz = self.hierarchy_level_nnz()
        return sum(nnz) / nnz[0] if nnz else 0.0

    def _info(self, level):
        n, nnz, pn = C.c_int64(), C.c_int64(), C.c_int64()
        self.lib.cfdxg_amg_level_info(self.handle, level, C.byref(n), C.byref(nnz), C.byref(pn))
        return n.value, nnz.value, pn.value

    def export_level(self, level: int) -> dict:
        n, nnz, pn = self._info(level)
        out = dict(row_offsets=np.empty(n + 1, np.int64), columns=np.empty(nnz, np.int64), values=np.empty(nnz),
                   inv_diag=np.empty(n), p_offsets=np.empty(n + 1, np.int64), p_columns=np.empty(pn, np.int64),
                   p_values=np.empty(pn), aggregate=np.empty(n, np.int64))
        rc = self.lib.cfdxg_amg_export_level(self.handle, level, *(N.ptr(out[k]) for k in (
            "row_offsets", "columns", "values", "inv_diag", "p_offsets", "p_columns", "p_values", "aggregate")))
        if rc != 0:
            raise CfdxgError(rc, "export level")
        if pn == 0:
            out["p_offsets"] = None
            out["aggregate"] = None
        return out

    def __del__(self):  # pragma: no cover
        try:
            if self.handle:
                self.lib.cfdxg_amg_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class ReusablePreconditionerContext:
    """ReusablePreconditionerContext (core/linalg/linear_solver_context.h:15-65):
    owns the lifecycle of one preconditioner across a sequence of matrices --
    a full setup when the CSR structure changed, the numeric refresh when only
    the values changed (a full setup again if the refresh is refused), nothing
    when the matrix is unchanged -- with the reference's statistics
    (full_setups, numeric_updates, unchanged_reuses, solves).

    ``prepare`` takes a device ``SparseMatrix`` (device setup and refresh) or
    host CSR arrays ``(row_offsets, columns, values)`` (host setup and refresh).
    The comparison is against a snapshot of the last prepared matrix, as the
    reference keeps one."""

    def __init__(self, preconditioner: NativeBoomerAMGPreconditioner):
        self.pc = preconditioner
        self.stats = dict(full_setups=0, numeric_updates=0, unchanged_reuses=0, solves=0)
        self._snapshot = None

    def invalidate(self):
        self._snapshot = None

    def prepare(self, A) -> bool:
        if isinstance(A, SparseMatrix):
            ro, co, va = A.to_csr()
            setup, update = (lambda: self.pc.setup(A)), (lambda: self.pc.update_values(A))
        else:
            ro, co, va = (np.ascontiguousarray(A[0], np.int64), np.ascontiguousarray(A[1], np.int64),
                          np.ascontiguousarray(A[2], np.float64))
            setup, update = (lambda: self.pc.setup_host(ro, co, va)), (lambda: self.pc.update_values_host(ro, co, va))
        if ro.size < 2 or ro[-1] != co.size or co.size != va.size or not np.all(np.isfinite(va)):
            return False
        snap = self._snapshot
        same_structure = snap is not None and np.array_equal(snap[0], ro) and np.array_equal(snap[1], co)
        same_values = same_structure and np.array_equal(snap[2], va)
        if not same_structure:
            ready = setup()
            self.stats["full_setups"] += int(ready)
        elif not same_values:
            ready = update()
            if ready:
                self.stats["numeric_updates"] += 1
            else:                              # a refused refresh rebuilds from the current matrix
                ready = setup()
                self.stats["full_setups"] += int(ready)
        else:
            ready = True
            self.stats["unchanged_reuses"] += 1
        if not ready:
            self.invalidate()
            return False
        self._snapshot = (ro.copy(), co.copy(), va.copy())
        return True

    def solve(self, A: SparseMatrix, rhs, x0=None, **kw):
        """prepare(A), then the prepared solve (solve_gmres; krylov="cg" for CG) -> (x, report)."""
        if not self.prepare(A):
            raise CfdxgError(N.CFDXG_ERR_SETUP, f"preconditioner preparation failed: {self.pc.last_error()}")
        self.stats["solves"] += 1
        return solve_gmres(A, rhs, x0=x0, amg=self.pc, **kw)


def make_request(krylov="gmres", preconditioner="native_amg", restart=40, precision="fp64", learned=None,
                 problem="pressure_poisson", scaling="none", null_space="none", **kw):
    """A cfdxg_request; krylov / preconditioner "auto" select the plan from the measured matrix.
    null_space="constant": the projected solves of a pure-Neumann operator (NullSpaceModel::Constant)."""
    lib = N.load()
    r = N.Request()
    lib.cfdxg_request_default(C.byref(r))
    r.krylov = N.KRYLOV[krylov]
    r.preconditioner = N.PRECONDITIONER[preconditioner]
    r.gmres_restart = restart
    r.precision = N.PRECISION[precision]
    r.learned = learned.handle if learned is not None else None
    r.problem = N.PROBLEMS.index(problem)
    r.scaling = N.SCALINGS.index(scaling)
    r.null_space = N.NULL_SPACES.index(null_space)
    for k, v in kw.items():
        setattr(r, k, v)
    return r


def measure_matrix_characteristics(row_offsets, columns, values, saddle_point=False,
                                   symmetry_tolerance=1e-12) -> dict:
    """core/linalg/matrix_diagnostics.h:285 measure_matrix_characteristics, on the host."""
    lib = N.load()
    ro, co, va = _i64(row_offsets), _i64(columns), _f64(values)
    c = N.MatrixCharacteristics()
    rc = lib.cfdxg_measure_matrix_characteristics(ro.size - 1, N.ptr(ro), N.ptr(co), N.ptr(va),
                                                  int(bool(saddle_point)), float(symmetry_tolerance), C.byref(c))
    if rc != 0:
        raise CfdxgError(rc, lib.cfdxg_plan_last_error().decode())
    return c.as_dict()


def diagnose_matrix(row_offsets, columns, values, n_cols=None, diagonal_relative_tolerance=1e-14,
                    include_topology=True) -> dict:
    """core/linalg/matrix_diagnostics.h:126 diagnose_matrix on the host (MatrixDiagnostics fields)."""
    lib = N.load()
    ro, co, va = _i64(row_offsets), _i64(columns), _f64(values)
    n = ro.size - 1
    d = N.MatrixDiagnostics()
    rc = lib.cfdxg_diagnose_matrix(n, n if n_cols is None else int(n_cols), N.ptr(ro), N.ptr(co), N.ptr(va),
                                   float(diagonal_relative_tolerance), int(bool(include_topology)), C.byref(d))
    if rc != 0:
        raise CfdxgError(rc, lib.cfdxg_plan_last_error().decode())
    return d.as_dict()


def scale_matrix(row_offsets, columns, values, scaling: str, zero_tolerance=0.0):
    """core/linalg/matrix_diagnostics.h:410 scale_matrix on the host -> dict of the
    row and column scales, the scaled values (same pattern) and the zero counts."""
    lib = N.load()
    ro, co, va = _i64(row_offsets), _i64(columns), _f64(values)
    n = ro.size - 1
    out = dict(row_scale=np.empty(n), column_scale=np.empty(n), values=np.empty(va.size))
    zc = np.zeros(2, np.int64)
    rc = lib.cfdxg_scale_matrix(n, N.ptr(ro), N.ptr(co), N.ptr(va), N.SCALINGS.index(scaling), float(zero_tolerance),
                                N.ptr(out["row_scale"]), N.ptr(out["column_scale"]), N.ptr(out["values"]), N.ptr(zc))
    if rc != 0:
        raise CfdxgError(rc, lib.cfdxg_plan_last_error().decode())
    out.update(zero_rows=int(zc[0]), zero_columns=int(zc[1]))
    return out


def select_linear_solver(problem: str, characteristics: dict, krylov="auto", preconditioner="auto",
                         gmres_restart=40, null_space="none", scaling="none", braess_sarazin_alpha=1.0) -> dict:
    """core/linalg/linear_solver_models.h:228 select_linear_solver -> plan (model names and flags).

    Raises CfdxgError where the reference throws std::invalid_argument."""
    lib = N.load()
    c = N.MatrixCharacteristics(**{k: characteristics[k] for k, _ in N.MatrixCharacteristics._fields_})
    r = N.PlanRequest(N.KRYLOV_MODELS.index(krylov), N.PRECONDITIONER_MODELS.index(preconditioner),
                      int(gmres_restart), N.NULL_SPACES.index(null_space), N.SCALINGS.index(scaling),
                      float(braess_sarazin_alpha))
    plan = N.SolverPlan()
    rc = lib.cfdxg_select_linear_solver(N.PROBLEMS.index(problem), C.byref(c), C.byref(r), C.byref(plan))
    if rc != 0:
        raise CfdxgError(rc, lib.cfdxg_plan_last_error().decode())
    return dict(problem=N.PROBLEMS[plan.problem], krylov=N.KRYLOV_MODELS[plan.krylov],
                preconditioner=N.PRECONDITIONER_MODELS[plan.preconditioner], null_space=N.NULL_SPACES[plan.null_space],
                automatic_krylov=bool(plan.automatic_krylov),
                automatic_preconditioner=bool(plan.automatic_preconditioner), reason=plan.reason.decode())


def solve_linear_system(A: SparseMatrix, rhs, x0=None, krylov="gmres", preconditioner="native_amg",
                        restart=40, precision="fp64", max_iterations=1000, tolerance=1e-12, learned=None,
                        linear_capture_path=None, **kw):
    """core/linalg/linear_solver_dispatch.h:227 for PressurePoisson systems -> (x, report).

    ``linear_capture_path`` (opt-in, as LinearSolverRequest::linear_capture_path)
    writes the system with its initial guess to a .cfdxlin file before the
    solve (linear_solver_dispatch.h:236-239)."""
    ctx = A.ctx
    b = _f64(rhs, A.n)
    x = np.zeros(A.n) if x0 is None else _f64(x0, A.n).copy()
    if linear_capture_path:
        ro, co, va = A.to_csr()
        write_linear_system_capture(linear_capture_path, ro, co, va, b, x, problem=CAPTURE_PRESSURE_POISSON,
                                    null_space=N.NULL_SPACES.index(kw.get("null_space", "none")),
                                    scaling=N.SCALINGS.index(kw.get("scaling", "none")),
                                    max_iterations=max_iterations, tolerance=tolerance)
    req = make_request(krylov, preconditioner, restart, precision, learned, **kw)
    rep = N.Report()
    rc = ctx.lib.cfdxg_solve_linear_system(ctx.handle, A.handle, N.ptr(b), N.ptr(x), N.CFDXG_MEM_HOST,
                                           C.byref(req), int(max_iterations), float(tolerance), C.byref(rep))
    ctx.check(rc, "solve_linear_system")
    return x, rep.as_dict()


def solve_gmres(A: SparseMatrix, rhs, x0=None, amg: NativeBoomerAMGPreconditioner | None = None, restart=30,
                max_iterations=1000, tolerance=1e-12, krylov="gmres", learned=None, **kw):
    """core/linalg/gmres_solver.h:28 with a prepared preconditioner -> (x, report)."""
    ctx = A.ctx
    b = _f64(rhs, A.n)
    x = np.zeros(A.n) if x0 is None else _f64(x0, A.n).copy()
    req = make_request(krylov, "native_amg" if amg else "none", restart, "fp64", learned, **kw)
    rep = N.Report()
    rc = ctx.lib.cfdxg_solve_gmres(ctx.handle, A.handle, amg.handle if amg else None, N.ptr(b), N.ptr(x),
                                   N.CFDXG_MEM_HOST, C.byref(req), int(max_iterations), float(tolerance),
                                   C.byref(rep))
    ctx.check(rc, "solve_gmres")
    return x, rep.as_dict()


def solve_fgmres(A, rhs, x0=None, amg=None, restart=30, max_iterations=1000, tolerance=1e-12, **kw):
    return solve_gmres(A, rhs, x0, amg, restart, max_iterations, tolerance, krylov="fgmres", **kw)


def solve_cg(A: SparseMatrix, rhs, x0=None, amg: NativeBoomerAMGPreconditioner | None = None, max_iterations=1000,
             tolerance=1e-12):
    """core/linalg/cg_solver.h:605 solve_cg(A, b, x, preconditioner) with a
    prepared native AMG (or the identity) -> (x, report)."""
    return solve_gmres(A, rhs, x0, amg, 30, max_iterations, tolerance, krylov="cg")


# ---------------------------------------------------------------- pressure gauge
class ReferenceCellGauge:
    """Gauge of a pure-Neumann system on the device.

    ``mode="eliminate"``: the pure-Neumann branch of the pressure corrector
    (physics/steady_incompressible_solver.h:8617-8654) -- the system without
    cell ``ref``; ``expand`` gives the full correction with 0 at ``ref``.
    ``mode="identity_row"``: apply_reference_cell_gauge
    (core/solvers/scalar_diffusion.h:177-210) -- a unit row at ``ref`` and
    rhs_i -= a_i,ref * value.  The plan is built once from A's pattern; each
    ``apply`` gathers the current values and right-hand side on the device."""

    MODES = {"eliminate": 0, "identity_row": 1}

    def __init__(self, ctx: Context, A: SparseMatrix, ref: int = 0, mode: str = "eliminate", value: float = 0.0):
        self.ctx, self.lib = ctx, ctx.lib
        h = C.c_void_p()
        ctx.check(self.lib.cfdxg_gauge_create(ctx.handle, A.handle, self.MODES[mode], int(ref), float(value),
                                              C.byref(h)), "gauge")
        self.handle = h
        n, nnz = C.c_int64(), C.c_int64()
        self.lib.cfdxg_gauge_size(h, C.byref(n), C.byref(nnz))
        self.n_out, self.nnz_out = n.value, nnz.value
        self.n = A.n
        self._gauged = None

    def apply(self, A: SparseMatrix, rhs):
        """-> (gauged SparseMatrix, gauged right-hand side); the matrix object is
        reused (values refreshed) on later calls."""
        b = _f64(rhs, self.n)
        out = np.empty(self.n_out)
        h = C.c_void_p(self._gauged.handle.value if self._gauged is not None else None)
        self.ctx.check(self.lib.cfdxg_gauge_apply(self.ctx.handle, self.handle, A.handle, N.ptr(b),
                                                  N.CFDXG_MEM_HOST, C.byref(h), N.ptr(out)), "gauge apply")
        if self._gauged is None:
            self._gauged = SparseMatrix(self.ctx, h)
        return self._gauged, out

    def expand(self, x_reduced) -> np.ndarray:
        xr = _f64(x_reduced, self.n_out)
        x = np.empty(self.n)
        self.ctx.check(self.lib.cfdxg_gauge_expand(self.ctx.handle, self.handle, N.ptr(xr), N.CFDXG_MEM_HOST,
                                                   N.ptr(x)), "gauge expand")
        return x

    def __del__(self):  # pragma: no cover
        try:
            if self.handle:
                self.lib.cfdxg_gauge_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


# ---------------------------------------------------------------- learned preconditioner
class LearnedPreconditioner:
    """4-round, 32-feature message-passing network on the matrix graph (no
    reference counterpart), applied in front of the AMG V-cycle inside FGMRES.
    Training runs on the GPU (FP32 forward/backward + Adam); inference uses
    BF16 tensor-core MLPs with FP32 state and accumulation."""

    def __init__(self, ctx: Context, seed: int = 0):
        self.ctx, self.lib = ctx, ctx.lib
        h = C.c_void_p()
        ctx.check(self.lib.cfdxg_mpnn_create(ctx.handle, seed, C.byref(h)), "mpnn create")
        self.handle = h
        cnt = C.c_int64()
        self.lib.cfdxg_mpnn_num_parameters(h, C.byref(cnt))
        self.n_params = cnt.value
        self.n = None

    def bind(self, mesh: Mesh, A: SparseMatrix, a_P):
        a = _f64(a_P, A.n)
        self.ctx.check(self.lib.cfdxg_mpnn_bind(self.ctx.handle, self.handle, mesh.handle, A.handle, N.ptr(a),
                                                N.CFDXG_MEM_HOST), "mpnn bind")
        self.n = A.n

    def set_vcycle(self, amg):
        """Train in front of this V-cycle (composed-preconditioner loss); None: the network alone."""
        self.ctx.check(self.lib.cfdxg_mpnn_set_vcycle(self.ctx.handle, self.handle, amg.handle if amg else None))

    def parameters(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        self.ctx.check(self.lib.cfdxg_mpnn_get_parameters(self.ctx.handle, self.handle, N.ptr(p)))
        return p

    def set_parameters(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self.ctx.check(self.lib.cfdxg_mpnn_set_parameters(self.ctx.handle, self.handle, N.ptr(p)))

    def save(self, path):
        self.ctx.check(self.lib.cfdxg_mpnn_save(self.ctx.handle, self.handle, str(path).encode()), "save")

    def load(self, path):
        self.ctx.check(self.lib.cfdxg_mpnn_load(self.ctx.handle, self.handle, str(path).encode()), "load")

    def apply(self, r) -> np.ndarray:
        r = _f64(r, self.n)
        y = np.empty(self.n)
        self.ctx.check(self.lib.cfdxg_mpnn_apply(self.ctx.handle, self.handle, N.ptr(r), N.ptr(y), N.CFDXG_MEM_HOST))
        return y

    def loss_grad(self, R, E):
        R, E = np.ascontiguousarray(R, np.float64), np.ascontiguousarray(E, np.float64)
        B = R.shape[0]
        loss = C.c_double()
        g = np.empty(self.n_params, np.float32)
        self.ctx.check(self.lib.cfdxg_mpnn_loss_grad(self.ctx.handle, self.handle, N.ptr(R), N.ptr(E), B,
                                                     N.CFDXG_MEM_HOST, C.byref(loss), N.ptr(g)), "loss_grad")
        return loss.value, g

    def train_step(self, R, E, lr=1e-3) -> float:
        R, E = np.ascontiguousarray(R, np.float64), np.ascontiguousarray(E, np.float64)
        loss = C.c_double()
        self.ctx.check(self.lib.cfdxg_mpnn_train_step(self.ctx.handle, self.handle, N.ptr(R), N.ptr(E), R.shape[0],
                                                      float(lr), N.CFDXG_MEM_HOST, C.byref(loss)), "train_step")
        return loss.value

    def __del__(self):  # pragma: no cover
        try:
            if self.handle:
                self.lib.cfdxg_mpnn_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


# ---------------------------------------------------------------------------
# linear-system replay files (.cfdxlin)
# ---------------------------------------------------------------------------
# LinearProblemKind (core/linalg/linear_solver_models.h:11-18): General 0,
# PressurePoisson 1, Diffusion 2, Momentum 3, ScalarTransport 4,
# CoupledPressureVelocity 5; NullSpaceModel None 0 / Constant 1.
CAPTURE_GENERAL, CAPTURE_PRESSURE_POISSON, CAPTURE_DIFFUSION = 0, 1, 2


def parse_linear_capture_iterations(csv: str, max_count: int = 32) -> list[int]:
    """parse_linear_capture_iterations (core/linalg/linear_system_capture.h:39-65):
    a comma-separated list of distinct positive outer iterations; ValueError on
    an empty, malformed, zero, duplicated or over-long list."""
    if not csv or max_count == 0:
        raise ValueError("capture iterations: missing selection")
    values = []
    for token in csv.split(","):
        if not token or len(values) >= max_count or not all("0" <= ch <= "9" for ch in token):
            raise ValueError("capture iterations: malformed list")
        number = int(token)
        if number == 0 or number > 2**64 - 1:
            raise ValueError("capture iterations: invalid value")
        values.append(number)
    if not values or csv.endswith(","):
        raise ValueError("capture iterations: empty selection")
    if len(set(values)) != len(values):
        raise ValueError("capture iterations: duplicated selection")
    return values


def read_linear_system_capture(path) -> dict:
    """read_linear_system_capture (core/linalg/linear_system_capture.h:233-284):
    CSR, right-hand side, initial guess and solver metadata of a .cfdxlin file.
    Raises CfdxgError on a malformed, truncated or corrupted file."""
    lib = N.load()
    h = C.c_void_p()
    info = N.CaptureInfo()
    rc = lib.cfdxg_capture_read(str(path).encode(), C.byref(h), C.byref(info))
    if rc != 0:
        raise CfdxgError(rc, lib.cfdxg_capture_last_error().decode())
    try:
        out = dict(row_offsets=np.empty(info.n + 1, np.int64), columns=np.empty(info.nnz, np.int64),
                   values=np.empty(info.nnz), rhs=np.empty(info.n), initial_solution=np.empty(info.n))
        lib.cfdxg_capture_export(h, *(N.ptr(out[k]) for k in ("row_offsets", "columns", "values", "rhs",
                                                               "initial_solution")))
    finally:
        lib.cfdxg_capture_destroy(h)
    out.update(problem=info.problem, null_space=info.null_space, scaling=info.scaling,
               max_iterations=info.max_iterations, tolerance=info.tolerance, checksum=info.checksum)
    return out


def write_linear_system_capture(path, row_offsets, columns, values, rhs, initial_solution,
                                problem=CAPTURE_PRESSURE_POISSON, null_space=0, scaling=0, max_iterations=1000,
                                tolerance=1e-8) -> int:
    """write_linear_system_capture (core/linalg/linear_system_capture.h:170-231);
    returns the file's checksum.  Invalid input raises before a file exists."""
    lib = N.load()
    ro, co, va = _i64(row_offsets), _i64(columns), _f64(values)
    n = ro.size - 1
    if n < 1 or co.size != ro[-1] or va.size != ro[-1]:
        raise ValueError("linear capture: CSR arrays of inconsistent sizes")
    b, x = _f64(rhs, n), _f64(initial_solution, n)
    info = N.CaptureInfo(problem, null_space, scaling, n, va.size, max_iterations, tolerance, 0)
    rc = lib.cfdxg_capture_write(str(path).encode(), n, N.ptr(ro), N.ptr(co), N.ptr(va), N.ptr(b), N.ptr(x),
                                 C.byref(info))
    if rc != 0:
        raise CfdxgError(rc, lib.cfdxg_capture_last_error().decode())
    return int(info.checksum)
