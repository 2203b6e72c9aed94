"""The allocation-free Rhie-Chow face-flux entry point.

Some callers cannot let a library allocate GPU memory while they run: a host
solver that reserves all device memory when it starts, or one working under a
memory-pool policy that forbids new allocations after start-up (and
cudaMalloc/cudaFree can also stall the whole device).  For them the library
offers cfdxg_rhie_chow_flux_noalloc, which keeps its scratch (the cell
pressure gradient and the boundary-patch table) in a static device array and
calls no allocator.

These tests call it through the C ABI and check that:

* two calls in a row give exactly the face fluxes of the ordinary entry point
  cfdxg_rhie_chow_flux (the same kernels in the same order, so the results are
  bit-identical);
* a call after a warm-up call leaves the device's free memory unchanged;
* NULL patch tables (no fixed-pressure patch), a mesh without patches and a
  mesh with the largest supported patch count (32) work, and 33 patches or a
  mesh beyond the static array's 262,144 cells are refused before any device
  access (every pointer passed is a real device buffer of the mesh's size).

The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import cfdx_dev_b200 as cg
from cfdx_dev_b200 import _native as N
from tests import cases

pytestmark = pytest.mark.gpu

MAX_CELLS = 262_144
MAX_PATCHES = 32


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class _Case:
    """A mesh on the device with the Rhie-Chow inputs as device tensors."""

    def __init__(self, ctx, m):
        import torch
        self.ctx, self.m = ctx, m
        self.mesh = cg.Mesh(ctx, m)
        g = self.mesh.geometry()
        # the benchmark's HbyA and rAU (tests/cases.py seeds); no patch table needed
        U = cg.fourier_field(g["cell_centres"], 8, 0.01, cases.SEED_HBYA)
        rAU = np.concatenate([1.0 / cg.random_field(m.n_cells, "loguniform", 1.0, 100.0, cases.SEED_AP)] * 3)
        self.U, self.rAU = U, rAU
        self.cc = g["cell_centres"].reshape(3, -1)
        dev = torch.device("cuda", 0)
        self.dev = dev
        self.U_d = torch.from_numpy(U).to(dev)
        self.rAU_d = torch.from_numpy(rAU).to(dev)
        self.p_d = torch.zeros(m.n_cells, dtype=torch.float64, device=dev)
        self.flux_d = torch.empty(m.n_faces, dtype=torch.float64, device=dev)

    def noalloc(self, p, fixed, value):
        import torch
        self.p_d.copy_(torch.from_numpy(np.ascontiguousarray(p, np.float64)))
        self.flux_d.fill_(np.nan)
        torch.cuda.synchronize()
        fx = None if fixed is None else np.ascontiguousarray(fixed, np.int32)
        va = None if value is None else np.ascontiguousarray(value, np.float64)
        rc = self.ctx.lib.cfdxg_rhie_chow_flux_noalloc(
            self.ctx.handle, self.mesh.handle, _ptr(self.U_d), _ptr(self.rAU_d), _ptr(self.p_d), 1.0,
            None if fx is None else N.ptr(fx), None if va is None else N.ptr(va), _ptr(self.flux_d))
        return rc, self.flux_d.cpu().numpy()

    def allocating(self, p, fixed, value):
        fx = np.zeros(self.m.n_patches, np.int32) if fixed is None else fixed
        va = np.zeros(self.m.n_patches) if value is None else value
        return cg.make_rhie_chow_mass_flux(self.mesh, self.U, self.rAU, p, 1.0, fx, va)


def _error(ctx):
    return ctx.lib.cfdxg_last_error(ctx.handle).decode()


def _repatched(m, n_patches):
    """The same mesh with its boundary faces dealt round-robin over n_patches patches."""
    out = cg.HostMesh(**{k: getattr(m, k).copy() for k in (
        "px", "py", "pz", "face_offsets", "face_vertices", "owner", "neighbour", "cell_offsets", "cell_faces",
        "patch_of_face", "patch_types")})
    bnd = np.flatnonzero(m.neighbour < 0)
    if n_patches == 0:
        out.patch_of_face[bnd] = -1
        out.patch_types = np.zeros(0, np.int32)
    else:
        out.patch_of_face[bnd] = (np.arange(bnd.size) % n_patches).astype(np.int32)
        out.patch_types = m.patch_types[np.arange(n_patches) % m.n_patches].astype(np.int32)
    return out


@pytest.fixture(scope="module")
def ctx():
    c = cg.Context(0)
    yield c
    c.close()


def test_noalloc_flux_equals_allocating_entry_point_on_two_calls_in_a_row(ctx):
    K = _Case(ctx, cases.simple_mesh(8))
    _, _, _, _, fixed, value = cases.simple_fields(K.m, K.cc.ravel())
    value1 = value.copy()
    value1[0] = 0.5
    for call, (p, val) in enumerate([(np.sin(2 * K.cc[0]) * K.cc[2], value), (K.cc[1] - 0.3 * K.cc[0], value1)]):
        expected = K.allocating(p, fixed, val)
        rc, got = K.noalloc(p, fixed, val)
        assert rc == 0, _error(ctx)
        assert np.array_equal(got, expected), (call, np.abs(got - expected).max())


def test_noalloc_flux_allocates_no_device_memory(ctx):
    import torch
    K = _Case(ctx, cases.simple_mesh(8))
    _, _, _, _, fixed, value = cases.simple_fields(K.m, K.cc.ravel())
    p = np.cos(3 * K.cc[1]) + K.cc[0]
    rc, _ = K.noalloc(p, fixed, value)           # warm-up: loads the device code if it is not yet loaded
    assert rc == 0, _error(ctx)
    fx = np.ascontiguousarray(fixed, np.int32)
    va = np.ascontiguousarray(value, np.float64)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    rc = ctx.lib.cfdxg_rhie_chow_flux_noalloc(ctx.handle, K.mesh.handle, _ptr(K.U_d), _ptr(K.rAU_d), _ptr(K.p_d),
                                              1.0, N.ptr(fx), N.ptr(va), _ptr(K.flux_d))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert rc == 0, _error(ctx)
    assert free1 == free0, (free0, free1)


def test_noalloc_flux_null_patch_tables_and_patch_counts(ctx):
    base = cases.simple_mesh(5)
    for n_patches in (0, 6, MAX_PATCHES):
        m = base if n_patches == 6 else _repatched(base, n_patches)
        K = _Case(ctx, m)
        p = np.sin(K.cc[0] + 2 * K.cc[1])
        # no fixed-pressure patch: NULL tables
        rc, got = K.noalloc(p, None, None)
        assert rc == 0, (n_patches, _error(ctx))
        assert np.array_equal(got, K.allocating(p, None, None)), n_patches
        if n_patches:
            fixed = (np.arange(n_patches) % 3 == 0).astype(np.int32)
            value = np.linspace(-0.5, 0.5, n_patches)
            rc, got = K.noalloc(p, fixed, value)
            assert rc == 0, (n_patches, _error(ctx))
            assert np.array_equal(got, K.allocating(p, fixed, value)), n_patches


def test_noalloc_flux_rejects_more_than_32_patches(ctx):
    K = _Case(ctx, _repatched(cases.simple_mesh(5), MAX_PATCHES + 1))
    fixed = np.zeros(MAX_PATCHES + 1, np.int32)
    value = np.zeros(MAX_PATCHES + 1)
    rc, got = K.noalloc(np.zeros(K.m.n_cells), fixed, value)
    assert rc == N.ERRORS_BY_NAME["invalid_argument"]
    assert "32" in _error(ctx)
    assert np.isnan(got).all()                   # nothing was written


def test_noalloc_flux_rejects_meshes_beyond_its_static_scratch(ctx):
    m = cases.simple_mesh(36)                    # 279,936 cells
    assert m.n_cells > MAX_CELLS
    K = _Case(ctx, m)
    _, _, _, _, fixed, value = cases.simple_fields(m, K.cc.ravel())
    rc, got = K.noalloc(np.zeros(m.n_cells), fixed, value)
    assert rc == N.ERRORS_BY_NAME["invalid_argument"]
    assert str(MAX_CELLS) in _error(ctx)
    assert np.isnan(got).all()
