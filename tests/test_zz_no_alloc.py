"""The allocation-free Rhie-Chow face-flux entry point.

Some callers cannot let a library allocate GPU memory while they run: a host
solver that reserves all device memory when it starts, or one working under a
memory-pool policy that forbids new allocations after start-up (and
cudaMalloc/cudaFree can also stall the whole device).  For them the library
offers cfdxg_rhie_chow_flux_noalloc, which keeps its scratch (the cell
pressure gradient and the boundary-patch table) in a static device array and
calls no allocator.

This file checks, through the C ABI, that two calls in a row give the same face
fluxes as the ordinary entry point cfdxg_rhie_chow_flux, and that a mesh
larger than the static array is refused.  It is named so that pytest collects
it last.
"""
import ctypes as C

import numpy as np
import pytest

import cfdx_dev_b200 as cg
from cfdx_dev_b200 import _native as N
from tests import cases

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10   # same face-flux tolerance as the parity tests


def _flux_reference(mesh, U, rAU, p, fixed, value):
    return cg.make_rhie_chow_mass_flux(mesh, U, rAU, p, 1.0, fixed, value)


def test_noalloc_flux_matches_allocating_entry_point_twice():
    import torch
    ctx = cg.Context(0)
    try:
        m = cases.simple_mesh(8)
        mesh = cg.Mesh(ctx, m)
        g = mesh.geometry()
        U, rAU, aP, p0, fixed, value = cases.simple_fields(m, g["cell_centres"])
        cc = g["cell_centres"].reshape(3, -1)
        value1 = value.copy()
        value1[0] = 0.5
        dev = torch.device("cuda", 0)
        U_d = torch.from_numpy(U).to(dev)
        rAU_d = torch.from_numpy(rAU).to(dev)
        flux_d = torch.empty(m.n_faces, dtype=torch.float64, device=dev)
        fixed_h = np.ascontiguousarray(fixed, np.int32)
        for call, (p, val) in enumerate([(np.sin(2 * cc[0]) * cc[2], value), (cc[1] - 0.3 * cc[0], value1)]):
            expected = _flux_reference(mesh, U, rAU, p, fixed, val)
            p_d = torch.from_numpy(p).to(dev)
            val_h = np.ascontiguousarray(val, np.float64)
            flux_d.fill_(np.nan)
            torch.cuda.synchronize()
            rc = ctx.lib.cfdxg_rhie_chow_flux_noalloc(
                ctx.handle, mesh.handle, C.c_void_p(U_d.data_ptr()), C.c_void_p(rAU_d.data_ptr()),
                C.c_void_p(p_d.data_ptr()), 1.0, N.ptr(fixed_h), N.ptr(val_h), C.c_void_p(flux_d.data_ptr()))
            assert rc == 0, ctx.lib.cfdxg_last_error(ctx.handle).decode()
            got = flux_d.cpu().numpy()
            err = np.linalg.norm(got - expected) / np.linalg.norm(expected)
            assert err <= REL_TOL, (call, err)
    finally:
        ctx.close()


def test_noalloc_flux_rejects_meshes_beyond_its_static_scratch():
    ctx = cg.Context(0)
    try:
        m = cases.simple_mesh(36)   # 279,936 cells > 262,144
        mesh = cg.Mesh(ctx, m)
        rc = ctx.lib.cfdxg_rhie_chow_flux_noalloc(ctx.handle, mesh.handle, C.c_void_p(1), C.c_void_p(1),
                                                  C.c_void_p(1), 1.0, None, None, C.c_void_p(1))
        assert rc == N.ERRORS_BY_NAME["invalid_argument"]
        assert "262144" in ctx.lib.cfdxg_last_error(ctx.handle).decode()
    finally:
        ctx.close()
