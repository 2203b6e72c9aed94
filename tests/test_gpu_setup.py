"""The AMG setup with its Galerkin products on the device (cfdxg_amg_setup):
the symbolic graphs by expand-sort-unique and the numeric products and
pruning of the refresh kernels, against the host setup (csrc/amg_setup.cpp,
pinned level by level to the reference's own setup by the CPU tests) and, at
32^3 (196,608 cells), against the fingerprints of the reference's own setup.
Every level's CSR, inverse diagonal, prolongation and the damping must be
bit-identical; a numeric refresh through the plan the device setup left
behind must equal the host refresh."""
import json
import time
from pathlib import Path

import numpy as np
import pytest

import cfdx_dev_b200 as cg
from tests import cases

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def _system(oracle, case, seed_offset=0):
    if case.startswith("tet") or case == "neumann":
        m = cases.simple_mesh(10 if case != "neumann" else 8, seed_offset=0)
        g = oracle.geometry(m)
        U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"], seed_offset=seed_offset)
        if case == "neumann":
            fixed = np.zeros_like(fixed)
        r = oracle.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
        return r["row_offsets"], r["columns"], r["values"]
    if case == "hex16":
        m, bc, src = cases.poisson_case(16)
    else:   # anisotropic boundary layer
        m = cg.boundary_layer_case(12, 10, 6, dy0=1e-3, growth=1.2, jitter=0.05, seed=5)
        bc = np.full(m.n_faces, np.nan)
        bc[m.patch_of_face == 0] = 0.0
        src = cg.random_field(m.n_cells, "uniform", -1.0, 1.0, 3)
    ro, co, va, rhs = oracle.assemble_diffusion(m, bc, 1.0, src)
    return ro, co, va


def _assert_same_hierarchy(a, b):
    sizes = a.hierarchy_level_sizes()
    assert list(sizes) == list(b.hierarchy_level_sizes())
    for l in range(len(sizes)):
        x, y = a.export_level(l), b.export_level(l)
        for k in ("row_offsets", "columns", "values", "inv_diag", "p_offsets", "p_columns", "p_values", "aggregate"):
            if x.get(k) is None:
                assert y.get(k) is None, (l, k)
            else:
                assert np.array_equal(x[k], y[k]), (l, k)
    assert a.omega == b.omega


@pytest.mark.parametrize("case", ["tet10", "hex16", "boundary_layer", "neumann"])
def test_device_galerkin_setup_equals_host_setup(ctx, oracle, case):
    ro, co, va = _system(oracle, case)
    opts = {"constant_null_space": 1} if case == "neumann" else {}
    dev = cg.NativeBoomerAMGPreconditioner(ctx, **opts)
    assert dev.setup(cg.SparseMatrix.from_csr(ctx, ro, co, va)), dev.last_error()
    host = cg.NativeBoomerAMGPreconditioner(None, **opts)
    assert host.setup_host(ro, co, va), host.last_error()
    assert len(host.hierarchy_level_sizes()) > 2
    _assert_same_hierarchy(dev, host)


def test_refresh_through_the_device_setup_plan(ctx, oracle):
    """update_values on the device with the plan the device setup built
    (P^T adjacency, AP and C graphs, keep positions) equals the host refresh."""
    ro, co, va1 = _system(oracle, "tet10")
    _, _, va2 = _system(oracle, "tet10", seed_offset=11)
    A = cg.SparseMatrix.from_csr(ctx, ro, co, va1)
    dev = cg.NativeBoomerAMGPreconditioner(ctx)
    assert dev.setup(A)
    A2 = cg.SparseMatrix.from_csr(ctx, ro, co, va2)
    assert dev.update_values(A2)
    host = cg.NativeBoomerAMGPreconditioner(None)
    assert host.setup_host(ro, co, va1) and host.update_values_host(ro, co, va2)
    _assert_same_hierarchy(dev, host)


def test_device_setup_reproduces_the_reference_setup_at_32(ctx, oracle):
    path = GOLDEN / "tet32_hierarchy.json"
    if not path.exists():
        pytest.skip("tet32_hierarchy.json not generated")
    from oracle import ref
    gold = json.loads(path.read_text())
    m = cases.simple_mesh(32)
    g = oracle.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    r = oracle.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    A = cg.SparseMatrix.from_csr(ctx, r["row_offsets"], r["columns"], r["values"])
    dev = cg.NativeBoomerAMGPreconditioner(ctx)
    t0 = time.perf_counter()
    assert dev.setup(A), dev.last_error()
    seconds = time.perf_counter() - t0
    sizes = dev.hierarchy_level_sizes()
    assert [lv["n_rows"] for lv in gold["levels"]] == list(sizes)
    for l in range(len(sizes)):
        mine = ref.fingerprint_levels([dev.export_level(l)])[0]
        want = {k: v for k, v in gold["levels"][l].items() if k != "p_nnz"}
        assert mine == want, l
    assert float(dev.omega).hex() == gold["omega_hex"]
    print(f"device-Galerkin setup of the 32^3 x 6 tet system: {seconds:.2f} s")
