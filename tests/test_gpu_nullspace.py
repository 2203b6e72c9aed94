"""The constant null space on the GPU (NullSpaceModel::Constant) against the
oracle, itself pinned bit for bit to the reference's solve_linear_system by
tests/test_oracle_pin.py.

* The native AMG's constant-null-space cycle: bit-identical to the oracle's in
  reference order (means summed in index order), for a hierarchy ending in
  the bordered dense LU and for one ending in 24 damped-Jacobi sweeps; within
  1e-12 with the default fixed-order tree sums.
* solve_projected_gmres (GMRES, FGMRES) and the projected CG through
  cfdxg_solve_linear_system: the oracle's iteration count and pressure to
  1e-10 (Jacobi / identity CG: +-2 iterations and 1e-7, the reductions'
  order, as for the ordinary CG); the unprojected physical residual certifies.
* Refusals: an incompatible right-hand side, an operator without the null
  space, CG's smoother certificate on a singular coarsest level --
  NOT_APPLICABLE with x untouched, as the reference; null space + scaling is
  an invalid request.
* The FP32 cycle with the bordered dense coarse inverse.
"""
import numpy as np
import pytest

import cfdx_dev_b200 as cg
from tests import cases

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10
CG_LONG_TOL = 1e-7


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def oracle_hierarchy(oracle, amg):
    n = len(amg.hierarchy_level_sizes())
    return oracle.Hierarchy([amg.export_level(l) for l in range(n)], amg.omega, constant_null_space=True)


@pytest.fixture(scope="module")
def neumann_tet(ctx):
    """The pressure-correction system of 8^3 x 6 Kuhn tets with no fixed-pressure
    patch, and its right-hand side less its mean."""
    m = cases.simple_mesh(8)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, np.zeros_like(fixed), value)
    return mesh, A, b - b.mean()


@pytest.fixture(scope="module")
def neumann_hex(ctx, oracle):
    """All-Neumann 10^3 hex Poisson (its one-row coarsest level is singular)."""
    m = cg.hex_case(10)
    ro, co, va, rhs = oracle.assemble_diffusion(m, np.full(m.n_faces, np.nan), 1.0,
                                                cg.random_field(m.n_cells, "uniform", -1.0, 1.0, 7))
    return cg.SparseMatrix.from_csr(ctx, ro, co, va), rhs - rhs.mean()


@pytest.mark.parametrize("case", ["tet_bordered_lu", "hex_swept_coarsest"])
def test_null_space_vcycle_bit_exact(ctx, oracle, neumann_tet, neumann_hex, case):
    A = neumann_tet[1] if case == "tet_bordered_lu" else neumann_hex[0]
    opts = dict(reference_order=1, constant_null_space=1)
    if case == "hex_swept_coarsest":
        opts["max_levels"] = 4   # the cycle ends at a 52-row level: 24 sweeps, each mean-removed
    amg = cg.NativeBoomerAMGPreconditioner(ctx, **opts)
    assert amg.setup(A), amg.last_error()
    sizes = amg.hierarchy_level_sizes()
    assert (sizes[-1] <= 16) == (case == "tet_bordered_lu")
    H = oracle_hierarchy(oracle, amg)
    for seed in (0, 1):
        r = np.random.default_rng(seed).standard_normal(A.n)
        assert np.array_equal(amg.apply(r), H.apply(r))
    # the default fixed-order tree sums: the same cycle to rounding
    fast = cg.NativeBoomerAMGPreconditioner(ctx, **{k: v for k, v in opts.items() if k != "reference_order"})
    assert fast.setup(A)
    r = np.random.default_rng(2).standard_normal(A.n)
    z = fast.apply(r)
    assert rel_l2(z, H.apply(r)) <= 1e-12
    assert abs(z.sum()) <= 1e-12 * np.abs(z).sum()


@pytest.mark.parametrize("krylov", ["fgmres", "gmres"])
def test_projected_gmres_matches_oracle(ctx, oracle, neumann_tet, krylov):
    mesh, A, b = neumann_tet
    ro, co, va = A.to_csr()
    amg = cg.NativeBoomerAMGPreconditioner(ctx, constant_null_space=1)
    assert amg.setup(A)
    x_ref, rep_ref = oracle.solve_projected_gmres(ro, co, va, b, oracle_hierarchy(oracle, amg), restart=30,
                                                  tolerance=1e-8)
    x0 = np.full(A.n, 0.3)   # a gauge the solve removes
    x, rep = cg.solve_linear_system(A, b, x0=x0, krylov=krylov, restart=30, tolerance=1e-8,
                                    null_space="constant")
    assert rep_ref["status"] == 0 and rep["status_name"] == "converged"
    assert rep["iterations"] == rep_ref["iterations"]
    assert rel_l2(x, x_ref) <= REL_TOL
    assert rep["physical_residual_relative"] <= 1e-8
    assert abs(x.sum()) <= 1e-10 * np.abs(x).sum()
    # the prepared form (solve_gmres with the hierarchy, no setup inside)
    xp, repp = cg.solve_gmres(A, b, x0=x0, amg=amg, restart=30, tolerance=1e-8, krylov=krylov,
                              null_space="constant")
    assert repp["iterations"] == rep_ref["iterations"] and rel_l2(xp, x_ref) <= REL_TOL


@pytest.mark.parametrize("pc", ["native_amg", "jacobi", "none"])
def test_projected_cg_matches_oracle(ctx, oracle, neumann_tet, pc):
    mesh, A, b = neumann_tet
    ro, co, va = A.to_csr()
    H = None
    if pc == "native_amg":
        amg = cg.NativeBoomerAMGPreconditioner(ctx, require_smoother_certificate=True, constant_null_space=1)
        assert amg.setup(A), amg.last_error()
        H = oracle_hierarchy(oracle, amg)
    x_ref, rep_ref = oracle.solve_cg(ro, co, va, b, pc, H, max_iterations=3000, tolerance=1e-10, null_space=True)
    x, rep = cg.solve_linear_system(A, b, krylov="cg", preconditioner=pc, max_iterations=3000, tolerance=1e-10,
                                    null_space="constant")
    assert rep_ref["status"] == 0 and rep["status_name"] == "converged"
    assert rep["physical_residual_relative"] <= 1e-10
    if pc == "native_amg":
        assert rep["iterations"] == rep_ref["iterations"]
        assert rel_l2(x, x_ref) <= REL_TOL
    else:
        assert abs(rep["iterations"] - rep_ref["iterations"]) <= 2
        assert rel_l2(x, x_ref) <= CG_LONG_TOL


def test_null_space_refusals(ctx, oracle, neumann_tet, neumann_hex):
    mesh, A, b = neumann_tet
    x0 = np.full(A.n, 0.25)
    # an incompatible right-hand side: NOT_APPLICABLE, x untouched
    for krylov in ("fgmres", "cg"):
        x, rep = cg.solve_linear_system(A, b + 1.0, x0=x0, krylov=krylov, tolerance=1e-8, null_space="constant")
        assert rep["status_name"] == "not_applicable" and np.array_equal(x, x0)
    # an operator without the constant null space (p fixed on one patch)
    m = cases.simple_mesh(8)
    g = mesh.geometry()
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    Ad, bd, _, _ = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    x, rep = cg.solve_linear_system(Ad, bd - bd.mean(), x0=x0, krylov="fgmres", tolerance=1e-8,
                                    null_space="constant")
    assert rep["status_name"] == "not_applicable" and np.array_equal(x, x0)
    # CG's AMG keeps the smoother certificate, which the hex system's singular
    # one-row coarsest level fails (the reference's solve is NOT_APPLICABLE too)
    Ah, bh = neumann_hex
    x, rep = cg.solve_linear_system(Ah, bh, krylov="cg", tolerance=1e-8, null_space="constant")
    assert rep["status_name"] == "not_applicable"
    # GMRES has no certificate: the same system solves
    x, rep = cg.solve_linear_system(Ah, bh, krylov="fgmres", restart=30, tolerance=1e-8, null_space="constant")
    assert rep["status_name"] == "converged"
    # scaling is not combined with a projected null space
    with pytest.raises(cg.CfdxgError):
        cg.solve_linear_system(A, b, krylov="fgmres", scaling="row", null_space="constant")


def test_fp32_cycle_with_bordered_dense_inverse(ctx, neumann_tet):
    mesh, A, b = neumann_tet
    # the whole fine level (3,072 rows) under the dense limit: the cycle is the
    # bordered inverse itself (stored FP32), so FGMRES needs a few iterations
    x, rep = cg.solve_linear_system(A, b, krylov="fgmres", precision="fp32_vcycle", restart=30, tolerance=1e-8,
                                    null_space="constant")
    assert rep["status_name"] == "converged" and rep["iterations"] <= 3
    assert rep["physical_residual_relative"] <= 1e-8
    # a multilevel FP32 cycle ending in a bordered dense level of <= 100 rows
    amg = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp32_vcycle", coarse_dense_limit=100,
                                           constant_null_space=1)
    assert amg.setup(A)
    z = amg.apply(np.random.default_rng(3).standard_normal(A.n))
    assert abs(z.sum()) <= 1e-5 * np.abs(z).sum()
    x, rep = cg.solve_fgmres(A, b, amg=amg, restart=30, tolerance=1e-8, null_space="constant")
    assert rep["status_name"] == "converged" and rep["physical_residual_relative"] <= 1e-8
