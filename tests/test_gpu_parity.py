"""GPU parity against the oracle, through the C ABI.

The checker is the plain-C restatement (oracle/cfdx_oracle.c), itself pinned
bit-for-bit to the reference by tests/test_oracle_pin.py.

Bit-exact: geometry, Poisson assembly, pressure-corrector assembly (CSR
values, b, phiHbyA, grad p), Gauss gradient, Rhie-Chow face flux, SpMV, one
FP64 V-cycle in reference summation order.  Tolerance-bound (relative L2
<= 1e-10): pressure after the full GMRES+AMG solve, and the corrected face
fluxes; the iteration count must match.  Where the reference build is present
the same solve is also compared with the reference itself.
"""
import numpy as np
import pytest

import cfdx_dev_b200 as cg
from tests import cases

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10   # pressure / face-flux parity with the FP64 oracle


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def oracle_hierarchy(oracle, amg):
    """The oracle's V-cycle on the hierarchy the library built (its host setup is
    pinned bit-exact to the reference's by the CPU tests)."""
    n = len(amg.hierarchy_level_sizes())
    return oracle.Hierarchy([amg.export_level(l) for l in range(n)], amg.omega)


@pytest.fixture(scope="module")
def tet_setup(ctx):
    m = cases.simple_mesh(10)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    return m, mesh, g, (U, rAU, aP, p, fixed, value)


@pytest.mark.parametrize("kind", ["hex", "tet", "bl"])
def test_geometry_bit_exact(ctx, oracle, kind):
    m = {"hex": lambda: cases.poisson_case(6)[0], "tet": lambda: cases.simple_mesh(6),
         "bl": lambda: cg.boundary_layer_case(8, 6, 5)}[kind]()
    mine = cg.Mesh(ctx, m).geometry()
    theirs = oracle.geometry(m)
    for k in mine:
        assert np.array_equal(mine[k], theirs[k]), k


def test_poisson_assembly_bit_exact(ctx, oracle):
    m, bc, src = cases.poisson_case(8)
    mesh = cg.Mesh(ctx, m)
    A, rhs = cg.assemble_cell_diffusion_matrix(mesh, bc, 1.0, src)
    ro, co, va, rhs_ref = oracle.assemble_diffusion(m, bc, 1.0, src)
    r2, c2, v2 = A.to_csr()
    assert np.array_equal(r2, ro) and np.array_equal(c2, co)
    assert np.array_equal(v2, va)
    assert np.array_equal(rhs, rhs_ref)


def test_pressure_assembly_bit_exact(ctx, oracle, tet_setup):
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    r = oracle.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    assert np.array_equal(ro, r["row_offsets"]) and np.array_equal(co, r["columns"])
    assert np.array_equal(va, r["values"])
    assert np.array_equal(b, r["b"])
    assert np.array_equal(phi, r["phiHbyA"])
    assert np.array_equal(grad, r["grad_p"])


@pytest.mark.parametrize("kind", ["hex", "bl", "prism"])
def test_pressure_assembly_other_cells_bit_exact(ctx, oracle, kind):
    # hexahedra take the assembly's form unrolled for six faces, the five-face
    # prisms its general form; p != 0 and a non-zero fixed value, so every
    # term is live
    m = {"hex": lambda: cases.poisson_case(7)[0], "bl": lambda: cg.boundary_layer_case(9, 7, 5),
         "prism": lambda: cases.prism_case(6, 5, 4)}[kind]()
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    cc = g["cell_centres"].reshape(3, -1)
    p1 = np.cos(2 * cc[0]) + cc[1] * cc[2]
    value1 = value.copy()
    value1[0] = -0.5
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p1, 1.1, fixed, value1)
    r = oracle.simple_assemble(m, U, rAU, p1, 1.1, fixed, value1)
    ro, co, va = A.to_csr()
    assert np.array_equal(ro, r["row_offsets"]) and np.array_equal(co, r["columns"])
    assert np.array_equal(va, r["values"])
    assert np.array_equal(b, r["b"])
    assert np.array_equal(phi, r["phiHbyA"])
    assert np.array_equal(grad, r["grad_p"])


def test_prism_pressure_solve_matches_oracle(ctx, oracle):
    # five-face cells end to end: the device setup equals the host setup, the
    # reference-order cycle is bit-identical to the oracle's, and the solve
    # matches it (the oracle's is pinned to the reference's on this system)
    m = cases.prism_case(9, 8, 7)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    amg = cg.NativeBoomerAMGPreconditioner(ctx, reference_order=1)
    assert amg.setup(A), amg.last_error()
    host = cg.NativeBoomerAMGPreconditioner(None)
    assert host.setup_host(ro, co, va)
    for l in range(len(host.hierarchy_level_sizes())):
        a, d = host.export_level(l), amg.export_level(l)
        for k in ("values", "inv_diag", "p_values"):
            assert np.array_equal(a[k], d[k]), (l, k)
    H = oracle_hierarchy(oracle, amg)
    r = np.random.default_rng(0).standard_normal(A.n)
    assert np.array_equal(amg.apply(r), H.apply(r))
    x_ref, rep_ref = oracle.solve_gmres(ro, co, va, b, H, restart=30, tolerance=1e-8)
    x, rep = cg.solve_gmres(A, b, amg=amg, restart=30, tolerance=1e-8)
    assert rep["status_name"] == "converged" and rep["iterations"] == rep_ref["iterations"]
    assert rel_l2(x, x_ref) <= REL_TOL


def test_pressure_assembly_nonzero_pressure_bit_exact(ctx, oracle, tet_setup):
    # a later corrector: p != 0, so the gradient and deferred fluxes are active
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    cc = g["cell_centres"].reshape(3, -1)
    p1 = np.sin(3 * cc[0]) + cc[1] * cc[2]
    value1 = value.copy()
    value1[0] = 0.25
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p1, 1.3, fixed, value1)
    r = oracle.simple_assemble(m, U, rAU, p1, 1.3, fixed, value1)
    assert np.array_equal(A.to_csr()[2], r["values"])
    assert np.array_equal(b, r["b"])
    assert np.array_equal(grad, r["grad_p"])
    assert np.array_equal(cg.gauss_gradient_with_boundary(mesh, p1, fixed, value1),
                          oracle.gauss_gradient(m, p1, fixed, value1))
    assert np.array_equal(cg.make_rhie_chow_mass_flux(mesh, U, rAU, p1, 1.3, fixed, value1),
                          oracle.rhie_chow_flux(m, U, rAU, p1, 1.3, fixed, value1))


def test_spmv_bit_exact(ctx, oracle, tet_setup):
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    x = np.random.default_rng(3).standard_normal(A.n)
    assert np.array_equal(A.matvec(x), oracle.spmv(ro, co, va, x))


def test_vcycle_bit_exact(ctx, oracle, tet_setup):
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    amg = cg.NativeBoomerAMGPreconditioner(ctx, reference_order=1)
    assert amg.setup(A)
    H = oracle_hierarchy(oracle, amg)
    fast = cg.NativeBoomerAMGPreconditioner(ctx)
    assert fast.setup(A)
    for seed in (0, 1):
        r = np.random.default_rng(seed).standard_normal(A.n)
        z_ref = H.apply(r)
        assert np.array_equal(amg.apply(r), z_ref)
        # cooperative row reductions on the dense coarse levels: same cycle, other summation order
        assert rel_l2(fast.apply(r), z_ref) < 1e-12


def test_poisson_solve_matches_oracle(ctx, oracle):
    m, bc, src = cases.poisson_case(12)
    mesh = cg.Mesh(ctx, m)
    A, rhs = cg.assemble_cell_diffusion_matrix(mesh, bc, 1.0, src)
    ro, co, va = A.to_csr()
    amg = cg.NativeBoomerAMGPreconditioner(ctx)
    assert amg.setup(A)
    x_ref, rep_ref = oracle.solve_gmres(ro, co, va, rhs, oracle_hierarchy(oracle, amg), restart=30, tolerance=1e-8)
    x, rep = cg.solve_linear_system(A, rhs, krylov="gmres", preconditioner="native_amg", restart=30,
                                    tolerance=1e-8)
    assert rep["status_name"] == "converged" and rep_ref["status"] == 0
    assert rep["iterations"] == rep_ref["iterations"]
    assert rel_l2(x, x_ref) <= REL_TOL
    assert rep["physical_residual_relative"] <= 1e-8


def test_pressure_solve_and_flux_match_oracle(ctx, oracle, tet_setup):
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    amg = cg.NativeBoomerAMGPreconditioner(ctx)
    assert amg.setup(A)
    x_ref, rep_ref = oracle.solve_gmres(ro, co, va, b, oracle_hierarchy(oracle, amg), restart=30, tolerance=1e-8)
    x, rep = cg.solve_linear_system(A, b, restart=30, tolerance=1e-8)
    assert rep["iterations"] == rep_ref["iterations"]
    assert rel_l2(x, x_ref) <= REL_TOL
    flux = cg.make_rhie_chow_mass_flux(mesh, U, rAU, x, 1.0, fixed, value)
    flux_ref = oracle.rhie_chow_flux(m, U, rAU, x_ref, 1.0, fixed, value)
    assert rel_l2(flux, flux_ref) <= REL_TOL


def test_prepared_gmres_matches_oracle(ctx, oracle, tet_setup):
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    amg = cg.NativeBoomerAMGPreconditioner(ctx)
    assert amg.setup(A)
    x_ref, rep_ref = oracle.solve_gmres(ro, co, va, b, oracle_hierarchy(oracle, amg), restart=30, tolerance=1e-8)
    x, rep = cg.solve_gmres(A, b, amg=amg, restart=30, tolerance=1e-8)
    assert rep["status_name"] == "converged"
    assert rep["iterations"] == rep_ref["iterations"]
    assert rel_l2(x, x_ref) <= REL_TOL


def test_golden_fixture_solve(ctx):
    # the reference's own outputs for the 4^3 x 6 tet system (tests/golden/)
    from pathlib import Path
    z = dict(np.load(Path(__file__).resolve().parent / "golden" / "pressure_tet4.npz"))
    m = cases.simple_mesh(int(z["n"]))
    mesh = cg.Mesh(ctx, m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, mesh.geometry()["cell_centres"])
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    assert np.array_equal(A.to_csr()[2], z["values"]) and np.array_equal(b, z["b"])
    x, rep = cg.solve_linear_system(A, b, restart=30, tolerance=1e-8)
    assert rep["iterations"] == int(z["iterations"])
    assert rel_l2(x, z["x"]) <= REL_TOL
    assert rel_l2(cg.make_rhie_chow_mass_flux(mesh, U, rAU, x, 1.0, fixed, value), z["flux_solved"]) <= REL_TOL


def test_pressure_solve_matches_reference_build(ctx, ref, tet_setup):
    # the reference's own solve_linear_system (setup + GMRES), where its build is present
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    x_ref, rep_ref = ref.solve_linear_system(ro, co, va, b, restart=30, tolerance=1e-8)
    x, rep = cg.solve_linear_system(A, b, restart=30, tolerance=1e-8)
    assert rep["iterations"] == rep_ref["iterations"]
    assert rel_l2(x, x_ref) <= REL_TOL


def test_poisson_hex32_end_to_end_matches_reference(ctx, ref):
    # The 32^3 hex Poisson benchmark system (32,768 cells) through the
    # reference's own assemble_cell_diffusion_matrix and solve_linear_system
    # (linear_solver_dispatch.h:227; its AMG setup included) against the GPU
    # path end to end: the same matrix bit for bit, the reference's hierarchy
    # level by level, the same iteration count, the pressure to 1e-10.
    m, bc, src = cases.poisson_case(32)
    mesh = cg.Mesh(ctx, m)
    A, rhs = cg.assemble_cell_diffusion_matrix(mesh, bc, 1.0, src)
    ro, co, va, rhs_ref, _ = ref.assemble_diffusion(m, bc, 1.0, src)
    for got, want in zip(A.to_csr(), (ro, co, va)):
        assert np.array_equal(got, want)
    assert np.array_equal(rhs, rhs_ref)
    x_ref, rep_ref = ref.solve_linear_system(ro, co, va, rhs_ref, restart=30, tolerance=1e-8)
    x, rep = cg.solve_linear_system(A, rhs, krylov="gmres", preconditioner="native_amg", restart=30,
                                    tolerance=1e-8)
    assert rep_ref["status"] == 0 and rep["status_name"] == "converged"
    assert rep["iterations"] == rep_ref["iterations"]
    assert rel_l2(x, x_ref) <= REL_TOL
    assert rep["physical_residual_relative"] <= 1e-8
    amg = cg.NativeBoomerAMGPreconditioner(ctx)
    assert amg.setup(A), amg.last_error()
    R = ref.Amg(ro, co, va)
    assert R.num_levels() == len(amg.hierarchy_level_sizes())
    for l in range(R.num_levels()):
        a, b = R.level(l), amg.export_level(l)
        for k in ("row_offsets", "columns", "values", "inv_diag", "p_columns", "p_values"):
            assert np.array_equal(a[k], b[k]), (l, k)
        if a["aggregate"] is not None:
            assert np.array_equal(a["aggregate"], b["aggregate"]), l
    assert R.omega == amg.omega


def test_fp32_vcycle_solve_reaches_fp64_tolerance(ctx, tet_setup):
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    x64, rep64 = cg.solve_linear_system(A, b, restart=30, tolerance=1e-8)
    x32, rep32 = cg.solve_linear_system(A, b, krylov="fgmres", restart=30, precision="fp32_vcycle", tolerance=1e-8)
    assert rep32["status_name"] == "converged"
    assert rep32["physical_residual_relative"] <= 1e-8
    assert rel_l2(x32, x64) < 1e-6
    for cs in (6, 1, 0):   # the reference's V(6,6) everywhere, the default, fine-level-only smoothing
        amg = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp32_vcycle", coarse_sweeps=cs)
        assert amg.setup(A)
        x32, rep32 = cg.solve_fgmres(A, b, amg=amg, restart=30, tolerance=1e-8)
        assert rep32["status_name"] == "converged"
        assert rep32["physical_residual_relative"] <= 1e-8
        # error against the FP64 solution is stated and small
        assert rel_l2(x32, x64) < 1e-6


@pytest.mark.parametrize("limit", [2000, 300])
def test_fp32_vcycle_fp64_dense_coarse_solve(ctx, ref, tet_setup, limit):
    # The mixed-precision configuration's FP64 coarsest-level direct solve:
    # the cycle ends at the first level with <= limit rows in a dense inverse
    # formed and applied in FP64.  Converges to the FP64 true residual, and
    # the solution agrees with the reference's own solve.
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    x_ref, rep_ref = ref.solve_linear_system(ro, co, va, b, restart=30, tolerance=1e-8)
    amg = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp32_vcycle", coarse_dense_limit=limit, dense_fp64=1)
    assert amg.setup(A)
    sizes = amg.hierarchy_level_sizes()
    assert any(s <= limit for s in sizes), sizes
    x32, rep32 = cg.solve_fgmres(A, b, amg=amg, restart=30, tolerance=1e-8, orthogonalization=1)
    assert rep32["status_name"] == "converged"
    assert rep32["physical_residual_relative"] <= 1e-8
    assert rel_l2(x32, x_ref) < 1e-6


def test_solve_is_deterministic(ctx, tet_setup):
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    x1, _ = cg.solve_linear_system(A, b, restart=30, tolerance=1e-8)
    x2, _ = cg.solve_linear_system(A, b, restart=30, tolerance=1e-8)
    assert np.array_equal(x1, x2)


def test_zero_rhs_and_invalid_requests(ctx, tet_setup):
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    x, rep = cg.solve_linear_system(A, np.zeros(A.n), restart=30, tolerance=1e-8)
    assert rep["status_name"] == "converged" and np.all(x == 0)
    with pytest.raises(cg.CfdxgError):
        cg.solve_linear_system(A, b, restart=0)
    amg = cg.NativeBoomerAMGPreconditioner(ctx)
    with pytest.raises(cg.CfdxgError):
        amg.apply(b)   # not set up


def test_device_numeric_refresh_bit_exact(ctx, oracle):
    """update_values on the device (Galerkin products, inverse diagonals,
    damping) against the host restatement, itself pinned to the reference's
    update_values by the CPU tests."""
    m = cases.simple_mesh(10)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    systems = []
    A = None
    for off in (0, 11):
        U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"], seed_offset=off)
        A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value, matrix=A)
        systems.append((A.to_csr(), b))
        if off == 0:
            dev = cg.NativeBoomerAMGPreconditioner(ctx, reference_order=1)
            assert dev.setup(A)
            dev32 = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp32_vcycle")
            assert dev32.setup(A)
    (ro, co, va1), b1 = systems[0]
    (_, _, va2), b2 = systems[1]
    host = cg.NativeBoomerAMGPreconditioner(None)
    assert host.setup_host(ro, co, va1)
    assert host.update_values_host(ro, co, va2)
    assert dev.update_values(A) and dev32.update_values(A)
    for amg in (dev, dev32):
        assert amg.omega == host.omega
        for l in range(len(host.hierarchy_level_sizes())):
            a, b = host.export_level(l), amg.export_level(l)
            for k in ("values", "inv_diag"):
                assert np.array_equal(a[k], b[k]), (l, k)
    H = oracle.Hierarchy([host.export_level(l) for l in range(len(host.hierarchy_level_sizes()))], host.omega)
    r = np.random.default_rng(9).standard_normal(A.n)
    assert np.array_equal(dev.apply(r), H.apply(r))
    x, rep = cg.solve_fgmres(A, b2, amg=dev32, restart=30, tolerance=1e-8)
    assert rep["status_name"] == "converged" and rep["physical_residual_relative"] <= 1e-8


def test_simple_outer_iterations_small(ctx):
    """Five SIMPLE outer iterations on a small anisotropic boundary-layer mesh:
    every pressure solve converges after the device numeric refresh and the
    continuity defect falls."""
    from cfdx_dev_b200 import simple_loop as sl
    m = cg.boundary_layer_case(24, 24, 8, 10.0, 1.0, 1e-4, 1.08, 0.05, sl.SEED)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    nu_t = sl.smoothed_eddy_ratio(m, sl.SEED + 2)
    for form in ("plain_fp64", "fp32_vcycle"):
        out = sl.run_form(ctx, form, m, mesh, g, nu_t, 5, 0.3, None, ctx.synchronize)
        assert all(r["status"] == "converged" for r in out["records"])
        assert out["final_continuity_l2"] < out["first_continuity_l2"]


# ---------------------------------------------------------------- CG
# CG's dots and norms are fixed-order parallel reductions here and sequential
# sums in the reference, so the iterates agree to rounding, not bit for bit.
# With AMG (8-10 iterations) the iteration count must match and the pressure
# agree to REL_TOL; the identity / Jacobi objects take hundreds of iterations,
# over which rounding differences grow, so there the count may differ by 2 and
# the pressure by CG_LONG_TOL, each solution certified to the solve tolerance.
CG_LONG_TOL = 1e-7


@pytest.mark.parametrize("pc", ["native_amg", "jacobi", "none"])
def test_cg_matches_oracle(ctx, oracle, tet_setup, pc):
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    H = None
    if pc == "native_amg":
        amg = cg.NativeBoomerAMGPreconditioner(ctx, require_smoother_certificate=True)
        assert amg.setup(A)
        H = oracle_hierarchy(oracle, amg)
    x_ref, rep_ref = oracle.solve_cg(ro, co, va, b, pc, H, max_iterations=3000, tolerance=1e-10)
    x, rep = cg.solve_linear_system(A, b, krylov="cg", preconditioner=pc, max_iterations=3000, tolerance=1e-10)
    assert rep["status_name"] == "converged" and rep_ref["status"] == 0
    assert rep["physical_residual_relative"] <= 1e-10
    if pc == "native_amg":
        assert rep["iterations"] == rep_ref["iterations"]
        assert rel_l2(x, x_ref) <= REL_TOL
    else:
        assert abs(rep["iterations"] - rep_ref["iterations"]) <= 2
        assert rel_l2(x, x_ref) <= CG_LONG_TOL


def test_prepared_cg_matches_oracle(ctx, oracle, tet_setup):
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    amg = cg.NativeBoomerAMGPreconditioner(ctx, require_smoother_certificate=True)
    assert amg.setup(A)
    x0 = np.random.default_rng(4).standard_normal(A.n) * 1e-2
    x_ref, rep_ref = oracle.solve_cg(ro, co, va, b, "native_amg", oracle_hierarchy(oracle, amg), x0=x0,
                                     tolerance=1e-10)
    x, rep = cg.solve_cg(A, b, x0=x0, amg=amg, tolerance=1e-10)
    assert rep["status_name"] == "converged"
    assert rep["iterations"] == rep_ref["iterations"]
    assert rel_l2(x, x_ref) <= REL_TOL


def test_cg_golden_fixture(ctx):
    # the reference's own CG + native AMG solve of the 4^3 x 6 tet system
    from pathlib import Path
    z = dict(np.load(Path(__file__).resolve().parent / "golden" / "pressure_tet4.npz"))
    A = cg.SparseMatrix.from_csr(ctx, z["row_offsets"], z["columns"], z["values"])
    x, rep = cg.solve_linear_system(A, z["b"], krylov="cg", max_iterations=1000, tolerance=1e-10)
    assert rep["status_name"] == "converged"
    assert rep["iterations"] == int(z["cg_iterations"])
    assert rel_l2(x, z["cg_x"]) <= REL_TOL


def test_cg_rejects_nonsymmetric_or_nonpositive_diagonal(ctx, tet_setup):
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    x0 = np.full(A.n, 0.25)
    off = next(k for k in range(ro[1]) if co[k] != 0)      # an off-diagonal entry of row 0
    skew = va.copy()
    skew[off] *= 1.5
    diag0 = next(k for k in range(ro[1]) if co[k] == 0)
    negdiag = va.copy()
    negdiag[diag0] = -negdiag[diag0]
    for bad in (skew, negdiag):
        B = cg.SparseMatrix.from_csr(ctx, ro, co, bad)
        x, rep = cg.solve_linear_system(B, b, x0=x0, krylov="cg", tolerance=1e-10)
        assert rep["status_name"] == "not_applicable"
        assert np.array_equal(x, x0)
    # the same system with symmetric coefficients is accepted
    x, rep = cg.solve_linear_system(A, b, krylov="cg", tolerance=1e-10)
    assert rep["status_name"] == "converged"
    with pytest.raises(cg.CfdxgError):
        cg.solve_linear_system(A, b, krylov="cg", learned=cg.LearnedPreconditioner(ctx))


# ---------------------------------------------------------------- .cfdxlin replay
def test_capture_replay_matches_reference_solution(ctx, tmp_path):
    """A pressure system written by the reference's write_linear_system_capture
    replays through the library: same CSR and right-hand side, and the solve
    with the file's tolerance and iteration limit reproduces the reference's
    solution and iteration count.  The library's own opt-in capture of the
    same solve is byte-identical to the reference's file."""
    from pathlib import Path
    golden = Path(__file__).resolve().parent / "golden"
    c = cg.read_linear_system_capture(golden / "pressure_tet4.cfdxlin")
    z = dict(np.load(golden / "pressure_tet4.npz"))
    A = cg.SparseMatrix.from_csr(ctx, c["row_offsets"], c["columns"], c["values"])
    path = tmp_path / "replay.cfdxlin"
    x, rep = cg.solve_linear_system(A, c["rhs"], c["initial_solution"], restart=30,
                                    max_iterations=c["max_iterations"], tolerance=c["tolerance"],
                                    linear_capture_path=str(path))
    assert rep["status_name"] == "converged"
    assert rep["iterations"] == int(z["iterations"])
    assert rel_l2(x, z["x"]) <= REL_TOL
    assert path.read_bytes() == (golden / "pressure_tet4.cfdxlin").read_bytes()


# ---------------------------------------------------------------- CGS2 option
def test_classical_gram_schmidt_matches_oracle(ctx, oracle, tet_setup):
    """orthogonalization = CGS2 forms the same projections as the reference's
    two-pass MGS with different rounding: the FP64 AMG-GMRES iterate agrees
    with the oracle's to REL_TOL at the same iteration count, and the FP32
    V-cycle FGMRES still reaches the FP64 certificate."""
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    amg = cg.NativeBoomerAMGPreconditioner(ctx)
    assert amg.setup(A)
    x_ref, rep_ref = oracle.solve_gmres(ro, co, va, b, oracle_hierarchy(oracle, amg), restart=30, tolerance=1e-8)
    x, rep = cg.solve_gmres(A, b, amg=amg, restart=30, tolerance=1e-8, orthogonalization=1)
    assert rep["status_name"] == "converged"
    assert rep["iterations"] == rep_ref["iterations"]
    assert rel_l2(x, x_ref) <= REL_TOL
    amg32 = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp32_vcycle")
    assert amg32.setup(A)
    x_m, rep_m = cg.solve_fgmres(A, b, amg=amg32, restart=30, tolerance=1e-8)
    x_c, rep_c = cg.solve_fgmres(A, b, amg=amg32, restart=30, tolerance=1e-8, orthogonalization=1)
    assert rep_c["status_name"] == "converged" and rep_c["physical_residual_relative"] <= 1e-8
    assert abs(rep_c["iterations"] - rep_m["iterations"]) <= 1
    assert rel_l2(x_c, x_ref) < 1e-6
    # Arnoldi cycles longer than one 16-vector chunk: Jacobi-preconditioned GMRES(40)
    kw = dict(krylov="gmres", preconditioner="jacobi", restart=40, tolerance=1e-8, max_iterations=4000)
    x0, rep0 = cg.solve_linear_system(A, b, **kw)
    x1, rep1 = cg.solve_linear_system(A, b, orthogonalization=1, **kw)
    assert rep1["status_name"] == rep0["status_name"] == "converged"
    assert rep0["iterations"] > 40
    assert abs(rep1["iterations"] - rep0["iterations"]) <= max(2, 0.05 * rep0["iterations"])
    assert rel_l2(x1, x0) < 1e-6
    with pytest.raises(cg.CfdxgError):
        cg.solve_gmres(A, b, amg=amg, orthogonalization=7)


# ---------------------------------------------------------------- FP16 level values
def test_half_values_fp32_vcycle(ctx, tet_setup):
    """half_values = 1 stores each level's rows as FP16 fractions of the row's
    largest magnitude: the FP32 V-cycle stays within 1e-2 of the FP32-value
    cycle, FGMRES reaches the FP64 certificate within one extra iteration, and
    after a numeric refresh on the device (which quantises the new values on
    the device) the cycle again stays within 1e-2 of the refreshed FP32-value
    cycle and FGMRES converges."""
    m, mesh, g, (U, rAU, aP, p, fixed, value) = tet_setup
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    full = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp32_vcycle", half_values=0)
    half = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp32_vcycle", half_values=1)
    assert full.setup(A) and half.setup(A)
    r = np.random.default_rng(3).standard_normal(A.n)
    z_full, z_half = full.apply(r), half.apply(r)
    assert rel_l2(z_half, z_full) < 1e-2
    x_f, rep_f = cg.solve_fgmres(A, b, amg=full, restart=30, tolerance=1e-8)
    x_h, rep_h = cg.solve_fgmres(A, b, amg=half, restart=30, tolerance=1e-8)
    assert rep_h["status_name"] == "converged" and rep_h["physical_residual_relative"] <= 1e-8
    assert rep_h["iterations"] <= rep_f["iterations"] + 1
    assert rel_l2(x_h, x_f) < 1e-6
    # numeric refresh on the device: the same values quantised on the device
    U2, rAU2, aP2, p2, fixed2, value2 = cases.simple_fields(m, g["cell_centres"], seed_offset=11)
    A2, b2, _, _ = cg.assemble_pressure_correction(mesh, U2, rAU2, p2, 1.0, fixed2, value2)
    assert half.update_values(A2) and full.update_values(A2)
    assert rel_l2(half.apply(r), full.apply(r)) < 1e-2
    x2, rep2 = cg.solve_fgmres(A2, b2, amg=half, restart=30, tolerance=1e-8)
    assert rep2["status_name"] == "converged" and rep2["physical_residual_relative"] <= 1e-8


# ---------------------------------------------------------------- pure-Neumann gauge
def test_pure_neumann_gauge_matches_oracle(ctx, oracle):
    """Every patch zero-gradient: the corrector's reference-cell elimination
    (steady_incompressible_solver.h:8617-8654) and apply_reference_cell_gauge
    (scalar_diffusion.h:177-210) on the device equal the oracle's bit for bit,
    twice on one plan (the second time with new values); the eliminated
    system's AMG-GMRES solve and its expansion match the oracle's."""
    m = cases.simple_mesh(8)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    ref_cell = 37
    gauge = ident = None
    A = None
    for off in (0, 5):
        U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"], seed_offset=off)
        fixed[:] = 0
        A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value, matrix=A)
        ro, co, va = A.to_csr()
        if gauge is None:
            gauge = cg.ReferenceCellGauge(ctx, A, ref=ref_cell)
            ident = cg.ReferenceCellGauge(ctx, A, ref=ref_cell, mode="identity_row", value=0.5)
        B, bB = gauge.apply(A, b)
        expect = oracle.gauge_eliminate(ro, co, va, b, ref_cell)
        for got, want in zip(B.to_csr() + (bB,), expect):
            assert np.array_equal(got, want)
        C, bC = ident.apply(A, b)
        expect = oracle.gauge_identity_row(ro, co, va, b, ref_cell, 0.5)
        for got, want in zip(C.to_csr() + (bC,), expect):
            assert np.array_equal(got, want)
    amg = cg.NativeBoomerAMGPreconditioner(ctx)
    assert amg.setup(B)
    e_ro, e_co, e_va, e_b = expect_elim = oracle.gauge_eliminate(ro, co, va, b, ref_cell)
    x_ref, rep_ref = oracle.solve_gmres(e_ro, e_co, e_va, e_b, oracle_hierarchy(oracle, amg), restart=30,
                                        tolerance=1e-8)
    xr, rep = cg.solve_gmres(B, bB, amg=amg, restart=30, tolerance=1e-8)
    assert rep["status_name"] == "converged" and rep["iterations"] == rep_ref["iterations"]
    assert rel_l2(xr, x_ref) <= REL_TOL
    x = gauge.expand(xr)
    assert x[ref_cell] == 0.0 and np.array_equal(x, oracle.gauge_expand(xr, ref_cell))
    # the full system is satisfied on every row but the reference cell's
    res = b - oracle.spmv(ro, co, va, x)
    assert np.linalg.norm(np.delete(res, ref_cell)) <= 1e-8 * np.linalg.norm(np.delete(b, ref_cell)) * 1.0001
    with pytest.raises(cg.CfdxgError):
        cg.ReferenceCellGauge(ctx, A, ref=A.n)


# ---------------------------------------------------------------- Poisson driver
@pytest.mark.parametrize("kind", ["dirichlet", "neumann"])
def test_poisson_driver_matches_oracle(ctx, oracle, kind):
    """solve_poisson_mixed (scalar_diffusion.h:294-340) on the device against
    the oracle's composition, itself bit-identical to the reference's driver:
    the apps/poisson case and a pure-Neumann case with the reference-cell
    gauge.  The own-diagonal CG takes tens of iterations with parallel dots, so
    the count may differ by 2 and the solution by CG_LONG_TOL; each solve is
    certified to its 1e-10 residual."""
    from tests.test_poisson_driver import apps_poisson_case, neumann_case, oracle_poisson_mixed
    if kind == "dirichlet":
        m, bc, src = apps_poisson_case(8)
        types, cell, value = None, 0, 0.0
    else:
        m, bc, src, types = neumann_case(8)
        cell, value = 11, 1.5
    x_ref, rep_ref = oracle_poisson_mixed(m, bc, src, types, ref_cell=cell, ref_value=value)
    mesh = cg.Mesh(ctx, m)
    out = cg.solve_poisson_mixed(mesh, bc, src, types, reference_cell=cell, reference_value=value)
    rep = out["report"]
    assert rep["status_name"] == "converged" and rep_ref["status"] == 0
    assert rep["physical_residual_relative"] <= 1e-10
    assert abs(rep["iterations"] - rep_ref["iterations"]) <= 2
    assert rel_l2(out["solution"], x_ref) <= CG_LONG_TOL
    if kind == "neumann":
        assert out["solution"][cell] == value
        with pytest.raises(ValueError):
            cg.solve_poisson_mixed(mesh, bc, src + 1.0, types)
