"""Pins the plain-C oracle (oracle/cfdx_oracle.c) to the reference itself.

No GPU: the restatement must reproduce, bit for bit, what the reference's
own code (compiled from its sources into oracle/_ref) computes -- geometry,
Gauss gradient, pressure-corrector assembly, Rhie-Chow face flux, Poisson
assembly, SpMV, one V-cycle on the reference's own hierarchy and a whole
AMG-GMRES solve -- and, without the reference tree, the committed golden
fixtures of tests/golden/ (made by tests/golden/make_golden.py from the
reference build).
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import cfdx_oracle as co
from tests import cases

GOLDEN = Path(__file__).resolve().parent / "golden"


def _pressure_inputs(n, seed_offset=0):
    m = cases.simple_mesh(n, seed_offset=seed_offset)
    g = co.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"], seed_offset=seed_offset)
    return m, g, U, rAU, p, fixed, value


@pytest.mark.parametrize("kind", ["hex", "tet", "bl", "prism"])
def test_geometry_matches_reference(ref, kind):
    import cfdx_dev_b200 as cg
    m = {"hex": lambda: cases.poisson_case(5)[0], "tet": lambda: cases.simple_mesh(5),
         "bl": lambda: cg.boundary_layer_case(6, 5, 4), "prism": lambda: cases.prism_case(4, 3, 3)}[kind]()
    mine = co.geometry(m)
    for which in ("fv", "cache"):   # build_fv_geometry and compute_geometry_cache agree
        theirs = ref.geometry(m, which)
        for k in mine:
            assert np.array_equal(mine[k], theirs[k]), (which, k)


@pytest.mark.parametrize("nonzero_p", [False, True])
def test_pressure_assembly_and_flux_match_reference(ref, nonzero_p):
    m, g, U, rAU, p, fixed, value = _pressure_inputs(6)
    rho = 1.0
    if nonzero_p:
        cc = g["cell_centres"].reshape(3, -1)
        p = np.sin(3 * cc[0]) + cc[1] * cc[2]
        value = value.copy()
        value[0] = 0.25
        rho = 1.3
    a = co.simple_assemble(m, U, rAU, p, rho, fixed, value)
    b = ref.simple_assemble(m, U, rAU, p, rho, fixed, value)
    for k in ("row_offsets", "columns", "values", "b", "phiHbyA", "grad_p"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(co.gauss_gradient(m, p, fixed, value), ref.gauss_gradient(m, p, fixed, value))
    assert np.array_equal(co.rhie_chow_flux(m, U, rAU, p, rho, fixed, value),
                          ref.rhie_chow_flux(m, U, rAU, p, rho, fixed, value))


@pytest.mark.parametrize("kind", ["hex", "prism"])
def test_pressure_assembly_on_other_cells_matches_reference(ref, kind):
    # six- and five-face cells (the GPU assembly's unrolled and general forms)
    m = cases.poisson_case(5)[0] if kind == "hex" else cases.prism_case(4, 3, 3)
    g = co.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    cc = g["cell_centres"].reshape(3, -1)
    p = np.cos(2 * cc[0]) + cc[1] * cc[2]
    value = value.copy()
    value[0] = -0.5
    a = co.simple_assemble(m, U, rAU, p, 1.1, fixed, value)
    b = ref.simple_assemble(m, U, rAU, p, 1.1, fixed, value)
    for k in ("row_offsets", "columns", "values", "b", "phiHbyA", "grad_p"):
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(co.rhie_chow_flux(m, U, rAU, p, 1.1, fixed, value),
                          ref.rhie_chow_flux(m, U, rAU, p, 1.1, fixed, value))


def test_poisson_assembly_matches_reference(ref):
    m, bc, src = cases.poisson_case(6)
    ro, co_, va, rhs = co.assemble_diffusion(m, bc, 1.0, src)
    r_ro, r_co, r_va, r_rhs, _ = ref.assemble_diffusion(m, bc, 1.0, src)
    assert np.array_equal(ro, r_ro) and np.array_equal(co_, r_co)
    assert np.array_equal(va, r_va) and np.array_equal(rhs, r_rhs)


@pytest.mark.parametrize("mesh", ["tet", "prism"])
def test_spmv_vcycle_and_solve_match_reference(ref, mesh):
    if mesh == "tet":
        m, g, U, rAU, p, fixed, value = _pressure_inputs(7)
    else:   # five-face cells
        m = cases.prism_case(9, 8, 7)
        g = co.geometry(m)
        U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    A = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    ro, cols, va, b = A["row_offsets"], A["columns"], A["values"], A["b"]
    x = np.random.default_rng(5).standard_normal(ro.size - 1)
    assert np.array_equal(co.spmv(ro, cols, va, x), ref.spmv(ro, cols, va, x))
    R = ref.Amg(ro, cols, va)
    H = co.Hierarchy([R.level(l) for l in range(R.num_levels())], R.omega)
    for seed in (0, 1):
        r = np.random.default_rng(seed).standard_normal(ro.size - 1)
        assert np.array_equal(H.apply(r), R.apply(r))
    x_ref, rep_ref = R.solve_gmres(b, restart=30, tolerance=1e-8)
    x_co, rep_co = co.solve_gmres(ro, cols, va, b, H, restart=30, tolerance=1e-8)
    assert rep_co["status"] == rep_ref["status"] == 0
    assert rep_co["iterations"] == rep_ref["iterations"]
    assert np.array_equal(x_co, x_ref)


@pytest.mark.parametrize("pc", ["native_amg", "jacobi", "none", "internal_jacobi"])
def test_cg_matches_reference(ref, pc):
    """CG (cg_solver.h:45-560) with each preconditioner object the dispatch
    builds (solve_linear_system, KrylovModel::CG) and with the solver's own
    diagonal (the legacy solve_cg overload): iterate and count bit-identical."""
    m, g, U, rAU, p, fixed, value = _pressure_inputs(7)
    A = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    ro, cols, va, b = A["row_offsets"], A["columns"], A["values"], A["b"]
    x0 = np.random.default_rng(9).standard_normal(b.size) * 1e-2
    if pc == "internal_jacobi":
        x_ref, rep_ref = ref.solve_cg_internal(ro, cols, va, b, x0=x0, max_iterations=2000, tolerance=1e-10)
        H = None
    else:
        x_ref, rep_ref = ref.solve_linear_system(ro, cols, va, b, x0=x0, krylov=1,
                                                 preconditioner={"native_amg": 6, "jacobi": 2, "none": 1}[pc],
                                                 max_iterations=2000, tolerance=1e-10)
        R = ref.Amg(ro, cols, va) if pc == "native_amg" else None
        H = co.Hierarchy([R.level(l) for l in range(R.num_levels())], R.omega) if R else None
    x_co, rep_co = co.solve_cg(ro, cols, va, b, pc, H, x0=x0, max_iterations=2000, tolerance=1e-10)
    assert rep_co["status"] == rep_ref["status"] == 0
    assert rep_co["iterations"] == rep_ref["iterations"]
    assert np.array_equal(x_co, x_ref)


def test_cg_edge_cases():
    ro = np.array([0, 2, 5, 7], np.int64)
    cols = np.array([0, 1, 0, 1, 2, 1, 2], np.int64)
    vals = np.array([4.0, 1.0, 1.0, 3.0, 1.0, 1.0, 2.0])
    # SPD 3x3: CG is exact in at most 3 steps
    x, rep = co.solve_cg(ro, cols, vals, np.array([1.0, 2.0, 3.0]), "jacobi", max_iterations=10, tolerance=1e-13)
    A = np.array([[4.0, 1.0, 0.0], [1.0, 3.0, 1.0], [0.0, 1.0, 2.0]])
    assert rep["status"] == 0 and rep["iterations"] <= 3
    assert np.allclose(A @ x, [1.0, 2.0, 3.0], rtol=0, atol=1e-12)
    # b = 0, x0 = 0: converged before any preconditioner work
    x, rep = co.solve_cg(ro, cols, vals, np.zeros(3), "none")
    assert rep["status"] == 0 and rep["iterations"] == 0 and rep["preconditioner_applications"] == 0
    # a non-positive diagonal: the solver's own Jacobi scaling is not applicable
    x, rep = co.solve_cg(ro, cols, -vals, np.ones(3), "internal_jacobi")
    assert rep["status"] == 3
    # an indefinite operator: non-positive curvature -> not applicable
    x, rep = co.solve_cg(ro, cols, np.array([1.0, 2.0, 2.0, 1.0, 0.0, 0.0, 1.0]), np.array([1.0, -1.0, 0.0]),
                         "none", max_iterations=10)
    assert rep["status"] == 3
    # non-finite input: diverged
    bad = vals.copy()
    bad[3] = np.nan
    assert co.solve_cg(ro, cols, bad, np.ones(3), "none")[1]["status"] == 2


def test_small_dense_coarsest_and_unpreconditioned_gmres(ref):
    # 1-D Poisson (known-answer shape of the reference's GMRES tests): the
    # hierarchy ends in a <= 16-row level, so the dense pivoted LU runs.
    n = 40
    rows, cols, vals = [], [], []
    for i in range(n):
        for j, v in ((i - 1, -1.0), (i, 2.0), (i + 1, -1.0)):
            if 0 <= j < n:
                rows.append(i); cols.append(j); vals.append(v)
    cols = np.array(cols, np.int64)
    vals = np.array(vals)
    ro = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int64)
    b = np.ones(n)
    R = ref.Amg(ro, cols, vals)
    levels = [R.level(l) for l in range(R.num_levels())]
    assert levels[-1]["inv_diag"].size <= 16
    H = co.Hierarchy(levels, R.omega)
    r = np.random.default_rng(2).standard_normal(n)
    assert np.array_equal(H.apply(r), R.apply(r))
    x_co, rep = co.solve_gmres(ro, cols, vals, b, None, restart=30, tolerance=1e-10, max_iterations=200)
    assert rep["status"] == 0
    exact = np.array([(i + 1) * (n - i) / 2.0 for i in range(n)])
    assert np.linalg.norm(x_co - exact) / np.linalg.norm(exact) < 1e-8


def test_exact_3x3_gmres():
    # the reference's exact 3x3 GMRES test shape: GMRES(3) is exact in 3 steps
    ro = np.array([0, 2, 5, 7], np.int64)
    cols = np.array([0, 1, 0, 1, 2, 1, 2], np.int64)
    vals = np.array([4.0, 1.0, 1.0, 3.0, 1.0, 1.0, 2.0])
    b = np.array([1.0, 2.0, 3.0])
    x, rep = co.solve_gmres(ro, cols, vals, b, None, restart=3, tolerance=1e-12, max_iterations=10)
    A = np.array([[4.0, 1.0, 0.0], [1.0, 3.0, 1.0], [0.0, 1.0, 2.0]])
    assert rep["status"] == 0 and rep["iterations"] <= 3
    assert np.allclose(A @ x, b, rtol=0, atol=1e-12)


def test_zero_rhs_shifted_solve():
    ro = np.array([0, 2, 5, 7], np.int64)
    cols = np.array([0, 1, 0, 1, 2, 1, 2], np.int64)
    vals = np.array([4.0, 1.0, 1.0, 3.0, 1.0, 1.0, 2.0])
    x, rep = co.solve_gmres(ro, cols, vals, np.zeros(3), None, x0=np.array([1.0, -2.0, 0.5]), restart=3,
                            tolerance=1e-12, max_iterations=10)
    assert rep["status"] == 0
    assert np.abs(x).max() < 1e-10


def test_invalid_inputs_fail_loudly():
    m = cases.simple_mesh(2)
    bad = cases.simple_mesh(2)
    bad.face_offsets = bad.face_offsets.copy()
    bad.face_offsets[1] = bad.face_offsets[0] + 2   # a two-vertex face
    with pytest.raises(RuntimeError):
        co.geometry(bad)
    x, rep = co.solve_gmres(np.array([0, 1], np.int64), np.array([0], np.int64), np.array([1.0]), np.ones(1),
                            restart=0)
    assert rep["status"] == 3
    assert co.geometry(m)["cell_volumes"].min() > 0


def _golden_levels(z):
    levels = []
    for l in range(int(z["n_levels"])):
        lv = {k: z[f"L{l}_{k}"] for k in ("row_offsets", "columns", "values", "inv_diag")}
        if f"L{l}_p_offsets" in z:
            lv.update({k: z[f"L{l}_{k}"] for k in ("p_offsets", "p_columns", "p_values")})
        levels.append(lv)
    return levels


def _neumann_pressure(n):
    """The pressure-correction system without a fixed-pressure patch (a
    constant null space), its right-hand side less its mean."""
    m, g, U, rAU, p, fixed, value = _pressure_inputs(n)
    a = co.simple_assemble(m, U, rAU, p, 1.0, np.zeros_like(fixed), value)
    return a["row_offsets"], a["columns"], a["values"], a["b"] - a["b"].mean()


def _neumann_poisson(n):
    import cfdx_dev_b200 as cg
    m = cg.hex_case(n)
    ro, cols, va, rhs = co.assemble_diffusion(m, np.full(m.n_faces, np.nan), 1.0,
                                              cg.random_field(m.n_cells, "uniform", -1.0, 1.0, 7))
    return ro, cols, va, rhs - rhs.mean()


@pytest.mark.parametrize("case", ["tet6", "tet8", "hex10"])
def test_null_space_solves_match_reference(ref, case):
    """NullSpaceModel::Constant (linear_solver_dispatch.h:354-400): the native
    AMG's constant-null-space cycle (mean removals, bordered coarsest LU),
    solve_projected_gmres for FGMRES and GMRES, and the projected CG with each
    preconditioner object -- iterate and count bit-identical to the reference's
    solve_linear_system."""
    ro, cols, va, b = _neumann_poisson(10) if case == "hex10" else _neumann_pressure(int(case[3:]))
    assert co.null_space_checks(ro, cols, va, b) == (True, True, True)
    R = ref.Amg(ro, cols, va, constant_null_space=True)
    H = co.Hierarchy([R.level(l) for l in range(R.num_levels())], R.omega, constant_null_space=True)
    assert H.n_rows[-1] <= 16
    for seed in (0, 1):
        r = np.random.default_rng(seed).standard_normal(b.size)
        assert np.array_equal(H.apply(r), R.apply(r))
    for krylov in (4, 3):   # FGMRES, GMRES
        x_ref, rep_ref = ref.solve_linear_system_null_space(ro, cols, va, b, krylov=krylov, preconditioner=6,
                                                            restart=30, tolerance=1e-8)
        x_co, rep_co = co.solve_projected_gmres(ro, cols, va, b, H, restart=30, tolerance=1e-8)
        assert rep_co["status"] == rep_ref["status"] == 0
        assert rep_co["iterations"] == rep_ref["iterations"]
        assert np.array_equal(x_co, x_ref)
    try:
        Rc = ref.Amg(ro, cols, va, require_smoother_certificate=True, constant_null_space=True)
        Hc = co.Hierarchy([Rc.level(l) for l in range(Rc.num_levels())], Rc.omega, constant_null_space=True)
    except RuntimeError:
        # the Jacobi certificate of CG's AMG refuses the hierarchy (the hex
        # case's one-row coarsest level has a zero diagonal): NOT_APPLICABLE
        Hc = None
    for pc, model in (("native_amg", 6), ("jacobi", 2), ("none", 1)):
        x_ref, rep_ref = ref.solve_linear_system_null_space(ro, cols, va, b, krylov=1, preconditioner=model,
                                                            tolerance=1e-8)
        if pc == "native_amg" and Hc is None:
            assert rep_ref["status"] == 3
            continue
        x_co, rep_co = co.solve_cg(ro, cols, va, b, pc, Hc if pc == "native_amg" else None, tolerance=1e-8,
                                   null_space=True)
        assert rep_co["status"] == rep_ref["status"] == 0
        assert rep_co["iterations"] == rep_ref["iterations"]
        assert np.array_equal(x_co, x_ref)


def test_null_space_cycle_with_swept_coarsest_level(ref):
    """A hierarchy cut at a 52-row level: the coarsest treatment is 24 damped-
    Jacobi sweeps from zero, each followed by the mean removal."""
    ro, cols, va, b = _neumann_poisson(10)
    R = ref.Amg(ro, cols, va, constant_null_space=True)
    levels = [R.level(l) for l in range(4)]
    assert levels[-1]["inv_diag"].size > 16
    RT = ref.AmgFromLevels(levels, R.omega, constant_null_space=True)
    H = co.Hierarchy(levels, R.omega, constant_null_space=True)
    for seed in (0, 1, 2):
        r = np.random.default_rng(seed).standard_normal(b.size)
        assert np.array_equal(H.apply(r), RT.apply(r))


def test_null_space_refusals(ref):
    """An incompatible right-hand side or an operator without the constant
    null space: NOT_APPLICABLE with the iterate untouched."""
    ro, cols, va, b = _neumann_pressure(6)
    bad_b = b + 1.0
    assert co.null_space_checks(ro, cols, va, bad_b) == (False, True, True)
    x0 = np.full(b.size, 0.25)
    for krylov in (4, 1):
        x_ref, rep_ref = ref.solve_linear_system_null_space(ro, cols, va, bad_b, x0=x0, krylov=krylov,
                                                            preconditioner=1)
        assert rep_ref["status"] == 3 and np.array_equal(x_ref, x0)
    x_co, rep = co.solve_projected_gmres(ro, cols, va, bad_b, None, x0=x0)
    assert rep["status"] == 3 and np.array_equal(x_co, x0)
    x_co, rep = co.solve_cg(ro, cols, va, bad_b, "none", x0=x0, null_space=True)
    assert rep["status"] == 3 and np.array_equal(x_co, x0)
    # a Dirichlet-fixed system has no constant null space
    m, g, U, rAU, p, fixed, value = _pressure_inputs(6)
    a = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    checks = co.null_space_checks(a["row_offsets"], a["columns"], a["values"], a["b"] - a["b"].mean())
    assert checks[1:] == (False, False)
    x_ref, rep_ref = ref.solve_linear_system_null_space(a["row_offsets"], a["columns"], a["values"],
                                                        a["b"] - a["b"].mean(), krylov=4, preconditioner=1)
    assert rep_ref["status"] == 3


@pytest.mark.parametrize("name", sorted(p.stem for p in GOLDEN.glob("*.npz")))
def test_oracle_reproduces_golden_fixtures(name):
    z = dict(np.load(GOLDEN / f"{name}.npz"))
    n = int(z["n"])
    if name.startswith("pressure"):
        m, g, U, rAU, p, fixed, value = _pressure_inputs(n)
        a = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
        for k in ("row_offsets", "columns", "values", "b"):
            assert np.array_equal(a[k], z[k]), k
        assert np.array_equal(co.rhie_chow_flux(m, U, rAU, p, 1.0, fixed, value), z["flux"])
        levels = []
        for l in range(int(z["n_levels"])):
            lv = {k: z[f"L{l}_{k}"] for k in ("row_offsets", "columns", "values", "inv_diag")}
            if f"L{l}_p_offsets" in z:
                lv.update({k: z[f"L{l}_{k}"] for k in ("p_offsets", "p_columns", "p_values")})
            levels.append(lv)
        H = co.Hierarchy(levels, float(z["omega"]))
        assert np.array_equal(H.apply(z["vcycle_r"]), z["vcycle_z"])
        x, rep = co.solve_gmres(a["row_offsets"], a["columns"], a["values"], a["b"], H, restart=30, tolerance=1e-8)
        assert rep["iterations"] == int(z["iterations"])
        assert np.array_equal(x, z["x"])
        assert np.array_equal(co.rhie_chow_flux(m, U, rAU, x, 1.0, fixed, value), z["flux_solved"])
        xc, repc = co.solve_cg(a["row_offsets"], a["columns"], a["values"], a["b"], "native_amg", H,
                               max_iterations=1000, tolerance=1e-10)
        assert repc["status"] == 0 and repc["iterations"] == int(z["cg_iterations"])
        assert np.array_equal(xc, z["cg_x"])
    elif name.startswith("neumann"):
        m, g, U, rAU, p, fixed, value = _pressure_inputs(n)
        a = co.simple_assemble(m, U, rAU, p, 1.0, np.zeros_like(fixed), value)
        for k in ("row_offsets", "columns", "values"):
            assert np.array_equal(a[k], z[k]), k
        assert np.array_equal(a["b"] - a["b"].mean(), z["b"])
        ro, cols, va, b = z["row_offsets"], z["columns"], z["values"], z["b"]
        assert co.null_space_checks(ro, cols, va, b) == (True, True, True)
        H = co.Hierarchy(_golden_levels(z), float(z["omega"]), constant_null_space=True)
        assert np.array_equal(H.apply(z["vcycle_r"]), z["vcycle_z"])
        x, rep = co.solve_projected_gmres(ro, cols, va, b, H, restart=30, tolerance=1e-8)
        assert rep["status"] == 0 and rep["iterations"] == int(z["iterations"])
        assert np.array_equal(x, z["x"])
        xc, repc = co.solve_cg(ro, cols, va, b, "native_amg", H, tolerance=1e-10, null_space=True)
        assert repc["status"] == 0 and repc["iterations"] == int(z["cg_iterations"])
        assert np.array_equal(xc, z["cg_x"])
    elif name.startswith("poisson"):
        m, bc, src = cases.poisson_case(n)
        ro, cols, va, rhs = co.assemble_diffusion(m, bc, 1.0, src)
        for k, v in (("row_offsets", ro), ("columns", cols), ("values", va), ("rhs", rhs)):
            assert np.array_equal(v, z[k]), k
    else:
        pytest.fail(f"unknown fixture {name}")
