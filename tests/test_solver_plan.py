"""Automatic solver selection on CPU, pinned to the reference.

``measure_matrix_characteristics`` (core/linalg/matrix_diagnostics.h:285) and
``select_linear_solver`` (core/linalg/linear_solver_models.h:228) are what
``solve_linear_system`` runs before every solve; the library restates them
on the host (cfdxg_measure_matrix_characteristics, cfdxg_select_linear_solver)
for requests whose Krylov method or preconditioner is "auto".  Here both are
compared with the reference's own functions built into oracle/_ref: the
characteristics field by field (floating-point fields bit for bit) on
pressure, diffusion and deliberately pathological matrices, and the plan
(Krylov, preconditioner, null space, automatic flags, or a rejection) over
every problem kind, model and characteristics profile."""
import itertools

import numpy as np
import pytest

import cfdx_dev_b200 as cg
from cfdx_dev_b200 import _native as N
from cfdx_dev_b200.api import CfdxgError
from oracle import cfdx_oracle as co
from tests import cases

GOLDEN = cases.ROOT / "tests" / "golden"
FLAGS = ("square", "numerically_symmetric", "diagonally_dominant", "strongly_scaled",
         "large_diagonal_dynamic_range", "strongly_directional_coupling", "positive_diagonal", "saddle_point")


def _csr_from_dense(D):
    ro, co_, va = [0], [], []
    for row in D:
        nz = np.nonzero(row)[0]
        co_ += nz.tolist()
        va += row[nz].tolist()
        ro.append(len(co_))
    return np.array(ro), np.array(co_), np.array(va, float)


def _matrices():
    z = np.load(GOLDEN / "pressure_tet4.npz")
    ro, co_, va = z["row_offsets"], z["columns"], z["values"]
    out = {"pressure_tet4": (ro, co_, va)}
    m = cases.simple_mesh(5)
    g = co.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    a = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    out["pressure_tet5"] = (a["row_offsets"], a["columns"], a["values"])
    hm, bc, src = cases.poisson_case(5)
    dro, dco, dva, _ = co.assemble_diffusion(hm, bc, 1.0, src)
    out["poisson_hex5"] = (dro, dco, dva)
    v = va.copy()
    v[1] *= 1.0 + 1e-6                                             # one asymmetric coupling
    out["asymmetric"] = (ro, co_, v)
    v = va.copy()
    for i in range(ro.size - 1):                                    # rows scaled over 9 decades
        v[ro[i]:ro[i + 1]] *= 10.0 ** (i % 10)
    out["strongly_scaled"] = (ro, co_, v)
    s = 10.0 ** (1.5 * (np.arange(ro.size - 1) % 3))              # S A S: diagonal spread 1e6, symmetric
    rows = np.repeat(np.arange(ro.size - 1), np.diff(ro))
    out["diagonal_range"] = (ro, co_, va * s[rows] * s[co_])
    # anisotropic 2-D Laplacian: x couplings 1, y couplings 1e-4
    nx = 6
    D = np.zeros((nx * nx, nx * nx))
    for j in range(nx):
        for i in range(nx):
            r = j * nx + i
            for di, dj, w in ((1, 0, 1.0), (-1, 0, 1.0), (0, 1, 1e-4), (0, -1, 1e-4)):
                ii, jj = i + di, j + dj
                D[r, r] += w
                if 0 <= ii < nx and 0 <= jj < nx:
                    D[r, jj * nx + ii] -= w
    D[0, 0] += 1.0
    out["anisotropic"] = _csr_from_dense(D)
    E = D.copy()
    E[3, 3] = 0.0                                                   # missing diagonal entry
    out["missing_diagonal"] = _csr_from_dense(E)
    E = D.copy()
    E[5, 5] = -E[5, 5]                                              # negative diagonal
    out["negative_diagonal"] = _csr_from_dense(E)
    E = D.copy()
    E[7, :] = 0.0                                                   # empty row
    out["empty_row"] = _csr_from_dense(E)
    out["one_by_one"] = (np.array([0, 1]), np.array([0]), np.array([2.5]))
    out["weak_dominance"] = _csr_from_dense(np.array([[1.0, -0.6, -0.5], [-0.6, 2.0, -0.3], [-0.5, -0.3, 1.0]]))
    return out


MATRICES = _matrices()


@pytest.mark.parametrize("name", sorted(MATRICES))
@pytest.mark.parametrize("tol,saddle", [(1e-12, False), (0.0, False), (1e-5, True)])
def test_characteristics_match_reference(ref, name, tol, saddle):
    ro, co_, va = MATRICES[name]
    mine = cg.measure_matrix_characteristics(ro, co_, va, saddle_point=saddle, symmetry_tolerance=tol)
    theirs = ref.measure_characteristics(ro, co_, va, saddle_point=saddle, symmetry_tolerance=tol)
    for k, v in theirs.items():
        if isinstance(v, float):
            assert np.float64(mine[k]).tobytes() == np.float64(v).tobytes(), (k, mine[k], v)
        else:
            assert mine[k] == v, (k, mine[k], v)


def test_characteristics_of_the_profiles():
    c = {k: cg.measure_matrix_characteristics(*MATRICES[k]) for k in ("pressure_tet4", "asymmetric", "anisotropic",
                                                                      "strongly_scaled", "missing_diagonal")}
    assert c["pressure_tet4"]["numerically_symmetric"] and c["pressure_tet4"]["positive_diagonal"]
    assert not c["asymmetric"]["numerically_symmetric"]
    assert c["anisotropic"]["strongly_directional_coupling"]
    assert c["strongly_scaled"]["strongly_scaled"]
    assert not c["missing_diagonal"]["positive_diagonal"]


def test_characteristics_reject_bad_input():
    ro, co_, va = MATRICES["pressure_tet4"]
    bad = co_.copy()
    bad[0], bad[1] = bad[1], bad[0]
    with pytest.raises(CfdxgError, match="increase"):
        cg.measure_matrix_characteristics(ro, bad, va)
    with pytest.raises(CfdxgError, match="tolerance"):
        cg.measure_matrix_characteristics(ro, co_, va, symmetry_tolerance=-1.0)
    # a non-finite value stops the diagnosis: coefficient evidence stays at its defaults
    v = va.copy()
    v[5] = np.nan
    c = cg.measure_matrix_characteristics(ro, co_, v)
    assert c["coefficient_range"] == 1.0 and not c["diagonally_dominant"] and not c["strongly_scaled"]


def _profiles():
    """Characteristic profiles that reach every branch of the selection."""
    out = []
    for bits in itertools.product((0, 1), repeat=7):
        sym, dd, pos, directional, ddr, scaled, saddle = bits
        for eq in (10, 5000):
            out.append(dict(equations=eq, average_nnz_per_row=5.0, coefficient_range=1e9 if scaled else 10.0,
                            square=1, numerically_symmetric=sym, diagonally_dominant=dd, strongly_scaled=scaled,
                            large_diagonal_dynamic_range=ddr, strongly_directional_coupling=directional,
                            positive_diagonal=pos, saddle_point=saddle))
    return out


def _compare(problem, c, k, p, null_space, scaling, restart=40, alpha=1.0, ref=None):
    theirs = ref.select_linear_solver(problem, c, k, p, restart, null_space, scaling, alpha)
    try:
        plan = cg.select_linear_solver(N.PROBLEMS[problem], c, N.KRYLOV_MODELS[k], N.PRECONDITIONER_MODELS[p],
                                       restart, N.NULL_SPACES[null_space], N.SCALINGS[scaling], alpha)
        mine = (N.KRYLOV_MODELS.index(plan["krylov"]), N.PRECONDITIONER_MODELS.index(plan["preconditioner"]),
                N.NULL_SPACES.index(plan["null_space"]), int(plan["automatic_krylov"]),
                int(plan["automatic_preconditioner"]))
    except CfdxgError:
        mine = None
    assert mine == theirs, (problem, c, k, p, null_space, scaling)


def test_selection_matches_reference_on_auto_requests(ref):
    for problem in range(6):
        for c in _profiles():
            for null_space in (0, 1):
                for scaling in range(5):
                    _compare(problem, c, 0, 0, null_space, scaling, ref=ref)


def test_selection_matches_reference_on_explicit_models(ref):
    rng = np.random.default_rng(20240611)
    profiles = _profiles()
    for _ in range(6000):
        c = profiles[rng.integers(len(profiles))]
        _compare(int(rng.integers(6)), c, int(rng.integers(8)), int(rng.integers(23)), int(rng.integers(2)),
                 int(rng.integers(5)), ref=ref)
    for k in range(8):                       # every model pair on the pressure profile
        for p in range(23):
            _compare(1, cg.measure_matrix_characteristics(*MATRICES["pressure_tet4"]), k, p, 0, 0, ref=ref)


def test_selection_rejects_what_the_reference_rejects(ref):
    c = cg.measure_matrix_characteristics(*MATRICES["pressure_tet4"])
    for restart, alpha in ((0, 1.0), (-3, 1.0), (40, 0.2), (40, 4.5), (40, float("nan"))):
        _compare(1, c, 0, 0, 0, 0, restart=restart, alpha=alpha, ref=ref)
    nonsquare = dict(c, square=0)
    _compare(1, nonsquare, 0, 0, 0, 0, ref=ref)


def test_pressure_systems_select_cg_with_native_amg():
    for name in ("pressure_tet4", "pressure_tet5", "poisson_hex5"):
        plan = cg.select_linear_solver("pressure_poisson", cg.measure_matrix_characteristics(*MATRICES[name]))
        assert (plan["krylov"], plan["preconditioner"]) == ("cg", "native_amg"), name
    plan = cg.select_linear_solver("pressure_poisson", cg.measure_matrix_characteristics(*MATRICES["anisotropic"]))
    assert (plan["krylov"], plan["preconditioner"]) == ("fgmres", "native_amg")
    for name in ("asymmetric", "diagonal_range"):
        plan = cg.select_linear_solver("pressure_poisson", cg.measure_matrix_characteristics(*MATRICES[name]))
        assert (plan["krylov"], plan["preconditioner"]) == ("gmres", "ilu0"), name


@pytest.mark.parametrize("name", sorted(MATRICES))
@pytest.mark.parametrize("scaling", ["none", "row", "column", "row_column", "symmetric_diagonal"])
@pytest.mark.parametrize("zero_tolerance", [0.0, 0.5])
def test_scaling_matches_reference(ref, name, scaling, zero_tolerance):
    ro, co_, va = MATRICES[name]
    mine = cg.scale_matrix(ro, co_, va, scaling, zero_tolerance)
    rs, cs, sv, zr, zc = ref.scale_matrix(ro, co_, va, N.SCALINGS.index(scaling), zero_tolerance)
    for a, b in ((mine["row_scale"], rs), (mine["column_scale"], cs), (mine["values"], sv)):
        assert a.tobytes() == b.tobytes()
    assert (mine["zero_rows"], mine["zero_columns"]) == (zr, zc)


def test_symmetric_diagonal_scaling_gives_a_unit_diagonal():
    ro, co_, va = MATRICES["pressure_tet5"]
    s = cg.scale_matrix(ro, co_, va, "symmetric_diagonal")
    rows = np.repeat(np.arange(ro.size - 1), np.diff(ro))
    diag = s["values"][rows == co_]
    assert np.allclose(diag, 1.0, rtol=1e-15, atol=0)
    c = cg.measure_matrix_characteristics(ro, co_, s["values"])
    assert c["numerically_symmetric"] and c["positive_diagonal"]
    with pytest.raises(CfdxgError):
        cg.scale_matrix(ro, co_, va, "row", zero_tolerance=-1.0)


# ---------------------------------------------- tests/unit/test_matrix_characteristics.cpp
def test_reference_case_coupled_dispatch():
    c = cg.measure_matrix_characteristics([0, 2, 5, 7], [0, 1, 0, 1, 2, 1, 2], [4.0, -1.0, -1.0, 4.0, -1.0, -1.0, 4.0],
                                          saddle_point=True)
    assert c["square"] and c["saddle_point"] and c["numerically_symmetric"] and c["diagonally_dominant"]
    assert abs(c["average_nnz_per_row"] - 7.0 / 3.0) < 1e-14
    plan = cg.select_linear_solver("coupled_pressure_velocity", c)
    assert (plan["krylov"], plan["preconditioner"]) == ("fgmres", "coupled_block_schur")


def test_reference_case_nonsymmetry_and_scaling():
    c = cg.measure_matrix_characteristics([0, 2, 4], [0, 1, 0, 1], [1.0e9, 1.0, 0.5, 1.0e-2])
    assert c["square"] and not c["numerically_symmetric"] and c["strongly_scaled"]
    assert c["coefficient_range"] > 1.0e10


def test_reference_case_diagonal_dynamic_range_avoids_cg_amg():
    c = cg.measure_matrix_characteristics([0, 2, 4], [0, 1, 0, 1], [1.0e5, -1.0e-1, -1.0e-1, 1.0])
    assert c["numerically_symmetric"] and c["diagonally_dominant"] and c["large_diagonal_dynamic_range"]
    assert not c["strongly_scaled"]
    plan = cg.select_linear_solver("pressure_poisson", c)
    assert (plan["krylov"], plan["preconditioner"]) == ("gmres", "jacobi")


# ------------------------------------------------------------- diagnose_matrix
@pytest.mark.parametrize("name", sorted(MATRICES))
@pytest.mark.parametrize("tol,topology", [(1e-14, True), (0.5, False)])
def test_diagnosis_matches_reference(ref, name, tol, topology):
    ro, co_, va = MATRICES[name]
    mine = cg.diagnose_matrix(ro, co_, va, diagonal_relative_tolerance=tol, include_topology=topology)
    theirs = ref.diagnose_matrix(ro, co_, va, tolerance=tol, topology=topology)
    for k, v in theirs.items():
        if isinstance(v, float):
            assert np.float64(mine[k]).tobytes() == np.float64(v).tobytes(), (k, mine[k], v)
        else:
            assert mine[k] == v, (k, mine[k], v)


def test_diagnosis_of_a_rectangular_matrix_and_an_inconsistent_one(ref):
    # 3 x 4 with an empty column, and the chain of a block-diagonal pattern (two components)
    ro, co_, va = np.array([0, 2, 3, 4]), np.array([0, 1, 1, 3]), np.array([2.0, -1.0, 3.0, 4.0])
    mine = cg.diagnose_matrix(ro, co_, va, n_cols=4)
    theirs = ref.diagnose_matrix(ro, co_, va, n_cols=4)
    assert np.isnan(mine["minimum_gershgorin_margin"]) and np.isnan(theirs["minimum_gershgorin_margin"])
    for k in theirs:
        if k != "minimum_gershgorin_margin":
            assert mine[k] == theirs[k], k
    assert mine["empty_columns"] == 1 and mine["connected_components"] == 3
    bad = cg.diagnose_matrix([0, 2, 3], [1, 0, 1], [1.0, 2.0, 3.0])   # unsorted row: not consistent
    assert bad["structurally_consistent"] == 0 and bad["finite"] == 0 and bad["rows"] == 2
