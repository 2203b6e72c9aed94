"""Automatic solver selection through the C ABI on the GPU.

``solve_linear_system`` with Krylov method and preconditioner "auto" measures
the matrix, selects the plan as the reference's select_linear_solver does
(pinned on CPU by tests/test_solver_plan.py) and runs it: the benign SPD
pressure systems here get CG + native AMG and must give the reference's own
CG solve (golden fixture) and the reference's automatic dispatch (oracle/_ref,
where built); a plan naming a model outside this library fails closed."""
from pathlib import Path

import numpy as np
import pytest

import cfdx_dev_b200 as cg
from cfdx_dev_b200 import _native as N

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "pressure_tet4.npz"


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_auto_plan_runs_cg_with_native_amg(ctx):
    z = dict(np.load(GOLDEN))
    A = cg.SparseMatrix.from_csr(ctx, z["row_offsets"], z["columns"], z["values"])
    x, rep = cg.solve_linear_system(A, z["b"], krylov="auto", preconditioner="auto", max_iterations=1000,
                                    tolerance=1e-10)
    assert (rep["plan_krylov"], rep["plan_preconditioner"]) == (N.KRYLOV["cg"], N.PRECONDITIONER["native_amg"])
    assert "cg + native_amg" in ctx.lib.cfdxg_plan_reason(ctx.handle).decode()
    assert rep["status_name"] == "converged"
    assert rep["iterations"] == int(z["cg_iterations"])
    assert rel_l2(x, z["cg_x"]) <= 1e-10


def test_auto_plan_matches_reference_dispatch(ctx):
    from oracle import ref
    if not ref.available():
        pytest.skip("reference oracle not built")
    z = dict(np.load(GOLDEN))
    A = cg.SparseMatrix.from_csr(ctx, z["row_offsets"], z["columns"], z["values"])
    x, rep = cg.solve_linear_system(A, z["b"], krylov="auto", preconditioner="auto", tolerance=1e-10)
    xr, rr = ref.solve_linear_system(z["row_offsets"], z["columns"], z["values"], z["b"], krylov=0,
                                     preconditioner=0, restart=40, tolerance=1e-10)
    assert rr["status"] == 0 and rep["iterations"] == rr["iterations"]
    assert rel_l2(x, xr) <= 1e-10


def test_auto_plan_outside_the_library_fails_closed(ctx):
    z = dict(np.load(GOLDEN))
    va = z["values"].copy()
    va[1] *= 1.5                                   # nonsymmetric: the plan is GMRES + ILU0
    A = cg.SparseMatrix.from_csr(ctx, z["row_offsets"], z["columns"], va)
    x0 = np.full(A.n, 0.125)
    x, rep = cg.solve_linear_system(A, z["b"], x0=x0, krylov="auto", preconditioner="auto", tolerance=1e-10)
    assert rep["status_name"] == "not_applicable" and np.array_equal(x, x0)
    assert "ilu0" in ctx.lib.cfdxg_plan_reason(ctx.handle).decode()
    # an explicit Krylov method with an automatic preconditioner keeps the method
    x, rep = cg.solve_linear_system(A, z["b"], krylov="gmres", preconditioner="auto", tolerance=1e-10)
    assert rep["status_name"] == "not_applicable"
