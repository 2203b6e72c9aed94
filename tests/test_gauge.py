"""Pressure gauge of a pure-Neumann system, on CPU: the oracle's restatement
against the reference's apply_reference_cell_gauge (core/solvers/
scalar_diffusion.h:177-210, built into oracle/_ref) and, for the corrector's
reference-cell elimination (physics/steady_incompressible_solver.h:8617-8654,
not a callable symbol), against its definition: the principal submatrix."""
import numpy as np
import pytest

from oracle import cfdx_oracle as co
from tests import cases


def _neumann_pressure_system(n=4):
    # every patch zero-gradient: the pure-Neumann pressure corrector
    m = cases.simple_mesh(n)
    g = co.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    fixed[:] = 0
    a = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    return a["row_offsets"], a["columns"], a["values"], a["b"]


def _dense(ro, cols, va, n):
    A = np.zeros((n, n))
    for i in range(n):
        for k in range(ro[i], ro[i + 1]):
            A[i, cols[k]] += va[k]
    return A


@pytest.mark.parametrize("cell", [0, 17, -1])
def test_elimination_is_the_principal_submatrix(cell):
    ro, cols, va, b = _neumann_pressure_system()
    n = b.size
    ref = cell % n
    r_ro, r_co, r_va, r_b = co.gauge_eliminate(ro, cols, va, b, ref)
    keep = np.array([i for i in range(n) if i != ref])
    assert np.array_equal(_dense(r_ro, r_co, r_va, n - 1), _dense(ro, cols, va, n)[np.ix_(keep, keep)])
    assert np.array_equal(r_b, b[keep])
    for i in range(n - 1):   # columns stay sorted
        assert np.all(np.diff(r_co[r_ro[i]:r_ro[i + 1]]) > 0)
    x = co.gauge_expand(np.arange(1.0, n), ref)
    assert x[ref] == 0.0 and np.array_equal(np.delete(x, ref), np.arange(1.0, n))


@pytest.mark.parametrize("cell,value", [(0, 0.0), (5, 2.5), (-1, -1.25)])
def test_identity_row_matches_reference(ref, cell, value):
    ro, cols, va, b = _neumann_pressure_system()
    cell = cell % b.size
    mine = co.gauge_identity_row(ro, cols, va, b, cell, value)
    theirs = ref.apply_reference_cell_gauge(ro, cols, va, b, cell, value)
    for a, t in zip(mine, theirs):
        assert np.array_equal(a, t)


def test_invalid_gauges_fail_loudly():
    with pytest.raises(RuntimeError):
        co.gauge_eliminate([0, 1], [0], [1.0], [1.0], 0)          # the only unknown
    with pytest.raises(RuntimeError):
        co.gauge_identity_row([0, 1], [0], [1.0], [1.0], 3, 0.0)   # out of range

