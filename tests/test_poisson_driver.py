"""The reference's Poisson driver (core/solvers/scalar_diffusion.h:294-340,
solve_poisson_mixed, called by apps/poisson) restated by composing the C
oracle's diffusion assembly, identity-row gauge and own-diagonal CG, pinned
bit for bit to the reference built into oracle/_ref: the apps/poisson case
(homogeneous Dirichlet on every boundary face, unit source) and a
pure-Neumann case (zero-flux walls, zero-mean source, reference-cell gauge)."""
import numpy as np
import pytest

from oracle import cfdx_oracle as co
from tests import cases


def oracle_poisson_mixed(m, bc, src, types=None, max_iterations=2000, tolerance=1e-10, ref_cell=0, ref_value=0.0):
    ro, cols, va, rhs = co.assemble_diffusion(m, bc, 1.0, src, types)
    t = np.zeros(bc.size, np.int32) if types is None else types
    x0 = np.zeros(rhs.size)
    if not np.any(np.isfinite(bc) & (t == 0)):
        ro, cols, va, rhs = co.gauge_identity_row(ro, cols, va, rhs, ref_cell, ref_value)
        x0[ref_cell] = ref_value
    return co.solve_cg(ro, cols, va, rhs, "internal_jacobi", None, x0=x0, max_iterations=max_iterations,
                       tolerance=tolerance)


def apps_poisson_case(n=6):
    import cfdx_dev_b200 as cg
    m = cg.hex_case(n)
    bc = np.full(m.n_faces, np.nan)
    bc[m.neighbour < 0] = 0.0
    return m, bc, np.ones(m.n_cells)


def neumann_case(n=6):
    import cfdx_dev_b200 as cg
    m = cg.hex_case(n)
    g = co.geometry(m)
    vol = g["cell_volumes"]
    f = cg.random_field(m.n_cells, "uniform", -1.0, 1.0, 7)
    src = f - np.sum(f * vol) / np.sum(vol)
    bc = np.full(m.n_faces, np.nan)
    bc[m.neighbour < 0] = 0.0
    types = np.ones(m.n_faces, np.int32)
    return m, bc, src, types


def test_apps_poisson_case_matches_reference(ref):
    m, bc, src = apps_poisson_case()
    x, rep = oracle_poisson_mixed(m, bc, src)
    x_ref, rep_ref = ref.solve_poisson_mixed(m, bc, src)
    assert rep["status"] == rep_ref["status"] == 0
    assert rep["iterations"] == rep_ref["iterations"]
    assert np.array_equal(x, x_ref)


@pytest.mark.parametrize("cell,value", [(0, 0.0), (11, 1.5)])
def test_pure_neumann_case_matches_reference(ref, cell, value):
    m, bc, src, types = neumann_case()
    x, rep = oracle_poisson_mixed(m, bc, src, types, ref_cell=cell, ref_value=value)
    x_ref, rep_ref = ref.solve_poisson_mixed(m, bc, src, types, reference_cell=cell, reference_value=value)
    assert rep["status"] == rep_ref["status"] == 0
    assert rep["iterations"] == rep_ref["iterations"]
    assert np.array_equal(x, x_ref)
    assert x[cell] == value


def test_incompatible_pure_neumann_data_is_refused(ref):
    m, bc, src, types = neumann_case()
    with pytest.raises(RuntimeError):
        ref.solve_poisson_mixed(m, bc, src + 1.0, types)
