"""The FP32 cycle's sparsified smoothing operators (coarse_drop_tolerance).

Between the fine and the coarsest level the FP32 cycle may smooth with a
sparser operator than the Galerkin one: each row keeps its diagonal and the
off-diagonal entries with |a_ij| >= theta * max_k!=i |a_ik|, the dropped
entries added to the diagonal.  Checked against a numpy FP64 restatement of
the same cycle (fine level V(pre, post), levels >= 1 V(0, 1), dense inverse
at the coarsest level) built from the exported Galerkin levels:

* the GPU FP32 cycle equals the restatement to FP32 rounding for theta = 0
  and theta = 0.02, on a tet pressure system and on an anisotropic
  boundary-layer one, and the two differ by far more than that rounding;
* after a numeric refresh the kept pattern is the setup's and the values
  and lumped diagonals are the new operator's;
* FGMRES with the sparsified cycle reaches the FP64 certificate.
(The option's validation is a CPU test, tests/test_abi.py.)
"""
import numpy as np
import pytest
import scipy.sparse as sp

import cfdx_dev_b200 as cg
from tests import cases

pytestmark = pytest.mark.gpu

THETA = 0.02
FP32_TOL = 1e-4
OPTS = dict(precision="fp32_vcycle", half_values=0, coarse_dense_limit=100, pre_sweeps=2, post_sweeps=2,
            coarse_pre_sweeps=0, coarse_post_sweeps=1)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def keep_mask(A, theta):
    """Kept entries of each row of A: the diagonal and |a_ij| >= theta * max off-diagonal."""
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    off = A.indices != rows
    mag = np.where(off, np.abs(A.data), 0.0)
    rmax = np.zeros(A.shape[0])
    np.maximum.at(rmax, rows, mag)
    return ~off | (np.abs(A.data) >= theta * rmax[rows])


def sparsified(A, keep):
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    off = A.indices != rows
    drop = ~keep
    d = A.diagonal() + np.bincount(rows[drop], weights=A.data[drop], minlength=A.shape[0])
    K = sp.csr_matrix((np.where(off, A.data, 0.0)[keep], (rows[keep], A.indices[keep])), shape=A.shape)
    return (K + sp.diags(d)).tocsr(), 1.0 / d


def levels_of(amg):
    out = []
    for l in range(len(amg.hierarchy_level_sizes())):
        e = amg.export_level(l)
        n = len(e["row_offsets"]) - 1
        A = sp.csr_matrix((e["values"], e["columns"], e["row_offsets"]), shape=(n, n))
        P = None
        if len(e["p_columns"]):
            P = sp.csr_matrix((e["p_values"], e["p_columns"], e["p_offsets"]),
                              shape=(n, int(e["p_columns"].max()) + 1))
        out.append(dict(A=A, dinv=e["inv_diag"], P=P))
    return out


def restated_cycle(levels, omega, theta, masks=None, dense_limit=100, pre=2, post=2):
    """z = V-cycle(r) of the FP32 cycle's structure in FP64; masks (one per
    level, or None) fix the kept pattern (a refresh keeps the setup's)."""
    used = next(l for l, lv in enumerate(levels) if lv["A"].shape[0] <= dense_limit) + 1
    ops = []
    for l in range(used):
        A = levels[l]["A"]
        if theta > 0 and 1 <= l < used - 1:
            keep = masks[l] if masks is not None else keep_mask(A, theta)
            ops.append(sparsified(A, keep))
        else:
            ops.append((A, levels[l]["dinv"]))
    dense = np.linalg.inv(levels[used - 1]["A"].toarray())

    def cyc(l, r):
        if l == used - 1:
            return dense @ r
        A, dinv = ops[l]
        P = levels[l]["P"]
        if l == 0:
            x = omega * dinv * r
            for _ in range(pre - 1):
                x = x + omega * dinv * (r - A @ x)
            x = x + P @ cyc(1, P.T @ (r - A @ x))
            for _ in range(post):
                x = x + omega * dinv * (r - A @ x)
            return x
        x = P @ cyc(l + 1, P.T @ r)
        return x + omega * dinv * (r - A @ x)

    return lambda r: cyc(0, r)


def _systems(ctx, m):
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    out = []
    for off in (0, 11):
        U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"], seed_offset=off)
        A, b, _, _ = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
        out.append((A, b))
    return out


@pytest.fixture(scope="module")
def system(ctx):
    return _systems(ctx, cases.simple_mesh(10))


@pytest.fixture(scope="module")
def boundary_layer(ctx):
    # anisotropic hexahedra (wall spacing 1e-3 growing 1.2 per cell), as in config 5
    return _systems(ctx, cg.boundary_layer_case(16, 12, 8, dy0=1e-3, growth=1.2, jitter=0.05, seed=5))


@pytest.mark.parametrize("case", ["tet", "boundary_layer"])
def test_sparsified_cycle_matches_restatement(ctx, system, boundary_layer, case):
    A, b = (system if case == "tet" else boundary_layer)[0]
    r = np.random.default_rng(5).standard_normal(A.n)
    z = {}
    for theta in (0.0, THETA):
        amg = cg.NativeBoomerAMGPreconditioner(ctx, coarse_drop_tolerance=theta, **OPTS)
        assert amg.setup(A), amg.last_error()
        assert len(amg.hierarchy_level_sizes()) >= 4
        z[theta] = amg.apply(r)
        want = restated_cycle(levels_of(amg), amg.omega, theta)(r)
        assert rel_l2(z[theta], want) < FP32_TOL, theta
    # the sparsification changes the cycle by far more than FP32 rounding
    # (1.7e-2 on the tets, 6.3e-3 on the boundary layer in FP64)
    assert rel_l2(z[THETA], z[0.0]) > 10 * FP32_TOL


def test_sparsified_pattern_survives_refresh(ctx, system):
    (A1, _), (A2, b2) = system
    amg = cg.NativeBoomerAMGPreconditioner(ctx, coarse_drop_tolerance=THETA, **OPTS)
    assert amg.setup(A1)
    masks = [keep_mask(lv["A"], THETA) for lv in levels_of(amg)]
    assert amg.update_values(A2)
    lv2 = levels_of(amg)
    r = np.random.default_rng(6).standard_normal(A1.n)
    want = restated_cycle(lv2, amg.omega, THETA, masks=masks)(r)
    assert rel_l2(amg.apply(r), want) < FP32_TOL
    # FGMRES with the refreshed sparsified cycle reaches the FP64 certificate
    x, rep = cg.solve_fgmres(A2, b2, amg=amg, restart=30, tolerance=1e-8)
    assert rep["status_name"] == "converged" and rep["physical_residual_relative"] <= 1e-8


def test_default_fp32_solve_with_sparsified_levels(ctx, system):
    """The default FP32 plan (theta 0.02, FP16 values) on a multilevel cycle:
    the FP64 certificate, and the solution within 1e-6 of the FP64 solve."""
    A, b = system[0]
    x64, rep64 = cg.solve_linear_system(A, b, restart=30, tolerance=1e-8)
    amg = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp32_vcycle", coarse_dense_limit=100)
    assert amg.setup(A)
    x, rep = cg.solve_fgmres(A, b, amg=amg, restart=30, tolerance=1e-8)
    assert rep["status_name"] == "converged" and rep["physical_residual_relative"] <= 1e-8
    assert rel_l2(x, x64) < 1e-6
