"""Solve options on a B200 that compose verified entry points: the request's
algebraic scaling (scale_matrix, solved scaled and certified unscaled) and the
distributed V-cycle of the domain decomposition (the library's FP64 SpMV per
part and level, torch element-wise updates).

The distributed V-cycle sums every product in the global row order and
updates element-wise in the reference's operation order, so on the device it
must equal the oracle's undivided V-cycle bit for bit; the solve keeps the
undivided iteration count for any number of parts (to one iteration: the
Krylov reductions are summed part by part)."""
import numpy as np
import pytest
import torch

import cfdx_dev_b200 as cg
from cfdx_dev_b200 import domain
from oracle import cfdx_oracle as co
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system():
    m = cases.simple_mesh(10)
    g = co.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    a = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    return a["row_offsets"], a["columns"], a["values"], a["b"]


@pytest.mark.parametrize("krylov,scaling", [("cg", "symmetric_diagonal"), ("gmres", "row"),
                                            ("fgmres", "row_column")])
def test_scaled_solve_is_certified_on_the_original_system(ctx, system, krylov, scaling):
    ro, co_, va, b = system
    A = cg.SparseMatrix.from_csr(ctx, ro, co_, va)
    x0, r0 = cg.solve_linear_system(A, b, krylov=krylov, tolerance=1e-10)
    x, rep = cg.solve_linear_system(A, b, krylov=krylov, scaling=scaling, tolerance=1e-10)
    assert rep["status_name"] == "converged"
    true = np.linalg.norm(b - co.spmv(ro, co_, va, x)) / np.linalg.norm(b)
    assert true <= 1e-10 and rep["physical_residual_relative"] == pytest.approx(true, rel=1e-6)
    assert rep["residual_relative"] == rep["physical_residual_relative"]
    assert np.linalg.norm(x - x0) <= 1e-5 * np.linalg.norm(x0)


def test_cg_refuses_nonsymmetric_scaling(ctx, system):
    ro, co_, va, b = system
    A = cg.SparseMatrix.from_csr(ctx, ro, co_, va)
    with pytest.raises(cg.CfdxgError):
        cg.solve_linear_system(A, b, krylov="cg", scaling="row", tolerance=1e-10)


def _device_vcycle(ctx, ro, co_, va, parts, replicate_below):
    plan = domain.DomainPlan(ro, co_, parts)
    comm = domain.PartComm(parts)
    amg = cg.NativeBoomerAMGPreconditioner()
    assert amg.setup_host(ro, co_, va)
    levels = [amg.export_level(l) for l in range(len(amg.hierarchy_level_sizes()))]
    stream = torch.cuda.ExternalStream(ctx.stream)
    dev = torch.device("cuda", torch.cuda.current_device())
    with torch.cuda.stream(stream):
        dm = domain.DistributedAMG(comm, levels, amg.omega, plan.row_splits,
                                   lambda r, c, v, nr, nc: domain.CudaOperator(ctx, r, c, v, nr, nc), dev,
                                   replicate_below=replicate_below)
    return plan, dm, levels, amg.omega, stream, dev


@pytest.mark.parametrize("parts,replicate_below", [(1, 4096), (3, 64)])
def test_device_distributed_vcycle_is_the_undivided_vcycle(ctx, system, parts, replicate_below):
    ro, co_, va, b = system
    plan, dm, levels, omega, stream, dev = _device_vcycle(ctx, ro, co_, va, parts, replicate_below)
    r = np.random.default_rng(parts).standard_normal(ro.size - 1)
    S = plan.row_splits
    with torch.cuda.stream(stream):
        rin = {p: torch.as_tensor(r[S[p]:S[p + 1]], device=dev) for p in range(parts)}
        z = {p: torch.empty(int(S[p + 1] - S[p]), dtype=torch.float64, device=dev) for p in range(parts)}
        dm.apply(rin, z)
        got = np.concatenate([z[p].cpu().numpy() for p in range(parts)])
    want = co.Hierarchy(levels, omega).apply(r)
    assert np.array_equal(got, want)


def test_device_distributed_solve_keeps_the_iteration_count(ctx, system):
    ro, co_, va, b = system
    its = []
    for parts in (1, 3):
        x, rep = domain.solve_distributed(ctx, ro, co_, va, b, parts, preconditioner="vcycle", replicate_below=64,
                                          tolerance=1e-8)
        xg = np.concatenate([x[p] for p in range(parts)])
        assert rep["status_name"] == "converged"
        assert np.linalg.norm(b - co.spmv(ro, co_, va, xg)) <= 1e-8 * np.linalg.norm(b)
        its.append(rep["iterations"])
    assert abs(its[0] - its[1]) <= 1          # only the order of the Krylov reductions differs
