"""Domain decomposition on one GPU: every part of the plan held by one
process (the halo exchange is then device copies), computed through the C ABI.

Checks: the parts' products after an exchange equal the undivided FP64 SpMV
bit for bit; the distributed FGMRES with a native AMG per part (FP64 and FP32
V-cycles) reaches the FP64 true relative residual 1e-8, measured by the
oracle's product on the host, and agrees with the undivided solve."""
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
    m = cases.simple_mesh(12)
    g = co.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    a = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    return a["row_offsets"], a["columns"], a["values"], a["b"]


def test_cuda_parts_product_is_bit_identical(ctx, system):
    ro, co_, va, b = system
    x = np.random.default_rng(11).standard_normal(b.size)
    A = cg.SparseMatrix.from_csr(ctx, ro, co_, va)
    y = A.matvec(x)
    plan = domain.DomainPlan(ro, co_, 3)
    comm = domain.PartComm(3)
    parts = {p: domain.CudaPart(ctx, plan.part(p), va) for p in range(3)}
    dev = parts[0].device
    comm.prepare({p: P.layout for p, P in parts.items()}, dev)
    with torch.cuda.stream(parts[0].stream):
        vec = {}
        for p, P in parts.items():
            L = P.layout
            v = torch.full((L.n_local,), float("nan"), dtype=torch.float64, device=dev)
            v[L.owned] = torch.as_tensor(x[L.row_begin:L.row_end], device=dev)
            vec[p] = v
        comm.exchange(vec)
        for p, P in parts.items():
            L = P.layout
            assert not torch.isnan(vec[p]).any()
            assert np.array_equal(P.matvec(vec[p]).cpu().numpy(), y[L.row_begin:L.row_end])


@pytest.mark.parametrize("precision", ["fp64", "fp32_vcycle"])
def test_cuda_parts_solve(ctx, system, precision):
    ro, co_, va, b = system
    launches = ctx.kernel_launches
    x, rep = domain.solve_distributed(ctx, ro, co_, va, b, 3, preconditioner="block_jacobi", precision=precision,
                                      tolerance=1e-8)
    assert ctx.kernel_launches > launches
    xg = np.concatenate([x[p] for p in range(3)])
    res = np.linalg.norm(b - co.spmv(ro, co_, va, xg)) / np.linalg.norm(b)
    assert rep["status_name"] == "converged" and res <= 1e-8, rep
    A = cg.SparseMatrix.from_csr(ctx, ro, co_, va)
    xr, rr = cg.solve_linear_system(A, b, tolerance=1e-12)
    assert np.linalg.norm(xg - xr) <= 1e-6 * np.linalg.norm(xr)
