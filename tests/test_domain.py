"""Domain decomposition on CPU: the partition/halo plan of the C ABI, the
halo exchange, and the distributed FGMRES driver over gloo ranks.

The reference has no distributed solve, so nothing here is compared with
it: the plan is checked against the undivided system (every local row is
the global row renumbered, a distributed product equals the global one bit
for bit), and the distributed solve against the FP64 true residual and the
undivided oracle GMRES solution.  The device parts (``CudaPart``) need a GPU;
here each part is the plain-C oracle's product and V-cycle (with the
library's host AMG setup of the part's diagonal block), which is what the
tests may use as a stand-in for the device."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from cfdx_dev_b200 import domain
from cfdx_dev_b200.api import CfdxgError, NativeBoomerAMGPreconditioner
from oracle import cfdx_oracle as co
from tests import cases

GOLDEN = cases.ROOT / "tests" / "golden"


def _golden():
    z = np.load(GOLDEN / "pressure_tet4.npz")
    return z["row_offsets"], z["columns"], z["values"], z["b"], z["x"]


def _system(n=8):
    m = cases.simple_mesh(n)
    g = co.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    a = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    return a["row_offsets"], a["columns"], a["values"], a["b"]


class OraclePart:
    """A part computed by the plain-C oracle: product of the local rows and a
    V-cycle of the AMG hierarchy the library sets up on the diagonal block."""

    device = torch.device("cpu")

    def __init__(self, layout, values, block_amg=True):
        self.layout = layout
        self.lv = np.ascontiguousarray(values[layout.local_source])
        if block_amg:
            bv = np.ascontiguousarray(values[layout.block_source])
            amg = NativeBoomerAMGPreconditioner()
            assert amg.setup_host(layout.block_row_offsets, layout.block_columns, bv), amg.last_error()
            self.H = co.Hierarchy([amg.export_level(l) for l in range(len(amg.hierarchy_level_sizes()))],
                                  amg.omega)

    def matvec(self, x_local):
        y = co.spmv(self.layout.local_row_offsets, self.layout.local_columns, self.lv, x_local.numpy())
        return torch.from_numpy(y[self.layout.owned])

    def precondition(self, r, z):
        z.copy_(torch.from_numpy(self.H.apply(r.numpy())))


# ------------------------------------------------------------------ the plan
@pytest.mark.parametrize("parts,splits", [(1, None), (2, None), (3, None), (5, None), (3, [0, 7, 200, 384]),
                                          (4, [0, 1, 2, 3, 384])])
def test_plan_rows_are_the_global_rows_renumbered(parts, splits):
    ro, co_, va, b, _ = _golden()
    plan = domain.DomainPlan(ro, co_, parts, splits)
    assert plan.parts == parts and plan.row_splits[0] == 0 and plan.row_splits[-1] == ro.size - 1
    if splits is not None:
        assert plan.row_splits.tolist() == splits
    for p in range(parts):
        L = plan.part(p)
        assert (L.row_begin, L.row_end) == (plan.row_splits[p], plan.row_splits[p + 1])
        g = L.local_to_global()
        assert np.all(np.diff(g) > 0)                         # numbering increasing in the global order
        assert L.local_row_offsets.size == L.n_local + 1
        assert np.all(np.diff(L.local_row_offsets[:L.owned_offset + 1]) == 0)             # ghost rows empty
        assert np.all(np.diff(L.local_row_offsets[L.owned_offset + L.n_owned:]) == 0)
        for i in range(L.row_begin, L.row_end):
            li = L.owned_offset + i - L.row_begin
            s = slice(L.local_row_offsets[li], L.local_row_offsets[li + 1])
            assert np.array_equal(g[L.local_columns[s]], co_[ro[i]:ro[i + 1]])
            assert np.array_equal(L.local_source[s], np.arange(ro[i], ro[i + 1]))
            bi = i - L.row_begin
            bs = slice(L.block_row_offsets[bi], L.block_row_offsets[bi + 1])
            own = (co_[ro[i]:ro[i + 1]] >= L.row_begin) & (co_[ro[i]:ro[i + 1]] < L.row_end)
            assert np.array_equal(L.block_columns[bs] + L.row_begin, co_[ro[i]:ro[i + 1]][own])
            assert np.array_equal(L.block_source[bs], np.arange(ro[i], ro[i + 1])[own])
        # the ghosts are exactly the foreign columns of the owned rows
        cols = co_[ro[L.row_begin]:ro[L.row_end]]
        assert np.array_equal(L.ghost_rows, np.unique(cols[(cols < L.row_begin) | (cols >= L.row_end)]))


@pytest.mark.parametrize("parts", [2, 3, 6])
def test_send_lists_match_the_receivers_ghosts(parts):
    ro, co_, va, b, _ = _golden()
    plan = domain.DomainPlan(ro, co_, parts)
    L = [plan.part(p) for p in range(parts)]
    for p in range(parts):
        for k, q in enumerate(L[p].neighbours.tolist()):
            assert q != p
            kq = L[q].neighbours.tolist().index(p)            # links are mutual
            recv = L[p].ghost_rows[L[p].recv_offsets[k]:L[p].recv_offsets[k + 1]]
            sent = L[q].send_rows[L[q].send_slice(kq)] + L[q].row_begin
            assert np.array_equal(recv, sent)
            g = L[p].local_to_global()
            assert np.array_equal(g[L[p].recv_slice(k)], recv)  # received straight into place


@pytest.mark.parametrize("parts", [1, 2, 4, 7])
def test_distributed_product_is_bit_identical(parts):
    ro, co_, va, b = _system(6)
    x = np.random.default_rng(3).standard_normal(ro.size - 1)
    y = co.spmv(ro, co_, va, x)
    plan = domain.DomainPlan(ro, co_, parts)
    comm = domain.PartComm(parts)
    layouts = {p: plan.part(p) for p in range(parts)}
    comm.prepare(layouts, torch.device("cpu"))
    vec = {}
    for p, L in layouts.items():
        v = torch.full((L.n_local,), np.nan, dtype=torch.float64)
        v[L.owned] = torch.from_numpy(x[L.row_begin:L.row_end])
        vec[p] = v
    comm.exchange(vec)
    for p, L in layouts.items():
        assert not torch.isnan(vec[p]).any()
        yl = co.spmv(L.local_row_offsets, L.local_columns, va[L.local_source], vec[p].numpy())
        assert np.array_equal(yl[L.owned], y[L.row_begin:L.row_end])


def test_balanced_splits_even_out_entries():
    ro, co_, va, b = _system(6)
    for parts in (2, 3, 8):
        plan = domain.DomainPlan(ro, co_, parts)
        nnz = np.diff(ro[plan.row_splits])
        widest = np.diff(ro).max()
        assert np.all(np.abs(nnz - ro[-1] / parts) <= widest), nnz


def test_plan_rejects_bad_input():
    ro, co_, va, b, _ = _golden()
    n = ro.size - 1
    for parts, splits in ((0, None), (n + 1, None), (2, [0, 5, n - 1]), (2, [0, 0, n]), (3, [0, 9, 9, n])):
        with pytest.raises(CfdxgError):
            domain.DomainPlan(ro, co_, parts, splits)
    bad = co_.copy()
    bad[0], bad[1] = bad[1], bad[0]
    with pytest.raises(CfdxgError, match="increasing"):
        domain.DomainPlan(ro, bad, 2)
    bad = co_.copy()
    bad[-1] = n
    with pytest.raises(CfdxgError, match="range"):
        domain.DomainPlan(ro, bad, 2)
    with pytest.raises(ValueError):
        domain.DomainPlan(ro, co_, 2, [0, n])
    with pytest.raises(ValueError):
        domain.PartComm(2, rank=0, world_size=3)
    with pytest.raises(ValueError):
        domain.PartComm(2, rank=0, world_size=2, owners=[1, 1])


# ------------------------------------------------------- the distributed solve
def _solve_parts(ro, co_, va, b, parts, comm, restart=30, tol=1e-8, max_iterations=500):
    plan = domain.DomainPlan(ro, co_, parts)
    local = {p: OraclePart(plan.part(p), va) for p in comm.local_parts}
    solver = domain.DistributedFGMRES(comm, local, restart=restart)
    return plan, solver.solve(domain.split_rows(plan, comm, b), max_iterations=max_iterations, tolerance=tol)


@pytest.mark.parametrize("parts", [1, 3])
def test_serial_parts_reach_the_true_residual(parts):
    ro, co_, va, b = _system(8)
    plan, (x, rep) = _solve_parts(ro, co_, va, b, parts, domain.PartComm(parts))
    xg = np.concatenate([x[p] for p in range(parts)])
    res = np.linalg.norm(b - co.spmv(ro, co_, va, xg)) / np.linalg.norm(b)
    assert rep["status_name"] == "converged" and res <= 1e-8
    assert rep["residual_relative"] == pytest.approx(res, rel=1e-6)
    xr, _ = co.solve_gmres(ro, co_, va, b, None, restart=60, tolerance=1e-12, max_iterations=3000)
    assert np.linalg.norm(xg - xr) <= 1e-6 * np.linalg.norm(xr)
    assert rep["preconditioner_applications"] == rep["iterations"]


def test_one_part_matches_undivided_amg_gmres_iterations():
    ro, co_, va, b, xg = _golden()
    amg = NativeBoomerAMGPreconditioner()
    assert amg.setup_host(ro, co_, va)
    H = co.Hierarchy([amg.export_level(l) for l in range(len(amg.hierarchy_level_sizes()))], amg.omega)
    _, ref = co.solve_gmres(ro, co_, va, b, H, restart=30, tolerance=1e-8)
    _, (x, rep) = _solve_parts(ro, co_, va, b, 1, domain.PartComm(1))
    # one part: FGMRES with the whole matrix's V-cycle; only the orthogonalisation differs
    assert abs(rep["iterations"] - ref["iterations"]) <= 1
    assert np.linalg.norm(x[0] - xg) <= 1e-6 * np.linalg.norm(xg)


def test_iteration_limit_and_zero_rhs():
    ro, co_, va, b = _system(6)
    plan, (x, rep) = _solve_parts(ro, co_, va, b, 2, domain.PartComm(2), restart=3, max_iterations=2)
    assert rep["status_name"] == "max_iterations_reached" and rep["iterations"] == 2
    plan, (x, rep) = _solve_parts(ro, co_, va, np.zeros_like(b), 2, domain.PartComm(2))
    assert rep["status_name"] == "converged" and rep["iterations"] == 0 and not any(v.any() for v in x.values())


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, parts, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ro, co_, va, b = _system(8)
        comm = domain.PartComm(parts, rank, world)
        plan, (x, rep) = _solve_parts(ro, co_, va, b, parts, comm)
        out.put((rank, {p: v for p, v in x.items()}, rep, comm.exchanges))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("parts", [2, 4])
def test_gloo_ranks_solve_one_system(parts):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, parts, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    x = {}
    for rank, xr, rep, ex in results:
        x.update(xr)
    reps = [r[2] for r in results]
    assert reps[0]["iterations"] == reps[1]["iterations"] and reps[0]["status_name"] == "converged"
    assert results[0][3] == results[1][3]                     # same number of halo exchanges
    ro, co_, va, b = _system(8)
    xg = np.concatenate([x[p] for p in range(parts)])
    assert np.linalg.norm(b - co.spmv(ro, co_, va, xg)) <= 1e-8 * np.linalg.norm(b)
    # the same parts on one process give the same iterate up to the order of the reductions
    _, (xs, rs) = _solve_parts(ro, co_, va, b, parts, domain.PartComm(parts))
    assert rs["iterations"] == reps[0]["iterations"]
    assert np.linalg.norm(np.concatenate([xs[p] for p in range(parts)]) - xg) <= 1e-9 * np.linalg.norm(xg)


# ------------------------------------------------- the distributed V-cycle
class HostOperator:
    """The oracle's product with a host CSR operator (the CPU stand-in for CudaOperator)."""

    def __init__(self, ro, co_, va, n_rows, n_cols):
        self.ro, self.co, self.va = (np.ascontiguousarray(ro, np.int64), np.ascontiguousarray(co_, np.int64),
                                     np.ascontiguousarray(va, np.float64))

    def __call__(self, x):
        return torch.from_numpy(co.spmv(self.ro, self.co, self.va, x.contiguous().numpy()))


def _hierarchy(ro, co_, va):
    amg = NativeBoomerAMGPreconditioner()
    assert amg.setup_host(ro, co_, va), amg.last_error()
    levels = [amg.export_level(l) for l in range(len(amg.hierarchy_level_sizes()))]
    return levels, amg.omega


def _distributed_amg(ro, co_, va, parts, comm, replicate_below, levels=None):
    levels, omega = levels or _hierarchy(ro, co_, va)
    plan = domain.DomainPlan(ro, co_, parts)
    dm = domain.DistributedAMG(comm, levels, omega, plan.row_splits, HostOperator, torch.device("cpu"),
                               replicate_below=replicate_below)
    return plan, dm, levels, omega


@pytest.mark.parametrize("parts,replicate_below", [(1, 4096), (2, 64), (3, 64), (5, 200), (4, 10 ** 9), (3, 16)])
def test_distributed_vcycle_is_the_undivided_vcycle_bit_for_bit(parts, replicate_below):
    ro, co_, va, b = _system(8)
    levels, omega = _hierarchy(ro, co_, va)
    plan, dm, _, _ = _distributed_amg(ro, co_, va, parts, domain.PartComm(parts), replicate_below, (levels, omega))
    if replicate_below == 64:
        assert sum(dm.dist) >= 3                                  # several split levels, then replicated ones
    H = co.Hierarchy(levels, omega)
    rng = np.random.default_rng(parts)
    for _ in range(2):
        r = rng.standard_normal(ro.size - 1)
        want = H.apply(r)
        z = {p: torch.empty(int(plan.row_splits[p + 1] - plan.row_splits[p]), dtype=torch.float64)
             for p in range(parts)}
        dm.apply({p: torch.from_numpy(r[plan.row_splits[p]:plan.row_splits[p + 1]].copy()) for p in range(parts)},
                 z)
        got = np.concatenate([z[p].numpy() for p in range(parts)])
        assert np.array_equal(got, want)


def test_coarse_blocks_follow_the_fine_blocks():
    ro, co_, va, b = _system(8)
    levels, omega = _hierarchy(ro, co_, va)
    plan, dm, _, _ = _distributed_amg(ro, co_, va, 4, domain.PartComm(4), 64, (levels, omega))
    for l in range(1, len(dm.splits)):
        S = dm.splits[l]
        assert S[0] == 0 and S[-1] == dm.n[l] and np.all(np.diff(S) > 0)
    # the first transfer: each part interpolates almost only from its own coarse block
    lv, F, S = levels[0], dm.splits[0], dm.splits[1]
    inside = 0
    for p in range(4):
        cols = lv["p_columns"][lv["p_offsets"][F[p]]:lv["p_offsets"][F[p + 1]]]
        inside += np.count_nonzero((cols >= S[p]) & (cols < S[p + 1]))
    assert inside >= 0.95 * lv["p_columns"].size


def test_fgmres_with_the_distributed_vcycle_keeps_the_iteration_count():
    ro, co_, va, b = _system(8)
    levels, omega = _hierarchy(ro, co_, va)
    its = {}
    for parts in (1, 2, 4, 7):
        comm = domain.PartComm(parts)
        plan, dm, _, _ = _distributed_amg(ro, co_, va, parts, comm, 64, (levels, omega))
        local = {p: OraclePart(plan.part(p), va, block_amg=False) for p in comm.local_parts}
        solver = domain.DistributedFGMRES(comm, local, restart=30, preconditioner=dm)
        x, rep = solver.solve(domain.split_rows(plan, comm, b), tolerance=1e-8)
        xg = np.concatenate([x[p] for p in range(parts)])
        assert rep["status_name"] == "converged"
        assert np.linalg.norm(b - co.spmv(ro, co_, va, xg)) <= 1e-8 * np.linalg.norm(b)
        its[parts] = rep["iterations"]
    assert len(set(its.values())) == 1, its                        # block-Jacobi needed 35-116 here
    _, ref = co.solve_gmres(ro, co_, va, b, co.Hierarchy(levels, omega), restart=30, tolerance=1e-8)
    assert abs(its[1] - ref["iterations"]) <= 1


def _rank_vcycle(rank, world, port, parts, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ro, co_, va, b = _system(8)
        comm = domain.PartComm(parts, rank, world)
        plan, dm, levels, omega = _distributed_amg(ro, co_, va, parts, comm, 64)
        r = np.random.default_rng(9).standard_normal(ro.size - 1)
        z = {p: torch.empty(int(plan.row_splits[p + 1] - plan.row_splits[p]), dtype=torch.float64)
             for p in comm.local_parts}
        dm.apply({p: torch.from_numpy(r[plan.row_splits[p]:plan.row_splits[p + 1]].copy())
                  for p in comm.local_parts}, z)
        local = {p: OraclePart(plan.part(p), va, block_amg=False) for p in comm.local_parts}
        x, rep = domain.DistributedFGMRES(comm, local, preconditioner=dm).solve(domain.split_rows(plan, comm, b),
                                                                               tolerance=1e-8)
        out.put((rank, {p: v.numpy() for p, v in z.items()}, x, rep["iterations"]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_ranks_run_the_distributed_vcycle():
    world, parts = 2, 4
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_vcycle, args=(r, world, port, parts, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ro, co_, va, b = _system(8)
    levels, omega = _hierarchy(ro, co_, va)
    want = co.Hierarchy(levels, omega).apply(np.random.default_rng(9).standard_normal(ro.size - 1))
    z, x = {}, {}
    for rank, zr, xr, its in results:
        z.update(zr)
        x.update(xr)
    assert np.array_equal(np.concatenate([z[p] for p in range(parts)]), want)
    assert results[0][3] == results[1][3]
    xg = np.concatenate([x[p] for p in range(parts)])
    assert np.linalg.norm(b - co.spmv(ro, co_, va, xg)) <= 1e-8 * np.linalg.norm(b)


def test_one_level_hierarchy_uses_the_dense_coarsest_solve():
    # 12 rows: the setup stops at one level, whose V-cycle is the pivoted dense solve
    n = 12
    D = 2.0 * np.eye(n) - 0.9 * np.eye(n, k=1) - 0.9 * np.eye(n, k=-1)
    D[0, 0] += 1.0
    ro = np.concatenate([[0], np.cumsum(np.count_nonzero(D, axis=1))])
    co_ = np.nonzero(D)[1]
    va = D[np.nonzero(D)]
    levels, omega = _hierarchy(ro, co_, va)
    assert len(levels) == 1
    plan, dm, _, _ = _distributed_amg(ro, co_, va, 3, domain.PartComm(3), 4096, (levels, omega))
    r = np.random.default_rng(1).standard_normal(n)
    S = plan.row_splits
    z = {p: torch.empty(int(S[p + 1] - S[p]), dtype=torch.float64) for p in range(3)}
    dm.apply({p: torch.from_numpy(r[S[p]:S[p + 1]].copy()) for p in range(3)}, z)
    got = np.concatenate([z[p].numpy() for p in range(3)])
    assert np.array_equal(got, co.Hierarchy(levels, omega).apply(r))
    np.testing.assert_allclose(D @ got, r, rtol=0, atol=1e-12)
