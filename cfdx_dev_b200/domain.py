"""Domain decomposition: one pressure system split over several GPUs.

The reference solves each pressure system on one rank
(core/linalg/linear_solver_dispatch.h:227-234 takes the whole matrix); this
module spreads one system over row blocks ("parts"), any number per process
and one process per GPU:

* ``DomainPlan`` -- the host-built partition and halo plan of the C ABI
  (``cfdxg_domain_plan_*``): per part its local rows in the numbering
  [ghosts below | owned | ghosts above], its diagonal block, and per
  neighbour the ghost slice it receives and the owned rows it sends;
* ``PartComm`` -- which process holds which part, the sum over processes
  (``torch.distributed.all_reduce``) and the halo exchange (copies between
  parts of one process, ``batch_isend_irecv`` between processes: NCCL
  send/recv over NVLink on GPUs, gloo on CPU);
* ``CudaPart`` -- a part on the device: its local matrix (the library's FP64
  SpMV, which sums each row in the global order, so a distributed product is
  bit-identical to the undivided one) and its own native AMG on the diagonal
  block (block-Jacobi, i.e. additive Schwarz without overlap);
* ``DistributedAMG`` -- the undivided native-AMG hierarchy (the reference's
  bit-exact setup, run on every process) applied as one V-cycle over the
  parts: each level is split into row blocks with its own halo plan, the
  transfers P and P^T get rectangular plans, and below a size threshold the
  coarse levels run replicated on every process after one all-reduce.  The
  cycle is the reference's (amg_preconditioner.h:2369-2443, 2564-2666) with
  every sum in the reference's order, so it equals the undivided V-cycle bit
  for bit and the solve keeps the one-GPU iteration count;
* ``DistributedFGMRES`` -- restarted right-preconditioned FGMRES in FP64 over
  the parts, classical Gram-Schmidt applied twice (one reduction of j+1
  values per pass instead of j+1 reductions of one), the Hessenberg and
  Givens work on the host as in core/linalg/gmres_solver.h:28-600, and the
  same stopping rule: the FP64 true relative residual ||b - Ax|| / ||b||.

Every control decision is taken from reduced values that are identical on
all processes, so all ranks run the same collectives in the same order.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from .api import CfdxgError, Context, NativeBoomerAMGPreconditioner, SparseMatrix

CONVERGED, MAX_ITER_REACHED, DIVERGED = 0, 1, 2
_STATUS = {CONVERGED: "converged", MAX_ITER_REACHED: "max_iterations_reached", DIVERGED: "diverged"}


@dataclass
class PartLayout:
    """One part of a DomainPlan (all arrays int64 unless noted)."""

    index: int
    row_begin: int
    row_end: int
    n_local: int
    owned_offset: int
    local_row_offsets: np.ndarray
    local_columns: np.ndarray
    local_source: np.ndarray
    block_row_offsets: np.ndarray
    block_columns: np.ndarray
    block_source: np.ndarray
    neighbours: np.ndarray        # int32
    recv_offsets: np.ndarray
    recv_start: np.ndarray
    ghost_rows: np.ndarray
    send_offsets: np.ndarray
    send_rows: np.ndarray
    col_begin: int = 0
    col_end: int = 0
    n_local_rows: int = 0
    first_row: int = 0

    @property
    def n_owned(self) -> int:
        """Owned rows."""
        return self.row_end - self.row_begin

    @property
    def n_owned_cols(self) -> int:
        return self.col_end - self.col_begin

    @property
    def owned(self) -> slice:
        """The owned entries' slice of the local (input) vector."""
        return slice(self.owned_offset, self.owned_offset + self.n_owned_cols)

    @property
    def rows(self) -> slice:
        """The owned rows' slice of a local product's output."""
        return slice(self.first_row, self.first_row + self.n_owned)

    def local_to_global(self) -> np.ndarray:
        """Global index of every local vector position."""
        g = np.empty(self.n_local, np.int64)
        below = self.owned_offset
        g[:below] = self.ghost_rows[:below]
        g[self.owned] = np.arange(self.col_begin, self.col_end)
        g[below + self.n_owned_cols:] = self.ghost_rows[below:]
        return g

    def recv_slice(self, k: int) -> slice:
        s = int(self.recv_start[k])
        return slice(s, s + int(self.recv_offsets[k + 1] - self.recv_offsets[k]))

    def send_slice(self, k: int) -> slice:
        return slice(int(self.send_offsets[k]), int(self.send_offsets[k + 1]))


class DomainPlan:
    """Row-block partition with halos of a CSR pattern: square (cfdxg_domain_plan_create)
    or, given ``n_cols`` and ``col_splits``, rectangular (cfdxg_domain_plan_create_rect)."""

    def __init__(self, row_offsets, columns, parts: int, row_splits=None, n_cols=None, col_splits=None):
        self.lib = N.load()
        self.handle = None
        ro = np.ascontiguousarray(row_offsets, np.int64)
        co = np.ascontiguousarray(columns, np.int64)
        self.n = ro.size - 1
        splits = None if row_splits is None else np.ascontiguousarray(row_splits, np.int64)
        if splits is not None and splits.size != parts + 1:
            raise ValueError("row_splits needs parts + 1 entries")
        h = C.c_void_p()
        if n_cols is None:
            rc = self.lib.cfdxg_domain_plan_create(self.n, N.ptr(ro), N.ptr(co), int(parts), N.ptr(splits),
                                                   C.byref(h))
        else:
            cs = np.ascontiguousarray(col_splits, np.int64)
            if splits is None or cs.size != parts + 1:
                raise ValueError("a rectangular plan needs row and column splits of parts + 1 entries")
            rc = self.lib.cfdxg_domain_plan_create_rect(self.n, int(n_cols), N.ptr(ro), N.ptr(co), int(parts),
                                                        N.ptr(splits), N.ptr(cs), C.byref(h))
        if rc != 0:
            raise CfdxgError(rc, self.lib.cfdxg_domain_last_error().decode())
        self.handle = h
        self.row_splits = np.empty(parts + 1, np.int64)
        self.col_splits = np.empty(parts + 1, np.int64)
        self.parts = self.lib.cfdxg_domain_plan_parts(h, N.ptr(self.row_splits), N.ptr(self.col_splits))

    def part(self, p: int) -> PartLayout:
        info = N.DomainPartInfo()
        rc = self.lib.cfdxg_domain_plan_info(self.handle, int(p), C.byref(info))
        if rc != 0:
            raise CfdxgError(rc, self.lib.cfdxg_domain_last_error().decode())
        n_own, nb = info.row_end - info.row_begin, info.n_neighbours
        sizes = dict(local_row_offsets=info.n_local_rows + 1, local_columns=info.nnz_local,
                     local_source=info.nnz_local,
                     block_row_offsets=n_own + 1, block_columns=info.nnz_block, block_source=info.nnz_block,
                     neighbours=nb, recv_offsets=nb + 1, recv_start=nb, ghost_rows=info.n_recv,
                     send_offsets=nb + 1, send_rows=info.n_send)
        arrays = {k: np.empty(v, np.int32 if k == "neighbours" else np.int64) for k, v in sizes.items()}
        out = N.DomainPartArrays(**{k: arrays[k].ctypes.data for k in N.DOMAIN_ARRAYS})
        rc = self.lib.cfdxg_domain_plan_export(self.handle, int(p), C.byref(out))
        if rc != 0:
            raise CfdxgError(rc, self.lib.cfdxg_domain_last_error().decode())
        return PartLayout(index=int(p), row_begin=info.row_begin, row_end=info.row_end, n_local=info.n_local,
                          owned_offset=info.owned_offset, col_begin=info.col_begin, col_end=info.col_end,
                          n_local_rows=info.n_local_rows, first_row=info.first_row, **arrays)

    def __del__(self):  # pragma: no cover
        try:
            if self.handle:
                self.lib.cfdxg_domain_plan_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


def contiguous_owners(parts: int, world_size: int) -> list[int]:
    """Part p goes to process p * world_size // parts (blocks of neighbouring parts)."""
    if world_size < 1 or parts < world_size:
        raise ValueError("need at least one part per process")
    return [p * world_size // parts for p in range(parts)]


class PartComm:
    """Which process holds which part, and the collectives between parts.

    ``rank``/``world_size`` are those of ``torch.distributed`` (one process
    per GPU); with ``world_size == 1`` every part is local and no process
    group is needed."""

    def __init__(self, parts: int, rank: int = 0, world_size: int = 1, owners=None, group=None):
        self.parts, self.rank, self.world_size, self.group = parts, rank, world_size, group
        self.owners = list(owners) if owners is not None else contiguous_owners(parts, world_size)
        if len(self.owners) != parts or any(o < 0 or o >= world_size for o in self.owners):
            raise ValueError("owners must map every part to a process")
        self.local_parts = [p for p in range(parts) if self.owners[p] == rank]
        if not self.local_parts:
            raise ValueError(f"process {rank} holds no part")
        self.exchanges = 0

    def allreduce_(self, t: torch.Tensor) -> torch.Tensor:
        """Sum over processes, in place (parts of one process are summed by the caller)."""
        if self.world_size > 1:
            import torch.distributed as dist
            dist.all_reduce(t, group=self.group)
        return t

    def prepare(self, layouts: dict[int, PartLayout], device) -> None:
        """The halo of the solver's own system (its square plan)."""
        self._halo = Halo(self, layouts, device)

    def exchange(self, vectors: dict[int, torch.Tensor]) -> None:
        """Fill the ghost slices of every local part's local vector from the owners' owned values."""
        self.exchanges += 1
        self._halo.exchange(vectors)

    def allgather(self, pieces: dict[int, torch.Tensor], splits, n: int) -> torch.Tensor:
        """The whole vector from the parts' owned pieces (a zero-padded sum over processes)."""
        first = next(iter(pieces.values()))
        full = torch.zeros(n, dtype=first.dtype, device=first.device)
        for p, v in pieces.items():
            full[int(splits[p]):int(splits[p + 1])] = v
        return self.allreduce_(full)


class Halo:
    """Ghost exchange of one plan: the local vectors of the process's parts are
    filled from the owners' owned entries -- copies between local parts,
    ``batch_isend_irecv`` between processes, posted on both sides in
    (source part, destination part) order."""

    def __init__(self, comm: PartComm, layouts: dict[int, PartLayout], device):
        self.comm = comm
        self._send, self._copy, self._recv = [], [], []
        for p in comm.local_parts:
            L = layouts[p]
            for k, q in enumerate(L.neighbours.tolist()):
                rs, ss = L.recv_slice(k), L.send_slice(k)
                if rs.stop > rs.start:
                    if comm.owners[q] == comm.rank:
                        src = layouts[q]
                        idx = L.ghost_rows[L.recv_offsets[k]:L.recv_offsets[k + 1]] - src.col_begin + src.owned_offset
                        self._copy.append((p, rs, q, torch.as_tensor(idx, device=device)))
                    else:
                        self._recv.append(((q, p), rs))
                if ss.stop > ss.start and comm.owners[q] != comm.rank:
                    idx = L.send_rows[ss] + L.owned_offset
                    self._send.append(((p, q), torch.as_tensor(idx, device=device)))
        self._send.sort(key=lambda e: e[0])
        self._recv.sort(key=lambda e: e[0])

    def exchange(self, vectors: dict[int, torch.Tensor]) -> None:
        for p, rs, q, idx in self._copy:
            vectors[p][rs] = vectors[q].index_select(0, idx)
        if not self._send and not self._recv:
            return
        import torch.distributed as dist
        comm = self.comm
        ops, bufs = [], []
        for (p, q), idx in self._send:
            buf = vectors[p].index_select(0, idx)
            bufs.append(buf)
            ops.append(dist.P2POp(dist.isend, buf, comm.owners[q], comm.group, tag=p * comm.parts + q))
        for (q, p), rs in self._recv:
            ops.append(dist.P2POp(dist.irecv, vectors[p][rs], comm.owners[q], comm.group, tag=q * comm.parts + p))
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class CudaPart:
    """A part on the device: local FP64 SpMV and a native AMG V-cycle on its diagonal block."""

    def __init__(self, ctx: Context, layout: PartLayout, values, precision: str = "fp64", block_amg: bool = True,
                 **amg_options):
        if not torch.cuda.is_available():
            raise RuntimeError("CudaPart needs a CUDA device (the distributed path has no CPU fallback)")
        self.ctx, self.layout = ctx, layout
        self.lib = ctx.lib
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.ExternalStream(ctx.stream, device=self.device)
        self.A = SparseMatrix.from_csr(ctx, layout.local_row_offsets, layout.local_columns,
                                       np.asarray(values)[layout.local_source])
        self.amg = None
        if block_amg:
            self.B = SparseMatrix.from_csr(ctx, layout.block_row_offsets, layout.block_columns,
                                           np.asarray(values)[layout.block_source])
            self.amg = NativeBoomerAMGPreconditioner(ctx, precision=precision, **amg_options)
            if not self.amg.setup(self.B):
                raise CfdxgError(N.CFDXG_ERR_SETUP,
                                 f"part {layout.index}: AMG setup failed: {self.amg.last_error()}")
        self._y = torch.empty(layout.n_local, dtype=torch.float64, device=self.device)

    def matvec(self, x_local: torch.Tensor) -> torch.Tensor:
        """Owned rows of A_loc x_loc (ghosts filled); a view of an internal buffer."""
        self.ctx.check(self.lib.cfdxg_matrix_spmv(self.ctx.handle, self.A.handle, C.c_void_p(x_local.data_ptr()),
                                                  C.c_void_p(self._y.data_ptr()), N.CFDXG_MEM_DEVICE), "part SpMV")
        return self._y[self.layout.owned]

    def precondition(self, r: torch.Tensor, z: torch.Tensor) -> None:
        """z = one V-cycle of the part's AMG on r (both owned-length, contiguous)."""
        self.ctx.check(self.lib.cfdxg_amg_apply(self.ctx.handle, self.amg.handle, C.c_void_p(r.data_ptr()),
                                                C.c_void_p(z.data_ptr()), N.CFDXG_MEM_DEVICE), "part V-cycle")


class DistributedFGMRES:
    """Restarted FGMRES(m) over the parts a process holds (see the module docstring).

    ``parts`` maps each local part to an object with ``layout``, ``device``,
    ``matvec(x_local) -> owned y`` and ``precondition(r, z)``; a
    ``preconditioner`` with ``apply(r, z)`` over all local parts at once (the
    distributed V-cycle) replaces the parts' own (block-Jacobi) one."""

    def __init__(self, comm: PartComm, parts: dict, restart: int = 30, preconditioner=None):
        if sorted(parts) != comm.local_parts:
            raise ValueError("parts must be exactly the process's local parts")
        if restart < 1:
            raise ValueError("restart must be at least 1")
        self.comm, self.parts, self.m = comm, parts, restart
        self.preconditioner = preconditioner
        first = parts[comm.local_parts[0]]
        self.device = first.device
        self.stream = getattr(first, "stream", None)
        comm.prepare({p: P.layout for p, P in parts.items()}, self.device)
        f64 = dict(dtype=torch.float64, device=self.device)
        m = restart
        self.V = {p: torch.zeros(m + 1, P.layout.n_owned, **f64) for p, P in parts.items()}
        # Z rows and the iterate are local vectors (halo slots included), so the
        # exchange fills their ghosts in place before a product
        self.Z = {p: torch.zeros(m, P.layout.n_local, **f64) for p, P in parts.items()}
        self.X = {p: torch.zeros(P.layout.n_local, **f64) for p, P in parts.items()}
        self.applications = 0

    # ------------------------------------------------------------ reductions
    def _sum(self, local: torch.Tensor) -> torch.Tensor:
        return self.comm.allreduce_(local)

    def _norm(self, vecs: dict) -> float:
        s = sum((v * v).sum() for v in vecs.values()).reshape(1)
        return math.sqrt(float(self._sum(s)[0]))

    def _residual(self, b: dict) -> dict:
        self.comm.exchange(self.X)
        return {p: b[p] - P.matvec(self.X[p]) for p, P in self.parts.items()}

    # ------------------------------------------------------------------ solve
    def solve(self, rhs: dict, x0: dict | None = None, max_iterations: int = 1000, tolerance: float = 1e-8) -> dict:
        """Solve for the local parts' owned rows; returns (x per part as numpy, report)."""
        with torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext():
            return self._solve(rhs, x0, max_iterations, tolerance)

    def _solve(self, rhs, x0, max_iterations, tolerance):
        parts, m = self.parts, self.m
        self.applications = 0
        b = {p: torch.as_tensor(np.asarray(rhs[p], np.float64), device=self.device) for p in parts}
        for p, P in parts.items():
            if b[p].numel() != P.layout.n_owned:
                raise ValueError(f"part {p}: right-hand side has {b[p].numel()} rows, expected {P.layout.n_owned}")
            own = self.X[p][P.layout.owned]
            own.zero_()
            if x0 is not None:
                own.copy_(torch.as_tensor(np.asarray(x0[p], np.float64), device=self.device))
        bnorm = self._norm(b)
        report = dict(status=CONVERGED, iterations=0, cycles=0, residual=0.0, residual_relative=0.0,
                      preconditioner_applications=0)
        if bnorm == 0.0:
            for p, P in parts.items():
                self.X[p][P.layout.owned].zero_()
            return self._finish(report)
        target = tolerance * bnorm
        it = 0
        while True:
            r = self._residual(b)
            beta = self._norm(r)
            report.update(residual=beta, residual_relative=beta / bnorm)
            if not math.isfinite(beta):
                report["status"] = DIVERGED
                break
            if beta <= target:
                report["status"] = CONVERGED
                break
            if it >= max_iterations:
                report["status"] = MAX_ITER_REACHED
                break
            report["cycles"] += 1
            for p in parts:
                self.V[p][0] = r[p] / beta
            H = np.zeros((m + 1, m))
            g = np.zeros(m + 1)
            g[0] = beta
            cs, sn = np.zeros(m), np.zeros(m)
            k = 0
            for j in range(m):
                if it >= max_iterations:
                    break
                w = {}
                if self.preconditioner is not None:
                    self.preconditioner.apply({p: self.V[p][j] for p in parts},
                                              {p: self.Z[p][j][P.layout.owned] for p, P in parts.items()})
                else:
                    for p, P in parts.items():
                        P.precondition(self.V[p][j], self.Z[p][j][P.layout.owned])
                self.applications += 1
                self.comm.exchange({p: self.Z[p][j] for p in parts})
                for p, P in parts.items():
                    w[p] = P.matvec(self.Z[p][j]).clone()
                h = np.zeros(j + 1)
                for _ in range(2):          # classical Gram-Schmidt, twice
                    c = self._sum(sum(self.V[p][:j + 1] @ w[p] for p in parts))
                    for p in parts:
                        w[p] -= self.V[p][:j + 1].T @ c
                    h += c.cpu().numpy()
                hn = self._norm(w)
                it += 1
                k = j + 1
                H[:j + 1, j] = h
                H[j + 1, j] = hn
                for i in range(j):          # previous Givens rotations
                    a, bb = H[i, j], H[i + 1, j]
                    H[i, j], H[i + 1, j] = cs[i] * a + sn[i] * bb, -sn[i] * a + cs[i] * bb
                den = math.hypot(H[j, j], H[j + 1, j])
                if not math.isfinite(den) or den == 0.0:
                    k = j
                    break
                cs[j], sn[j] = H[j, j] / den, H[j + 1, j] / den
                H[j, j], H[j + 1, j] = den, 0.0
                g[j], g[j + 1] = cs[j] * g[j], -sn[j] * g[j]
                if hn == 0.0 or abs(g[j + 1]) <= target:
                    break
                for p in parts:
                    self.V[p][j + 1] = w[p] / hn
            if k > 0:
                y = np.zeros(k)
                for i in range(k - 1, -1, -1):
                    y[i] = (g[i] - H[i, i + 1:k] @ y[i + 1:k]) / H[i, i]
                yt = torch.as_tensor(y, device=self.device)
                for p, P in parts.items():
                    self.X[p][P.layout.owned] += self.Z[p][:k, P.layout.owned].T @ yt
            elif it >= max_iterations:
                continue
            else:                           # no usable direction: stop on the true residual
                r = self._residual(b)
                beta = self._norm(r)
                report.update(residual=beta, residual_relative=beta / bnorm,
                              status=CONVERGED if beta <= target else DIVERGED)
                break
        report["iterations"] = it
        return self._finish(report)

    def _finish(self, report):
        report["preconditioner_applications"] = self.applications
        report["status_name"] = _STATUS[report["status"]]
        x = {p: self.X[p][P.layout.owned].cpu().numpy().copy() for p, P in self.parts.items()}
        return x, report


def _transpose(n_rows: int, n_cols: int, ro, co, va):
    """CSR of the transpose; each of its rows lists the original rows in increasing order."""
    counts = np.bincount(co, minlength=n_cols)
    tro = np.zeros(n_cols + 1, np.int64)
    np.cumsum(counts, out=tro[1:])
    order = np.argsort(co, kind="stable")
    rows = np.repeat(np.arange(n_rows, dtype=np.int64), np.diff(ro))
    return tro, rows[order], np.ascontiguousarray(va[order])


def _augment(n_rows: int, ro, co, va, shift: int, first=0):
    """[I | M]: row i is 1 at column first + i, then M's row with columns + shift.

    Applied to [x; y] it sums 1*x_i and then M's entries in row order, which
    is the reference's prolongation x_i += sum_k p_ik y_k entry by entry."""
    nnz = np.diff(ro)
    aro = np.zeros(n_rows + 1, np.int64)
    np.cumsum(nnz + 1, out=aro[1:])
    aco = np.empty(aro[-1], np.int64)
    ava = np.empty(aro[-1])
    head = aro[:-1]
    aco[head] = first + np.arange(n_rows)
    ava[head] = 1.0
    body = np.ones(aro[-1], bool)
    body[head] = False
    aco[body] = co + shift
    ava[body] = va
    return aro, aco, ava


def _coarse_splits(fine_splits, p_ro, p_co, p_va, n_coarse: int):
    """Row blocks of the next level that follow the fine blocks.  A coarse
    point's home is the first fine row that P maps to it with weight 1 (its
    C point; RS numbers coarse points in fine order, so homes nearly
    increase); coarse block k starts at the number of coarse points whose home
    lies below fine split k."""
    parts = len(fine_splits) - 1
    n_fine = p_ro.size - 1
    rows = np.repeat(np.arange(n_fine, dtype=np.int64), np.diff(p_ro))
    home = np.full(n_coarse, n_fine, np.int64)
    one = p_va == 1.0
    np.minimum.at(home, p_co[one], rows[one])
    s = np.zeros(parts + 1, np.int64)
    s[parts] = n_coarse
    for k in range(1, parts):
        v = int(np.count_nonzero(home < int(fine_splits[k])))
        s[k] = min(max(v, s[k - 1] + 1), n_coarse - (parts - k))
    return s


class DistributedAMG:
    """One V-cycle of an undivided AMG hierarchy over the parts of a ``PartComm``.

    ``levels`` are the hierarchy's levels as ``NativeBoomerAMGPreconditioner.
    export_level`` gives them (each process holds the whole hierarchy; the
    setup is the reference's, bit-exact and deterministic, so every process
    builds the same one); ``row_splits`` are the finest level's blocks.
    ``make_operator(row_offsets, columns, values, n_rows, n_cols)`` returns a
    callable computing the product with a host CSR operator on the vectors'
    device (``CudaOperator`` for the library's SpMV).

    Levels with at least ``replicate_below`` rows (and two per part) are split
    into row blocks that follow the finer level's; the first level below that
    and all coarser ones run on every process, entered by one all-reduce of the
    fine residual.  The arithmetic is the reference's damped-Jacobi V(pre,
    post) cycle in its summation order: products sum each row in the global
    order, the restriction gathers P^T rows in increasing fine order (the
    order of the reference's scatter), the prolongation adds P's entries one at
    a time, and the coarsest level is the pivoted dense solve (at most 16 rows)
    or 24 sweeps (amg_preconditioner.h:2369-2443, 2564-2666)."""

    def __init__(self, comm: PartComm, levels: list, omega: float, row_splits, make_operator, device,
                 pre_sweeps: int = 6, post_sweeps: int = 6, replicate_below: int = 4096):
        self.comm, self.device = comm, device
        self.omega, self.pre, self.post = float(omega), int(pre_sweeps), int(post_sweeps)
        f64 = dict(dtype=torch.float64, device=device)
        L = len(levels)
        n = [int(lv["inv_diag"].size) for lv in levels]
        parts = comm.parts
        # a one-level hierarchy of at most 16 rows is the dense coarsest solve: replicated
        dist = [not (L == 1 and n[0] <= 16)]
        for l in range(1, L):
            dist.append(dist[-1] and n[l] >= max(replicate_below, 2 * parts) and not (l == L - 1 and n[l] <= 16))
        self.L, self.n, self.dist = L, n, dist
        self.splits = [np.ascontiguousarray(row_splits, np.int64)]
        self.levels = []
        for l in range(L):
            lv = levels[l]
            last = l + 1 == L
            d = {}
            if dist[l]:
                S = self.splits[l]
                plan = DomainPlan(lv["row_offsets"], lv["columns"], parts, S)
                lay = {p: plan.part(p) for p in comm.local_parts}
                d["layouts"] = lay
                d["halo"] = Halo(comm, lay, device)
                d["A"] = {p: make_operator(L_.local_row_offsets, L_.local_columns, lv["values"][L_.local_source],
                                           L_.n_local_rows, L_.n_local) for p, L_ in lay.items()}
                d["inv"] = {p: torch.as_tensor(lv["inv_diag"][L_.row_begin:L_.row_end], **f64)
                            for p, L_ in lay.items()}
                if not last:
                    pro, pco, pva = lv["p_offsets"], lv["p_columns"], lv["p_values"]
                    nc = n[l + 1]
                    tro, tco, tva = _transpose(n[l], nc, pro, pco, pva)
                    if dist[l + 1]:
                        Sc = _coarse_splits(S, pro, pco, pva, nc)
                        self.splits.append(Sc)
                        rplan = DomainPlan(tro, tco, parts, Sc, n_cols=n[l], col_splits=S)
                        rl = {p: rplan.part(p) for p in comm.local_parts}
                        d["R_layouts"], d["R_halo"] = rl, Halo(comm, rl, device)
                        d["R"] = {p: make_operator(L_.local_row_offsets, L_.local_columns, tva[L_.local_source],
                                                   L_.n_local_rows, L_.n_local) for p, L_ in rl.items()}
                        pplan = DomainPlan(pro, pco, parts, S, n_cols=nc, col_splits=Sc)
                        pl = {p: pplan.part(p) for p in comm.local_parts}
                        d["P_layouts"], d["P_halo"] = pl, Halo(comm, pl, device)
                        d["AUG"] = {}
                        for p, L_ in pl.items():
                            aro, aco, ava = _augment(L_.n_owned, L_.local_row_offsets, L_.local_columns,
                                                     pva[L_.local_source], L_.n_owned)
                            d["AUG"][p] = make_operator(aro, aco, ava, L_.n_owned, L_.n_owned + L_.n_local)
                    else:
                        # the next level is replicated: the fine residual is gathered whole
                        d["R_full"] = make_operator(tro, tco, tva, nc, n[l])
                        d["AUG"] = {}
                        for p, L_ in lay.items():
                            r0, r1 = L_.row_begin, L_.row_end
                            sub_ro = pro[r0:r1 + 1] - pro[r0]
                            sl = slice(int(pro[r0]), int(pro[r1]))
                            aro, aco, ava = _augment(r1 - r0, sub_ro, pco[sl], pva[sl], r1 - r0)
                            d["AUG"][p] = make_operator(aro, aco, ava, r1 - r0, (r1 - r0) + nc)
            else:
                d["A_full"] = make_operator(lv["row_offsets"], lv["columns"], lv["values"], n[l], n[l])
                d["inv_full"] = torch.as_tensor(lv["inv_diag"], **f64)
                if last and n[l] <= 16:
                    d["dense"] = (lv["row_offsets"].copy(), lv["columns"].copy(), lv["values"].copy())
                if not last:
                    pro, pco, pva = lv["p_offsets"], lv["p_columns"], lv["p_values"]
                    tro, tco, tva = _transpose(n[l], n[l + 1], pro, pco, pva)
                    d["R_full"] = make_operator(tro, tco, tva, n[l + 1], n[l])
                    aro, aco, ava = _augment(n[l], pro, pco, pva, n[l])
                    d["AUG_full"] = make_operator(aro, aco, ava, n[l], n[l] + n[l + 1])
            self.levels.append(d)

    # ---------------------------------------------------------------- cycle
    def apply(self, r: dict, z: dict) -> None:
        """z = V-cycle(r) for every local part (owned pieces of the finest level)."""
        if not self.dist[0]:
            S = self.splits[0]
            x = self._cycle_full(0, self.comm.allgather(r, S, self.n[0]))
            for p in z:
                z[p].copy_(x[int(S[p]):int(S[p + 1])])
            return
        x = self._cycle_split(0, r)
        for p in z:
            z[p].copy_(x[p])

    def _smooth_split(self, l, r, x, sweeps, from_zero):
        d = self.levels[l]
        for s in range(sweeps):
            if s == 0 and from_zero:        # A * 0 is +0: the same update without the product
                ax = {p: torch.zeros_like(r[p]) for p in r}
            else:
                d["halo"].exchange(x)
                ax = {p: d["A"][p](x[p])[L_.rows] for p, L_ in d["layouts"].items()}
            for p, L_ in d["layouts"].items():
                x[p][L_.owned] += self.omega * (d["inv"][p] * (r[p] - ax[p]))

    def _cycle_split(self, l, r):
        d = self.levels[l]
        lay = d["layouts"]
        x = {p: torch.zeros(L_.n_local, dtype=torch.float64, device=self.device) for p, L_ in lay.items()}
        if l + 1 == self.L:                 # a split coarsest level: 24 sweeps from zero
            self._smooth_split(l, r, x, 24, True)
            return {p: x[p][L_.owned] for p, L_ in lay.items()}
        self._smooth_split(l, r, x, self.pre, True)
        d["halo"].exchange(x)
        res = {p: r[p] - d["A"][p](x[p])[L_.rows] for p, L_ in lay.items()}
        own = {p: x[p][L_.owned] for p, L_ in lay.items()}
        if self.dist[l + 1]:
            rl = d["R_layouts"]
            loc = {p: torch.zeros(R_.n_local, dtype=torch.float64, device=self.device) for p, R_ in rl.items()}
            for p, R_ in rl.items():
                loc[p][R_.owned] = res[p]
            d["R_halo"].exchange(loc)
            rc = {p: d["R"][p](loc[p]).clone() for p in rl}
            xc = self._cycle_split(l + 1, rc)
            pl = d["P_layouts"]
            cl = {p: torch.zeros(P_.n_local, dtype=torch.float64, device=self.device) for p, P_ in pl.items()}
            for p, P_ in pl.items():
                cl[p][P_.owned] = xc[p]
            d["P_halo"].exchange(cl)
            for p in lay:
                own[p].copy_(d["AUG"][p](torch.cat([own[p], cl[p]])))
        else:
            full = self.comm.allgather(res, self.splits[l], self.n[l])
            xc = self._cycle_full(l + 1, d["R_full"](full).clone())
            for p in lay:
                own[p].copy_(d["AUG"][p](torch.cat([own[p], xc])))
        self._smooth_split(l, r, x, self.post, False)
        return {p: x[p][L_.owned] for p, L_ in lay.items()}

    def _smooth_full(self, l, r, x, sweeps, from_zero):
        d = self.levels[l]
        for s in range(sweeps):
            ax = torch.zeros_like(r) if (s == 0 and from_zero) else d["A_full"](x)
            x += self.omega * (d["inv_full"] * (r - ax))

    def _cycle_full(self, l, r):
        d = self.levels[l]
        if l + 1 == self.L:
            if "dense" in d:
                return torch.as_tensor(_dense_coarsest(*d["dense"], r.cpu().numpy()), device=self.device)
            x = torch.zeros_like(r)
            self._smooth_full(l, r, x, 24, True)
            return x
        x = torch.zeros_like(r)
        self._smooth_full(l, r, x, self.pre, True)
        res = r - d["A_full"](x)
        xc = self._cycle_full(l + 1, d["R_full"](res).clone())
        x = d["AUG_full"](torch.cat([x, xc])).clone()
        self._smooth_full(l, r, x, self.post, False)
        return x


def _dense_coarsest(ro, co, va, b):
    """Pivoted Gaussian elimination of the coarsest level (at most 16 rows), as
    smooth_coarsest does it (amg_preconditioner.h:2564-2666): the entries
    summed into a dense matrix, partial pivoting on the largest magnitude,
    singular below 128 eps max(1, max|a|)."""
    n = ro.size - 1
    m = [[0.0] * n for _ in range(n)]
    rhs = [float(v) for v in b]
    for i in range(n):
        for k in range(int(ro[i]), int(ro[i + 1])):
            m[i][int(co[k])] += float(va[k])
    scale = 0.0
    for row in m:
        for v in row:
            scale = max(scale, abs(v))
    tol = 128.0 * np.finfo(np.float64).eps * max(1.0, scale)
    for k in range(n):
        piv, pa = k, abs(m[k][k])
        for i in range(k + 1, n):
            if abs(m[i][k]) > pa:
                pa, piv = abs(m[i][k]), i
        if not math.isfinite(pa) or pa <= tol:
            raise CfdxgError(N.CFDXG_ERR_SETUP, "singular coarsest level")
        if piv != k:
            m[k][k:], m[piv][k:] = m[piv][k:], m[k][k:]
            rhs[k], rhs[piv] = rhs[piv], rhs[k]
        dg = m[k][k]
        for i in range(k + 1, n):
            f = m[i][k] / dg
            if not math.isfinite(f):
                raise CfdxgError(N.CFDXG_ERR_SETUP, "non-finite elimination factor")
            m[i][k] = 0.0
            for j in range(k + 1, n):
                m[i][j] -= f * m[k][j]
            rhs[i] -= f * rhs[k]
    sol = [0.0] * n
    for i in range(n - 1, -1, -1):
        acc = rhs[i]
        for j in range(i + 1, n):
            acc -= m[i][j] * sol[j]
        if not math.isfinite(m[i][i]) or abs(m[i][i]) <= tol:
            raise CfdxgError(N.CFDXG_ERR_SETUP, "singular coarsest level")
        sol[i] = acc / m[i][i]
    return np.array(sol)


class CudaOperator:
    """A host CSR operator (n_rows x n_cols) on the device through the library's
    FP64 SpMV (rows summed in order); padded to a square matrix, whose extra
    rows are empty.  Calling it returns a view of an internal buffer."""

    def __init__(self, ctx: Context, ro, co, va, n_rows: int, n_cols: int):
        self.ctx, self.lib = ctx, ctx.lib
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.n_rows, self.n_cols = int(n_rows), int(n_cols)
        n = max(self.n_rows, self.n_cols)
        ro = np.asarray(ro, np.int64)
        self.A = None
        if ro[-1] > 0:
            ro_sq = np.concatenate([ro, np.full(n - self.n_rows, ro[-1], np.int64)])
            self.A = SparseMatrix.from_csr(ctx, ro_sq, co, va)
        self._x = torch.zeros(n, dtype=torch.float64, device=self.device) if self.n_cols < n else None
        self._y = torch.zeros(n, dtype=torch.float64, device=self.device)

    def __call__(self, x: torch.Tensor) -> torch.Tensor:
        if self.A is None:
            return self._y[:self.n_rows]
        if self._x is not None:
            self._x[:self.n_cols].copy_(x)
            x = self._x
        elif not x.is_contiguous():
            x = x.contiguous()
        self.ctx.check(self.lib.cfdxg_matrix_spmv(self.ctx.handle, self.A.handle, C.c_void_p(x.data_ptr()),
                                                  C.c_void_p(self._y.data_ptr()), N.CFDXG_MEM_DEVICE), "operator")
        return self._y[:self.n_rows]


def split_rows(plan: DomainPlan, comm: PartComm, v) -> dict:
    """The local parts' owned pieces of a global vector."""
    v = np.asarray(v, np.float64)
    return {p: v[plan.row_splits[p]:plan.row_splits[p + 1]] for p in comm.local_parts}


def solve_distributed(ctx: Context, row_offsets, columns, values, rhs, parts: int, comm: PartComm | None = None,
                      x0=None, restart: int = 30, max_iterations: int = 1000, tolerance: float = 1e-8,
                      row_splits=None, preconditioner: str = "vcycle", precision: str = "fp64",
                      replicate_below: int = 4096, **amg_options):
    """Solve one FP64 system split into ``parts`` row blocks over the processes of ``comm``.

    Every process passes the whole CSR system and right-hand side (host
    arrays) and gets back its own parts' rows of the solution and the report.
    ``preconditioner``: "vcycle" -- the undivided native-AMG hierarchy (host
    setup on every process) as a distributed FP64 V-cycle, the one-GPU
    preconditioner and iteration count; "block_jacobi" -- a native AMG on
    each part's diagonal block (``precision`` selects its V-cycle)."""
    if preconditioner not in ("vcycle", "block_jacobi"):
        raise ValueError("preconditioner must be 'vcycle' or 'block_jacobi'")
    comm = comm or PartComm(parts)
    plan = DomainPlan(row_offsets, columns, parts, row_splits)
    va = np.ascontiguousarray(values, np.float64)
    blocks = preconditioner == "block_jacobi"
    local = {p: CudaPart(ctx, plan.part(p), va, precision=precision, block_amg=blocks, **amg_options)
             for p in comm.local_parts}
    pc = None
    if not blocks:
        amg = NativeBoomerAMGPreconditioner(None, **amg_options)
        if not amg.setup_host(row_offsets, columns, va):
            raise CfdxgError(N.CFDXG_ERR_SETUP, f"AMG setup failed: {amg.last_error()}")
        levels = [amg.export_level(l) for l in range(len(amg.hierarchy_level_sizes()))]
        first = local[comm.local_parts[0]]
        with torch.cuda.stream(first.stream):
            pc = DistributedAMG(comm, levels, amg.omega, plan.row_splits,
                                lambda ro, co, v, nr, nc: CudaOperator(ctx, ro, co, v, nr, nc), first.device,
                                replicate_below=replicate_below)
    solver = DistributedFGMRES(comm, local, restart=restart, preconditioner=pc)
    x0p = None if x0 is None else split_rows(plan, comm, x0)
    return solver.solve(split_rows(plan, comm, rhs), x0p, max_iterations=max_iterations, tolerance=tolerance)
