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

    @property
    def n_owned(self) -> int:
        return self.row_end - self.row_begin

    @property
    def owned(self) -> slice:
        """The owned rows' slice of the local vector."""
        return slice(self.owned_offset, self.owned_offset + self.n_owned)

    def local_to_global(self) -> np.ndarray:
        """Global row of every local vector position."""
        g = np.empty(self.n_local, np.int64)
        below = self.owned_offset
        g[:below] = self.ghost_rows[:below]
        g[self.owned] = np.arange(self.row_begin, self.row_end)
        g[below + self.n_owned:] = self.ghost_rows[below:]
        return g

    def recv_slice(self, k: int) -> slice:
        s = int(self.recv_start[k])
        return slice(s, s + int(self.recv_offsets[k + 1] - self.recv_offsets[k]))

    def send_slice(self, k: int) -> slice:
        return slice(int(self.send_offsets[k]), int(self.send_offsets[k + 1]))


class DomainPlan:
    """Row-block partition with halos of a square CSR pattern (cfdxg_domain_plan_create)."""

    def __init__(self, row_offsets, columns, parts: int, row_splits=None):
        self.lib = N.load()
        ro = np.ascontiguousarray(row_offsets, np.int64)
        co = np.ascontiguousarray(columns, np.int64)
        self.n = ro.size - 1
        splits = None if row_splits is None else np.ascontiguousarray(row_splits, np.int64)
        if splits is not None and splits.size != parts + 1:
            raise ValueError("row_splits needs parts + 1 entries")
        h = C.c_void_p()
        rc = self.lib.cfdxg_domain_plan_create(self.n, N.ptr(ro), N.ptr(co), int(parts), N.ptr(splits), C.byref(h))
        if rc != 0:
            raise CfdxgError(rc, self.lib.cfdxg_domain_last_error().decode())
        self.handle = h
        self.row_splits = np.empty(parts + 1, np.int64)
        self.parts = self.lib.cfdxg_domain_plan_parts(h, N.ptr(self.row_splits))

    def part(self, p: int) -> PartLayout:
        info = N.DomainPartInfo()
        rc = self.lib.cfdxg_domain_plan_info(self.handle, int(p), C.byref(info))
        if rc != 0:
            raise CfdxgError(rc, self.lib.cfdxg_domain_last_error().decode())
        n_own, nb = info.row_end - info.row_begin, info.n_neighbours
        sizes = dict(local_row_offsets=info.n_local + 1, local_columns=info.nnz_local, local_source=info.nnz_local,
                     block_row_offsets=n_own + 1, block_columns=info.nnz_block, block_source=info.nnz_block,
                     neighbours=nb, recv_offsets=nb + 1, recv_start=nb, ghost_rows=info.n_recv,
                     send_offsets=nb + 1, send_rows=info.n_send)
        arrays = {k: np.empty(v, np.int32 if k == "neighbours" else np.int64) for k, v in sizes.items()}
        out = N.DomainPartArrays(**{k: arrays[k].ctypes.data for k in N.DOMAIN_ARRAYS})
        rc = self.lib.cfdxg_domain_plan_export(self.handle, int(p), C.byref(out))
        if rc != 0:
            raise CfdxgError(rc, self.lib.cfdxg_domain_last_error().decode())
        return PartLayout(index=int(p), row_begin=info.row_begin, row_end=info.row_end, n_local=info.n_local,
                          owned_offset=info.owned_offset, **arrays)

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
        """Index tensors of the exchange, on the vectors' device."""
        self._layouts = layouts
        self._send, self._copy, self._recv = [], [], []
        for p in self.local_parts:
            L = layouts[p]
            for k, q in enumerate(L.neighbours.tolist()):
                rs, ss = L.recv_slice(k), L.send_slice(k)
                if rs.stop > rs.start:
                    if self.owners[q] == self.rank:
                        src = layouts[q]
                        idx = L.ghost_rows[L.recv_offsets[k]:L.recv_offsets[k + 1]] - src.row_begin + src.owned_offset
                        self._copy.append((p, rs, q, torch.as_tensor(idx, device=device)))
                    else:
                        self._recv.append(((q, p), rs))
                if ss.stop > ss.start and self.owners[q] != self.rank:
                    idx = L.send_rows[ss] + L.owned_offset
                    self._send.append(((p, q), torch.as_tensor(idx, device=device)))
        # every pair of processes posts its messages in (source part, destination part) order
        self._send.sort(key=lambda e: e[0])
        self._recv.sort(key=lambda e: e[0])

    def exchange(self, vectors: dict[int, torch.Tensor]) -> None:
        """Fill the ghost slices of every local part's local vector from the owners' owned values."""
        self.exchanges += 1
        for p, rs, q, idx in self._copy:
            vectors[p][rs] = vectors[q].index_select(0, idx)
        if not self._send and not self._recv:
            return
        import torch.distributed as dist
        ops, bufs = [], []
        for (p, q), idx in self._send:
            buf = vectors[p].index_select(0, idx)
            bufs.append(buf)
            ops.append(dist.P2POp(dist.isend, buf, self.owners[q], self.group, tag=p * self.parts + q))
        for (q, p), rs in self._recv:
            ops.append(dist.P2POp(dist.irecv, vectors[p][rs], self.owners[q], self.group, tag=q * self.parts + p))
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class CudaPart:
    """A part on the device: local FP64 SpMV and a native AMG V-cycle on its diagonal block."""

    def __init__(self, ctx: Context, layout: PartLayout, values, precision: str = "fp64", **amg_options):
        if not torch.cuda.is_available():
            raise RuntimeError("CudaPart needs a CUDA device (the distributed path has no CPU fallback)")
        self.ctx, self.layout = ctx, layout
        self.lib = ctx.lib
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = torch.cuda.ExternalStream(ctx.stream, device=self.device)
        self.A = SparseMatrix.from_csr(ctx, layout.local_row_offsets, layout.local_columns,
                                       np.asarray(values)[layout.local_source])
        self.B = SparseMatrix.from_csr(ctx, layout.block_row_offsets, layout.block_columns,
                                       np.asarray(values)[layout.block_source])
        self.amg = NativeBoomerAMGPreconditioner(ctx, precision=precision, **amg_options)
        if not self.amg.setup(self.B):
            raise CfdxgError(N.CFDXG_ERR_SETUP, f"part {layout.index}: AMG setup failed: {self.amg.last_error()}")
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
    ``matvec(x_local) -> owned y`` and ``precondition(r, z)``."""

    def __init__(self, comm: PartComm, parts: dict, restart: int = 30):
        if sorted(parts) != comm.local_parts:
            raise ValueError("parts must be exactly the process's local parts")
        if restart < 1:
            raise ValueError("restart must be at least 1")
        self.comm, self.parts, self.m = comm, parts, restart
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
                for p, P in parts.items():
                    z = self.Z[p][j]
                    zo = z[P.layout.owned]
                    P.precondition(self.V[p][j], zo)
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


def split_rows(plan: DomainPlan, comm: PartComm, v) -> dict:
    """The local parts' owned pieces of a global vector."""
    v = np.asarray(v, np.float64)
    return {p: v[plan.row_splits[p]:plan.row_splits[p + 1]] for p in comm.local_parts}


def solve_distributed(ctx: Context, row_offsets, columns, values, rhs, parts: int, comm: PartComm | None = None,
                      x0=None, restart: int = 30, max_iterations: int = 1000, tolerance: float = 1e-8,
                      row_splits=None, precision: str = "fp64", **amg_options):
    """Solve one FP64 system split into ``parts`` row blocks over the processes of ``comm``.

    Every process passes the whole CSR system and right-hand side (host
    arrays) and gets back its own parts' rows of the solution and the report.
    Preconditioner: the library's native AMG on each part's diagonal block."""
    comm = comm or PartComm(parts)
    plan = DomainPlan(row_offsets, columns, parts, row_splits)
    va = np.ascontiguousarray(values, np.float64)
    local = {p: CudaPart(ctx, plan.part(p), va, precision=precision, **amg_options) for p in comm.local_parts}
    solver = DistributedFGMRES(comm, local, restart=restart)
    x0p = None if x0 is None else split_rows(plan, comm, x0)
    return solver.solve(split_rows(plan, comm, rhs), x0p, max_iterations=max_iterations, tolerance=tolerance)
