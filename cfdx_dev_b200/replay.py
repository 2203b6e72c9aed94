"""Replay a captured linear system on the GPU.

The counterpart of the reference's tools/diagnostics/cfdx_linear_replay.cpp:
reads a ``.cfdxlin`` capture (core/linalg/linear_system_capture.h), prints its
CSR diagnosis to stderr, solves it once per requested preconditioner with the
automatic Krylov choice through ``solve_linear_system`` (the capture's problem
kind, scaling, iteration limit and tolerance; the initial guess from the
file) and prints one CSV row per candidate:

    preconditioner,krylov,status,iterations,total_ms,true_abs_l2,true_relative

Each candidate must pass the capture's tolerance on the FP64 true residual of
the original system (the rhs norm, or the initial residual for b = 0);
otherwise the exit status is 1.  Candidates: auto, jacobi, native, none.
Models this library does not provide (ilu0, directional, energy) and
captures with a projected constant null space are reported as
``not_applicable`` rows.

    python -m cfdx_dev_b200.replay pressure.cfdxlin [auto|jacobi|native|none ...]
"""
from __future__ import annotations

import sys
import time

import numpy as np

from . import _native as N
from .api import (CfdxgError, Context, SparseMatrix, diagnose_matrix, read_linear_system_capture,
                  solve_linear_system)

CANDIDATES = {"auto": "auto", "jacobi": "jacobi", "native": "native_amg", "none": "none"}
NOT_PROVIDED = ("ilu0", "directional", "energy")
HEADER = "preconditioner,krylov,status,iterations,total_ms,true_abs_l2,true_relative"


def diagnosis(c: dict) -> str:
    """The reference tool's CSR line from diagnose_matrix (rows, nnz, missing and
    near-zero diagonals) and the capture's checksum."""
    d = diagnose_matrix(c["row_offsets"], c["columns"], c["values"])
    return (f"CSR rows={d['rows']} nnz={d['nnz']} missing_diagonal={d['missing_diagonal']} "
            f"near_zero_diagonal={d['near_zero_diagonal']} checksum={c['checksum']:x}")


def _true_residual(ro, co, va, x, b):
    rows = np.repeat(np.arange(ro.size - 1), np.diff(ro))
    r = b - np.bincount(rows, weights=va * x[co], minlength=b.size)
    return float(np.linalg.norm(r))


def replay(path, candidates=("auto",), ctx: Context | None = None) -> tuple[list[str], bool]:
    """CSV rows (without the header) and whether every candidate passed."""
    unknown = [n for n in candidates if n not in CANDIDATES and n not in NOT_PROVIDED]
    if unknown:
        raise ValueError(f"unknown preconditioner: {unknown[0]}")
    c = read_linear_system_capture(path)
    ctx = ctx or Context(0)
    A = SparseMatrix.from_csr(ctx, c["row_offsets"], c["columns"], c["values"])
    b, x0 = c["rhs"], c["initial_solution"]
    rhs_norm = float(np.linalg.norm(b))
    initial = _true_residual(c["row_offsets"], c["columns"], c["values"], x0, b)
    reference = rhs_norm if rhs_norm > 0.0 else initial
    rows, passed = [], True
    for name in candidates:
        if name in NOT_PROVIDED or c["null_space"] != 0:
            rows.append(f"{name},none,not_applicable,0,0,nan,nan")
            passed = False
            continue
        t0 = time.perf_counter()
        try:
            x, rep = solve_linear_system(A, b, x0=x0, krylov="auto", preconditioner=CANDIDATES[name],
                                         max_iterations=int(c["max_iterations"]), tolerance=float(c["tolerance"]),
                                         problem=N.PROBLEMS[c["problem"]], scaling=N.SCALINGS[c["scaling"]])
        except CfdxgError as e:
            print(f"REPLAY_SOLVE_FAILED {name}: {e}", file=sys.stderr)
            rows.append(f"{name},none,exception,0,0,nan,nan")
            passed = False
            continue
        ms = (time.perf_counter() - t0) * 1e3
        absolute = _true_residual(c["row_offsets"], c["columns"], c["values"], x, b)
        relative = absolute / reference if reference > 0.0 else (0.0 if absolute == 0.0 else float("inf"))
        ok = rep["status"] == 0 and np.isfinite(relative) and relative <= c["tolerance"]
        passed = passed and ok
        krylov = N.KRYLOV_MODELS[rep["plan_krylov"]] if 0 <= rep["plan_krylov"] < len(N.KRYLOV_MODELS) else "none"
        rows.append(f"{name},{krylov},{rep['status_name']},{rep['iterations']},{ms:.17g},{absolute:.17g},"
                    f"{relative:.17g}")
    return rows, passed


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if not argv:
        print("Usage: python -m cfdx_dev_b200.replay file.cfdxlin [auto|jacobi|native|none ...]", file=sys.stderr)
        return 2
    try:
        c = read_linear_system_capture(argv[0])
        print(diagnosis(c), file=sys.stderr)
        rows, passed = replay(argv[0], argv[1:] or ["auto"])
    except Exception as e:  # noqa: BLE001 - the tool reports every failure the same way
        print(f"CFDX_LINEAR_REPLAY_FAIL: {e}", file=sys.stderr)
        return 1
    print(HEADER)
    for r in rows:
        print(r)
    if not passed:
        print("CFDX_LINEAR_REPLAY_FAIL: at least one candidate failed", file=sys.stderr)
    return 0 if passed else 1


if __name__ == "__main__":
    sys.exit(main())
