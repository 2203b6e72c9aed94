"""SIMPLE pressure-correction outer iterations on an anisotropic boundary-layer
hex mesh: the steps either side of the pressure solve, repeated.

Mesh: nx x ny x nz hex cells on [0, lx] x [0, 1] x [0, lz] (default
256 x 256 x 64 = 4,194,304 cells on [0,10] x [0,1] x [0,1]); the wall-normal
spacing grows geometrically from 1e-4 at y = 0 by 1.08 per cell (capped so the
column spans [0, 1]), x and z lattice lines are jittered by +-0.05h (seeded).
Per-cell eddy-viscosity ratio log-uniform on [1, 1e3], smoothed by 3 Jacobi
sweeps (average of the cell and its face neighbours).

The momentum solve is outside this library's path, so the loop drives the
reference's pressure-side steps with a momentum operator of its own: a
viscous-plus-upwind-convection matrix on the cell graph built from the previous
iteration's face fluxes (the same matrix for the three velocity components,
zero-gradient velocity boundaries),

  a_oo += G_f + max(phi_f, 0),   a_on = -G_f - max(-phi_f, 0),
  a_nn += G_f + max(-phi_f, 0),  a_no = -G_f - max(phi_f, 0),
  G_f = (1 + nu_t,f) |S_f| / |d_f|   (boundary faces: owner diagonal only),

with right-hand side -grad(p) V, taking the current cell velocity as the
momentum solution.  Each outer iteration then runs the reference's chain:

  rAU = 1 / diag(M);  HbyA = build_hbya (steady_incompressible_solver.h:6430-6465);
  pressure-corrector assembly (:8048-8181);  AMG setup, then numeric refresh on the
  unchanged pattern (amg_preconditioner.h:245-314);  the pressure solve;
  p += alpha_p p' (:9339-9343, fixed-pressure boundary: no gauge shift);
  phi = make_rhie_chow_mass_flux(HbyA, p) (:2064-2217);  grad p;  U = HbyA - V rAU grad p.

The initial velocity is a unit stream in x plus an 8-mode divergence-free
Fourier field; p = 0 is fixed on the x = 0 patch.  tests/test_gpu_simple.py
checks five iterations of this chain on the GPU against the same chain built
from the C oracle (HbyA, assembly, flux and gradient bit-identical; the
pressure to 1e-10 with equal iteration counts).

Forms: plain FP64 GMRES(30) + FP64 AMG (the reference's method); FP64
FGMRES(30) + FP32 V-cycle; and the same with the learned stage in front
(optionally fine-tuned on pairs from this mesh).  Each form runs the whole
loop from the same initial state; the JSON report has per-iteration
continuity residuals, Krylov iterations and the seconds spent in assembly,
AMG setup/refresh, solve and face flux.

    python -m cfdx_dev_b200.simple_loop --nx 256 --ny 256 --nz 64 --iterations 20
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import cfdx_dev_b200 as cg  # noqa: E402

SEED = 20240605
WEIGHTS = Path(__file__).resolve().parent / "weights" / "mpnn.bin"


def face_graph(m):
    internal = m.neighbour >= 0
    return m.owner[internal], m.neighbour[internal]


def smoothed_eddy_ratio(m, seed, sweeps=3):
    nu = cg.random_field(m.n_cells, "loguniform", 1.0, 1.0e3, seed)
    o, n = face_graph(m)
    deg = np.bincount(o, minlength=m.n_cells) + np.bincount(n, minlength=m.n_cells)
    for _ in range(sweeps):
        s = nu.copy()
        np.add.at(s, o, nu[n])
        np.add.at(s, n, nu[o])
        nu = s / (1.0 + deg)
    return nu


def viscous_diagonal(m, g, nu_t):
    """sum over faces of (1 + nu_t,f) |S_f| / |d_f| per cell (face value: mean of the two cells)."""
    nf, nc = m.n_faces, m.n_cells
    S = g["face_Sf"].reshape(3, nf)
    area = np.sqrt((S * S).sum(0))
    cc = g["cell_centres"].reshape(3, nc)
    fc = g["face_centres"].reshape(3, nf)
    o, nb = m.owner, m.neighbour
    internal = nb >= 0
    other = np.where(internal, nb, 0)
    d = np.where(internal[None, :], cc[:, other] - cc[:, o], fc - cc[:, o])
    dist = np.sqrt((d * d).sum(0))
    nu_f = np.where(internal, 0.5 * (nu_t[o] + nu_t[other]), nu_t[o])
    coef = (1.0 + nu_f) * area / dist
    aP = np.bincount(o, weights=coef, minlength=nc)
    aP += np.bincount(nb[internal], weights=coef[internal], minlength=nc)
    return aP


def outflow(m, phi):
    """sum_f max(phi_f, 0) leaving each cell (owner side +phi, neighbour side -phi)."""
    nc = m.n_cells
    out = np.bincount(m.owner, weights=np.maximum(phi, 0.0), minlength=nc)
    internal = m.neighbour >= 0
    out += np.bincount(m.neighbour[internal], weights=np.maximum(-phi[internal], 0.0), minlength=nc)
    return out


def cell_pattern(m):
    """CSR pattern of the cell graph (sorted rows, diagonal included) and, per
    interior face, the positions of (owner, neighbour) and (neighbour, owner)."""
    nc = m.n_cells
    internal = np.flatnonzero(m.neighbour >= 0)
    o, n = m.owner[internal], m.neighbour[internal]
    rows = np.concatenate([np.arange(nc), o, n])
    cols = np.concatenate([np.arange(nc), n, o])
    order = np.lexsort((cols, rows))
    ro = np.zeros(nc + 1, np.int64)
    np.add.at(ro, rows + 1, 1)
    ro = np.cumsum(ro)
    co = cols[order].astype(np.int64)
    pos = np.empty(rows.size, np.int64)
    pos[order] = np.arange(rows.size)
    diag_pos = pos[:nc]
    on_pos, no_pos = pos[nc:nc + internal.size], pos[nc + internal.size:]
    return ro, co, diag_pos, internal, on_pos, no_pos


def momentum_values(m, g, nu_t, phi, pattern):
    """Values of the synthetic momentum matrix (see the module docstring) on cell_pattern's pattern."""
    ro, co, diag_pos, internal, on_pos, no_pos = pattern
    nf, nc = m.n_faces, m.n_cells
    S = g["face_Sf"].reshape(3, nf)
    area = np.sqrt((S * S).sum(0))
    cc = g["cell_centres"].reshape(3, nc)
    fc = g["face_centres"].reshape(3, nf)
    o, nb = m.owner, m.neighbour
    isin = nb >= 0
    other = np.where(isin, nb, 0)
    d = np.where(isin[None, :], cc[:, other] - cc[:, o], fc - cc[:, o])
    dist = np.sqrt((d * d).sum(0))
    nu_f = np.where(isin, 0.5 * (nu_t[o] + nu_t[other]), nu_t[o])
    G = (1.0 + nu_f) * area / dist
    va = np.zeros(co.size)
    diag = np.bincount(o, weights=G + np.maximum(phi, 0.0), minlength=nc)
    diag += np.bincount(nb[internal], weights=G[internal] + np.maximum(-phi[internal], 0.0), minlength=nc)
    va[diag_pos] = diag
    va[on_pos] = -G[internal] - np.maximum(-phi[internal], 0.0)
    va[no_pos] = -G[internal] - np.maximum(phi[internal], 0.0)
    return va, diag


def finetune(ctx, net, mesh, A, aP, amg64, amg32, pairs, epochs, seed):
    rng = np.random.default_rng(seed)
    R, E = [], []
    for q in range(pairs):
        r = rng.standard_normal(A.n) if q % 2 else A.matvec(rng.standard_normal(A.n))
        r /= np.sqrt(np.mean(r * r))
        e, rep = cg.solve_gmres(A, r, amg=amg64, restart=30, tolerance=1e-10, max_iterations=2000)
        if q >= pairs // 2:
            for _ in range(1 + q % 3):
                e = e - amg32.apply(r)
                r = A.matvec(e)
            s = 1.0 / np.sqrt(np.mean(r * r))
            r, e = r * s, e * s
        R.append(r)
        E.append(e)
    R, E = np.array(R), np.array(E)
    net.bind(mesh, A, aP)
    net.set_vcycle(amg32)
    losses = []
    for ep in range(epochs):
        for b in range(0, pairs, 8):
            losses.append(net.train_step(R[b:b + 8], E[b:b + 8], lr=5e-4))
    net.set_vcycle(None)
    return losses


def initial_state(m, g):
    """(U, p, phi) at the first outer iteration."""
    U = cg.fourier_field(g["cell_centres"], 8, 0.01, SEED + 1)
    U[:m.n_cells] += 1.0   # unit stream in x
    return U, np.zeros(m.n_cells), np.zeros(m.n_faces)


def run_form(ctx, form, m, mesh, g, nu_t, iterations, alpha_p, net, sync, keep=False):
    nc = m.n_cells
    fixed = np.zeros(m.n_patches, np.int32)
    fixed[0] = 1
    value = np.zeros(m.n_patches)
    vol = g["cell_volumes"]
    U, p, phi = initial_state(m, g)
    gradp = np.zeros(3 * nc)
    pattern = cell_pattern(m)
    precision = "fp64" if form == "plain_fp64" else "fp32_vcycle"
    krylov = "gmres" if form == "plain_fp64" else "fgmres"
    A = None
    amg = None
    records, states = [], []
    for k in range(iterations):
        rec = {"iteration": k}
        t = time.perf_counter()
        va, aP = momentum_values(m, g, nu_t, phi, pattern)
        rAU = np.concatenate([1.0 / aP] * 3)
        rhs = -(gradp.reshape(3, nc) * vol[None, :]).ravel()
        M = cg.SparseMatrix.from_csr(ctx, pattern[0], pattern[1], va)
        HbyA = cg.build_hbya(mesh, M, rhs, U, gradp, rAU)
        rec["momentum_s"] = time.perf_counter() - t
        t = time.perf_counter()
        A, b, phiH, _ = cg.assemble_pressure_correction(mesh, HbyA, rAU, p, 1.0, fixed, value, matrix=A)
        sync()
        rec["assembly_s"] = time.perf_counter() - t
        rec["continuity_l2"] = float(np.linalg.norm(b))
        t = time.perf_counter()
        if amg is None:
            # The FP32 forms end the cycle at <= 2,000 rows in an FP64 dense
            # inverse (the mixed-precision configuration as specified), which
            # every numeric refresh re-forms by LU.
            extra = {} if precision == "fp64" else {"coarse_dense_limit": 2000, "dense_fp64": 1}
            amg = cg.NativeBoomerAMGPreconditioner(ctx, precision=precision, **extra)
            if not amg.setup(A):
                raise RuntimeError(amg.last_error())
            rec["amg_setup_s"] = time.perf_counter() - t
            rec["amg_levels"] = amg.hierarchy_level_sizes()
        elif amg.update_values(A):
            rec["amg_refresh_s"] = time.perf_counter() - t
        else:
            # the numeric refresh refuses a changed pruned coarse pattern (as the
            # reference's update_values does); the owner then sets up afresh
            if not amg.setup(A):
                raise RuntimeError(amg.last_error())
            rec["amg_resetup_s"] = time.perf_counter() - t
        kw = {}
        if form == "learned_fp32":
            t = time.perf_counter()
            net.bind(mesh, A, aP)
            rec["learned_bind_s"] = time.perf_counter() - t
            kw = dict(learned=net)
        t = time.perf_counter()
        ortho = {} if form == "plain_fp64" else {"orthogonalization": 1}
        dp, rep = cg.solve_gmres(A, b, amg=amg, restart=30, tolerance=1e-8, krylov=krylov, max_iterations=1000,
                                 **ortho, **kw)
        sync()
        rec["solve_s"] = time.perf_counter() - t
        rec["krylov_iterations"] = rep["iterations"]
        rec["status"] = rep["status_name"]
        rec["physical_residual_relative"] = rep["physical_residual_relative"]
        t = time.perf_counter()
        p = p + alpha_p * dp
        phi = cg.make_rhie_chow_mass_flux(mesh, HbyA, rAU, p, 1.0, fixed, value)
        gradp = cg.gauss_gradient_with_boundary(mesh, p, fixed, value)
        sync()
        rec["flux_s"] = time.perf_counter() - t
        # cell velocity correction with dAU = V rAU (the volume enters at the projection)
        U = (HbyA.reshape(3, nc) - vol[None, :] * rAU.reshape(3, nc) * gradp.reshape(3, nc)).ravel()
        records.append(rec)
        if keep:
            states.append({"HbyA": HbyA, "b": b, "dp": dp, "p": p.copy(), "phi": phi, "iterations": rep["iterations"]})
        print(json.dumps({"form": form, **{q: v for q, v in rec.items() if q != "amg_levels"}}), flush=True)
    total = {q: float(sum(r.get(q, 0.0) for r in records))
             for q in ("momentum_s", "assembly_s", "amg_setup_s", "amg_refresh_s", "amg_resetup_s", "learned_bind_s",
                       "solve_s", "flux_s")}
    total["refreshes"] = sum(1 for r in records if "amg_refresh_s" in r)
    total["resetups"] = sum(1 for r in records if "amg_resetup_s" in r)
    total["krylov_iterations"] = int(sum(r["krylov_iterations"] for r in records))
    out = {"records": records, "totals": total,
           "final_continuity_l2": records[-1]["continuity_l2"], "first_continuity_l2": records[0]["continuity_l2"]}
    if keep:
        out["states"] = states
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--nz", type=int, default=64)
    ap.add_argument("--iterations", type=int, default=20)
    ap.add_argument("--alpha-p", type=float, default=0.3)
    ap.add_argument("--forms", default="plain_fp64,fp32_vcycle,learned_fp32")
    ap.add_argument("--finetune-pairs", type=int, default=0, help="pairs from this mesh to fine-tune the network on")
    ap.add_argument("--finetune-epochs", type=int, default=4)
    ap.add_argument("--json", type=Path, default=None)
    args = ap.parse_args(argv)
    ctx = cg.Context(0)
    t = time.perf_counter()
    m = cg.boundary_layer_case(args.nx, args.ny, args.nz, 10.0, 1.0, 1e-4, 1.08, 0.05, SEED)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    nu_t = smoothed_eddy_ratio(m, SEED + 2)
    case_s = time.perf_counter() - t
    out = {"workload": f"boundary-layer hex {args.nx}x{args.ny}x{args.nz} = {m.n_cells} cells, {args.iterations} "
                       f"SIMPLE outer iterations, alpha_p {args.alpha_p}", "cells": m.n_cells, "case_s": case_s,
           "forms": {}}
    net = None
    forms = [f for f in args.forms.split(",") if f]
    if "learned_fp32" in forms:
        if not WEIGHTS.exists():
            forms.remove("learned_fp32")
        else:
            net = cg.LearnedPreconditioner(ctx)
            net.load(WEIGHTS)
            if args.finetune_pairs > 0:
                fixed = np.zeros(m.n_patches, np.int32)
                fixed[0] = 1
                U0 = cg.fourier_field(g["cell_centres"], 8, 0.01, SEED + 1)
                aP0 = viscous_diagonal(m, g, nu_t)
                A0, _, _, _ = cg.assemble_pressure_correction(mesh, U0, np.concatenate([1.0 / aP0] * 3),
                                                              np.zeros(m.n_cells), 1.0, fixed, np.zeros(m.n_patches))
                a64 = cg.NativeBoomerAMGPreconditioner(ctx)
                a32 = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp32_vcycle")
                assert a64.setup(A0) and a32.setup(A0)
                t = time.perf_counter()
                losses = finetune(ctx, net, mesh, A0, aP0, a64, a32, args.finetune_pairs, args.finetune_epochs, SEED)
                out["finetune"] = {"pairs": args.finetune_pairs, "epochs": args.finetune_epochs,
                                   "seconds": time.perf_counter() - t, "first_loss": losses[0], "last_loss": losses[-1]}
    for form in forms:
        out["forms"][form] = run_form(ctx, form, m, mesh, g, nu_t, args.iterations, args.alpha_p, net, ctx.synchronize)
    summary = {f: v["totals"] for f, v in out["forms"].items()}
    print(json.dumps({"summary": summary, "workload": out["workload"]}), flush=True)
    if args.json:
        args.json.write_text(json.dumps(out))


if __name__ == "__main__":
    main()
