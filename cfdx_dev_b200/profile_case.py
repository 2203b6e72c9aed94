"""A small, self-contained workload for kernel profilers (ncu).

Builds the seeded Kuhn-tet pressure-correction system of an n^3 lattice
(6 tets per hex cell, interior vertices jittered by +-0.15h; divergence-free
Fourier HbyA, log-uniform a_P on [1, 100], p = 0 fixed on the x = 0 patch),
sets up the AMG hierarchy and runs each hot-path kernel a few times:

  * ``vcycle``: three V-cycle applications (``--precision fp32_vcycle|fp64``);
  * ``solve``: one FGMRES(30) solve to 1e-8 with the FP32 V-cycle, two
    applications of the learned stage (when trained weights are present) and
    the Rhie-Chow face flux of the solution;
  * ``face``: the face loop alone -- ``--cycles`` pressure-corrector
    assemblies (Gauss gradient + assembly) and Rhie-Chow fluxes with a
    non-zero pressure, inputs on the device, L2 flushed before each call;
    prints each kernel's device time from the library's live profiler;
  * ``setup``: the AMG setup with its Galerkin products on the device
    (cfdxg_amg_setup) and the all-host setup of the same matrix, timed;
  * ``refresh``: ``--cycles`` numeric refreshes (update_values) of the same
    matrix, each refresh stage's device time.

Example (one kernel, one launch, at 663,552 cells):

    ncu --set full --clock-control none --kernel-name-base demangled \\
        -k 'regex:k_sweep<float, float, \\(int\\)1>' -s 1 -c 1 -o sweep \\
        python -m cfdx_dev_b200.profile_case --n 48 --mode solve
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import cfdx_dev_b200 as cg  # noqa: E402

SEED_MESH, SEED_HBYA, SEED_AP = 20240601, 20240602, 20240603
WEIGHTS = Path(__file__).resolve().parent / "weights" / "mpnn.bin"


def build_system(ctx, n):
    m = cg.tet_case(n, 0.15, SEED_MESH)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    U = cg.fourier_field(g["cell_centres"], 8, 0.01, SEED_HBYA)
    aP = cg.random_field(m.n_cells, "loguniform", 1.0, 100.0, SEED_AP)
    rAU = np.concatenate([1.0 / aP] * 3)
    p = np.zeros(m.n_cells)
    fixed = np.zeros(m.n_patches, np.int32)
    fixed[0] = 1
    value = np.zeros(m.n_patches)
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    return m, mesh, (U, rAU, aP, p, fixed, value), A, b


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--n", type=int, default=48, help="lattice size (cells = 6 n^3)")
    ap.add_argument("--mode", choices=["vcycle", "solve", "face", "setup", "refresh"], default="solve")
    ap.add_argument("--precision", choices=["fp32_vcycle", "fp64"], default="fp32_vcycle")
    ap.add_argument("--wide-columns", action="store_true", help="int32 columns on every level (narrow_columns = 0)")
    ap.add_argument("--cycles", type=int, default=3, help="V-cycle applications in --mode vcycle")
    args = ap.parse_args(argv)
    ctx = cg.Context(0)
    m, mesh, (U, rAU, aP, p, fixed, value), A, b = build_system(ctx, args.n)
    if args.mode == "face":
        face_loop(ctx, m, mesh, (U, rAU, p, fixed, value), A, args.cycles)
        return
    if args.mode == "setup":
        import time
        amg = cg.NativeBoomerAMGPreconditioner(ctx, precision=args.precision)
        t0 = time.perf_counter()
        if not amg.setup(A):
            raise SystemExit(amg.last_error())
        t1 = time.perf_counter()
        host = cg.NativeBoomerAMGPreconditioner(None)
        ro, co, va = A.to_csr()
        t2 = time.perf_counter()
        if not host.setup_host(ro, co, va):
            raise SystemExit(host.last_error())
        t3 = time.perf_counter()
        same = all(np.array_equal(amg.export_level(l)["values"], host.export_level(l)["values"])
                   for l in range(len(host.hierarchy_level_sizes())))
        print(f"setup n={args.n} cells={A.n} levels={len(amg.hierarchy_level_sizes())} "
              f"device-Galerkin setup {t1 - t0:.3f} s (with the device upload), host setup {t3 - t2:.3f} s, "
              f"identical level values: {same}")
        return
    if args.mode == "refresh":
        amg = cg.NativeBoomerAMGPreconditioner(ctx, precision=args.precision)
        if not amg.setup(A):
            raise SystemExit(amg.last_error())
        import time
        ctx.profile(True)
        t0 = time.perf_counter()
        for k in range(args.cycles):
            if not amg.update_values(A):
                raise SystemExit(amg.last_error())
        ctx.synchronize()
        print(f"refresh n={args.n} cells={A.n}: {(time.perf_counter() - t0) / args.cycles:.3f} s per refresh")
        ctx.synchronize()
        for e in ctx.profile_read():
            if e["launches"] and e["name"].startswith("refresh"):
                print(f"{e['name']}: {e['launches']} launches, {e['total_ms'] / e['launches']:.2f} ms each")
        return
    amg = cg.NativeBoomerAMGPreconditioner(ctx, precision=args.precision,
                                           narrow_columns=0 if args.wide_columns else 1)
    if not amg.setup(A):
        raise SystemExit(amg.last_error())
    if args.mode == "vcycle":
        for _ in range(args.cycles):
            z = amg.apply(b)
        print(f"vcycle n={args.n} cells={A.n} levels={amg.hierarchy_level_sizes()} |z|={np.linalg.norm(z):.6e}")
        return
    # the benchmark's FGMRES form: two-pass classical Gram-Schmidt
    x, rep = cg.solve_fgmres(A, b, amg=amg, restart=30, tolerance=1e-8, orthogonalization=1)
    if rep["status_name"] != "converged":
        raise SystemExit(f"solve did not converge: {rep}")
    if WEIGHTS.exists():
        net = cg.LearnedPreconditioner(ctx)
        net.load(WEIGHTS)
        net.bind(mesh, A, aP)
        for _ in range(2):
            y = net.apply(b)
    flux = cg.make_rhie_chow_mass_flux(mesh, U, rAU, x, 1.0, fixed, value)
    print(f"solve n={args.n} cells={A.n} iterations={rep['iterations']} |flux|={np.linalg.norm(flux):.6e}")
    ctx.close()


def face_loop(ctx, m, mesh, fields, A, calls):
    import ctypes as C

    import torch

    from cfdx_dev_b200 import _native as N
    U, rAU, p, fixed, value = fields
    dev = torch.device("cuda", 0)
    cc = mesh.geometry()["cell_centres"].reshape(3, -1)
    p = np.sin(3.0 * cc[0]) * cc[1] + cc[2]     # non-zero pressure: every term of the face loop is live
    Ud, rd, pd = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (U, rAU, p))
    nc, nf = m.n_cells, m.n_faces
    bd = torch.empty(nc, dtype=torch.float64, device=dev)
    phid = torch.empty(nf, dtype=torch.float64, device=dev)
    gd = torch.empty(3 * nc, dtype=torch.float64, device=dev)
    fl = torch.empty(nf, dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    fx = np.ascontiguousarray(fixed, np.int32)
    vv = np.ascontiguousarray(value, np.float64)
    h = C.c_void_p(A.handle.value)
    ptr = lambda t: C.c_void_p(t.data_ptr())
    lib = ctx.lib
    ctx.profile(True)
    for s in range(calls):
        flush.fill_(float(s))
        torch.cuda.synchronize()
        ctx.check(lib.cfdxg_assemble_pressure_correction(ctx.handle, mesh.handle, ptr(Ud), ptr(rd), ptr(pd), 1.0,
                                                         N.ptr(fx), N.ptr(vv), N.CFDXG_MEM_DEVICE, C.byref(h),
                                                         ptr(bd), ptr(phid), ptr(gd)), "assembly")
        flush.fill_(float(s))
        torch.cuda.synchronize()
        ctx.check(lib.cfdxg_rhie_chow_flux(ctx.handle, mesh.handle, ptr(Ud), ptr(rd), ptr(pd), 1.0, N.ptr(fx),
                                           N.ptr(vv), N.CFDXG_MEM_DEVICE, ptr(fl)), "flux")
    torch.cuda.synchronize()
    for e in ctx.profile_read():
        if e["launches"]:
            ms = e["total_ms"] / e["launches"]
            print(f"{e['name']}: {e['launches']} launches, {ms * 1e3:.1f} us, "
                  f"{e['bytes'] / e['launches'] / (ms / 1e3) / 1e9:.0f} GB/s on the algorithmic bytes")
    ctx.profile(False)
    print(f"face n={m.n_cells} cells |b|={float(bd.norm()):.6e} |flux|={float(fl.norm()):.6e}")


if __name__ == "__main__":
    main()
