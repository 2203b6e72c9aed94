#!/usr/bin/env python
"""Benchmark: seconds to an FP64 true relative residual of 1e-8 for the SIMPLE
pressure-correction solve on one B200.

Workload (one GPU): the 64^3 Kuhn-tet mesh (1,572,864 cells, interior vertices
jittered by U[+-0.15h]), pressure-correction system assembled on the GPU from a
divergence-free 8-mode Fourier HbyA (+U[+-0.01]) and log-uniform a_P in
[1,100]; p = 0 fixed on the x = 0 patch.  16 seeded right-hand sides (HbyA seeds)
share the matrix; one step solves one of them, cycling.  The AMG hierarchy is
built once per matrix (setup seconds are reported separately) and every solve
starts from p' = 0.

Forms timed: plain FP64 AMG-GMRES (the reference's algorithm, two-pass
modified Gram-Schmidt), FP32 V-cycle inside FP64 FGMRES, and -- when trained
weights are present -- the learned message-passing preconditioner in front of
the FP32 V-cycle; the two FGMRES forms orthogonalise with two-pass classical
Gram-Schmidt.  `value` is the headline form, the FP32 V-cycle (the learned
form is timed beside it: with the full training set it saves 0.1 iteration
per solve and costs more than that).

Inputs are larger than L2 (the hierarchy alone is > 2 GB), and L2 is also
flushed before every timed step.  Rank-local device timing with CUDA events on
the library's stream, max over ranks.  N > 1 runs independent replicas (each
rank its own right-hand sides); there is no data-path collective.

`parity` (rank 0, one GPU): the reference's own solve of the first right-hand
side on its own hierarchy (one host core, also the `cpu_baseline`), its
corrector assembly compared bit for bit with the GPU's, and each GPU form's
pressure and corrected face fluxes against the reference's (relative L2) with
the iteration counts.

`--impl reference` times the reference's own CPU implementation (oracle/_ref,
one host core): its assembly of the same system, its own AMG hierarchy
rebuilt from the stored output of its complete setup, and one complete
GMRES(30) solve per step; it loads only oracle libraries.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

TOL = 1e-8
RESTART = 30
N_RHS = 16
FALLBACK_HBM_GBS = 6650.0
WEIGHTS = ROOT / "cfdx_dev_b200" / "weights" / "mpnn.bin"
METRIC = "s to 1e-8 FP64 residual/pressure solve: learned+FP32 vs plain AMG-GMRES, 1xB200"


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cfdxg", "reference"], default="cfdxg")
    ap.add_argument("--n", type=int, default=64, help="lattice size (cells = 6 n^3)")
    ap.add_argument("--config", type=int, default=2, choices=[2, 5],
                    help="2 (default): the pressure solve benchmark above; 5: SIMPLE outer iterations on the "
                         "256x256x64 boundary-layer mesh in three forms (a separate record, one JSON line)")
    ap.add_argument("--outer-iterations", type=int, default=20, help="--config 5: SIMPLE outer iterations")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned+FP32 form")
    ap.add_argument("--no-c3", action="store_true", help="skip the FP64-coarse-solve FP32 form")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain FP64 form (profiling runs; no speed-ups or errors against it)")
    ap.add_argument("--no-assembly", action="store_true", help="skip the face-loop timing")
    ap.add_argument("--half-values", type=int, default=1,
                    help="FP32 V-cycle coarse levels store FP16 row-scaled values (1, the library default) "
                         "or FP32 values (0)")
    return ap.parse_args()


def dist_env():
    from cfdx_dev_b200.replicas import dist_env as env
    return env()


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic():
    """ncu DRAM bytes per launch recorded in profiles/*.md as `traffic[<kernel>] = <bytes>`."""
    out = {}
    for f in (ROOT / "profiles").glob("*.md"):
        for line in f.read_text().splitlines():
            line = line.strip().strip("`")
            if line.startswith("traffic[") and "=" in line:
                k, v = line.split("=", 1)
                try:
                    out[k.strip()[len("traffic["):-1]] = float(v.split()[0])
                except ValueError:
                    pass
    return out


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"cfdxg_clocks_{os.getpid()}.csv"

    def start(self):
        """Starts sampling every 50 ms and returns once the first sample is in
        (nvidia-smi takes ~0.1-0.3 s to start; the timed region of one form is
        ~0.2 s), so that the samples after this call fall in the timed region."""
        self.skip = 0
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(self.device)], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            n = len(self.path.read_text().splitlines())
            if n:
                self.skip = n
                break
            time.sleep(0.01)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.path.read_text().splitlines()
        # the samples taken after start() returned; the one before, if none came later
        window = lines[self.skip:] or lines[-1:]
        for line in window:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_cfdxg(args):
    import torch

    import cfdx_dev_b200 as cg
    from cfdx_dev_b200 import _native as N
    from cfdx_dev_b200.replicas import max_over_ranks, seed_offsets
    from tests import cases

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local_rank)

    ctx = cg.Context(local_rank)
    lib = ctx.lib
    lstream = torch.cuda.ExternalStream(ctx.stream, device=dev)

    t0 = time.time()
    m = cases.simple_mesh(args.n)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    rhs_list = []
    A = None
    seeds = seed_offsets(rank, N_RHS)   # each replica its own right-hand sides
    for k in range(N_RHS):
        U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"], seed_offset=seeds[k])
        if k == 0:
            base_rAU = rAU
        # the matrix depends on rAU and geometry only; HbyA changes b
        A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, base_rAU, p, 1.0, fixed, value, matrix=A)
        if k == 0:
            base_aP = aP
            base_fields = (U, rAU, p, fixed, value)
        rhs_list.append(b)
    case_s = time.time() - t0
    n_cells = A.n

    # (form, V-cycle precision, Krylov method, learned stage).  fp32_vcycle_fp64_coarse is
    # the mixed-precision configuration with its FP64 coarsest-level direct solve at
    # <= 2,000 unknowns; fp32_vcycle ends instead at <= 6,000 rows in an FP32-stored inverse.
    plan = [("plain_fp64", "fp64", "gmres", False), ("fp32_vcycle_fp64_coarse", "fp32_c3", "fgmres", False),
            ("fp32_vcycle", "fp32_vcycle", "fgmres", False)]
    if args.no_c3:
        plan = [e for e in plan if e[0] != "fp32_vcycle_fp64_coarse"]
    if args.no_plain:
        plan = plan[1:]
    net = None
    if WEIGHTS.exists() and not args.no_learned:
        net = cg.LearnedPreconditioner(ctx)
        net.load(str(WEIGHTS))
        net.bind(mesh, A, base_aP)
        plan.append(("learned_fp32", "fp32_vcycle", "fgmres", True))
    # The headline is the FP32 V-cycle form: trained on the full config-4 set
    # (4,096 pairs on 256 meshes of 16^3-48^3) the learned stage saves no
    # FGMRES iteration per solve at 64^3 in front of the default cycle and
    # costs about 0.5 ms, so it is timed and reported as its own form but
    # does not set `value`.
    headline = "fp32_vcycle" if any(e[0] == "fp32_vcycle" for e in plan) else plan[-1][0]
    forms = {}
    amgs = {}
    by_precision = {}   # one hierarchy per V-cycle precision, shared by the forms that use it
    for form, prec, krylov, learned in plan:
        if prec not in by_precision:
            extra = {"half_values": args.half_values} if prec.startswith("fp32") else {}
            if prec == "fp32_c3":
                extra.update(coarse_dense_limit=2000, dense_fp64=1)
            amg = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp64" if prec == "fp64" else "fp32_vcycle",
                                                   **extra)
            t = time.time()
            if not amg.setup(A):
                raise RuntimeError(amg.last_error())
            by_precision[prec] = (amg, {"setup_s": time.time() - t, "host_setup_s": amg.setup_seconds})
        amgs[form] = by_precision[prec][0]
        forms[form] = dict(by_precision[prec][1])
    levels = amgs[plan[0][0]].hierarchy_level_sizes()
    level_nnz = amgs[plan[0][0]].hierarchy_level_nnz()

    b_dev = [torch.from_numpy(b).to(dev) for b in rhs_list]
    x_dev = torch.zeros(n_cells, dtype=torch.float64, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MB > L2

    def request(krylov, learned):
        # The plain form is the reference's algorithm (two-pass modified
        # Gram-Schmidt); the FGMRES forms use two-pass classical Gram-Schmidt.
        ortho = 0 if krylov == "gmres" else 1
        return cg.make_request(krylov, "native_amg", RESTART, "fp64", net if learned else None,
                               orthogonalization=ortho)

    def solve_device(amg, req, k):
        rep = N.Report()
        rc = lib.cfdxg_solve_gmres(ctx.handle, A.handle, amg.handle, C.c_void_p(b_dev[k].data_ptr()),
                                   C.c_void_p(x_dev.data_ptr()), N.CFDXG_MEM_DEVICE, C.byref(req), 1000, TOL,
                                   C.byref(rep))
        ctx.check(rc, "solve")
        return rep.as_dict()

    ref_solutions = {}
    first_solution = {}   # per form, its solution of right-hand side 0 (parity against the reference)
    sampler = ClockSampler(local_rank)
    for form, prec, krylov, learned in plan:
        amg = amgs[form]
        req = request(krylov, learned)
        for w in range(args.warmup):
            x_dev.zero_()
            torch.cuda.synchronize()
            solve_device(amg, req, w % N_RHS)
        times, iters, errs, fallbacks = [], [], [], []
        launches0 = ctx.kernel_launches
        if form == headline:
            sampler.start()
        for s in range(args.steps):
            k = s % N_RHS
            x_dev.zero_()
            flush.fill_(float(s))
            torch.cuda.synchronize()
            if world > 1:
                torch.distributed.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(lstream)
            rep = solve_device(amg, req, k)
            e1.record(lstream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
            iters.append(rep["iterations"])
            fallbacks.append(rep["learned_fallbacks"])
            if rep["status_name"] != "converged" or rep["physical_residual_relative"] > TOL:
                raise RuntimeError(f"{form} did not converge: {rep}")
            x = x_dev.cpu().numpy()
            if k == 0 and form not in first_solution:
                first_solution[form] = (x.copy(), rep["iterations"])
            if form == "plain_fp64":
                ref_solutions[k] = x.copy()
            elif k in ref_solutions:
                errs.append(float(np.linalg.norm(x - ref_solutions[k]) / np.linalg.norm(ref_solutions[k])))
        if form == headline:
            clocks = sampler.stop()
            launches = ctx.kernel_launches - launches0
            # Per-kernel live timing (CUDA events on the library stream around
            # every kernel class) is a second pass over the same solves: the
            # events would otherwise sit inside the timed region above.
            ctx.profile(True)
            for s in range(args.steps):
                x_dev.zero_()
                flush.fill_(float(s))
                torch.cuda.synchronize()
                solve_device(amg, req, s % N_RHS)
            torch.cuda.synchronize()
            prof = ctx.profile_read()
            ctx.profile(False)
        forms[form].update(s_per_solve=float(np.mean(times)), s_min=float(np.min(times)),
                           iterations=float(np.mean(iters)),
                           rel_error_vs_fp64=(float(np.max(errs)) if errs else 0.0))
        if learned:
            forms[form]["learned_fallback_applications"] = float(np.mean(fallbacks))
    for form in forms:
        if "plain_fp64" in forms:
            forms[form]["speedup_vs_plain_fp64"] = forms["plain_fp64"]["s_per_solve"] / forms[form]["s_per_solve"]

    # ---- the face loop: pressure-corrector assembly and Rhie-Chow face flux ----
    assembly = None
    if not args.no_assembly:
        assembly = time_face_loop(ctx, lib, N, mesh, A, base_fields, dev, lstream, flush, args)

    # ---- end to end through the C ABI with pinned host buffers ----
    e2e = None
    if not args.no_e2e:
        amg = amgs[headline]
        b_host = torch.empty(n_cells, dtype=torch.float64, pin_memory=True)
        x_host = torch.empty(n_cells, dtype=torch.float64, pin_memory=True)
        bh, xh = b_host.numpy(), x_host.numpy()
        hk = next(e for e in plan if e[0] == headline)
        req = request(hk[2], hk[3])
        e2e_times = []
        for s in range(args.warmup + args.steps):
            k = s % N_RHS
            bh[:] = rhs_list[k]
            xh[:] = 0.0
            flush.fill_(float(s))
            torch.cuda.synchronize()
            rep = N.Report()
            t = time.perf_counter()
            rc = lib.cfdxg_solve_gmres(ctx.handle, A.handle, amg.handle, N.ptr(bh), N.ptr(xh), N.CFDXG_MEM_HOST,
                                       C.byref(req), 1000, TOL, C.byref(rep))
            dt = time.perf_counter() - t
            ctx.check(rc, "e2e solve")
            if s >= args.warmup:
                e2e_times.append(dt)
        e2e = {"value": float(np.mean(e2e_times)), "unit": "s",
               "h2d_bytes_per_step": int(16 * n_cells), "d2h_bytes_per_step": int(8 * n_cells)}

    # ---- max over ranks ----
    value, e2e_max = max_over_ranks([forms[headline]["s_per_solve"], e2e["value"] if e2e else 0.0], dev)
    if e2e:
        e2e["value"] = e2e_max

    # ---- roofline of the dominant kernel (live CUDA-event timing in the timed region) ----
    peak, peak_kind = measured_peak()
    traffic = profiled_traffic()
    kernels = []
    for e in prof:
        if e["total_ms"] > 0:
            gbs = e["bytes"] / (e["total_ms"] / 1e3) / 1e9
            kernels.append(dict(name=e["name"], launches=e["launches"], total_ms=round(e["total_ms"], 3),
                                achieved_gbs=round(gbs, 1), frac=round(gbs / peak, 3)))
    # step budget: device time of every library kernel class in the profiled pass
    # (the same solves as the timed pass) against the timed time per solve
    device_ms = sum(e["total_ms"] for e in prof) / max(1, args.steps)
    budget = {"device_ms_per_solve": round(device_ms, 4),
              "ms_per_solve": round(forms[headline]["s_per_solve"] * 1e3, 4),
              "device_fraction": round(device_ms / (forms[headline]["s_per_solve"] * 1e3), 3)}
    single = [k for k in kernels if "graph" not in k["name"]]
    dom = max(single, key=lambda k: k["total_ms"]) if single else None
    dom_e = next(e for e in prof if dom and e["name"] == dom["name"]) if dom else None
    roofline = None
    if dom:
        roofline = {"kernel": dom["name"], "bound": "hbm", "achieved": dom["achieved_gbs"], "peak": peak,
                    "peak_kind": f"{peak_kind} ({'of measured' if peak_kind == 'measured' else 'of fallback'})",
                    "unit": "GB/s", "frac": dom["frac"],
                    "bytes_per_launch": dom_e["bytes"] / dom_e["launches"],
                    "traffic": traffic.get(dom["name"])}

    result = None
    if rank == 0:
        cpu = parity = None
        if world == 1 and not args.no_cpu_baseline and "plain_fp64" in amgs:
            cpu, parity = cpu_baseline_and_parity(args.n, amgs["plain_fp64"], A, rhs_list[0], m, mesh, base_fields,
                                                  first_solution)
        result = {
            "metric": METRIC,
            "value": value, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (Krylov) / f32 (V-cycle)", "data": "synthetic (seeded)",
            "config": dict(_config(args.n, n_cells, int(A.nnz), headline), amg_levels=levels,
                           operator_complexity=round(sum(level_nnz) / level_nnz[0], 2),
                           parallelism=f"replicas x{world}"),
            "forms": forms, "case_build_s": case_s,
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks, "roofline": roofline,
            "assembly": assembly,
            "kernels": kernels, "budget": budget, "cpu_baseline": cpu, "parity": parity,
        }
        print(json.dumps(result), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return result


def time_face_loop(ctx, lib, N, mesh, A, fields, dev, lstream, flush, args):
    """Device time of the pressure-corrector assembly (Gauss gradient + face loop
    writing the CSR values, b and phiHbyA) and of the Rhie-Chow face flux, inputs
    resident on the device, L2 flushed before each call; per-kernel achieved
    bandwidth from the library's profiler (CUDA events on its stream)."""
    import torch
    U, rAU, p, fixed, value = fields
    nc, nf = A.n, mesh.host.n_faces
    Ud, rd, pd = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (U, rAU, p))
    bd = torch.empty(nc, dtype=torch.float64, device=dev)
    phid = torch.empty(nf, dtype=torch.float64, device=dev)
    gd = torch.empty(3 * nc, dtype=torch.float64, device=dev)
    fl = torch.empty(nf, dtype=torch.float64, device=dev)
    fx = np.ascontiguousarray(fixed, np.int32)
    vv = np.ascontiguousarray(value, np.float64)
    h = C.c_void_p(A.handle.value)
    ptr = lambda t: C.c_void_p(t.data_ptr())

    def assemble():
        ctx.check(lib.cfdxg_assemble_pressure_correction(ctx.handle, mesh.handle, ptr(Ud), ptr(rd), ptr(pd), 1.0,
                                                         N.ptr(fx), N.ptr(vv), N.CFDXG_MEM_DEVICE, C.byref(h),
                                                         ptr(bd), ptr(phid), ptr(gd)), "assembly")

    def flux():
        ctx.check(lib.cfdxg_rhie_chow_flux(ctx.handle, mesh.handle, ptr(Ud), ptr(rd), ptr(pd), 1.0, N.ptr(fx),
                                           N.ptr(vv), N.CFDXG_MEM_DEVICE, ptr(fl)), "rhie-chow flux")

    out = {}
    for name, fn in (("assembly", assemble), ("rhie_chow_flux", flux)):
        for _ in range(args.warmup):
            fn()
        ctx.profile(True)
        ts = []
        for s in range(args.steps):
            flush.fill_(float(s))
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(lstream)
            fn()
            e1.record(lstream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        prof = ctx.profile_read()
        ctx.profile(False)
        out[f"{name}_ms"] = float(np.mean(ts))
        for e in prof:
            if e["total_ms"] > 0:
                gbs = e["bytes"] / (e["total_ms"] / 1e3) / 1e9
                out.setdefault("kernels", {})[e["name"]] = {
                    "launches": e["launches"], "ms_per_launch": e["total_ms"] / e["launches"],
                    "bytes_per_launch": e["bytes"] / e["launches"], "achieved_gbs": round(gbs, 1)}
    peak, kind = measured_peak()
    for v in out.get("kernels", {}).values():
        v["frac"] = round(v["achieved_gbs"] / peak, 3)
    out["peak_gbs"] = peak
    out["peak_kind"] = kind
    out["workload"] = f"{nc} cells, {nf} faces, {A.nnz} nonzeros"
    return out


def _export_levels(amg):
    return [amg.export_level(l) for l in range(len(amg.hierarchy_level_sizes()))]


def reference_hierarchy(n, ro, co, va):
    """The reference's own AMG hierarchy of the n^3 system: its setup's stored
    C/F interpolation (oracle/_ref/tet{n}_transfers.npz, written by
    oracle/reference_hierarchy.py from a complete run of the reference's setup)
    with every other setup step -- Galerkin products, diagonals, damping -- run
    by the reference's own code, then checked level by level against the
    committed SHA-256 of that complete setup.  -> (ref.Amg, info) or (None, info)."""
    from oracle import ref
    from oracle import reference_hierarchy as rh
    got = rh.load_transfers(n) if ref.available() else None
    if got is None:
        return None, {"hierarchy": "stored reference transfers absent"}
    transfers, rows, gold = got
    t = time.perf_counter()
    R = ref.AmgFromTransfers(ro, co, va, transfers, rows)
    rebuild_s = time.perf_counter() - t
    hashes = ref.hierarchy_sha256(R)
    match = len(hashes) == len(gold["levels"]) and R.omega == gold["omega"] and all(
        all(g.get(k) == v for k, v in h.items()) for h, g in zip(hashes, gold["levels"]))
    what = ("the reference's own setup (stored C/F interpolation of a complete run, Galerkin products rebuilt by "
            "its code); per-level SHA-256 " + ("equal to that run's" if match else "DIFFERENT from that run's"))
    return R, {"hierarchy": what, "fingerprint_match": bool(match), "rebuild_s": rebuild_s,
               "reference_setup_s": gold["setup_seconds"], "levels": len(hashes), "fingerprint": hashes}


class _CpuSolver:
    """The reference's CPU solve phase: the reference itself (oracle/_ref, kind
    "reference") on its own hierarchy where that is stored, else on the library's
    host-built hierarchy (bit-identical to the reference's, as the tests check);
    the plain-C restatement (oracle/cfdx_oracle.c, kind "port") where the
    reference build is absent."""

    def __init__(self, n, amg, ro, co, va):
        from oracle import ref
        self.info = {}
        self.R = None
        if ref.available():
            self.kind = "reference"
            self.R, self.info = reference_hierarchy(n, ro, co, va)
            if self.R is None:
                self.R = ref.AmgFromLevels(_export_levels(amg), amg.omega)
                self.info["hierarchy"] = "library host setup loaded into the reference's V-cycle"
        else:
            from oracle import cfdx_oracle as co_
            self.kind = "port"
            self.co = co_
            self.H = co_.Hierarchy(_export_levels(amg), amg.omega)
            self.csr = (ro, co, va)
            self.info["hierarchy"] = "library host setup (C restatement of the V-cycle)"

    def solve(self, b, max_iterations=1000):
        """-> (solution, iterations, solve seconds)"""
        if self.kind == "reference":
            x, rep = self.R.solve_gmres(b, restart=RESTART, max_iterations=max_iterations, tolerance=TOL)
            return x, rep["iterations"], rep["solve_seconds"]
        t = time.perf_counter()
        x, rep = self.co.solve_gmres(*self.csr, b, self.H, restart=RESTART, max_iterations=max_iterations,
                                     tolerance=TOL)
        return x, rep["iterations"], time.perf_counter() - t


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def cpu_baseline_and_parity(n, amg, A, b, m, mesh, fields, first_solution):
    """The reference's solve phase on the same system and first right-hand side
    (one host core), and the GPU forms' parity against its solution: pressure
    relative L2, iteration count and the corrected face fluxes of each
    solution (make_rhie_chow_mass_flux: the library's on the GPU, the
    reference's own on the host)."""
    import cfdx_dev_b200 as cg
    ro, co, va = (np.ascontiguousarray(a, t) for a, t in zip(A.to_csr(), (np.int64, np.int64, np.float64)))
    S = _CpuSolver(n, amg, ro, co, va)
    t = time.time()
    x_ref, iters, sec = S.solve(b)
    cpu = {"value": sec, "unit": "s", "cores": 1, "kind": S.kind, "iterations": iters, "wall_s": time.time() - t,
           "sample": "one complete GMRES(30)+NativeAMG solve phase to 1e-8 on the full system, first right-hand "
                     "side; hierarchy: " + S.info.get("hierarchy", "")}
    U, rAU, p, fixed, value = fields
    parity = {"tolerance_rel_l2": 1e-10, "reference": S.kind, "reference_iterations": int(iters),
              "hierarchy": S.info.get("hierarchy")}
    if "rebuild_s" in S.info:
        parity["reference_hierarchy_fingerprint_match"] = S.info["fingerprint_match"]
        parity["reference_rebuild_s"] = S.info["rebuild_s"]
        parity["reference_setup_s"] = S.info["reference_setup_s"]
        # the library's own host setup against the reference's setup, level by level
        parity["library_hierarchy_equals_reference"] = _library_fingerprint(amg) == S.info["fingerprint"]
    if S.kind == "reference":
        from oracle import ref
        r = ref.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
        parity["assembly_bit_exact"] = bool(np.array_equal(r["row_offsets"], ro) and np.array_equal(
            r["columns"], co) and np.array_equal(r["values"], va) and np.array_equal(r["b"], b))
        flux_ref = ref.rhie_chow_flux(m, U, rAU, x_ref, 1.0, fixed, value)
    else:
        from oracle import cfdx_oracle as co_
        flux_ref = co_.rhie_chow_flux(m, U, rAU, x_ref, 1.0, fixed, value)
    forms = {}
    for form, (x, its) in first_solution.items():
        flux = cg.make_rhie_chow_mass_flux(mesh, U, rAU, x, 1.0, fixed, value)
        forms[form] = {"pressure_rel_l2": rel_l2(x, x_ref), "flux_rel_l2": rel_l2(flux, flux_ref),
                       "iterations": int(its)}
    parity["forms"] = forms
    if "plain_fp64" in forms:
        f = forms["plain_fp64"]
        parity["plain_fp64_within_tolerance"] = bool(f["pressure_rel_l2"] <= 1e-10 and f["flux_rel_l2"] <= 1e-10)
        parity["plain_fp64_same_iterations"] = f["iterations"] == int(iters)
    return cpu, parity


def _library_fingerprint(amg):
    from oracle import ref
    out = []
    for l in range(len(amg.hierarchy_level_sizes())):
        out += ref.fingerprint_levels([amg.export_level(l)])
    return out


def run_reference(args):
    """Reference arm: the reference's own CPU implementation of the path on this
    config, loading only oracle libraries -- inputs from the generator compiled
    alone (oracle/cases.py), geometry and corrector assembly by the reference's
    code, its own AMG hierarchy (reference_hierarchy), and one complete
    GMRES(30) solve to 1e-8 per step (about 27 s each on one core, so the arm
    runs at most one warm-up and three timed solves)."""
    rank, local_rank, world = dist_env()
    if rank != 0:
        return None
    from oracle import cases as oc
    from oracle import ref
    from oracle import reference_hierarchy as rh
    base = {"impl": "reference", "metric": METRIC}
    if not ref.available() or rh.load_transfers(args.n) is None:
        out = dict(base, unavailable="the reference build (oracle/_ref) or its stored 64^3 AMG transfers are "
                                     "absent; its own setup takes hours at this size")
        print(json.dumps(out), flush=True)
        return out
    t0 = time.time()
    m = oc.simple_mesh(args.n)
    g = ref.geometry(m)
    U, rAU, aP, p, fixed, value = oc.simple_fields(m, g["cell_centres"])
    r = ref.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    case_s = time.time() - t0
    gold = rh.load_transfers(args.n)[2]
    system_match = rh.system_sha256(r) == gold["system"]
    R, info = reference_hierarchy(args.n, r["row_offsets"], r["columns"], r["values"])
    warmup, steps = min(args.warmup, 1), min(args.steps, 3)
    for _ in range(warmup):
        R.solve_gmres(r["b"], restart=RESTART, tolerance=TOL)
    ts, its = [], []
    for _ in range(steps):
        x, rep = R.solve_gmres(r["b"], restart=RESTART, tolerance=TOL)
        if rep["status"] != 0:
            raise RuntimeError(f"reference solve did not converge: {rep}")
        ts.append(rep["solve_seconds"])
        its.append(rep["iterations"])
    v = float(np.mean(ts))
    out = dict(base, value=v, unit="s", n_gpus=world, steps=steps, warmup=warmup, steps_requested=args.steps,
               warmup_requested=args.warmup, ms_per_step=v * 1e3, higher_is_better=False, scaling="weak",
               vs_baseline=None, dtype="f64", data="synthetic (seeded)",
               config=_config(args.n, m.n_cells, int(r["columns"].size), "plain_fp64 (the reference, host)"),
               iterations=float(np.mean(its)), case_build_s=case_s, hierarchy_rebuild_s=info["rebuild_s"],
               hierarchy_fingerprint_match=info["fingerprint_match"], system_fingerprint_match=system_match,
               reference_setup_s=gold["setup_seconds"],
               cpu_baseline={"value": v, "unit": "s", "cores": 1, "kind": "reference",
                             "sample": f"{steps} complete GMRES(30)+NativeAMG solves to 1e-8 of the full system "
                                       f"(one per step, first right-hand side) on the reference's own hierarchy "
                                       f"({info['hierarchy']}; its setup took {gold['setup_seconds']:.0f} s once, "
                                       f"not timed here)"},
               e2e={"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    print(json.dumps(out), flush=True)
    return out


def _config(n, cells, nnz, form):
    return {"workload": f"Kuhn-tet {n}^3 x6 = {cells} cells, SIMPLE pressure correction, "
                        f"{N_RHS} seeded RHS, GMRES/FGMRES({RESTART}) + native RS AMG to 1e-8",
            "form": form, "cells": cells, "nnz": nnz,
            "l2": "inputs > L2 and L2 flushed before every timed step", "parallelism": "replicas x1"}


def run_config5(args):
    """SIMPLE outer iterations (cfdx_dev_b200/simple_loop.py) on the anisotropic
    boundary-layer hex mesh, 256 x 256 x 64 = 4,194,304 cells, in the three
    forms; per form the AMG setup, numeric refreshes, solves, assembly, face
    flux and host-side momentum stand-in are reported separately (wall clock
    around each synchronised step) with the continuity defect per iteration."""
    import torch

    import cfdx_dev_b200 as cg
    from cfdx_dev_b200 import simple_loop as sl
    rank, local_rank, world = dist_env()
    if rank != 0:
        return None
    torch.cuda.set_device(local_rank)
    ctx = cg.Context(local_rank)
    t = time.perf_counter()
    m = cg.boundary_layer_case(256, 256, 64, 10.0, 1.0, 1e-4, 1.08, 0.05, sl.SEED)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    nu_t = sl.smoothed_eddy_ratio(m, sl.SEED + 2)
    case_s = time.perf_counter() - t
    net = None
    forms = ["plain_fp64", "fp32_vcycle"]
    if WEIGHTS.exists() and not args.no_learned:
        net = cg.LearnedPreconditioner(ctx)
        net.load(str(WEIGHTS))
        forms.append("learned_fp32")
    out = {}
    for form in forms:
        r = sl.run_form(ctx, form, m, mesh, g, nu_t, args.outer_iterations, 0.3, net, ctx.synchronize)
        tot = r["totals"]
        out[form] = {"totals": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in tot.items()},
                     "continuity_l2": [round(x["continuity_l2"], 9) for x in r["records"]],
                     "krylov_iterations": [x["krylov_iterations"] for x in r["records"]],
                     "solve_s_per_iteration": round(tot["solve_s"] / args.outer_iterations, 5),
                     "refresh_s_per_refresh": round(tot["amg_refresh_s"] / max(1, tot["refreshes"]), 5)}
    line = {"metric": "SIMPLE outer iterations on the 256x256x64 boundary-layer mesh (config 5)",
            "unit": "s", "n_gpus": 1, "outer_iterations": args.outer_iterations, "cells": m.n_cells,
            "case_build_s": case_s, "data": "synthetic (seeded)", "forms": out}
    print(json.dumps(line), flush=True)
    ctx.close()
    return line


def main():
    args = parse_args()
    if args.config == 5:
        run_config5(args)
        return
    if args.warmup < 3 and args.impl == "cfdxg":
        raise SystemExit("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_cfdxg(args)


if __name__ == "__main__":
    main()
