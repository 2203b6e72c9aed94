"""Train the learned message-passing preconditioner on the GPU.

Training data are (residual, error) pairs that the plain solver itself
generates: on seeded Kuhn-tet meshes of lattice sizes between --min-n and
--max-n (6 tets per hex, interior vertices jittered by +-0.15h) the
pressure-correction system is assembled, and for each residual r the error
e = A^-1 r is obtained with plain FP64 AMG-GMRES to a relative residual of
1e-10.  Residuals mix the assembled continuity right-hand sides (other HbyA
seeds), white noise, and smooth fields mapped through A; half of them are then
advanced 1..--richardson-steps steps of the V-cycle-preconditioned Richardson
iteration (the error is updated exactly alongside), which leaves the slowly
converging components the learned stage is meant to remove.  The loss is the
A-norm of the error of the composed preconditioner z = N(r) + M(r - A N(r))
with M the FP32 AMG V-cycle, ||(I - M A)(e - N(r))||_A^2 / ||(I - M A) e||_A^2
(below 1 when the learned stage improves on the V-cycle alone), minimised with
Adam by the library's own forward and backward kernels.

    python -m cfdx_dev_b200.train_mpnn --meshes 64 --pairs-per-mesh 16 \
        --min-n 16 --max-n 40 --epochs 30 --out weights.bin

Data-parallel over the GPUs of one node (one process per GPU, NCCL):

    torchrun --nproc-per-node 8 --master-addr 127.0.0.1 -m cfdx_dev_b200.train_mpnn --meshes 64 ...

Each rank generates and holds its own meshes (mesh i goes to rank i mod
world); every step each rank takes the loss gradient of its own batch with the
library's kernels, one all-reduce averages the gradients weighted by the pair
counts, and every rank applies the same FP32 Adam update, so the parameters
stay identical everywhere.
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

SEED_BASE = 7_000_000


class DataParallelAdam:
    """Adam on gradients averaged over the processes of a torch.distributed group.

    ``step(grad, loss, count)`` takes this process's mean loss gradient over
    ``count`` pairs; one all-reduce of [count * grad, count * loss, count]
    gives the mean over every pair of every process, and the update is the
    library's FP32 Adam (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected:
    the k_adam kernel of train_step) applied identically on every process.
    Without a process group it is plain Adam on one process's gradient."""

    def __init__(self, params, lr: float, group=None):
        self.p = np.array(params, np.float32)
        self.m = np.zeros_like(self.p)
        self.v = np.zeros_like(self.p)
        self.t = 0
        self.lr = np.float32(lr)
        self.group = group

    def _allreduce(self, buf: np.ndarray) -> np.ndarray:
        import torch
        import torch.distributed as dist
        if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(self.group) == 1:
            return buf
        backend = dist.get_backend(self.group)
        dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        t = torch.as_tensor(buf, device=dev)
        dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def step(self, grad, loss: float, count: int, lr: float | None = None):
        """One update; returns (mean loss over all pairs, new parameters)."""
        g = np.asarray(grad, np.float64)
        buf = np.concatenate([g * count, [loss * count, float(count)]])
        buf = self._allreduce(buf)
        total = buf[-1]
        g = (buf[:-2] / total).astype(np.float32)
        self.t += 1
        f32 = np.float32
        bc1 = f32(1.0) - f32(0.9) ** f32(self.t)
        bc2 = f32(1.0) - f32(0.999) ** f32(self.t)
        self.m = f32(0.9) * self.m + f32(0.1) * g
        self.v = f32(0.999) * self.v + f32(0.001) * g * g
        step_lr = self.lr if lr is None else f32(lr)
        self.p = self.p - step_lr * (self.m / bc1) / (np.sqrt(self.v / bc2) + f32(1e-8))
        return float(buf[-2] / total), self.p


def make_system(ctx, n, seed):
    """Jittered Kuhn-tet mesh, pressure-correction matrix and its inputs."""
    m = cg.tet_case(n, 0.15, SEED_BASE + seed)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    aP = cg.random_field(m.n_cells, "loguniform", 1.0, 100.0, SEED_BASE + 1000 + seed)
    rAU = np.concatenate([1.0 / aP] * 3)
    fixed = np.zeros(m.n_patches, np.int32)
    fixed[0] = 1
    value = np.zeros(m.n_patches)
    U = cg.fourier_field(g["cell_centres"], 8, 0.01, SEED_BASE + 2000 + seed)
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, np.zeros(m.n_cells), 1.0, fixed, value)
    return dict(m=m, mesh=mesh, g=g, aP=aP, rAU=rAU, fixed=fixed, value=value, A=A)


def make_pairs(ctx, sysd, k, seed, richardson_steps=0):
    """k (r, e) pairs; e solved with the plain FP64 AMG-GMRES path.

    With richardson_steps > 0, the second half of the pairs are carried
    1..richardson_steps steps of the preconditioned Richardson iteration with
    the FP32 V-cycle M (e <- e - M r, r <- A e): the residuals the Krylov
    solver meets after the V-cycle has removed what it handles well."""
    A, m, g = sysd["A"], sysd["m"], sysd["g"]
    amg = cg.NativeBoomerAMGPreconditioner(ctx)
    if not amg.setup(A):
        raise RuntimeError(amg.last_error())
    # the FP32 V-cycle the learned stage runs in front of
    sysd["vcycle"] = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp32_vcycle")
    if not sysd["vcycle"].setup(A):
        raise RuntimeError(sysd["vcycle"].last_error())
    rng = np.random.default_rng(SEED_BASE + 3000 + seed)
    R, E = [], []
    for q in range(k):
        kind = q % 3
        if kind == 0:   # continuity residual of another predictor field
            U = cg.fourier_field(g["cell_centres"], 8, 0.01, SEED_BASE + 4000 + 97 * seed + q)
            _, r, _, _ = cg.assemble_pressure_correction(sysd["mesh"], U, sysd["rAU"], np.zeros(m.n_cells), 1.0,
                                                         sysd["fixed"], sysd["value"])
        elif kind == 1:  # white noise
            r = rng.standard_normal(m.n_cells)
        else:            # smooth field through the operator
            u = cg.fourier_field(g["cell_centres"], 4, 0.0, SEED_BASE + 5000 + 97 * seed + q)[:m.n_cells]
            r = A.matvec(u + 0.1 * rng.standard_normal(m.n_cells))
        r = r / np.sqrt(np.mean(r * r))
        e, rep = cg.solve_gmres(A, r, amg=amg, restart=30, tolerance=1e-10, max_iterations=2000)
        if rep["status_name"] != "converged":
            raise RuntimeError(f"training pair solve failed: {rep}")
        if richardson_steps and q >= k // 2:
            for _ in range(1 + q % richardson_steps):
                e = e - sysd["vcycle"].apply(r)
                r = A.matvec(e)
            scale = 1.0 / np.sqrt(np.mean(r * r))
            r, e = r * scale, e * scale
        R.append(r)
        E.append(e)
    return np.array(R), np.array(E)


def train(args):
    from cfdx_dev_b200 import replicas
    rank, local_rank, world = replicas.dist_env()
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if args.meshes % world:
            raise SystemExit("--meshes must be a multiple of the number of processes")
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ctx = cg.Context(local_rank)
    net = cg.LearnedPreconditioner(ctx, seed=args.seed)
    opt = DataParallelAdam(net.parameters(), args.lr) if world > 1 else None
    sizes = np.linspace(args.min_n, args.max_n, args.meshes).round().astype(int)
    data = []
    t0 = time.time()
    for i, n in enumerate(sizes):
        if i % world != rank:
            continue
        sysd = make_system(ctx, int(n), i)
        R, E = make_pairs(ctx, sysd, args.pairs_per_mesh, i, args.richardson_steps)
        data.append((sysd, R, E))
        print(f"mesh {i} n={n} cells={sysd['m'].n_cells} pairs={len(R)} ({time.time() - t0:.1f}s)", flush=True)
    gen_s = time.time() - t0
    rng = np.random.default_rng(args.seed)
    history = []
    t1 = time.time()
    lr = args.lr
    for epoch in range(args.epochs):
        losses = []
        for i in rng.permutation(len(data)):
            sysd, R, E = data[i]
            net.bind(sysd["mesh"], sysd["A"], sysd["aP"])
            net.set_vcycle(sysd["vcycle"] if args.composed else None)
            for b in range(0, len(R), args.batch):
                Rb, Eb = R[b:b + args.batch], E[b:b + args.batch]
                if opt is None:
                    losses.append(net.train_step(Rb, Eb, lr=lr))
                else:
                    loss, grad = net.loss_grad(Rb, Eb)
                    loss, params = opt.step(grad, loss, len(Rb), lr=lr)
                    net.set_parameters(params)
                    losses.append(loss)
        if epoch == int(0.7 * args.epochs):
            lr *= 0.3
        history.append(float(np.mean(losses)))
        print(f"epoch {epoch} loss {history[-1]:.4f} ({time.time() - t1:.1f}s)", flush=True)
    if rank == 0:
        net.save(args.out)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    summary = {"meshes": len(data), "pairs": int(sum(len(R) for _, R, _ in data)), "rank": rank, "world": world,
               "sizes": [int(s) for s in sizes], "generation_s": gen_s, "training_s": time.time() - t1,
               "loss_history": history, "params": net.n_params, "out": str(args.out)}
    print(json.dumps(summary), flush=True)
    return net, summary


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--meshes", type=int, default=64)
    ap.add_argument("--pairs-per-mesh", type=int, default=16)
    ap.add_argument("--min-n", type=int, default=16)
    ap.add_argument("--max-n", type=int, default=40)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--richardson-steps", type=int, default=4,
                    help="carry half of the pairs up to this many V-cycle Richardson steps (0: off)")
    ap.add_argument("--composed", type=int, default=1,
                    help="1: loss of the learned stage in front of the FP32 V-cycle; 0: the network alone")
    ap.add_argument("--out", type=Path, default=ROOT / "cfdx_dev_b200" / "weights" / "mpnn.bin")
    args = ap.parse_args(argv)
    args.out.parent.mkdir(parents=True, exist_ok=True)
    train(args)


if __name__ == "__main__":
    main()
