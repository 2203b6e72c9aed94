"""Data-parallel training of the learned preconditioner, on CPU.

The training step of ``cfdx_dev_b200.train_mpnn`` over several processes is:
each rank's loss gradient over its own pairs, one all-reduce that averages the
gradients weighted by the pair counts, and the library's FP32 Adam update
applied identically on every rank.  Here the gradients come from the FP64
oracle of the network (oracle/mpnn_oracle.py), the stand-in for the
library's backward kernels, and two gloo ranks are checked against one
process that sees every pair: the same losses and parameters, and parameters
bit-identical across the ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cfdx_dev_b200.train_mpnn import DataParallelAdam
from oracle import cfdx_oracle as co
from oracle import mpnn_oracle as mo
from tests import cases


def _graph_and_pairs(count, seed):
    m = cases.simple_mesh(3)
    g = co.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    a = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    G = mo.Graph(a["row_offsets"], a["columns"], a["values"], g["cell_volumes"], aP)
    rng = np.random.default_rng(seed)
    pairs = []
    for _ in range(count):
        e = rng.standard_normal(G.n)
        pairs.append((G.matvec(e), e))
    return G, pairs


def _adam_reference(p, grads, lr):
    """Textbook bias-corrected Adam in FP64."""
    p = p.astype(np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    for t, g in enumerate(grads, start=1):
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g * g
        p = p - lr * (m / (1 - 0.9 ** t)) / (np.sqrt(v / (1 - 0.999 ** t)) + 1e-8)
    return p


def test_adam_update_is_bias_corrected_adam():
    rng = np.random.default_rng(0)
    p0 = rng.standard_normal(50).astype(np.float32)
    grads = [rng.standard_normal(50) for _ in range(5)]
    opt = DataParallelAdam(p0, 1e-2)
    for g in grads:
        loss, p = opt.step(g, 1.0, 4)
        assert p.dtype == np.float32 and loss == 1.0
    np.testing.assert_allclose(p, _adam_reference(p0, grads, 1e-2), rtol=1e-5, atol=1e-6)
    # the first step moves every parameter by the learning rate against its gradient
    opt = DataParallelAdam(p0, 1e-2)
    _, p = opt.step(grads[0], 0.0, 1)
    np.testing.assert_allclose(p0 - p, 1e-2 * np.sign(grads[0]), rtol=1e-4)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


STEPS, PAIRS = 3, (3, 2)          # rank 0 holds three pairs per step, rank 1 two


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        G, pairs = _graph_and_pairs(STEPS * sum(PAIRS), 11)
        theta = mo.init_params(5).astype(np.float32)
        opt = DataParallelAdam(theta, 3e-3)
        losses = []
        for s in range(STEPS):
            batch = pairs[s * sum(PAIRS):(s + 1) * sum(PAIRS)]
            mine = batch[:PAIRS[0]] if rank == 0 else batch[PAIRS[0]:]
            loss, grad = mo.loss_and_grad(opt.p.astype(np.float64), G, mine)
            loss, _ = opt.step(grad, loss, len(mine))
            losses.append(loss)
        out.put((rank, losses, opt.p))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_train_as_one_process():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, l0, p0), (_, l1, p1) = results
    assert np.array_equal(p0, p1) and l0 == l1                      # every rank holds the same network
    # one process with every pair of each step
    G, pairs = _graph_and_pairs(STEPS * sum(PAIRS), 11)
    opt = DataParallelAdam(mo.init_params(5).astype(np.float32), 3e-3)
    for s in range(STEPS):
        batch = pairs[s * sum(PAIRS):(s + 1) * sum(PAIRS)]
        loss, grad = mo.loss_and_grad(opt.p.astype(np.float64), G, batch)
        loss, _ = opt.step(grad, loss, len(batch))
        assert loss == pytest.approx(l0[s], rel=1e-10)
    np.testing.assert_allclose(p0, opt.p, rtol=1e-5, atol=1e-7)
