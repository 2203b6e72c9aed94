"""Replica bookkeeping of multi-GPU runs, on CPU: two gloo ranks.

The pressure solve runs as independent replicas (one per GPU) with no data-path
collective; the ranks share only the launcher environment, disjoint seed blocks
and the MAX-over-ranks reduction of the time per step.  Here two processes
each solve their own seeded system with the plain-C oracle (the CPU stand-in
for a GPU replica) and reduce their timings as the benchmark does."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cfdx_dev_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    r, lr, w = replicas.dist_env()
    dist.init_process_group("gloo", rank=r, world_size=w, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import cfdx_oracle as co
        from tests import cases
        seeds = replicas.seed_offsets(r, 2)
        m = cases.simple_mesh(3)
        g = co.geometry(m)
        iters, checks = [], []
        for s in seeds:
            U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"], seed_offset=s)
            a = co.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
            x, rep = co.solve_gmres(a["row_offsets"], a["columns"], a["values"], a["b"], None, restart=30,
                                    tolerance=1e-8, max_iterations=500)
            iters.append(rep["iterations"])
            checks.append(float(np.abs(a["b"]).sum()))
        t = replicas.max_over_ranks([10.0 * (r + 1), 5.0 - r, float(max(iters))])
        all_checks = [None] * w
        dist.all_gather_object(all_checks, checks)
        out.put((r, lr, w, seeds, t, all_checks, rep["status"]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_seed_blocks_are_disjoint():
    blocks = [replicas.seed_offsets(r, 16) for r in range(8)]
    flat = [s for b in blocks for s in b]
    assert len(flat) == len(set(flat)) == 128 and blocks[1][0] == 16
    with pytest.raises(ValueError):
        replicas.seed_offsets(-1, 4)


def test_max_over_ranks_without_a_group_is_the_identity():
    assert replicas.max_over_ranks([1.5, -2.0]) == [1.5, -2.0]


def test_two_gloo_ranks_reduce_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, lr0, w0, s0, t0, c0, st0), (r1, lr1, w1, s1, t1, c1, st1) = results
    assert (r0, r1, w0, w1, lr0, lr1) == (0, 1, 2, 2, 0, 1)
    assert set(s0).isdisjoint(s1)
    assert t0 == t1 and t0[:2] == [20.0, 5.0]          # the slowest rank's time, identical on every rank
    assert c0 == c1 and c0[0] != c0[1]                 # the two replicas solved different systems
    assert st0 == st1 == 0
