"""The FP64 CPU oracle of the learned preconditioner: its analytic gradient
agrees with central finite differences (this pins the oracle the GPU kernels
are checked against)."""
import numpy as np

import cfdx_dev_b200 as cg
from oracle import mpnn_oracle as mo
from tests import cases


def small_graph(ref, n=3):
    m = cases.simple_mesh(n)
    g = ref.geometry(m)
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    r = ref.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    G = mo.Graph(r["row_offsets"], r["columns"], r["values"], g["cell_volumes"], aP)
    return G, r


def test_param_count():
    assert mo.N_PARAMS == 4 * 32 + 32 + 4 * (32 * 64 + 32 + 32 * 32 + 32) + 32 + 1


def test_oracle_gradient_matches_finite_differences(ref):
    G, r = small_graph(ref)
    rng = np.random.default_rng(0)
    theta = mo.init_params(1)
    pairs = []
    for _ in range(2):
        e = rng.standard_normal(G.n)
        pairs.append((G.matvec(e) + 0.1 * rng.standard_normal(G.n), e))
    L, grad = mo.loss_and_grad(theta, G, pairs)
    idx = rng.choice(theta.size, 40, replace=False)
    for i in idx:
        h = 1e-6 * max(1.0, abs(theta[i]))
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (mo.loss_and_grad(tp, G, pairs)[0] - mo.loss_and_grad(tm, G, pairs)[0]) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, grad[i])


def test_oracle_is_homogeneous_in_the_residual(ref):
    G, r = small_graph(ref)
    theta = mo.init_params(2)
    x = np.random.default_rng(1).standard_normal(G.n)
    y1 = mo.forward(theta, G, x)
    y2 = mo.forward(theta, G, 3.5 * x)
    assert np.allclose(3.5 * y1, y2, rtol=1e-12, atol=0)
    assert np.all(mo.forward(theta, G, 0 * x) == 0)


def test_oracle_composed_gradient_matches_finite_differences(ref):
    """Loss of N in front of the (symmetric) reference V-cycle."""
    G, r = small_graph(ref, 4)
    R = ref.Amg(r["row_offsets"], r["columns"], r["values"])
    rng = np.random.default_rng(2)
    theta = mo.init_params(3)
    pairs = []
    for _ in range(2):
        e = rng.standard_normal(G.n)
        pairs.append((G.matvec(e), e))
    L, grad = mo.loss_and_grad(theta, G, pairs, M=R.apply)
    for i in rng.choice(theta.size, 30, replace=False):
        h = 1e-6 * max(1.0, abs(theta[i]))
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (mo.loss_and_grad(tp, G, pairs, M=R.apply)[0] - mo.loss_and_grad(tm, G, pairs, M=R.apply)[0]) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, grad[i])
