"""GPU kernels of the learned preconditioner against the FP64 oracle
(oracle/mpnn_oracle.py, itself pinned by finite differences)."""
import numpy as np
import pytest

import cfdx_dev_b200 as cg
from oracle import mpnn_oracle as mo
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bound(ctx):
    m = cases.simple_mesh(6)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    ro, co, va = A.to_csr()
    G = mo.Graph(ro, co, va, g["cell_volumes"], aP)
    net = cg.LearnedPreconditioner(ctx, seed=3)
    net.bind(mesh, A, aP)
    theta = mo.init_params(5)
    net.set_parameters(theta.astype(np.float32))
    theta32 = net.parameters().astype(np.float64)
    return dict(mesh=mesh, A=A, b=b, G=G, net=net, theta=theta32, aP=aP, m=m)


def _pairs(G, k=2, seed=0):
    rng = np.random.default_rng(seed)
    R, E = [], []
    for _ in range(k):
        e = rng.standard_normal(G.n)
        R.append(G.matvec(e) + 0.05 * rng.standard_normal(G.n))
        E.append(e)
    return np.array(R), np.array(E)


def test_parameter_count_matches_oracle(bound):
    assert bound["net"].n_params == mo.N_PARAMS


def test_training_gradient_matches_oracle(bound):
    G, net, theta = bound["G"], bound["net"], bound["theta"]
    R, E = _pairs(G)
    loss, grad = net.loss_grad(R, E)
    loss_ref, grad_ref = mo.loss_and_grad(theta, G, list(zip(R, E)))
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    # FP32 kernels vs FP64 oracle
    assert np.linalg.norm(grad - grad_ref) <= 1e-4 * np.linalg.norm(grad_ref)


def test_composed_training_gradient_matches_oracle(bound, oracle):
    """Gradient of the learned stage in front of the V-cycle; the oracle runs the
    same hierarchy with the reference's V-cycle (bit-identical to the device's in
    reference summation order)."""
    G, net, theta, A = bound["G"], bound["net"], bound["theta"], bound["A"]
    amg = cg.NativeBoomerAMGPreconditioner(net.ctx, reference_order=1)
    assert amg.setup(A)
    R_amg = oracle.Hierarchy([amg.export_level(l) for l in range(len(amg.hierarchy_level_sizes()))], amg.omega)
    net.set_vcycle(amg)
    try:
        R, E = _pairs(G, seed=7)
        loss, grad = net.loss_grad(R, E)
        loss_ref, grad_ref = mo.loss_and_grad(theta, G, list(zip(R, E)), M=R_amg.apply)
    finally:
        net.set_vcycle(None)
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    assert np.linalg.norm(grad - grad_ref) <= 1e-4 * np.linalg.norm(grad_ref)


def test_tensor_core_inference_matches_oracle(bound):
    G, net, theta = bound["G"], bound["net"], bound["theta"]
    r = np.random.default_rng(4).standard_normal(G.n)
    y = net.apply(r)
    y_ref = mo.forward(theta, G, r)
    # BF16 operands, FP32 accumulation
    assert np.linalg.norm(y - y_ref) <= 3e-2 * np.linalg.norm(y_ref)
    assert np.allclose(net.apply(2.0 * r), 2.0 * y, rtol=1e-5, atol=1e-12 * np.abs(y).max())


def test_training_reduces_loss_and_weights_roundtrip(bound, tmp_path):
    G, net = bound["G"], bound["net"]
    R, E = _pairs(G, 4, seed=1)
    l0 = net.train_step(R, E, lr=3e-3)
    for _ in range(30):
        l1 = net.train_step(R, E, lr=3e-3)
    assert l1 < 0.7 * l0
    p = net.parameters()
    path = tmp_path / "w.bin"
    net.save(path)
    net2 = cg.LearnedPreconditioner(net.ctx, seed=99)
    net2.load(path)
    assert np.array_equal(net2.parameters(), p)
    raw = bytearray(path.read_bytes())
    raw[40] ^= 0xFF
    path.write_bytes(bytes(raw))
    with pytest.raises(cg.CfdxgError):
        net2.load(path)


def test_learned_fgmres_converges_with_fallback_accounting(bound):
    A, b, net = bound["A"], bound["b"], bound["net"]
    x, rep = cg.solve_linear_system(A, b, krylov="fgmres", precision="fp32_vcycle", restart=30, tolerance=1e-8,
                                    learned=net)
    assert rep["status_name"] == "converged"
    assert rep["physical_residual_relative"] <= 1e-8
    assert 0 <= rep["learned_fallbacks"] <= rep["preconditioner_applications"]


WEIGHTS = cases.ROOT / "cfdx_dev_b200" / "weights" / "mpnn.bin"


@pytest.mark.skipif(not WEIGHTS.exists(), reason="no trained weights committed")
def test_trained_network_gain_over_vcycle_alone(ctx, capsys):
    """What the trained network gains over the method without it, on a mesh it
    was not trained on: the A-norm error of the learned stage in front of the
    FP32 V-cycle, against the V-cycle alone, on solver residuals (the
    right-hand side and white noise, each also after two V-cycle Richardson
    steps); an untrained network of the same shape is the control.  The FGMRES
    iteration counts with and without the learned stage are reported."""
    m = cases.simple_mesh(20, seed_offset=77)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"], seed_offset=77)
    A, b, phi, grad = cg.assemble_pressure_correction(mesh, U, rAU, p, 1.0, fixed, value)
    M = cg.NativeBoomerAMGPreconditioner(ctx, precision="fp32_vcycle")
    assert M.setup(A)
    M64 = cg.NativeBoomerAMGPreconditioner(ctx)
    assert M64.setup(A)
    trained = cg.LearnedPreconditioner(ctx)
    trained.load(WEIGHTS)
    trained.bind(mesh, A, aP)
    control = cg.LearnedPreconditioner(ctx, seed=1)
    control.bind(mesh, A, aP)

    def energy(v):
        return float(v @ A.matvec(v))

    ratios = {"trained": [], "control": []}
    rng = np.random.default_rng(5)
    for r0 in (b, rng.standard_normal(A.n)):
        r0 = r0 / np.sqrt(np.mean(r0 * r0))
        e0, rep = cg.solve_gmres(A, r0, amg=M64, restart=30, tolerance=1e-12)
        assert rep["status_name"] == "converged"
        for steps in (0, 2):
            r, e = r0.copy(), e0.copy()
            for _ in range(steps):
                e = e - M.apply(r)
                r = A.matvec(e)
            base = energy(e - M.apply(r))
            for label, net in (("trained", trained), ("control", control)):
                y = net.apply(r)
                z = y + M.apply(r - A.matvec(y))
                ratios[label].append(energy(e - z) / base)
    its = {}
    for label, kw in (("fp32_vcycle", {}), ("learned_first", dict(learned=trained, learned_applications=1)),
                      ("learned_every", dict(learned=trained, learned_applications=0))):
        x, rep = cg.solve_fgmres(A, b, amg=M, restart=30, tolerance=1e-8, **kw)
        assert rep["status_name"] == "converged" and rep["physical_residual_relative"] <= 1e-8
        its[label] = rep["iterations"]
    with capsys.disabled():
        print(f"\nlearned-stage A-norm error / V-cycle alone: trained {np.round(ratios['trained'], 3)}, "
              f"untrained {np.round(ratios['control'], 3)}; FGMRES iterations {its}")
    assert max(ratios["trained"]) < 0.8
    assert np.mean(ratios["trained"]) < 0.8 * np.mean(ratios["control"])
