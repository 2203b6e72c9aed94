"""The SIMPLE outer iteration on the GPU against the same chain built from the
C oracle.

cfdx_dev_b200/simple_loop.py runs the reference's pressure-side chain per
outer iteration: rAU from the momentum diagonal, HbyA by build_hbya
(physics/steady_incompressible_solver.h:6430-6465), the pressure-corrector
assembly (:8048-8181), AMG setup then numeric refresh, the pressure solve,
p += alpha_p p' (:9339-9343), the corrected face fluxes
(make_rhie_chow_mass_flux, :2064-2217), grad p and the velocity correction.
The oracle chain below takes the same steps with oracle/cfdx_oracle.c (HbyA,
assembly, GMRES on the same hierarchy, flux, gradient; the hierarchy from the
library's host setup and host refresh, which the CPU tests pin to the
reference's).  Five iterations: HbyA, b and the fluxes agree to 1e-10 (the
first iteration's HbyA and b bit for bit), the pressure to 1e-10, with equal
Krylov iteration counts.
"""
import numpy as np
import pytest

import cfdx_dev_b200 as cg
from cfdx_dev_b200 import simple_loop as sl

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10
ITERATIONS = 5
ALPHA_P = 0.3


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def oracle_chain(oracle, m, nu_t, iterations, alpha_p):
    g = oracle.geometry(m)
    nc = m.n_cells
    vol = g["cell_volumes"]
    fixed = np.zeros(m.n_patches, np.int32)
    fixed[0] = 1
    value = np.zeros(m.n_patches)
    U, p, phi = sl.initial_state(m, g)
    gradp = np.zeros(3 * nc)
    pattern = sl.cell_pattern(m)
    amg = cg.NativeBoomerAMGPreconditioner(None)
    states = []
    for k in range(iterations):
        va, aP = sl.momentum_values(m, g, nu_t, phi, pattern)
        rAU = np.concatenate([1.0 / aP] * 3)
        rhs = -(gradp.reshape(3, nc) * vol[None, :]).ravel()
        HbyA = oracle.build_hbya(pattern[0], pattern[1], np.tile(va, 3), rhs, U, gradp, vol, rAU)
        r = oracle.simple_assemble(m, HbyA, rAU, p, 1.0, fixed, value)
        csr = (r["row_offsets"], r["columns"], r["values"])
        if k == 0 or not amg.update_values_host(*csr):
            assert amg.setup_host(*csr), amg.last_error()
        H = oracle.Hierarchy([amg.export_level(l) for l in range(len(amg.hierarchy_level_sizes()))], amg.omega)
        dp, rep = oracle.solve_gmres(*csr, r["b"], H, restart=30, tolerance=1e-8)
        assert rep["status"] == 0, rep
        p = p + alpha_p * dp
        phi = oracle.rhie_chow_flux(m, HbyA, rAU, p, 1.0, fixed, value)
        gradp = oracle.gauss_gradient(m, p, fixed, value)
        U = (HbyA.reshape(3, nc) - vol[None, :] * rAU.reshape(3, nc) * gradp.reshape(3, nc)).ravel()
        states.append({"HbyA": HbyA, "b": r["b"], "p": p.copy(), "phi": phi, "iterations": rep["iterations"]})
    return states


def test_build_hbya_bit_exact(ctx, oracle):
    m = cg.boundary_layer_case(10, 8, 6, 10.0, 1.0, 1e-3, 1.2, 0.05, 11)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    nc = m.n_cells
    rng = np.random.default_rng(3)
    pattern = sl.cell_pattern(m)
    va3 = [sl.momentum_values(m, g, sl.smoothed_eddy_ratio(m, s), rng.standard_normal(m.n_faces), pattern)[0]
           for s in (1, 2, 3)]
    rhs, U, gradp = (rng.standard_normal(3 * nc) for _ in range(3))
    rAU = 1.0 / rng.uniform(1.0, 100.0, 3 * nc)
    mats = [cg.SparseMatrix.from_csr(ctx, pattern[0], pattern[1], v) for v in va3]
    got = cg.build_hbya(mesh, mats, rhs, U, gradp, rAU)
    want = oracle.build_hbya(pattern[0], pattern[1], np.concatenate(va3), rhs, U, gradp, g["cell_volumes"], rAU)
    assert np.array_equal(got, want)
    # a non-finite HbyA is refused, as the reference throws
    bad = rAU.copy()
    bad[5] = np.inf
    with pytest.raises(cg.CfdxgError):
        cg.build_hbya(mesh, mats, rhs, U, gradp, bad)


def test_simple_outer_iterations_match_oracle_chain(ctx, oracle):
    m = cg.boundary_layer_case(16, 12, 8, 10.0, 1.0, 1e-3, 1.15, 0.05, sl.SEED)
    mesh = cg.Mesh(ctx, m)
    g = mesh.geometry()
    nu_t = sl.smoothed_eddy_ratio(m, sl.SEED + 2)
    got = sl.run_form(ctx, "plain_fp64", m, mesh, g, nu_t, ITERATIONS, ALPHA_P, None, ctx.synchronize,
                      keep=True)["states"]
    want = oracle_chain(oracle, m, nu_t, ITERATIONS, ALPHA_P)
    # the first iteration starts from identical inputs: bit-identical HbyA and b
    assert np.array_equal(got[0]["HbyA"], want[0]["HbyA"])
    assert np.array_equal(got[0]["b"], want[0]["b"])
    for k, (a, b) in enumerate(zip(got, want)):
        assert a["iterations"] == b["iterations"], k
        for key in ("HbyA", "b", "p", "phi"):
            assert rel_l2(a[key], b[key]) <= REL_TOL, (k, key, rel_l2(a[key], b[key]))
    # the chain reduces the continuity defect
    assert np.linalg.norm(got[-1]["b"]) < np.linalg.norm(got[0]["b"])
