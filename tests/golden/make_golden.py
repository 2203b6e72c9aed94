"""Regenerates the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own code, compiled from its sources into oracle/_ref
(``make -C oracle ref``; needs the reference source tree), on the seeded
inputs of tests/cases.py and stores its outputs:

* pressure_tet4.npz -- Kuhn-tet 4^3 x 6 pressure-correction system: CSR,
  right-hand side, Rhie-Chow face flux at p = 0 and at the solved pressure,
  the AMG hierarchy (every level's CSR, inverse diagonal and prolongation,
  damping omega), one V-cycle (r, z), the AMG-GMRES(30) solution to 1e-8
  with its iteration count, and the CG + native-AMG solution of the
  reference's solve_linear_system to 1e-10 (cg_x, cg_iterations);
* poisson_hex6.npz -- hex 6^3 Poisson system (CSR and right-hand side);
* neumann_tet5.npz -- the Kuhn-tet 5^3 x 6 pressure-correction system with
  no fixed-pressure patch (a constant null space) and its right-hand side
  less its mean: CSR, the hierarchy of the native AMG built with
  constant_null_space, one V-cycle of it (r, z), and the solutions of the
  reference's solve_linear_system with NullSpaceModel::Constant -- FGMRES(30)
  + native AMG to 1e-8 (projected GMRES) and CG + native AMG to 1e-10;
* pressure_tet4.cfdxlin -- the pressure system of pressure_tet4.npz with a
  zero initial guess, written by the reference's write_linear_system_capture
  (PressurePoisson, no null space, tolerance 1e-8, 1000 iterations).

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import ref  # noqa: E402
from tests import cases  # noqa: E402


def pressure(n: int):
    m = cases.simple_mesh(n)
    g = ref.geometry(m, "fv")
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    a = ref.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    ro, co, va, b = a["row_offsets"], a["columns"], a["values"], a["b"]
    R = ref.Amg(ro, co, va)
    out = dict(n=n, row_offsets=ro, columns=co, values=va, b=b,
               flux=ref.rhie_chow_flux(m, U, rAU, p, 1.0, fixed, value),
               n_levels=R.num_levels(), omega=R.omega)
    for l in range(R.num_levels()):
        lv = R.level(l)
        for k in ("row_offsets", "columns", "values", "inv_diag"):
            out[f"L{l}_{k}"] = lv[k]
        if lv["p_offsets"] is not None:
            for k in ("p_offsets", "p_columns", "p_values"):
                out[f"L{l}_{k}"] = lv[k]
    r = np.random.default_rng(11).standard_normal(ro.size - 1)
    out.update(vcycle_r=r, vcycle_z=R.apply(r))
    x, rep = R.solve_gmres(b, restart=30, tolerance=1e-8)
    assert rep["status"] == 0
    out.update(x=x, iterations=rep["iterations"],
               flux_solved=ref.rhie_chow_flux(m, U, rAU, x, 1.0, fixed, value))
    xc, repc = ref.solve_linear_system(ro, co, va, b, krylov=1, preconditioner=6, max_iterations=1000,
                                       tolerance=1e-10)
    assert repc["status"] == 0
    out.update(cg_x=xc, cg_iterations=repc["iterations"])
    np.savez_compressed(HERE / f"pressure_tet{n}.npz", **out)


def neumann(n: int):
    m = cases.simple_mesh(n)
    g = ref.geometry(m, "fv")
    U, rAU, aP, p, fixed, value = cases.simple_fields(m, g["cell_centres"])
    fixed[:] = 0
    a = ref.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    ro, co, va = a["row_offsets"], a["columns"], a["values"]
    b = a["b"] - a["b"].mean()
    R = ref.Amg(ro, co, va, constant_null_space=True)
    out = dict(n=n, row_offsets=ro, columns=co, values=va, b=b, n_levels=R.num_levels(), omega=R.omega)
    for l in range(R.num_levels()):
        lv = R.level(l)
        for k in ("row_offsets", "columns", "values", "inv_diag"):
            out[f"L{l}_{k}"] = lv[k]
        if lv["p_offsets"] is not None:
            for k in ("p_offsets", "p_columns", "p_values"):
                out[f"L{l}_{k}"] = lv[k]
    r = np.random.default_rng(13).standard_normal(ro.size - 1)
    out.update(vcycle_r=r, vcycle_z=R.apply(r))
    x, rep = ref.solve_linear_system_null_space(ro, co, va, b, krylov=4, preconditioner=6, restart=30,
                                                tolerance=1e-8)
    assert rep["status"] == 0
    out.update(x=x, iterations=rep["iterations"])
    xc, repc = ref.solve_linear_system_null_space(ro, co, va, b, krylov=1, preconditioner=6, tolerance=1e-10)
    assert repc["status"] == 0
    out.update(cg_x=xc, cg_iterations=repc["iterations"])
    np.savez_compressed(HERE / f"neumann_tet{n}.npz", **out)


def capture(n: int):
    z = np.load(HERE / f"pressure_tet{n}.npz")
    b = z["b"]
    ref.write_capture(HERE / f"pressure_tet{n}.cfdxlin", z["row_offsets"], z["columns"], z["values"], b,
                      np.zeros_like(b), problem=1, null_space=0, scaling=0, max_iterations=1000, tolerance=1e-8)


def poisson(n: int):
    m, bc, src = cases.poisson_case(n)
    ro, co, va, rhs, _ = ref.assemble_diffusion(m, bc, 1.0, src)
    np.savez_compressed(HERE / f"poisson_hex{n}.npz", n=n, row_offsets=ro, columns=co, values=va, rhs=rhs)


if __name__ == "__main__":
    pressure(4)
    capture(4)
    poisson(6)
    neumann(5)
    for p in sorted(HERE.glob("*.npz")) + sorted(HERE.glob("*.cfdxlin")):
        print(p.name, p.stat().st_size)
