"""Run the reference's own AMG setup on a Kuhn-tet pressure-correction system
and store what the CPU reference legs need to rebuild its hierarchy quickly.

TEST INFRASTRUCTURE ONLY.  Usage (needs oracle/_ref, i.e. the reference build):

    python -m oracle.reference_hierarchy 64      # hours at 64^3 on one core

Steps, all in the reference's own code (oracle/_ref): geometry
(build_fv_geometry), the pressure-corrector assembly, and
MatrixFreeVcyclePreconditioner::setup with the Balanced NativeAMG parameters
(core/linalg/hypre_amg.cpp:172-219) -- the setup takes about O(n^2.2) time
because its Ruge-Stueben second pass restarts after every promotion
(core/linalg/amg_preconditioner.h:1613-1660).  Then one GMRES(30) solve to
1e-8 on that hierarchy and the corrected face fluxes
(make_rhie_chow_mass_flux) of its solution.

Writes
* tests/golden/tet{n}_hierarchy.json (committed): the system's and every
  level's SHA-256 per array, level sizes, the damping, the reference's setup
  seconds, its solve report and the SHA-256 of its solution and fluxes;
* oracle/_ref/tet{n}_transfers.npz (not committed; travels with oracle/_ref):
  each level's prolongation and aggregates, from which
  ref.AmgFromTransfers rebuilds the identical hierarchy with the reference's
  own Galerkin products in seconds instead of hours.
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from oracle import cases as oc  # noqa: E402
from oracle import ref  # noqa: E402


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def transfers_path(n: int) -> Path:
    return ROOT / "oracle" / "_ref" / f"tet{n}_transfers.npz"


def golden_path(n: int) -> Path:
    return ROOT / "tests" / "golden" / f"tet{n}_hierarchy.json"


def reference_system(n: int):
    """(mesh, fields, assembled system) of the n^3 x 6 Kuhn-tet pressure correction, reference code only."""
    m = oc.simple_mesh(n)
    g = ref.geometry(m)
    fields = oc.simple_fields(m, g["cell_centres"])
    U, rAU, aP, p, fixed, value = fields
    r = ref.simple_assemble(m, U, rAU, p, 1.0, fixed, value)
    return m, fields, r


def system_sha256(r) -> dict:
    return {k: sha(np.asarray(r[k], np.int64 if k in ("row_offsets", "columns") else np.float64))
            for k in ("row_offsets", "columns", "values", "b")}


def load_transfers(n: int):
    """-> (transfers dict, level row counts, golden dict) or None where either file is missing."""
    t, g = transfers_path(n), golden_path(n)
    if not (t.exists() and g.exists()):
        return None
    gold = json.loads(g.read_text())
    z = np.load(t)
    return {k: z[k] for k in z.files}, [lv["n_rows"] for lv in gold["levels"]], gold


def main(n: int) -> None:
    t0 = time.time()
    m, (U, rAU, aP, p, fixed, value), r = reference_system(n)
    t = time.time()
    R = ref.Amg(r["row_offsets"], r["columns"], r["values"])
    setup_s = time.time() - t
    levels = ref.hierarchy_sha256(R)
    transfers = {}
    for l in range(R.num_levels()):
        lv = R.level(l)
        if lv["p_offsets"] is not None:
            levels[l]["p_nnz"] = int(lv["p_columns"].size)
            for k in ("p_offsets", "p_columns", "p_values", "aggregate"):
                transfers[f"{k}_{l}"] = lv[k]
    transfers_path(n).parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(transfers_path(n), **transfers)
    x, rep = R.solve_gmres(r["b"], restart=30, max_iterations=1000, tolerance=1e-8)
    flux = ref.rhie_chow_flux(m, U, rAU, x, 1.0, fixed, value)
    info = {"cells": int(m.n_cells), "setup_seconds": setup_s, "omega": R.omega, "omega_hex": float(R.omega).hex(),
            "system": system_sha256(r), "levels": levels,
            "solve": {k: (float(v) if isinstance(v, float) else int(v)) for k, v in rep.items()},
            "solution_sha256": sha(x), "flux_sha256": sha(flux), "total_seconds": time.time() - t0}
    golden_path(n).write_text(json.dumps(info, indent=1) + "\n")


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 64)
