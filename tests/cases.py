"""Seeded synthetic inputs shared by the tests and the benchmark.

Each configuration follows the benchmark definitions (hex Poisson on the unit
cube; jittered Kuhn tets with log-uniform a_P and a divergence-free Fourier
HbyA; p = 0 fixed on the x = 0 patch).  Seeds are fixed so both the CUDA path
and the reference oracle see identical arrays.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

import cfdx_dev_b200 as cg

ROOT = Path(__file__).resolve().parents[1]

SEED_MESH = 20240601
SEED_HBYA = 20240602
SEED_AP = 20240603
SEED_SOURCE = 20240604


def poisson_case(n: int):
    """Config-1 style: hex n^3, Dirichlet p=0 on x=0 (west), S ~ U[-1,1] (seeded)."""
    m = cg.hex_case(n)
    bc = np.full(m.n_faces, np.nan)
    bc[m.patch_of_face == 0] = 0.0
    src = cg.random_field(m.n_cells, "uniform", -1.0, 1.0, SEED_SOURCE)
    return m, bc, src


def simple_mesh(n: int, jitter: float = 0.15, seed_offset: int = 0):
    """Config-2 style mesh: Kuhn tets of an n^3 lattice, interior vertices jittered."""
    return cg.tet_case(n, jitter, SEED_MESH + seed_offset)


def simple_fields(m, centres, seed_offset: int = 0):
    """HbyA (8 Fourier modes + U[-0.01,0.01]), rAU = 1/a_P with a_P log-uniform on [1,100],
    p = 0, fixed p = 0 on patch 0 (x = 0).  Returns (U, rAU, aP, p, fixed, value)."""
    U = cg.fourier_field(centres, 8, 0.01, SEED_HBYA + seed_offset)
    aP = cg.random_field(m.n_cells, "loguniform", 1.0, 100.0, SEED_AP + seed_offset)
    rAU = np.concatenate([1.0 / aP] * 3)
    p = np.zeros(m.n_cells)
    fixed = np.zeros(m.n_patches, np.int32)
    fixed[0] = 1
    value = np.zeros(m.n_patches)
    return U, rAU, aP, p, fixed, value
