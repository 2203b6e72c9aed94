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


def prism_case(nx: int, ny: int, nz: int, jitter: float = 0.1, seed: int = SEED_MESH) -> "cg.HostMesh":
    """Triangular prisms (five faces each): every cell of an nx x ny x nz
    lattice split along its (x0, y0)-(x1, y1) diagonal plane into prism A
    (x0y0, x1y0, x1y1) and prism B (x0y0, x1y1, x0y1), cells 2h and 2h + 1 of
    hexahedron h.  Interior points jittered by +-jitter of the spacing.
    Patches: 0 x = 0, 1 x = 1, 2 the y walls, 3 the z walls (type 0).  Face
    orientation is left to the geometry build (owner = lower cell)."""
    rng = np.random.default_rng(seed)
    X, Y, Z = np.meshgrid(np.linspace(0, 1, nx + 1), np.linspace(0, 1, ny + 1), np.linspace(0, 1, nz + 1),
                          indexing="ij")
    pts = np.stack([X, Y, Z], -1)
    inner = (slice(1, nx), slice(1, ny), slice(1, nz))
    h = np.array([1.0 / nx, 1.0 / ny, 1.0 / nz])
    pts[inner] += jitter * h * rng.uniform(-1, 1, pts[inner].shape)

    def pid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    def cell(i, j, k, half):
        return 2 * ((i * ny + j) * nz + k) + half

    faces, owners, neighs, patches = [], [], [], []
    cell_faces = [[] for _ in range(2 * nx * ny * nz)]

    def add(verts, a, b, patch=-1):
        f = len(faces)
        faces.append(verts)
        o, n = (a, b) if b < 0 or a < b else (b, a)
        owners.append(o)
        neighs.append(n)
        patches.append(patch)
        cell_faces[o].append(f)
        if n >= 0:
            cell_faces[n].append(f)

    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                A, B = cell(i, j, k, 0), cell(i, j, k, 1)
                p00, p10, p11, p01 = pid(i, j, k), pid(i + 1, j, k), pid(i + 1, j + 1, k), pid(i, j + 1, k)
                q00, q10, q11, q01 = (pid(i, j, k + 1), pid(i + 1, j, k + 1), pid(i + 1, j + 1, k + 1),
                                      pid(i, j + 1, k + 1))
                add([p00, p11, q11, q00], A, B)                                   # diagonal plane
                # x = i + 1 face: A here, B of the next column (or the x = 1 wall)
                add([p10, p11, q11, q10], A, cell(i + 1, j, k, 1) if i + 1 < nx else -1, -1 if i + 1 < nx else 1)
                if i == 0:
                    add([p00, p01, q01, q00], B, -1, 0)
                # y = j + 1 face: B here, A of the next row (or the y wall)
                add([p01, p11, q11, q01], B, cell(i, j + 1, k, 0) if j + 1 < ny else -1, -1 if j + 1 < ny else 2)
                if j == 0:
                    add([p00, p10, q10, q00], A, -1, 2)
                # z = k + 1 triangles, or the z wall
                up = k + 1 < nz
                add([q00, q10, q11], A, cell(i, j, k + 1, 0) if up else -1, -1 if up else 3)
                add([q00, q11, q01], B, cell(i, j, k + 1, 1) if up else -1, -1 if up else 3)
                if k == 0:
                    add([p00, p10, p11], A, -1, 3)
                    add([p00, p11, p01], B, -1, 3)
    fo = np.zeros(len(faces) + 1, np.int64)
    fo[1:] = np.cumsum([len(f) for f in faces])
    co = np.zeros(len(cell_faces) + 1, np.int64)
    co[1:] = np.cumsum([len(c) for c in cell_faces])
    pts = pts.reshape(-1, 3)
    return cg.HostMesh(px=np.ascontiguousarray(pts[:, 0]), py=np.ascontiguousarray(pts[:, 1]),
                       pz=np.ascontiguousarray(pts[:, 2]), face_offsets=fo,
                       face_vertices=np.concatenate([np.asarray(f, np.int64) for f in faces]),
                       owner=np.asarray(owners, np.int64), neighbour=np.asarray(neighs, np.int64),
                       cell_offsets=co, cell_faces=np.concatenate([np.asarray(c, np.int64) for c in cell_faces]),
                       patch_of_face=np.asarray(patches, np.int32), patch_types=np.zeros(4, np.int32))
