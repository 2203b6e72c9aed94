"""Seeded synthetic inputs for the CPU reference legs, without the CUDA library.

TEST INFRASTRUCTURE ONLY.  oracle/_build/libcfdx_cases.so is the package's
own input generator (cfdx_dev_b200/csrc/cases.cpp) compiled alone with the
package's host flags, so the reference legs of bench.py can build the same
meshes and fields as tests/cases.py (bit for bit; tested) while loading only
oracle libraries.  The seeds are those of tests/cases.py.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import threading
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libcfdx_cases.so"

SEED_MESH = 20240601
SEED_HBYA = 20240602
SEED_AP = 20240603

_lib = None
_lock = threading.Lock()


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
            _lib = C.CDLL(str(LIB_PATH))
            _lib.cfdxg_case_tet.argtypes = [C.c_int64, C.c_double, C.c_uint64, C.c_void_p]
            _lib.cfdxg_case_hex.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_void_p]
            _lib.cfdxg_case_sizes.argtypes = [C.c_void_p, C.c_void_p]
            _lib.cfdxg_case_export.argtypes = [C.c_void_p] * 12
            _lib.cfdxg_case_destroy.argtypes = [C.c_void_p]
            _lib.cfdxg_field_fourier.argtypes = [C.c_int64, C.c_void_p, C.c_int32, C.c_double, C.c_uint64,
                                                 C.c_void_p]
            _lib.cfdxg_field_random.argtypes = [C.c_int64, C.c_int32, C.c_double, C.c_double, C.c_uint64,
                                                C.c_void_p]
    return _lib


@dataclass
class CaseMesh:
    px: np.ndarray
    py: np.ndarray
    pz: np.ndarray
    face_offsets: np.ndarray
    face_vertices: np.ndarray
    owner: np.ndarray
    neighbour: np.ndarray
    cell_offsets: np.ndarray
    cell_faces: np.ndarray
    patch_of_face: np.ndarray
    patch_types: np.ndarray

    @property
    def n_faces(self):
        return self.owner.size

    @property
    def n_cells(self):
        return self.cell_offsets.size - 1

    @property
    def n_patches(self):
        return self.patch_types.size


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _export(h) -> CaseMesh:
    L = lib()
    s = np.zeros(6, np.int64)
    L.cfdxg_case_sizes(h, _p(s))
    npnt, nf, nfv, nc, ncf, npat = (int(v) for v in s)
    m = CaseMesh(px=np.empty(npnt), py=np.empty(npnt), pz=np.empty(npnt),
                 face_offsets=np.empty(nf + 1, np.int64), face_vertices=np.empty(nfv, np.int64),
                 owner=np.empty(nf, np.int64), neighbour=np.empty(nf, np.int64),
                 cell_offsets=np.empty(nc + 1, np.int64), cell_faces=np.empty(ncf, np.int64),
                 patch_of_face=np.empty(nf, np.int32), patch_types=np.empty(npat, np.int32))
    L.cfdxg_case_export(h, *(_p(getattr(m, f)) for f in (
        "px", "py", "pz", "face_offsets", "face_vertices", "owner", "neighbour", "cell_offsets", "cell_faces",
        "patch_of_face", "patch_types")))
    L.cfdxg_case_destroy(h)
    return m


def tet_case(n: int, jitter: float, seed: int) -> CaseMesh:
    h = C.c_void_p()
    if lib().cfdxg_case_tet(n, jitter, seed, C.byref(h)) != 0:
        raise RuntimeError("tet case")
    return _export(h)


def simple_mesh(n: int, jitter: float = 0.15, seed_offset: int = 0) -> CaseMesh:
    return tet_case(n, jitter, SEED_MESH + seed_offset)


def simple_fields(m, centres, seed_offset: int = 0):
    """(U, rAU, aP, p, fixed, value) exactly as tests/cases.py.simple_fields."""
    centres = np.ascontiguousarray(centres, np.float64)
    n = m.n_cells
    U = np.empty(3 * n)
    if lib().cfdxg_field_fourier(n, _p(centres), 8, 0.01, SEED_HBYA + seed_offset, _p(U)) != 0:
        raise RuntimeError("fourier field")
    aP = np.empty(n)
    if lib().cfdxg_field_random(n, 0, 1.0, 100.0, SEED_AP + seed_offset, _p(aP)) != 0:
        raise RuntimeError("random field")
    rAU = np.concatenate([1.0 / aP] * 3)
    p = np.zeros(n)
    fixed = np.zeros(m.n_patches, np.int32)
    fixed[0] = 1
    value = np.zeros(m.n_patches)
    return U, rAU, aP, p, fixed, value
