"""The C ABI library loads and exports every entry point include/cfdxg.h declares."""
import pytest
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "cfdxg.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cfdxg_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    from cfdx_dev_b200 import _native
    lib = _native.load()
    syms = declared_symbols()
    assert len(syms) > 40
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # and every declared entry point has a ctypes prototype in the binding
    assert not [s for s in syms if s not in _native.PROTOTYPES]


def test_build_targets_sm100a_only():
    from cfdx_dev_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_host_only_calls_need_no_device():
    import cfdx_dev_b200 as cg
    m = cg.hex_case(3)
    assert m.n_cells == 27 and m.n_faces == 108
    amg = cg.NativeBoomerAMGPreconditioner(None)
    assert amg.name() == "NativeBoomerStyleAMG"


def test_amg_option_defaults():
    """cfdxg_amg_options_default: the reference's smoother and coarsening
    parameters, and the FP32 cycle's own defaults (host-only, no device)."""
    import ctypes as C
    from cfdx_dev_b200 import _native as N
    o = N.AmgOptions()
    assert N.load().cfdxg_amg_options_default(C.byref(o)) == 0
    assert (o.omega, o.strength_threshold, o.max_levels) == (0.7, 0.25, 25)
    assert (o.pre_sweeps, o.post_sweeps, o.coarse_pre_sweeps, o.coarse_post_sweeps) == (-1, -1, -1, -1)
    assert (o.coarse_dense_limit, o.narrow_columns, o.half_values, o.dense_fp64) == (6000, 1, 1, 0)
    assert (o.reference_order, o.constant_null_space) == (0, 0)
    assert o.coarse_drop_tolerance == 0.02


def test_amg_options_are_validated():
    """cfdxg_amg_create refuses out-of-range options (host-only, no device)."""
    import cfdx_dev_b200 as cg
    for bad in (dict(omega=0.0), dict(omega=2.0), dict(strength_threshold=1.5), dict(max_levels=0),
                dict(coarse_drop_tolerance=-0.1), dict(coarse_drop_tolerance=1.0),
                dict(coarse_drop_tolerance=float("nan"))):
        with pytest.raises(cg.CfdxgError):
            cg.NativeBoomerAMGPreconditioner(None, **bad)
    cg.NativeBoomerAMGPreconditioner(None, precision="fp32_vcycle", coarse_drop_tolerance=0.0)
    cg.NativeBoomerAMGPreconditioner(None, precision="fp32_vcycle", coarse_drop_tolerance=0.5)


def test_header_is_plain_c_and_links_from_c(tmp_path):
    """include/cfdxg.h is a C header (C99, no warnings under -Wall -Wextra
    -pedantic) and a C program links against libcfdxg.so and calls a host-only
    entry point."""
    import subprocess
    from tests.conftest import ROOT
    src = tmp_path / "abi.c"
    src.write_text('#include "cfdxg.h"\n'
                   "int main(void) { cfdxg_request r; cfdxg_request_default(&r);\n"
                   "  return r.krylov == CFDXG_KRYLOV_GMRES && r.problem == CFDXG_PROBLEM_PRESSURE_POISSON ? 0 : 1; }\n")
    lib_dir = ROOT / "cfdx_dev_b200" / "_lib"
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", f"-I{ROOT / 'include'}", str(src),
                    f"-L{lib_dir}", "-lcfdxg", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    assert subprocess.run([str(exe)]).returncode == 0
