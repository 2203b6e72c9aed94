"""The CFDX-side adapters (include/cfdxg_cfdx.hpp) compile against the
reference's own headers, link against libcfdxg.so with the reference's
native-AMG object, and run: a GpuNativeAMGPreconditioner and
solve_linear_system_gpu on a CFDX SparseMatrix, and the apps/poisson driver
shim on a one-cell CFDX Mesh (tests/cfdx_adapter_demo.cpp).

* CPU: the program compiles and links against the reference's headers (needs
  the reference source tree and oracle/_ref); without a device it stops after
  the context creation fails and prints "no device".
* GPU: the same program, prebuilt by `make -C oracle adapter` into
  oracle/_ref/cfdx_adapter_demo (it travels with oracle/_ref), must solve both
  systems through the adapters and print "solved 0"."""
import os
import subprocess

import pytest

from tests.conftest import REF_SRC, ROOT

OBJ = ROOT / "oracle" / "_ref" / "obj" / "core_linalg" / "hypre_amg.o"
DEMO_SRC = ROOT / "tests" / "cfdx_adapter_demo.cpp"
DEMO_EXE = ROOT / "oracle" / "_ref" / "cfdx_adapter_demo"


@pytest.mark.skipif(not (REF_SRC / "src").exists() or not OBJ.exists(), reason="needs the reference tree and build")
def test_adapters_compile_link_and_run(tmp_path):
    exe = tmp_path / "adapter"
    lib_dir = ROOT / "cfdx_dev_b200" / "_lib"
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-std=c++17", "-w", "-DCFDX_HAS_MPI=0", "-DCFDX_HAS_HDF5=0", f"-I{ROOT / 'include'}",
           f"-I{REF_SRC / 'src'}", str(DEMO_SRC), str(OBJ), f"-L{lib_dir}", "-lcfdxg", f"-Wl,-rpath,{lib_dir}",
           "-Wl,--push-state,--no-as-needed", "-l:libstdc++.so.6", "-Wl,--pop-state", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith(("no device", "solved 0"))


@pytest.mark.gpu
def test_adapters_solve_on_the_gpu():
    if not DEMO_EXE.exists():
        pytest.skip("oracle/_ref/cfdx_adapter_demo not built (make -C oracle adapter, needs the reference tree)")
    out = subprocess.run([str(DEMO_EXE)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("solved 0"), out.stdout
