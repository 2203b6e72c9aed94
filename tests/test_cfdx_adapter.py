"""The CFDX-side adapters (include/cfdxg_cfdx.hpp) compile against the
reference's own headers, link against libcfdxg.so with the reference's
native-AMG object, and run: a GpuNativeAMGPreconditioner and
solve_linear_system_gpu on a CFDX SparseMatrix.  Without a device the program
stops after the context creation fails; on a GPU host it solves a 2x2 system
through the adapters.  Needs the reference source tree (its headers) and the
reference build in oracle/_ref (its hypre_amg object)."""
import os
import subprocess
from pathlib import Path

import pytest

from tests.conftest import REF_SRC, ROOT

OBJ = ROOT / "oracle" / "_ref" / "obj" / "core_linalg" / "hypre_amg.o"

PROGRAM = r'''
#include "cfdxg_cfdx.hpp"
#include <cstdio>
int main() {
    cfdxg_context* ctx = nullptr;
    if (cfdxg_context_create(0, &ctx) != CFDXG_OK) { std::puts("no device"); return 0; }
    cfdx::core::SparseMatrix A(2, 2);
    A.push_back(0, 0, 2.0); A.push_back(0, 1, -1.0); A.push_back(1, 0, -1.0); A.push_back(1, 1, 3.0);
    A.finalize();
    cfdx::core::Vector b(2, 1.0), x(2, 0.0), z(2, 0.0);
    cfdxg_cfdx::GpuNativeAMGPreconditioner pc(ctx);
    if (!pc.setup(A) || !pc.apply(b, z)) return 2;
    const auto rep = cfdxg_cfdx::solve_linear_system_gpu(ctx, A, b, x, cfdx::core::LinearProblemKind::PressurePoisson);
    cfdxg_context_destroy(ctx);
    std::printf("solved %d %.17g %.17g\n", static_cast<int>(rep.result.status), x(0), x(1));
    return rep.result.status == cfdx::core::SolverStatus::CONVERGED ? 0 : 1;
}
'''


@pytest.mark.skipif(not (REF_SRC / "src").exists() or not OBJ.exists(), reason="needs the reference tree and build")
def test_adapters_compile_link_and_run(tmp_path):
    src = tmp_path / "adapter.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "adapter"
    lib_dir = ROOT / "cfdx_dev_b200" / "_lib"
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-std=c++17", "-w", "-DCFDX_HAS_MPI=0", "-DCFDX_HAS_HDF5=0", f"-I{ROOT / 'include'}",
           f"-I{REF_SRC / 'src'}", str(src), str(OBJ), f"-L{lib_dir}", "-lcfdxg", f"-Wl,-rpath,{lib_dir}",
           "-Wl,--push-state,--no-as-needed", "-l:libstdc++.so.6", "-Wl,--pop-state", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith(("no device", "solved 0"))
