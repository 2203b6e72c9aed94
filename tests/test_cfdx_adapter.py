"""The CFDX-side adapters (include/cfdxg_cfdx.hpp) compile against the
reference's own headers, link against libcfdxg.so with the reference's
native-AMG object, and run: a GpuNativeAMGPreconditioner and
solve_linear_system_gpu on a CFDX SparseMatrix, and the apps/poisson driver
shim on a one-cell CFDX Mesh.  Without a device the program stops after the
context creation fails; on a GPU host it solves both through the adapters.  Needs the reference source tree (its headers) and the
reference build in oracle/_ref (its hypre_amg object)."""
import os
import subprocess
from pathlib import Path

import pytest

from tests.conftest import REF_SRC, ROOT

OBJ = ROOT / "oracle" / "_ref" / "obj" / "core_linalg" / "hypre_amg.o"

PROGRAM = r'''
#include "cfdxg_cfdx.hpp"
#include <cmath>
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
    // the apps/poisson driver on one unit hex cell with phi = 1 on every face
    cfdx::core::Mesh m;
    m.points().resize(8);
    const double p[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};
    for (int q = 0; q < 8; ++q) m.points().set(q, p[q][0], p[q][1], p[q][2]);
    const std::vector<std::vector<cfdx::core::FaceIndex>> faces = {
        {0,4,7,3}, {1,2,6,5}, {0,1,5,4}, {3,7,6,2}, {0,3,2,1}, {4,5,6,7}};
    for (const auto& f : faces) m.faces().push_face(f);
    m.cells().push_cell({0, 1, 2, 3, 4, 5});
    m.ownership().resize(6);
    for (int f = 0; f < 6; ++f) {
        m.ownership().set_owner(f, 0);
        m.ownership().set_neighbour(f, cfdx::core::FaceOwnership::BOUNDARY);
    }
    cfdx::core::Patch walls;
    walls.name = "walls";
    walls.type = cfdx::core::PatchType::WALL;
    walls.face_ids = {0, 1, 2, 3, 4, 5};
    m.boundary().add_patch(walls);
    auto bc = cfdx::core::PoissonBoundaryCondition::dirichlet(6);
    for (int f = 0; f < 6; ++f) bc.face_values[f] = 1.0;
    const auto poisson = cfdxg_cfdx::solve_poisson_dirichlet_gpu(ctx, m, bc, std::vector<double>(1, 0.0));
    cfdxg_context_destroy(ctx);
    std::printf("solved %d %.17g %.17g %.17g\n", static_cast<int>(rep.result.status), x(0), x(1),
                poisson.solution(0));
    return rep.result.status == cfdx::core::SolverStatus::CONVERGED &&
           poisson.linear_result.status == cfdx::core::SolverStatus::CONVERGED &&
           std::abs(poisson.solution(0) - 1.0) < 1e-12 ? 0 : 1;
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
