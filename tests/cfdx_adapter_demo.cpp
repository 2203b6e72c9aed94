// cfdx_adapter_demo.cpp -- runs the CFDX-side adapters (include/cfdxg_cfdx.hpp)
// on CFDX types: a GpuNativeAMGPreconditioner and solve_linear_system_gpu on a
// 2x2 CFDX SparseMatrix, and the apps/poisson driver shim
// solve_poisson_dirichlet_gpu on a one-cell CFDX Mesh with phi = 1 on every
// face.  Prints "no device" when no CUDA device is present, else
// "solved <status> x0 x1 phi"; exits 0 when both solves converged and the
// Poisson solution is 1.
//
// TEST PROGRAM: built by `make -C oracle adapter` against the reference's
// headers and its hypre_amg object (oracle/_ref), linked with libcfdxg.so;
// tests/test_cfdx_adapter.py runs it.
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
