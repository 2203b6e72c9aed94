// ref_common.h -- shared helpers of the reference-built oracle adapters.
//
// TEST INFRASTRUCTURE ONLY: builds reference `cfdx::core::Mesh` objects from
// flat arrays so that the reference's own functions can be called on the same
// inputs as the CUDA path.  Compiled only by oracle/Makefile.
#pragma once
#include "ref_abi.h"

#include "cfdx/core/mesh/mesh.h"
#include "cfdx/core/linalg/sparse_matrix.h"

#include <chrono>
#include <cstdint>
#include <exception>
#include <string>
#include <vector>

namespace cfdx_ref {

inline thread_local std::string g_error;

inline void set_error(const std::exception& e) { g_error = e.what(); }

inline double now_seconds() {
    using clock = std::chrono::steady_clock;
    return std::chrono::duration<double>(clock::now().time_since_epoch()).count();
}

// Mesh built from flat arrays exactly as the reference fixtures build theirs:
// push_face / push_cell in array order, owner/neighbour set per face, one
// boundary patch per distinct patch id (names "p0", "p1", ...).
inline cfdx::core::Mesh make_mesh(const ref_mesh_t& a) {
    using namespace cfdx::core;
    Mesh m;
    m.points().resize(static_cast<std::size_t>(a.n_points));
    for (int64_t i = 0; i < a.n_points; ++i)
        m.points().set(static_cast<std::size_t>(i), a.px[i], a.py[i], a.pz[i]);
    std::vector<FaceIndex> fv;
    for (int64_t f = 0; f < a.n_faces; ++f) {
        fv.assign(a.face_vertices + a.face_offsets[f], a.face_vertices + a.face_offsets[f + 1]);
        m.faces().push_face(fv);
    }
    std::vector<FaceIndex> cf;
    for (int64_t c = 0; c < a.n_cells; ++c) {
        cf.assign(a.cell_faces + a.cell_offsets[c], a.cell_faces + a.cell_offsets[c + 1]);
        m.cells().push_cell(cf);
    }
    m.ownership().resize(static_cast<std::size_t>(a.n_faces));
    for (int64_t f = 0; f < a.n_faces; ++f) {
        m.ownership().set_owner(static_cast<std::size_t>(f), static_cast<CellIndex>(a.owner[f]));
        m.ownership().set_neighbour(static_cast<std::size_t>(f), a.neighbour[f] < 0 ? FaceOwnership::BOUNDARY : a.neighbour[f]);
    }
    std::vector<Patch> patches(static_cast<std::size_t>(a.n_patches));
    for (int32_t p = 0; p < a.n_patches; ++p) {
        patches[p].name = "p" + std::to_string(p);
        patches[p].type = static_cast<PatchType>(a.patch_types[p]);
    }
    for (int64_t f = 0; f < a.n_faces; ++f) {
        const int32_t p = a.patch_of_face ? a.patch_of_face[f] : -1;
        if (p >= 0 && p < a.n_patches) patches[p].face_ids.push_back(static_cast<FaceIndex>(f));
    }
    for (auto& p : patches) m.boundary().add_patch(p);
    return m;
}

inline cfdx::core::SparseMatrix make_csr(int64_t n, const int64_t* ro, const int64_t* co,
                                         const double* va) {
    using cfdx::core::SparseMatrix;
    std::vector<SparseMatrix::Index> off(static_cast<std::size_t>(n) + 1), col;
    std::vector<double> val;
    for (int64_t i = 0; i <= n; ++i) off[i] = static_cast<SparseMatrix::Index>(ro[i]);
    col.resize(static_cast<std::size_t>(ro[n]));
    val.resize(static_cast<std::size_t>(ro[n]));
    for (int64_t k = 0; k < ro[n]; ++k) {
        col[k] = static_cast<SparseMatrix::Index>(co[k]);
        val[k] = va[k];
    }
    return SparseMatrix::from_sorted_csr(static_cast<std::size_t>(n), static_cast<std::size_t>(n),
                                         std::move(off), std::move(col), std::move(val));
}

inline int64_t export_csr(const cfdx::core::SparseMatrix& A, int64_t* ro, int64_t* co, double* va) {
    const std::size_t n = A.n_rows();
    for (std::size_t i = 0; i <= n; ++i) ro[i] = A.row_offsets_data()[i];
    for (std::size_t k = 0; k < A.nnz(); ++k) {
        co[k] = A.columns_data()[k];
        va[k] = A.values_data()[k];
    }
    return static_cast<int64_t>(A.nnz());
}

}  // namespace cfdx_ref
