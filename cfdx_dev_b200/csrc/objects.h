// objects.h -- internal definitions of the opaque C-ABI handles.
#pragma once
#include <cuda_fp16.h>
#include <memory>
#include <string>
#include <vector>

#include "amg_setup.h"
#include "device.cuh"

namespace cfdxg {

// Pressure-correction / diffusion CSR pattern of a mesh: rows sorted, one
// entry per (cell, neighbour) plus the diagonal; per (cell, local face) the
// CSR slot of the neighbour column (-1 on boundary faces).
struct MeshPattern {
    bool built = false;
    int64_t nnz = 0;
    std::vector<uint32_t> ro, co;
    DevBuf<int> d_ro, d_co, d_slot, d_diag;
};

template <class T>
struct DevLevel {
    int n = 0, nnz = 0, nc = 0;
    DevBuf<int> ro, co;
    // Narrow columns: when every |column - row| of the level fits in 16 bits,
    // the columns are stored as int16 offsets from the row (co16) and co is
    // left empty -- 2 bytes instead of 4 per nonzero on the HBM-bound sweeps.
    DevBuf<int16_t> co16;
    bool narrow = false;
    // Half values (FP32 cycle, option half_values): each row of A stored as
    // FP16 fractions of its largest magnitude (vh) times that magnitude
    // (rscale); va is then left empty.
    DevBuf<__half> vh;
    DevBuf<T> rscale;
    bool half = false;
    // Sparsified smoothing operator (FP32 cycle, coarse_drop_tolerance): ro,
    // co and the values hold the Galerkin operator's diagonal and its kept
    // off-diagonal entries (one bit per Galerkin entry in keep), the dropped
    // entries added to the diagonal; inv_diag is that diagonal's inverse.
    DevBuf<uint32_t> keep;
    bool sparsified = false;
    DevBuf<T> va, inv_diag;
    DevBuf<int> p_off, p_col, r_off, r_row;
    DevBuf<T> p_val, r_val;
    DevBuf<T> r, x, x2, res;
    T* xout = nullptr;   // where the level's result lives after enqueue
    int tpr = 1;         // threads cooperating on one row of A (1 = reference order)
    int tpr_r = 1;       // threads cooperating on one row of P^T
    int tpr_p = 1;       // threads cooperating on one row of P (prolongation)
};

template <class T>
struct DevHierarchy {
    std::vector<DevLevel<T>> L;
    int used = 0;              // levels visited by the cycle
    T omega = T(0.7);
    int pre = 6, post = 6;
    int coarse_pre = 6, coarse_post = 6;   // sweeps on levels >= 1
    int coarse_mode = 0;       // 0: 24 Jacobi sweeps, 1: reference dense LU (n <= 16), 2: dense inverse
    DevBuf<float> dense;       // mode 2: the n*n inverse (row-major), formed in FP64, stored FP32
    DevBuf<double> dense64;    // mode 2 with dense_fp64: the same inverse stored FP64
    bool dense_fp64 = false;
    // the dense inverse's LU solver handle and work arrays, kept for refreshes
    std::shared_ptr<void> solver;
    DevBuf<double> lu_a, lu_x, lu_work;
    DevBuf<int> lu_ipiv, lu_info;
    bool dense_cholesky = false;   // the last inverse came from a Cholesky factor (symmetric level)
    // constant null space: the cycle's mean removals (in index order with
    // reference_order) and the bordered coarsest solve
    bool null_space = false;
    bool ns_in_order = false;
    DevBuf<double> ns_partials;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t graph_kernels = 0;
    double graph_bytes = 0.0;   // algorithmic bytes of one replay
    int* status = nullptr;
    ~DevHierarchy() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};


}  // namespace cfdxg

struct cfdxg_mesh {
    int64_t n_points = 0, n_faces = 0, n_cells = 0, n_internal = 0;
    int32_t n_patches = 0;
    int max_cell_faces = 0;
    cfdxg::DevBuf<double> px, py, pz;
    cfdxg::DevBuf<int> face_off, face_vert, owner, neigh, cell_off, cell_face, cell_sorted,
        patch_of_face, patch_type;
    // geometry (SoA)
    bool geometry_ready = false;
    cfdxg::DevBuf<double> face_centre, face_sf, cell_centre, cell_volume;
    cfdxg::MeshPattern pattern;
    // face-loop tables, built with the geometry (assembly.cu): per cell-face
    // slot (cell-face order) the face id, with bit 31 set where the cell is
    // the face's neighbour, and the other cell (-1 on the boundary); the Gauss
    // gradient's interpolation weight of the cell's side; per face the
    // corrector's geometric terms d, e, Sf . e (5 x n_faces, SoA)
    cfdxg::DevBuf<int2> slot_rec;
    cfdxg::DevBuf<double> slot_w, face_geo;
    // per-call boundary table and gradient scratch, kept so the face-loop entry
    // points neither allocate nor free device memory after their first call
    cfdxg::DevBuf<int> bc_fixed;
    cfdxg::DevBuf<double> bc_value, grad_scratch;
    // host copies needed by the pattern build
    std::vector<int64_t> h_owner, h_neigh, h_cell_off, h_cell_face;
    std::vector<int32_t> h_patch_types;
};

struct cfdxg_matrix {
    int64_t n = 0, nnz = 0;
    cfdxg::DevBuf<int> ro, co;
    cfdxg::DevBuf<double> va;
    // host mirror of the CSR (pattern always valid; values refreshed on demand)
    cfdxg::HostCsr host;
    bool host_values_valid = false;
    const cfdxg_mesh* mesh = nullptr;   // set when assembled from a mesh pattern
};

namespace cfdxg {
// FP64 device copy of the hierarchy's numeric state and of the symbolic
// Galerkin plans, for the numeric refresh on the GPU (galerkin.cu).
struct DevRefreshLevel {
    int n = 0, n_coarse = 0;
    int64_t nnz = 0;
    DevBuf<int> ro, co;                       // this level's CSR pattern
    DevBuf<double> va, inv_diag;              // this level's values (FP64)
    DevBuf<int> p_off, p_col;                 // P to the next level
    DevBuf<double> p_val;
    DevBuf<int> ap_off, ap_col, c_off, c_col, t_off, t_row, t_pos, keep_pos;
    DevBuf<double> ap, cv;
};
struct DevRefresh {
    std::vector<DevRefreshLevel> L;
    DevBuf<double> bounds;                    // per-level normalised Gershgorin bound
    DevBuf<double> sqrt_diag;                 // scratch: sqrt(1 / inv_diag) of one level
};
}  // namespace cfdxg

struct cfdxg_amg {
    cfdxg_amg_options opts{};
    cfdxg::AmgHierarchy host;
    bool ready = false;
    std::string error;
    double setup_seconds = 0.0;
    std::unique_ptr<cfdxg::DevHierarchy<double>> d64;
    std::unique_ptr<cfdxg::DevHierarchy<float>> d32;
    int64_t applications = 0;
    // numeric refresh on the device; the host mirror of the level values is
    // then stale until amg_sync_host_values
    std::unique_ptr<cfdxg::DevRefresh> refresh;
    bool host_values_stale = false;
    cfdxg_context* ctx = nullptr;   // context the device hierarchy lives on
};

namespace cfdxg {

// The Galerkin products of a first setup on the device (galerkin.cu), as the
// setup's GalerkinHook: symbolic graphs by expand, sort, unique, numeric
// products and pruning by the refresh kernels -- the host restatement's
// coarse operators bit for bit.  It keeps every level's plan; take() hands
// them over as the hierarchy's refresh plan.
class DeviceGalerkin {
public:
    DeviceGalerkin(cfdxg_context* ctx, const cfdxg_matrix* A);
    ~DeviceGalerkin();
    DeviceGalerkin(const DeviceGalerkin&) = delete;
    DeviceGalerkin& operator=(const DeviceGalerkin&) = delete;
    bool operator()(int level, const HostCsr& A, const AmgLevel& P, int64_t coarse_n, HostCsr& coarse);
    std::unique_ptr<DevRefresh> take(int levels);

private:
    cfdxg_context* ctx_;
    const cfdxg_matrix* A_;
    std::unique_ptr<DevRefresh> R_;
    // grow-only scratch shared by the levels: expansion keys and their sorted
    // and unique copies, per-entry lengths and offsets, integer flags, CUB
    // temporaries
    DevBuf<unsigned long long> keys_, sorted_, uniq_;
    DevBuf<int64_t> len_, eoff_, count_;
    DevBuf<int> ints_, ints2_, counts_;
    DevBuf<unsigned char> temp_;
    // two pinned chunks staging the coarse operators' downloads
    static constexpr std::size_t kStageBytes = std::size_t{32} << 20;
    void* stage_[2] = {nullptr, nullptr};
    cudaEvent_t staged_[2] = {nullptr, nullptr};
    void download(const void* src, void* dst, std::size_t bytes);
};

// numeric refresh of the hierarchy on the device (galerkin.cu): the
// reference's update_values (amg_preconditioner.h:245-314) with the Galerkin
// products, pruning check, inverse diagonals and damping computed in its
// order on the GPU; false (hierarchy unchanged) when the pruned pattern or a
// diagonal no longer qualifies
bool amg_refresh_device(cfdxg_context* ctx, cfdxg_amg* amg, const cfdxg_matrix* A, std::string& error);
// copies refreshed level values and inverse diagonals back to the host mirror
void amg_sync_host_values(cfdxg_context* ctx, cfdxg_amg* amg);
template <class T>
void set_hierarchy_values_device(cfdxg_context* ctx, DevHierarchy<T>& d, const DevRefresh& R, double omega);

// matrix helpers (matrix.cu)
void matrix_sync_host_values(cfdxg_context* ctx, cfdxg_matrix* A);
void spmv_fp64(cfdxg_context* ctx, const cfdxg_matrix* A, const double* x, double* y);

// hierarchy (vcycle.cu)
// Device layout choices for one hierarchy.
struct UploadOptions {
    int coarse_dense_limit = 0;   // FP32: dense FP64 inverse at the first level with <= this many rows
    bool reference_order = false; // one thread per row everywhere (the reference's sums)
    bool narrow_columns = true;   // int16 column offsets on one-thread-per-row levels
    bool half_values = false;     // FP32: FP16 row-scaled matrix values
    bool dense_fp64 = false;      // FP32: the dense coarse inverse stored (and applied) in FP64
    bool constant_null_space = false;   // the cycle of a pure-Neumann operator (mean removals)
    double coarse_drop_tolerance = 0.0; // FP32: sparsified smoothing operators between fine and coarsest
};

// From the host hierarchy, or, with R (the device levels a device-Galerkin
// setup left), from the device copy -- the same layout and values.
template <class T>
std::unique_ptr<DevHierarchy<T>> upload_hierarchy(cfdxg_context* ctx, const AmgHierarchy& h,
                                                  const UploadOptions& opt, const DevRefresh* R = nullptr);
// z = V-cycle(r); r, z are FP64 device vectors.
template <class T>
void vcycle_apply(cfdxg_context* ctx, DevHierarchy<T>& d, const double* r, double* z);
template <class T>
void destroy_hierarchy(DevHierarchy<T>* d);

// z = one V-cycle of a device-ready hierarchy applied to r (device vectors)
void amg_apply_device(cfdxg_context* ctx, cfdxg_amg* amg, const double* r, double* z);

// status word helpers (context.cu)
void clear_status(cfdxg_context* ctx);
int read_status(cfdxg_context* ctx);   // synchronises
constexpr int kStatusNonFinite = 1;
constexpr int kStatusGeometry = 2;

}  // namespace cfdxg
