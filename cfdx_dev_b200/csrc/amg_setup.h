// amg_setup.h -- host construction of the classical Ruge-Stueben hierarchy.
//
// Restates the reference's native Boomer-style AMG setup
// (core/linalg/amg_preconditioner.h:76-243 setup, :1401-1421 build_diagonal,
// :1466-1509 build_strength_graph, :1511-1885 build_cf_interpolation,
// :1322-1399 smoother damping certificate; core/linalg/galerkin_csr_product.h
// symbolic/numeric/numeric_into_existing) with identical floating-point
// operation order, so the C/F splitting, aggregates, prolongation weights and
// Galerkin coarse operators are bit-identical to the reference's.  The work
// is reorganised for speed only where the result cannot change: the RS second
// pass resumes after each promotion instead of rescanning from row 0, and all
// per-row work (strength rows, interpolation rows, Galerkin rows) runs on
// host threads, each row still computed in the reference's order.
#pragma once
#include <functional>
#include <cstdint>
#include <memory>
#include <type_traits>
#include <utility>
#include <string>
#include <vector>

namespace cfdxg {

// CSR with the reference's 32-bit index type (core/linalg/sparse_matrix.h:30).
// Allocator whose resize() leaves new elements default-initialised (for
// arithmetic types: unwritten), so that a large level filled by a copy right
// after is touched once, not zero-filled first.
template <class T>
struct DefaultInitAllocator : std::allocator<T> {
    template <class U>
    struct rebind { using other = DefaultInitAllocator<U>; };
    DefaultInitAllocator() = default;
    template <class U>
    DefaultInitAllocator(const DefaultInitAllocator<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... Args>
    void construct(U* p, Args&&... args) {
        ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
    }
};
template <class T>
using HostVec = std::vector<T, DefaultInitAllocator<T>>;

struct HostCsr {
    int64_t n = 0;
    HostVec<uint32_t> ro;   // n + 1
    HostVec<uint32_t> co;   // nnz, strictly increasing per row
    HostVec<double> va;     // nnz
    int64_t nnz() const { return static_cast<int64_t>(co.size()); }
};

// Symbolic Galerkin plan (galerkin_csr_product.h:33-138), kept for the
// numeric-only refresh of update_values.
struct GalerkinPlan {
    int64_t n_fine = 0, n_coarse = 0;
    std::vector<uint32_t> t_off, t_row, t_pos;   // P^T adjacency in stable order
    std::vector<uint32_t> ap_off, ap_col;        // symbolic A*P
    std::vector<uint32_t> c_off, c_col;          // symbolic P^T (A P), before pruning
};

struct AmgLevel {
    HostCsr A;
    std::vector<double> inv_diag;
    // Prolongation P (fine rows x coarse columns), entries in the reference's
    // per-row order (sorted by coarse index), and the first-level "aggregate"
    // diagnostic (strongest interpolation column of each fine row).
    std::vector<uint32_t> p_off, p_col;
    std::vector<double> p_val;
    std::vector<uint32_t> aggregate;
    GalerkinPlan plan;
};

struct AmgOptions {
    double omega = 0.7;
    int pre = 6;
    int post = 6;
    int coarse_pre = -1;    // sweeps on levels >= 1 (-1: the V-cycle precision's default)
    int coarse_post = -1;
    double strength_threshold = 0.25;
    int max_levels = 25;
    bool require_smoother_certificate = false;
    bool constant_null_space = false;   // the finest operator must have the constant null space
};

struct AmgHierarchy {
    std::vector<AmgLevel> levels;
    double omega = 0.7;
    AmgOptions options;
    std::string error;
};

// The Galerkin product P^T A P of one setup level computed elsewhere (on the
// device): (level index, A, the level's prolongation in p_off/p_col/p_val,
// coarse size, out: the pruned coarse operator).  The product must be the one
// galerkin_symbolic + galerkin_numeric give, bit for bit; the level's host
// plan then stays empty.
using GalerkinHook = std::function<bool(int, const HostCsr&, const AmgLevel&, int64_t, HostCsr&)>;

// Full setup.  Returns false (and leaves `out` untouched) on failure, with the
// reason in `error`.
bool amg_setup(const HostCsr& A, const AmgOptions& options, AmgHierarchy& out, std::string& error,
               const GalerkinHook* galerkin = nullptr);

// Numeric refresh on an unchanged fine pattern (amg_preconditioner.h:245-314).
// Transactional: on failure the hierarchy is unchanged.
bool amg_update_values(AmgHierarchy& h, const HostCsr& A, std::string& error);

// Helpers shared with the device upload.
bool build_inverse_diagonal(const HostCsr& A, std::vector<double>& inv_diag);
bool has_constant_null_space(const HostCsr& A);
int host_threads();

}  // namespace cfdxg
