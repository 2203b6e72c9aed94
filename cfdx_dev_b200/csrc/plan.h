// plan.h -- automatic solver selection on the host.
//
// measure_characteristics restates measure_matrix_characteristics
// (core/linalg/matrix_diagnostics.h:285-358) together with the part of
// diagnose_matrix (:126-225) it reads; select_solver (plan.cpp) restates
// select_linear_solver (core/linalg/linear_solver_models.h:228-425).  Both
// run on the host arrays the library already mirrors, only when a request
// asks for automatic selection.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <string>
#include <vector>

#include "cfdxg.h"

namespace cfdxg {

// std::min / std::max as the reference calls them: the first argument wins
// unless the second compares strictly less / greater (a NaN never replaces).
inline double ref_min(double a, double b) { return b < a ? b : a; }
inline double ref_max(double a, double b) { return a < b ? b : a; }

// Characteristics of a square CSR matrix whose columns increase strictly in
// each row (the caller validates the structure).  A non-finite value makes the
// reference's diagnosis stop early (SparseMatrix::is_consistent is false:
// sparse_matrix.h:256-275), which leaves its coefficient evidence at the
// defaults; that is kept.
template <class I>
void measure_characteristics(int64_t n, const I* ro, const I* co, const double* va, bool saddle_point,
                             double symmetry_tolerance, cfdxg_matrix_characteristics& c) {
    const double inf = std::numeric_limits<double>::infinity();
    const int64_t nnz = static_cast<int64_t>(ro[n]);
    bool consistent = true;
    for (int64_t k = 0; k < nnz && consistent; ++k) consistent = std::isfinite(va[k]);

    // diagnose_matrix(matrix, 1e-14, false): the fields the profile reads
    double max_abs = 0.0, min_nonzero_abs = inf, max_abs_diag = 0.0, min_nonzero_abs_diag = inf;
    double gershgorin = inf, diag_range = 1.0;
    int64_t missing_diagonal = 0;
    if (consistent) {
        for (int64_t i = 0; i < n; ++i) {
            bool present = false;
            double diagonal = 0.0, offdiag = 0.0;
            for (int64_t k = static_cast<int64_t>(ro[i]); k < static_cast<int64_t>(ro[i + 1]); ++k) {
                const double m = std::fabs(va[k]);
                max_abs = ref_max(max_abs, m);
                if (m > 0.0) min_nonzero_abs = ref_min(min_nonzero_abs, m);
                if (static_cast<int64_t>(co[k]) == i) {
                    present = true;
                    diagonal += va[k];
                }
            }
            if (!present) ++missing_diagonal;
            const double dabs = std::fabs(diagonal);
            if (dabs > 0.0) {
                max_abs_diag = ref_max(max_abs_diag, dabs);
                min_nonzero_abs_diag = ref_min(min_nonzero_abs_diag, dabs);
            }
            for (int64_t k = static_cast<int64_t>(ro[i]); k < static_cast<int64_t>(ro[i + 1]); ++k)
                if (static_cast<int64_t>(co[k]) != i) offdiag += std::fabs(va[k]);
            gershgorin = ref_min(gershgorin, dabs - offdiag);
        }
        if (min_nonzero_abs_diag < inf) diag_range = max_abs_diag / min_nonzero_abs_diag;
    }

    c.equations = n;
    c.average_nnz_per_row = n == 0 ? 0.0 : static_cast<double>(nnz) / static_cast<double>(n);
    c.coefficient_range = min_nonzero_abs == inf ? 1.0 : max_abs / min_nonzero_abs;
    c.square = 1;
    c.diagonally_dominant = std::isfinite(gershgorin) && gershgorin >= -1e-14 * ref_max(1.0, max_abs_diag);
    c.strongly_scaled = std::isfinite(c.coefficient_range) && c.coefficient_range >= 1.0e8;
    c.large_diagonal_dynamic_range = std::isfinite(diag_range) && diag_range >= 1.0e4;
    c.saddle_point = saddle_point ? 1 : 0;
    c.strongly_directional_coupling = 0;
    c.positive_diagonal = missing_diagonal == 0;
    for (int64_t i = 0; i < n; ++i) {
        // per row: the diagonal sum and the spread of the negative couplings
        double diag = 0.0, weakest = inf, strongest = 0.0;
        for (int64_t k = static_cast<int64_t>(ro[i]); k < static_cast<int64_t>(ro[i + 1]); ++k) {
            if (static_cast<int64_t>(co[k]) == i) diag += va[k];
            else if (va[k] < 0.0) {
                weakest = ref_min(weakest, -va[k]);
                strongest = ref_max(strongest, -va[k]);
            }
        }
        if (!(diag > 0.0) || !std::isfinite(diag)) c.positive_diagonal = 0;
        if (weakest < inf && strongest / weakest >= 1.0e3) c.strongly_directional_coupling = 1;
    }
    // numerical symmetry against max(1, max|a|) (a_ji = 0 where absent)
    const double tol = symmetry_tolerance * ref_max(1.0, max_abs);
    c.numerically_symmetric = n > 0 ? 1 : 0;
    for (int64_t i = 0; i < n && c.numerically_symmetric; ++i) {
        for (int64_t k = static_cast<int64_t>(ro[i]); k < static_cast<int64_t>(ro[i + 1]); ++k) {
            const int64_t j = static_cast<int64_t>(co[k]);
            double aji = 0.0;
            for (int64_t q = static_cast<int64_t>(ro[j]); q < static_cast<int64_t>(ro[j + 1]); ++q)
                if (static_cast<int64_t>(co[q]) == i) aji += va[q];
            if (std::fabs(va[k] - aji) > tol) {
                c.numerically_symmetric = 0;
                break;
            }
        }
    }
}

// scale_matrix (core/linalg/matrix_diagnostics.h:410-490): row/column scales
// 1 / max|a| (Row, Column, RowColumn) or 1 / sqrt|a_ii| on both sides
// (SymmetricDiagonal, a_ii = the sum of the row's diagonal entries), left at 1
// where the maximum (or |a_ii|) is <= zero_tolerance, which is counted; the
// scaled entry is (a_ij * r_i) * c_j, re-stored as 0 + value the way the
// reference's finalize re-accumulates each entry.
template <class I>
void scale_values(int32_t mode, int64_t n, const I* ro, const I* co, const double* va, double zero_tolerance,
                  double* row_scale, double* col_scale, double* scaled, int64_t& zero_rows, int64_t& zero_cols) {
    zero_rows = zero_cols = 0;
    for (int64_t i = 0; i < n; ++i) row_scale[i] = col_scale[i] = 1.0;
    const bool rows = mode == 1 || mode == 3, cols = mode == 2 || mode == 3;
    if (rows || cols) {
        std::vector<double> row_max(static_cast<size_t>(n), 0.0), col_max(static_cast<size_t>(n), 0.0);
        for (int64_t i = 0; i < n; ++i)
            for (int64_t k = static_cast<int64_t>(ro[i]); k < static_cast<int64_t>(ro[i + 1]); ++k) {
                const double m = std::fabs(va[k]);
                row_max[i] = ref_max(row_max[i], m);
                col_max[co[k]] = ref_max(col_max[co[k]], m);
            }
        for (int64_t i = 0; i < n && rows; ++i) {
            if (row_max[i] <= zero_tolerance) ++zero_rows;
            else row_scale[i] = 1.0 / row_max[i];
        }
        for (int64_t j = 0; j < n && cols; ++j) {
            if (col_max[j] <= zero_tolerance) ++zero_cols;
            else col_scale[j] = 1.0 / col_max[j];
        }
    }
    if (mode == 4) {
        for (int64_t i = 0; i < n; ++i) {
            double d = 0.0;
            for (int64_t k = static_cast<int64_t>(ro[i]); k < static_cast<int64_t>(ro[i + 1]); ++k)
                if (static_cast<int64_t>(co[k]) == i) d += va[k];
            d = std::fabs(d);
            if (d <= zero_tolerance) {
                ++zero_rows;
                ++zero_cols;
            } else {
                row_scale[i] = col_scale[i] = 1.0 / std::sqrt(d);
            }
        }
    }
    for (int64_t i = 0; i < n; ++i)
        for (int64_t k = static_cast<int64_t>(ro[i]); k < static_cast<int64_t>(ro[i + 1]); ++k)
            scaled[k] = 0.0 + va[k] * row_scale[i] * col_scale[co[k]];
}

// select_linear_solver; false with the reason in `why` where the reference
// throws std::invalid_argument.
bool select_solver(int32_t problem, const cfdxg_matrix_characteristics& c, const cfdxg_plan_request& r,
                   cfdxg_solver_plan& plan, std::string& why);

const char* krylov_model_name(int32_t model);
const char* preconditioner_model_name(int32_t model);

}  // namespace cfdxg
