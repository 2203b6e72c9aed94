// mpnn.h -- learned message-passing preconditioner (internal interface).
#pragma once
#include <functional>

#include "objects.h"

namespace cfdxg {

// Binds the network to the matrix a solve uses (edge weights, features).
void bind_learned_to_matrix(cfdxg_context* ctx, cfdxg_mpnn* net, const cfdxg_matrix* A);

// z = y + M(v - A y) with y = N(v) and M the AMG V-cycle.  The caller drops
// the learned stage (plain M) when the Krylov iteration stops converging.
bool learned_then_amg(cfdxg_context* ctx, cfdxg_mpnn* net, const cfdxg_matrix* A, const double* v, double* z,
                      const std::function<void(const double*, double*)>& amg, int64_t* fallbacks);

}  // namespace cfdxg
