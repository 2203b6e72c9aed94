// mpnn.h -- learned message-passing preconditioner (internal interface).
#pragma once
#include <functional>

#include "objects.h"

namespace cfdxg {

// Binds the network to the matrix a solve uses (edge weights, features).
void bind_learned_to_matrix(cfdxg_context* ctx, cfdxg_mpnn* net, const cfdxg_matrix* A);

// z = y + M(v - A y) with y = N(v); falls back to z = M(v) (and counts it)
// when y does not reduce the residual, i.e. ||v - A y|| >= ||v||.
bool learned_then_amg(cfdxg_context* ctx, cfdxg_mpnn* net, const cfdxg_matrix* A, const double* v, double* z,
                      const std::function<void(const double*, double*)>& amg, int64_t* fallbacks);

// Fallbacks recorded on the device since the last call (synchronises).
int64_t learned_take_fallbacks(cfdxg_context* ctx, cfdxg_mpnn* net);

}  // namespace cfdxg
