// Domain decomposition plan: contiguous row blocks with halos.
//
// A square plan splits a system's rows and, with the same splits, its
// unknowns; a rectangular plan (a transfer operator between two AMG levels)
// splits its rows and its columns separately, each part owning a block of
// each.
//
// The reference solves each pressure system on one rank
// (core/linalg/linear_solver_dispatch.h:227-234 takes the whole SparseMatrix,
// and the Krylov and AMG code has no distributed form), so this plan has no
// reference counterpart: it is what lets one system spread over several
// GPUs.  A part owns the global rows [r0, r1).  Its local vector is
//
//   [ghosts below r0 | owned rows r0..r1-1 | ghosts above r1]
//
// with the ghosts (the columns of owned rows that other parts own) in
// increasing global order.  That numbering is increasing in the global
// column, so every local row lists its entries in the global row's order
// and a local product y = A_loc x_loc sums each owned row exactly as the
// global product does.  Because parts own contiguous row ranges, the ghosts
// that one neighbour owns form one contiguous slice of the local vector, so
// a halo exchange receives straight into place; the sender packs its owned
// values in the same increasing global order.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "cfdxg.h"

namespace {

struct Part {
    int64_t r0 = 0, r1 = 0;                  // owned rows
    int64_t c0 = 0, c1 = 0;                  // owned columns (= rows for a square plan)
    int64_t below = 0;                       // ghosts below c0
    int64_t first_row = 0;                   // local row of r0
    std::vector<int64_t> lro, lco, lsrc;     // local system
    std::vector<int64_t> bro, bco, bsrc;     // owned-column block
    std::vector<int64_t> ghosts;             // global columns, increasing
    std::vector<int32_t> nb;                 // neighbours (receive from or send to)
    std::vector<int64_t> recv_off, recv_start, send_off, send_rows;
};

thread_local std::string g_error;

int fail(int code, const std::string& why) {
    g_error = why;
    return code;
}

int owner_of(const std::vector<int64_t>& splits, int64_t index) {
    return static_cast<int>(std::upper_bound(splits.begin(), splits.end(), index) - splits.begin()) - 1;
}

}  // namespace

struct cfdxg_domain_plan {
    int64_t n_rows = 0, n_cols = 0;
    bool square = true;
    std::vector<int64_t> row_splits, col_splits;
    std::vector<Part> parts;
};

namespace {

std::string validate_pattern(int64_t n_rows, int64_t n_cols, const int64_t* ro, const int64_t* co) {
    if (ro[0] != 0) return "domain plan: row offsets must start at 0";
    for (int64_t i = 0; i < n_rows; ++i) {
        if (ro[i + 1] < ro[i]) return "domain plan: row offsets decrease";
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k) {
            if (co[k] < 0 || co[k] >= n_cols) return "domain plan: column out of range";
            if (k > ro[i] && co[k - 1] >= co[k]) return "domain plan: columns not strictly increasing in a row";
        }
    }
    return {};
}

std::string validate_splits(const std::vector<int64_t>& s, int64_t n, const char* what) {
    if (s.front() != 0 || s.back() != n) return std::string("domain plan: ") + what + " splits must run from 0 to n";
    for (size_t k = 0; k + 1 < s.size(); ++k)
        if (s[k + 1] <= s[k]) return std::string("domain plan: every part must own at least one ") + what;
    return {};
}

// Blocks of nearly equal entry counts: split k starts at the first row whose
// offset reaches k * nnz / parts, kept strictly increasing with at least one
// row per block.
std::vector<int64_t> balanced_splits(int64_t n, const int64_t* ro, int parts) {
    std::vector<int64_t> s(parts + 1, 0);
    const int64_t nnz = ro[n];
    for (int k = 1; k < parts; ++k) {
        const int64_t target = static_cast<int64_t>((static_cast<__int128>(nnz) * k) / parts);
        int64_t r = std::lower_bound(ro, ro + n + 1, target) - ro;
        r = std::max(r, s[k - 1] + 1);
        r = std::min(r, n - (parts - k));
        s[k] = r;
    }
    s[parts] = n;
    return s;
}

// Local numbering of the column space [ghosts below | owned | ghosts above].
// A square plan pads the local rows to the local vector (owned rows at the
// owned columns' positions, ghost rows empty), so one square product maps a
// local vector to a local vector; a rectangular plan keeps the owned rows only.
void build_local(const int64_t* ro, const int64_t* co, bool square, Part& P) {
    const int64_t r0 = P.r0, r1 = P.r1, c0 = P.c0, c1 = P.c1, owned = c1 - c0;
    for (int64_t i = r0; i < r1; ++i)
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k)
            if (co[k] < c0 || co[k] >= c1) P.ghosts.push_back(co[k]);
    std::sort(P.ghosts.begin(), P.ghosts.end());
    P.ghosts.erase(std::unique(P.ghosts.begin(), P.ghosts.end()), P.ghosts.end());
    P.below = std::lower_bound(P.ghosts.begin(), P.ghosts.end(), c0) - P.ghosts.begin();
    const int64_t n_local = owned + static_cast<int64_t>(P.ghosts.size());
    auto local_of = [&](int64_t c) -> int64_t {
        if (c >= c0 && c < c1) return P.below + (c - c0);
        const int64_t g = std::lower_bound(P.ghosts.begin(), P.ghosts.end(), c) - P.ghosts.begin();
        return c < c0 ? g : g + owned;
    };
    P.first_row = square ? P.below : 0;
    P.lro.assign(static_cast<size_t>(P.first_row) + 1, 0);
    P.bro.assign(1, 0);
    for (int64_t i = r0; i < r1; ++i) {
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k) {
            P.lco.push_back(local_of(co[k]));
            P.lsrc.push_back(k);
            if (co[k] >= c0 && co[k] < c1) {
                P.bco.push_back(co[k] - c0);
                P.bsrc.push_back(k);
            }
        }
        P.lro.push_back(static_cast<int64_t>(P.lco.size()));
        P.bro.push_back(static_cast<int64_t>(P.bco.size()));
    }
    if (square)
        while (static_cast<int64_t>(P.lro.size()) < n_local + 1) P.lro.push_back(static_cast<int64_t>(P.lco.size()));
}

int create(int64_t n_rows, int64_t n_cols, const int64_t* ro, const int64_t* co, int32_t parts,
           const int64_t* row_splits, const int64_t* col_splits, bool square, cfdxg_domain_plan** out) {
    if (!out) return fail(CFDXG_ERR_INVALID_ARGUMENT, "domain plan: null argument");
    *out = nullptr;
    if (n_rows <= 0 || n_cols <= 0 || !ro || (ro[n_rows] > 0 && !co))
        return fail(CFDXG_ERR_INVALID_ARGUMENT, "domain plan: empty or null system");
    if (parts < 1 || parts > n_rows || parts > n_cols)
        return fail(CFDXG_ERR_INVALID_ARGUMENT, "domain plan: need 1 <= parts <= rows and columns");
    if (!square && (!row_splits || !col_splits))
        return fail(CFDXG_ERR_INVALID_ARGUMENT, "domain plan: a rectangular plan needs row and column splits");
    try {
        std::string why = validate_pattern(n_rows, n_cols, ro, co);
        if (!why.empty()) return fail(CFDXG_ERR_INVALID_ARGUMENT, why);
        auto plan = std::make_unique<cfdxg_domain_plan>();
        plan->n_rows = n_rows;
        plan->n_cols = n_cols;
        plan->square = square;
        if (row_splits) {
            plan->row_splits.assign(row_splits, row_splits + parts + 1);
            why = validate_splits(plan->row_splits, n_rows, "row");
            if (!why.empty()) return fail(CFDXG_ERR_INVALID_ARGUMENT, why);
        } else {
            plan->row_splits = balanced_splits(n_rows, ro, parts);
        }
        if (square) {
            plan->col_splits = plan->row_splits;
        } else {
            plan->col_splits.assign(col_splits, col_splits + parts + 1);
            why = validate_splits(plan->col_splits, n_cols, "column");
            if (!why.empty()) return fail(CFDXG_ERR_INVALID_ARGUMENT, why);
        }
        const auto& cs = plan->col_splits;
        plan->parts.resize(parts);
        for (int p = 0; p < parts; ++p) {
            Part& P = plan->parts[p];
            P.r0 = plan->row_splits[p];
            P.r1 = plan->row_splits[p + 1];
            P.c0 = cs[p];
            P.c1 = cs[p + 1];
            build_local(ro, co, square, P);
        }
        // per part and neighbour: [ghost range received] and [owned columns sent]
        std::vector<std::map<int, std::pair<std::pair<int64_t, int64_t>, std::vector<int64_t>>>> links(parts);
        for (int p = 0; p < parts; ++p) {
            const Part& P = plan->parts[p];
            for (size_t g = 0; g < P.ghosts.size();) {
                const int q = owner_of(cs, P.ghosts[g]);
                size_t e = g;
                while (e < P.ghosts.size() && P.ghosts[e] < cs[q + 1]) ++e;
                links[p][q].first = {static_cast<int64_t>(g), static_cast<int64_t>(e)};
                auto& send = links[q][p].second;
                for (size_t t = g; t < e; ++t) send.push_back(P.ghosts[t] - cs[q]);
                g = e;
            }
        }
        for (int p = 0; p < parts; ++p) {
            Part& P = plan->parts[p];
            const int64_t owned = P.c1 - P.c0;
            P.recv_off.push_back(0);
            P.send_off.push_back(0);
            for (auto& [q, link] : links[p]) {
                const auto [g0, g1] = link.first;
                P.nb.push_back(q);
                P.recv_off.push_back(P.recv_off.back() + (g1 - g0));
                // an empty receive range keeps the slice position where it would sit
                const int64_t at = g1 > g0 ? g0 : static_cast<int64_t>(q < p ? P.below : P.ghosts.size());
                P.recv_start.push_back(q < p ? at : at + owned);
                P.send_rows.insert(P.send_rows.end(), link.second.begin(), link.second.end());
                P.send_off.push_back(static_cast<int64_t>(P.send_rows.size()));
            }
        }
        *out = plan.release();
    } catch (const std::bad_alloc&) {
        return fail(CFDXG_ERR_OUT_OF_MEMORY, "domain plan: out of host memory");
    }
    g_error.clear();
    return CFDXG_OK;
}

}  // namespace

extern "C" {

int cfdxg_domain_plan_create(int64_t n, const int64_t* ro, const int64_t* co, int32_t parts,
                             const int64_t* row_splits, cfdxg_domain_plan** out) {
    return create(n, n, ro, co, parts, row_splits, nullptr, true, out);
}

int cfdxg_domain_plan_create_rect(int64_t n_rows, int64_t n_cols, const int64_t* ro, const int64_t* co,
                                  int32_t parts, const int64_t* row_splits, const int64_t* col_splits,
                                  cfdxg_domain_plan** out) {
    return create(n_rows, n_cols, ro, co, parts, row_splits, col_splits, false, out);
}

int cfdxg_domain_plan_parts(const cfdxg_domain_plan* plan, int64_t* row_splits, int64_t* col_splits) {
    if (!plan) return fail(CFDXG_ERR_INVALID_ARGUMENT, "domain plan: null handle");
    if (row_splits) std::memcpy(row_splits, plan->row_splits.data(), plan->row_splits.size() * sizeof(int64_t));
    if (col_splits) std::memcpy(col_splits, plan->col_splits.data(), plan->col_splits.size() * sizeof(int64_t));
    return static_cast<int>(plan->parts.size());
}

int cfdxg_domain_plan_info(const cfdxg_domain_plan* plan, int32_t part, cfdxg_domain_part_info* info) {
    if (!plan || !info) return fail(CFDXG_ERR_INVALID_ARGUMENT, "domain plan: null argument");
    if (part < 0 || part >= static_cast<int32_t>(plan->parts.size()))
        return fail(CFDXG_ERR_INVALID_ARGUMENT, "domain plan: part out of range");
    const Part& P = plan->parts[part];
    info->row_begin = P.r0;
    info->row_end = P.r1;
    info->n_local = (P.c1 - P.c0) + static_cast<int64_t>(P.ghosts.size());
    info->owned_offset = P.below;
    info->nnz_local = static_cast<int64_t>(P.lco.size());
    info->nnz_block = static_cast<int64_t>(P.bco.size());
    info->n_neighbours = static_cast<int32_t>(P.nb.size());
    info->n_recv = static_cast<int64_t>(P.ghosts.size());
    info->n_send = static_cast<int64_t>(P.send_rows.size());
    info->col_begin = P.c0;
    info->col_end = P.c1;
    info->n_local_rows = static_cast<int64_t>(P.lro.size()) - 1;
    info->first_row = P.first_row;
    return CFDXG_OK;
}

int cfdxg_domain_plan_export(const cfdxg_domain_plan* plan, int32_t part, const cfdxg_domain_part_arrays* out) {
    if (!plan || !out) return fail(CFDXG_ERR_INVALID_ARGUMENT, "domain plan: null argument");
    if (part < 0 || part >= static_cast<int32_t>(plan->parts.size()))
        return fail(CFDXG_ERR_INVALID_ARGUMENT, "domain plan: part out of range");
    const Part& P = plan->parts[part];
    auto put = [](auto* dst, const auto& v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    put(out->local_row_offsets, P.lro);
    put(out->local_columns, P.lco);
    put(out->local_source, P.lsrc);
    put(out->block_row_offsets, P.bro);
    put(out->block_columns, P.bco);
    put(out->block_source, P.bsrc);
    put(out->neighbours, P.nb);
    put(out->recv_offsets, P.recv_off);
    put(out->recv_start, P.recv_start);
    put(out->ghost_rows, P.ghosts);
    put(out->send_offsets, P.send_off);
    put(out->send_rows, P.send_rows);
    return CFDXG_OK;
}

int cfdxg_domain_plan_destroy(cfdxg_domain_plan* plan) {
    delete plan;
    return CFDXG_OK;
}

const char* cfdxg_domain_last_error(void) { return g_error.c_str(); }

}  // extern "C"
