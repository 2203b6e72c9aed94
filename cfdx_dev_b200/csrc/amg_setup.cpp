// amg_setup.cpp -- bit-exact, fast host restatement of the reference's
// classical RS AMG setup.  See amg_setup.h for the contract.
#include "amg_setup.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <limits>
#include <queue>
#include <thread>
#include <chrono>
#include <cstdio>
#include <utility>

namespace cfdxg {

namespace {
bool profile_setup() {
    static const bool on = std::getenv("CFDXG_SETUP_PROFILE") != nullptr;
    return on;
}
double tnow() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
}  // namespace

int host_threads() {
    static int n = [] {
        if (const char* s = std::getenv("CFDXG_HOST_THREADS")) {
            const int v = std::atoi(s);
            if (v > 0) return v;
        }
        const unsigned hc = std::thread::hardware_concurrency();
        return static_cast<int>(std::max(1u, std::min(hc, 32u)));
    }();
    return n;
}

namespace {

// Runs fn(begin, end, worker) over [0, n) in contiguous blocks, one per worker.
template <class Fn>
void parallel_blocks(int64_t n, Fn&& fn, int64_t min_per_thread = 4096) {
    int workers = host_threads();
    if (n < min_per_thread * 2) workers = 1;
    workers = static_cast<int>(std::min<int64_t>(workers, std::max<int64_t>(1, n / std::max<int64_t>(1, min_per_thread))));
    if (workers <= 1) {
        fn(int64_t(0), n, 0);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(workers);
    for (int w = 0; w < workers; ++w) {
        const int64_t b = n * w / workers, e = n * (w + 1) / workers;
        pool.emplace_back([&fn, b, e, w] { fn(b, e, w); });
    }
    for (auto& t : pool) t.join();
}

// Dynamic schedule: workers pull chunks of `chunk` rows from a shared counter,
// so dense rows do not leave threads idle.  fn(begin, end, worker).
template <class Fn>
void parallel_chunks(int64_t n, int64_t chunk, Fn&& fn) {
    const int workers = static_cast<int>(std::min<int64_t>(host_threads(), (n + chunk - 1) / chunk));
    if (workers <= 1) {
        fn(int64_t(0), n, 0);
        return;
    }
    std::atomic<int64_t> next{0};
    std::vector<std::thread> pool;
    pool.reserve(workers);
    for (int w = 0; w < workers; ++w)
        pool.emplace_back([&, w] {
            for (;;) {
                const int64_t b = next.fetch_add(chunk);
                if (b >= n) break;
                fn(b, std::min(n, b + chunk), w);
            }
        });
    for (auto& t : pool) t.join();
}

inline int workers_for(int64_t n, int64_t min_per_thread = 4096) {
    int workers = host_threads();
    if (n < min_per_thread * 2) return 1;
    return static_cast<int>(std::min<int64_t>(workers, std::max<int64_t>(1, n / min_per_thread)));
}

// amg_preconditioner.h:1258-1275 matrix_is_valid + sparse_matrix.h:248 is_consistent
bool matrix_is_valid(const HostCsr& A) {
    if (A.n <= 0 || static_cast<int64_t>(A.ro.size()) != A.n + 1 || A.ro[0] != 0 ||
        A.ro[A.n] != static_cast<uint32_t>(A.co.size()) || A.co.size() != A.va.size())
        return false;
    for (int64_t i = 0; i < A.n; ++i)
        if (A.ro[i + 1] < A.ro[i]) return false;
    std::atomic<bool> ok{true};
    parallel_chunks(A.n, 4096, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e && ok.load(std::memory_order_relaxed); ++i)
            for (uint32_t k = A.ro[i]; k < A.ro[i + 1]; ++k) {
                if (A.co[k] >= A.n || !std::isfinite(A.va[k]) || (k > A.ro[i] && A.co[k] <= A.co[k - 1])) {
                    ok = false;
                    return;
                }
            }
    });
    return ok;
}

// Value lookup on a row with sorted unique columns: identical to the
// reference's linear matrix_value scan (amg_preconditioner.h:1668-1674),
// which returns 0.0 + a_ij, i.e. a_ij, or 0.0 when absent.
inline double row_value(const HostCsr& A, int64_t i, uint32_t j) {
    const uint32_t* b = A.co.data() + A.ro[i];
    const uint32_t* e = A.co.data() + A.ro[i + 1];
    const uint32_t* it = std::lower_bound(b, e, j);
    if (it == e || *it != j) return 0.0;
    return 0.0 + A.va[static_cast<std::size_t>(it - A.co.data())];
}

struct Strength {
    // padded CSR: row i owns [A.ro[i], A.ro[i] + len[i]) of col
    std::vector<uint32_t> col, len;
    const HostCsr* A = nullptr;
    const uint32_t* begin(int64_t i) const { return col.data() + A->ro[i]; }
    const uint32_t* end(int64_t i) const { return col.data() + A->ro[i] + len[i]; }
    uint32_t size(int64_t i) const { return len[i]; }
};

// amg_preconditioner.h:1466-1509
void build_strength_graph(const HostCsr& A, const std::vector<double>& inv_diag,
                          double threshold, Strength& s) {
    const int64_t n = A.n;
    s.A = &A;
    s.col.assign(A.co.size(), 0);
    s.len.assign(static_cast<std::size_t>(n), 0);
    constexpr double max_row_sum = 0.9;
    parallel_blocks(n, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e; ++i) {
            const double di = 1.0 / inv_diag[i];
            double row_sum = di;
            double opposite_max = 0.0;
            double absolute_max = 0.0;
            for (uint32_t k = A.ro[i]; k < A.ro[i + 1]; ++k) {
                if (A.co[k] == i) continue;
                row_sum += A.va[k];
                absolute_max = std::max(absolute_max, std::abs(A.va[k]));
                if (di * A.va[k] < 0.0) opposite_max = std::max(opposite_max, std::abs(A.va[k]));
            }
            if (std::abs(row_sum) > std::abs(di) * max_row_sum) continue;
            const bool use_opposite = opposite_max > 0.0;
            const double scale = use_opposite ? opposite_max : absolute_max;
            if (!(scale > 0.0) || !std::isfinite(scale)) continue;
            uint32_t cnt = 0;
            for (uint32_t k = A.ro[i]; k < A.ro[i + 1]; ++k) {
                const uint32_t j = A.co[k];
                if (j == i || j >= n) continue;
                if (use_opposite && di * A.va[k] >= 0.0) continue;
                if (std::abs(A.va[k]) + std::numeric_limits<double>::epsilon() < threshold * scale) continue;
                s.col[A.ro[i] + cnt++] = j;   // CSR columns are sorted and unique
            }
            s.len[i] = cnt;
        }
    });
}

enum : uint8_t { kUndecided = 0, kFine = 1, kCoarse = 2 };

// The undecided points of the first pass by influence: per influence value a
// three-level 64-ary bitmap over the point indices, so that the selection --
// the largest influence, then the smallest index -- and every insertion and
// removal take a few word operations.  It selects exactly the point the
// reference's heap over (measure, n - i) with lazily skipped stale entries
// selects.
class InfluenceBuckets {
public:
    explicit InfluenceBuckets(int64_t n)
        : w0_((n + 63) / 64), w1_((w0_ + 63) / 64), w2_((w1_ + 63) / 64) {}
    void insert(uint32_t m, uint32_t i) {
        if (m >= words_.size()) {
            words_.resize(static_cast<std::size_t>(m) + 1);
            count_.resize(static_cast<std::size_t>(m) + 1, 0);
        }
        auto& b = words_[m];
        if (b.empty()) b.assign(static_cast<std::size_t>(w0_ + w1_ + w2_), 0);
        uint64_t* l0 = b.data();
        uint64_t* l1 = l0 + w0_;
        uint64_t* l2 = l1 + w1_;
        l0[i >> 6] |= uint64_t{1} << (i & 63);
        l1[i >> 12] |= uint64_t{1} << ((i >> 6) & 63);
        l2[i >> 18] |= uint64_t{1} << ((i >> 12) & 63);
        ++count_[m];
        if (static_cast<int64_t>(m) > top_) top_ = m;
    }
    void erase(uint32_t m, uint32_t i) {
        auto& b = words_[m];
        uint64_t* l0 = b.data();
        uint64_t* l1 = l0 + w0_;
        uint64_t* l2 = l1 + w1_;
        l0[i >> 6] &= ~(uint64_t{1} << (i & 63));
        if (l0[i >> 6] == 0) {
            l1[i >> 12] &= ~(uint64_t{1} << ((i >> 6) & 63));
            if (l1[i >> 12] == 0) l2[i >> 18] &= ~(uint64_t{1} << ((i >> 12) & 63));
        }
        --count_[m];
    }
    // the largest non-empty influence and its smallest index; false when empty
    bool best(uint32_t& m, uint32_t& i) {
        while (top_ >= 0 && count_[top_] == 0) --top_;
        if (top_ < 0) return false;
        const auto& b = words_[top_];
        const uint64_t* l0 = b.data();
        const uint64_t* l1 = l0 + w0_;
        const uint64_t* l2 = l1 + w1_;
        int64_t w2 = 0;
        while (w2 < w2_ && l2[w2] == 0) ++w2;
        if (w2 == w2_) return false;
        const int64_t w1 = w2 * 64 + __builtin_ctzll(l2[w2]);
        const int64_t w0 = w1 * 64 + __builtin_ctzll(l1[w1]);
        i = static_cast<uint32_t>(w0 * 64 + __builtin_ctzll(l0[w0]));
        m = static_cast<uint32_t>(top_);
        return true;
    }

private:
    int64_t w0_, w1_, w2_;
    std::vector<std::vector<uint64_t>> words_;
    std::vector<int64_t> count_;
    int64_t top_ = -1;
};

// amg_preconditioner.h:1511-1885 (DirectCF, no row cap)
bool build_cf_interpolation(const HostCsr& A, const std::vector<double>& inv_diag,
                            double threshold, AmgLevel& level, int64_t& coarse_n) {
    const int64_t n = A.n;
    const double t_start = tnow();
    Strength strong;
    build_strength_graph(A, inv_diag, threshold, strong);
    const double t_strength = tnow();

    // transpose of the strength graph, rows in increasing source order
    std::vector<uint32_t> t_off(static_cast<std::size_t>(n) + 1, 0), t_col;
    for (int64_t i = 0; i < n; ++i)
        for (const uint32_t* p = strong.begin(i); p != strong.end(i); ++p) ++t_off[*p + 1];
    for (int64_t i = 0; i < n; ++i) t_off[i + 1] += t_off[i];
    t_col.resize(t_off[n]);
    {
        std::vector<uint32_t> cursor(t_off.begin(), t_off.end() - 1);
        for (int64_t i = 0; i < n; ++i)
            for (const uint32_t* p = strong.begin(i); p != strong.end(i); ++p)
                t_col[cursor[*p]++] = static_cast<uint32_t>(i);
    }

    // First pass: dynamic-influence selection (the largest influence, the
    // lowest index among equals), the undecided points kept by influence.
    std::vector<uint8_t> point(static_cast<std::size_t>(n), kUndecided);
    std::vector<uint32_t> influence(static_cast<std::size_t>(n));
    InfluenceBuckets candidates(n);
    for (int64_t i = 0; i < n; ++i) {
        influence[i] = t_off[i + 1] - t_off[i];
        candidates.insert(influence[i], static_cast<uint32_t>(i));
    }
    int64_t undecided = n;
    while (undecided > 0) {
        uint32_t measure = 0, best = 0;
        if (!candidates.best(measure, best)) return false;
        candidates.erase(measure, best);
        point[best] = kCoarse;
        --undecided;
        for (uint32_t t = t_off[best]; t < t_off[best + 1]; ++t) {
            const uint32_t j = t_col[t];
            if (point[j] != kUndecided) continue;
            candidates.erase(influence[j], j);
            point[j] = kFine;
            --undecided;
            for (const uint32_t* p = strong.begin(j); p != strong.end(j); ++p) {
                const uint32_t k = *p;
                if (point[k] == kUndecided) {
                    candidates.erase(influence[k], k);
                    ++influence[k];
                    candidates.insert(influence[k], k);
                }
            }
        }
    }

    const double t_pass1 = tnow();
    // Second pass.  The reference restarts its scan at row 0 after each
    // promotion; promotions only grow the C set, which can neither create an
    // uncovered F-F edge at an earlier row nor un-cover a covered one, so a
    // scan that resumes at the next row selects exactly the same points.
    // After the first pass no point is undecided, so the neighbourhood
    // marking of the reference is a no-op and is omitted.
    // Same boolean as the reference's nested scan (is there a C point in
    // S_i intersect S_j?), evaluated by merging the two sorted rows.
    const auto has_common_coarse = [&](int64_t i, int64_t j) {
        const uint32_t *a = strong.begin(i), *ae = strong.end(i);
        const uint32_t *b = strong.begin(j), *be = strong.end(j);
        while (a != ae && b != be) {
            if (*a < *b) ++a;
            else if (*b < *a) ++b;
            else {
                if (point[*a] == kCoarse) return true;
                ++a;
                ++b;
            }
        }
        return false;
    };
    for (int64_t i = 0; i < n; ++i) {
        if (point[i] != kFine) continue;
        for (const uint32_t* p = strong.begin(i); p != strong.end(i); ++p) {
            const uint32_t j = *p;
            if (point[j] != kFine) continue;
            if (has_common_coarse(i, j)) continue;
            point[i] = kCoarse;
            break;
        }
    }
    // Promote F points without a strong C neighbour (sequential, order matters).
    for (int64_t i = 0; i < n; ++i) {
        if (point[i] != kFine) continue;
        bool has_strong_c = false;
        for (const uint32_t* p = strong.begin(i); p != strong.end(i); ++p)
            if (point[*p] == kCoarse) { has_strong_c = true; break; }
        if (!has_strong_c) point[i] = kCoarse;
    }

    const double t_pass2 = tnow();
    std::vector<uint32_t> coarse_index(static_cast<std::size_t>(n), static_cast<uint32_t>(n));
    coarse_n = 0;
    for (int64_t i = 0; i < n; ++i)
        if (point[i] == kCoarse) coarse_index[i] = static_cast<uint32_t>(coarse_n++);

    // Interpolation rows, computed independently per fine row.
    const int workers = workers_for(n, 2048);
    std::vector<std::vector<uint32_t>> w_len(workers), w_col(workers), w_agg(workers);
    std::vector<std::vector<double>> w_val(workers);
    std::atomic<bool> failed{false};
    std::vector<int64_t> bounds(workers + 1);
    for (int w = 0; w <= workers; ++w) bounds[w] = n * w / workers;
    auto rows_job = [&](int w) {
        auto& len = w_len[w];
        auto& col = w_col[w];
        auto& val = w_val[w];
        auto& agg = w_agg[w];
        std::vector<std::pair<uint32_t, double>> weights;
        // stamped sparse accumulator (amg_preconditioner.h:1688-1700): O(1) lookups
        std::vector<int64_t> stamp(static_cast<std::size_t>(coarse_n), -1);
        std::vector<uint32_t> slot_of(static_cast<std::size_t>(coarse_n), 0);
        std::vector<uint32_t> kc;
        for (int64_t i = bounds[w]; i < bounds[w + 1] && !failed.load(std::memory_order_relaxed); ++i) {
            if (point[i] == kCoarse) {
                len.push_back(1);
                col.push_back(coarse_index[i]);
                val.push_back(1.0);
                agg.push_back(coarse_index[i]);
                continue;
            }
            const double diagonal = 1.0 / inv_diag[i];
            bool any_c = false;
            for (const uint32_t* p = strong.begin(i); p != strong.end(i); ++p)
                if (point[*p] == kCoarse) { any_c = true; break; }
            if (!any_c) { failed = true; return; }
            double weak_sum = 0.0;
            for (uint32_t k = A.ro[i]; k < A.ro[i + 1]; ++k) {
                const uint32_t j = A.co[k];
                if (j == i) continue;
                if (!std::binary_search(strong.begin(i), strong.end(i), j)) weak_sum += A.va[k];
            }
            const double denominator = diagonal + weak_sum;
            if (!std::isfinite(denominator) || std::abs(denominator) <= 1e-30) { failed = true; return; }
            // Sparse accumulator in first-touch order, entries start at 0.0.
            weights.clear();
            const auto accumulate = [&](uint32_t coarse, double contribution) {
                if (stamp[coarse] != i) {
                    stamp[coarse] = i;
                    slot_of[coarse] = static_cast<uint32_t>(weights.size());
                    weights.emplace_back(coarse, 0.0);
                }
                weights[slot_of[coarse]].second += contribution;
            };
            for (const uint32_t* p = strong.begin(i); p != strong.end(i); ++p)
                if (point[*p] == kCoarse) accumulate(coarse_index[*p], row_value(A, i, *p));
            for (const uint32_t* p = strong.begin(i); p != strong.end(i); ++p) {
                const uint32_t k = *p;
                if (point[k] != kFine) continue;
                double c_sum = 0.0;
                kc.clear();
                for (const uint32_t* q = strong.begin(k); q != strong.end(k); ++q) {
                    if (point[*q] == kCoarse) {
                        c_sum += row_value(A, k, *q);
                        kc.push_back(*q);
                    }
                }
                if (!std::isfinite(c_sum) || std::abs(c_sum) <= 1e-30) { failed = true; return; }
                const double aik = row_value(A, i, k);
                for (const uint32_t j : kc) {
                    const double akj = row_value(A, k, j);
                    accumulate(coarse_index[j], aik * akj / c_sum);
                }
            }
            std::sort(weights.begin(), weights.end(),
                      [](const auto& l, const auto& r) { return l.first < r.first; });
            double largest = -1.0;
            uint32_t aggregate = 0;
            const std::size_t start = val.size();
            for (const auto& [coarse, numerator] : weights) {
                const double weight = -numerator / denominator;
                if (!std::isfinite(weight)) { failed = true; return; }
                col.push_back(coarse);
                val.push_back(weight);
                if (std::abs(weight) > largest) {
                    largest = std::abs(weight);
                    aggregate = coarse;
                }
            }
            if (val.size() == start) { failed = true; return; }
            double row_sum = 0.0;
            for (std::size_t q = start; q < val.size(); ++q) row_sum += val[q];
            if (!std::isfinite(row_sum) || std::abs(row_sum) <= 1e-30) { failed = true; return; }
            for (std::size_t q = start; q < val.size(); ++q) {
                val[q] /= row_sum;
                if (!std::isfinite(val[q])) { failed = true; return; }
            }
            len.push_back(static_cast<uint32_t>(val.size() - start));
            agg.push_back(aggregate);
        }
    };
    if (workers == 1) {
        rows_job(0);
    } else {
        std::vector<std::thread> pool;
        for (int w = 0; w < workers; ++w) pool.emplace_back(rows_job, w);
        for (auto& t : pool) t.join();
    }
    if (failed) return false;
    if (profile_setup())
        std::fprintf(stderr, "[cfdxg setup] n=%lld strength %.3fs pass1 %.3fs pass2 %.3fs weights %.3fs\n",
                     static_cast<long long>(n), t_strength - t_start, t_pass1 - t_strength, t_pass2 - t_pass1,
                     tnow() - t_pass2);
    level.p_off.assign(static_cast<std::size_t>(n) + 1, 0);
    level.p_col.clear();
    level.p_val.clear();
    level.aggregate.clear();
    level.aggregate.reserve(static_cast<std::size_t>(n));
    int64_t row = 0;
    for (int w = 0; w < workers; ++w) {
        level.p_col.insert(level.p_col.end(), w_col[w].begin(), w_col[w].end());
        level.p_val.insert(level.p_val.end(), w_val[w].begin(), w_val[w].end());
        level.aggregate.insert(level.aggregate.end(), w_agg[w].begin(), w_agg[w].end());
        for (const uint32_t l : w_len[w]) {
            level.p_off[row + 1] = level.p_off[row] + l;
            ++row;
        }
    }
    return row == n;
}

// galerkin_csr_product.h:33-138 symbolic
bool galerkin_symbolic(const HostCsr& A, const AmgLevel& L, int64_t coarse_n, GalerkinPlan& plan) {
    const int64_t n = A.n;
    plan.n_fine = n;
    plan.n_coarse = coarse_n;
    plan.t_off.assign(static_cast<std::size_t>(coarse_n) + 1, 0);
    for (int64_t i = 0; i < n; ++i)
        for (uint32_t q = L.p_off[i]; q < L.p_off[i + 1]; ++q) {
            if (L.p_col[q] >= coarse_n || !std::isfinite(L.p_val[q])) return false;
            ++plan.t_off[L.p_col[q] + 1];
        }
    for (int64_t c = 0; c < coarse_n; ++c) plan.t_off[c + 1] += plan.t_off[c];
    plan.t_row.resize(plan.t_off[coarse_n]);
    plan.t_pos.resize(plan.t_off[coarse_n]);
    {
        std::vector<uint32_t> cursor(plan.t_off.begin(), plan.t_off.end() - 1);
        for (int64_t i = 0; i < n; ++i)
            for (uint32_t q = L.p_off[i]; q < L.p_off[i + 1]; ++q) {
                const uint32_t pos = cursor[L.p_col[q]]++;
                plan.t_row[pos] = static_cast<uint32_t>(i);
                plan.t_pos[pos] = q - L.p_off[i];
            }
    }
    // symbolic A*P rows, then P^T(AP) rows; both sorted unique
    // Rows are produced in chunks by a dynamic schedule; each chunk's rows
    // are stored separately and concatenated in chunk order.
    const auto build_rows = [coarse_n](int64_t rows, auto&& gather, std::vector<uint32_t>& off,
                                       std::vector<uint32_t>& col) {
        constexpr int64_t kChunk = 64;
        const int64_t n_chunks = (rows + kChunk - 1) / kChunk;
        std::vector<std::vector<uint32_t>> cc(n_chunks), cl(n_chunks);
        std::vector<std::vector<int64_t>> seen_by(host_threads());
        parallel_chunks(rows, kChunk, [&](int64_t b, int64_t e, int w) {
            auto& seen = seen_by[w];
            if (seen.size() != static_cast<std::size_t>(coarse_n)) seen.assign(static_cast<std::size_t>(coarse_n), -1);
            auto& outc = cc[b / kChunk];
            auto& outl = cl[b / kChunk];
            std::vector<uint32_t> scratch;
            for (int64_t r = b; r < e; ++r) {
                scratch.clear();
                gather(r, [&](uint32_t c) {
                    if (seen[c] != r) { seen[c] = r; scratch.push_back(c); }
                });
                std::sort(scratch.begin(), scratch.end());
                outc.insert(outc.end(), scratch.begin(), scratch.end());
                outl.push_back(static_cast<uint32_t>(scratch.size()));
            }
        });
        off.assign(static_cast<std::size_t>(rows) + 1, 0);
        col.clear();
        int64_t r = 0;
        uint64_t total = 0;
        for (int64_t c = 0; c < n_chunks; ++c) {
            col.insert(col.end(), cc[c].begin(), cc[c].end());
            for (const uint32_t l : cl[c]) {
                total += l;
                off[r + 1] = static_cast<uint32_t>(total);
                ++r;
            }
        }
        return total < std::numeric_limits<uint32_t>::max() && r == rows;
    };
    if (!build_rows(n, [&](int64_t i, auto&& push) {
            for (uint32_t k = A.ro[i]; k < A.ro[i + 1]; ++k) {
                const uint32_t j = A.co[k];
                for (uint32_t q = L.p_off[j]; q < L.p_off[j + 1]; ++q) push(L.p_col[q]);
            }
        }, plan.ap_off, plan.ap_col)) return false;
    if (!build_rows(coarse_n, [&](int64_t c, auto&& push) {
            for (uint32_t t = plan.t_off[c]; t < plan.t_off[c + 1]; ++t) {
                const uint32_t i = plan.t_row[t];
                for (uint32_t p = plan.ap_off[i]; p < plan.ap_off[i + 1]; ++p) push(plan.ap_col[p]);
            }
        }, plan.c_off, plan.c_col)) return false;
    return true;
}

// galerkin_csr_product.h:231-291 accumulate: same per-entry operation order.
// Column -> position lookups use per-thread marker arrays (the reference's
// `lookup` vector), reset after each row.
bool galerkin_accumulate(const HostCsr& A, const AmgLevel& L, const GalerkinPlan& plan,
                         std::vector<double>& c_values) {
    std::vector<double> ap(plan.ap_col.size(), 0.0);
    c_values.assign(plan.c_col.size(), 0.0);
    std::atomic<bool> failed{false};
    const int nw = host_threads();
    std::vector<std::vector<int64_t>> lookups(nw);
    const auto lookup_for = [&](int w) -> std::vector<int64_t>& {
        auto& v = lookups[w];
        if (v.size() != static_cast<std::size_t>(plan.n_coarse)) v.assign(static_cast<std::size_t>(plan.n_coarse), -1);
        return v;
    };
    parallel_chunks(plan.n_fine, 256, [&](int64_t b, int64_t e, int w) {
        auto& lookup = lookup_for(w);
        for (int64_t i = b; i < e && !failed.load(std::memory_order_relaxed); ++i) {
            for (uint32_t p = plan.ap_off[i]; p < plan.ap_off[i + 1]; ++p) lookup[plan.ap_col[p]] = p;
            for (uint32_t k = A.ro[i]; k < A.ro[i + 1]; ++k) {
                const uint32_t j = A.co[k];
                for (uint32_t q = L.p_off[j]; q < L.p_off[j + 1]; ++q) {
                    const int64_t pos = lookup[L.p_col[q]];
                    if (pos < 0 || !std::isfinite(L.p_val[q])) { failed = true; break; }
                    double& dst = ap[static_cast<std::size_t>(pos)];
                    dst += A.va[k] * L.p_val[q];
                    if (!std::isfinite(dst)) { failed = true; break; }
                }
            }
            for (uint32_t p = plan.ap_off[i]; p < plan.ap_off[i + 1]; ++p) lookup[plan.ap_col[p]] = -1;
        }
    });
    if (failed) return false;
    parallel_chunks(plan.n_coarse, 16, [&](int64_t b, int64_t e, int w) {
        auto& lookup = lookup_for(w);
        for (int64_t c = b; c < e && !failed.load(std::memory_order_relaxed); ++c) {
            for (uint32_t p = plan.c_off[c]; p < plan.c_off[c + 1]; ++p) lookup[plan.c_col[p]] = p;
            for (uint32_t t = plan.t_off[c]; t < plan.t_off[c + 1]; ++t) {
                const uint32_t i = plan.t_row[t];
                const uint32_t entry = plan.t_pos[t];
                const double weight = L.p_val[L.p_off[i] + entry];
                for (uint32_t p = plan.ap_off[i]; p < plan.ap_off[i + 1]; ++p) {
                    const int64_t pos = lookup[plan.ap_col[p]];
                    if (pos < 0) { failed = true; break; }
                    double& dst = c_values[static_cast<std::size_t>(pos)];
                    dst += weight * ap[p];
                    if (!std::isfinite(dst)) { failed = true; break; }
                }
            }
            for (uint32_t p = plan.c_off[c]; p < plan.c_off[c + 1]; ++p) lookup[plan.c_col[p]] = -1;
        }
    });
    return !failed;
}

// galerkin_csr_product.h:141-167 numeric (prune |v| <= 1e-30)
bool galerkin_numeric(const HostCsr& A, const AmgLevel& L, const GalerkinPlan& plan, HostCsr& out) {
    std::vector<double> cv;
    if (!galerkin_accumulate(A, L, plan, cv)) return false;
    out.n = plan.n_coarse;
    out.ro.assign(static_cast<std::size_t>(plan.n_coarse) + 1, 0);
    out.co.clear();
    out.va.clear();
    out.co.reserve(plan.c_col.size());
    out.va.reserve(plan.c_col.size());
    for (int64_t c = 0; c < plan.n_coarse; ++c) {
        for (uint32_t p = plan.c_off[c]; p < plan.c_off[c + 1]; ++p)
            if (std::abs(cv[p]) > 1e-30) {
                out.co.push_back(plan.c_col[p]);
                out.va.push_back(cv[p]);
            }
        out.ro[c + 1] = static_cast<uint32_t>(out.co.size());
    }
    return true;
}

// galerkin_csr_product.h:183-212 numeric_into_existing: the pruned graph must be unchanged
bool galerkin_numeric_into_existing(const HostCsr& A, const AmgLevel& L, const GalerkinPlan& plan,
                                    HostCsr& out) {
    if (out.n != plan.n_coarse) return false;
    std::vector<double> cv;
    if (!galerkin_accumulate(A, L, plan, cv)) return false;
    for (int64_t c = 0; c < plan.n_coarse; ++c) {
        uint32_t cursor = out.ro[c];
        for (uint32_t p = plan.c_off[c]; p < plan.c_off[c + 1]; ++p) {
            if (std::abs(cv[p]) > 1e-30) {
                if (cursor == out.ro[c + 1] || out.co[cursor] != plan.c_col[p]) return false;
                ++cursor;
            }
        }
        if (cursor != out.ro[c + 1]) return false;
    }
    std::size_t pos = 0;
    for (const double v : cv)
        if (std::abs(v) > 1e-30) out.va[pos++] = v;
    return true;
}

// amg_preconditioner.h:1322-1347
double normalized_gershgorin_upper_bound(const AmgLevel& level) {
    const HostCsr& A = level.A;
    const int64_t n = A.n;
    if (static_cast<int64_t>(level.inv_diag.size()) != n || n == 0)
        return std::numeric_limits<double>::infinity();
    std::vector<double> diagonal(static_cast<std::size_t>(n));
    for (int64_t i = 0; i < n; ++i) {
        if (!(level.inv_diag[i] > 0.0) || !std::isfinite(level.inv_diag[i]))
            return std::numeric_limits<double>::infinity();
        diagonal[i] = 1.0 / level.inv_diag[i];
        if (!(diagonal[i] > 0.0) || !std::isfinite(diagonal[i]))
            return std::numeric_limits<double>::infinity();
    }
    const int workers = workers_for(n, 8192);
    std::vector<double> part(workers, 0.0);
    std::vector<uint8_t> bad(workers, 0);
    parallel_blocks(n, [&](int64_t b, int64_t e, int w) {
        double ub = 0.0;
        for (int64_t i = b; i < e; ++i) {
            double row_sum = 0.0;
            for (uint32_t k = A.ro[i]; k < A.ro[i + 1]; ++k) {
                const uint32_t j = A.co[k];
                const double scale = std::sqrt(diagonal[i]) * std::sqrt(diagonal[j]);
                if (!(scale > 0.0) || !std::isfinite(scale)) { bad[w] = 1; return; }
                row_sum += std::abs(A.va[k]) / scale;
            }
            if (!std::isfinite(row_sum)) { bad[w] = 1; return; }
            ub = std::max(ub, row_sum);
        }
        part[w] = ub;
    }, 8192);
    double upper = 0.0;
    for (int w = 0; w < workers; ++w) {
        if (bad[w]) return std::numeric_limits<double>::infinity();
        upper = std::max(upper, part[w]);   // max is order-independent
    }
    return upper;
}

// amg_preconditioner.h:1362-1399
bool stable_omega(const std::vector<AmgLevel>& levels, double configured, double& omega,
                  std::string& reason) {
    if (levels.empty()) { reason = "empty AMG hierarchy"; return false; }
    double maximum_bound = 0.0;
    for (std::size_t l = 0; l < levels.size(); ++l) {
        const auto& L = levels[l];
        if (static_cast<int64_t>(L.inv_diag.size()) != L.A.n) {
            reason = "diagonal size mismatch at level " + std::to_string(l);
            return false;
        }
        for (int64_t r = 0; r < L.A.n; ++r)
            if (!(L.inv_diag[r] > 0.0) || !std::isfinite(L.inv_diag[r])) {
                reason = "Jacobi stability certificate requires positive finite diagonal; level=" +
                         std::to_string(l) + " row=" + std::to_string(r);
                return false;
            }
        const double bound = normalized_gershgorin_upper_bound(L);
        if (!std::isfinite(bound) || !(bound > 0.0)) {
            reason = "normalized Gershgorin bound is invalid at level " + std::to_string(l);
            return false;
        }
        maximum_bound = std::max(maximum_bound, bound);
    }
    if (!(maximum_bound > 0.0) || !std::isfinite(maximum_bound)) {
        reason = "maximum normalized Gershgorin bound is invalid";
        return false;
    }
    omega = std::min(configured, 1.8 / maximum_bound);
    if (!std::isfinite(omega) || !(omega > 0.0 && omega < 2.0)) {
        reason = "computed Jacobi damping is outside (0,2)";
        return false;
    }
    return true;
}

}  // namespace

// amg_preconditioner.h:1401-1421
bool build_inverse_diagonal(const HostCsr& A, std::vector<double>& inv_diag) {
    inv_diag.assign(static_cast<std::size_t>(A.n), 0.0);
    std::atomic<bool> ok{true};
    parallel_blocks(A.n, [&](int64_t b, int64_t e, int) {
        for (int64_t i = b; i < e; ++i) {
            double diagonal = 0.0;
            for (uint32_t k = A.ro[i]; k < A.ro[i + 1]; ++k)
                if (A.co[k] == i) diagonal += A.va[k];
            if (!std::isfinite(diagonal) || std::abs(diagonal) <= 1e-30) { ok = false; return; }
            inv_diag[i] = 1.0 / diagonal;
            if (!std::isfinite(inv_diag[i])) { ok = false; return; }
        }
    }, 16384);
    return ok;
}

// amg_preconditioner.h:1289-1308 has_constant_null_space: every |row sum|
// within 256 eps max(1, largest absolute row sum), rows summed in CSR order
bool has_constant_null_space(const HostCsr& A) {
    double matrix_scale = 0.0, residual_scale = 0.0;
    for (int64_t i = 0; i < A.n; ++i) {
        double row_sum = 0.0, row_norm = 0.0;
        for (uint32_t k = A.ro[i]; k < A.ro[i + 1]; ++k) {
            row_sum += A.va[k];
            row_norm += std::abs(A.va[k]);
        }
        matrix_scale = std::max(matrix_scale, row_norm);
        residual_scale = std::max(residual_scale, std::abs(row_sum));
    }
    const double tolerance = 256.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, matrix_scale);
    return std::isfinite(residual_scale) && residual_scale <= tolerance;
}

bool amg_setup(const HostCsr& A, const AmgOptions& opt, AmgHierarchy& out, std::string& error,
               const GalerkinHook* galerkin) {
    error.clear();
    if (A.n == 0 || !matrix_is_valid(A) || (opt.constant_null_space && !has_constant_null_space(A))) {
        error = "invalid finest matrix, dimensions, CSR, or null-space contract";
        return false;
    }
    std::vector<AmgLevel> levels;
    levels.emplace_back();
    levels.back().A = A;
    if (!build_inverse_diagonal(levels.back().A, levels.back().inv_diag)) {
        error = "invalid or zero diagonal on finest level";
        return false;
    }
    constexpr int64_t coarse_direct_limit = 16;
    while (levels.back().A.n > coarse_direct_limit &&
           static_cast<int>(levels.size()) < opt.max_levels) {
        AmgLevel& cur = levels.back();
        int64_t coarse_n = 0;
        AmgLevel staged;
        if (!build_cf_interpolation(cur.A, cur.inv_diag, opt.strength_threshold, staged, coarse_n)) {
            error = "Direct-CF interpolation construction failed at level " + std::to_string(levels.size() - 1);
            return false;
        }
        if (coarse_n == 0 || coarse_n >= cur.A.n) break;
        GalerkinPlan plan;
        HostCsr coarse;
        const double tg0 = tnow();
        bool sym_ok = true, num_ok = true;
        double tg1 = tg0;
        if (galerkin) {
            // the product on the device; the plan stays there for the refresh
            num_ok = (*galerkin)(static_cast<int>(levels.size() - 1), cur.A, staged, coarse_n, coarse);
            tg1 = tnow();
        } else {
            sym_ok = galerkin_symbolic(cur.A, staged, coarse_n, plan);
            tg1 = tnow();
            num_ok = sym_ok && galerkin_numeric(cur.A, staged, plan, coarse);
        }
        if (profile_setup())
            std::fprintf(stderr, "[cfdxg setup]   galerkin symbolic %.3fs numeric %.3fs -> %lld rows %lld nnz\n",
                         tg1 - tg0, tnow() - tg1, static_cast<long long>(coarse.n),
                         static_cast<long long>(coarse.co.size()));
        if (!sym_ok || !num_ok || !matrix_is_valid(coarse)) {
            error = "invalid Galerkin coarse matrix from level " + std::to_string(levels.size() - 1);
            return false;
        }
        AmgLevel next;
        next.A = std::move(coarse);
        if (!build_inverse_diagonal(next.A, next.inv_diag)) {
            error = "invalid or zero diagonal on coarse level " + std::to_string(levels.size());
            return false;
        }
        cur.p_off = std::move(staged.p_off);
        cur.p_col = std::move(staged.p_col);
        cur.p_val = std::move(staged.p_val);
        cur.aggregate = std::move(staged.aggregate);
        cur.plan = std::move(plan);
        levels.push_back(std::move(next));
    }
    double omega = opt.omega;
    std::string reason;
    if (stable_omega(levels, opt.omega, omega, reason)) {
        // certified damping
    } else if (opt.require_smoother_certificate) {
        error = reason;
        return false;
    } else {
        omega = opt.omega;
    }
    out.levels = std::move(levels);
    out.omega = omega;
    out.options = opt;
    out.error.clear();
    return true;
}

bool amg_update_values(AmgHierarchy& h, const HostCsr& A, std::string& error) {
    error.clear();
    if (h.levels.empty() || A.n != h.levels.front().A.n || A.ro != h.levels.front().A.ro ||
        A.co != h.levels.front().A.co || !matrix_is_valid(A) ||
        (h.options.constant_null_space && !has_constant_null_space(A))) {
        error = "native AMG numeric update requires an unchanged CSR pattern";
        return false;
    }
    std::vector<HostCsr> mats(h.levels.size());
    std::vector<std::vector<double>> diags(h.levels.size());
    mats[0] = A;
    if (!build_inverse_diagonal(mats[0], diags[0])) {
        error = "native AMG numeric update failed";
        return false;
    }
    for (std::size_t l = 0; l + 1 < h.levels.size(); ++l) {
        mats[l + 1] = h.levels[l + 1].A;
        AmgLevel view;
        view.p_off = h.levels[l].p_off;   // prolongation is unchanged
        view.p_col = h.levels[l].p_col;
        view.p_val = h.levels[l].p_val;
        if (!galerkin_numeric_into_existing(mats[l], view, h.levels[l].plan, mats[l + 1]) ||
            !matrix_is_valid(mats[l + 1]) || !build_inverse_diagonal(mats[l + 1], diags[l + 1])) {
            error = "native AMG numeric update failed";
            return false;
        }
    }
    std::vector<AmgLevel> staged_levels(h.levels.size());
    for (std::size_t l = 0; l < h.levels.size(); ++l) {
        staged_levels[l].A = mats[l];
        staged_levels[l].inv_diag = diags[l];
    }
    double omega = h.omega;
    std::string reason;
    if (!stable_omega(staged_levels, h.options.omega, omega, reason)) {
        if (h.options.require_smoother_certificate) {
            error = "native AMG numeric update failed";
            return false;
        }
        omega = h.omega;
    }
    for (std::size_t l = 0; l < h.levels.size(); ++l) {
        h.levels[l].A = std::move(mats[l]);
        h.levels[l].inv_diag = std::move(diags[l]);
    }
    h.omega = omega;
    return true;
}

}  // namespace cfdxg
