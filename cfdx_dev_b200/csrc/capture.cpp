// Linear-system replay files (".cfdxlin").
//
// Reads and writes the reference's single-rank CSR capture format
// (core/linalg/linear_system_capture.h:67-284) so that a pressure system that
// CFDX wrote during a run replays here bit for bit, and a system assembled
// here can be replayed by the reference's own tools
// (tools/diagnostics/cfdx_linear_replay.cpp).  The format is a text file:
//
//   CFDX_LINEAR_REPLAY_V1
//   problem null_space scaling          (decimal enum values)
//   rows cols nnz max_iterations        (decimal)
//   tolerance                           (hex IEEE-754 bit pattern)
//   row_offsets[0..rows]                (hex, one per line)
//   column value                        (hex, hex bits; nnz lines)
//   rhs initial_solution                (hex bits; rows lines)
//   checksum                            (hex FNV-1a over every word)
//
// The checksum is 64-bit FNV-1a over the little-endian bytes of every header
// number, offset, column and FP64 bit pattern, in file order (offset basis
// 14695981039346656037, prime 1099511628211: linear_system_capture.h:78-100,
// :138-160).  Writes go to "<path>.tmp" and are renamed into place, so a
// reader never sees a partial file.  Limits match the reference's bounded
// reader: rows <= 2,000,000, nnz <= 100,000,000, max_iterations <= 1e8.
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "cfdxg.h"

struct cfdxg_capture {
    int64_t n = 0;
    std::vector<int64_t> row_offsets, columns;
    std::vector<double> values, rhs, guess;
    cfdxg_capture_info info{};
};

namespace {

constexpr uint64_t kOffset = 14695981039346656037ULL;
constexpr uint64_t kPrime = 1099511628211ULL;
constexpr int64_t kMaxRows = 2000000;
constexpr int64_t kMaxNnz = 100000000;
constexpr int64_t kMaxIterations = 100000000;
// LinearProblemKind General..CoupledPressureVelocity, LinearScalingModel
// None..SymmetricDiagonal (core/linalg/linear_solver_models.h)
constexpr int kProblemMax = 5;
constexpr int kScalingMax = 4;

thread_local std::string g_error;

int fail(int code, const std::string& why) {
    g_error = why;
    return code;
}

uint64_t bits(double x) {
    uint64_t u;
    std::memcpy(&u, &x, sizeof u);
    return u;
}

double from_bits(uint64_t u) {
    double x;
    std::memcpy(&x, &u, sizeof x);
    return x;
}

struct Fnv {
    uint64_t h = kOffset;
    void add(uint64_t w) {
        for (int i = 0; i < 8; ++i) {
            h ^= (w >> (8 * i)) & 0xffu;
            h *= kPrime;
        }
    }
};

// Checks of linear_system_capture.h:117-137 (verify) and of the CSR
// invariants the reference's SparseMatrix holds (sparse_matrix.h:136-163,
// 256-276).  Returns an empty string when the system is valid.
std::string validate(int64_t n, const int64_t* ro, const int64_t* co, const double* va, const double* rhs,
                     const double* guess, const cfdxg_capture_info& info) {
    if (n <= 0) return "linear capture: invalid square finalized CSR";
    if (n > kMaxRows) return "linear capture: dimensions exceed replay format limits";
    if (ro[0] != 0) return "linear capture: invalid square finalized CSR";
    for (int64_t i = 0; i < n; ++i)
        if (ro[i + 1] < ro[i]) return "linear capture: invalid square finalized CSR";
    const int64_t nnz = ro[n];
    if (nnz > kMaxNnz) return "linear capture: dimensions exceed replay format limits";
    for (int64_t i = 0; i < n; ++i)
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k) {
            if (co[k] < 0 || co[k] >= n || !std::isfinite(va[k]) || (k > ro[i] && co[k] <= co[k - 1]))
                return "linear capture: invalid square finalized CSR";
        }
    if (info.problem < 0 || info.problem > kProblemMax || (info.null_space != 0 && info.null_space != 1) ||
        info.scaling < 0 || info.scaling > kScalingMax)
        return "linear capture: invalid solver metadata";
    if (info.max_iterations <= 0 || info.max_iterations > kMaxIterations || !(info.tolerance > 0.0) ||
        !std::isfinite(info.tolerance))
        return "linear capture: invalid iteration controls";
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(rhs[i]) || !std::isfinite(guess[i])) return "linear capture: nonfinite vector";
    return {};
}

uint64_t fingerprint(int64_t n, const int64_t* ro, const int64_t* co, const double* va, const double* rhs,
                     const double* guess, const cfdxg_capture_info& info) {
    Fnv f;
    const int64_t nnz = ro[n];
    f.add(uint64_t(n));
    f.add(uint64_t(n));
    f.add(uint64_t(nnz));
    f.add(uint64_t(info.problem));
    f.add(uint64_t(info.null_space));
    f.add(uint64_t(info.scaling));
    f.add(uint64_t(info.max_iterations));
    f.add(bits(info.tolerance));
    for (int64_t i = 0; i <= n; ++i) f.add(uint64_t(ro[i]));
    for (int64_t k = 0; k < nnz; ++k) {
        f.add(uint64_t(co[k]));
        f.add(bits(va[k]));
    }
    for (int64_t i = 0; i < n; ++i) {
        f.add(bits(rhs[i]));
        f.add(bits(guess[i]));
    }
    return f.h;
}

// Whitespace-separated tokens from a buffered file, as std::istream's >>.
class Tokens {
public:
    explicit Tokens(FILE* f) : f_(f), buf_(1 << 20) {}
    // Next token; false at end of file.
    bool next(std::string& tok) {
        tok.clear();
        int c;
        while ((c = get()) != EOF && is_space(c)) {}
        if (c == EOF) return false;
        do {
            tok.push_back(char(c));
        } while ((c = get()) != EOF && !is_space(c));
        return true;
    }
    bool next_hex(uint64_t& w) {
        std::string t;
        if (!next(t)) return false;
        size_t i = 0;
        if (t.size() > 2 && t[0] == '0' && (t[1] == 'x' || t[1] == 'X')) i = 2;
        if (i == t.size()) return false;
        uint64_t v = 0;
        for (; i < t.size(); ++i) {
            const char ch = t[i];
            int d;
            if (ch >= '0' && ch <= '9') d = ch - '0';
            else if (ch >= 'a' && ch <= 'f') d = ch - 'a' + 10;
            else if (ch >= 'A' && ch <= 'F') d = ch - 'A' + 10;
            else return false;
            if (v >> 60) return false;  // more than 64 bits
            v = (v << 4) | uint64_t(d);
        }
        w = v;
        return true;
    }
    bool next_dec(int64_t& v, bool allow_negative) {
        std::string t;
        if (!next(t) || t.empty()) return false;
        size_t i = 0;
        bool neg = false;
        if (t[0] == '+' || t[0] == '-') {
            neg = t[0] == '-';
            if (neg && !allow_negative) return false;
            i = 1;
        }
        if (i == t.size()) return false;
        uint64_t u = 0;
        for (; i < t.size(); ++i) {
            if (t[i] < '0' || t[i] > '9') return false;
            if (u > (uint64_t(INT64_MAX) - 9) / 10) return false;
            u = u * 10 + uint64_t(t[i] - '0');
        }
        v = neg ? -int64_t(u) : int64_t(u);
        return true;
    }

private:
    static bool is_space(int c) { return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }
    int get() {
        if (pos_ == len_) {
            len_ = std::fread(buf_.data(), 1, buf_.size(), f_);
            pos_ = 0;
            if (len_ == 0) return EOF;
        }
        return static_cast<unsigned char>(buf_[pos_++]);
    }
    FILE* f_;
    std::vector<char> buf_;
    size_t pos_ = 0, len_ = 0;
};

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

int read_capture(const char* path, cfdxg_capture& c) {
    File file;
    file.f = std::fopen(path, "rb");
    if (!file.f) return fail(CFDXG_ERR_IO, "linear capture: cannot open file");
    Tokens in(file.f);
    std::string header;
    if (!in.next(header) || header != "CFDX_LINEAR_REPLAY_V1")
        return fail(CFDXG_ERR_IO, "linear capture: unsupported format");
    int64_t problem, null_space, scaling, rows, cols, nnz, iterations;
    if (!in.next_dec(problem, true) || !in.next_dec(null_space, true) || !in.next_dec(scaling, true) ||
        !in.next_dec(rows, false) || !in.next_dec(cols, false) || !in.next_dec(nnz, false) ||
        !in.next_dec(iterations, false))
        return fail(CFDXG_ERR_IO, "linear capture: invalid header");
    if (problem < 0 || problem > kProblemMax || (null_space != 0 && null_space != 1) || scaling < 0 ||
        scaling > kScalingMax)
        return fail(CFDXG_ERR_IO, "linear capture: invalid solver metadata");
    // bounded before anything is allocated
    if (rows <= 0 || rows != cols || rows > kMaxRows || nnz > kMaxNnz)
        return fail(CFDXG_ERR_IO, "linear capture: dimensions exceed supported limits");
    uint64_t w;
    if (!in.next_hex(w)) return fail(CFDXG_ERR_IO, "linear capture: truncated or invalid hexadecimal number");
    c.info = cfdxg_capture_info{};
    c.info.problem = int32_t(problem);
    c.info.null_space = int32_t(null_space);
    c.info.scaling = int32_t(scaling);
    c.info.n = rows;
    c.info.nnz = nnz;
    c.info.max_iterations = iterations;
    c.info.tolerance = from_bits(w);
    c.n = rows;
    c.row_offsets.assign(size_t(rows) + 1, 0);
    c.columns.assign(size_t(nnz), 0);
    c.values.assign(size_t(nnz), 0.0);
    c.rhs.assign(size_t(rows), 0.0);
    c.guess.assign(size_t(rows), 0.0);
    const char* trunc = "linear capture: truncated or invalid hexadecimal number";
    for (auto& v : c.row_offsets) {
        if (!in.next_hex(w)) return fail(CFDXG_ERR_IO, trunc);
        if (w > 0xffffffffULL) return fail(CFDXG_ERR_IO, "linear capture: overflowing CSR offset");
        v = int64_t(w);
    }
    for (int64_t k = 0; k < nnz; ++k) {
        if (!in.next_hex(w)) return fail(CFDXG_ERR_IO, trunc);
        if (w >= uint64_t(cols)) return fail(CFDXG_ERR_IO, "linear capture: invalid CSR column");
        c.columns[k] = int64_t(w);
        if (!in.next_hex(w)) return fail(CFDXG_ERR_IO, trunc);
        c.values[k] = from_bits(w);
    }
    for (int64_t i = 0; i < rows; ++i) {
        if (!in.next_hex(w)) return fail(CFDXG_ERR_IO, trunc);
        c.rhs[i] = from_bits(w);
        if (!in.next_hex(w)) return fail(CFDXG_ERR_IO, trunc);
        c.guess[i] = from_bits(w);
    }
    uint64_t expected;
    if (!in.next_hex(expected)) return fail(CFDXG_ERR_IO, trunc);
    std::string trailing;
    if (in.next(trailing)) return fail(CFDXG_ERR_IO, "linear capture: unexpected trailing data");
    if (c.row_offsets[rows] != nnz) return fail(CFDXG_ERR_IO, "linear capture: invalid CSR offsets");
    const std::string why = validate(rows, c.row_offsets.data(), c.columns.data(), c.values.data(), c.rhs.data(),
                                     c.guess.data(), c.info);
    if (!why.empty()) return fail(CFDXG_ERR_IO, why);
    if (fingerprint(rows, c.row_offsets.data(), c.columns.data(), c.values.data(), c.rhs.data(), c.guess.data(),
                    c.info) != expected)
        return fail(CFDXG_ERR_IO, "linear capture: checksum mismatch");
    c.info.checksum = expected;
    return CFDXG_OK;
}

bool put(FILE* f, const char* fmt, unsigned long long a) { return std::fprintf(f, fmt, a) > 0; }

bool put2(FILE* f, unsigned long long a, unsigned long long b) { return std::fprintf(f, "%llx %llx\n", a, b) > 0; }

}  // namespace

extern "C" {

int cfdxg_capture_read(const char* path, cfdxg_capture** out, cfdxg_capture_info* info) {
    if (!path || !out) return fail(CFDXG_ERR_INVALID_ARGUMENT, "linear capture: null argument");
    *out = nullptr;
    auto* c = new (std::nothrow) cfdxg_capture;
    if (!c) return fail(CFDXG_ERR_OUT_OF_MEMORY, "linear capture: out of host memory");
    int rc;
    try {
        rc = read_capture(path, *c);
    } catch (const std::bad_alloc&) {
        rc = fail(CFDXG_ERR_OUT_OF_MEMORY, "linear capture: out of host memory");
    }
    if (rc != CFDXG_OK) {
        delete c;
        return rc;
    }
    if (info) *info = c->info;
    *out = c;
    g_error.clear();
    return CFDXG_OK;
}

int cfdxg_capture_export(const cfdxg_capture* c, int64_t* row_offsets, int64_t* columns, double* values,
                         double* rhs, double* initial_solution) {
    if (!c) return fail(CFDXG_ERR_INVALID_ARGUMENT, "linear capture: null handle");
    if (row_offsets) std::memcpy(row_offsets, c->row_offsets.data(), c->row_offsets.size() * sizeof(int64_t));
    if (columns) std::memcpy(columns, c->columns.data(), c->columns.size() * sizeof(int64_t));
    if (values) std::memcpy(values, c->values.data(), c->values.size() * sizeof(double));
    if (rhs) std::memcpy(rhs, c->rhs.data(), c->rhs.size() * sizeof(double));
    if (initial_solution) std::memcpy(initial_solution, c->guess.data(), c->guess.size() * sizeof(double));
    return CFDXG_OK;
}

int cfdxg_capture_write(const char* path, int64_t n, const int64_t* ro, const int64_t* co, const double* va,
                        const double* rhs, const double* guess, cfdxg_capture_info* info) {
    if (!path || !*path) return fail(CFDXG_ERR_INVALID_ARGUMENT, "linear capture: empty path");
    if (!info || !rhs || !guess || !ro || (n > 0 && ro[n] > 0 && (!co || !va)))
        return fail(CFDXG_ERR_INVALID_ARGUMENT, "linear capture: null argument");
    if (n <= 0) return fail(CFDXG_ERR_INVALID_ARGUMENT, "linear capture: invalid square finalized CSR");
    if (n > kMaxRows) return fail(CFDXG_ERR_INVALID_ARGUMENT, "linear capture: dimensions exceed replay format limits");
    const std::string why = validate(n, ro, co, va, rhs, guess, *info);
    if (!why.empty()) return fail(CFDXG_ERR_INVALID_ARGUMENT, why);
    const int64_t nnz = ro[n];
    const uint64_t fp = fingerprint(n, ro, co, va, rhs, guess, *info);
    const std::string tmp = std::string(path) + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return fail(CFDXG_ERR_IO, "linear capture: cannot create temporary file");
    bool ok = std::fprintf(f, "CFDX_LINEAR_REPLAY_V1\n%d %d %d\n%lld %lld %lld %lld\n", int(info->problem),
                           int(info->null_space), int(info->scaling), (long long)n, (long long)n, (long long)nnz,
                           (long long)info->max_iterations) > 0;
    ok = ok && put(f, "%llx\n", bits(info->tolerance));
    for (int64_t i = 0; ok && i <= n; ++i) ok = put(f, "%llx\n", (unsigned long long)ro[i]);
    for (int64_t k = 0; ok && k < nnz; ++k) ok = put2(f, (unsigned long long)co[k], bits(va[k]));
    for (int64_t i = 0; ok && i < n; ++i) ok = put2(f, bits(rhs[i]), bits(guess[i]));
    ok = ok && put(f, "%llx\n", fp);
    ok = (std::fflush(f) == 0) && ok;
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) {
        std::remove(tmp.c_str());
        return fail(CFDXG_ERR_IO, ok ? "linear capture: disk close failed" : "linear capture: disk write failed");
    }
    if (std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        return fail(CFDXG_ERR_IO, "linear capture: atomic rename failed");
    }
    info->n = n;
    info->nnz = nnz;
    info->checksum = fp;
    g_error.clear();
    return CFDXG_OK;
}

int cfdxg_capture_destroy(cfdxg_capture* c) {
    delete c;
    return CFDXG_OK;
}

const char* cfdxg_capture_last_error(void) { return g_error.c_str(); }

}  // extern "C"
