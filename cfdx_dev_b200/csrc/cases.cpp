// cases.cpp -- seeded synthetic meshes and fields for the benchmark configurations.
//
// The hex and Kuhn-tet generators number faces exactly as the reference's
// own mesh fixtures do (tests/validation/thermal_3d_mesh_v36.h:18-80 and
// tests/validation/radiation_tetrahedral_mesh_v52.h:14-92): cells are visited
// in lattice order, each cell's faces in the fixture's local order, a face gets
// the next id at its first occurrence, and the second visiting cell becomes its
// neighbour.  Random numbers come from std::mt19937_64 mapped to [0,1) by
// taking the top 53 bits, so every platform draws the same values.
#include "../../include/cfdxg.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <new>
#include <random>
#include <unordered_map>
#include <vector>

struct cfdxg_case {
    std::vector<double> px, py, pz;
    std::vector<int64_t> face_off{0}, face_vert, owner, neighbour, cell_off{0}, cell_face;
    std::vector<int32_t> patch_of_face, patch_types;
};

namespace {

inline double uniform01(std::mt19937_64& g) {
    return static_cast<double>(g() >> 11) * 0x1.0p-53;
}

struct V3 {
    double x, y, z;
    V3 operator+(const V3& o) const { return {x + o.x, y + o.y, z + o.z}; }
    V3 operator-(const V3& o) const { return {x - o.x, y - o.y, z - o.z}; }
    V3 operator*(double s) const { return {x * s, y * s, z * s}; }
    double dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
    V3 cross(const V3& o) const { return {y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x}; }
};

}  // namespace

extern "C" int cfdxg_case_hex(int64_t nx, int64_t ny, int64_t nz, cfdxg_case** out) {
    if (!out || nx < 1 || ny < 1 || nz < 1) return CFDXG_ERR_INVALID_ARGUMENT;
    auto* c = new (std::nothrow) cfdxg_case();
    if (!c) return CFDXG_ERR_OUT_OF_MEMORY;
    const auto pid = [&](int64_t i, int64_t j, int64_t k) { return (k * (ny + 1) + j) * (nx + 1) + i; };
    const int64_t np = (nx + 1) * (ny + 1) * (nz + 1);
    c->px.resize(np); c->py.resize(np); c->pz.resize(np);
    for (int64_t k = 0; k <= nz; ++k)
        for (int64_t j = 0; j <= ny; ++j)
            for (int64_t i = 0; i <= nx; ++i) {
                const int64_t p = pid(i, j, k);
                c->px[p] = double(i) / double(nx);
                c->py[p] = double(j) / double(ny);
                c->pz[p] = double(k) / double(nz);
            }
    // A face shared by two lattice cells is met first from the lower cell.
    // Interior faces of the structured lattice are found by direct index
    // instead of a map: the x-face between (i-1,j,k) and (i,j,k) is that
    // cell's east face, and likewise for y (north) and z (top).
    const int64_t ncell = nx * ny * nz;
    std::vector<int64_t> east(ncell, -1), north(ncell, -1), top(ncell, -1);
    std::vector<int32_t> kinds;
    c->owner.reserve(3 * ncell + nx * ny + ny * nz + nx * nz);
    const auto add = [&](std::array<int64_t, 4> v, int64_t cell, int kind) {
        const int64_t f = static_cast<int64_t>(c->owner.size());
        c->face_vert.insert(c->face_vert.end(), v.begin(), v.end());
        c->face_off.push_back(static_cast<int64_t>(c->face_vert.size()));
        c->owner.push_back(cell);
        c->neighbour.push_back(-1);
        kinds.push_back(kind);
        return f;
    };
    for (int64_t k = 0; k < nz; ++k)
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                const int64_t cell = (k * ny + j) * nx + i;
                const int64_t a = pid(i, j, k), b = pid(i + 1, j, k), d = pid(i, j + 1, k), e = pid(i + 1, j + 1, k);
                const int64_t A = pid(i, j, k + 1), B = pid(i + 1, j, k + 1), D = pid(i, j + 1, k + 1), E = pid(i + 1, j + 1, k + 1);
                int64_t fb, fw, fs;
                if (k > 0) { fb = top[cell - nx * ny]; c->neighbour[fb] = cell; }
                else fb = add({a, d, e, b}, cell, 4);
                const int64_t ft = add({A, B, E, D}, cell, 5);
                if (i > 0) { fw = east[cell - 1]; c->neighbour[fw] = cell; }
                else fw = add({d, a, A, D}, cell, 0);
                const int64_t fe = add({b, e, E, B}, cell, 1);
                if (j > 0) { fs = north[cell - nx]; c->neighbour[fs] = cell; }
                else fs = add({a, b, B, A}, cell, 2);
                const int64_t fn = add({e, d, D, E}, cell, 3);
                east[cell] = fe; north[cell] = fn; top[cell] = ft;
                for (const int64_t f : {fb, ft, fw, fe, fs, fn}) c->cell_face.push_back(f);
                c->cell_off.push_back(static_cast<int64_t>(c->cell_face.size()));
            }
    const int64_t nf = static_cast<int64_t>(c->owner.size());
    c->patch_of_face.assign(nf, -1);
    for (int64_t f = 0; f < nf; ++f)
        if (c->neighbour[f] < 0) c->patch_of_face[f] = kinds[f];
    c->patch_types.assign(6, 0);   // PatchType::WALL
    *out = c;
    return CFDXG_OK;
}

namespace {

// Kuhn split shared by the tet generator: (tests/validation/radiation_tetrahedral_mesh_v52.h:30-85)
int build_kuhn(cfdxg_case* c, int64_t n) {
    const int64_t nv = n + 1;
    const auto vid = [nv](int64_t i, int64_t j, int64_t k) { return i + nv * (j + nv * k); };
    static const int corners[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};
    static const int tets[6][4] = {{0,1,2,6},{0,1,5,6},{0,3,2,6},{0,3,7,6},{0,4,5,6},{0,4,7,6}};
    const int64_t ncell = 6 * n * n * n;
    std::unordered_map<uint64_t, int64_t> faces;
    faces.reserve(static_cast<std::size_t>(ncell * 2.2));
    c->owner.reserve(ncell * 2 + 12 * n * n);
    c->cell_face.reserve(4 * ncell);
    const auto point = [&](int64_t id) { return V3{c->px[id], c->py[id], c->pz[id]}; };
    for (int64_t k = 0; k < n; ++k)
        for (int64_t j = 0; j < n; ++j)
            for (int64_t i = 0; i < n; ++i) {
                int64_t p[8];
                for (int q = 0; q < 8; ++q) p[q] = vid(i + corners[q][0], j + corners[q][1], k + corners[q][2]);
                for (const auto& t : tets) {
                    const int64_t v[4] = {p[t[0]], p[t[1]], p[t[2]], p[t[3]]};
                    const V3 centre = (point(v[0]) + point(v[1]) + point(v[2]) + point(v[3])) * 0.25;
                    const int64_t sides[4][3] = {{v[0], v[1], v[2]}, {v[0], v[1], v[3]},
                                                 {v[0], v[2], v[3]}, {v[1], v[2], v[3]}};
                    const int64_t cid = static_cast<int64_t>(c->cell_off.size()) - 1;
                    for (const auto& side : sides) {
                        int64_t s[3] = {side[0], side[1], side[2]};
                        int64_t key3[3] = {s[0], s[1], s[2]};
                        std::sort(key3, key3 + 3);
                        const uint64_t key = (static_cast<uint64_t>(key3[0]) << 42) |
                                             (static_cast<uint64_t>(key3[1]) << 21) |
                                             static_cast<uint64_t>(key3[2]);
                        const auto it = faces.find(key);
                        if (it == faces.end()) {
                            const V3 A = point(s[0]), B = point(s[1]), C = point(s[2]);
                            if ((B - A).cross(C - A).dot((A + B + C) * (1. / 3.) - centre) < 0.)
                                std::swap(s[1], s[2]);
                            const int64_t fid = static_cast<int64_t>(c->owner.size());
                            c->face_vert.insert(c->face_vert.end(), {s[0], s[1], s[2]});
                            c->face_off.push_back(static_cast<int64_t>(c->face_vert.size()));
                            faces.emplace(key, fid);
                            c->owner.push_back(cid);
                            c->neighbour.push_back(-1);
                            c->cell_face.push_back(fid);
                        } else {
                            const int64_t fid = it->second;
                            if (c->neighbour[fid] != -1 || c->owner[fid] == cid) return CFDXG_ERR_GEOMETRY;
                            c->neighbour[fid] = cid;
                            c->cell_face.push_back(fid);
                        }
                    }
                    c->cell_off.push_back(static_cast<int64_t>(c->cell_face.size()));
                }
            }
    // Patches by the lattice plane every vertex of a boundary face lies on.
    const int64_t nf = static_cast<int64_t>(c->owner.size());
    c->patch_of_face.assign(nf, -1);
    for (int64_t f = 0; f < nf; ++f) {
        if (c->neighbour[f] >= 0) continue;
        int lo[3] = {1, 1, 1}, hi[3] = {1, 1, 1};
        for (int64_t q = c->face_off[f]; q < c->face_off[f + 1]; ++q) {
            const int64_t v = c->face_vert[q];
            const int64_t ijk[3] = {v % nv, (v / nv) % nv, v / (nv * nv)};
            for (int d = 0; d < 3; ++d) {
                if (ijk[d] != 0) lo[d] = 0;
                if (ijk[d] != n) hi[d] = 0;
            }
        }
        int patch = -1;
        for (int d = 0; d < 3 && patch < 0; ++d) {
            if (lo[d]) patch = 2 * d;
            else if (hi[d]) patch = 2 * d + 1;
        }
        if (patch < 0) return CFDXG_ERR_GEOMETRY;
        c->patch_of_face[f] = patch;
    }
    c->patch_types.assign(6, 0);   // PatchType::WALL
    return CFDXG_OK;
}

}  // namespace

extern "C" int cfdxg_case_tet(int64_t n, double jitter, uint64_t seed, cfdxg_case** out) {
    if (!out || n < 1 || n > 2000 || !(jitter >= 0.0 && jitter < 0.5)) return CFDXG_ERR_INVALID_ARGUMENT;
    auto* c = new (std::nothrow) cfdxg_case();
    if (!c) return CFDXG_ERR_OUT_OF_MEMORY;
    const int64_t nv = n + 1;
    const int64_t np = nv * nv * nv;
    c->px.resize(np); c->py.resize(np); c->pz.resize(np);
    std::mt19937_64 g(seed);
    const double h = 1.0 / double(n);
    for (int64_t k = 0; k <= n; ++k)
        for (int64_t j = 0; j <= n; ++j)
            for (int64_t i = 0; i <= n; ++i) {
                const int64_t id = i + nv * (j + nv * k);
                double x = double(i) / double(n), y = double(j) / double(n), z = double(k) / double(n);
                if (jitter > 0.0 && i > 0 && i < n && j > 0 && j < n && k > 0 && k < n) {
                    x += (2.0 * uniform01(g) - 1.0) * jitter * h;
                    y += (2.0 * uniform01(g) - 1.0) * jitter * h;
                    z += (2.0 * uniform01(g) - 1.0) * jitter * h;
                }
                c->px[id] = x; c->py[id] = y; c->pz[id] = z;
            }
    const int rc = build_kuhn(c, n);
    if (rc != CFDXG_OK) { delete c; return rc; }
    *out = c;
    return CFDXG_OK;
}

extern "C" int cfdxg_case_boundary_layer(int64_t nx, int64_t ny, int64_t nz, double lx, double lz,
                                         double dy0, double growth, double jitter, uint64_t seed,
                                         cfdxg_case** out) {
    if (!out || nx < 1 || ny < 1 || nz < 1 || !(lx > 0) || !(lz > 0) || !(dy0 > 0) || !(growth >= 1.0) ||
        !(jitter >= 0.0 && jitter < 0.5) || dy0 * ny >= 1.0)
        return CFDXG_ERR_INVALID_ARGUMENT;
    cfdxg_case* c = nullptr;
    int rc = cfdxg_case_hex(nx, ny, nz, &c);
    if (rc != CFDXG_OK) return rc;
    // y lines: dy_j = min(dy0 * growth^j, cap), cap chosen by bisection so the column sums to 1.
    const auto total = [&](double cap) {
        double s = 0.0, d = dy0;
        for (int64_t j = 0; j < ny; ++j) { s += std::min(d, cap); d *= growth; }
        return s;
    };
    double lo = dy0, hi = 1.0;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        (total(mid) < 1.0 ? lo : hi) = mid;
    }
    std::vector<double> ys(ny + 1, 0.0);
    {
        double d = dy0;
        for (int64_t j = 0; j < ny; ++j) { ys[j + 1] = ys[j] + std::min(d, hi); d *= growth; }
        for (int64_t j = 1; j <= ny; ++j) ys[j] /= ys[ny];
    }
    std::mt19937_64 g(seed);
    std::vector<double> xs(nx + 1), zs(nz + 1);
    for (int64_t i = 0; i <= nx; ++i) {
        xs[i] = lx * double(i) / double(nx);
        if (i > 0 && i < nx) xs[i] += (2.0 * uniform01(g) - 1.0) * jitter * lx / double(nx);
    }
    for (int64_t k = 0; k <= nz; ++k) {
        zs[k] = lz * double(k) / double(nz);
        if (k > 0 && k < nz) zs[k] += (2.0 * uniform01(g) - 1.0) * jitter * lz / double(nz);
    }
    for (int64_t k = 0; k <= nz; ++k)
        for (int64_t j = 0; j <= ny; ++j)
            for (int64_t i = 0; i <= nx; ++i) {
                const int64_t p = (k * (ny + 1) + j) * (nx + 1) + i;
                c->px[p] = xs[i]; c->py[p] = ys[j]; c->pz[p] = zs[k];
            }
    *out = c;
    return CFDXG_OK;
}

extern "C" int cfdxg_case_destroy(cfdxg_case* c) {
    delete c;
    return CFDXG_OK;
}

extern "C" int cfdxg_case_sizes(const cfdxg_case* c, int64_t* s) {
    if (!c || !s) return CFDXG_ERR_INVALID_ARGUMENT;
    s[0] = static_cast<int64_t>(c->px.size());
    s[1] = static_cast<int64_t>(c->owner.size());
    s[2] = static_cast<int64_t>(c->face_vert.size());
    s[3] = static_cast<int64_t>(c->cell_off.size()) - 1;
    s[4] = static_cast<int64_t>(c->cell_face.size());
    s[5] = static_cast<int64_t>(c->patch_types.size());
    return CFDXG_OK;
}

extern "C" int cfdxg_case_export(const cfdxg_case* c, double* px, double* py, double* pz,
                                 int64_t* fo, int64_t* fv, int64_t* owner, int64_t* neighbour,
                                 int64_t* co, int64_t* cf, int32_t* pf, int32_t* pt) {
    if (!c) return CFDXG_ERR_INVALID_ARGUMENT;
    const auto cp = [](auto* dst, const auto& v) {
        if (dst) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(px, c->px); cp(py, c->py); cp(pz, c->pz);
    cp(fo, c->face_off); cp(fv, c->face_vert); cp(owner, c->owner); cp(neighbour, c->neighbour);
    cp(co, c->cell_off); cp(cf, c->cell_face); cp(pf, c->patch_of_face); cp(pt, c->patch_types);
    return CFDXG_OK;
}

extern "C" int cfdxg_field_fourier(int64_t n, const double* centres, int32_t n_modes,
                                   double perturbation, uint64_t seed, double* u) {
    if (n < 0 || !centres || !u || n_modes < 0) return CFDXG_ERR_INVALID_ARGUMENT;
    constexpr double two_pi = 6.283185307179586476925286766559;
    std::mt19937_64 g(seed);
    struct Mode { V3 k, amp; double phase; };
    std::vector<Mode> modes;
    for (int32_t m = 0; m < n_modes; ++m) {
        int64_t ki[3];
        do {
            for (auto& q : ki) q = static_cast<int64_t>(std::floor(uniform01(g) * 7.0)) - 3;
        } while (ki[0] == 0 && ki[1] == 0 && ki[2] == 0);
        const V3 k{two_pi * double(ki[0]), two_pi * double(ki[1]), two_pi * double(ki[2])};
        const V3 a{2.0 * uniform01(g) - 1.0, 2.0 * uniform01(g) - 1.0, 2.0 * uniform01(g) - 1.0};
        const double k2 = k.dot(k);
        // a x k is orthogonal to k, so the mode is divergence-free.
        modes.push_back({k, a.cross(k) * (1.0 / k2), two_pi * uniform01(g)});
    }
    for (int64_t c = 0; c < n; ++c) {
        const V3 x{centres[c], centres[n + c], centres[2 * n + c]};
        V3 s{0.0, 0.0, 0.0};
        for (const auto& m : modes) s = s + m.amp * std::cos(m.k.dot(x) + m.phase);
        u[c] = s.x; u[n + c] = s.y; u[2 * n + c] = s.z;
    }
    for (int64_t q = 0; q < 3 * n; ++q) u[q] += (2.0 * uniform01(g) - 1.0) * perturbation;
    return CFDXG_OK;
}

extern "C" int cfdxg_field_random(int64_t n, int32_t kind, double lo, double hi, uint64_t seed,
                                  double* v) {
    if (n < 0 || !v) return CFDXG_ERR_INVALID_ARGUMENT;
    std::mt19937_64 g(seed);
    if (kind == 0) {
        if (!(lo > 0.0) || !(hi >= lo)) return CFDXG_ERR_INVALID_ARGUMENT;
        const double a = std::log(lo), b = std::log(hi);
        for (int64_t i = 0; i < n; ++i) v[i] = std::exp(a + (b - a) * uniform01(g));
    } else {
        for (int64_t i = 0; i < n; ++i) v[i] = lo + (hi - lo) * uniform01(g);
    }
    return CFDXG_OK;
}
