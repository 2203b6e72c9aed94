/*
 * cfdx_oracle.c -- plain-C restatement of the CFDX pressure-correction hot
 * path (declarations and reference citations in cfdx_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY.  The loops follow the reference's own loop
 * structure (face-ordered where the reference loops over faces, cell-ordered
 * where it loops over cells), so every sum is formed in the reference's order.
 */
#include "cfdx_oracle.h"

#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static __thread char g_error[256];

const char* co_last_error(void) { return g_error; }

static int fail(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof g_error, fmt, ap);
    va_end(ap);
    return -1;
}

/* ---------------------------------------------------------------- vectors */

typedef struct {
    double x, y, z;
} v3;

static inline v3 mk(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 ld(const double* a, int64_t n, int64_t i) { return mk(a[i], a[n + i], a[2 * n + i]); }
static inline void st(double* a, int64_t n, int64_t i, v3 v) { a[i] = v.x; a[n + i] = v.y; a[2 * n + i] = v.z; }
static inline v3 vsub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vadd(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vscale(v3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double vmag(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

/* --------------------------------------------------------------- geometry */

typedef struct {
    int64_t nf, nc;
    double *fc, *sf, *cc, *cv;   /* SoA, owned */
} geom_t;

static void geom_free(geom_t* g) {
    free(g->fc); free(g->sf); free(g->cc); free(g->cv);
    memset(g, 0, sizeof *g);
}

/* compute_cell_geometry_oriented (cell_geometry.h:121-147) feeding
 * compute_cell_geometry (:49-118): Sf signed by ownership, area-weighted
 * centre, signed pyramid volume (2-D flat cells: summed face areas). */
static int cell_geometry(const co_mesh_t* m, int64_t c, const double* fc, const double* sf, v3* centre,
                         double* volume) {
    const int64_t b = m->cell_offsets[c], e = m->cell_offsets[c + 1];
    if (e == b) return fail("cell %lld has no faces", (long long)c);
    int is_2d = 1;
    for (int64_t k = b; k < e; ++k) {
        const int64_t f = m->cell_faces[k];
        if (m->owner[f] != c && m->neighbour[f] != c) return fail("face %lld not attached to cell %lld", (long long)f, (long long)c);
        v3 s = ld(sf, m->n_faces, f);
        if (m->owner[f] != c) s = vscale(s, -1.0);
        if (fabs(fc[2 * m->n_faces + f]) > 1e-12) { is_2d = 0; break; }
        if (fabs(s.x) > 1e-12 || fabs(s.y) > 1e-12) { is_2d = 0; break; }
    }
    v3 ws = mk(0.0, 0.0, 0.0);
    double total = 0.0;
    for (int64_t k = b; k < e; ++k) {
        const int64_t f = m->cell_faces[k];
        v3 s = ld(sf, m->n_faces, f);
        if (m->owner[f] != c) s = vscale(s, -1.0);
        const double a = vmag(s);
        ws = vadd(ws, vscale(ld(fc, m->n_faces, f), a));
        total += a;
    }
    const v3 cen = total > 0.0 ? vscale(ws, 1.0 / total) : mk(0.0, 0.0, 0.0);
    double sv = 0.0;
    for (int64_t k = b; k < e; ++k) {
        const int64_t f = m->cell_faces[k];
        v3 s = ld(sf, m->n_faces, f);
        if (m->owner[f] != c) s = vscale(s, -1.0);
        const double area = vmag(s);
        if (!(area > 0.0)) return fail("degenerate face %lld", (long long)f);
        if (is_2d) sv += area;
        else sv += vdot(vsub(ld(fc, m->n_faces, f), cen), s);
    }
    if (!is_2d) sv /= 3.0;
    *centre = cen;
    *volume = fabs(sv);
    return 0;
}

static int build_geometry(const co_mesh_t* m, geom_t* g) {
    const int64_t nf = m->n_faces, nc = m->n_cells;
    memset(g, 0, sizeof *g);
    g->nf = nf; g->nc = nc;
    g->fc = malloc(sizeof(double) * 3 * nf);
    g->sf = malloc(sizeof(double) * 3 * nf);
    g->cc = malloc(sizeof(double) * 3 * nc);
    g->cv = malloc(sizeof(double) * nc);
    if (!g->fc || !g->sf || !g->cc || !g->cv) { geom_free(g); return fail("out of memory"); }
    /* face_geometry.h:50-90: triangle fan around the first vertex */
    for (int64_t f = 0; f < nf; ++f) {
        const int64_t off = m->face_offsets[f], nv = m->face_offsets[f + 1] - off;
        if (nv < 3) { geom_free(g); return fail("face %lld has fewer than 3 vertices", (long long)f); }
        const int64_t v0 = m->face_vertices[off];
        const v3 p0 = mk(m->px[v0], m->py[v0], m->pz[v0]);
        v3 S = mk(0.0, 0.0, 0.0), awc = mk(0.0, 0.0, 0.0);
        double tri_area = 0.0;
        for (int64_t k = 1; k + 1 < nv; ++k) {
            const int64_t va = m->face_vertices[off + k], vb = m->face_vertices[off + k + 1];
            const v3 pa = mk(m->px[va], m->py[va], m->pz[va]);
            const v3 pb = mk(m->px[vb], m->py[vb], m->pz[vb]);
            const v3 tS = vscale(vcross(vsub(pa, p0), vsub(pb, p0)), 0.5);
            const double ta = vmag(tS);
            S = vadd(S, tS);
            awc = vadd(awc, vscale(vadd(vadd(p0, pa), pb), ta / 3.0));
            tri_area += ta;
        }
        const double area = vmag(S);
        if (!(tri_area > 0.0) || !(area > 0.0) || !isfinite(area)) {
            geom_free(g);
            return fail("degenerate face %lld", (long long)f);
        }
        st(g->fc, nf, f, vscale(awc, 1.0 / tri_area));
        st(g->sf, nf, f, S);
    }
    /* finite_volume_transport.h:115-127 first cell pass */
    for (int64_t c = 0; c < nc; ++c) {
        v3 cen;
        double vol;
        if (cell_geometry(m, c, g->fc, g->sf, &cen, &vol)) { geom_free(g); return -1; }
        if (!(vol > 0.0) || !isfinite(vol)) { geom_free(g); return fail("non-positive cell volume %lld", (long long)c); }
        st(g->cc, nc, c, cen);
        g->cv[c] = vol;
    }
    /* :129-151 ensure_face_orientation (face_geometry.h:115-127) */
    for (int64_t f = 0; f < nf; ++f) {
        const int64_t o = m->owner[f], n = m->neighbour[f];
        const v3 co = ld(g->cc, nc, o);
        const v3 d = n >= 0 ? vsub(ld(g->cc, nc, n), co) : vsub(ld(g->fc, nf, f), co);
        const v3 s = ld(g->sf, nf, f);
        if (vdot(s, d) < 0.0) st(g->sf, nf, f, vscale(s, -1.0));
    }
    /* :153-165 second cell pass with owner-oriented face vectors */
    for (int64_t c = 0; c < nc; ++c) {
        v3 cen;
        double vol;
        if (cell_geometry(m, c, g->fc, g->sf, &cen, &vol)) { geom_free(g); return -1; }
        if (!(vol > 0.0) || !isfinite(vol)) { geom_free(g); return fail("non-positive cell volume %lld", (long long)c); }
        st(g->cc, nc, c, cen);
        g->cv[c] = vol;
    }
    return 0;
}

int co_fv_geometry(const co_mesh_t* m, double* fc, double* sf, double* cc, double* cv) {
    geom_t g;
    if (build_geometry(m, &g)) return -1;
    memcpy(fc, g.fc, sizeof(double) * 3 * g.nf);
    memcpy(sf, g.sf, sizeof(double) * 3 * g.nf);
    memcpy(cc, g.cc, sizeof(double) * 3 * g.nc);
    memcpy(cv, g.cv, sizeof(double) * g.nc);
    geom_free(&g);
    return 0;
}

/* ------------------------------------------------------ boundary patches */

static int patch_type(const co_mesh_t* m, int64_t f) {
    const int32_t p = m->patch_of_face ? m->patch_of_face[f] : -1;
    if (p < 0 || p >= m->n_patches || !m->patch_types) return -1;
    return m->patch_types[p];
}

static int fixed_value(const co_mesh_t* m, const int32_t* fixed, const double* value, int64_t f, double* v) {
    const int32_t p = m->patch_of_face ? m->patch_of_face[f] : -1;
    if (p < 0 || p >= m->n_patches || !fixed || !fixed[p]) return 0;
    *v = value ? value[p] : 0.0;
    return 1;
}

/* -------------------------------------------------------- gauss gradient */

static int gauss_gradient(const co_mesh_t* m, const geom_t* g, const double* p, const int32_t* fixed,
                          const double* value, double* grad) {
    const int64_t nc = m->n_cells, nf = m->n_faces;
    for (int64_t c = 0; c < nc; ++c) {
        v3 sum = mk(0.0, 0.0, 0.0);
        for (int64_t k = m->cell_offsets[c]; k < m->cell_offsets[c + 1]; ++k) {
            const int64_t f = m->cell_faces[k];
            const int own = m->owner[f] == c;
            v3 S = ld(g->sf, nf, f);
            if (!own) S = vscale(S, -1.0);
            double vf = p[c];
            if (m->neighbour[f] >= 0) {
                const int64_t other = own ? m->neighbour[f] : m->owner[f];
                const v3 fcv = ld(g->fc, nf, f);
                const double dc = vmag(vsub(fcv, ld(g->cc, nc, c)));
                const double dn = vmag(vsub(ld(g->cc, nc, other), fcv));
                if (!(dc + dn > 0.0)) return fail("degenerate face distance at face %lld", (long long)f);
                const double w = dn / (dc + dn);
                vf = w * p[c] + (1.0 - w) * p[other];
            } else {
                if (patch_type(m, f) == CO_PATCH_EMPTY) continue;
                double v;
                if (fixed_value(m, fixed, value, f, &v)) vf = v;
            }
            sum = vadd(sum, vscale(S, vf));
        }
        const double invV = 1.0 / g->cv[c];
        const v3 gc = mk(sum.x * invV, sum.y * invV, sum.z * invV);
        if (!isfinite(gc.x) || !isfinite(gc.y) || !isfinite(gc.z)) return fail("non-finite gradient at cell %lld", (long long)c);
        st(grad, nc, c, gc);
    }
    return 0;
}

int co_gauss_gradient(const co_mesh_t* m, const double* p, const int32_t* fixed, const double* value,
                      double* grad) {
    geom_t g;
    if (build_geometry(m, &g)) return -1;
    const int rc = gauss_gradient(m, &g, p, fixed, value, grad);
    geom_free(&g);
    return rc;
}

/* ------------------------------------------- pressure-correction face terms */

/* :1914-1935 pressure_face_orthogonal_coefficient */
static int orthogonal_coefficient(v3 S, v3 dvec, v3 dau, double* out) {
    const double d = vmag(dvec), area = vmag(S);
    if (!(d > 0.0) || !isfinite(d) || !(area > 0.0) || !isfinite(area)) return fail("invalid face geometry");
    const v3 e = mk(dvec.x / d, dvec.y / d, dvec.z / d);
    const double oa = vdot(S, e);
    if (!(oa > 0.0) || !isfinite(oa)) return fail("face orientation inconsistent with the cell-centre direction");
    const double rfn = dau.x * e.x * e.x + dau.y * e.y * e.y + dau.z * e.z * e.z;
    *out = rfn * oa / d;
    if (!isfinite(*out)) return fail("non-finite face coefficient");
    return 0;
}

/* :1941-1965 pressure_face_nonorthogonal_flux */
static int nonorthogonal_flux(v3 S, v3 dvec, v3 dau, v3 gp, double* out) {
    const double d = vmag(dvec);
    if (!(d > 0.0) || !isfinite(d)) return fail("invalid centre distance");
    const v3 e = mk(dvec.x / d, dvec.y / d, dvec.z / d);
    const double oa = vdot(S, e);
    const double rfn = dau.x * e.x * e.x + dau.y * e.y * e.y + dau.z * e.z * e.z;
    const double full = dau.x * gp.x * S.x + dau.y * gp.y * S.y + dau.z * gp.z * S.z;
    const double implicit_flux = rfn * vdot(gp, e) * oa;
    *out = full - implicit_flux;
    if (!isfinite(*out)) return fail("non-finite deferred flux");
    return 0;
}

/* the face-interpolated V*rAU of :1991-1999 and :6491-6499 (wn = 0.5: no projected interpolation) */
static v3 face_dau(const geom_t* g, const double* rau, int64_t o, int64_t n) {
    const int64_t nc = g->nc;
    const double wn = 0.5, wo = 1.0 - wn;
    return mk(wo * g->cv[o] * rau[o] + wn * g->cv[n] * rau[n],
              wo * g->cv[o] * rau[nc + o] + wn * g->cv[n] * rau[nc + n],
              wo * g->cv[o] * rau[2 * nc + o] + wn * g->cv[n] * rau[2 * nc + n]);
}

/* :1967-2024 rhie_chow_pressure_flux_internal (interior face) */
static int rc_internal(const co_mesh_t* m, const geom_t* g, int64_t f, const double* p, const double* grad,
                       const double* rau, double rho, double* out) {
    const int64_t nc = m->n_cells, o = m->owner[f], n = m->neighbour[f];
    const v3 S = ld(g->sf, m->n_faces, f);
    const double area = vmag(S);
    if (!(area > 0.0) || !isfinite(area)) return fail("degenerate face %lld", (long long)f);
    const v3 dvec = vsub(ld(g->cc, nc, n), ld(g->cc, nc, o));
    const double d = vmag(dvec);
    if (!(d > 0.0) || !isfinite(d)) return fail("degenerate centre distance at face %lld", (long long)f);
    const double wn = 0.5, wo = 1.0 - wn;
    const v3 dau = face_dau(g, rau, o, n);
    const v3 gp = mk(wo * grad[o] + wn * grad[n], wo * grad[nc + o] + wn * grad[nc + n],
                     wo * grad[2 * nc + o] + wn * grad[2 * nc + n]);
    double ic, no;
    if (orthogonal_coefficient(S, dvec, dau, &ic) || nonorthogonal_flux(S, dvec, dau, gp, &no)) return -1;
    *out = rho * (ic * (p[n] - p[o]) + no);
    return 0;
}

/* :1842-1905 make_mass_flux with zero-gradient velocity patches */
static double mass_flux(const co_mesh_t* m, const geom_t* g, int64_t f, const double* U, double rho) {
    const int64_t nc = m->n_cells, o = m->owner[f], n = m->neighbour[f];
    v3 Uf = ld(U, nc, o);
    if (n >= 0) {
        const double wn = 0.5;
        Uf = vadd(vscale(Uf, 1.0 - wn), vscale(ld(U, nc, n), wn));
    } else {
        const int t = patch_type(m, f);
        if (t == CO_PATCH_EMPTY || t == CO_PATCH_SYMMETRY) return 0.0;
    }
    return rho * vdot(Uf, ld(g->sf, m->n_faces, f));
}

/* fixed-pressure boundary face: implicit coefficient and source (:8130-8175) */
static int fixed_boundary(const co_mesh_t* m, const geom_t* g, int64_t f, const double* p, const double* grad,
                          const double* rau, double rho, double value, double* coeff, double* source) {
    const int64_t nc = m->n_cells, o = m->owner[f];
    const v3 dvec = vsub(ld(g->fc, m->n_faces, f), ld(g->cc, nc, o));
    const v3 S = ld(g->sf, m->n_faces, f);
    const v3 dau = mk(g->cv[o] * rau[o], g->cv[o] * rau[nc + o], g->cv[o] * rau[2 * nc + o]);
    double bc, deferred;
    if (orthogonal_coefficient(S, dvec, dau, &bc)) return -1;
    if (nonorthogonal_flux(S, dvec, dau, ld(grad, nc, o), &deferred)) return -1;
    *coeff = bc;
    *source = rho * (bc * (value - p[o]) + deferred);
    return 0;
}

/* ---------------------------------------------------------- CSR pattern */

typedef struct {
    int64_t n, nnz;
    int64_t *ro, *co;
    double* va;
} csr_t;

static int cmp_i64(const void* a, const void* b) {
    const int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return (x > y) - (x < y);
}

/* cell graph: the diagonal plus one column per distinct face neighbour, sorted */
static int build_pattern(const co_mesh_t* m, csr_t* A) {
    const int64_t nc = m->n_cells;
    A->n = nc;
    A->ro = malloc(sizeof(int64_t) * (nc + 1));
    A->co = malloc(sizeof(int64_t) * (m->cell_offsets[nc] + nc));
    if (!A->ro || !A->co) return fail("out of memory");
    int64_t pos = 0;
    A->ro[0] = 0;
    for (int64_t c = 0; c < nc; ++c) {
        const int64_t start = pos;
        A->co[pos++] = c;
        for (int64_t k = m->cell_offsets[c]; k < m->cell_offsets[c + 1]; ++k) {
            const int64_t f = m->cell_faces[k];
            if (m->neighbour[f] < 0) continue;
            const int64_t other = m->owner[f] == c ? m->neighbour[f] : m->owner[f];
            int dup = 0;
            for (int64_t q = start; q < pos; ++q) dup |= A->co[q] == other;
            if (!dup) A->co[pos++] = other;
        }
        qsort(A->co + start, (size_t)(pos - start), sizeof(int64_t), cmp_i64);
        A->ro[c + 1] = pos;
    }
    A->nnz = pos;
    A->va = calloc((size_t)pos, sizeof(double));
    if (!A->va) return fail("out of memory");
    return 0;
}

static double* entry(csr_t* A, int64_t row, int64_t col) {
    for (int64_t k = A->ro[row]; k < A->ro[row + 1]; ++k)
        if (A->co[k] == col) return A->va + k;
    return NULL;
}

static void csr_free(csr_t* A) {
    free(A->ro); free(A->co); free(A->va);
    memset(A, 0, sizeof *A);
}

static int64_t export_csr(const csr_t* A, int64_t* ro, int64_t* co, double* va) {
    if (ro) memcpy(ro, A->ro, sizeof(int64_t) * (A->n + 1));
    if (co) memcpy(co, A->co, sizeof(int64_t) * A->nnz);
    if (va) memcpy(va, A->va, sizeof(double) * A->nnz);
    return A->nnz;
}

/* ------------------------------------------------- corrector assembly */

int64_t co_pressure_assemble(const co_mesh_t* m, const double* U, const double* rau, const double* p, double rho,
                             const int32_t* fixed, const double* value, double* phi_out, double* grad_out,
                             int64_t* ro, int64_t* co, double* va, double* b) {
    const int64_t nc = m->n_cells, nf = m->n_faces;
    geom_t g;
    csr_t A;
    memset(&A, 0, sizeof A);
    if (build_geometry(m, &g)) return -1;
    double* phi = malloc(sizeof(double) * nf);
    double* grad = malloc(sizeof(double) * 3 * nc);
    double* cont = calloc((size_t)nc, sizeof(double));
    double* diag = calloc((size_t)nc, sizeof(double));
    int64_t rc = -1;
    if (!phi || !grad || !cont || !diag) { fail("out of memory"); goto done; }
    if (build_pattern(m, &A)) goto done;
    /* :7894 phiHbyA = make_mass_flux(HbyA), face loop */
    for (int64_t f = 0; f < nf; ++f) phi[f] = mass_flux(m, &g, f, U, rho);
    /* :8060 gradient of the current pressure */
    if (gauss_gradient(m, &g, p, fixed, value, grad)) goto done;
    /* :8079-8098 continuity, cell-ordered loop over each cell's faces */
    for (int64_t c = 0; c < nc; ++c) {
        for (int64_t k = m->cell_offsets[c]; k < m->cell_offsets[c + 1]; ++k) {
            const int64_t f = m->cell_faces[k];
            const int own = m->owner[f] == c;
            cont[c] += own ? phi[f] : -phi[f];
            if (m->neighbour[f] >= 0) {
                double nonorth;
                if (rc_internal(m, &g, f, p, grad, rau, rho, &nonorth)) goto done;
                cont[c] += own ? -nonorth : nonorth;
            }
        }
    }
    /* :8100-8120 interior faces in face order: coefficient, diagonal, off-diagonals */
    for (int64_t f = 0; f < nf; ++f) {
        const int64_t n = m->neighbour[f];
        if (n < 0) continue;
        const int64_t o = m->owner[f];
        const v3 S = ld(g.sf, nf, f);
        const v3 dvec = vsub(ld(g.cc, nc, n), ld(g.cc, nc, o));
        double oc;
        if (orthogonal_coefficient(S, dvec, face_dau(&g, rau, o, n), &oc)) goto done;
        const double coeff = rho * oc;
        diag[o] += coeff;
        diag[n] += coeff;
        *entry(&A, o, n) -= coeff;
        *entry(&A, n, o) -= coeff;
    }
    /* :8122-8126 diagonal and right-hand side */
    for (int64_t c = 0; c < nc; ++c) {
        *entry(&A, c, c) += diag[c];
        b[c] = -cont[c];
    }
    /* :8130-8175 fixed-pressure boundary faces in face order */
    for (int64_t f = 0; f < nf; ++f) {
        if (m->neighbour[f] >= 0) continue;
        double v, bcoef, source;
        if (!fixed_value(m, fixed, value, f, &v)) continue;
        if (fixed_boundary(m, &g, f, p, grad, rau, rho, v, &bcoef, &source)) goto done;
        const int64_t o = m->owner[f];
        *entry(&A, o, o) += rho * bcoef;
        b[o] += source;
    }
    if (phi_out) memcpy(phi_out, phi, sizeof(double) * nf);
    if (grad_out) memcpy(grad_out, grad, sizeof(double) * 3 * nc);
    rc = export_csr(&A, ro, co, va);
done:
    free(phi); free(grad); free(cont); free(diag);
    csr_free(&A);
    geom_free(&g);
    return rc;
}

int co_rhie_chow_flux(const co_mesh_t* m, const double* U, const double* rau, const double* p, double rho,
                      const int32_t* fixed, const double* value, double* flux) {
    const int64_t nc = m->n_cells, nf = m->n_faces;
    geom_t g;
    if (build_geometry(m, &g)) return -1;
    double* grad = malloc(sizeof(double) * 3 * nc);
    int rc = -1;
    if (!grad) { fail("out of memory"); goto done; }
    if (gauss_gradient(m, &g, p, fixed, value, grad)) goto done;
    for (int64_t f = 0; f < nf; ++f) {
        const int64_t o = m->owner[f], n = m->neighbour[f];
        v3 Hf = ld(U, nc, o);
        double correction = 0.0;
        if (n >= 0) {
            const double wn = 0.5;
            Hf = vadd(vscale(Hf, 1.0 - wn), vscale(ld(U, nc, n), wn));
            if (rc_internal(m, &g, f, p, grad, rau, rho, &correction)) goto done;
        } else {
            const int t = patch_type(m, f);
            if (t == CO_PATCH_EMPTY || t == CO_PATCH_SYMMETRY) { flux[f] = 0.0; continue; }
            double v, bcoef;
            if (fixed_value(m, fixed, value, f, &v) &&
                fixed_boundary(m, &g, f, p, grad, rau, rho, v, &bcoef, &correction)) goto done;
        }
        flux[f] = rho * vdot(Hf, ld(g.sf, nf, f)) - correction;
    }
    rc = 0;
done:
    free(grad);
    geom_free(&g);
    return rc;
}

/* -------------------------------------------------- Poisson assembly */

int64_t co_assemble_diffusion(const co_mesh_t* m, const double* bcv, const int32_t* bct, double gamma,
                              const double* source, int64_t* ro, int64_t* co, double* va, double* rhs) {
    const int64_t nc = m->n_cells, nf = m->n_faces;
    if (!(gamma > 0.0) || !isfinite(gamma)) return fail("diffusivity must be positive");
    geom_t g;
    csr_t A;
    memset(&A, 0, sizeof A);
    if (build_geometry(m, &g)) return -1;
    int64_t rc = -1;
    if (build_pattern(m, &A)) goto done;
    for (int64_t c = 0; c < nc; ++c) rhs[c] = source[c] * g.cv[c];
    /* rows start as {(c, 0.0)}; face loop in face order (:84-140).  Each
     * off-diagonal appears once per face, so the consolidation of duplicate
     * columns (:143-158) is the single value 0.0 + (-g). */
    for (int64_t f = 0; f < nf; ++f) {
        const int64_t o = m->owner[f], n = m->neighbour[f];
        const double area = vmag(ld(g.sf, nf, f));
        if (!(area > 0.0) || !isfinite(area)) { fail("invalid face area"); goto done; }
        if (n >= 0) {
            const double d = vmag(vsub(ld(g.cc, nc, n), ld(g.cc, nc, o)));
            if (!(d > DBL_EPSILON) || !isfinite(d)) { fail("invalid cell-centre distance"); goto done; }
            const double gf = gamma * area / d;
            *entry(&A, o, o) += gf;
            *entry(&A, n, n) += gf;
            *entry(&A, o, n) = 0.0 + (-gf);
            *entry(&A, n, o) = 0.0 + (-gf);
        } else if (isfinite(bcv[f])) {
            const double d = vmag(vsub(ld(g.fc, nf, f), ld(g.cc, nc, o)));
            if (!(d > DBL_EPSILON) || !isfinite(d)) { fail("invalid boundary distance"); goto done; }
            const double gf = gamma * area / d;
            if (!bct || bct[f] == 0) {
                *entry(&A, o, o) += gf;
                rhs[o] += gf * bcv[f];
            } else {
                rhs[o] += bcv[f] * area;
            }
        }
    }
    /* consolidation: the diagonal is 0.0 + (accumulated diagonal) */
    for (int64_t c = 0; c < nc; ++c) *entry(&A, c, c) = 0.0 + *entry(&A, c, c);
    rc = export_csr(&A, ro, co, va);
done:
    csr_free(&A);
    geom_free(&g);
    return rc;
}

/* ------------------------------------------------------------- SpMV */

void co_spmv(int64_t n, const int64_t* ro, const int64_t* co, const double* va, const double* x, double* y) {
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k) s += va[k] * x[co[k]];
        y[i] = s;
    }
}

/* ----------------------------------------------------------- V-cycle */

/* amg_preconditioner.h:1310-1319 remove_constant: subtract the mean, summed in order */
static void remove_constant(int64_t n, double* v) {
    if (n == 0) return;
    double mean = 0.0;
    for (int64_t i = 0; i < n; ++i) mean += v[i];
    mean /= (double)n;
    for (int64_t i = 0; i < n; ++i) v[i] -= mean;
}

/* amg_preconditioner.h:2369-2409 damped Jacobi, x += omega * inv_diag (r - A x),
 * the mean removed after every sweep under the constant null space */
static int smooth(const co_hierarchy_t* h, int l, const double* r, double* x, int sweeps, double* ax) {
    const int64_t n = h->n_rows[l];
    for (int s = 0; s < sweeps; ++s) {
        co_spmv(n, h->row_offsets[l], h->columns[l], h->values[l], x, ax);
        for (int64_t i = 0; i < n; ++i) {
            const double delta = h->inv_diag[l][i] * (r[i] - ax[i]);
            x[i] += h->omega * delta;
            if (!isfinite(x[i])) return fail("non-finite smoother update");
        }
        if (h->constant_null_space) remove_constant(n, x);
    }
    return 0;
}

/* amg_preconditioner.h:2564-2666 smooth_coarsest */
static int coarsest(const co_hierarchy_t* h, int l, const double* r, double* x) {
    const int64_t n = h->n_rows[l];
    double* ax = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    if (!ax) return fail("out of memory");
    if (n > 16) {
        for (int64_t i = 0; i < n; ++i) x[i] = 0.0;
        const int rc = smooth(h, l, r, x, 24, ax);
        free(ax);
        return rc;
    }
    free(ax);
    /* :2590-2611 under the constant null space, the system bordered by a row
     * and a column of ones (a zero-mean correction) */
    const int64_t sn = n + (h->constant_null_space ? 1 : 0);
    double m[17 * 17], b[17], sol[17];
    for (int64_t q = 0; q < sn * sn; ++q) m[q] = 0.0;
    for (int64_t i = 0; i < sn; ++i) b[i] = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        b[i] = r[i];
        for (int64_t k = h->row_offsets[l][i]; k < h->row_offsets[l][i + 1]; ++k)
            m[i * sn + h->columns[l][k]] += h->values[l][k];
    }
    if (h->constant_null_space)
        for (int64_t i = 0; i < n; ++i) {
            m[i * sn + n] = 1.0;
            m[n * sn + i] = 1.0;
        }
    double scale = 0.0;
    for (int64_t q = 0; q < sn * sn; ++q) scale = fmax(scale, fabs(m[q]));
    const double tol = 128.0 * DBL_EPSILON * fmax(1.0, scale);
    for (int64_t k = 0; k < sn; ++k) {
        int64_t piv = k;
        double pa = fabs(m[k * sn + k]);
        for (int64_t i = k + 1; i < sn; ++i)
            if (fabs(m[i * sn + k]) > pa) { pa = fabs(m[i * sn + k]); piv = i; }
        if (!isfinite(pa) || pa <= tol) return fail("singular coarsest level");
        if (piv != k) {
            for (int64_t j = k; j < sn; ++j) { const double t = m[k * sn + j]; m[k * sn + j] = m[piv * sn + j]; m[piv * sn + j] = t; }
            const double t = b[k]; b[k] = b[piv]; b[piv] = t;
        }
        const double dg = m[k * sn + k];
        for (int64_t i = k + 1; i < sn; ++i) {
            const double factor = m[i * sn + k] / dg;
            if (!isfinite(factor)) return fail("non-finite elimination factor");
            m[i * sn + k] = 0.0;
            for (int64_t j = k + 1; j < sn; ++j) m[i * sn + j] -= factor * m[k * sn + j];
            b[i] -= factor * b[k];
        }
    }
    for (int64_t ii = sn; ii-- > 0;) {
        double sum = b[ii];
        for (int64_t j = ii + 1; j < sn; ++j) sum -= m[ii * sn + j] * sol[j];
        const double dg = m[ii * sn + ii];
        if (!isfinite(dg) || fabs(dg) <= tol) return fail("singular coarsest level");
        sol[ii] = sum / dg;
        if (!isfinite(sol[ii])) return fail("non-finite coarsest solution");
    }
    for (int64_t i = 0; i < n; ++i) x[i] = sol[i];
    if (h->constant_null_space) remove_constant(n, x);
    return 0;
}

/* amg_preconditioner.h:2411-2443 vcycle */
static int vcycle(const co_hierarchy_t* h, int l, const double* r, double* x) {
    if (l + 1 == h->n_levels) return coarsest(h, l, r, x);
    const int64_t n = h->n_rows[l], nc = h->n_rows[l + 1];
    double* ax = malloc(sizeof(double) * (size_t)n);
    double* cr = calloc((size_t)nc, sizeof(double));
    double* cx = calloc((size_t)nc, sizeof(double));
    int rc = -1;
    if (!ax || !cr || !cx) { fail("out of memory"); goto done; }
    if (smooth(h, l, r, x, h->pre_sweeps, ax)) goto done;
    co_spmv(n, h->row_offsets[l], h->columns[l], h->values[l], x, ax);
    /* restriction: scatter of P^T in increasing fine-row order */
    for (int64_t i = 0; i < n; ++i) {
        const double res = r[i] - ax[i];
        for (int64_t k = h->p_offsets[l][i]; k < h->p_offsets[l][i + 1]; ++k)
            cr[h->p_columns[l][k]] += h->p_values[l][k] * res;
    }
    if (h->constant_null_space) remove_constant(nc, cr);
    if (vcycle(h, l + 1, cr, cx)) goto done;
    /* prolongation: x_i += sum_k p_ik e_k in P's row order */
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t k = h->p_offsets[l][i]; k < h->p_offsets[l][i + 1]; ++k)
            x[i] += h->p_values[l][k] * cx[h->p_columns[l][k]];
        if (!isfinite(x[i])) { fail("non-finite prolongation"); goto done; }
    }
    if (h->constant_null_space) remove_constant(n, x);
    rc = smooth(h, l, r, x, h->post_sweeps, ax);
done:
    free(ax); free(cr); free(cx);
    return rc;
}

/* amg_preconditioner.h:1191-1203 apply: the cycle from z = 0 on r, with the
 * mean removed from a copy of r and from z under the constant null space */
int co_vcycle(const co_hierarchy_t* h, const double* r, double* z) {
    if (!h || h->n_levels <= 0) return fail("empty hierarchy");
    const int64_t n = h->n_rows[0];
    for (int64_t i = 0; i < n; ++i) {
        if (!isfinite(r[i])) return fail("non-finite residual");
        z[i] = 0.0;
    }
    if (h->constant_null_space) {
        double* rc = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
        if (!rc) return fail("out of memory");
        memcpy(rc, r, sizeof(double) * (size_t)n);
        remove_constant(n, rc);
        const int bad = vcycle(h, 0, rc, z);
        free(rc);
        if (bad) return -1;
        remove_constant(n, z);
    } else if (vcycle(h, 0, r, z)) {
        return -1;
    }
    for (int64_t i = 0; i < n; ++i)
        if (!isfinite(z[i])) return fail("non-finite V-cycle result");
    return 0;
}

/* ------------------------------------------------------------- GMRES */

/* krylov_reductions.h:84-115 krylov_norm2: scaled two-pass norm */
static double norm2(int64_t n, const double* a) {
    double scale = 0.0, invalid = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        if (!isfinite(a[i])) invalid = 1.0;
        scale = fmax(scale, fabs(a[i]));
    }
    if (invalid > 0.0) return NAN;
    if (scale == 0.0) return 0.0;
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double q = a[i] / scale;
        s += q * q;
    }
    if (!isfinite(s)) return NAN;
    return scale * sqrt(fmax(0.0, s));
}

/* krylov_reductions.h:63-82 krylov_dot_view: sequential sum */
static double dot(int64_t n, const double* a, const double* b) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* krylov_controls.h:28-51 choose_gmres_restart */
static int choose_restart(int current, double reduction) {
    const int rmin = 10, rmax = 512;
    const double target = 0.1;
    if (reduction > target * 2.0) return current > rmax - 5 ? rmax : current + 5;
    if (reduction < target * 0.5) return current - 5 > rmin ? current - 5 : rmin;
    return current < rmin ? rmin : (current > rmax ? rmax : current);
}

/* ------------------------------------------------------- null space */

/* null_space.h:58-62 constant(n): ones scaled by 1 / their hypot-accumulated
 * norm (:141-146 stable_norm), so every entry is this one value */
double co_null_space_entry(int64_t n) {
    double norm = 0.0;
    for (int64_t i = 0; i < n; ++i) norm = hypot(norm, 1.0);
    return 1.0 * (1.0 / norm);
}

/* null_space.h:64-71 remove: v -= (v . e) e with every e_i = e, the dot in order */
static int ns_remove(int64_t n, double e, double* v) {
    double c = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        if (!isfinite(v[i])) return fail("cannot project a non-finite vector");
        c += v[i] * e;
    }
    for (int64_t i = 0; i < n; ++i) v[i] -= c * e;
    return 0;
}

static double hypot_norm(int64_t n, const double* a) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s = hypot(s, a[i]);
    return s;
}

int co_null_space_checks(int64_t n, const int64_t* ro, const int64_t* co, const double* va, const double* b,
                         int32_t* out) {
    out[0] = out[1] = out[2] = 0;
    if (n <= 0) return 0;
    const double e = co_null_space_entry(n);
    /* :97-105 is_compatible: |b . e| <= 1e-14 + 1e-12 ||b|| */
    double c = 0.0;
    for (int64_t i = 0; i < n; ++i) c += b[i] * e;
    const double component = sqrt(fmax(0.0, c * c));
    out[0] = component <= 1e-14 + 1e-12 * hypot_norm(n, b);
    /* :107-134 operator_residual: ||A e|| / ||A||_F (hypot sums), <= 1e-12 */
    double fro = 0.0;
    for (int64_t k = 0; k < ro[n]; ++k) {
        if (!isfinite(va[k])) return fail("null space operator contains non-finite values");
        fro = hypot(fro, va[k]);
    }
    double* y = calloc((size_t)n, sizeof(double));
    if (!y) return fail("out of memory");
    double pn = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double sum = 0.0;
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k) sum += va[k] * e;
        pn = hypot(pn, sum);
    }
    out[1] = pn / fmax(fro, DBL_MIN) <= 1e-12;
    /* projected_gmres.h:53-82: and ||A^T e|| <= 1e-12 ||A||_F */
    for (int64_t i = 0; i < n; ++i)
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k) y[co[k]] += va[k] * e;
    out[2] = out[1] && !(hypot_norm(n, y) > 1e-12 * fmax(fro, DBL_MIN));
    free(y);
    return 0;
}

typedef struct {
    int64_t n;
    const int64_t *ro, *co;
    const double* va;
    const co_hierarchy_t* h;
    double ns;          /* entry of the constant null-space vector; 0: no projection */
    double* scratch;    /* n values for the projected operator */
} system_t;

/* The Krylov operator: A, or projected_gmres.h:122-131 P A P */
static int op_apply(const system_t* S, const double* in, double* out) {
    if (S->ns == 0.0) {
        co_spmv(S->n, S->ro, S->co, S->va, in, out);
        return 0;
    }
    memcpy(S->scratch, in, sizeof(double) * (size_t)S->n);
    if (ns_remove(S->n, S->ns, S->scratch)) return -1;
    co_spmv(S->n, S->ro, S->co, S->va, S->scratch, out);
    return ns_remove(S->n, S->ns, out);
}

static int gmres(const system_t* S, const double* b, double* x, int restart, int64_t max_iter, double tolerance,
                 co_report_t* R);

static void finish(co_report_t* R, int status, int64_t it, double res, double rel) {
    R->status = status;
    R->iterations = it;
    R->residual = res;
    R->residual_relative = rel;
}

static int gmres(const system_t* S, const double* b, double* x, int restart, int64_t max_iter, double tolerance,
                 co_report_t* R) {
    const int64_t n = S->n;
    memset(R, 0, sizeof *R);
    if (n == 0 || restart <= 0 || max_iter == 0 || !isfinite(tolerance) || tolerance <= 0.0) {
        R->status = 3;
        return 0;
    }
    int cur = restart < 10 ? 10 : (restart > 512 ? 512 : restart);
    if (n < cur) cur = (int)n;
    const double b_norm = norm2(n, b);
    if (!isfinite(b_norm)) { R->status = 2; return 0; }
    if (b_norm == 0.0) {
        /* :64-134: shifted solve A y = -A x0 */
        double* ax0 = malloc(sizeof(double) * n);
        if (!ax0) return fail("out of memory");
        if (op_apply(S, x, ax0)) { free(ax0); return -1; }
        const double ax0n = norm2(n, ax0);
        if (!isfinite(ax0n)) { free(ax0); finish(R, 2, 0, ax0n, ax0n); return 0; }
        if (ax0n > 0.0) {
            double* sh = malloc(sizeof(double) * n);
            double* y = calloc((size_t)n, sizeof(double));
            if (!sh || !y) { free(ax0); free(sh); free(y); return fail("out of memory"); }
            for (int64_t i = 0; i < n; ++i) sh[i] = -ax0[i];
            co_report_t inner;
            if (gmres(S, sh, y, restart, max_iter, tolerance, &inner)) { free(ax0); free(sh); free(y); return -1; }
            for (int64_t i = 0; i < n; ++i) x[i] += y[i];
            if (op_apply(S, x, ax0)) { free(ax0); free(sh); free(y); return -1; }
            for (int64_t i = 0; i < n; ++i) sh[i] = b[i] - ax0[i];
            const double res = norm2(n, sh), rel = res / ax0n;
            const int ok = isfinite(res) && isfinite(rel) && rel <= tolerance;
            *R = inner;
            finish(R, ok ? 0 : (inner.status == 3 ? 3 : 2), inner.iterations, res, rel);
            free(ax0); free(sh); free(y);
            return 0;
        }
        free(ax0);
    }
    const double rhs_scale = fmax(b_norm, 1e-300);
    const double tol = b_norm == 0.0 ? 0.0 : tolerance * b_norm;
    const size_t N = (size_t)n;
    double *r = malloc(sizeof(double) * N), *w = malloc(sizeof(double) * N), *best = malloc(sizeof(double) * N);
    double *trial = malloc(sizeof(double) * N), *tmp = malloc(sizeof(double) * N);
    double *V = NULL, *Z = NULL, *H = NULL, *cs = NULL, *sn = NULL, *g = NULL, *y = NULL;
    int rc = -1;
    if (!r || !w || !best || !trial || !tmp) { fail("out of memory"); goto out; }
#define TRUE_RESIDUAL(dst)                                      \
    do {                                                        \
        if (op_apply(S, x, tmp)) goto out;                      \
        for (int64_t i_ = 0; i_ < n; ++i_) r[i_] = b[i_] - tmp[i_]; \
        dst = norm2(n, r);                                      \
    } while (0)
    double beta;
    TRUE_RESIDUAL(beta);
    if (!isfinite(beta)) { finish(R, 2, 0, beta, 0.0); rc = 0; goto out; }
    if (b_norm == 0.0) {
        const double xn = norm2(n, x);
        const double ref = fmax(fmax(xn, 1.0), 1e-300);
        finish(R, beta <= tolerance * ref ? 0 : 2, 0, beta, beta / ref);
        rc = 0;
        goto out;
    }
    if (beta <= tol) { finish(R, 0, 0, beta, beta / rhs_scale); rc = 0; goto out; }
    int64_t iterations = 0;
    double previous = beta, best_res = beta;
    memcpy(best, x, sizeof(double) * N);
    int m_alloc = 0;
    while (iterations < max_iter) {
        const int m = cur;
        if (m > m_alloc) {
            free(V); free(Z); free(H); free(cs); free(sn); free(g); free(y);
            V = malloc(sizeof(double) * N * (size_t)(m + 1));
            Z = malloc(sizeof(double) * N * (size_t)m);
            H = malloc(sizeof(double) * (size_t)(m + 1) * (size_t)m);
            cs = malloc(sizeof(double) * m); sn = malloc(sizeof(double) * m);
            g = malloc(sizeof(double) * (m + 1)); y = malloc(sizeof(double) * m);
            if (!V || !Z || !H || !cs || !sn || !g || !y) { fail("out of memory"); goto out; }
            m_alloc = m;
        }
#define HH(i, j) H[(size_t)(i) * (size_t)m + (size_t)(j)]
        TRUE_RESIDUAL(beta);
        if (!isfinite(beta)) { memcpy(x, best, sizeof(double) * N); finish(R, 2, iterations, best_res, best_res / rhs_scale); rc = 0; goto out; }
        if (beta <= tol) break;
        for (int64_t i = 0; i < n; ++i) V[i] = r[i] / beta;
        memset(H, 0, sizeof(double) * (size_t)(m + 1) * (size_t)m);
        memset(cs, 0, sizeof(double) * m);
        memset(sn, 0, sizeof(double) * m);
        memset(g, 0, sizeof(double) * (m + 1));
        g[0] = beta;
        int used = 0, breakdown = 0, reliable_restart = 0;
        double est = beta, action = 0.0;
        for (int j = 0; j < m && iterations < max_iter; ++j) {
            double* vj = V + (size_t)j * N;
            double* zj = Z + (size_t)j * N;
            if (S->h || S->ns != 0.0) {
                /* projected_gmres.h:32-44 ProjectedPreconditioner: P M P */
                const double* in = vj;
                if (S->ns != 0.0) {
                    memcpy(trial, vj, sizeof(double) * N);
                    if (ns_remove(n, S->ns, trial)) goto out;
                    in = trial;
                }
                int bad = 0;
                if (S->h) bad = co_vcycle(S->h, in, zj) != 0;
                else memcpy(zj, in, sizeof(double) * N);
                if (!bad && S->ns != 0.0) {
                    for (int64_t i = 0; i < n; ++i) bad |= !isfinite(zj[i]);
                    if (!bad) ns_remove(n, S->ns, zj);
                }
                if (bad) {
                    memcpy(x, best, sizeof(double) * N);
                    finish(R, 3, iterations, best_res, best_res / rhs_scale);
                    rc = 0;
                    goto out;
                }
                ++R->preconditioner_applications;
            } else {
                memcpy(zj, vj, sizeof(double) * N);
            }
            if (op_apply(S, zj, w)) goto out;
            action = norm2(n, w);
            if (!isfinite(action)) { memcpy(x, best, sizeof(double) * N); finish(R, 2, iterations, best_res, best_res / rhs_scale); rc = 0; goto out; }
            /* :271-290 two passes of modified Gram-Schmidt */
            for (int i = 0; i <= j; ++i) {
                const double* vi = V + (size_t)i * N;
                const double hv = dot(n, vi, w);
                HH(i, j) = hv;
                for (int64_t k = 0; k < n; ++k) w[k] -= hv * vi[k];
            }
            for (int i = 0; i <= j; ++i) {
                const double* vi = V + (size_t)i * N;
                const double corr = dot(n, vi, w);
                HH(i, j) += corr;
                for (int64_t k = 0; k < n; ++k) w[k] -= corr * vi[k];
            }
            const double hnext = norm2(n, w);
            if (!isfinite(hnext)) { memcpy(x, best, sizeof(double) * N); finish(R, 2, iterations, best_res, best_res / rhs_scale); rc = 0; goto out; }
            HH(j + 1, j) = hnext;
            const double floor_ = 4096.0 * DBL_EPSILON * fmax(action, 1e-300);
            const int bd = hnext <= floor_ && action > 0.0;
            if (hnext > 0.0) {
                double* vn = V + (size_t)(j + 1) * N;
                for (int64_t k = 0; k < n; ++k) vn[k] = w[k] / hnext;
            }
            /* :324-350 Givens rotations */
            for (int i = 0; i < j; ++i) {
                const double h0 = HH(i, j), h1 = HH(i + 1, j);
                HH(i, j) = cs[i] * h0 + sn[i] * h1;
                HH(i + 1, j) = -sn[i] * h0 + cs[i] * h1;
            }
            const double a = HH(j, j), b2 = HH(j + 1, j);
            const double rho = hypot(a, b2);
            if (rho > 0.0) {
                cs[j] = a / rho;
                sn[j] = b2 / rho;
                HH(j, j) = rho;
                HH(j + 1, j) = 0.0;
                const double gj = g[j], gj1 = g[j + 1];
                g[j] = cs[j] * gj + sn[j] * gj1;
                g[j + 1] = -sn[j] * gj + cs[j] * gj1;
            }
            ++iterations;
            ++used;
            est = fabs(g[j + 1]);
            if (bd) { breakdown = 1; break; }
            if (est <= tol) break;
            /* :380-455 periodic check of the updated candidate's true residual */
            if (iterations % 50 == 0) {
                int usable = 1;
                for (int i = used; i-- > 0;) {
                    double sum = g[i];
                    for (int k = i + 1; k < used; ++k) sum -= HH(i, k) * y[k];
                    const double dg = HH(i, i);
                    if (!isfinite(sum) || !isfinite(dg) || fabs(dg) <= 128.0 * DBL_EPSILON * fmax(action, 1e-300)) {
                        usable = 0;
                        break;
                    }
                    y[i] = sum / dg;
                }
                if (usable) {
                    memcpy(trial, x, sizeof(double) * N);
                    for (int k = 0; k < used; ++k) {
                        const double* zk = Z + (size_t)k * N;
                        for (int64_t i = 0; i < n; ++i) trial[i] += y[k] * zk[i];
                    }
                    if (op_apply(S, trial, tmp)) goto out;
                    for (int64_t i = 0; i < n; ++i) tmp[i] = b[i] - tmp[i];
                    const double verified = norm2(n, tmp);
                    if (!isfinite(verified) || verified / fmax(est, 1e-300) > 10.0) {
                        reliable_restart = 1;
                        break;
                    }
                }
            }
        }
        if (used == 0) break;
        /* :463-495 back substitution */
        for (int i = 0; i < m; ++i) y[i] = 0.0;
        for (int i = used; i-- > 0;) {
            double sum = g[i];
            for (int jj = i + 1; jj < used; ++jj) sum -= HH(i, jj) * y[jj];
            const double dg = HH(i, i);
            double hs = fabs(dg);
            for (int k = 0; k < used; ++k) hs = fmax(hs, fabs(HH(k, i)));
            const double dfloor = 128.0 * DBL_EPSILON * fmax(hs, 1e-300);
            if (fabs(dg) <= dfloor) {
                if (fabs(sum) <= dfloor) { y[i] = 0.0; continue; }
                double bres;
                TRUE_RESIDUAL(bres);
                if (!isfinite(bres) || best_res < bres) { memcpy(x, best, sizeof(double) * N); bres = best_res; }
                finish(R, 2, iterations, bres, bres / rhs_scale);
                rc = 0;
                goto out;
            }
            y[i] = sum / dg;
        }
        /* :497-501 x += sum_j y_j z_j, one basis vector at a time */
        for (int jj = 0; jj < used; ++jj) {
            const double alpha = y[jj];
            const double* zk = Z + (size_t)jj * N;
            for (int64_t i = 0; i < n; ++i) x[i] += alpha * zk[i];
        }
        TRUE_RESIDUAL(beta);
        if (reliable_restart && isfinite(beta)) ++R->residual_replacements;
        if (!isfinite(beta)) { memcpy(x, best, sizeof(double) * N); finish(R, 2, iterations, best_res, best_res / rhs_scale); rc = 0; goto out; }
        if (beta < best_res) { best_res = beta; memcpy(best, x, sizeof(double) * N); }
        if (beta <= tol) { finish(R, 0, iterations, beta, beta / rhs_scale); rc = 0; goto out; }
        if (breakdown) {
            if (best_res < beta) { memcpy(x, best, sizeof(double) * N); beta = best_res; }
            finish(R, 2, iterations, beta, beta / rhs_scale);
            rc = 0;
            goto out;
        }
        const double reduction = beta / fmax(previous, 1e-300);
        if (!isfinite(reduction)) { memcpy(x, best, sizeof(double) * N); finish(R, 2, iterations, best_res, best_res / rhs_scale); rc = 0; goto out; }
        cur = choose_restart(cur, reduction);
        if (n < cur) cur = (int)n;
        previous = beta;
#undef HH
    }
    if (best_res < beta) { memcpy(x, best, sizeof(double) * N); beta = best_res; }
    finish(R, 1, iterations, beta, beta / rhs_scale);
    rc = 0;
#undef TRUE_RESIDUAL
out:
    free(r); free(w); free(best); free(trial); free(tmp);
    free(V); free(Z); free(H); free(cs); free(sn); free(g); free(y);
    return rc;
}

int co_solve_gmres(int64_t n, const int64_t* ro, const int64_t* co, const double* va, const co_hierarchy_t* h,
                   const double* b, double* x, int32_t restart, int64_t max_iterations, double tolerance,
                   co_report_t* report) {
    const system_t S = {n, ro, co, va, h, 0.0, NULL};
    co_report_t local;
    co_report_t* R = report ? report : &local;
    return gmres(&S, b, x, restart, max_iterations, tolerance, R);
}

int co_solve_projected_gmres(int64_t n, const int64_t* ro, const int64_t* co, const double* va,
                             const co_hierarchy_t* h, const double* b, double* x, int32_t restart,
                             int64_t max_iterations, double tolerance, co_report_t* report) {
    co_report_t local;
    co_report_t* R = report ? report : &local;
    memset(R, 0, sizeof *R);
    R->status = 3;
    if (n <= 0 || restart <= 0 || max_iterations <= 0 || !(tolerance > 0.0) || !isfinite(tolerance)) return 0;
    for (int64_t i = 0; i < n; ++i)
        if (!isfinite(b[i]) || !isfinite(x[i])) return 0;
    int32_t checks[3];
    if (co_null_space_checks(n, ro, co, va, b, checks)) return -1;
    if (!checks[0] || !checks[2]) return 0;
    const size_t N = (size_t)n;
    double* gf = malloc(sizeof(double) * N);
    double* ax = malloc(sizeof(double) * N);
    double* scratch = malloc(sizeof(double) * N);
    int rc = -1;
    if (!gf || !ax || !scratch) { fail("out of memory"); goto done; }
    /* :101-104 a gauge-free copy of the iterate */
    const double e = co_null_space_entry(n);
    memcpy(gf, x, sizeof(double) * N);
    if (ns_remove(n, e, gf)) goto done;
    /* :105-119 already satisfied in physical coordinates */
    co_spmv(n, ro, co, va, gf, ax);
    double r0 = 0.0;
    for (int64_t i = 0; i < n; ++i) r0 = hypot(r0, b[i] - ax[i]);
    const double bn = hypot_norm(n, b);
    if (r0 == 0.0 || (bn > 0.0 && r0 <= tolerance * bn)) {
        R->status = 0;
        R->residual = r0;
        R->residual_relative = bn > 0.0 ? r0 / bn : 0.0;
        memcpy(x, gf, sizeof(double) * N);
        rc = 0;
        goto done;
    }
    /* :120-141 FGMRES on P A P, preconditioned by P M P */
    const system_t S = {n, ro, co, va, h, e, scratch};
    if (gmres(&S, b, gf, restart, max_iterations, tolerance, R)) goto done;
    int valid = 1;
    for (int64_t i = 0; i < n; ++i) valid &= isfinite(gf[i]) != 0;
    if (R->status != 3 && valid) {
        if (ns_remove(n, e, gf)) goto done;
        memcpy(x, gf, sizeof(double) * N);
    }
    rc = 0;
done:
    free(gf); free(ax); free(scratch);
    return rc;
}

/* ---------------------------------------------------------------- CG */

/* The preconditioner of one CG solve: the solver's own diagonal (no object,
 * the legacy solve_cg overload), or one of the objects the dispatch builds
 * (linear_solver_dispatch.h:169-189): identity, Jacobi, native AMG. */
typedef struct {
    int32_t kind;
    const co_hierarchy_t* h;
    const double* diag;      /* kind 0: first diagonal entry; kind 2: its inverse */
    double ns;               /* entry of the constant null-space vector; 0: none */
} cg_pc_t;

/* cg_solver.h:203-216 apply_preconditioner: z = M^-1 r (projected under a
 * null space), every entry finite */
static int cg_apply(const cg_pc_t* P, int64_t n, const double* r, double* z) {
    switch (P->kind) {
        case CO_CG_INTERNAL_JACOBI:
            for (int64_t i = 0; i < n; ++i) z[i] = r[i] / P->diag[i];
            break;
        case CO_CG_IDENTITY:                       /* preconditioner.h:39-45 */
            memcpy(z, r, sizeof(double) * (size_t)n);
            break;
        case CO_CG_JACOBI:                         /* preconditioner.h:87-91 */
            for (int64_t i = 0; i < n; ++i) z[i] = P->diag[i] * r[i];
            break;
        default:
            if (co_vcycle(P->h, r, z)) return 0;
    }
    if (P->ns != 0.0) {
        for (int64_t i = 0; i < n; ++i)
            if (!isfinite(z[i])) return 0;
        ns_remove(n, P->ns, z);
    }
    for (int64_t i = 0; i < n; ++i)
        if (!isfinite(z[i])) return 0;
    return 1;
}

int co_solve_cg(int64_t n, const int64_t* ro, const int64_t* co, const double* va, int32_t preconditioner,
                const co_hierarchy_t* h, const double* b, double* x, int64_t max_iter, double tolerance,
                co_report_t* report) {
    return co_solve_cg_ns(n, ro, co, va, preconditioner, h, b, x, max_iter, tolerance, 0, report);
}

int co_solve_cg_ns(int64_t n, const int64_t* ro, const int64_t* co, const double* va, int32_t preconditioner,
                   const co_hierarchy_t* h, const double* b, double* x, int64_t max_iter, double tolerance,
                   int32_t null_space, co_report_t* report) {
    co_report_t local;
    co_report_t* R = report ? report : &local;
    memset(R, 0, sizeof *R);
    if (n <= 0) { R->status = 3; return 0; }
    if (preconditioner == CO_CG_AMG && !h) return fail("CG with native AMG needs a hierarchy");
    if (preconditioner != CO_CG_INTERNAL_JACOBI && preconditioner != CO_CG_IDENTITY &&
        preconditioner != CO_CG_JACOBI && preconditioner != CO_CG_AMG)
        return fail("unknown CG preconditioner %d", (int)preconditioner);
    const int has_pc = preconditioner != CO_CG_INTERNAL_JACOBI;
    double ns = 0.0;
    if (null_space) {
        /* :74-79 a compatible right-hand side and A e = 0, else NOT_APPLICABLE */
        int32_t checks[3];
        if (co_null_space_checks(n, ro, co, va, b, checks)) return -1;
        if (!checks[0] || !checks[1]) { R->status = 3; return 0; }
        ns = co_null_space_entry(n);
    }
    for (int64_t k = 0; k < ro[n]; ++k)
        if (!isfinite(va[k])) { R->status = 2; return 0; }
    for (int64_t i = 0; i < n; ++i)
        if (!isfinite(b[i]) || !isfinite(x[i])) { R->status = 2; return 0; }
    if (ns != 0.0) ns_remove(n, ns, x);                            /* :93 */
    const size_t N = (size_t)n;
    double *r = malloc(sizeof(double) * N), *rv = malloc(sizeof(double) * N), *z = malloc(sizeof(double) * N);
    double *p = malloc(sizeof(double) * N), *Ap = malloc(sizeof(double) * N), *M = calloc(N, sizeof(double));
    int rc = -1;
    if (!r || !rv || !z || !p || !Ap || !M) { fail("out of memory"); goto out; }
    cg_pc_t P = {preconditioner, h, M, ns};
#define NS_REMOVE(v) do { if (ns != 0.0) ns_remove(n, ns, (v)); } while (0)
    double homogeneous = 0.0;
    /* cg_solver.h:108-120 update_true_residual (reports of failed solves) */
#define TRUE_RES()                                                                   \
    do {                                                                             \
        co_spmv(n, ro, co, va, x, Ap);                                               \
        for (int64_t i_ = 0; i_ < n; ++i_) rv[i_] = b[i_] - Ap[i_];                  \
    } while (0)
#define FAILED_REPORT(st, it)                                                        \
    do {                                                                             \
        R->status = (st);                                                            \
        R->iterations = (it);                                                        \
        TRUE_RES();                                                                  \
        R->residual = norm2(n, rv);                                                  \
        const double bn_ = norm2(n, b);                                              \
        R->residual_relative = bn_ > 0.0 ? R->residual / bn_                         \
            : (homogeneous > 0.0 ? R->residual / homogeneous                         \
               : (R->residual == 0.0 ? 0.0 : INFINITY));                             \
        rc = 0;                                                                      \
        goto out;                                                                    \
    } while (0)
#define FINISH(st, it, res)                                                          \
    do {                                                                             \
        R->status = (st);                                                            \
        R->iterations = (it);                                                        \
        R->residual = (res);                                                         \
        R->residual_relative = reference > 0.0 ? (res) / reference : 0.0;            \
        rc = 0;                                                                      \
        goto out;                                                                    \
    } while (0)
#define APPLY() (++R->preconditioner_applications, cg_apply(&P, n, r, z))
    /* :149-169 initial true residual, converged before any preconditioner work */
    TRUE_RES();
    NS_REMOVE(rv);                                                 /* :149 */
    memcpy(r, rv, sizeof(double) * N);
    const double b_norm = norm2(n, b);
    const double initial = norm2(n, rv);
    homogeneous = b_norm == 0.0 ? initial : 0.0;
    const double reference = b_norm > 0.0 ? b_norm : initial;
    const double tol_abs = tolerance * reference;
    if (initial <= tol_abs) FINISH(0, 0, initial);
    /* :171-189 the solver's own diagonal / the Jacobi object's inverse diagonal */
    if (preconditioner == CO_CG_INTERNAL_JACOBI || preconditioner == CO_CG_JACOBI) {
        for (int64_t i = 0; i < n; ++i) {
            int found = 0;
            for (int64_t k = ro[i]; k < ro[i + 1]; ++k)
                if (co[k] == i) {
                    M[i] = preconditioner == CO_CG_JACOBI ? 1.0 / va[k] : va[k];
                    found = 1;
                    break;
                }
            if (preconditioner == CO_CG_INTERNAL_JACOBI ? (!(M[i] > 0.0) || !isfinite(M[i]))
                                                        : (!found || !isfinite(M[i])))
                FAILED_REPORT(3, 0);
        }
    }
    if (!APPLY()) FAILED_REPORT(3, 0);
    memcpy(p, z, sizeof(double) * N);
    double rsold = dot(n, r, z);
    if (!isfinite(rsold)) FAILED_REPORT(2, 0);
    if (!(rsold > 0.0)) FAILED_REPORT(3, 0);
    double at_last_replacement = INFINITY;
    for (int64_t iter = 1; iter <= max_iter; ++iter) {
        co_spmv(n, ro, co, va, p, Ap);
        NS_REMOVE(Ap);                                             /* :262 */
        const double pAp = dot(n, p, Ap);
        if (!(pAp > 0.0) || !isfinite(pAp)) FAILED_REPORT(3, iter);
        const double alpha = rsold / pAp;
        if (!isfinite(alpha)) FAILED_REPORT(2, iter);
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
        }
        if (ns != 0.0) {                                           /* :295-298 */
            for (int64_t i = 0; i < n; ++i)
                if (!isfinite(x[i]) || !isfinite(r[i])) FAILED_REPORT(2, iter);
            ns_remove(n, ns, x);
            ns_remove(n, ns, r);
        }
        for (int64_t i = 0; i < n; ++i)
            if (!isfinite(x[i]) || !isfinite(r[i])) FAILED_REPORT(2, iter);
        if (!APPLY()) FAILED_REPORT(3, iter);
        const double rsnew = dot(n, r, z);
        if (!isfinite(rsnew)) FAILED_REPORT(2, iter);
        TRUE_RES();
        const double res = norm2(n, rv);
        if (res <= tol_abs) FINISH(0, iter, res);
        if (!has_pc) {
            /* :321-352 the internal-Jacobi residual replacement */
            double rr = 0.0;
            for (int64_t i = 0; i < n; ++i) rr = hypot(rr, r[i]);
            if (isfinite(rr) && rr <= tol_abs && res > tol_abs) {
                ++R->residual_replacements;
                memcpy(r, rv, sizeof(double) * N);
                NS_REMOVE(r);                                      /* :376 */
                if (!APPLY()) { R->status = 3; R->iterations = iter; rc = 0; goto out; }
                const double replaced = dot(n, r, z);
                if (!isfinite(replaced) || !(replaced > 0.0)) FINISH(1, iter, res);
                memcpy(p, z, sizeof(double) * N);
                rsold = replaced;
                continue;
            }
        } else {
            /* :399-525 adaptive residual replacement and collapse repair */
            double rr2 = 0.0;
            for (int64_t i = 0; i < n; ++i) rr2 += r[i] * r[i];
            const double rr = sqrt(rr2);
            const double gap = fabs(res - rr);
            const double scale = fmax(res, rr);
            const int progress = res < 0.5 * at_last_replacement;
            const int collapsed = !(rsnew > 0.0);
            const int adaptive = isfinite(rr) && scale > 0.0 && gap > 0.25 * scale && progress;
            const int repair = collapsed && progress;
            if (collapsed && !repair) FINISH(1, iter, res);
            if (adaptive || repair) {
                ++R->residual_replacements;
                at_last_replacement = res;
                memcpy(r, rv, sizeof(double) * N);
                NS_REMOVE(r);                                      /* :517 */
                if (!APPLY()) FAILED_REPORT(3, iter);
                const double replaced = dot(n, r, z);
                if (!isfinite(replaced) || !(replaced > 0.0)) FAILED_REPORT(3, iter);
                memcpy(p, z, sizeof(double) * N);
                rsold = replaced;
                continue;
            }
        }
        const double beta = rsnew / rsold;
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        NS_REMOVE(p);                                              /* :558 */
        rsold = rsnew;
    }
    TRUE_RES();
    FINISH(1, max_iter, norm2(n, rv));
#undef TRUE_RES
#undef FAILED_REPORT
#undef FINISH
#undef APPLY
#undef NS_REMOVE
out:
    free(r); free(rv); free(z); free(p); free(Ap); free(M);
    return rc;
}

/* ------------------------------------------------------------- gauge */

/* physics/steady_incompressible_solver.h:8617-8654, the pure-Neumann branch of
 * the pressure corrector: skip row ref, skip column ref in every other row,
 * shift later indices down by one, keep b without entry ref. */
int64_t co_gauge_eliminate(int64_t n, const int64_t* ro, const int64_t* co, const double* va, const double* b,
                           int64_t ref, int64_t* ro_out, int64_t* co_out, double* va_out, double* b_out) {
    if (n <= 1 || ref < 0 || ref >= n) return fail("gauge: invalid size or reference cell");
    int64_t nnz = 0, r = 0;
    ro_out[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (i == ref) continue;
        b_out[r] = b[i];
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k) {
            if (co[k] == ref) continue;
            co_out[nnz] = co[k] < ref ? co[k] : co[k] - 1;
            va_out[nnz] = va[k];
            ++nnz;
        }
        ro_out[++r] = nnz;
    }
    return nnz;
}

/* :8645-8653: p_corr(cell) = reduced(cell < ref ? cell : cell - 1), p_corr(ref) = 0 */
void co_gauge_expand(int64_t n, const double* x_reduced, int64_t ref, double* x) {
    for (int64_t i = 0; i < n; ++i) x[i] = i == ref ? 0.0 : x_reduced[i < ref ? i : i - 1];
}

/* core/solvers/scalar_diffusion.h:177-210 apply_reference_cell_gauge */
int64_t co_gauge_identity_row(int64_t n, const int64_t* ro, const int64_t* co, const double* va, const double* b,
                              int64_t ref, double value, int64_t* ro_out, int64_t* co_out, double* va_out,
                              double* b_out) {
    if (n <= 0 || ref < 0 || ref >= n || !isfinite(value)) return fail("gauge: invalid arguments");
    int64_t nnz = 0;
    ro_out[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        double a_iref = 0.0;   /* matrix(i, ref): the sum of the row's entries in column ref */
        for (int64_t k = ro[i]; k < ro[i + 1]; ++k)
            if (co[k] == ref) a_iref += va[k];
        b_out[i] = i == ref ? value : b[i] - a_iref * value;
        if (i == ref) {
            co_out[nnz] = ref;
            va_out[nnz] = 1.0;
            ++nnz;
        } else {
            for (int64_t k = ro[i]; k < ro[i + 1]; ++k) {
                if (co[k] == ref) continue;
                co_out[nnz] = co[k];
                va_out[nnz] = va[k];
                ++nnz;
            }
        }
        ro_out[i + 1] = nnz;
    }
    return nnz;
}

/* ---------------------------------------------------- momentum-inverse HbyA */

/* physics/steady_incompressible_solver.h:6430-6465 (build_hbya): h starts at
 * the component's momentum right-hand side plus gradp * V (:6437), subtracts
 * the off-diagonal products in the row's CSR order (:6438-6443), and HbyA is
 * rAU * h (:6459), refused when not finite (:6460-6461). */
int co_build_hbya(int64_t n, const int64_t* ro, const int64_t* co, const double* va, const double* rhs,
                  const double* U, const double* gradp, const double* vol, const double* rAU, double* HbyA) {
    const int64_t nnz = ro[n];
    for (int d = 0; d < 3; ++d) {
        const double* a = va + d * nnz;
        for (int64_t c = 0; c < n; ++c) {
            double h = rhs[d * n + c] + gradp[d * n + c] * vol[c];
            for (int64_t k = ro[c]; k < ro[c + 1]; ++k) {
                const int64_t col = co[k];
                if (col != c) h -= a[k] * U[d * n + col];
            }
            HbyA[d * n + c] = rAU[d * n + c] * h;
            if (!isfinite(HbyA[d * n + c])) return fail("solve_steady_incompressible: non-finite HbyA");
        }
    }
    return 0;
}
