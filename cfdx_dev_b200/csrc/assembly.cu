// assembly.cu -- mesh upload, finite-volume geometry and the pressure-correction
// face loop on the GPU.
//
// Geometry restates compute_face_geometry (core/geometry/face_geometry.h:50-90),
// compute_cell_geometry(_oriented) (core/geometry/cell_geometry.h:49-147) and the
// two-pass orientation of build_fv_geometry (physics/finite_volume_transport.h:92-176);
// compute_geometry_cache (core/geometry/geometry_cache.h:66-237) yields the same
// values.  The Gauss gradient and the corrector assembly are cell-centric: a
// thread per cell recomputes the quantities of its faces (identical inputs and
// operations from either side of a face) and sums them in the order the
// reference does -- cell-face order for continuity and the gradient, global
// face order for the diagonal and the boundary sources -- so no atomics are
// needed and every FP64 result is bit-identical to the reference's (this file
// is compiled without FMA contraction).  The geometry build also forms
// per-mesh tables so that no call repeats geometric work: per cell-face slot
// the face, side and other cell in one 8-byte record (no owner/neighbour
// lookup chain), the gradient weight of the cell's side, and per face the
// corrector's d, e and Sf . e (no square roots or divisions of geometry per
// call).  (A warp-per-tile variant with one lane per slot and the per-cell
// sums formed in order through shuffles was bit-identical but measured 1.8x
// slower for the assembly on the 64^3 tets: the shuffles cost more
// instructions than the extra parallelism saved.)
#include <algorithm>
#include <cmath>
#include <numeric>
#include <string>

#include "io.h"

namespace cfdxg {
namespace {

constexpr int kT = 128;
constexpr int kMaxCellFaces = 16;
constexpr int kPatchSymmetry = 3;
constexpr int kPatchEmpty = 6;
constexpr int kOtherSide = int(0x80000000u);   // slot record: the cell is the face's neighbour

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 ld3(const double* a, int64_t n, int64_t i) { return {a[i], a[n + i], a[2 * n + i]}; }
__device__ __forceinline__ D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 mul(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ double mag(D3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

// face_geometry.h:50-90 -- triangle fan around the first vertex
__global__ void k_face_geometry(int nf, const int* __restrict__ fo, const int* __restrict__ fv,
                                const double* __restrict__ px, const double* __restrict__ py,
                                const double* __restrict__ pz, double* fc, double* sf, int* status) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int off = fo[f], nv = fo[f + 1] - off;
    if (nv < 3) { atomicOr(status, kStatusGeometry); return; }
    const int v0 = fv[off];
    const D3 p0{px[v0], py[v0], pz[v0]};
    D3 S{0.0, 0.0, 0.0}, awc{0.0, 0.0, 0.0};
    double tri_area = 0.0;
    for (int k = 1; k + 1 < nv; ++k) {
        const int va = fv[off + k], vb = fv[off + k + 1];
        const D3 pa{px[va], py[va], pz[va]}, pb{px[vb], py[vb], pz[vb]};
        const D3 tS = mul(cross(sub(pa, p0), sub(pb, p0)), 0.5);
        const double ta = mag(tS);
        S = add(S, tS);
        awc = add(awc, mul(add(add(p0, pa), pb), ta / 3.0));
        tri_area += ta;
    }
    const double area = mag(S);
    if (!(tri_area > 0.0) || !(area > 0.0) || !isfinite(area)) atomicOr(status, kStatusGeometry);
    const D3 c = mul(awc, 1.0 / tri_area);
    fc[f] = c.x; fc[nf + f] = c.y; fc[2 * nf + f] = c.z;
    sf[f] = S.x; sf[nf + f] = S.y; sf[2 * nf + f] = S.z;
}

// cell_geometry.h:49-147 with the ownership-signed local Sf
__global__ void k_cell_geometry(int nc, int nf, const int* __restrict__ co, const int* __restrict__ cf,
                                const int* __restrict__ owner, const double* __restrict__ fc,
                                const double* __restrict__ sf, double* cc, double* vol, int* status) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int b = co[c], e = co[c + 1];
    if (e == b) { atomicOr(status, kStatusGeometry); return; }
    bool is_2d = true;
    for (int k = b; k < e; ++k) {
        const int f = cf[k];
        if (fabs(fc[2 * nf + f]) > 1e-12) { is_2d = false; break; }
        if (fabs(sf[f]) > 1e-12 || fabs(sf[nf + f]) > 1e-12) { is_2d = false; break; }
    }
    D3 ws{0.0, 0.0, 0.0};
    double total = 0.0;
    for (int k = b; k < e; ++k) {
        const int f = cf[k];
        const D3 cfv = ld3(fc, nf, f);
        D3 s = ld3(sf, nf, f);
        if (owner[f] != c) s = mul(s, -1.0);
        const double a = mag(s);
        ws = add(ws, mul(cfv, a));
        total += a;
    }
    const D3 centre = total > 0.0 ? mul(ws, 1.0 / total) : D3{0.0, 0.0, 0.0};
    double sv = 0.0;
    for (int k = b; k < e; ++k) {
        const int f = cf[k];
        D3 s = ld3(sf, nf, f);
        if (owner[f] != c) s = mul(s, -1.0);
        const double area = mag(s);
        if (!(area > 0.0)) atomicOr(status, kStatusGeometry);
        if (is_2d) sv += area;
        else sv += dot(sub(ld3(fc, nf, f), centre), s);
    }
    if (!is_2d) sv /= 3.0;
    const double v = fabs(sv);
    if (!(v > 0.0) || !isfinite(v) || !isfinite(sv)) atomicOr(status, kStatusGeometry);
    cc[c] = centre.x; cc[nc + c] = centre.y; cc[2 * nc + c] = centre.z;
    if (vol) vol[c] = v;
}

// face_geometry.h:115-127 ensure_face_orientation
__global__ void k_orient(int nf, int nc, const int* __restrict__ owner, const int* __restrict__ neigh,
                         const double* __restrict__ fc, const double* __restrict__ cc, double* sf) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int o = owner[f], n = neigh[f];
    const D3 co = ld3(cc, nc, o);
    const D3 d = n >= 0 ? sub(ld3(cc, nc, n), co) : sub(ld3(fc, nf, f), co);
    const D3 s = ld3(sf, nf, f);
    if (dot(s, d) < 0.0) {
        const D3 t = mul(s, -1.0);
        sf[f] = t.x; sf[nf + f] = t.y; sf[2 * nf + f] = t.z;
    }
}

struct MeshView {
    int nc, nf;
    const int *co, *cf, *cs, *owner, *neigh, *patch, *ptype;
    const double *fc, *sf, *cc, *vol;
    const double* geo;   // per-face d, e, Sf . e (face-loop table), null until built
};

struct BcView {
    const int* fixed;     // per patch
    const double* value;  // per patch
    int n_patches;
};

// Geometry of one face as the corrector uses it (pressure_face_orthogonal_coefficient,
// steady_incompressible_solver.h:1914-1935, and the same terms of
// pressure_face_nonorthogonal_flux, :1941-1965): d = |dvec|, e = dvec / d and
// oa = Sf . e, with dvec = Cn - Co on an interior face and Cf - Co on a
// boundary face.  They depend on the geometry only, so k_face_terms forms them
// once per mesh with exactly these operations; the corrector reads them back
// and forms rfn = sum_d dAU_d e_d^2, which depends on rAU.  (The area check of
// those functions is the geometry build's: Sf never changes.)
struct FaceTerms {
    D3 e;
    double d, oa, rfn;
};

// per-face table layout (SoA, nf each): d, e.x, e.y, e.z, oa
constexpr int kFaceTermArrays = 5;

__device__ __forceinline__ FaceTerms face_terms(const double* __restrict__ geo, int nf, int f, D3 dau,
                                                int* status) {
    FaceTerms t;
    t.d = geo[f];
    t.e = D3{geo[nf + f], geo[2 * nf + f], geo[3 * nf + f]};
    t.oa = geo[4 * nf + f];
    if (!(t.d > 0.0) || !isfinite(t.d)) atomicOr(status, kStatusGeometry);
    if (!(t.oa > 0.0) || !isfinite(t.oa)) atomicOr(status, kStatusGeometry);
    t.rfn = dau.x * t.e.x * t.e.x + dau.y * t.e.y * t.e.y + dau.z * t.e.z * t.e.z;
    return t;
}

// :1914-1935 -- rfn (Sf . e) / d
__device__ __forceinline__ double ortho_coefficient(const FaceTerms& t, int* status) {
    const double coefficient = t.rfn * t.oa / t.d;
    if (!isfinite(coefficient)) atomicOr(status, kStatusGeometry);
    return coefficient;
}

// :1941-1965 -- (dAU o grad p) . Sf - rfn (grad p . e)(Sf . e)
__device__ __forceinline__ double nonortho_flux(const FaceTerms& t, D3 S, D3 dau, D3 gp, int* status) {
    const double full = dau.x * gp.x * S.x + dau.y * gp.y * S.y + dau.z * gp.z * S.z;
    const double implicit_flux = t.rfn * dot(gp, t.e) * t.oa;
    const double deferred = full - implicit_flux;
    if (!isfinite(deferred)) atomicOr(status, kStatusGeometry);
    return deferred;
}

// dAU face interpolation of rhie_chow_pressure_flux_internal (:1991-1999) / :6491-6499, wn = 0.5
__device__ __forceinline__ D3 face_dau(int o, int n, int nc, const double* vol, const double* rau) {
    const double wn = 0.5, wo = 1.0 - wn;
    return {wo * vol[o] * rau[o] + wn * vol[n] * rau[n],
            wo * vol[o] * rau[nc + o] + wn * vol[n] * rau[nc + n],
            wo * vol[o] * rau[2 * nc + o] + wn * vol[n] * rau[2 * nc + n]};
}

// rhie_chow_pressure_flux_internal (:1967-2024) for the interior face f with
// owner o and neighbour n; also returns the implicit coefficient (the
// pressure-matrix face coefficient before rho).
__device__ __forceinline__ double rc_internal(const MeshView& m, int f, int o, int n, const double* p,
                                              const double* grad, const double* rau, double rho,
                                              double* implicit_out, int* status) {
    const D3 S = ld3(m.sf, m.nf, f);
    const double wn = 0.5, wo = 1.0 - wn;
    const D3 dau = face_dau(o, n, m.nc, m.vol, rau);
    const D3 gp{wo * grad[o] + wn * grad[n], wo * grad[m.nc + o] + wn * grad[m.nc + n],
                wo * grad[2 * m.nc + o] + wn * grad[2 * m.nc + n]};
    const FaceTerms t = face_terms(m.geo, m.nf, f, dau, status);
    const double ic = ortho_coefficient(t, status);
    const double no = nonortho_flux(t, S, dau, gp, status);
    if (implicit_out) *implicit_out = ic;
    return rho * (ic * (p[n] - p[o]) + no);
}

// make_mass_flux (:1842-1905) on face f with owner o and neighbour n (< 0 on
// the boundary), zero-gradient velocity boundaries
__device__ __forceinline__ double mass_flux(const MeshView& m, int f, int o, int n, const double* U, double rho) {
    D3 Uf = ld3(U, m.nc, o);
    if (n >= 0) {
        const double wn = 0.5;
        Uf = add(mul(Uf, 1.0 - wn), mul(ld3(U, m.nc, n), wn));
    } else {
        const int p = m.patch[f];
        if (p >= 0 && (m.ptype[p] == kPatchEmpty || m.ptype[p] == kPatchSymmetry)) return 0.0;
    }
    return rho * dot(Uf, ld3(m.sf, m.nf, f));
}

// Fixed-pressure boundary coefficient and source (:8130-8175 / :2176-2205)
__device__ __forceinline__ void fixed_boundary(const MeshView& m, int f, int o, const double* p, const double* grad,
                                               const double* rau, double rho, double value,
                                               double* coeff, double* source, int* status) {
    const D3 S = ld3(m.sf, m.nf, f);
    const D3 dau{m.vol[o] * rau[o], m.vol[o] * rau[m.nc + o], m.vol[o] * rau[2 * m.nc + o]};
    const FaceTerms t = face_terms(m.geo, m.nf, f, dau, status);
    const double bc = ortho_coefficient(t, status);
    const D3 gp = ld3(grad, m.nc, o);
    const double deferred = nonortho_flux(t, S, dau, gp, status);
    *coeff = bc;
    *source = rho * (bc * (value - p[o]) + deferred);
}

__device__ __forceinline__ bool boundary_fixed(const MeshView& m, const BcView& bc, int f, double* value) {
    const int p = m.patch[f];
    if (p < 0 || p >= bc.n_patches) return false;
    if (!bc.fixed[p]) return false;
    *value = bc.value[p];
    return true;
}

// gauss_gradient_with_boundary (:1634-1744), single sweep, distance weight:
// a thread per cell over its slots in cell-face order.  The slot records give
// the face, the side and the other cell in one load, and the interpolation
// weight of the cell's side comes from the table (no face-centre or
// cell-centre reads, no square roots or divisions per call).
__global__ void k_gauss_gradient(MeshView m, BcView bc, const int2* __restrict__ rec,
                                 const double* __restrict__ wslot, const double* __restrict__ p, double* grad,
                                 int* status) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int b = m.co[c], e = m.co[c + 1];
    const double pc = p[c];
    D3 sum{0.0, 0.0, 0.0};
#pragma unroll 4
    for (int k = b; k < e; ++k) {
        const int2 r = rec[k];
        const int f = r.x & 0x7fffffff;
        D3 S = ld3(m.sf, m.nf, f);
        if (r.x < 0) S = mul(S, -1.0);
        double vf = pc;
        if (r.y >= 0) {
            const double w = wslot[k];
            vf = w * pc + (1.0 - w) * p[r.y];
        } else {
            const int pt = m.patch[f];
            if (pt >= 0 && m.ptype[pt] == kPatchEmpty) continue;
            double v;
            if (boundary_fixed(m, bc, f, &v)) vf = v;
        }
        sum = add(sum, mul(S, vf));
    }
    const double invV = 1.0 / m.vol[c];
    const double gx = sum.x * invV, gy = sum.y * invV, gz = sum.z * invV;
    if (!isfinite(gx) || !isfinite(gy) || !isfinite(gz)) atomicOr(status, kStatusNonFinite);
    grad[c] = gx; grad[m.nc + c] = gy; grad[2 * m.nc + c] = gz;
}

// coeff[k] of a cell's NF slots, k known only at run time: a select over the
// unrolled slots keeps the array in registers
template <int NF>
__device__ __forceinline__ double pick_slot(const double (&a)[NF], int k) {
    double v = a[0];
#pragma unroll
    for (int j = 1; j < NF; ++j)
        if (j == k) v = a[j];
    return v;
}

// Pressure-corrector block (:8048-8181) of cell c: its CSR row and b.
// Continuity is summed in cell-face order, the diagonal and the fixed-pressure
// boundary terms in global face order (the per-cell sorted permutation cs), as
// the reference sums them.  NF > 0: a cell of exactly NF faces, every loop
// unrolled and the face coefficients in registers; NF = 0: up to
// kMaxCellFaces faces, the coefficients in local memory.
template <int NF>
__device__ __forceinline__ void assemble_cell(const MeshView& m, const BcView& bc, const int2* __restrict__ rec,
                                              const double* __restrict__ U, const double* __restrict__ rau,
                                              const double* __restrict__ p, const double* __restrict__ grad,
                                              double rho, const int* __restrict__ slot,
                                              const int* __restrict__ diag_pos, double* __restrict__ values,
                                              double* __restrict__ b, double* __restrict__ phi_out, int* status,
                                              int c, int beg, int nfc) {
    constexpr int kCap = NF > 0 ? NF : kMaxCellFaces;
    const int n_slots = NF > 0 ? NF : nfc;
    double coeff[kCap];
    unsigned interior = 0;
    double cont = 0.0;
#pragma unroll
    for (int k = 0; k < n_slots; ++k) {
        const int2 r = rec[beg + k];
        const int f = r.x & 0x7fffffff;
        const bool own = r.x >= 0;
        const int o = own ? c : r.y, n = own ? r.y : c;
        const double phi = mass_flux(m, f, o, n, U, rho);
        if (phi_out && own) phi_out[f] = phi;
        cont += own ? phi : -phi;
        coeff[k] = 0.0;
        if (r.y >= 0) {
            interior |= 1u << k;
            double ic;
            const double rc = rc_internal(m, f, o, n, p, grad, rau, rho, &ic, status);
            cont += own ? -rc : rc;
            coeff[k] = rho * ic;
        }
    }
    double diag = 0.0;
#pragma unroll
    for (int q = 0; q < n_slots; ++q) {
        const int k = m.cs[beg + q];
        if (interior >> k & 1u) diag += NF > 0 ? pick_slot(coeff, k) : coeff[k];
    }
    double acc = 0.0 + diag;
    double bb = -cont;
    const unsigned all = n_slots >= 32 ? ~0u : (1u << n_slots) - 1u;
    if (interior != all) {
        for (int q = 0; q < n_slots; ++q) {
            const int k = m.cs[beg + q];
            if (interior >> k & 1u) continue;
            const int f = rec[beg + k].x & 0x7fffffff;
            double value;
            if (!boundary_fixed(m, bc, f, &value)) continue;
            double bcoef, source;
            fixed_boundary(m, f, c, p, grad, rau, rho, value, &bcoef, &source, status);
            acc += rho * bcoef;
            bb += source;
        }
    }
    values[diag_pos[c]] = acc;
#pragma unroll
    for (int k = 0; k < n_slots; ++k)
        if (slot[beg + k] >= 0) values[slot[beg + k]] = 0.0 - coeff[k];
    b[c] = bb;
}

// One thread per cell; tetrahedra and hexahedra take the unrolled forms.
// Capped at 64 registers (eight 128-thread blocks per SM instead of six at
// 80): 180 instead of 192 us at 64^3, despite a few spilled registers.
__global__ void __launch_bounds__(kT, 8) k_pressure_assembly(MeshView m, BcView bc, const int2* __restrict__ rec,
                                    const double* __restrict__ U, const double* __restrict__ rau,
                                    const double* __restrict__ p, const double* __restrict__ grad, double rho,
                                    const int* __restrict__ slot, const int* __restrict__ diag_pos,
                                    double* __restrict__ values, double* __restrict__ b,
                                    double* __restrict__ phi_out, int* status) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int beg = m.co[c], nfc = m.co[c + 1] - beg;
    if (nfc > kMaxCellFaces) { atomicOr(status, kStatusGeometry); return; }
    if (nfc == 4)
        assemble_cell<4>(m, bc, rec, U, rau, p, grad, rho, slot, diag_pos, values, b, phi_out, status, c, beg, nfc);
    else if (nfc == 6)
        assemble_cell<6>(m, bc, rec, U, rau, p, grad, rho, slot, diag_pos, values, b, phi_out, status, c, beg, nfc);
    else
        assemble_cell<0>(m, bc, rec, U, rau, p, grad, rho, slot, diag_pos, values, b, phi_out, status, c, beg, nfc);
}

// make_rhie_chow_mass_flux (:2064-2217), HBYA_PREDICTOR, zero-gradient velocity boundaries
__global__ void k_rhie_chow_flux(MeshView m, BcView bc, const double* __restrict__ U,
                                 const double* __restrict__ rau, const double* __restrict__ p,
                                 const double* __restrict__ grad, double rho, double* __restrict__ flux,
                                 int* status) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= m.nf) return;
    const int o = m.owner[f], n = m.neigh[f];
    D3 Hf = ld3(U, m.nc, o);
    double correction = 0.0;
    if (n >= 0) {
        const double wn = 0.5;
        Hf = add(mul(Hf, 1.0 - wn), mul(ld3(U, m.nc, n), wn));
        correction = rc_internal(m, f, o, n, p, grad, rau, rho, nullptr, status);
    } else {
        const int pt = m.patch[f];
        if (pt >= 0 && (m.ptype[pt] == kPatchEmpty || m.ptype[pt] == kPatchSymmetry)) {
            flux[f] = 0.0;
            return;
        }
        double value;
        if (boundary_fixed(m, bc, f, &value)) {
            double bcoef, source;
            fixed_boundary(m, f, o, p, grad, rau, rho, value, &bcoef, &source, status);
            correction = source;
        }
    }
    flux[f] = rho * dot(Hf, ld3(m.sf, m.nf, f)) - correction;
}

// The corrector's geometric face terms (see FaceTerms): d, e and Sf . e with
// dvec = Cn - Co (interior) or Cf - Co (boundary), the operations of
// pressure_face_orthogonal_coefficient (:1914-1935).
__global__ void k_face_terms(int nf, int nc, const int* __restrict__ owner, const int* __restrict__ neigh,
                             const double* __restrict__ fc, const double* __restrict__ sf,
                             const double* __restrict__ cc, double* geo) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int o = owner[f], n = neigh[f];
    const D3 dvec = n >= 0 ? sub(ld3(cc, nc, n), ld3(cc, nc, o)) : sub(ld3(fc, nf, f), ld3(cc, nc, o));
    const double d = mag(dvec);
    const D3 e{dvec.x / d, dvec.y / d, dvec.z / d};
    geo[f] = d;
    geo[nf + f] = e.x;
    geo[2 * nf + f] = e.y;
    geo[3 * nf + f] = e.z;
    geo[4 * nf + f] = dot(ld3(sf, nf, f), e);
}

// Gauss-gradient weight of each interior slot from its cell's side,
// w = dn / (dc + dn) with dc = |Cf - Cc| and dn = |Cother - Cf| (:1660-1700):
// geometry only, so formed once with the geometry.
__global__ void k_slot_weights(int nc, int nf, const int* __restrict__ co, const int2* __restrict__ rec,
                               const double* __restrict__ fc, const double* __restrict__ cc, double* w,
                               int* status) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const D3 ccv = ld3(cc, nc, c);
    for (int k = co[c]; k < co[c + 1]; ++k) {
        const int2 r = rec[k];
        if (r.y < 0) {
            w[k] = 0.0;
            continue;
        }
        const D3 fcv = ld3(fc, nf, r.x & 0x7fffffff);
        const double dc = mag(sub(fcv, ccv));
        const double dn = mag(sub(ld3(cc, nc, r.y), fcv));
        if (!(dc + dn > 0.0)) atomicOr(status, kStatusGeometry);
        w[k] = dn / (dc + dn);
    }
}

// assemble_cell_diffusion_matrix (core/solvers/scalar_diffusion.h:39-163), one thread per cell.
__global__ void k_diffusion_assembly(MeshView m, const double* __restrict__ bcv, const int* __restrict__ bct,
                                     double gamma, const double* __restrict__ source,
                                     const int* __restrict__ slot, const int* __restrict__ diag_pos,
                                     double* __restrict__ values, double* __restrict__ rhs, int* status) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.nc) return;
    const int beg = m.co[c], nfc = m.co[c + 1] - beg;
    double r = source[c] * m.vol[c];
    double diag = 0.0;
    for (int q = 0; q < nfc; ++q) {
        const int k = m.cs[beg + q];
        const int f = m.cf[beg + k];
        const int o = m.owner[f], n = m.neigh[f];
        const double area = mag(ld3(m.sf, m.nf, f));
        if (!(area > 0.0) || !isfinite(area)) atomicOr(status, kStatusGeometry);
        if (n >= 0) {
            const double d = mag(sub(ld3(m.cc, m.nc, n), ld3(m.cc, m.nc, o)));
            if (!(d > 2.220446049250313080847e-16) || !isfinite(d)) atomicOr(status, kStatusGeometry);
            const double g = gamma * area / d;
            diag += g;
            values[slot[beg + k]] = 0.0 + (-g);
        } else if (isfinite(bcv[f])) {
            const double d = mag(sub(ld3(m.fc, m.nf, f), ld3(m.cc, m.nc, o)));
            if (!(d > 2.220446049250313080847e-16) || !isfinite(d)) atomicOr(status, kStatusGeometry);
            const double g = gamma * area / d;
            if (!bct || bct[f] == 0) {
                diag += g;
                r += g * bcv[f];
            } else {
                r += bcv[f] * area;
            }
        }
    }
    values[diag_pos[c]] = 0.0 + diag;
    rhs[c] = r;
}

// The build_hbya step of solve_steady_incompressible (:6430-6465), one
// thread per (cell, component): h = rhs + gradp * V (:6437), minus the
// off-diagonal products of the component's momentum row in CSR order
// (:6438-6443), HbyA = rAU * h (:6459); non-finite HbyA is flagged (:6460).
__global__ void k_build_hbya(int n, const int* __restrict__ ro, const int* __restrict__ co,
                             const double* __restrict__ va0, const double* __restrict__ va1,
                             const double* __restrict__ va2, const double* __restrict__ rhs,
                             const double* __restrict__ U, const double* __restrict__ gradp,
                             const double* __restrict__ vol, const double* __restrict__ rau,
                             double* __restrict__ hbya, int* status) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= 3 * static_cast<int64_t>(n)) return;
    const int d = static_cast<int>(t / n), c = static_cast<int>(t % n);
    const double* va = d == 0 ? va0 : (d == 1 ? va1 : va2);
    const double* Ud = U + static_cast<int64_t>(d) * n;
    double h = rhs[t] + gradp[t] * vol[c];
    for (int k = ro[c]; k < ro[c + 1]; ++k) {
        const int col = co[k];
        if (col != c) h -= va[k] * Ud[col];
    }
    const double v = rau[t] * h;
    hbya[t] = v;
    if (!isfinite(v)) atomicOr(status, kStatusNonFinite);
}

MeshView view(const cfdxg_mesh* m) {
    return {static_cast<int>(m->n_cells), static_cast<int>(m->n_faces), m->cell_off.get(), m->cell_face.get(),
            m->cell_sorted.get(), m->owner.get(), m->neigh.get(), m->patch_of_face.get(), m->patch_type.get(),
            m->face_centre.get(), m->face_sf.get(), m->cell_centre.get(), m->cell_volume.get(),
            m->face_geo.get()};
}

void launch_gradient(cfdxg_context* ctx, const cfdxg_mesh* m, const MeshView& mv, const BcView& bc,
                     const double* p, double* grad) {
    k_gauss_gradient<<<blocks_for(m->n_cells, kT), kT, 0, ctx->stream>>>(mv, bc, m->slot_rec.get(), m->slot_w.get(),
                                                                        p, grad, ctx->scratch.status);
    check_launch(ctx);
}

// The face-loop tables of the mesh (slot records, gradient weights, face
// terms); called by the geometry build, after the geometry.
void build_face_tables(cfdxg_context* ctx, cfdxg_mesh* m) {
    const int64_t nc = m->n_cells, nf = m->n_faces, nslot = static_cast<int64_t>(m->h_cell_face.size());
    std::vector<int2> rec(nslot);
    for (int64_t c = 0; c < nc; ++c)
        for (int64_t k = m->h_cell_off[c]; k < m->h_cell_off[c + 1]; ++k) {
            const int64_t f = m->h_cell_face[k];
            const bool own = m->h_owner[f] == c;
            const int64_t n = m->h_neigh[f];
            rec[k].x = static_cast<int>(f) | (own ? 0 : kOtherSide);
            rec[k].y = n < 0 ? -1 : static_cast<int>(own ? n : m->h_owner[f]);
        }
    m->slot_rec.upload(rec, ctx->stream);
    m->slot_w.resize(static_cast<std::size_t>(nslot));
    k_slot_weights<<<blocks_for(nc, kT), kT, 0, ctx->stream>>>(
        static_cast<int>(nc), static_cast<int>(nf), m->cell_off.get(), m->slot_rec.get(), m->face_centre.get(),
        m->cell_centre.get(), m->slot_w.get(), ctx->scratch.status);
    check_launch(ctx);
    m->face_geo.resize(static_cast<std::size_t>(kFaceTermArrays) * nf);
    k_face_terms<<<blocks_for(nf, kT), kT, 0, ctx->stream>>>(static_cast<int>(nf), static_cast<int>(nc),
                                                             m->owner.get(), m->neigh.get(), m->face_centre.get(),
                                                             m->face_sf.get(), m->cell_centre.get(),
                                                             m->face_geo.get());
    check_launch(ctx);
}

// Algorithmic (compulsory) bytes of the face-loop kernels, FP64 values and
// 32-bit indices, each array read or written once:
//   Gauss gradient: per face owner + neighbour (8), Sf (24); per cell p (8),
//   grad out (24)
//   pressure assembly: per face owner + neighbour (8), Sf (24), phiHbyA out (8);
//   per cell centre (24), volume (8), rAU (8, one component), p (8), grad (24),
//   b out (8); CSR values out (8 per nonzero)
//   Rhie-Chow flux: per face owner + neighbour (8), Sf (24), flux out (8);
//   per cell HbyA (24), rAU (24), p (8), grad (24), centre (24), volume (8)
double gradient_bytes(const cfdxg_mesh* m) { return 32.0 * m->n_faces + 32.0 * m->n_cells; }
double assembly_bytes(const cfdxg_mesh* m, int64_t nnz) {
    return 40.0 * m->n_faces + 72.0 * m->n_cells + 8.0 * nnz + 8.0 * m->n_cells;
}
double flux_bytes(const cfdxg_mesh* m) { return 40.0 * m->n_faces + 112.0 * m->n_cells; }

void require_geometry(const cfdxg_mesh* m) {
    if (!m->geometry_ready) throw Error(CFDXG_ERR_NOT_READY, "geometry not built: call cfdxg_geometry_build");
}

void check_device_status(cfdxg_context* ctx, const char* what) {
    const int st = read_status(ctx);
    if (st & kStatusGeometry) throw Error(CFDXG_ERR_GEOMETRY, std::string(what) + ": invalid or inconsistent face geometry");
    if (st & kStatusNonFinite) throw Error(CFDXG_ERR_NONFINITE, std::string(what) + ": non-finite result");
}

// CSR pattern of the cell graph (one entry per neighbour plus the diagonal),
// built once per mesh on the host.
void build_pattern(cfdxg_context* ctx, cfdxg_mesh* m) {
    MeshPattern& P = m->pattern;
    if (P.built) return;
    const int64_t nc = m->n_cells;
    P.ro.assign(nc + 1, 0);
    P.co.clear();
    std::vector<int> slot(m->h_cell_face.size(), -1), diag(nc, 0);
    std::vector<std::pair<uint32_t, int>> row;   // (column, local face or -1)
    for (int64_t c = 0; c < nc; ++c) {
        row.clear();
        row.emplace_back(static_cast<uint32_t>(c), -1);
        for (int64_t k = m->h_cell_off[c]; k < m->h_cell_off[c + 1]; ++k) {
            const int64_t f = m->h_cell_face[k];
            const int64_t n = m->h_neigh[f];
            if (n < 0) continue;
            const int64_t other = m->h_owner[f] == c ? n : m->h_owner[f];
            row.emplace_back(static_cast<uint32_t>(other), static_cast<int>(k - m->h_cell_off[c]));
        }
        std::sort(row.begin(), row.end());
        for (std::size_t q = 1; q < row.size(); ++q)
            if (row[q].first == row[q - 1].first)
                throw Error(CFDXG_ERR_GEOMETRY, "two faces join the same pair of cells (unsupported)");
        for (const auto& [col, local] : row) {
            const int pos = static_cast<int>(P.co.size());
            if (local < 0) diag[c] = pos;
            else slot[m->h_cell_off[c] + local] = pos;
            P.co.push_back(col);
        }
        P.ro[c + 1] = static_cast<uint32_t>(P.co.size());
    }
    P.nnz = static_cast<int64_t>(P.co.size());
    std::vector<int> ro(P.ro.begin(), P.ro.end()), co(P.co.begin(), P.co.end());
    P.d_ro.upload(ro, ctx->stream);
    P.d_co.upload(co, ctx->stream);
    P.d_slot.upload(slot, ctx->stream);
    P.d_diag.upload(diag, ctx->stream);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    P.built = true;
}

cfdxg_matrix* new_pattern_matrix(cfdxg_context* ctx, cfdxg_mesh* m) {
    build_pattern(ctx, m);
    auto* A = new cfdxg_matrix();
    A->n = m->n_cells;
    A->nnz = m->pattern.nnz;
    A->ro.resize(A->n + 1);
    A->co.resize(A->nnz);
    CFDXG_CUDA(cudaMemcpyAsync(A->ro.get(), m->pattern.d_ro.get(), sizeof(int) * (A->n + 1), cudaMemcpyDeviceToDevice, ctx->stream));
    CFDXG_CUDA(cudaMemcpyAsync(A->co.get(), m->pattern.d_co.get(), sizeof(int) * A->nnz, cudaMemcpyDeviceToDevice, ctx->stream));
    A->va.resize(A->nnz);
    A->host.n = A->n;
    A->host.ro.assign(m->pattern.ro.begin(), m->pattern.ro.end());
    A->host.co.assign(m->pattern.co.begin(), m->pattern.co.end());
    A->host_values_valid = false;
    A->mesh = m;
    return A;
}

}  // namespace
}  // namespace cfdxg

using namespace cfdxg;

extern "C" int cfdxg_mesh_upload(cfdxg_context* ctx, const cfdxg_mesh_desc* d, cfdxg_mesh** out) {
    if (!ctx) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    if (!d || !out || d->n_faces <= 0 || d->n_cells <= 0 || d->n_points <= 0 || !d->px || !d->py || !d->pz ||
        !d->face_offsets || !d->face_vertices || !d->owner || !d->neighbour || !d->cell_offsets ||
        !d->cell_faces || (d->n_patches > 0 && !d->patch_types))
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "mesh descriptor is incomplete");
    if (d->n_faces > INT32_MAX / 2 || d->n_cells > INT32_MAX / 2 || d->n_points > INT32_MAX / 2)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "mesh too large for 32-bit device indices");
    auto m = std::make_unique<cfdxg_mesh>();
    m->n_points = d->n_points; m->n_faces = d->n_faces; m->n_cells = d->n_cells; m->n_patches = d->n_patches;
    const int64_t nf = d->n_faces, nc = d->n_cells, np = d->n_points;
    const int64_t nfv = d->face_offsets[nf], ncf = d->cell_offsets[nc];
    if (d->face_offsets[0] != 0 || d->cell_offsets[0] != 0 || nfv <= 0 || ncf <= 0)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "invalid CSR offsets");
    std::vector<int> fo(nf + 1), fv(nfv), own(nf), nb(nf), co(nc + 1), cf(ncf), sorted(ncf), pf(nf, -1), pt;
    for (int64_t f = 0; f <= nf; ++f) {
        fo[f] = static_cast<int>(d->face_offsets[f]);
        if (f && fo[f] < fo[f - 1]) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "face offsets not monotone");
    }
    for (int64_t q = 0; q < nfv; ++q) {
        if (d->face_vertices[q] < 0 || d->face_vertices[q] >= np) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "face vertex out of range");
        fv[q] = static_cast<int>(d->face_vertices[q]);
    }
    int64_t n_internal = 0;
    for (int64_t f = 0; f < nf; ++f) {
        if (d->owner[f] < 0 || d->owner[f] >= nc || d->neighbour[f] >= nc)
            throw Error(CFDXG_ERR_INVALID_ARGUMENT, "owner/neighbour out of range");
        own[f] = static_cast<int>(d->owner[f]);
        nb[f] = d->neighbour[f] < 0 ? -1 : static_cast<int>(d->neighbour[f]);
        if (nb[f] >= 0) ++n_internal;
        if (d->patch_of_face) {
            pf[f] = d->patch_of_face[f];
            if (pf[f] >= d->n_patches) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "patch id out of range");
        }
    }
    int maxf = 0;
    for (int64_t c = 0; c <= nc; ++c) {
        co[c] = static_cast<int>(d->cell_offsets[c]);
        if (c && co[c] < co[c - 1]) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "cell offsets not monotone");
        if (c) maxf = std::max(maxf, co[c] - co[c - 1]);
    }
    if (maxf > kMaxCellFaces) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "cells with more than 16 faces are not supported");
    std::vector<int> local;
    for (int64_t c = 0; c < nc; ++c) {
        local.resize(co[c + 1] - co[c]);
        for (int k = co[c]; k < co[c + 1]; ++k) {
            const int64_t f = d->cell_faces[k];
            if (f < 0 || f >= nf) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "cell face out of range");
            if (own[f] != c && nb[f] != c) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "cell face not attached to its cell");
            cf[k] = static_cast<int>(f);
        }
        std::iota(local.begin(), local.end(), 0);
        std::stable_sort(local.begin(), local.end(), [&](int a, int b) { return cf[co[c] + a] < cf[co[c] + b]; });
        for (std::size_t r = 0; r < local.size(); ++r) sorted[co[c] + r] = local[r];
    }
    for (int32_t p = 0; p < d->n_patches; ++p) pt.push_back(d->patch_types[p]);
    if (pt.empty()) pt.push_back(0);
    cudaStream_t s = ctx->stream;
    m->px.upload(d->px, np, s); m->py.upload(d->py, np, s); m->pz.upload(d->pz, np, s);
    m->face_off.upload(fo, s); m->face_vert.upload(fv, s); m->owner.upload(own, s); m->neigh.upload(nb, s);
    m->cell_off.upload(co, s); m->cell_face.upload(cf, s); m->cell_sorted.upload(sorted, s);
    m->patch_of_face.upload(pf, s); m->patch_type.upload(pt, s);
    m->n_internal = n_internal;
    m->max_cell_faces = maxf;
    m->h_owner.assign(d->owner, d->owner + nf);
    m->h_neigh.assign(d->neighbour, d->neighbour + nf);
    for (auto& v : m->h_neigh) if (v < 0) v = -1;
    m->h_cell_off.assign(d->cell_offsets, d->cell_offsets + nc + 1);
    m->h_cell_face.assign(d->cell_faces, d->cell_faces + ncf);
    m->h_patch_types.assign(pt.begin(), pt.end());
    CFDXG_CUDA(cudaStreamSynchronize(s));
    *out = m.release();
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_mesh_destroy(cfdxg_mesh* mesh) {
    delete mesh;
    return CFDXG_OK;
}

extern "C" int cfdxg_geometry_build(cfdxg_context* ctx, cfdxg_mesh* m) {
    if (!ctx || !m) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    cudaStream_t s = ctx->stream;
    const int nf = static_cast<int>(m->n_faces), nc = static_cast<int>(m->n_cells);
    m->face_centre.resize(3 * static_cast<size_t>(nf));
    m->face_sf.resize(3 * static_cast<size_t>(nf));
    m->cell_centre.resize(3 * static_cast<size_t>(nc));
    m->cell_volume.resize(nc);
    clear_status(ctx);
    int* st = ctx->scratch.status;
    k_face_geometry<<<blocks_for(nf, kT), kT, 0, s>>>(nf, m->face_off.get(), m->face_vert.get(), m->px.get(),
                                                      m->py.get(), m->pz.get(), m->face_centre.get(),
                                                      m->face_sf.get(), st);
    check_launch(ctx);
    // first pass: centres with the raw face vectors signed by ownership
    k_cell_geometry<<<blocks_for(nc, kT), kT, 0, s>>>(nc, nf, m->cell_off.get(), m->cell_face.get(), m->owner.get(),
                                                      m->face_centre.get(), m->face_sf.get(), m->cell_centre.get(),
                                                      m->cell_volume.get(), st);
    check_launch(ctx);
    k_orient<<<blocks_for(nf, kT), kT, 0, s>>>(nf, nc, m->owner.get(), m->neigh.get(), m->face_centre.get(),
                                               m->cell_centre.get(), m->face_sf.get());
    check_launch(ctx);
    // second pass with owner-oriented face vectors
    k_cell_geometry<<<blocks_for(nc, kT), kT, 0, s>>>(nc, nf, m->cell_off.get(), m->cell_face.get(), m->owner.get(),
                                                      m->face_centre.get(), m->face_sf.get(), m->cell_centre.get(),
                                                      m->cell_volume.get(), st);
    check_launch(ctx);
    build_face_tables(ctx, m);
    check_device_status(ctx, "geometry");
    m->geometry_ready = true;
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_geometry_download(cfdxg_context* ctx, const cfdxg_mesh* m, double* fc, double* sf, double* cc,
                                       double* cv) {
    if (!ctx || !m) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    require_geometry(m);
    if (fc) m->face_centre.download(fc, ctx->stream);
    if (sf) m->face_sf.download(sf, ctx->stream);
    if (cc) m->cell_centre.download(cc, ctx->stream);
    if (cv) m->cell_volume.download(cv, ctx->stream);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_assemble_cell_diffusion(cfdxg_context* ctx, cfdxg_mesh* m, const double* bc_values,
                                             const int32_t* bc_types, double gamma, const double* source,
                                             int32_t mem, cfdxg_matrix** A_out, double* rhs) {
    if (!ctx || !m) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    check_mem_flag(mem);
    if (!A_out || !rhs || !source || !bc_values) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "missing argument");
    if (!(gamma > 0.0) || !std::isfinite(gamma)) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "diffusivity must be positive");
    require_geometry(m);
    const int64_t nf = m->n_faces, nc = m->n_cells;
    In<double> bv(ctx, bc_values, nf, mem), src(ctx, source, nc, mem);
    In<int32_t> bt(ctx, bc_types, bc_types ? nf : 0, mem);
    Out<double> r(ctx, rhs, nc, mem);
    std::unique_ptr<cfdxg_matrix> A(new_pattern_matrix(ctx, m));
    clear_status(ctx);
    k_diffusion_assembly<<<blocks_for(nc, kT), kT, 0, ctx->stream>>>(view(m), bv.get(), bt.get(), gamma, src.get(),
                                                                     m->pattern.d_slot.get(), m->pattern.d_diag.get(),
                                                                     A->va.get(), r.get(), ctx->scratch.status);
    check_launch(ctx);
    r.finish();
    check_device_status(ctx, "assemble_cell_diffusion_matrix");
    *A_out = A.release();
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

namespace {
// Per-patch fixed-pressure table in the mesh's own device buffers.
BcView make_bc(cfdxg_context* ctx, cfdxg_mesh* m, const int32_t* fixed, const double* value) {
    const int np = std::max<int>(1, m->n_patches);
    std::vector<int> f(np, 0);
    std::vector<double> v(np, 0.0);
    for (int p = 0; p < m->n_patches; ++p) {
        f[p] = fixed ? fixed[p] : 0;
        v[p] = value ? value[p] : 0.0;
    }
    m->bc_fixed.upload(f, ctx->stream);
    m->bc_value.upload(v, ctx->stream);
    return {m->bc_fixed.get(), m->bc_value.get(), static_cast<int>(m->n_patches)};
}

double* gradient_scratch(cfdxg_mesh* m) {
    m->grad_scratch.resize(3 * static_cast<std::size_t>(m->n_cells));
    return m->grad_scratch.get();
}
}  // namespace

extern "C" int cfdxg_gauss_gradient(cfdxg_context* ctx, cfdxg_mesh* m, const double* p, const int32_t* fixed,
                                    const double* value, int32_t mem, double* grad) {
    if (!ctx || !m) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    check_mem_flag(mem);
    require_geometry(m);
    if (!p || !grad) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "missing argument");
    const int64_t nc = m->n_cells;
    const BcView bc = make_bc(ctx, m, fixed, value);
    In<double> pin(ctx, p, nc, mem);
    Out<double> g(ctx, grad, 3 * nc, mem);
    clear_status(ctx);
    {
        ProfScope ps(ctx, "gauss_gradient", gradient_bytes(m));
        launch_gradient(ctx, m, view(m), bc, pin.get(), g.get());
    }
    g.finish();
    check_device_status(ctx, "gauss_gradient_with_boundary");
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_assemble_pressure_correction(cfdxg_context* ctx, cfdxg_mesh* m, const double* HbyA,
                                                  const double* rAU, const double* p, double rho,
                                                  const int32_t* fixed, const double* value, int32_t mem,
                                                  cfdxg_matrix** A_inout, double* b, double* phiHbyA,
                                                  double* grad_p) {
    if (!ctx || !m) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    NvtxRange nvtx_range("cfdxg.assemble_pressure_correction");
    check_mem_flag(mem);
    require_geometry(m);
    if (!HbyA || !rAU || !p || !A_inout || !b) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "missing argument");
    if (!std::isfinite(rho) || !(rho > 0.0)) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "density must be positive");
    const int64_t nc = m->n_cells, nf = m->n_faces;
    const BcView bc = make_bc(ctx, m, fixed, value);
    In<double> U(ctx, HbyA, 3 * nc, mem), rau(ctx, rAU, 3 * nc, mem), pin(ctx, p, nc, mem);
    Out<double> bout(ctx, b, nc, mem), phi(ctx, phiHbyA, phiHbyA ? nf : 0, mem);
    Out<double> gout(ctx, grad_p, grad_p ? 3 * nc : 0, mem);
    double* g = gout.get();
    if (!g) g = gradient_scratch(m);
    std::unique_ptr<cfdxg_matrix> fresh;
    cfdxg_matrix* A = *A_inout;
    if (!A) {
        fresh.reset(new_pattern_matrix(ctx, m));
        A = fresh.get();
    } else if (A->mesh != m) {
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "matrix was not assembled on this mesh");
    }
    clear_status(ctx);
    const MeshView mv = view(m);
    {
        ProfScope ps(ctx, "gauss_gradient", gradient_bytes(m));
        launch_gradient(ctx, m, mv, bc, pin.get(), g);
    }
    {
        ProfScope ps(ctx, "pressure_assembly", assembly_bytes(m, A->nnz));
        k_pressure_assembly<<<blocks_for(nc, kT), kT, 0, ctx->stream>>>(mv, bc, m->slot_rec.get(), U.get(), rau.get(),
                                                                        pin.get(), g, rho, m->pattern.d_slot.get(),
                                                                        m->pattern.d_diag.get(), A->va.get(),
                                                                        bout.get(), phi.get(), ctx->scratch.status);
        check_launch(ctx);
    }
    bout.finish();
    phi.finish();
    gout.finish();
    check_device_status(ctx, "pressure-correction assembly");
    A->host_values_valid = false;
    if (fresh) *A_inout = fresh.release();
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_rhie_chow_flux(cfdxg_context* ctx, cfdxg_mesh* m, const double* HbyA, const double* rAU,
                                    const double* p, double rho, const int32_t* fixed, const double* value,
                                    int32_t mem, double* flux) {
    if (!ctx || !m) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    NvtxRange nvtx_range("cfdxg.rhie_chow_flux");
    check_mem_flag(mem);
    require_geometry(m);
    if (!HbyA || !rAU || !p || !flux) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "missing argument");
    const int64_t nc = m->n_cells, nf = m->n_faces;
    const BcView bc = make_bc(ctx, m, fixed, value);
    In<double> U(ctx, HbyA, 3 * nc, mem), rau(ctx, rAU, 3 * nc, mem), pin(ctx, p, nc, mem);
    Out<double> fl(ctx, flux, nf, mem);
    double* g = gradient_scratch(m);
    clear_status(ctx);
    const MeshView mv = view(m);
    {
        ProfScope ps(ctx, "gauss_gradient", gradient_bytes(m));
        launch_gradient(ctx, m, mv, bc, pin.get(), g);
    }
    {
        ProfScope ps(ctx, "rhie_chow_flux", flux_bytes(m));
        k_rhie_chow_flux<<<blocks_for(nf, kT), kT, 0, ctx->stream>>>(mv, bc, U.get(), rau.get(), pin.get(),
                                                                     g, rho, fl.get(), ctx->scratch.status);
        check_launch(ctx);
    }
    fl.finish();
    check_device_status(ctx, "make_rhie_chow_mass_flux");
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

// ---------------------------------------------------------------------------
// cfdxg_rhie_chow_flux_noalloc: the Rhie-Chow face flux with its scratch in a
// static device array, for callers that cannot allocate device memory.
namespace cfdxg {
namespace {

constexpr int kNoAllocMaxCells = 1 << 18;   // 262,144 cells
constexpr int kNoAllocMaxPatches = 32;
// layout: [3 * kNoAllocMaxCells doubles: gradient SoA][32 doubles: patch value][32 ints: patch fixed flag]
constexpr std::size_t kNoAllocGradBytes = sizeof(double) * 3 * kNoAllocMaxCells;
constexpr std::size_t kNoAllocBytes = kNoAllocGradBytes + sizeof(double) * kNoAllocMaxPatches +
                                      sizeof(int) * kNoAllocMaxPatches;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct PatchTable {
    int n;
    int fixed[kNoAllocMaxPatches];
    double value[kNoAllocMaxPatches];
};

__global__ void k_fill_patch_table(PatchTable t, int* fixed, double* value) {
    const int k = threadIdx.x;
    if (k < kNoAllocMaxPatches) {
        fixed[k] = k < t.n ? t.fixed[k] : 0;
        value[k] = k < t.n ? t.value[k] : 0.0;
    }
}

// Device address of g_noalloc_scratch in the calling thread's current context.
// Looked up on every call rather than cached: the address belongs to the
// module as loaded in that context, and a context that is destroyed and made
// again (cudaDeviceReset, or a driver-API context made current by the caller)
// loads the module at another address.  The lookup allocates nothing.
void* noalloc_scratch_address() {
    void* ptr = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (rc != cudaSuccess || !ptr)
        throw Error(CFDXG_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") +
                                        cudaGetErrorString(rc));
    return ptr;
}

// Makes the context's device current for the call and gives the caller's
// current device back on every exit path.
class CurrentDevice {
public:
    explicit CurrentDevice(int device) {
        CFDXG_CUDA(cudaGetDevice(&saved_));
        if (saved_ != device) CFDXG_CUDA(cudaSetDevice(device));
        switched_ = saved_ != device;
    }
    ~CurrentDevice() {
        if (switched_) cudaSetDevice(saved_);
    }
    CurrentDevice(const CurrentDevice&) = delete;
    CurrentDevice& operator=(const CurrentDevice&) = delete;

private:
    int saved_ = 0;
    bool switched_ = false;
};

}  // namespace
}  // namespace cfdxg

extern "C" int cfdxg_rhie_chow_flux_noalloc(cfdxg_context* ctx, cfdxg_mesh* m, const double* HbyA,
                                            const double* rAU, const double* p, double rho,
                                            const int32_t* fixed, const double* value, double* flux) {
    if (!ctx || !m) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    require_geometry(m);
    if (!HbyA || !rAU || !p || !flux) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "missing argument");
    if (m->n_cells > kNoAllocMaxCells)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT,
                    "cfdxg_rhie_chow_flux_noalloc: the mesh has " + std::to_string(m->n_cells) +
                        " cells; its static scratch holds at most " + std::to_string(kNoAllocMaxCells));
    if (m->n_patches > kNoAllocMaxPatches)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT,
                    "cfdxg_rhie_chow_flux_noalloc: at most 32 boundary patches are supported");
    const CurrentDevice on_device(ctx->device);
    auto* base = static_cast<unsigned char*>(noalloc_scratch_address());
    double* grad = reinterpret_cast<double*>(base);
    double* tvalue = reinterpret_cast<double*>(base + kNoAllocGradBytes);
    int* tfixed = reinterpret_cast<int*>(base + kNoAllocGradBytes + sizeof(double) * kNoAllocMaxPatches);
    PatchTable t{};
    t.n = m->n_patches;
    for (int k = 0; k < m->n_patches; ++k) {
        t.fixed[k] = fixed ? fixed[k] : 0;
        t.value[k] = value ? value[k] : 0.0;
    }
    const int64_t nc = m->n_cells, nf = m->n_faces;
    clear_status(ctx);
    k_fill_patch_table<<<1, kNoAllocMaxPatches, 0, ctx->stream>>>(t, tfixed, tvalue);
    check_launch(ctx);
    const BcView bc{tfixed, tvalue, static_cast<int>(m->n_patches)};
    const MeshView mv = view(m);
    launch_gradient(ctx, m, mv, bc, p, grad);
    k_rhie_chow_flux<<<blocks_for(nf, kT), kT, 0, ctx->stream>>>(mv, bc, HbyA, rAU, p, grad, rho, flux,
                                                                 ctx->scratch.status);
    check_launch(ctx);
    check_device_status(ctx, "make_rhie_chow_mass_flux (no-alloc)");
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_build_hbya(cfdxg_context* ctx, cfdxg_mesh* m, const cfdxg_matrix* const* momentum,
                                const double* rhs, const double* U, const double* gradp, const double* rAU,
                                int32_t mem, double* HbyA) {
    if (!ctx || !m) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    NvtxRange nvtx_range("cfdxg.build_hbya");
    check_mem_flag(mem);
    require_geometry(m);
    if (!momentum || !rhs || !U || !gradp || !rAU || !HbyA)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "missing argument");
    const int64_t nc = m->n_cells;
    for (int d = 0; d < 3; ++d) {
        const cfdxg_matrix* M = momentum[d];
        if (!M || M->n != nc) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "momentum matrix size differs from the mesh");
        if (d > 0 && (M->nnz != momentum[0]->nnz || M->host.ro != momentum[0]->host.ro ||
                      M->host.co != momentum[0]->host.co))
            throw Error(CFDXG_ERR_INVALID_ARGUMENT, "the three momentum matrices must share one pattern");
    }
    In<double> b(ctx, rhs, 3 * nc, mem), u(ctx, U, 3 * nc, mem), gp(ctx, gradp, 3 * nc, mem),
        rau(ctx, rAU, 3 * nc, mem);
    Out<double> out(ctx, HbyA, 3 * nc, mem);
    clear_status(ctx);
    {
        // momentum values of three components + pattern, rhs/U/gradp/rAU reads, V, HbyA write
        ProfScope ps(ctx, "build_hbya", 3.0 * 8.0 * momentum[0]->nnz + 4.0 * (nc + 1) + 4.0 * momentum[0]->nnz +
                                            (4 * 24.0 + 8.0 + 24.0) * nc);
        k_build_hbya<<<blocks_for(3 * nc, kT), kT, 0, ctx->stream>>>(
            static_cast<int>(nc), momentum[0]->ro.get(), momentum[0]->co.get(), momentum[0]->va.get(),
            momentum[1]->va.get(), momentum[2]->va.get(), b.get(), u.get(), gp.get(), m->cell_volume.get(),
            rau.get(), out.get(), ctx->scratch.status);
        check_launch(ctx);
    }
    out.finish();
    const int st = read_status(ctx);
    if (st & kStatusNonFinite) throw Error(CFDXG_ERR_NONFINITE, "solve_steady_incompressible: non-finite HbyA");
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}
