// ref_simple.cpp -- oracle adapter: SIMPLE pressure-correction assembly and
// Rhie-Chow face flux through the reference's own physics functions.
//
// TEST INFRASTRUCTURE ONLY (see ref_abi.h).  build_fv_geometry, make_mass_flux,
// gauss_gradient_with_boundary, rhie_chow_pressure_flux_internal,
// pressure_face_orthogonal_coefficient, pressure_face_nonorthogonal_flux and
// make_rhie_chow_mass_flux are the reference's inline functions, called as-is.
// The corrector block of solve_steady_incompressible
// (physics/steady_incompressible_solver.h:8048-8181, 8605-8608) is not a
// callable symbol; ref_simple_assemble restates it line by line around those
// calls for the default controls (SIMPLE, no compensated assembly, no skew
// correction, no projected interpolation, fixed-pressure boundary present).
#include "cfdx/physics/steady_incompressible_solver.h"

#include "ref_common.h"

using namespace cfdx::core;
using namespace cfdx::physics;

namespace {

ScalarBoundaryConditions make_pressure_bcs(const ref_mesh_t& m, const int32_t* fixed,
                                           const double* value) {
    ScalarBoundaryConditions bcs;
    for (int32_t p = 0; p < m.n_patches; ++p) {
        ScalarBoundaryCondition bc;
        bc.type = fixed[p] ? ScalarBoundaryType::FIXED_VALUE : ScalarBoundaryType::ZERO_GRADIENT;
        bc.value = value[p];
        bcs["p" + std::to_string(p)] = bc;
    }
    return bcs;
}

Field<double, Location::CELL> make_vector_field(const double* soa, std::size_t n) {
    Field<double, Location::CELL> U(n, "HbyA", "m/s", 3);
    for (std::size_t d = 0; d < 3; ++d)
        for (std::size_t c = 0; c < n; ++c) U.component_data(d)[c] = soa[d * n + c];
    return U;
}

Field<double, Location::CELL> make_scalar_field(const double* v, std::size_t n) {
    Field<double, Location::CELL> p(n, "p", "Pa", 1);
    for (std::size_t c = 0; c < n; ++c) p(c) = v[c];
    return p;
}

std::array<std::vector<double>, 3> make_rau(const double* soa, std::size_t n) {
    std::array<std::vector<double>, 3> r;
    for (std::size_t d = 0; d < 3; ++d) r[d].assign(soa + d * n, soa + (d + 1) * n);
    return r;
}

}  // namespace

extern "C" int ref_fv_geometry(const ref_mesh_t* m, double* fc, double* sf, double* cc, double* cv) {
    try {
        const Mesh mesh = cfdx_ref::make_mesh(*m);
        const FvGeometry g = build_fv_geometry(mesh);
        const std::size_t nf = mesh.n_faces(), nc = mesh.n_cells();
        for (std::size_t f = 0; f < nf; ++f) {
            fc[f] = g.face_centres[f].x; fc[nf + f] = g.face_centres[f].y; fc[2 * nf + f] = g.face_centres[f].z;
            sf[f] = g.face_area_vectors[f].x; sf[nf + f] = g.face_area_vectors[f].y; sf[2 * nf + f] = g.face_area_vectors[f].z;
        }
        for (std::size_t c = 0; c < nc; ++c) {
            cc[c] = g.cell_centres[c].x; cc[nc + c] = g.cell_centres[c].y; cc[2 * nc + c] = g.cell_centres[c].z;
            cv[c] = g.cell_volumes[c];
        }
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

extern "C" int ref_gauss_gradient(const ref_mesh_t* m, const double* p, const int32_t* fixed,
                                  const double* value, double* grad) {
    try {
        const Mesh mesh = cfdx_ref::make_mesh(*m);
        const FvGeometry g = build_fv_geometry(mesh);
        const auto bcs = make_pressure_bcs(*m, fixed, value);
        const auto pf = make_scalar_field(p, mesh.n_cells());
        const auto gp = gauss_gradient_with_boundary(pf, mesh, g, bcs, false, false);
        const std::size_t nc = mesh.n_cells();
        for (std::size_t d = 0; d < 3; ++d)
            for (std::size_t c = 0; c < nc; ++c) grad[d * nc + c] = gp.component_data(d)[c];
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

extern "C" int64_t ref_simple_assemble(const ref_mesh_t* m, const double* HbyA_soa,
                                       const double* rAU_soa, const double* p_in, double rho,
                                       const int32_t* fixed, const double* value,
                                       double* phi_out, double* grad_out, int64_t* ro,
                                       int64_t* co, double* va, double* b_out, double* seconds) {
    try {
        const Mesh mesh = cfdx_ref::make_mesh(*m);
        const FvGeometry geometry = build_fv_geometry(mesh);
        const std::size_t nc = mesh.n_cells();
        const auto pressure_bcs = make_pressure_bcs(*m, fixed, value);
        const VelocityBoundaryConditions velocity_bcs;
        const auto HbyA = make_vector_field(HbyA_soa, nc);
        const auto p = make_scalar_field(p_in, nc);
        const auto rAU = make_rau(rAU_soa, nc);

        const double t0 = cfdx_ref::now_seconds();
        // :7894 phiHbyA = make_mass_flux(HbyA)
        const auto phiHbyA = make_mass_flux(mesh, geometry, HbyA, rho, velocity_bcs, {}, false, nullptr);

        // :6485-6500 directional_face_coefficient
        const auto directional_face_coefficient =
            [&](const std::array<std::vector<double>, 3>& coeff, std::size_t f, std::size_t o,
                std::size_t n, const Vec3& Sf, const Vec3& dvec) {
                const double wn = pressure_face_neighbour_weight(geometry, f, o, n, false);
                const double wo = 1.0 - wn;
                const double cx = wo * geometry.cell_volumes[o] * coeff[0][o] + wn * geometry.cell_volumes[n] * coeff[0][n];
                const double cy = wo * geometry.cell_volumes[o] * coeff[1][o] + wn * geometry.cell_volumes[n] * coeff[1][n];
                const double cz = wo * geometry.cell_volumes[o] * coeff[2][o] + wn * geometry.cell_volumes[n] * coeff[2][n];
                return pressure_face_orthogonal_coefficient(Sf, dvec, {cx, cy, cz});
            };

        // :8048-8181 one corrector, default (non-compensated) path
        SparseMatrix A(nc, nc);
        Vector b(nc, 0.0);
        std::vector<std::map<std::size_t, double>> rows(nc);
        std::vector<double> diag(nc, 0.0);
        std::vector<double> continuity(nc, 0.0);
        const auto current_grad_p = gauss_gradient_with_boundary(p, mesh, geometry, pressure_bcs, false, false);
        const auto* cell_faces = mesh.cells().faces_data();
        const auto* cell_offsets = mesh.cells().offsets_data();
        for (std::size_t c = 0; c < nc; ++c) {
            const Offset off = cell_offsets[c];
            const Offset count = cell_offsets[c + 1] - off;
            for (Offset k = 0; k < count; ++k) {
                const std::size_t f = cell_faces[off + k];
                continuity[c] += mesh.ownership().owner(f) == c ? phiHbyA(f) : -phiHbyA(f);
                if (mesh.ownership().neighbour(f) >= 0) {
                    const double phi_nonorth = rhie_chow_pressure_flux_internal(
                        mesh, geometry, f, p, current_grad_p, rAU, rho, false);
                    continuity[c] += mesh.ownership().owner(f) == c ? -phi_nonorth : phi_nonorth;
                }
            }
        }
        for (std::size_t f = 0; f < mesh.n_faces(); ++f) {
            const auto nr = mesh.ownership().neighbour(f);
            if (nr < 0) continue;
            const std::size_t o = mesh.ownership().owner(f);
            const std::size_t n = static_cast<std::size_t>(nr);
            const Vec3 Sf = geometry.face_area_vectors[f];
            const Vec3 dvec = geometry.cell_centres[n] - geometry.cell_centres[o];
            const double coeff = rho * directional_face_coefficient(rAU, f, o, n, Sf, dvec);
            diag[o] += coeff;
            diag[n] += coeff;
            rows[o][n] -= coeff;
            rows[n][o] -= coeff;
        }
        for (std::size_t c = 0; c < nc; ++c) {
            rows[c][c] += diag[c];
            b(c) = -continuity[c];
        }
        for (std::size_t f = 0; f < mesh.n_faces(); ++f) {
            if (mesh.ownership().neighbour(f) >= 0) continue;
            const std::size_t patch = geometry.face_patch[f];
            if (patch >= mesh.boundary().n_patches()) continue;
            const auto& name = mesh.boundary().patch(patch).name;
            const auto it = pressure_bcs.find(name);
            if (it == pressure_bcs.end() || it->second.type != ScalarBoundaryType::FIXED_VALUE) continue;
            const std::size_t o = mesh.ownership().owner(f);
            const Vec3 dvec = geometry.face_centres[f] - geometry.cell_centres[o];
            const Vec3 Sf = geometry.face_area_vectors[f];
            const Vec3 dAU_boundary{geometry.cell_volumes[o] * rAU[0][o],
                                    geometry.cell_volumes[o] * rAU[1][o],
                                    geometry.cell_volumes[o] * rAU[2][o]};
            const double boundary_coeff = pressure_face_orthogonal_coefficient(Sf, dvec, dAU_boundary);
            rows[o][o] += rho * boundary_coeff;
            const Vec3 gp_boundary{current_grad_p.component_data(0)[o],
                                   current_grad_p.component_data(1)[o],
                                   current_grad_p.component_data(2)[o]};
            const double deferred_boundary = pressure_face_nonorthogonal_flux(Sf, dvec, dAU_boundary, gp_boundary);
            const double boundary_source = rho * (boundary_coeff * (it->second.value - p(o)) + deferred_boundary);
            b(o) += boundary_source;
        }
        // :8605-8608 fixed-pressure boundary: full system
        for (std::size_t row = 0; row < nc; ++row)
            for (const auto& [col, v] : rows[row]) A.push_back(row, col, v);
        A.finalize();
        if (seconds) *seconds = cfdx_ref::now_seconds() - t0;

        for (std::size_t f = 0; f < mesh.n_faces(); ++f) phi_out[f] = phiHbyA(f);
        for (std::size_t d = 0; d < 3; ++d)
            for (std::size_t c = 0; c < nc; ++c) grad_out[d * nc + c] = current_grad_p.component_data(d)[c];
        for (std::size_t c = 0; c < nc; ++c) b_out[c] = b(c);
        return cfdx_ref::export_csr(A, ro, co, va);
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}

extern "C" int ref_rhie_chow_flux(const ref_mesh_t* m, const double* HbyA_soa, const double* rAU_soa,
                                  const double* p_in, double rho, const int32_t* fixed,
                                  const double* value, double* flux_out) {
    try {
        const Mesh mesh = cfdx_ref::make_mesh(*m);
        const FvGeometry geometry = build_fv_geometry(mesh);
        const std::size_t nc = mesh.n_cells();
        const auto pressure_bcs = make_pressure_bcs(*m, fixed, value);
        const VelocityBoundaryConditions velocity_bcs;
        const auto HbyA = make_vector_field(HbyA_soa, nc);
        const auto p = make_scalar_field(p_in, nc);
        const auto rAU = make_rau(rAU_soa, nc);
        const auto flux = make_rhie_chow_mass_flux(
            mesh, geometry, HbyA, p, rAU, rho, velocity_bcs, pressure_bcs,
            RhieChowVelocityContract::HBYA_PREDICTOR, false, false, nullptr);
        for (std::size_t f = 0; f < mesh.n_faces(); ++f) flux_out[f] = flux(f);
        return 0;
    } catch (const std::exception& e) {
        cfdx_ref::set_error(e);
        return -1;
    }
}
