"""cfdx_dev_b200 -- B200-native CFDX pressure-correction hot path.

Unstructured finite-volume pressure-correction assembly and Rhie-Chow face
fluxes, plus the native-AMG-preconditioned GMRES/FGMRES solve, as sm_100a
CUDA kernels behind a C ABI (include/cfdxg.h).  See ``api`` for the
reference-shaped Python entry points, ``domain`` for one system split over
several GPUs, ``replay`` for replaying captured systems and ``train_mpnn`` for
training the learned stage.
"""
from .api import (  # noqa: F401
    CfdxgError,
    Context,
    HostMesh,
    LearnedPreconditioner,
    Mesh,
    NativeBoomerAMGPreconditioner,
    ReferenceCellGauge,
    ReusablePreconditionerContext,
    SparseMatrix,
    assemble_cell_diffusion_matrix,
    assemble_pressure_correction,
    boundary_layer_case,
    build_hbya,
    fourier_field,
    gauss_gradient_with_boundary,
    hex_case,
    diagnose_matrix,
    make_request,
    measure_matrix_characteristics,
    make_rhie_chow_mass_flux,
    parse_linear_capture_iterations,
    random_field,
    read_linear_system_capture,
    scale_matrix,
    select_linear_solver,
    solve_cg,
    solve_fgmres,
    solve_gmres,
    solve_linear_system,
    solve_poisson_mixed,
    tet_case,
    write_linear_system_capture,
)
