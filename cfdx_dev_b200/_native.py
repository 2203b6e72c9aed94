"""ctypes binding of libcfdxg.so (the C ABI declared in include/cfdxg.h).

The library is built in-tree by ``python -m cfdx_dev_b200.build``.  Loading
fails loudly if it is missing: there is no CPU fallback for the hot path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libcfdxg.so"

CFDXG_MEM_HOST = 0
CFDXG_MEM_DEVICE = 1
KRYLOV = {"auto": 0, "cg": 1, "gmres": 3, "fgmres": 4}
PRECONDITIONER = {"auto": 0, "none": 1, "jacobi": 2, "native_amg": 6, "own_diagonal": 32}
# the reference's full model enums (core/linalg/linear_solver_models.h:11-61), for plan selection
PROBLEMS = ["general", "pressure_poisson", "diffusion", "momentum", "scalar_transport", "coupled_pressure_velocity"]
KRYLOV_MODELS = ["auto", "cg", "bicgstab", "gmres", "fgmres", "lgmres", "pipecg", "pipefgmres"]
PRECONDITIONER_MODELS = [
    "auto", "none", "jacobi", "gauss_seidel", "ilu0", "ilut", "native_amg", "smoothed_aggregation_amg",
    "anisotropic_line_amg", "fsai", "ras", "native_fieldsplit", "coupled_block_schur", "pcd", "lsc", "mgr",
    "anisotropic_line", "anisotropic_boomer_amg", "anisotropic_smoothed_aggregation_amg",
    "directional_semi_coarsening_amg", "energy_minimizing_amg", "vanka_pressure_patch", "braess_sarazin"]
NULL_SPACES = ["none", "constant"]
SCALINGS = ["none", "row", "column", "row_column", "symmetric_diagonal"]
PRECISION = {"fp64": 0, "fp32_vcycle": 1}
STATUS = {0: "converged", 1: "max_iter_reached", 2: "diverged", 3: "not_applicable"}
ERRORS = {
    -1: "invalid_argument", -2: "cuda", -3: "setup", -4: "not_ready",
    -5: "nonfinite", -6: "geometry", -7: "out_of_memory", -8: "io",
}

ERRORS_BY_NAME = {v: k for k, v in ERRORS.items()}

c_double_p = C.POINTER(C.c_double)
c_float_p = C.POINTER(C.c_float)
c_int64_p = C.POINTER(C.c_int64)
c_int32_p = C.POINTER(C.c_int32)


class MeshDesc(C.Structure):
    _fields_ = [
        ("n_points", C.c_int64), ("n_faces", C.c_int64), ("n_cells", C.c_int64),
        ("px", c_double_p), ("py", c_double_p), ("pz", c_double_p),
        ("face_offsets", c_int64_p), ("face_vertices", c_int64_p),
        ("owner", c_int64_p), ("neighbour", c_int64_p),
        ("cell_offsets", c_int64_p), ("cell_faces", c_int64_p),
        ("n_patches", C.c_int32), ("patch_of_face", c_int32_p), ("patch_types", c_int32_p),
    ]


class AmgOptions(C.Structure):
    _fields_ = [
        ("omega", C.c_double), ("pre_sweeps", C.c_int32), ("post_sweeps", C.c_int32),
        ("strength_threshold", C.c_double), ("max_levels", C.c_int32),
        ("require_smoother_certificate", C.c_int32), ("precision", C.c_int32),
        ("coarse_dense_limit", C.c_int32), ("reference_order", C.c_int32),
        ("coarse_pre_sweeps", C.c_int32), ("coarse_post_sweeps", C.c_int32), ("narrow_columns", C.c_int32),
        ("half_values", C.c_int32), ("dense_fp64", C.c_int32), ("constant_null_space", C.c_int32),
        ("coarse_drop_tolerance", C.c_double),
    ]


class KernelProfile(C.Structure):
    _fields_ = [("name", C.c_char * 48), ("launches", C.c_int64), ("total_ms", C.c_double), ("bytes", C.c_double)]


class Request(C.Structure):
    _fields_ = [
        ("krylov", C.c_int32), ("preconditioner", C.c_int32), ("gmres_restart", C.c_int32),
        ("precision", C.c_int32), ("restart_min", C.c_int32), ("restart_max", C.c_int32),
        ("adaptive_restart", C.c_int32), ("residual_replacement", C.c_int32),
        ("residual_replacement_period", C.c_int64), ("residual_replacement_gap_ratio", C.c_double),
        ("target_reduction_per_cycle", C.c_double), ("learned", C.c_void_p),
        ("learned_applications", C.c_int32), ("orthogonalization", C.c_int32), ("problem", C.c_int32),
        ("scaling", C.c_int32), ("null_space", C.c_int32),
    ]


class Report(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("iterations", C.c_int64), ("residual", C.c_double),
        ("residual_relative", C.c_double), ("physical_residual_relative", C.c_double),
        ("residual_replacements", C.c_int64), ("max_true_recursive_gap", C.c_double),
        ("setup_seconds", C.c_double), ("solve_seconds", C.c_double),
        ("preconditioner_applications", C.c_int64), ("learned_fallbacks", C.c_int64),
        ("plan_krylov", C.c_int32), ("plan_preconditioner", C.c_int32),
    ]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["status_name"] = STATUS.get(self.status, ERRORS.get(self.status, str(self.status)))
        return d


class CaptureInfo(C.Structure):
    _fields_ = [
        ("problem", C.c_int32), ("null_space", C.c_int32), ("scaling", C.c_int32), ("n", C.c_int64),
        ("nnz", C.c_int64), ("max_iterations", C.c_int64), ("tolerance", C.c_double), ("checksum", C.c_uint64),
    ]


class MatrixCharacteristics(C.Structure):
    _fields_ = [
        ("equations", C.c_int64), ("average_nnz_per_row", C.c_double), ("coefficient_range", C.c_double),
        ("square", C.c_int32), ("numerically_symmetric", C.c_int32), ("diagonally_dominant", C.c_int32),
        ("strongly_scaled", C.c_int32), ("large_diagonal_dynamic_range", C.c_int32),
        ("strongly_directional_coupling", C.c_int32), ("positive_diagonal", C.c_int32), ("saddle_point", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


DIAG_COUNTS = ("empty_rows", "empty_columns", "missing_diagonal", "near_zero_diagonal", "isolated_dofs",
               "duplicate_entries")
DIAG_VALUES = ("max_abs_value", "min_nonzero_abs_value", "max_row_sum", "min_nonzero_row_sum", "max_column_sum",
               "min_nonzero_column_sum", "max_abs_diagonal", "min_nonzero_abs_diagonal", "diagonal_dynamic_range",
               "row_sum_dynamic_range", "column_sum_dynamic_range", "minimum_gershgorin_margin")


class MatrixDiagnostics(C.Structure):
    _fields_ = ([("rows", C.c_int64), ("columns", C.c_int64), ("nnz", C.c_int64), ("finite", C.c_int32),
                 ("structurally_consistent", C.c_int32)] + [(k, C.c_int64) for k in DIAG_COUNTS] +
                [(k, C.c_double) for k in DIAG_VALUES] + [("connected_components", C.c_int64)])

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class PlanRequest(C.Structure):
    _fields_ = [("krylov", C.c_int32), ("preconditioner", C.c_int32), ("gmres_restart", C.c_int32),
                ("null_space", C.c_int32), ("scaling", C.c_int32), ("braess_sarazin_alpha", C.c_double)]


class SolverPlan(C.Structure):
    _fields_ = [("problem", C.c_int32), ("krylov", C.c_int32), ("preconditioner", C.c_int32),
                ("null_space", C.c_int32), ("automatic_krylov", C.c_int32), ("automatic_preconditioner", C.c_int32),
                ("reason", C.c_char * 512)]


class DomainPartInfo(C.Structure):
    _fields_ = [
        ("row_begin", C.c_int64), ("row_end", C.c_int64), ("n_local", C.c_int64), ("owned_offset", C.c_int64),
        ("nnz_local", C.c_int64), ("nnz_block", C.c_int64), ("n_neighbours", C.c_int32), ("n_recv", C.c_int64),
        ("n_send", C.c_int64), ("col_begin", C.c_int64), ("col_end", C.c_int64), ("n_local_rows", C.c_int64),
        ("first_row", C.c_int64),
    ]


DOMAIN_ARRAYS = ("local_row_offsets", "local_columns", "local_source", "block_row_offsets", "block_columns",
                 "block_source", "neighbours", "recv_offsets", "recv_start", "ghost_rows", "send_offsets",
                 "send_rows")


class DomainPartArrays(C.Structure):
    _fields_ = [(name, C.c_void_p) for name in DOMAIN_ARRAYS]


_V = C.c_void_p
_P = C.POINTER
# name -> (restype, argtypes)
PROTOTYPES = {
    "cfdxg_context_create": (C.c_int, [C.c_int32, _P(_V)]),
    "cfdxg_context_destroy": (C.c_int, [_V]),
    "cfdxg_last_error": (C.c_char_p, [_V]),
    "cfdxg_kernel_launches": (C.c_int64, [_V]),
    "cfdxg_synchronize": (C.c_int, [_V]),
    "cfdxg_context_stream": (C.c_void_p, [_V]),
    "cfdxg_profile_enable": (C.c_int, [_V, C.c_int32]),
    "cfdxg_profile_read": (C.c_int, [_V, _V, C.c_int32, c_int32_p]),
    "cfdxg_mesh_upload": (C.c_int, [_V, _P(MeshDesc), _P(_V)]),
    "cfdxg_mesh_destroy": (C.c_int, [_V]),
    "cfdxg_geometry_build": (C.c_int, [_V, _V]),
    "cfdxg_geometry_download": (C.c_int, [_V, _V, _V, _V, _V, _V]),
    "cfdxg_matrix_create": (C.c_int, [_V, C.c_int64, _V, _V, _V, C.c_int32, _P(_V)]),
    "cfdxg_matrix_destroy": (C.c_int, [_V]),
    "cfdxg_matrix_size": (C.c_int, [_V, c_int64_p, c_int64_p]),
    "cfdxg_matrix_download": (C.c_int, [_V, _V, _V, _V, _V]),
    "cfdxg_matrix_spmv": (C.c_int, [_V, _V, _V, _V, C.c_int32]),
    "cfdxg_assemble_cell_diffusion": (C.c_int, [_V, _V, _V, _V, C.c_double, _V, C.c_int32, _P(_V), _V]),
    "cfdxg_assemble_pressure_correction": (
        C.c_int, [_V, _V, _V, _V, _V, C.c_double, _V, _V, C.c_int32, _P(_V), _V, _V, _V]),
    "cfdxg_rhie_chow_flux": (C.c_int, [_V, _V, _V, _V, _V, C.c_double, _V, _V, C.c_int32, _V]),
    "cfdxg_gauss_gradient": (C.c_int, [_V, _V, _V, _V, _V, C.c_int32, _V]),
    "cfdxg_build_hbya": (C.c_int, [_V, _V, _V, _V, _V, _V, _V, C.c_int32, _V]),
    "cfdxg_rhie_chow_flux_noalloc": (C.c_int, [_V, _V, _V, _V, _V, C.c_double, _V, _V, _V]),
    "cfdxg_amg_options_default": (C.c_int, [_P(AmgOptions)]),
    "cfdxg_amg_create": (C.c_int, [_V, _P(AmgOptions), _P(_V)]),
    "cfdxg_amg_destroy": (C.c_int, [_V]),
    "cfdxg_amg_setup": (C.c_int, [_V, _V, _V]),
    "cfdxg_amg_update_values_host": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cfdxg_amg_setup_host": (C.c_int, [_V, C.c_int64, _V, _V, _V]),
    "cfdxg_amg_update_values": (C.c_int, [_V, _V, _V]),
    "cfdxg_amg_apply": (C.c_int, [_V, _V, _V, _V, C.c_int32]),
    "cfdxg_amg_name": (C.c_char_p, [_V]),
    "cfdxg_amg_last_error": (C.c_char_p, [_V]),
    "cfdxg_amg_num_levels": (C.c_int32, [_V]),
    "cfdxg_amg_omega": (C.c_double, [_V]),
    "cfdxg_amg_level_info": (C.c_int, [_V, C.c_int32, c_int64_p, c_int64_p, c_int64_p]),
    "cfdxg_amg_export_level": (C.c_int, [_V, C.c_int32, _V, _V, _V, _V, _V, _V, _V, _V]),
    "cfdxg_amg_setup_seconds": (C.c_double, [_V]),
    "cfdxg_request_default": (C.c_int, [_P(Request)]),
    "cfdxg_solve_linear_system": (
        C.c_int, [_V, _V, _V, _V, C.c_int32, _P(Request), C.c_int64, C.c_double, _P(Report)]),
    "cfdxg_solve_gmres": (
        C.c_int, [_V, _V, _V, _V, _V, C.c_int32, _P(Request), C.c_int64, C.c_double, _P(Report)]),
    "cfdxg_case_hex": (C.c_int, [C.c_int64, C.c_int64, C.c_int64, _P(_V)]),
    "cfdxg_case_tet": (C.c_int, [C.c_int64, C.c_double, C.c_uint64, _P(_V)]),
    "cfdxg_case_boundary_layer": (
        C.c_int, [C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.c_double, C.c_uint64, _P(_V)]),
    "cfdxg_case_destroy": (C.c_int, [_V]),
    "cfdxg_case_sizes": (C.c_int, [_V, c_int64_p]),
    "cfdxg_case_export": (C.c_int, [_V] + [_V] * 11),
    "cfdxg_field_fourier": (C.c_int, [C.c_int64, _V, C.c_int32, C.c_double, C.c_uint64, _V]),
    "cfdxg_field_random": (C.c_int, [C.c_int64, C.c_int32, C.c_double, C.c_double, C.c_uint64, _V]),
    "cfdxg_mpnn_create": (C.c_int, [_V, C.c_uint64, _P(_V)]),
    "cfdxg_mpnn_destroy": (C.c_int, [_V]),
    "cfdxg_mpnn_num_parameters": (C.c_int, [_V, c_int64_p]),
    "cfdxg_mpnn_get_parameters": (C.c_int, [_V, _V, _V]),
    "cfdxg_mpnn_set_parameters": (C.c_int, [_V, _V, _V]),
    "cfdxg_mpnn_save": (C.c_int, [_V, _V, C.c_char_p]),
    "cfdxg_mpnn_load": (C.c_int, [_V, _V, C.c_char_p]),
    "cfdxg_mpnn_bind": (C.c_int, [_V, _V, _V, _V, _V, C.c_int32]),
    "cfdxg_mpnn_apply": (C.c_int, [_V, _V, _V, _V, C.c_int32]),
    "cfdxg_mpnn_set_vcycle": (C.c_int, [_V, _V, _V]),
    "cfdxg_mpnn_train_step": (C.c_int, [_V, _V, _V, _V, C.c_int32, C.c_float, C.c_int32, c_double_p]),
    "cfdxg_mpnn_loss_grad": (C.c_int, [_V, _V, _V, _V, C.c_int32, C.c_int32, c_double_p, _V]),
    "cfdxg_gauge_create": (C.c_int, [_V, _V, C.c_int32, C.c_int64, C.c_double, _P(_V)]),
    "cfdxg_gauge_apply": (C.c_int, [_V, _V, _V, _V, C.c_int32, _P(_V), _V]),
    "cfdxg_gauge_expand": (C.c_int, [_V, _V, _V, C.c_int32, _V]),
    "cfdxg_gauge_size": (C.c_int, [_V, c_int64_p, c_int64_p]),
    "cfdxg_gauge_destroy": (C.c_int, [_V]),
    "cfdxg_capture_read": (C.c_int, [C.c_char_p, _P(_V), _P(CaptureInfo)]),
    "cfdxg_capture_export": (C.c_int, [_V] * 6),
    "cfdxg_capture_write": (C.c_int, [C.c_char_p, C.c_int64] + [_V] * 5 + [_P(CaptureInfo)]),
    "cfdxg_capture_destroy": (C.c_int, [_V]),
    "cfdxg_capture_last_error": (C.c_char_p, []),
    "cfdxg_measure_matrix_characteristics": (C.c_int, [C.c_int64, _V, _V, _V, C.c_int32, C.c_double,
                                                      _P(MatrixCharacteristics)]),
    "cfdxg_select_linear_solver": (C.c_int, [C.c_int32, _P(MatrixCharacteristics), _P(PlanRequest),
                                            _P(SolverPlan)]),
    "cfdxg_plan_last_error": (C.c_char_p, []),
    "cfdxg_diagnose_matrix": (C.c_int, [C.c_int64, C.c_int64, _V, _V, _V, C.c_double, C.c_int32,
                                        _P(MatrixDiagnostics)]),
    "cfdxg_scale_matrix": (C.c_int, [C.c_int64, _V, _V, _V, C.c_int32, C.c_double, _V, _V, _V, _V]),
    "cfdxg_plan_reason": (C.c_char_p, [_V]),
    "cfdxg_domain_plan_create": (C.c_int, [C.c_int64, _V, _V, C.c_int32, _V, _P(_V)]),
    "cfdxg_domain_plan_create_rect": (C.c_int, [C.c_int64, C.c_int64, _V, _V, C.c_int32, _V, _V, _P(_V)]),
    "cfdxg_domain_plan_parts": (C.c_int, [_V, _V, _V]),
    "cfdxg_domain_plan_info": (C.c_int, [_V, C.c_int32, _P(DomainPartInfo)]),
    "cfdxg_domain_plan_export": (C.c_int, [_V, C.c_int32, _P(DomainPartArrays)]),
    "cfdxg_domain_plan_destroy": (C.c_int, [_V]),
    "cfdxg_domain_last_error": (C.c_char_p, []),
}

_lib = None


def load() -> C.CDLL:
    """Load libcfdxg.so (built in-tree).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m cfdx_dev_b200.build` "
            "(the CUDA path has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a):
    """Raw data pointer of a numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.c_void_p)
