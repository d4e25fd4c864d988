"""ctypes binding of the in-tree C-ABI library (include/philip_b200.h).

The library is the product: there is no CPU fallback. Loading fails loudly when
``libphilip_b200.so`` is missing or no CUDA device is visible.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("PHILIP_B200_LIB", os.path.join(_HERE, "libphilip_b200.so"))

PH_HOST, PH_DEVICE = 0, 1
PH_FP64, PH_FP32_RESIDUAL = 0, 1
PH_OK, PH_ERR_INVALID, PH_ERR_UNSUPPORTED, PH_ERR_CUDA, PH_ERR_NOMEM, PH_ERR_EXCHANGE = 0, 1, 2, 3, 4, 5
PH_HALO_STATE, PH_HALO_VISCOUS = 0, 1
PH_HALO_BEGIN, PH_HALO_END = 0, 1
# PeriodicTurbulence::IntegratedQuantitiesEnum (periodic_turbulence.h:176-186)
INTEGRATED_QUANTITIES = ("kinetic_energy", "enstrophy", "pressure_dilatation",
                         "viscosity_times_deviatoric_strain_rate_tensor_magnitude_sqr",
                         "viscosity_times_strain_rate_tensor_magnitude_sqr", "incompressible_kinetic_energy",
                         "incompressible_enstrophy", "incompressible_palinstrophy", "angular_momentum")
ERRORS = {1: "invalid argument", 2: "unsupported configuration", 3: "CUDA error", 4: "out of device memory",
          5: "halo exchange failed"}

EXPORTED = ["ph_ctx_create", "ph_ctx_destroy", "ph_ndofs", "ph_cell_ijk", "ph_set_state", "ph_get_state",
            "ph_residual", "ph_apply_inverse_mass", "ph_rk_step", "ph_integrals", "ph_status", "ph_sync",
            "ph_set_timing", "ph_get_timing", "ph_quotient_selftest", "ph_residual_noalloc", "ph_residual_noalloc_status", "ph_node_xyz",
            "ph_batch_create", "ph_batch_destroy", "ph_batch_bytes", "ph_batch_admit", "ph_batch_step",
            "ph_batch_progress", "ph_batch_active", "ph_batch_get_state", "ph_batch_status", "ph_batch_release",
            "ph_batch_poll", "ph_batch_fence", "ph_batch_fence_wait", "ph_batch_autotune", "ph_batch_set_variant",
            "ph_batch_launches", "ph_mesh_node_xyz", "ph_rk_error_norm", "ph_last_error",
            "ph_integrated_quantities", "ph_run", "ph_rk_relaxation", "ph_ctx_create_slab", "ph_set_halo_exchange",
            "ph_set_rank_sum",
            "ph_slab_connectivity", "ph_server_create", "ph_server_submit", "ph_server_poll", "ph_server_wait",
            "ph_server_result", "ph_server_stats", "ph_server_destroy", "ph_snapshots_create", "ph_snapshots_destroy",
            "ph_snapshots_add", "ph_snapshots_add_state", "ph_snapshots_add_batch", "ph_snapshots_count",
            "ph_snapshots_get", "ph_snapshots_pod", "ph_limit", "ph_kinetic_energy_rate"]
PH_SOLVE_QUEUED, PH_SOLVE_RUNNING, PH_SOLVE_DONE, PH_SOLVE_FAILED = 0, 1, 2, 3

# ph_halo_fn(user, what, phase, send_lo, send_hi, recv_lo, recv_hi, bytes, cuda_stream)
HALO_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)
# ph_rank_sum_fn(user, values, count)
RANK_SUM_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int)


class PhParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "poly_degree", "overintegration", "flux_nodes_type", "pde_type", "use_split_form",
        "two_point_num_flux_type", "conv_num_flux", "diss_num_flux", "flux_reconstruction",
        "flux_reconstruction_aux", "runge_kutta_method", "use_constant_viscosity", "non_physical_behavior",
        "precision")] + [(n, ctypes.c_double) for n in (
        "FR_user_specified_correction_parameter_value", "gamma_gas", "mach_infinity", "reynolds_number_inf",
        "prandtl_number", "temperature_inf", "nondimensionalized_constant_viscosity", "sipg_penalty_factor",
        "rk_atol", "rk_rtol", "pressure_shift")] + [
        ("use_relaxation_runge_kutta", ctypes.c_int), ("relaxation_runge_kutta_root_tolerance", ctypes.c_double),
        ("bound_preserving_limiter", ctypes.c_int), ("min_density", ctypes.c_double),
        ("angle_of_attack", ctypes.c_double), ("side_slip_angle", ctypes.c_double),
        ("thermal_boundary_condition_type", ctypes.c_int), ("isothermal_wall_temperature", ctypes.c_double),
        ("use_projected_entropy_variables_for_nsfr_boundary_term", ctypes.c_int)]


class PhMeshDesc(ctypes.Structure):
    _fields_ = [("n_cells_per_direction", ctypes.c_int), ("cell_order", ctypes.c_int),
                ("left", ctypes.c_double), ("right", ctypes.c_double),
                ("warp", ctypes.c_double), ("grid_degree", ctypes.c_int),
                ("mapping_support_points", ctypes.POINTER(ctypes.c_double)),
                ("boundary_type", ctypes.c_int * 6)]

# boundary_id of each boundary condition (Euler::boundary_face_values); 0 keeps a periodic pair of sides
BOUNDARY = {"periodic": 0, "wall": 1001, "pressure_outflow": 1002, "inflow": 1003, "riemann_farfield": 1004,
            "farfield": 1005, "slip_wall": 1006, "extrapolation": 1007}


def boundary_ids(types) -> list:
    """boundary_id values of six boundary types given by name or by id."""
    ids = [BOUNDARY[t] if isinstance(t, str) else int(t) for t in types]
    if len(ids) != 6:
        raise ValueError("boundaries: one type per side x-, x+, y-, y+, z-, z+")
    return ids


class PhError(RuntimeError):
    pass


_lib = None


def load(build_if_missing: bool = False):
    """Load the library (optionally building it first); raises if it cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise PhError(f"{LIB_PATH} is missing: run philip_b200.build.build() (or __graft_entry__.build())")
        from . import build as _build
        _build.build()
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    L.ph_ctx_create.argtypes = [ctypes.POINTER(PhMeshDesc), ctypes.POINTER(PhParams), vp, ctypes.POINTER(vp)]
    L.ph_ctx_destroy.argtypes = [vp]
    L.ph_ndofs.argtypes = [vp]; L.ph_ndofs.restype = ctypes.c_int64
    L.ph_cell_ijk.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
    L.ph_set_state.argtypes = [vp, vp, ctypes.c_int]
    L.ph_get_state.argtypes = [vp, vp, ctypes.c_int]
    L.ph_residual.argtypes = [vp, vp, vp, ctypes.c_int]
    L.ph_apply_inverse_mass.argtypes = [vp, vp, vp, ctypes.c_int]
    L.ph_rk_step.argtypes = [vp, ctypes.c_double, ctypes.c_int]
    L.ph_integrals.argtypes = [vp, dp]
    L.ph_integrated_quantities.argtypes = [vp, dp]
    L.ph_run.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, dp]
    L.ph_rk_relaxation.argtypes = [vp, dp, dp]
    L.ph_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32)]
    L.ph_limit.argtypes = [vp, ctypes.c_double]
    L.ph_kinetic_energy_rate.argtypes = [vp, dp]
    L.ph_sync.argtypes = [vp]
    L.ph_set_timing.argtypes = [vp, ctypes.c_int]
    L.ph_get_timing.argtypes = [vp, dp]
    L.ph_quotient_selftest.argtypes = [ctypes.c_uint64, ctypes.c_int, dp]
    sz = ctypes.c_size_t
    L.ph_batch_create.argtypes = [sz, ctypes.c_int, vp, ctypes.POINTER(vp)]
    L.ph_batch_destroy.argtypes = [vp]
    L.ph_batch_bytes.argtypes = [ctypes.POINTER(PhMeshDesc), ctypes.POINTER(PhParams), ctypes.POINTER(sz)]
    L.ph_batch_admit.argtypes = [vp, ctypes.POINTER(PhMeshDesc), ctypes.POINTER(PhParams), ctypes.POINTER(ctypes.c_double),
                                 ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.ph_batch_step.argtypes = [vp, ctypes.c_int]
    L.ph_batch_progress.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    L.ph_batch_active.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.ph_batch_get_state.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.ph_batch_status.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_uint32)]
    L.ph_batch_release.argtypes = [vp, ctypes.c_int]
    L.ph_batch_poll.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.ph_batch_fence.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.ph_batch_fence_wait.argtypes = [vp, ctypes.c_longlong]
    L.ph_batch_autotune.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    L.ph_batch_set_variant.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.ph_batch_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.ph_mesh_node_xyz.argtypes = [ctypes.POINTER(PhMeshDesc), ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.ph_rk_error_norm.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.ph_node_xyz.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
    L.ph_residual_noalloc.argtypes = [ctypes.POINTER(PhMeshDesc), ctypes.POINTER(PhParams), vp, vp, vp]
    L.ph_residual_noalloc_status.argtypes = [vp, ctypes.POINTER(ctypes.c_uint32)]
    L.ph_ctx_create_slab.argtypes = [ctypes.POINTER(PhMeshDesc), ctypes.POINTER(PhParams), ctypes.c_int, ctypes.c_int,
                                     vp, ctypes.POINTER(vp)]
    L.ph_set_halo_exchange.argtypes = [vp, HALO_FN, vp]
    L.ph_set_rank_sum.argtypes = [vp, RANK_SUM_FN, vp]
    L.ph_slab_connectivity.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int32),
                                       ctypes.POINTER(ctypes.c_int32)]
    ll = ctypes.c_longlong
    L.ph_server_create.argtypes = [sz, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.POINTER(vp)]
    L.ph_server_submit.argtypes = [vp, ctypes.POINTER(PhMeshDesc), ctypes.POINTER(PhParams), dp, ctypes.c_double,
                                   ctypes.c_int, ctypes.POINTER(ll)]
    L.ph_server_poll.argtypes = [vp, ll, ctypes.POINTER(ctypes.c_int)]
    L.ph_server_wait.argtypes = [vp, ll, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]
    L.ph_server_result.argtypes = [vp, ll, dp, ctypes.POINTER(ctypes.c_uint32), dp]
    L.ph_server_stats.argtypes = [vp, ctypes.POINTER(ll)]
    L.ph_server_destroy.argtypes = [vp]
    L.ph_snapshots_create.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.POINTER(vp)]
    L.ph_snapshots_destroy.argtypes = [vp]
    L.ph_snapshots_add.argtypes = [vp, vp, ctypes.c_int]
    L.ph_snapshots_add_state.argtypes = [vp, vp]
    L.ph_snapshots_add_batch.argtypes = [vp, vp, ctypes.c_int]
    L.ph_snapshots_count.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.ph_snapshots_get.argtypes = [vp, vp, ctypes.c_int]
    L.ph_snapshots_pod.argtypes = [vp, ctypes.c_double, vp, vp, vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.ph_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def check(rc: int):
    if rc != 0:
        msg = _lib.ph_last_error().decode() if _lib is not None else ""
        raise PhError(f"philip_b200 error {rc} ({ERRORS.get(rc, '?')}): {msg}")
