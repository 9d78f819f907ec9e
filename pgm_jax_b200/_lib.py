"""ctypes binding of the engine's C ABI (include/pgm_b200.h).

The library is the product: there is no fallback.  Loading fails loudly when it is missing.
"""

from __future__ import annotations

import ctypes as C
import os

from .build import LIB

_i32 = C.c_int32
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)
_pu = C.POINTER(C.c_uint32)

# every symbol the header declares (tests check the library exports them)
EXPORTS = (
    "pgm_create", "pgm_destroy", "pgm_compute", "pgm_compute_host", "pgm_energy", "pgm_energy_fixed_mu", "pgm_field",
    "pgm_set_row_capacity", "pgm_row_capacity", "pgm_set_elec_capacity", "pgm_elec_capacity", "pgm_max_vdw_count", "pgm_set_list_capacity", "pgm_list_capacity", "pgm_list_rebuilds", "pgm_max_row_count", "pgm_num_atoms", "pgm_num_systems",
    "pgm_last_error", "pgm_last_launch_count", "pgm_launches_per_iteration", "pgm_unrolled_iterations", "pgm_profile_kernel", "pgm_row_pairs", "pgm_rigid_create", "pgm_rigid_destroy",
    "pgm_rigid_begin_step", "pgm_rigid_set_step", "pgm_rigid_end_step", "pgm_rigid_kinetic", "pgm_rigid_scale_momenta", "pgm_rigid_last_error", "pgm_pimd_kick",
    "pgm_pimd_free_thermostat", "pgm_pimd_centroid_bussi", "pgm_pimd_free_thermostat_scaled", "pgm_water_bonded",
    "pgm_pimd_last_error", "pgm_graph_begin",
    "pgm_graph_end", "pgm_graph_launch", "pgm_graph_destroy", "pgm_field_static", "pgm_static_last_error",
    "pgm_set_nn_model", "pgm_nn_features", "pgm_nn_param_count", "pgm_nn_predict", "pgm_nn_loss_grad", "pgm_nn_adam",
    "pgm_nn_last_error", "pgm_set_nn_fallback", "pgm_nn_fallback_stats", "pgm_tuning", "pgm_set_tuning", "pgm_autotune",
    "pgm_iel_len", "pgm_tc_gemm", "pgm_tc_last_error", "pgm_mpnn_param_count", "pgm_set_mpnn_model", "pgm_nn_graph",
    "pgm_mpnn_work_bytes", "pgm_mpnn_predict", "pgm_mpnn_loss_grad", "pgm_mpnn_adam", "pgm_mpnn_last_error",
)

STATUS_ROW_OVERFLOW = 0x1
STATUS_CG_MAXITER = 0x2
STATUS_NONFINITE = 0x4
STATUS_BAD_BOX = 0x8
STATUS_LIST_OVERFLOW = 0x10
STATUS_SHORT_OVERFLOW = 0x20


class PgmTuning(C.Structure):
    _fields_ = [
        ("rowfield_lanes", C.c_int), ("forces_blocks_per_sm", C.c_int), ("rowfield_ms", C.c_double * 3),
        ("forces_ms", C.c_double * 3), ("tuned", C.c_int), ("from_cache", C.c_int), ("sweep_early", C.c_int),
        ("sweep_ms", C.c_double * 2), ("rowfield_grid", C.c_int), ("grid_ms", C.c_double * 3),
    ]


class PgmSettings(C.Structure):
    _fields_ = [
        ("elec", C.c_int), ("vdw", C.c_int), ("lj_lrc", C.c_int), ("precision", C.c_int), ("cutoff", C.c_double),
        ("ewald_beta", C.c_double), ("pme_order", C.c_int), ("dipole_tol", C.c_double), ("max_iter", C.c_int),
        ("predictor", C.c_int), ("fused", C.c_int), ("norm_refresh", C.c_int), ("peek", C.c_double),
        ("row_capacity", C.c_int), ("skin", C.c_double), ("list_capacity", C.c_int), ("elec_cutoff", C.c_double),
        ("elec_capacity", C.c_int), ("iel", C.c_int), ("iel_order", C.c_int), ("iel_custom", C.c_int),
        ("iel_kappa", C.c_double), ("iel_alpha", C.c_double), ("iel_omega", C.c_double), ("iel_precond", C.c_int),
        ("iel_iter", C.c_int), ("iel_no_shadow", C.c_int), ("local_cut", C.c_double), ("local_niter", C.c_int),
    ]


class PgmSystemDesc(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int), ("n_mol", C.c_int), ("mol_start", _pi), ("q", _pd), ("radius", _pd), ("alpha", _pd),
        ("lj_rmin_half", _pd), ("lj_sqrt_eps", _pd), ("masses", _pd), ("n_cov", C.c_int), ("cov_i", _pi),
        ("cov_j", _pi), ("cov_c", _pd), ("pme_grid", C.c_int * 3), ("box0", C.c_double * 9),
    ]


class PgmInduction(C.Structure):
    _fields_ = [("mu", C.c_void_p), ("hist", C.c_void_p), ("count", C.c_void_p), ("norm", C.c_void_p), ("xl", C.c_void_p)]


class PgmOutputs(C.Structure):
    _fields_ = [
        ("energy", C.c_void_p), ("forces", C.c_void_p), ("virial", C.c_void_p), ("iterations", C.c_void_p),
        ("residual", C.c_void_p), ("status", C.c_void_p),
    ]


_lib = None


def load(path: str | None = None):
    """Load libpgm_b200.so (built in-tree by pgm_jax_b200.build); raise if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB
    if not os.path.exists(p):
        raise RuntimeError(f"the engine library {p} is not built: run pgm_jax_b200.build.build() (nvcc, sm_100a)")
    lib = C.CDLL(p)
    H = C.c_void_p
    vp = C.c_void_p
    lib.pgm_create.argtypes = [C.POINTER(PgmSettings), C.POINTER(PgmSystemDesc), C.c_int, C.c_int, C.POINTER(H)]
    lib.pgm_destroy.argtypes = [H]
    lib.pgm_compute.argtypes = [H, vp, vp, vp, vp, C.c_int, C.POINTER(PgmInduction), C.POINTER(PgmOutputs)]
    lib.pgm_compute_host.argtypes = [H, vp, vp, C.POINTER(PgmInduction), C.POINTER(PgmOutputs)]
    lib.pgm_energy.argtypes = [H, vp, vp, vp, vp, C.c_int, C.POINTER(PgmInduction), vp, vp, vp]
    lib.pgm_energy_fixed_mu.argtypes = [H, vp, vp, vp, vp, C.c_int, vp, vp, vp, vp, vp]
    lib.pgm_field.argtypes = [H, vp, vp, vp, C.c_int, vp, vp]
    lib.pgm_set_row_capacity.argtypes = [H, C.c_int]
    lib.pgm_row_capacity.argtypes = [H]
    lib.pgm_set_elec_capacity.argtypes = [H, C.c_int]
    lib.pgm_set_elec_capacity.restype = C.c_int
    lib.pgm_elec_capacity.argtypes = [H]
    lib.pgm_max_vdw_count.argtypes = [H]
    lib.pgm_set_list_capacity.argtypes = [H, C.c_int]
    lib.pgm_set_list_capacity.restype = C.c_int
    lib.pgm_list_capacity.argtypes = [H]
    lib.pgm_list_rebuilds.argtypes = [H]
    lib.pgm_list_rebuilds.restype = C.c_longlong
    lib.pgm_max_row_count.argtypes = [H]
    lib.pgm_unrolled_iterations.argtypes = [H]
    lib.pgm_num_atoms.argtypes = [H]
    lib.pgm_num_systems.argtypes = [H]
    lib.pgm_last_launch_count.argtypes = [H]
    lib.pgm_last_launch_count.restype = C.c_longlong
    lib.pgm_last_error.restype = C.c_char_p
    lib.pgm_profile_kernel.argtypes = [H, vp, C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.pgm_profile_kernel.restype = C.c_int
    lib.pgm_row_pairs.argtypes = [H]
    lib.pgm_row_pairs.restype = C.c_longlong
    lib.pgm_launches_per_iteration.argtypes = [H]
    lib.pgm_launches_per_iteration.restype = C.c_longlong
    lib.pgm_rigid_create.argtypes = [C.c_int, vp, vp, vp, vp, vp, C.c_int, C.POINTER(H)]
    lib.pgm_rigid_destroy.argtypes = [H]
    lib.pgm_rigid_begin_step.argtypes = [H, vp, C.c_double, C.c_double, vp, C.c_uint64, vp, vp, vp, vp, vp, vp, vp]
    lib.pgm_rigid_set_step.argtypes = [H, C.c_uint64]
    lib.pgm_rigid_end_step.argtypes = [H, vp, C.c_double, vp, vp, vp, vp]
    lib.pgm_rigid_kinetic.argtypes = [H, vp, vp, vp, vp]
    lib.pgm_rigid_scale_momenta.argtypes = [H, vp, vp, vp, vp]
    lib.pgm_pimd_kick.argtypes = [vp, C.c_longlong, C.c_double, vp, vp]
    lib.pgm_pimd_free_thermostat.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, C.c_double, C.c_uint64, vp, vp,
                                             vp]
    lib.pgm_pimd_centroid_bussi.argtypes = [vp, C.c_int, C.c_int, vp, vp, C.c_double, C.c_double, C.c_double, C.c_uint64, vp, vp,
                                            vp]
    lib.pgm_pimd_free_thermostat_scaled.argtypes = [vp, C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, C.c_double, C.c_uint64,
                                                    vp, vp, vp, vp]
    lib.pgm_water_bonded.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp]
    lib.pgm_pimd_last_error.restype = C.c_char_p
    for n in ("pgm_pimd_kick", "pgm_pimd_free_thermostat", "pgm_pimd_centroid_bussi", "pgm_pimd_free_thermostat_scaled",
              "pgm_water_bonded"):
        getattr(lib, n).restype = C.c_int
    lib.pgm_rigid_last_error.restype = C.c_char_p
    lib.pgm_field_static.argtypes = [vp, C.c_int, vp, vp, vp, vp, C.c_double, C.c_double, vp, C.c_int, C.c_int, vp, vp]
    lib.pgm_field_static.restype = C.c_int
    lib.pgm_static_last_error.restype = C.c_char_p
    lib.pgm_set_nn_model.argtypes = [H, vp, C.c_float, C.c_float]
    lib.pgm_nn_features.argtypes = [H, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.pgm_nn_predict.argtypes = [vp, vp, vp, vp, C.c_int, vp]
    lib.pgm_nn_loss_grad.argtypes = [vp, vp, vp, vp, vp, C.c_int, C.c_float, vp, vp]
    lib.pgm_nn_adam.argtypes = [vp, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int]
    lib.pgm_nn_last_error.restype = C.c_char_p
    lib.pgm_set_mpnn_model.argtypes = [H, vp, C.c_float, C.c_float]
    lib.pgm_nn_graph.argtypes = [H, vp, vp, vp, C.c_int]
    lib.pgm_mpnn_work_bytes.argtypes = [C.c_int, C.c_int]
    lib.pgm_mpnn_work_bytes.restype = C.c_longlong
    lib.pgm_mpnn_predict.argtypes = [vp, vp, vp, vp, vp, vp, C.c_int, C.c_int, C.c_float, C.c_float, vp, vp]
    lib.pgm_mpnn_loss_grad.argtypes = [vp, vp, vp, vp, vp, vp, vp, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, vp, vp, vp]
    lib.pgm_mpnn_last_error.restype = C.c_char_p
    lib.pgm_mpnn_adam.argtypes = [vp, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int]
    for n in ("pgm_set_mpnn_model", "pgm_nn_graph", "pgm_mpnn_predict", "pgm_mpnn_loss_grad", "pgm_mpnn_adam"):
        getattr(lib, n).restype = C.c_int
    lib.pgm_tc_gemm.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, vp, vp, C.c_int, vp]
    lib.pgm_tc_gemm.restype = C.c_int
    lib.pgm_tc_last_error.restype = C.c_char_p
    lib.pgm_iel_len.argtypes = [C.c_int]
    lib.pgm_iel_len.restype = C.c_int
    lib.pgm_tuning.argtypes = [H, C.POINTER(PgmTuning)]
    lib.pgm_set_tuning.argtypes = [H, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.pgm_autotune.argtypes = [H, vp]
    for n in ("pgm_tuning", "pgm_set_tuning", "pgm_autotune"):
        getattr(lib, n).restype = C.c_int
    lib.pgm_set_nn_fallback.argtypes = [H, C.c_double]
    lib.pgm_nn_fallback_stats.argtypes = [H, vp, vp]
    for n in ("pgm_set_nn_model", "pgm_nn_features", "pgm_nn_predict", "pgm_nn_loss_grad", "pgm_nn_adam",
              "pgm_set_nn_fallback", "pgm_nn_fallback_stats"):
        getattr(lib, n).restype = C.c_int
    lib.pgm_graph_begin.argtypes = [vp]
    lib.pgm_graph_end.argtypes = [vp, C.POINTER(vp)]
    lib.pgm_graph_launch.argtypes = [vp, vp]
    lib.pgm_graph_destroy.argtypes = [vp]
    for n in ("pgm_rigid_create", "pgm_rigid_destroy", "pgm_rigid_begin_step", "pgm_rigid_set_step", "pgm_rigid_end_step", "pgm_rigid_kinetic",
              "pgm_rigid_scale_momenta",
              "pgm_graph_begin", "pgm_graph_end", "pgm_graph_launch", "pgm_graph_destroy"):
        getattr(lib, n).restype = C.c_int
    for n in ("pgm_create", "pgm_destroy", "pgm_compute", "pgm_compute_host", "pgm_energy", "pgm_energy_fixed_mu",
              "pgm_field", "pgm_set_row_capacity"):
        getattr(lib, n).restype = C.c_int
    _lib = lib
    return lib


def check_mpnn(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"pgm_b200 error {rc}: {load().pgm_mpnn_last_error().decode()}")


def check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"pgm_b200 error {rc}: {load().pgm_last_error().decode()}")
