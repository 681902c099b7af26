# SPDX-License-Identifier: Apache-2.0
"""ctypes binding of liballoy_dfsph.so (include/alloy_dfsph.h). There is no fallback: if the library is missing or
does not load, ``lib()`` raises."""

from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "liballoy_dfsph.so"

ADF_OK, ADF_ERR_VALUE, ADF_ERR_CAPACITY, ADF_ERR_CUDA, ADF_ERR_STATE = 0, 1, 2, 3, 4
ADF_NOALLOC_MAX_WORLDS, ADF_NOALLOC_MAX_CHUNKS = 16384, 65536  # include/alloy_dfsph.h

# every entry point of include/alloy_dfsph.h
EXPORTS = ("adf_last_error", "adf_create", "adf_destroy", "adf_step", "adf_density_ratio", "adf_get_report",
           "adf_active_mass", "adf_get_warm_starts", "adf_set_warm_starts", "adf_state_arrays", "adf_reset",
           "adf_add_emitter", "adf_set_emitter_pool", "adf_emitter_state", "adf_set_emitter_enabled", "adf_add_sink",
           "adf_neighbor_rows", "adf_debug_field", "adf_world_sum", "adf_kernel_launches", "adf_profile_enable",
           "adf_profile_read", "adf_list_stats", "adf_world_sum_noalloc", "adf_set_graphs", "adf_mlp_create",
           "adf_mlp_destroy", "adf_mlp_set_params", "adf_mlp_get_params", "adf_mlp_forward", "adf_mlp_gradient",
           "adf_mlp_train_step", "adf_mlp_status", "adf_set_warm_model", "adf_set_feature_recording",
           "adf_warm_features", "adf_set_warm_judging", "adf_set_autotune", "adf_tuned_configs", "adf_add_emitters",
           "adf_prime", "adf_iteration_work", "adf_set_tuned_config", "adf_get_state_storage", "adf_port_take",
           "adf_port_emit", "adf_energy", "adf_stable_dt", "adf_skin_flags",
           "adf_add_patch_emitter", "adf_trigger", "adf_mlp_set_wait_limit", "adf_mlp_clear_status",
           "adf_set_persistent", "adf_set_barrier_wait", "adf_clear_status", "adf_set_halo", "adf_halo_stats")
TUNE_KERNELS = ("density_alpha", "solve_init", "accel", "jacobi", "xsph", "lists")  # ADF_TUNE_KERNELS, in order
MLP_PARAMS, MLP_FEATURES = 5378, 16  # ADF_MLP_PARAMS, ADF_MLP_FEATURES
PROF_KINDS = ("sort", "lists", "wall_slots", "density_alpha", "solve_init", "accel", "jacobi", "reduce_check",
              "apply", "xsph", "finish", "emit", "warm_start", "halo")


class Params(C.Structure):
    """adf_params"""
    _fields_ = [("kind", C.c_int), ("particle_radius", C.c_double), ("h", C.c_double), ("sigma", C.c_double),
                ("n_full", C.c_double), ("tot_min", C.c_double), ("lattice_grad", C.c_double),
                ("wall_offset", C.c_double), ("wall_amplitude", C.c_double), ("taper0", C.c_double),
                ("taper1", C.c_double), ("reach", C.c_double), ("tol_den", C.c_double), ("tol_div", C.c_double),
                ("max_error_factor", C.c_double), ("min_it", C.c_int), ("max_it", C.c_int), ("omega", C.c_double),
                ("warm_den", C.c_double), ("warm_div", C.c_double), ("min_nb", C.c_double),
                ("divergence_solve", C.c_int), ("two_sided", C.c_int), ("xsph_c", C.c_double),
                ("capacity", C.c_int), ("v_sep", C.c_double), ("relief_speed", C.c_double),
                ("project_eps", C.c_double), ("has_bounds", C.c_int), ("bounds_lo", C.c_double * 3),
                ("bounds_hi", C.c_double * 3), ("cg", C.c_int), ("wall_friction", C.c_int), ("skin", C.c_double),
                ("skin_cap", C.c_int), ("jitter_speed", C.c_double), ("jitter_ratio", C.c_double),
                ("tol_den_min", C.c_double)]


class ModelDesc(C.Structure):
    """adf_model"""
    _fields_ = [("n", C.c_int), ("world_count", C.c_int), ("world_start", C.POINTER(C.c_int32)),
                ("q_host", C.POINTER(C.c_float)), ("mass", C.c_void_p), ("rest_density", C.c_void_p),
                ("radius", C.c_void_p), ("flags", C.c_void_p), ("phase", C.c_void_p), ("world", C.c_void_p),
                ("gravity", C.c_void_p), ("n_shapes", C.c_int), ("shape_start", C.POINTER(C.c_int32)),
                ("shape_ids", C.POINTER(C.c_int32)), ("shape_box", C.POINTER(C.c_float)), ("sweep_len", C.c_double),
                ("shape_geo", C.POINTER(C.c_int32)), ("shape_quat", C.POINTER(C.c_float))]


class Report(C.Structure):
    """adf_report"""
    _fields_ = [(name, C.c_void_p) for name in (
        "density_err", "divergence_err", "iters_density", "iters_divergence", "mass_in", "mass_out", "mass_initial",
        "escaped", "neighbor_overflow", "max_speed", "density_err_max", "projected", "nonfinite", "emitter_overflow",
        "density_tol", "learned_divergence", "learned_density", "swept")]


class StateStorage(C.Structure):
    """adf_state_storage"""
    _fields_ = [("mass_in", C.c_void_p), ("mass_out", C.c_void_p), ("escaped", C.c_void_p), ("emit_t", C.c_void_p),
                ("emit_cursor", C.c_void_p), ("emit_world", C.c_void_p), ("n_emitters", C.c_int32),
                ("port_stack", C.c_void_p), ("port_top", C.c_void_p), ("port_absorbed", C.c_void_p),
                ("port_emitted", C.c_void_p), ("port_retired", C.c_void_p), ("port_taken", C.c_void_p),
                ("port_granted", C.c_void_p), ("n_patch_entries", C.c_int32), ("patch_pending", C.c_void_p),
                ("patch_fired", C.c_void_p), ("patch_world", C.c_void_p), ("warm_probe_gap", C.c_void_p),
                ("warm_probe_wait", C.c_void_p)]


_lib = None


def lib() -> C.CDLL:
    """Load (once) and declare the library. Raises when it is missing: this package has no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"liballoy_dfsph.so not found at {LIB_PATH}; build it with `python -m alloy_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    P, vp, i = C.c_void_p, C.c_void_p, C.c_int
    L.adf_last_error.restype = C.c_char_p
    L.adf_create.argtypes = [C.POINTER(Params), C.POINTER(ModelDesc), i, C.POINTER(P)]
    L.adf_destroy.argtypes = [P]
    L.adf_destroy.restype = None
    L.adf_step.argtypes = [P, vp, vp, vp, vp, vp, C.c_double, vp]
    L.adf_density_ratio.argtypes = [P, vp, vp, vp, vp, vp]
    L.adf_get_report.argtypes = [P, C.POINTER(Report), vp]
    L.adf_active_mass.argtypes = [P, vp, vp]
    L.adf_get_warm_starts.argtypes = [P, vp, vp, vp]
    L.adf_set_warm_starts.argtypes = [P, vp, vp, vp]
    L.adf_state_arrays.argtypes = [P, C.POINTER(vp), C.POINTER(vp)]
    L.adf_reset.argtypes = [P, vp, vp, vp, vp]
    L.adf_add_emitter.argtypes = [P, i, vp, vp, i, vp, C.c_float, vp, i]
    L.adf_set_emitter_pool.argtypes = [P, i, vp, i]
    L.adf_add_emitters.argtypes = [P, i, vp, vp, vp, vp, vp, vp, vp, vp]
    L.adf_prime.argtypes = [P, vp, vp, C.c_double, C.c_double, i, vp, vp]
    L.adf_iteration_work.argtypes = [P, vp, vp]
    L.adf_set_tuned_config.argtypes = [P, i, i, i]
    L.adf_emitter_state.argtypes = [P, vp, vp]
    L.adf_set_emitter_enabled.argtypes = [P, i, i]
    L.adf_add_sink.argtypes = [P, i, vp, vp]
    L.adf_neighbor_rows.argtypes = [P, vp, vp, vp]
    L.adf_debug_field.argtypes = [P, C.c_char_p, vp, vp]
    L.adf_world_sum.argtypes = [P, vp, vp, vp, vp]
    L.adf_kernel_launches.argtypes = [P]
    L.adf_kernel_launches.restype = C.c_int64
    L.adf_profile_enable.argtypes = [P, i]
    L.adf_profile_read.argtypes = [P, vp, vp]
    L.adf_list_stats.argtypes = [P, vp, vp, vp]
    L.adf_world_sum_noalloc.argtypes = [vp, i, vp, i, vp, vp, vp]
    L.adf_set_graphs.argtypes = [P, i]
    L.adf_mlp_create.argtypes = [vp, i, C.POINTER(P)]
    L.adf_mlp_destroy.argtypes = [P]
    L.adf_mlp_destroy.restype = None
    L.adf_mlp_set_params.argtypes = [P, vp]
    L.adf_mlp_get_params.argtypes = [P, vp]
    L.adf_mlp_forward.argtypes = [P, vp, i, vp, vp]
    L.adf_mlp_gradient.argtypes = [P, vp, vp, vp, i, vp, vp, vp]
    L.adf_mlp_train_step.argtypes = [P, vp, vp, vp, i, C.c_float, vp, vp]
    L.adf_mlp_status.argtypes = [P]
    L.adf_set_warm_model.argtypes = [P, P, vp]
    L.adf_set_feature_recording.argtypes = [P, i]
    L.adf_warm_features.argtypes = [P, vp, vp]
    L.adf_set_warm_judging.argtypes = [P, i]
    L.adf_set_persistent.argtypes = [P, i]
    L.adf_set_halo.argtypes = [P, i]
    L.adf_halo_stats.argtypes = [P, vp, vp, vp]
    L.adf_set_barrier_wait.argtypes = [P, C.c_longlong, i]
    L.adf_clear_status.argtypes = [P]
    L.adf_set_autotune.argtypes = [P, i]
    L.adf_tuned_configs.argtypes = [P, vp, vp, vp]
    L.adf_get_state_storage.argtypes = [P, C.POINTER(StateStorage)]
    L.adf_port_take.argtypes = [P, vp, vp, i, vp]
    L.adf_port_emit.argtypes = [P, vp, vp, vp, vp, i, vp, vp]
    L.adf_energy.argtypes = [P, vp, vp, vp, vp, vp]
    L.adf_stable_dt.argtypes = [P, vp, C.c_double, C.c_double, C.c_double, vp, vp]
    L.adf_skin_flags.argtypes = [P, vp, vp]
    L.adf_add_patch_emitter.argtypes = [P, C.c_int, vp, vp, vp, vp, vp]
    L.adf_trigger.argtypes = [P, C.c_int, vp, C.c_int, vp]
    L.adf_mlp_set_wait_limit.argtypes = [P, C.c_uint32]
    L.adf_mlp_clear_status.argtypes = [P]
    for name in EXPORTS:
        if name not in ("adf_destroy", "adf_last_error", "adf_kernel_launches", "adf_mlp_destroy"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


class CapacityError(RuntimeError):
    """A fixed capacity was exceeded (alloy.core.errors.CapacityError's role)."""


def check(rc: int, what: str = "") -> int:
    """Map an ADF status code to the reference's exception types."""
    if rc >= 0 and rc == ADF_OK:
        return rc
    code = -rc if rc < 0 else rc
    msg = lib().adf_last_error().decode(errors="replace")
    text = f"{what}: {msg}" if what and msg and not msg.startswith(what) else (msg or what)
    if code == ADF_ERR_VALUE:
        raise ValueError(text)
    if code == ADF_ERR_CAPACITY:
        raise CapacityError(text)
    raise RuntimeError(f"liballoy_dfsph error {code}: {text}")
