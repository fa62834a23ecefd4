"""Loader and ctypes prototypes of libamrgpu.so (declared in include/amrgpu.h).

The library is built in-tree (``amr-demo_b200/lib/libamrgpu.so``) by
``make -C amr-demo_b200``. Loading fails loudly when it is missing: there is
no CPU fallback for the GPU path.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libamrgpu.so")

_lib = None

i32p = C.POINTER(C.c_int)
i64p = C.POINTER(C.c_int64)
f64p = C.POINTER(C.c_double)
f32p = C.POINTER(C.c_float)
u16p = C.POINTER(C.c_uint16)


class ConfigStruct(C.Structure):
    """amrgpu_config_t."""

    _fields_ = [
        ("dim", C.c_int), ("nfields", C.c_int), ("nelem_subgrid", C.c_int),
        ("coarse_grid_h", C.c_double),
        ("initial_condition", C.c_int),
        ("bc", C.c_int * 6),
        ("time_scheme", C.c_int), ("time_steps", C.c_int),
        ("dt", C.c_double), ("cfl", C.c_double),
        ("mach", C.c_double), ("alpha", C.c_double), ("beta", C.c_double),
        ("gamma", C.c_double), ("density", C.c_double), ("pressure", C.c_double),
        ("checkpoint_interval", C.c_int), ("visualization_interval", C.c_int),
        ("regrid_interval", C.c_int),
        ("amr_ntag_methods", C.c_int),
        ("amr_tag_methods", C.c_int * 5),
        ("amr_tag_tolerances", C.c_double * 5),
        ("form", C.c_int),
        ("final_time", C.c_double),
        ("ic_params", C.c_double * 8),
        ("ic_seed", C.c_uint64),
        ("noise_amplitude", C.c_double),
    ]


class MeshStruct(C.Structure):
    """amrgpu_mesh_t."""

    _fields_ = [("ncell", C.c_int), ("nghost", C.c_int), ("nface", C.c_int), ("dof", C.c_int),
                ("cell_info", i32p), ("face_info", i32p), ("geom", f64p)]


class JudgeStruct(C.Structure):
    """amrgpu_judge_t."""

    _fields_ = [("judged", C.c_int), ("disagree", C.c_int), ("rate", C.c_double), ("coarser", C.c_int)]


class ReportStruct(C.Structure):
    """amrgpu_report_t."""

    _fields_ = [("steps_done", C.c_int), ("time", C.c_double), ("dt_last", C.c_double),
                ("residual_norm", C.c_double), ("error", C.c_int), ("nan_detected", C.c_int)]


# name -> (restype, argtypes); the exported symbols of include/amrgpu.h
PROTOTYPES = {
    # Part 1: the reference ABI
    "hpc_amr_initialize_solver": (None, [i32p] * 2 + [f64p] + [i32p] * 9),
    "hpc_amr_initialize_quadrant": (None, [i32p] * 5 + [f64p] * 3),
    "hpc_amr_regrid_points": (None, [i32p, i32p, f64p, f64p]),
    "hpc_amr_tag_feature": (None, [i32p] * 5 + [f64p] * 3 + [i32p]),
    "hpc_amr_coarsen_operator_2d": (None, [i32p] * 4 + [f64p] * 7),
    "hpc_amr_refine_operator_2d": (None, [i32p] * 4 + [f64p] * 7),
    "hpc_amr_evolve_solver": (None, [i32p] * 15 + [f64p] * 2 + [i32p] * 5 + [C.c_ssize_t] + [f64p] * 3),
    "physics_go_gpu": (None, [i32p] * 15 + [f64p] * 2 + [i32p] * 5 + [C.c_ssize_t] + [f64p] * 3),
    # Part 2: errors and configuration
    "amrgpu_last_error": (C.c_int, []),
    "amrgpu_evolve_config": (C.c_int, [C.c_int, C.POINTER(ConfigStruct)]),
    "amrgpu_set_comm_ops": (C.c_int, [C.c_void_p]),
    "amrgpu_session_set_patch_rule": (C.c_int, [C.c_void_p, i32p, C.c_int]),
    "amrgpu_has_comm_ops": (C.c_int, []),
    "amrgpu_session_autotune": (C.c_int, [C.c_void_p, C.c_int]),
    "amrgpu_session_launch_variant_info": (C.c_int, [C.c_void_p, C.c_int, i32p, i32p, i32p, i32p]),
    "amrgpu_tune_cache_get": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, i32p, i32p, i32p, f64p]),
    "amrgpu_tune_cache_put": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_double]),
    "amrgpu_tune_cache_reload": (None, []),
    "amrgpu_error_string": (C.c_char_p, [C.c_int]),
    "amrgpu_last_error_message": (C.c_char_p, []),
    "amrgpu_clear_error": (None, []),
    "amrgpu_config_defaults": (None, [C.POINTER(ConfigStruct)]),
    "amrgpu_config_read": (C.c_int, [C.c_char_p, C.POINTER(ConfigStruct)]),
    "amrgpu_config_get": (C.c_int, [C.POINTER(ConfigStruct)]),
    "amrgpu_config_set": (C.c_int, [C.POINTER(ConfigStruct)]),
    # sessions
    "amrgpu_session_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(MeshStruct), C.POINTER(ConfigStruct)]),
    "amrgpu_session_destroy": (None, [C.c_void_p]),
    "amrgpu_session_set_form": (C.c_int, [C.c_void_p, C.c_int]),
    "amrgpu_session_set_launch": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "amrgpu_session_upload": (C.c_int, [C.c_void_p, f64p]),
    "amrgpu_session_download": (C.c_int, [C.c_void_p, f64p]),
    "amrgpu_session_step": (C.c_int, [C.c_void_p, C.c_int]),
    "amrgpu_session_step_graph": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "amrgpu_session_sync": (C.c_int, [C.c_void_p, C.POINTER(ReportStruct)]),
    "amrgpu_session_rhs": (C.c_int, [C.c_void_p, f64p]),
    "amrgpu_session_cfl_dt": (C.c_int, [C.c_void_p, f64p]),
    "amrgpu_session_state_device": (C.c_void_p, [C.c_void_p, C.c_int]),
    "amrgpu_session_cells": (C.c_int, [C.c_void_p]),
    "amrgpu_session_stream": (C.c_void_p, [C.c_void_p]),
    "amrgpu_session_launch_count": (C.c_int64, [C.c_void_p]),
    "amrgpu_session_totals": (C.c_int, [C.c_void_p, f64p]),
    "amrgpu_session_set_launch_variant": (C.c_int, [C.c_void_p, C.c_int]),
    "amrgpu_session_launch_variant": (C.c_int, [C.c_void_p]),
    "amrgpu_session_regrid_forest": (C.c_int, [C.c_void_p, C.c_void_p]),
    "amrgpu_forest_balance_device": (C.c_int, [C.c_void_p, C.c_void_p]),
    "amrgpu_forest_adapt": (C.c_int, [C.c_void_p, i32p, C.c_int, C.c_int, C.c_int, C.c_int]),
    "amrgpu_session_balance_regrid": (C.c_int, [C.c_void_p, C.c_void_p]),
    "amrgpu_session_adapt_regrid": (C.c_int, [C.c_void_p, C.c_void_p, i32p, i32p, C.c_int, C.c_int, C.c_int,
                                              C.c_int]),
    "amrgpu_session_holds_forest": (C.c_int, [C.c_void_p, C.c_void_p]),
    "amrgpu_session_reserve": (C.c_int, [C.c_void_p, C.c_longlong, C.c_int]),
    "amrgpu_session_balance_stall_test": (C.c_int, [C.c_void_p, C.c_void_p]),
    "amrgpu_session_quad_descriptors": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "amrgpu_session_face_count": (C.c_int, [C.c_void_p]),
    "amrgpu_session_step_stage": (C.c_int, [C.c_void_p, i32p, i32p]),
    "amrgpu_session_stage_input": (C.c_void_p, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "amrgpu_session_dt_slot": (C.c_void_p, [C.c_void_p]),
    "amrgpu_session_capture_mark": (C.c_int, [C.c_void_p]),
    "amrgpu_session_capture_rewind": (C.c_int, [C.c_void_p]),
    "amrgpu_session_advance": (C.c_int, [C.c_void_p, C.c_int]),
    "amrgpu_session_step_index": (C.c_longlong, [C.c_void_p]),
    "amrgpu_session_set_halo": (C.c_int, [C.c_void_p, i32p, C.c_int]),
    "amrgpu_session_halo_pack": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "amrgpu_session_halo_unpack": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "amrgpu_session_halo_unpack_edges": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "amrgpu_session_halo_pack_edges": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "amrgpu_session_local_scalars": (C.c_int, [C.c_void_p, f64p, i32p]),
    "amrgpu_session_tag": (C.c_int, [C.c_void_p, i32p]),
    "amrgpu_session_remap": (C.c_int, [C.c_void_p, C.c_void_p, i32p, i32p]),
    "amrgpu_session_regrid": (C.c_int, [C.c_void_p, C.c_void_p, i32p, i32p]),
    "amrgpu_session_launch_variants": (C.c_int, [C.c_void_p, i32p, i32p, C.c_int]),
    # forest
    "amrgpu_forest_new_brick": (C.c_void_p, [C.c_int] * 4 + [C.c_double] * 4 + [C.c_int]),
    "amrgpu_forest_destroy": (None, [C.c_void_p]),
    "amrgpu_forest_num_quads": (C.c_int, [C.c_void_p]),
    "amrgpu_forest_quads": (C.c_int, [C.c_void_p, i32p, i32p, i64p, i64p]),
    "amrgpu_forest_set_tags": (C.c_int, [C.c_void_p, i32p]),
    "amrgpu_forest_get_tags": (C.c_int, [C.c_void_p, i32p]),
    "amrgpu_forest_begin_regrid": (None, [C.c_void_p]),
    "amrgpu_forest_refine": (C.c_int, [C.c_void_p, i32p, C.c_int]),
    "amrgpu_forest_coarsen": (C.c_int, [C.c_void_p, i32p, C.c_int]),
    "amrgpu_forest_balance": (C.c_int, [C.c_void_p]),
    "amrgpu_forest_is_balanced": (C.c_int, [C.c_void_p]),
    "amrgpu_forest_remap": (C.c_int, [C.c_void_p, i32p, i32p]),
    "amrgpu_forest_max_faces": (C.c_int, [C.c_void_p]),
    "amrgpu_forest_external": (C.c_int, [C.c_void_p, C.c_int, C.c_int, i32p, i32p, f64p, i32p, i32p]),
    "amrgpu_forest_quad_h": (C.c_double, [C.c_void_p, C.c_int]),
    "amrgpu_forest_initialize": (C.c_int, [C.c_void_p, C.c_int, f64p]),
    # output
    "amrgpu_write_vtk": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, f64p, C.c_int]),
    "amrgpu_checkpoint_write": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, f64p, C.c_int, C.c_double]),
    "amrgpu_checkpoint_read_header": (C.c_int, [C.c_char_p, i32p, i32p, i32p, f64p]),
    "amrgpu_checkpoint_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p), f64p, C.c_longlong]),
    # learned refinement indicator
    "amrgpu_mlp_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_ulonglong]),
    "amrgpu_mlp_destroy": (None, [C.c_void_p]),
    "amrgpu_mlp_get_params": (C.c_int, [C.c_void_p, f32p]),
    "amrgpu_mlp_set_params": (C.c_int, [C.c_void_p, f32p]),
    "amrgpu_session_features": (C.c_int, [C.c_void_p, u16p]),
    "amrgpu_session_jumps": (C.c_int, [C.c_void_p, f64p]),
    "amrgpu_mlp_dataset_append": (C.c_longlong, [C.c_void_p, C.c_void_p, C.c_double, C.c_double]),
    "amrgpu_mlp_dataset_relabel": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_double, C.c_double]),
    "amrgpu_mlp_dataset_cover": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong, C.c_double, C.c_double]),
    "amrgpu_mlp_dataset_size": (C.c_longlong, [C.c_void_p]),
    "amrgpu_mlp_dataset_clear": (C.c_int, [C.c_void_p]),
    "amrgpu_mlp_dataset_labels": (C.c_int, [C.c_void_p, i32p, C.c_longlong]),
    "amrgpu_mlp_train_epoch": (C.c_int, [C.c_void_p, i32p, C.c_longlong, C.c_int, C.c_float, C.c_float, f64p, f64p]),
    "amrgpu_mlp_grad": (C.c_int, [C.c_void_p, u16p, i32p, C.c_int, f32p, f32p, f64p]),
    "amrgpu_mlp_predict": (C.c_int, [C.c_void_p, u16p, C.c_int, f32p]),
    "amrgpu_session_learned_tags": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_ulonglong, C.c_double,
                                              C.c_double, i32p, C.c_void_p]),
    # allocation-free entry point
    "amrgpu_totals_noalloc": (C.c_int, [C.c_void_p, C.c_longlong, C.c_void_p, C.c_int, C.c_int, f64p,
                                        C.c_void_p]),
}


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"libamrgpu.so not found at {LIB_PATH}; build it with `make -C amr-demo_b200` "
            "(there is no CPU fallback for the GPU path)")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


class AmrGpuError(RuntimeError):
    """A non-zero status from libamrgpu."""

    def __init__(self, code, where=""):
        L = lib()
        msg = L.amrgpu_last_error_message().decode(errors="replace")
        super().__init__(f"{where}: {L.amrgpu_error_string(code).decode()} ({code}): {msg}")
        self.code = code


def check(code, where=""):
    if code != 0:
        raise AmrGpuError(code, where)
    return code
