"""ctypes binding of libdense_b200.so (C ABI in include/dense_b200.h).

The shared library is the only compute path: if it is missing or cannot be
loaded, every call raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import re
from typing import List

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "_build", "libdense_b200.so")
HEADER = os.path.join(ROOT, "include", "dense_b200.h")

(DN_OK, DN_INVALID_ARG, DN_OUT_OF_MEMORY, DN_DEVICE_ERROR, DN_TIMEOUT, DN_NOT_READY,
 DN_OUT_OF_RANGE) = range(7)
DN_RUN_CLEAN, DN_RUN_PRUNE, DN_RUN_GRAPH, DN_RUN_INIT, DN_RUN_TIMING = 1, 2, 4, 8, 16
DN_RUN_LEARNED = 32

_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_f = ctypes.POINTER(ctypes.c_float)
_u8 = ctypes.POINTER(ctypes.c_uint8)
_i32 = ctypes.POINTER(ctypes.c_int32)
_vp = ctypes.c_void_p
_i = ctypes.c_int


class DenseError(RuntimeError):
    """A device-side failure reported by the library (status and message)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


_SIGNATURES = {
    "dn_last_error": ([], ctypes.c_char_p),
    "dn_version": ([], ctypes.c_char_p),
    "dn_device_count": ([], ctypes.c_int),
    "dn_set_device": ([ctypes.c_int], ctypes.c_int),
    "dn_estimator_create": ([ctypes.POINTER(_vp)], _i),
    "dn_estimator_destroy": ([_vp], _i),
    "dn_estimator_add_view": ([_vp, _d, _d, _d, _u8, _u8, _i, _i, _i], _i),
    "dn_estimator_set_depth_range": ([_vp, ctypes.c_double, ctypes.c_double, _i], _i),
    "dn_estimator_set_patchmatch_iterations": ([_vp, _i], _i),
    "dn_estimator_set_patch_size": ([_vp, _i], _i),
    "dn_estimator_set_min_patch_sd": ([_vp, ctypes.c_float], _i),
    "dn_estimator_set_seed": ([_vp, ctypes.c_uint64], _i),
    "dn_estimator_compute_brute_force": ([_vp, _f, _f, _f, _i32], _i),
    "dn_estimator_compute_patch_match": ([_vp, _f, _f, _f, _i32], _i),
    "dn_estimator_compute_patch_match_sample": ([_vp, _f, _f, _f, _i32], _i),
    "dn_estimator_score_planes": ([_vp, _f, _f, _i32], _i),
    "dn_estimator_compute_patch_match_init": ([_vp, _f, _f, _f, _f, _i32], _i),
    "dn_estimator_last_taps": ([_vp, ctypes.POINTER(ctypes.c_uint64)], _i),
    "dn_cleaner_create": ([ctypes.POINTER(_vp)], _i),
    "dn_cleaner_destroy": ([_vp], _i),
    "dn_cleaner_set_same_depth_threshold": ([_vp, ctypes.c_float], _i),
    "dn_cleaner_set_min_consistent_views": ([_vp, _i], _i),
    "dn_cleaner_add_view": ([_vp, _d, _d, _d, _f, _i, _i, _i], _i),
    "dn_cleaner_clean": ([_vp, _f], _i),
    "dn_pruner_create": ([ctypes.POINTER(_vp)], _i),
    "dn_pruner_destroy": ([_vp], _i),
    "dn_pruner_set_same_depth_threshold": ([_vp, ctypes.c_float], _i),
    "dn_pruner_add_view": ([_vp, _d, _d, _d, _f, _f, _u8, _u8, _i, _i], _i),
    "dn_pruner_prune": ([_vp, ctypes.POINTER(ctypes.c_int64)], _i),
    "dn_pruner_fetch": ([_vp, _f, _f, _u8, _u8, ctypes.c_int64], _i),
    "dn_batch_create": ([ctypes.POINTER(_vp)], _i),
    "dn_batch_destroy": ([_vp], _i),
    "dn_batch_add_view": ([_vp, _d, _d, _d, _u8, _u8, _i, _i, _i, ctypes.POINTER(_i)], _i),
    "dn_batch_add_depthmap": ([_vp, _i, _i32, _i, ctypes.c_double, ctypes.c_double,
                               ctypes.POINTER(_i)], _i),
    "dn_batch_set_clean_views": ([_vp, _i, _i32, _i], _i),
    "dn_batch_set_params": ([_vp, _i, ctypes.c_float, _i, ctypes.c_float, _i, ctypes.c_uint64], _i),
    "dn_batch_run": ([_vp, ctypes.c_uint], _i),
    "dn_batch_synchronize": ([_vp], _i),
    "dn_batch_get_depthmap": ([_vp, _i, _f, _f, _f, _i32, _f], _i),
    "dn_batch_get_depths": ([_vp, _i, _i32, _vp, _i], _i),
    "dn_batch_get_depths_async": ([_vp, _i, _i32, _vp, _i], _i),
    "dn_batch_set_init": ([_vp, _i, _f], _i),
    "dn_batch_set_schedule": ([_vp, _i, _i, _i, _i, ctypes.c_float, ctypes.c_float], _i),
    "dn_batch_set_candidate_views": ([_vp, _i], _i),
    "dn_batch_set_active_pixels": ([_vp, _i, ctypes.c_float], _i),
    "dn_batch_set_active_lists": ([_vp, _i], _i),
    "dn_batch_set_active_seed": ([_vp, ctypes.c_float], _i),
    "dn_batch_set_init_fallback": ([_vp, _i], _i),
    "dn_batch_set_proposal_scale": ([_vp, _i], _i),
    "dn_batch_set_knight_moves": ([_vp, _i], _i),
    "dn_batch_set_proposal_net": ([_vp, ctypes.POINTER(ctypes.c_uint16), _f, _i, _i], _i),
    "dn_batch_pruned_count": ([_vp, ctypes.POINTER(ctypes.c_int64)], _i),
    "dn_batch_get_points": ([_vp, _i, _f, _f, _u8, _u8, ctypes.c_int64,
                             ctypes.POINTER(ctypes.c_int64)], _i),
    "dn_batch_last_taps": ([_vp, ctypes.POINTER(ctypes.c_uint64)], _i),
    "dn_batch_set_view_image": ([_vp, _i, _u8, _i], _i),
    "dn_batch_upload_view_image": ([_vp, _i, _u8, _i], _i),
    "dn_batch_last_timings": ([_vp, _f, _i, ctypes.POINTER(ctypes.c_uint64)], _i),
    "dn_batch_copy_depth_device": ([_vp, _i, _vp], _i),
    "dn_batch_timer_record": ([_vp, _i], _i),
    "dn_batch_set_tuning": ([_vp, _i, _i, _i], _i),
    "dn_estimator_set_tuning": ([_vp, _i, _i, _i], _i),
    "dn_batch_timer_elapsed": ([_vp, _f], _i),
    "dn_postprocess_depth": ([_f, _f, _i, _i], _i),
    "dn_check_bounded_wait": ([_i, ctypes.c_int64, _f], _i),
    "dn_fp32_peak": ([ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)], _i),
    "dn_walk_ceiling": ([ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)], _i),
    "dn_batch_sweep_features": ([_vp, _vp, ctypes.c_int64, _i, _i], _i),
    "dn_batch_targets": ([_vp, _vp, ctypes.c_int64, ctypes.c_float, _i], _i),
    "dn_batch_init_from_output": ([_vp, _i, _vp], _i),
    "dn_nn_conv3x3_forward": ([_vp, _vp, _vp, ctypes.c_int64, _i, _i, _i, _i, _i, _vp, _vp, _vp], _i),
    "dn_nn_conv3x3_forward_mma_sync": ([_vp, _vp, _vp, ctypes.c_int64, _i, _i, _i, _i, _i, _vp,
                                        _vp, _vp], _i),
    "dn_nn_synchronize": ([_vp], _i),
    "dn_gpu_cleaner_create": ([ctypes.POINTER(_vp)], _i),
    "dn_gpu_cleaner_destroy": ([_vp], _i),
    "dn_gpu_cleaner_set_same_depth_threshold": ([_vp, ctypes.c_float], _i),
    "dn_gpu_cleaner_set_min_consistent_views": ([_vp, _i], _i),
    "dn_gpu_cleaner_set_carving_threshold": ([_vp, ctypes.c_float], _i),
    "dn_gpu_cleaner_set_max_carved_views": ([_vp, _i], _i),
    "dn_gpu_cleaner_set_device": ([_vp, _i], _i),
    "dn_gpu_cleaner_add_view": ([_vp, _d, _d, _d, _f, _i, _i, _i, ctypes.POINTER(_i)], _i),
    "dn_gpu_cleaner_clean": ([_vp, _i, _i32, _i, _f], _i),
    "dn_gpu_cleaner_clear": ([_vp], _i),
    "dn_fuser_create": ([ctypes.POINTER(_vp)], _i),
    "dn_fuser_destroy": ([_vp], _i),
    "dn_fuser_set_min_num_consistent": ([_vp, _i], _i),
    "dn_fuser_set_max_reproj_error": ([_vp, ctypes.c_float], _i),
    "dn_fuser_set_max_depth_error": ([_vp, ctypes.c_float], _i),
    "dn_fuser_set_max_normal_error": ([_vp, ctypes.c_float], _i),
    "dn_fuser_set_border_margin": ([_vp, _i], _i),
    "dn_fuser_set_sor_params": ([_vp, _i, ctypes.c_float], _i),
    "dn_fuser_set_behind_depth_factor": ([_vp, ctypes.c_float], _i),
    "dn_fuser_add_view": ([_vp, _d, _d, _d, _f, _f, _u8, _u8, _i, _i, _i32, _i, _i], _i),
    "dn_fuser_fuse": ([_vp, ctypes.POINTER(ctypes.c_int64)], _i),
    "dn_fuser_get": ([_vp, _f, _f, _u8, ctypes.c_int64], _i),
    "dn_fuser_last_error": ([], ctypes.c_char_p),
    "dn_fuser_last_removal_ms": ([_vp, ctypes.POINTER(ctypes.c_float)], _i),
    "dn_sor_filter": ([_f, ctypes.c_int64, _i, ctypes.c_float, _u8, _f], _i),
    "dn_svo_create": ([ctypes.POINTER(_vp)], _i),
    "dn_svo_destroy": ([_vp], _i),
    "dn_svo_set_voxel_size": ([_vp, ctypes.c_float], _i),
    "dn_svo_set_trunc_factor": ([_vp, ctypes.c_float], _i),
    "dn_svo_set_min_weight": ([_vp, ctypes.c_float], _i),
    "dn_svo_set_device": ([_vp, _i], _i),
    "dn_svo_set_bbox": ([_vp, _f, _f], _i),
    "dn_svo_add_view": ([_vp, _d, _d, _d, _f, _f, _u8, _u8, _f, _i, _i], _i),
    "dn_svo_count_voxels": ([_vp, ctypes.POINTER(ctypes.c_uint32)], _i),
    "dn_svo_fuse": ([_vp, ctypes.POINTER(ctypes.c_int64)], _i),
    "dn_svo_get": ([_vp, _f, _f, _u8, ctypes.c_int64], _i),
    "dn_svo_last_fuse_ms": ([_vp, ctypes.POINTER(ctypes.c_float)], _i),
    "dn_svo_last_error": ([], ctypes.c_char_p),
    "dn_acmmp_create": ([ctypes.POINTER(_vp)], _i),
    "dn_acmmp_destroy": ([_vp], _i),
    "dn_acmmp_set_max_iterations": ([_vp, _i], _i),
    "dn_acmmp_set_patch_size": ([_vp, _i], _i),
    "dn_acmmp_set_max_image_size": ([_vp, _i], _i),
    "dn_acmmp_set_hierarchy_levels": ([_vp, _i], _i),
    "dn_acmmp_set_sigma_spatial": ([_vp, ctypes.c_float], _i),
    "dn_acmmp_set_sigma_color": ([_vp, ctypes.c_float], _i),
    "dn_acmmp_set_top_k": ([_vp, _i], _i),
    "dn_acmmp_set_census_weight": ([_vp, ctypes.c_float], _i),
    "dn_acmmp_set_smooth_weight": ([_vp, ctypes.c_float], _i),
    "dn_acmmp_set_geom_consistency_weight": ([_vp, ctypes.c_float], _i),
    "dn_acmmp_set_device": ([_vp, _i], _i),
    "dn_acmmp_begin_ref_view": ([_vp, _d, _d, _d, _u8, _i, _i, _i, ctypes.c_float,
                                 ctypes.c_float, ctypes.POINTER(_i)], _i),
    "dn_acmmp_add_source_view": ([_vp, _d, _d, _d, _u8, _i, _i, _i], _i),
    "dn_acmmp_set_sfm_points": ([_vp, _d, ctypes.c_int64], _i),
    "dn_acmmp_add_geom_link": ([_vp, _i, _i, _i], _i),
    "dn_acmmp_run": ([_vp], _i),
    "dn_acmmp_num_refs": ([_vp, ctypes.POINTER(_i)], _i),
    "dn_acmmp_result_size": ([_vp, _i, ctypes.POINTER(_i), ctypes.POINTER(_i)], _i),
    "dn_acmmp_get_result": ([_vp, _i, _f, _f, _f, _f], _i),
    "dn_acmmp_last_run_ms": ([_vp, ctypes.POINTER(ctypes.c_float)], _i),
    "dn_acmmp_clear": ([_vp], _i),
    "dn_acmmp_last_error": ([], ctypes.c_char_p),
    "dn_delaunay_2d": ([_d, _i, _i, _i, ctypes.POINTER(_i), _i, ctypes.POINTER(_i)], _i),
    "dn_xxh32": ([_vp, ctypes.c_int64, ctypes.c_uint32], ctypes.c_uint32),
    "dn_lz4f_compress_bound": ([ctypes.c_int64], ctypes.c_int64),
    "dn_lz4f_compress": ([_vp, ctypes.c_int64, _vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)],
                         _i),
    "dn_lz4f_decompress": ([_vp, ctypes.c_int64, _vp, ctypes.c_int64,
                            ctypes.POINTER(ctypes.c_int64)], _i),
    "dn_io_last_error": ([], ctypes.c_char_p),
    "dn_nn_conv3x3_backward": ([_vp, _vp, _vp, _vp, ctypes.c_int64, _i, _i, _i, _i, _vp, _vp, _vp,
                                _vp, _vp], _i),
    "dn_nn_backward_scratch_bytes": ([ctypes.c_int64, _i], ctypes.c_int64),
    "dn_nn_conv3x3_backward_tc": ([_vp, _vp, _vp, _vp, ctypes.c_int64, _i, _i, _i, _i, _vp, _vp,
                                   _vp, _vp, ctypes.c_int64, _vp], _i),
    "dn_nn_l1_loss": ([_vp, _vp, ctypes.c_int64, ctypes.c_float, _vp, _vp, _vp, _vp], _i),
    "dn_nn_adam": ([_vp, _vp, _vp, _vp, _i, _vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                    ctypes.c_float, ctypes.c_float, ctypes.c_float, _vp, _vp], _i),
    "dn_prune_noalloc": ([_vp, _i, ctypes.c_float, _vp, _vp, _vp, _vp, ctypes.c_int64, _vp, _vp], _i),
    "dn_noalloc_last_error": ([], ctypes.c_char_p),
}


class PruneView(ctypes.Structure):
    """dn_prune_view (include/dense_b200.h): host camera, device buffers."""

    _fields_ = [("K", ctypes.c_double * 9), ("R", ctypes.c_double * 9), ("t", ctypes.c_double * 3),
                ("depth", ctypes.c_void_p), ("plane", ctypes.c_void_p), ("color", ctypes.c_void_p),
                ("label", ctypes.c_void_p), ("width", ctypes.c_int), ("height", ctypes.c_int)]


def header_symbols() -> List[str]:
    """Function names declared in include/dense_b200.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(dn_[a-z0-9_]+)\s*\(", text)))


def load():
    """Loads the library (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    lib = ctypes.CDLL(LIB_PATH)
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(status: int) -> None:
    if status == DN_OK:
        return
    msg = load().dn_last_error().decode(errors="replace")
    if status == DN_INVALID_ARG:
        raise ValueError(msg)
    if status == DN_OUT_OF_MEMORY:
        raise MemoryError(msg)
    if status == DN_OUT_OF_RANGE:
        raise IndexError(msg)
    raise DenseError(status, msg)


def ptr(a, t):
    return a.ctypes.data_as(t)
