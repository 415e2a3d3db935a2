"""Drop-in for the legacy ``pydense`` classes of OpenSfM's dense path.

Mirrors ``opensfm/src/lib/dense/pydense.pyi:28-77`` (DepthmapCleaner,
DepthmapEstimator, DepthmapPruner) over the C ABI of libdense_b200.so:
same method names, argument order and meaning, same return layout:

* ``DepthmapEstimator.compute_*()`` -> ``[depth (H,W) f32, plane (H,W,3) f32,
  score (H,W) f32, nghbr (H,W) i32]`` (``DepthmapEstimatorResult``,
  ``depthmap.h:50-55``);
* ``DepthmapCleaner.clean()`` -> ``(H,W) f32``;
* ``DepthmapPruner.prune()`` -> ``[points (N,3) f32, normals (N,3) f32,
  colors (N,3) u8, labels (N,) u8]``.

Arrays are converted to C-contiguous float64 / uint8 / float32 as pybind11's
``forcecast`` would; inputs are copied at ``add_view``.  Bad shapes or values
raise ``ValueError``; device failures raise ``RuntimeError``
(``opensfm_b200._lib.DenseError``).  The library releases no Python lock of
its own; ctypes drops the GIL for the duration of each call.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import _d, _f, _i32, _u8, check, ptr

__all__ = ["DepthmapEstimator", "DepthmapCleaner", "DepthmapPruner", "GPUDepthmapCleaner",
           "DepthmapFuser", "SVOFuser", "DepthmapClusterEstimator", "Batch", "postprocess_depth",
           "sor_filter", "fp32_peak", "walk_ceiling"]


def postprocess_depth(depth: np.ndarray) -> np.ndarray:
    """PostProcess (``depthmap.cc:489-502``) of a depth map on the device."""
    d = np.ascontiguousarray(depth, dtype=np.float32)
    if d.ndim != 2:
        raise ValueError("depth must be 2-D")
    out = np.zeros_like(d)
    check(_lib.load().dn_postprocess_depth(ptr(d, _f), ptr(out, _f), d.shape[1], d.shape[0]))
    return out


def fp32_peak() -> float:
    """Measured FP32 FMA throughput of the current device, TFLOP/s."""
    tf = ctypes.c_double()
    ms = ctypes.c_double()
    check(_lib.load().dn_fp32_peak(ctypes.byref(tf), ctypes.byref(ms)))
    return float(tf.value)


def walk_ceiling() -> float:
    """Measured ceiling of the scoring walk on the current device, G taps/s:
    affine 7 x 7 table walks with their NCC sums alone (dn_walk_ceiling)."""
    gt = ctypes.c_double()
    ms = ctypes.c_double()
    check(_lib.load().dn_walk_ceiling(ctypes.byref(gt), ctypes.byref(ms)))
    return float(gt.value)


def _mat(a, shape, name):
    m = np.ascontiguousarray(a, dtype=np.float64)
    if m.size != int(np.prod(shape)):
        raise ValueError(f"{name} must have {int(np.prod(shape))} elements, got {m.size}")
    return m.reshape(shape)


def _image(a, name):
    im = np.ascontiguousarray(a)
    if im.ndim != 2:
        raise ValueError(f"{name} must be a 2-D array, got shape {im.shape}")
    return np.ascontiguousarray(im, dtype=np.uint8)


class _Handle:
    _destroy = None

    def __init__(self, create: str, destroy: str):
        self._L = _lib.load()
        h = ctypes.c_void_p()
        check(getattr(self._L, create)(ctypes.byref(h)))
        self._h = h
        self._destroy = getattr(self._L, destroy)

    def close(self):
        if getattr(self, "_h", None) is not None and self._destroy is not None:
            self._destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DepthmapEstimator(_Handle):
    """``dense::DepthmapEstimator`` (``depthmap.h:57-111``) on the B200."""

    def __init__(self) -> None:
        super().__init__("dn_estimator_create", "dn_estimator_destroy")
        self._shape = None

    def add_view(self, K, R, t, image, mask) -> None:
        K = _mat(K, (3, 3), "K")
        R = _mat(R, (3, 3), "R")
        t = _mat(t, (3,), "t")
        im = _image(image, "image")
        mk = _image(mask, "mask") if mask is not None else None
        if mk is not None and mk.shape != im.shape:
            raise ValueError("mask must have the image's shape")
        H, W = im.shape
        check(self._L.dn_estimator_add_view(
            self._h, ptr(K, _d), ptr(R, _d), ptr(t, _d), ptr(im, _u8),
            ptr(mk, _u8) if mk is not None else None, W, H, W))
        if self._shape is None:
            self._shape = (H, W)

    def set_depth_range(self, min_depth: float, max_depth: float, num_planes: int) -> None:
        check(self._L.dn_estimator_set_depth_range(self._h, float(min_depth), float(max_depth),
                                                    int(num_planes)))

    def set_patchmatch_iterations(self, n: int) -> None:
        check(self._L.dn_estimator_set_patchmatch_iterations(self._h, int(n)))

    def set_patch_size(self, size: int) -> None:
        check(self._L.dn_estimator_set_patch_size(self._h, int(size)))

    def set_min_patch_sd(self, sd: float) -> None:
        check(self._L.dn_estimator_set_min_patch_sd(self._h, float(sd)))

    def set_seed(self, seed: int) -> None:
        """Seed of the counter-based PatchMatch RNG (no reference counterpart)."""
        check(self._L.dn_estimator_set_seed(self._h, int(seed) & (2**64 - 1)))

    def _outputs(self):
        if self._shape is None:
            raise ValueError("DepthmapEstimator has no views")
        H, W = self._shape
        return (np.zeros((H, W), np.float32), np.zeros((H, W, 3), np.float32),
                np.zeros((H, W), np.float32), np.zeros((H, W), np.int32))

    def _run(self, fn, *extra) -> list:
        depth, plane, score, nghbr = self._outputs()
        check(fn(self._h, *extra, ptr(depth, _f), ptr(plane, _f), ptr(score, _f),
                 ptr(nghbr, _i32)))
        return [depth, plane, score, nghbr]

    def compute_brute_force(self) -> list:
        return self._run(self._L.dn_estimator_compute_brute_force)

    def compute_patch_match(self) -> list:
        return self._run(self._L.dn_estimator_compute_patch_match)

    def compute_patch_match_sample(self) -> list:
        return self._run(self._L.dn_estimator_compute_patch_match_sample)

    def compute_patch_match_init(self, init_planes) -> list:
        """PatchMatch from a given plane field (planes with z == 0 are drawn at random)."""
        H, W = self._outputs()[0].shape
        pl = np.ascontiguousarray(init_planes, dtype=np.float32)
        if pl.shape != (H, W, 3):
            raise ValueError(f"init planes must have shape {(H, W, 3)}")
        return self._run(self._L.dn_estimator_compute_patch_match_init, ptr(pl, _f))

    def score_planes(self, planes):
        """ComputePlaneScore (``depthmap.cc:408-419``) for every interior pixel."""
        H, W = self._outputs()[0].shape
        pl = np.ascontiguousarray(planes, dtype=np.float32)
        if pl.shape != (H, W, 3):
            raise ValueError(f"planes must have shape {(H, W, 3)}")
        score = np.zeros((H, W), np.float32)
        nghbr = np.zeros((H, W), np.int32)
        check(self._L.dn_estimator_score_planes(self._h, ptr(pl, _f), ptr(score, _f),
                                                ptr(nghbr, _i32)))
        return score, nghbr

    def last_taps(self) -> int:
        v = ctypes.c_uint64()
        check(self._L.dn_estimator_last_taps(self._h, ctypes.byref(v)))
        return int(v.value)

    def set_tuning(self, bx: int = 32, by: int = 4, variant: int = 2) -> None:
        check(self._L.dn_estimator_set_tuning(self._h, int(bx), int(by), int(variant)))


class DepthmapCleaner(_Handle):
    """``dense::DepthmapCleaner`` (``depthmap.h:113-129``) on the B200."""

    def __init__(self) -> None:
        super().__init__("dn_cleaner_create", "dn_cleaner_destroy")
        self._shape = None

    def set_same_depth_threshold(self, t: float) -> None:
        check(self._L.dn_cleaner_set_same_depth_threshold(self._h, float(t)))

    def set_min_consistent_views(self, n: int) -> None:
        check(self._L.dn_cleaner_set_min_consistent_views(self._h, int(n)))

    def add_view(self, K, R, t, depth) -> None:
        K = _mat(K, (3, 3), "K")
        R = _mat(R, (3, 3), "R")
        t = _mat(t, (3,), "t")
        d = np.ascontiguousarray(depth, dtype=np.float32)
        if d.ndim != 2:
            raise ValueError("depth must be a 2-D array")
        H, W = d.shape
        check(self._L.dn_cleaner_add_view(self._h, ptr(K, _d), ptr(R, _d), ptr(t, _d),
                                          ptr(d, _f), W, H, W))
        if self._shape is None:
            self._shape = (H, W)

    def clean(self) -> np.ndarray:
        if self._shape is None:
            raise ValueError("DepthmapCleaner has no views")
        out = np.zeros(self._shape, np.float32)
        check(self._L.dn_cleaner_clean(self._h, ptr(out, _f)))
        return out


class GPUDepthmapCleaner(_Handle):
    """``dense::GPUDepthmapCleaner`` (``cleaner.h:16-60``, ``pydense.pyi:129-149``)
    on the B200: forward and backward consistency with space carving."""

    def __init__(self) -> None:
        super().__init__("dn_gpu_cleaner_create", "dn_gpu_cleaner_destroy")
        self._shapes = []

    @staticmethod
    def is_available() -> bool:
        try:
            return _lib.load().dn_device_count() > 0
        except OSError:
            return False

    def set_same_depth_threshold(self, t: float) -> None:
        check(self._L.dn_gpu_cleaner_set_same_depth_threshold(self._h, float(t)))

    def set_min_consistent_views(self, n: int) -> None:
        check(self._L.dn_gpu_cleaner_set_min_consistent_views(self._h, int(n)))

    def set_carving_threshold(self, t: float) -> None:
        check(self._L.dn_gpu_cleaner_set_carving_threshold(self._h, float(t)))

    def set_max_carved_views(self, n: int) -> None:
        check(self._L.dn_gpu_cleaner_set_max_carved_views(self._h, int(n)))

    def set_device(self, device: int) -> None:
        """Views added after this call live on `device` (the reference binds
        one OpenCL device per cleaner)."""
        if self._shapes:
            raise ValueError("set_device must come before the first add_view")
        check(self._L.dn_gpu_cleaner_set_device(self._h, int(device)))

    def add_view(self, K, R, t, depth) -> None:
        K = _mat(K, (3, 3), "K")
        R = _mat(R, (3, 3), "R")
        t = _mat(t, (3,), "t")
        d = np.ascontiguousarray(depth, dtype=np.float32)
        if d.ndim != 2:
            raise ValueError("depth must be a 2-D array")
        H, W = d.shape
        check(self._L.dn_gpu_cleaner_add_view(self._h, ptr(K, _d), ptr(R, _d), ptr(t, _d),
                                              ptr(d, _f), W, H, W, None))
        self._shapes.append((H, W))

    def clean(self, ref_idx: int, neighbor_ids) -> np.ndarray:
        ids = np.ascontiguousarray(np.asarray(neighbor_ids).reshape(-1), dtype=np.int32)
        if not 0 <= int(ref_idx) < len(self._shapes):
            raise IndexError(f"Clean: ref_idx {ref_idx} out of range [0, {len(self._shapes)})")
        out = np.zeros(self._shapes[int(ref_idx)], np.float32)
        check(self._L.dn_gpu_cleaner_clean(self._h, int(ref_idx), ptr(ids, _i32), len(ids),
                                           ptr(out, _f)))
        return out

    def clear(self) -> None:
        check(self._L.dn_gpu_cleaner_clear(self._h))
        self._shapes = []


class DepthmapFuser(_Handle):
    """``dense::DepthmapFuser`` (``fuser.h:28-77``, ``pydense.pyi:80-102``):
    per-pixel fusion into points; the candidate observations of every pixel
    run on the B200, the raster-order marks and medians on the host."""

    def __init__(self) -> None:
        super().__init__("dn_fuser_create", "dn_fuser_destroy")
        self._n_primary_px = 0

    def _check(self, st: int) -> None:
        if st == _lib.DN_OK:
            return
        msg = self._L.dn_fuser_last_error().decode(errors="replace")
        if st == _lib.DN_INVALID_ARG:
            raise ValueError(msg)
        if st == _lib.DN_OUT_OF_MEMORY:
            raise MemoryError(msg)
        raise _lib.DenseError(st, msg)

    def set_min_num_consistent(self, n: int) -> None:
        self._check(self._L.dn_fuser_set_min_num_consistent(self._h, int(n)))

    def set_max_reproj_error(self, px: float) -> None:
        self._check(self._L.dn_fuser_set_max_reproj_error(self._h, float(px)))

    def set_max_depth_error(self, ratio: float) -> None:
        self._check(self._L.dn_fuser_set_max_depth_error(self._h, float(ratio)))

    def set_max_normal_error(self, degrees: float) -> None:
        self._check(self._L.dn_fuser_set_max_normal_error(self._h, float(degrees)))

    def set_border_margin(self, px: int) -> None:
        self._check(self._L.dn_fuser_set_border_margin(self._h, int(px)))

    def set_num_threads(self, n: int) -> None:
        """Accepted for compatibility: the result is the reference's
        single-thread result whatever the count."""

    def set_sor_params(self, knn: int, stddev_factor: float) -> None:
        """Statistical outlier removal after fusion (fuser.cc:66-69,
        374-482): knn <= 0 skips it; the default is knn 12, factor 2.5."""
        self._check(self._L.dn_fuser_set_sor_params(self._h, int(knn), float(stddev_factor)))

    def last_removal_ms(self) -> float:
        """Device time of the last fuse's outlier removal (0 when skipped)."""
        ms = ctypes.c_float()
        self._check(self._L.dn_fuser_last_removal_ms(self._h, ctypes.byref(ms)))
        return float(ms.value)

    def set_behind_depth_factor(self, factor: float) -> None:
        self._check(self._L.dn_fuser_set_behind_depth_factor(self._h, float(factor)))

    def add_view(self, K, R, t, depth, normal, color, mask, neighbor_ids,
                 primary: bool = True) -> None:
        K = _mat(K, (3, 3), "K")
        R = _mat(R, (3, 3), "R")
        t = _mat(t, (3,), "t")
        d = np.ascontiguousarray(depth, dtype=np.float32)
        if d.ndim != 2:
            raise ValueError("depth must be a 2-D array")
        H, W = d.shape
        n = np.ascontiguousarray(normal, dtype=np.float32)
        c = np.ascontiguousarray(color, dtype=np.uint8)
        if n.shape != (H, W, 3):
            raise ValueError("depth and normal must have matching shapes.")
        if c.shape != (H, W, 3):
            raise ValueError("depth and color must have matching shapes.")
        m = None
        if mask is not None and np.asarray(mask).size:
            m = np.ascontiguousarray(mask, dtype=np.uint8)
            if m.shape != (H, W):
                raise ValueError("mask must have the depth's shape")
        nb = np.ascontiguousarray(np.asarray(neighbor_ids).reshape(-1), dtype=np.int32)
        self._check(self._L.dn_fuser_add_view(
            self._h, ptr(K, _d), ptr(R, _d), ptr(t, _d), ptr(d, _f), ptr(n, _f), ptr(c, _u8),
            ptr(m, _u8) if m is not None else None, W, H, ptr(nb, _i32), int(nb.size),
            int(bool(primary))))

    def fuse(self) -> list:
        cnt = ctypes.c_int64()
        self._check(self._L.dn_fuser_fuse(self._h, ctypes.byref(cnt)))
        n = int(cnt.value)
        pts = np.zeros((n, 3), np.float32)
        nrm = np.zeros((n, 3), np.float32)
        clr = np.zeros((n, 3), np.uint8)
        self._check(self._L.dn_fuser_get(self._h, ptr(pts, _f), ptr(nrm, _f), ptr(clr, _u8), n))
        return [pts, nrm, clr]


class SVOFuser(_Handle):
    """``dense::SVOFuser`` (``svo_fuser.h:14-68``, bound at
    ``python/pybind.cc:37-51``): TSDF fusion into a sparse voxel hash on the
    B200, surface points at the TSDF's zero crossings.  Points come in
    ascending voxel order (the reference's order follows an atomic counter)."""

    def __init__(self) -> None:
        super().__init__("dn_svo_create", "dn_svo_destroy")
        self._counted = False

    def _check(self, st: int) -> None:
        if st == _lib.DN_OK:
            return
        msg = self._L.dn_svo_last_error().decode(errors="replace")
        if st == _lib.DN_INVALID_ARG:
            raise ValueError(msg)
        if st == _lib.DN_OUT_OF_MEMORY:
            raise MemoryError(msg)
        raise _lib.DenseError(st, msg)

    @staticmethod
    def is_gpu_available() -> bool:
        try:
            return GPUDepthmapCleaner.is_available()
        except Exception:
            return False

    def set_voxel_size(self, size: float) -> None:
        self._check(self._L.dn_svo_set_voxel_size(self._h, float(size)))

    def set_trunc_factor(self, factor: float) -> None:
        self._check(self._L.dn_svo_set_trunc_factor(self._h, float(factor)))

    def set_min_weight(self, w: float) -> None:
        self._check(self._L.dn_svo_set_min_weight(self._h, float(w)))

    def set_device(self, device_idx: int) -> None:
        self._check(self._L.dn_svo_set_device(self._h, int(device_idx)))

    def set_bbox(self, min_world, max_world) -> None:
        lo = np.ascontiguousarray(min_world, dtype=np.float32).reshape(3)
        hi = np.ascontiguousarray(max_world, dtype=np.float32).reshape(3)
        self._check(self._L.dn_svo_set_bbox(self._h, ptr(lo, _f), ptr(hi, _f)))

    def add_view(self, K, R, t, depth, normal, color, mask, confidence=None,
                 name: str = "") -> None:
        K = _mat(K, (3, 3), "K")
        R = _mat(R, (3, 3), "R")
        t = _mat(t, (3,), "t")
        d = np.ascontiguousarray(depth, dtype=np.float32)
        if d.ndim != 2:
            raise ValueError("depth must be a 2-D array")
        H, W = d.shape
        n = np.ascontiguousarray(normal, dtype=np.float32)
        c = np.ascontiguousarray(color, dtype=np.uint8)
        if n.ndim != 3 or n.shape[:2] != (H, W):
            raise ValueError("depth and normal must have matching shapes.")
        if c.ndim != 3 or c.shape[:2] != (H, W):
            raise ValueError("depth and color must have matching shapes.")
        if n.shape[2] != 3 or c.shape[2] != 3:
            raise ValueError("normal and color must have 3 channels")
        m = None
        if mask is not None and np.asarray(mask).size:
            m = np.ascontiguousarray(mask, dtype=np.uint8)
            if m.shape != (H, W):
                raise ValueError("mask must have the depth's shape")
        w = None
        if confidence is not None:
            cf = np.ascontiguousarray(confidence, dtype=np.float32)
            if cf.shape == (H, W):  # any other shape is ignored, as the reference does
                w = cf
        self._check(self._L.dn_svo_add_view(
            self._h, ptr(K, _d), ptr(R, _d), ptr(t, _d), ptr(d, _f), ptr(n, _f), ptr(c, _u8),
            ptr(m, _u8) if m is not None else None, ptr(w, _f) if w is not None else None,
            W, H))

    def count_voxels(self) -> int:
        n = ctypes.c_uint32()
        self._check(self._L.dn_svo_count_voxels(self._h, ctypes.byref(n)))
        self._counted = self._counted or n.value > 0
        return int(n.value)

    def fuse(self) -> list:
        cnt = ctypes.c_int64()
        st = self._L.dn_svo_fuse(self._h, ctypes.byref(cnt))
        if st == _lib.DN_INVALID_ARG:
            # The reference throws std::runtime_error here.
            raise RuntimeError(self._L.dn_svo_last_error().decode(errors="replace"))
        self._check(st)
        n = int(cnt.value)
        pts = np.zeros((n, 3), np.float32)
        nrm = np.zeros((n, 3), np.float32)
        clr = np.zeros((n, 3), np.uint8)
        self._check(self._L.dn_svo_get(self._h, ptr(pts, _f), ptr(nrm, _f), ptr(clr, _u8), n))
        return [pts, nrm, clr]

    def last_fuse_ms(self) -> float:
        """Device time of the last fuse (integration and extraction)."""
        ms = ctypes.c_float()
        self._check(self._L.dn_svo_last_fuse_ms(self._h, ctypes.byref(ms)))
        return float(ms.value)


class DepthmapClusterEstimator(_Handle):
    """``dense::DepthmapClusterEstimator`` (``cluster.h``, bound at
    ``python/pybind.cc:53-104``) on the B200: the live path's PatchMatch
    estimator with its pyramid levels, geometric consistency and SfM planar
    prior.  ``run()`` returns,
    per reference view, ``[depth (H,W) f32, normal (H,W,3) f32, cost (H,W)
    f32, confidence (H,W) f32]``."""

    def __init__(self) -> None:
        super().__init__("dn_acmmp_create", "dn_acmmp_destroy")

    def _check(self, st: int) -> None:
        if st == _lib.DN_OK:
            return
        msg = self._L.dn_acmmp_last_error().decode(errors="replace")
        if st == _lib.DN_INVALID_ARG:
            raise ValueError(msg)
        if st == _lib.DN_OUT_OF_MEMORY:
            raise MemoryError(msg)
        if st == _lib.DN_OUT_OF_RANGE:
            raise IndexError(msg)
        raise _lib.DenseError(st, msg)

    @staticmethod
    def is_available() -> bool:
        return GPUDepthmapCleaner.is_available()

    @staticmethod
    def num_devices() -> int:
        try:
            return int(_lib.load().dn_device_count())
        except OSError:
            return 0

    def set_max_iterations(self, n: int) -> None:
        self._check(self._L.dn_acmmp_set_max_iterations(self._h, int(n)))

    def set_patch_size(self, size: int) -> None:
        self._check(self._L.dn_acmmp_set_patch_size(self._h, int(size)))

    def set_max_image_size(self, size: int) -> None:
        self._check(self._L.dn_acmmp_set_max_image_size(self._h, int(size)))

    def set_hierarchy_levels(self, levels: int) -> None:
        self._check(self._L.dn_acmmp_set_hierarchy_levels(self._h, int(levels)))

    def set_sigma_spatial(self, v: float) -> None:
        self._check(self._L.dn_acmmp_set_sigma_spatial(self._h, float(v)))

    def set_sigma_color(self, v: float) -> None:
        self._check(self._L.dn_acmmp_set_sigma_color(self._h, float(v)))

    def set_top_k(self, k: int) -> None:
        self._check(self._L.dn_acmmp_set_top_k(self._h, int(k)))

    def set_census_weight(self, w: float) -> None:
        self._check(self._L.dn_acmmp_set_census_weight(self._h, float(w)))

    def set_smooth_weight(self, w: float) -> None:
        self._check(self._L.dn_acmmp_set_smooth_weight(self._h, float(w)))

    def set_geom_consistency_weight(self, w: float) -> None:
        self._check(self._L.dn_acmmp_set_geom_consistency_weight(self._h, float(w)))

    def set_device(self, idx: int) -> None:
        self._check(self._L.dn_acmmp_set_device(self._h, int(idx)))

    def begin_ref_view(self, K, R, t, image, depth_min: float, depth_max: float) -> int:
        K, R, t = _mat(K, (3, 3), "K"), _mat(R, (3, 3), "R"), _mat(t, (3,), "t")
        im = _image(image, "image")
        idx = ctypes.c_int()
        self._check(self._L.dn_acmmp_begin_ref_view(
            self._h, ptr(K, _d), ptr(R, _d), ptr(t, _d), ptr(im, _u8), im.shape[1], im.shape[0],
            im.shape[1], float(depth_min), float(depth_max), ctypes.byref(idx)))
        return int(idx.value)

    def add_source_view(self, K, R, t, image) -> None:
        K, R, t = _mat(K, (3, 3), "K"), _mat(R, (3, 3), "R"), _mat(t, (3,), "t")
        im = _image(image, "image")
        st = self._L.dn_acmmp_add_source_view(self._h, ptr(K, _d), ptr(R, _d), ptr(t, _d),
                                               ptr(im, _u8), im.shape[1], im.shape[0],
                                               im.shape[1])
        if st == _lib.DN_INVALID_ARG and b"no ref view" in self._L.dn_acmmp_last_error():
            raise RuntimeError(self._L.dn_acmmp_last_error().decode())
        self._check(st)

    def set_sfm_points(self, points) -> None:
        p = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        self._check(self._L.dn_acmmp_set_sfm_points(self._h, ptr(p, _d), len(p)))

    def add_geom_link(self, ref_idx: int, source_view_idx: int, from_ref_idx: int) -> None:
        st = self._L.dn_acmmp_add_geom_link(self._h, int(ref_idx), int(source_view_idx),
                                             int(from_ref_idx))
        if st == _lib.DN_INVALID_ARG:
            raise RuntimeError(self._L.dn_acmmp_last_error().decode())
        self._check(st)

    def run(self) -> list:
        st = self._L.dn_acmmp_run(self._h)
        if st == _lib.DN_INVALID_ARG and b"no reference views" in self._L.dn_acmmp_last_error():
            raise RuntimeError(self._L.dn_acmmp_last_error().decode())
        self._check(st)
        n = ctypes.c_int()
        self._check(self._L.dn_acmmp_num_refs(self._h, ctypes.byref(n)))
        out = []
        for i in range(n.value):
            w, h = ctypes.c_int(), ctypes.c_int()
            self._check(self._L.dn_acmmp_result_size(self._h, i, ctypes.byref(w),
                                                      ctypes.byref(h)))
            H, W = h.value, w.value
            d = np.zeros((H, W), np.float32)
            nrm = np.zeros((H, W, 3), np.float32)
            c = np.zeros((H, W), np.float32)
            cf = np.zeros((H, W), np.float32)
            self._check(self._L.dn_acmmp_get_result(self._h, i, ptr(d, _f), ptr(nrm, _f),
                                                     ptr(c, _f), ptr(cf, _f)))
            out.append([d, nrm, c, cf])
        return out

    def last_run_ms(self) -> float:
        """Device time of the last run's kernels (all references)."""
        ms = ctypes.c_float()
        self._check(self._L.dn_acmmp_last_run_ms(self._h, ctypes.byref(ms)))
        return float(ms.value)

    def clear(self) -> None:
        self._check(self._L.dn_acmmp_clear(self._h))


def sor_filter(points, knn: int = 12, stddev_factor: float = 2.5):
    """The fuser's statistical outlier removal (``fuser.cc:374-482``) on any
    (N, 3) points: returns (keep (N,) bool, mean distance to the knn nearest
    other points (N,) f32).  knn <= 0 or N <= knn + 1 keeps every point."""
    p = np.ascontiguousarray(points, dtype=np.float32)
    if p.ndim != 2 or p.shape[1] != 3:
        raise ValueError("points must have shape (N, 3)")
    keep = np.ones(len(p), np.uint8)
    mk = np.zeros(len(p), np.float32)
    L = _lib.load()
    st = L.dn_sor_filter(ptr(p, _f), len(p), int(knn), float(stddev_factor), ptr(keep, _u8),
                         ptr(mk, _f))
    if st != _lib.DN_OK:
        msg = L.dn_fuser_last_error().decode(errors="replace")
        if st == _lib.DN_INVALID_ARG:
            raise ValueError(msg)
        if st == _lib.DN_OUT_OF_MEMORY:
            raise MemoryError(msg)
        raise _lib.DenseError(st, msg)
    return keep.astype(bool), mk


class DepthmapPruner(_Handle):
    """``dense::DepthmapPruner`` (``depthmap.h:131-153``) on the B200."""

    def __init__(self) -> None:
        super().__init__("dn_pruner_create", "dn_pruner_destroy")
        self._shape = None

    def set_same_depth_threshold(self, t: float) -> None:
        check(self._L.dn_pruner_set_same_depth_threshold(self._h, float(t)))

    def add_view(self, K, R, t, depth, plane, color, label) -> None:
        K = _mat(K, (3, 3), "K")
        R = _mat(R, (3, 3), "R")
        t = _mat(t, (3,), "t")
        d = np.ascontiguousarray(depth, dtype=np.float32)
        if d.ndim != 2:
            raise ValueError("depth must be a 2-D array")
        H, W = d.shape
        pl = np.ascontiguousarray(plane, dtype=np.float32)
        col = np.ascontiguousarray(color, dtype=np.uint8)
        lab = np.ascontiguousarray(label, dtype=np.uint8)
        if pl.shape != (H, W, 3) or col.shape != (H, W, 3) or lab.shape != (H, W):
            raise ValueError("plane/color must be (H,W,3) and label (H,W) like depth")
        check(self._L.dn_pruner_add_view(self._h, ptr(K, _d), ptr(R, _d), ptr(t, _d), ptr(d, _f),
                                         ptr(pl, _f), ptr(col, _u8), ptr(lab, _u8), W, H))
        if self._shape is None:
            self._shape = (H, W)

    def prune(self) -> list:
        if self._shape is None:
            raise ValueError("DepthmapPruner has no views")
        n = ctypes.c_int64()
        check(self._L.dn_pruner_prune(self._h, ctypes.byref(n)))
        n = int(n.value)
        pts = np.zeros((n, 3), np.float32)
        nrm = np.zeros((n, 3), np.float32)
        col = np.zeros((n, 3), np.uint8)
        lab = np.zeros((n,), np.uint8)
        check(self._L.dn_pruner_fetch(self._h, ptr(pts, _f), ptr(nrm, _f), ptr(col, _u8),
                                      ptr(lab, _u8), n))
        return [pts, nrm, col, lab]


class Batch(_Handle):
    """Every depthmap of a reconstruction in one batched run (no reference
    counterpart; OpenSfM's dense.py runs one estimator per view).

    ``add_view`` uploads a view once; ``add_depthmap`` declares a depthmap by
    reference view, matching views and depth range; ``set_clean_views`` lists
    the depthmaps a depthmap is cleaned against; ``run`` enqueues PatchMatch
    (and the cleaner) for all of them, optionally replaying a captured CUDA
    graph.
    """

    def __init__(self) -> None:
        super().__init__("dn_batch_create", "dn_batch_destroy")
        self._shapes: List[tuple] = []
        self._map_shapes: List[tuple] = []
        self._io_keep: list = []  # host buffers of pipelined copies in flight

    def add_view(self, K, R, t, image, mask=None) -> int:
        K = _mat(K, (3, 3), "K")
        R = _mat(R, (3, 3), "R")
        t = _mat(t, (3,), "t")
        im = _image(image, "image")
        mk = _image(mask, "mask") if mask is not None else None
        H, W = im.shape
        vid = ctypes.c_int()
        check(self._L.dn_batch_add_view(self._h, ptr(K, _d), ptr(R, _d), ptr(t, _d), ptr(im, _u8),
                                        ptr(mk, _u8) if mk is not None else None, W, H, W,
                                        ctypes.byref(vid)))
        self._shapes.append((H, W))
        return vid.value

    def add_depthmap(self, ref: int, matching: Sequence[int], min_depth: float,
                     max_depth: float) -> int:
        nb = np.ascontiguousarray(matching, dtype=np.int32)
        mid = ctypes.c_int()
        check(self._L.dn_batch_add_depthmap(self._h, int(ref), ptr(nb, _i32), len(nb),
                                            float(min_depth), float(max_depth), ctypes.byref(mid)))
        self._map_shapes.append(self._shapes[ref])
        return mid.value

    def set_clean_views(self, map_id: int, others: Sequence[int]) -> None:
        o = np.ascontiguousarray(others, dtype=np.int32)
        check(self._L.dn_batch_set_clean_views(self._h, int(map_id), ptr(o, _i32), len(o)))

    def set_params(self, patch_size=7, min_patch_sd=1.0, iterations=3, same_depth_threshold=0.01,
                   min_consistent_views=3, seed=1) -> None:
        check(self._L.dn_batch_set_params(self._h, int(patch_size), float(min_patch_sd),
                                          int(iterations), float(same_depth_threshold),
                                          int(min_consistent_views), int(seed)))

    def set_schedule(self, half_passes: int = -1, use_near: bool = True, use_far: bool = True,
                     n_refine: int = 6, depth_range0: float = 0.02,
                     normal_range0: float = 0.5) -> None:
        """PatchMatch half-passes and candidate sets (defaults: the reference's schedule)."""
        check(self._L.dn_batch_set_schedule(self._h, int(half_passes), int(bool(use_near)),
                                            int(bool(use_far)), int(n_refine), float(depth_range0),
                                            float(normal_range0)))

    def set_candidate_views(self, mode) -> None:
        """0 / False: every matching view per candidate (ComputePatchMatch);
        1 / True: full initialisation, then one view per candidate plus one
        random other view per update in the half-passes; 2: the reference's
        ComputePatchMatchSample (a random view at the initialisation too)."""
        check(self._L.dn_batch_set_candidate_views(self._h, int(mode)))

    def set_knight_moves(self, on: bool) -> None:
        """Also try the planes of the 8 knight-move pixels in every update."""
        check(self._L.dn_batch_set_knight_moves(self._h, int(bool(on))))

    def set_active_pixels(self, on: bool, min_change: float = 0.0) -> None:
        """From the third half-pass on, update only pixels whose own depth or a
        neighbour's depth moved at their last update (by more than
        ``min_change`` relative; 0: any change of the plane)."""
        check(self._L.dn_batch_set_active_pixels(self._h, int(bool(on)), float(min_change)))

    def set_init_fallback(self, on: bool) -> None:
        """Given planes (learned proposals) compete with the reference's random
        initialisation per pixel: the higher score on the same view(s) wins."""
        check(self._L.dn_batch_set_init_fallback(self._h, int(bool(on))))

    def set_active_seed(self, min_score: float) -> None:
        """Settled start: pixels whose initial score is at least ``min_score``
        start as settled and the active rule applies from the first
        half-pass; 0 (default): every pixel starts as moved."""
        check(self._L.dn_batch_set_active_seed(self._h, float(min_score)))

    def set_active_lists(self, on: bool) -> None:
        """Active half-passes over compacted lists of the active pixels (the
        default) or over every tile that holds one; the maps are the same."""
        check(self._L.dn_batch_set_active_lists(self._h, int(bool(on))))

    def set_proposal_net(self, weights: Optional[np.ndarray], biases: Optional[np.ndarray] = None,
                         n_planes: int = 8, stride: int = 2) -> None:
        """The network of learned runs (``run(learned=True)``): ``weights`` the
        BF16 bit patterns (uint16) of the 6 layers' [cout][288] matrices one
        after the other, ``biases`` their FP32 biases; None removes it."""
        if weights is None:
            check(self._L.dn_batch_set_proposal_net(self._h, None, None, 0, 0))
            return
        w = np.ascontiguousarray(weights, dtype=np.uint16)
        b = np.ascontiguousarray(biases, dtype=np.float32)
        if w.size != 5 * 32 * 288 + 4 * 288 or b.size != 5 * 32 + 4:
            raise ValueError("weights must hold 46080 BF16 values and biases 164 floats")
        check(self._L.dn_batch_set_proposal_net(
            self._h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), ptr(b, _f), int(n_planes),
            int(stride)))

    def set_proposal_scale(self, ref_dim: int) -> None:
        """The larger side of the network's training images: each map's
        proposal grid then uses the stride scaled by its own larger side over
        ``ref_dim`` (rounded down to 1, 2, 4 or 8); 0: one stride for all."""
        check(self._L.dn_batch_set_proposal_scale(self._h, int(ref_dim)))

    def set_init(self, map_id: int, planes: Optional[np.ndarray]) -> None:
        if planes is None:
            check(self._L.dn_batch_set_init(self._h, int(map_id), None))
            return
        pl = np.ascontiguousarray(planes, dtype=np.float32)
        if pl.shape != self._map_shapes[map_id] + (3,):
            raise ValueError("init planes must be (H, W, 3)")
        check(self._L.dn_batch_set_init(self._h, int(map_id), ptr(pl, _f)))

    def run(self, clean: bool = False, graph: bool = False, timing: bool = False,
            prune: bool = False, learned: bool = False) -> None:
        flags = ((_lib.DN_RUN_CLEAN if clean or prune else 0) | (_lib.DN_RUN_GRAPH if graph else 0) |
                 (_lib.DN_RUN_TIMING if timing else 0) | (_lib.DN_RUN_PRUNE if prune else 0) |
                 (_lib.DN_RUN_LEARNED if learned else 0))
        check(self._L.dn_batch_run(self._h, flags))

    def pruned_count(self) -> int:
        n = ctypes.c_int64()
        check(self._L.dn_batch_pruned_count(self._h, ctypes.byref(n)))
        return int(n.value)

    def get_points(self, map_id: int) -> list:
        """[points (N,3), normals (N,3), colors (N,3) u8, labels (N,) u8] of one map."""
        n = ctypes.c_int64()
        check(self._L.dn_batch_get_points(self._h, int(map_id), None, None, None, None, 0,
                                          ctypes.byref(n)))
        k = int(n.value)
        pts = np.zeros((k, 3), np.float32)
        nrm = np.zeros((k, 3), np.float32)
        col = np.zeros((k, 3), np.uint8)
        lab = np.zeros((k,), np.uint8)
        check(self._L.dn_batch_get_points(self._h, int(map_id), ptr(pts, _f), ptr(nrm, _f),
                                          ptr(col, _u8), ptr(lab, _u8), k, ctypes.byref(n)))
        return [pts, nrm, col, lab]

    def set_view_image(self, view_id: int, image: np.ndarray) -> None:
        """Asynchronous re-upload of a view's pixels; keep ``image`` alive until synchronize."""
        im = np.ascontiguousarray(image, dtype=np.uint8)
        H, W = self._shapes[view_id]
        if im.shape != (H, W):
            raise ValueError("image must keep the view's size")
        check(self._L.dn_batch_set_view_image(self._h, int(view_id), ptr(im, _u8), W))

    def upload_view_image(self, view_id: int, image: np.ndarray) -> None:
        """Pipelined re-upload of a view's pixels for the runs enqueued after
        it: the host copy runs beside a run already enqueued.  ``image``
        (pinned for the overlap) is kept referenced, and must stay unmodified,
        until ``synchronize``."""
        H, W = self._shapes[view_id]
        if image.dtype != np.uint8 or not image.flags.c_contiguous or image.shape != (H, W):
            raise ValueError("image must be a C-contiguous uint8 array of the view's size")
        check(self._L.dn_batch_upload_view_image(self._h, int(view_id), ptr(image, _u8), W))
        self._io_keep.append(image)

    def set_tuning(self, bx: int = 32, by: int = 4, variant: int = 2) -> None:
        check(self._L.dn_batch_set_tuning(self._h, int(bx), int(by), int(variant)))

    def timer_record(self, slot: int) -> None:
        check(self._L.dn_batch_timer_record(self._h, int(slot)))

    def timer_elapsed(self) -> float:
        ms = ctypes.c_float()
        check(self._L.dn_batch_timer_elapsed(self._h, ctypes.byref(ms)))
        return float(ms.value)

    def timings(self):
        """(per-stage ms [init, half-passes, post, clean and prune, total, learned
        proposal], [init taps, half-pass taps])."""
        t = np.zeros(6, np.float32)
        taps = (ctypes.c_uint64 * 2)()
        check(self._L.dn_batch_last_timings(self._h, ptr(t, _f), 6, taps))
        return t.astype(float).tolist(), [int(taps[0]), int(taps[1])]

    def synchronize(self) -> None:
        check(self._L.dn_batch_synchronize(self._h))
        self._io_keep = []

    def get(self, map_id: int, clean: bool = False) -> list:
        H, W = self._map_shapes[map_id]
        depth = np.zeros((H, W), np.float32)
        plane = np.zeros((H, W, 3), np.float32)
        score = np.zeros((H, W), np.float32)
        nghbr = np.zeros((H, W), np.int32)
        cl = np.zeros((H, W), np.float32) if clean else None
        check(self._L.dn_batch_get_depthmap(self._h, int(map_id), ptr(depth, _f), ptr(plane, _f),
                                            ptr(score, _f), ptr(nghbr, _i32),
                                            ptr(cl, _f) if clean else None))
        out = [depth, plane, score, nghbr]
        if clean:
            out.append(cl)
        return out

    def get_depth(self, map_id: int, clean: bool = False) -> np.ndarray:
        H, W = self._map_shapes[map_id]
        out = np.zeros((H, W), np.float32)
        if clean:
            check(self._L.dn_batch_get_depthmap(self._h, int(map_id), None, None, None, None,
                                                ptr(out, _f)))
        else:
            check(self._L.dn_batch_get_depthmap(self._h, int(map_id), ptr(out, _f), None, None,
                                                None, None))
        return out

    def get_depths(self, map_ids, outs=None, clean: bool = False):
        """Final (or cleaned) depths of several maps with one synchronisation.
        ``outs`` (optional) are C-contiguous float32 (H, W) host arrays, pinned
        ones copy asynchronously."""
        ids = [int(m) for m in map_ids]
        if outs is None:
            outs = [np.zeros(self._map_shapes[m], np.float32) for m in ids]
        for m, o in zip(ids, outs):
            if o.dtype != np.float32 or not o.flags.c_contiguous or o.shape != self._map_shapes[m]:
                raise ValueError("outputs must be C-contiguous float32 arrays of the map's shape")
        id_arr = (ctypes.c_int32 * len(ids))(*ids)
        ptr_arr = (ctypes.c_void_p * len(ids))(*[o.ctypes.data for o in outs])
        check(self._L.dn_batch_get_depths(self._h, len(ids), id_arr,
                                          ctypes.cast(ptr_arr, ctypes.c_void_p), int(bool(clean))))
        return outs

    def get_depths_async(self, map_ids, outs, clean: bool = False):
        """Pipelined readback of the final (or cleaned) depths as the runs
        enqueued before it leave them, into C-contiguous float32 (H, W) host
        arrays ``outs`` (pinned for the overlap); complete after
        ``synchronize``, which also releases the kept references."""
        ids = [int(m) for m in map_ids]
        if len(outs) != len(ids):
            raise ValueError("one output per map")
        for m, o in zip(ids, outs):
            if not 0 <= m < len(self._map_shapes):
                raise IndexError(f"depthmap id {m} out of range")
            if o.dtype != np.float32 or not o.flags.c_contiguous or o.shape != self._map_shapes[m]:
                raise ValueError("outputs must be C-contiguous float32 arrays of the map's shape")
        id_arr = (ctypes.c_int32 * len(ids))(*ids)
        ptr_arr = (ctypes.c_void_p * len(ids))(*[o.ctypes.data for o in outs])
        check(self._L.dn_batch_get_depths_async(self._h, len(ids), id_arr,
                                                ctypes.cast(ptr_arr, ctypes.c_void_p),
                                                int(bool(clean))))
        self._io_keep.append(list(outs))
        return outs

    def last_taps(self) -> int:
        v = ctypes.c_uint64()
        check(self._L.dn_batch_last_taps(self._h, ctypes.byref(v)))
        return int(v.value)
