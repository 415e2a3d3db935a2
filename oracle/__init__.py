"""CPU oracles for the dense depthmap path.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference legs import this package, and only as the checker or as the
timed CPU baseline.  The product (``opensfm_b200``) never imports it.

The oracles:

``port``
    ``depthmap_oracle.c``: this project's plain-C restatement of the
    reference's legacy path (``opensfm/src/lib/dense/src/depthmap.cc``):
    brute force, PatchMatch (raster schedule, seeded RNG), plane scoring,
    median post-process, cleaner, pruner.  The same library holds the C
    restatements of the steps either side of it: ``fuser_oracle.c``
    (``port_fuse``, ``port_sor``), ``svo_oracle.c`` (``port_svo``) and
    ``acmmp_oracle.c`` (``port_acmmp``, ``port_acmmp_cluster``); and
    ``gpu_clean_fp32`` restates the GPU cleaner's kernel in numpy.
``ref``
    The reference's own ``depthmap.cc`` compiled unmodified against the
    project's OpenCV shim (``oracle/Makefile`` -> ``oracle/_ref/``), driven
    through ``ref_capi.cc``.  Present wherever the reference's sources were
    available when ``make`` ran; ``ref_available()`` says whether it is.
``ncc_fp64``
    A numpy float64 restatement of ``ComputePlaneImageScore``
    (``depthmap.cc:441-487``), the yardstick for NCC error.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libdepthmap_ref.so")
# The reference checkout: $OPENSFM_REFERENCE, else a "reference" folder beside
# this repository.
REF_ROOT = os.environ.get("OPENSFM_REFERENCE",
                          os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
REF_DENSE = os.path.join(REF_ROOT, "opensfm", "src", "lib", "dense")

_port = None
_ref = None

_d = ctypes.POINTER(ctypes.c_double)
_f = ctypes.POINTER(ctypes.c_float)
_u8 = ctypes.POINTER(ctypes.c_uint8)
_i32 = ctypes.POINTER(ctypes.c_int32)


def build(with_ref: bool = True) -> None:
    """Builds the C restatement, and the compiled reference if its sources exist."""
    subprocess.check_call(["make", "-s", "-C", HERE, os.path.join(HERE, "_build", "liboracle.so")])
    if with_ref and os.path.isdir(REF_DENSE):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF_DENSE={REF_DENSE}"])


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def _P(a, t):
    return a.ctypes.data_as(t)


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_LIB):
            build(with_ref=False)
        L = ctypes.CDLL(PORT_LIB)
        L.or_compute.argtypes = [ctypes.c_int, ctypes.c_int, _d, _d, _d, _u8, _u8, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint64,
                                 _f, _f, _f, _i32]
        L.or_compute_redblack.argtypes = [ctypes.c_int, ctypes.c_int, _d, _d, _d, _u8, _u8,
                                          ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_float,
                                          ctypes.c_uint64, _f, _f, _f, _i32]
        L.or_score_planes.argtypes = [ctypes.c_int, _d, _d, _d, _u8, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, _f, _f, _i32]
        L.or_median5.argtypes = [_f, _f, ctypes.c_int, ctypes.c_int]
        L.or_clean.argtypes = [ctypes.c_int, _d, _d, _d, _f, ctypes.c_int, ctypes.c_int,
                               ctypes.c_float, ctypes.c_int, _f]
        L.or_prune.argtypes = [ctypes.c_int, _d, _d, _d, _f, _f, _u8, _u8, ctypes.c_int,
                               ctypes.c_int, ctypes.c_float, _f, _f, _u8, _u8, ctypes.c_long]
        L.or_prune.restype = ctypes.c_long
        L.or_inv3.argtypes = [_d, _d]
        L.or_patch_variance.argtypes = [_u8, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int]
        L.or_patch_variance.restype = ctypes.c_float
        _port = L
    return _port


def ref():
    global _ref
    if _ref is None:
        if not ref_available():
            raise FileNotFoundError("compiled reference oracle not built: " + REF_LIB)
        L = ctypes.CDLL(REF_LIB)
        L.ref_est_new.restype = ctypes.c_void_p
        L.ref_est_free.argtypes = [ctypes.c_void_p]
        L.ref_est_add_view.argtypes = [ctypes.c_void_p, _d, _d, _d, _u8, _u8, ctypes.c_int,
                                       ctypes.c_int]
        L.ref_est_set_depth_range.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_int]
        L.ref_est_set_patchmatch_iterations.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_est_set_patch_size.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_est_set_min_patch_sd.argtypes = [ctypes.c_void_p, ctypes.c_float]
        L.ref_est_compute.argtypes = [ctypes.c_void_p, ctypes.c_int, _f, _f, _f, _i32]
        L.ref_est_score_planes.argtypes = [ctypes.c_void_p, _f, _f, _i32]
        L.ref_est_plane_image_score.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _f,
                                                ctypes.c_int]
        L.ref_est_plane_image_score.restype = ctypes.c_float
        L.ref_patch_variance.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.ref_patch_variance.restype = ctypes.c_float
        L.ref_median5.argtypes = [_f, _f, ctypes.c_int, ctypes.c_int]
        L.ref_inv3.argtypes = [_d, _d]
        L.ref_srand.argtypes = [ctypes.c_uint]
        L.ref_cleaner_new.restype = ctypes.c_void_p
        L.ref_cleaner_free.argtypes = [ctypes.c_void_p]
        L.ref_cleaner_set_same_depth_threshold.argtypes = [ctypes.c_void_p, ctypes.c_float]
        L.ref_cleaner_set_min_consistent_views.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_cleaner_add_view.argtypes = [ctypes.c_void_p, _d, _d, _d, _f, ctypes.c_int,
                                           ctypes.c_int]
        L.ref_cleaner_clean.argtypes = [ctypes.c_void_p, _f, ctypes.c_int, ctypes.c_int]
        L.ref_pruner_new.restype = ctypes.c_void_p
        L.ref_pruner_free.argtypes = [ctypes.c_void_p]
        L.ref_pruner_set_same_depth_threshold.argtypes = [ctypes.c_void_p, ctypes.c_float]
        L.ref_pruner_add_view.argtypes = [ctypes.c_void_p, _d, _d, _d, _f, _f, _u8, _u8,
                                          ctypes.c_int, ctypes.c_int]
        L.ref_pruner_prune.argtypes = [ctypes.c_void_p]
        L.ref_pruner_prune.restype = ctypes.c_long
        L.ref_pruner_fetch.argtypes = [ctypes.c_void_p, _f, _f, _u8, _u8]
        _ref = L
    return _ref


# --------------------------------------------------------------------------
# Views: every oracle entry takes lists of K, R, t (float64) and images.

def _stack_cams(Ks, Rs, ts):
    K = np.ascontiguousarray(np.stack([np.asarray(k, np.float64).reshape(9) for k in Ks]))
    R = np.ascontiguousarray(np.stack([np.asarray(r, np.float64).reshape(9) for r in Rs]))
    t = np.ascontiguousarray(np.stack([np.asarray(x, np.float64).reshape(3) for x in ts]))
    return K, R, t


def port_compute(mode: int, Ks, Rs, ts, images, masks, patch_size=7, min_depth=1.0,
                 max_depth=10.0, num_planes=50, iterations=3, min_patch_sd=1.0, seed=1):
    """mode 0 brute force, 1 PatchMatch, 2 PatchMatch (sample)."""
    K, R, t = _stack_cams(Ks, Rs, ts)
    im = np.ascontiguousarray(np.stack(images).astype(np.uint8))
    mk = np.ascontiguousarray(np.stack(masks).astype(np.uint8))
    n, H, W = im.shape
    depth = np.zeros((H, W), np.float32)
    plane = np.zeros((H, W, 3), np.float32)
    score = np.zeros((H, W), np.float32)
    nghbr = np.zeros((H, W), np.int32)
    port().or_compute(mode, n, _P(K, _d), _P(R, _d), _P(t, _d), _P(im, _u8), _P(mk, _u8), W, H,
                      patch_size, min_depth, max_depth, num_planes, iterations, min_patch_sd,
                      seed, _P(depth, _f), _P(plane, _f), _P(score, _f), _P(nghbr, _i32))
    return depth, plane, score, nghbr


def port_compute_redblack(Ks, Rs, ts, images, masks, patch_size=7, min_depth=1.0,
                          max_depth=10.0, half_passes=6, min_patch_sd=1.0, seed=1, sample=False):
    """The GPU's red-black PatchMatch schedule with the reference's arithmetic
    (or_compute_redblack in depthmap_oracle.c), or its sample mode:
    [depth, plane, score, nghbr]."""
    K, R, t = _stack_cams(Ks, Rs, ts)
    im = np.ascontiguousarray(np.stack(images).astype(np.uint8))
    mk = np.ascontiguousarray(np.stack(masks).astype(np.uint8))
    n, H, W = im.shape
    depth = np.zeros((H, W), np.float32)
    plane = np.zeros((H, W, 3), np.float32)
    score = np.zeros((H, W), np.float32)
    nghbr = np.zeros((H, W), np.int32)
    port().or_compute_redblack(int(bool(sample)), n, _P(K, _d), _P(R, _d), _P(t, _d), _P(im, _u8),
                               _P(mk, _u8), W, H,
                               patch_size, min_depth, max_depth, half_passes, min_patch_sd, seed,
                               _P(depth, _f), _P(plane, _f), _P(score, _f), _P(nghbr, _i32))
    return depth, plane, score, nghbr


def port_score_planes(Ks, Rs, ts, images, planes, patch_size=7):
    K, R, t = _stack_cams(Ks, Rs, ts)
    im = np.ascontiguousarray(np.stack(images).astype(np.uint8))
    n, H, W = im.shape
    pl = np.ascontiguousarray(planes, np.float32)
    score = np.zeros((H, W), np.float32)
    nghbr = np.zeros((H, W), np.int32)
    port().or_score_planes(n, _P(K, _d), _P(R, _d), _P(t, _d), _P(im, _u8), W, H, patch_size,
                           _P(pl, _f), _P(score, _f), _P(nghbr, _i32))
    return score, nghbr


def port_median5(depth):
    d = np.ascontiguousarray(depth, np.float32)
    out = np.empty_like(d)
    port().or_median5(_P(d, _f), _P(out, _f), d.shape[1], d.shape[0])
    return out


def port_clean(Ks, Rs, ts, depths, threshold=0.01, min_views=2):
    K, R, t = _stack_cams(Ks, Rs, ts)
    d = np.ascontiguousarray(np.stack(depths).astype(np.float32))
    n, H, W = d.shape
    out = np.zeros((H, W), np.float32)
    port().or_clean(n, _P(K, _d), _P(R, _d), _P(t, _d), _P(d, _f), W, H, threshold, min_views,
                    _P(out, _f))
    return out


def port_prune(Ks, Rs, ts, depths, planes, colors, labels, threshold=0.01):
    K, R, t = _stack_cams(Ks, Rs, ts)
    d = np.ascontiguousarray(np.stack(depths).astype(np.float32))
    p = np.ascontiguousarray(np.stack(planes).astype(np.float32))
    c = np.ascontiguousarray(np.stack(colors).astype(np.uint8))
    lb = np.ascontiguousarray(np.stack(labels).astype(np.uint8))
    n, H, W = d.shape
    cap = H * W
    pts = np.zeros((cap, 3), np.float32)
    nrm = np.zeros((cap, 3), np.float32)
    col = np.zeros((cap, 3), np.uint8)
    lab = np.zeros((cap,), np.uint8)
    cnt = port().or_prune(n, _P(K, _d), _P(R, _d), _P(t, _d), _P(d, _f), _P(p, _f), _P(c, _u8),
                          _P(lb, _u8), W, H, threshold, _P(pts, _f), _P(nrm, _f), _P(col, _u8),
                          _P(lab, _u8), cap)
    return pts[:cnt].copy(), nrm[:cnt].copy(), col[:cnt].copy(), lab[:cnt].copy()


# --------------------------------------------------------------------------
# The compiled reference, through the same argument conventions.

class RefEstimator:
    """The reference's dense::DepthmapEstimator (compiled), pydense-style."""

    def __init__(self):
        self.L = ref()
        self.h = self.L.ref_est_new()
        self.shape = None
        self._keep = []

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_est_free(self.h)
            self.h = None

    def add_view(self, K, R, t, image, mask):
        K = np.ascontiguousarray(K, np.float64)
        R = np.ascontiguousarray(R, np.float64)
        t = np.ascontiguousarray(t, np.float64)
        im = np.ascontiguousarray(image, np.uint8)
        mk = np.ascontiguousarray(mask, np.uint8)
        self._keep += [K, R, t]
        if self.shape is None:
            self.shape = im.shape
        self.L.ref_est_add_view(self.h, _P(K, _d), _P(R, _d), _P(t, _d), _P(im, _u8),
                                _P(mk, _u8), im.shape[1], im.shape[0])

    def set_depth_range(self, mn, mx, n):
        self.L.ref_est_set_depth_range(self.h, mn, mx, n)

    def set_patchmatch_iterations(self, n):
        self.L.ref_est_set_patchmatch_iterations(self.h, n)

    def set_patch_size(self, n):
        self.L.ref_est_set_patch_size(self.h, n)

    def set_min_patch_sd(self, sd):
        self.L.ref_est_set_min_patch_sd(self.h, sd)

    def _compute(self, mode):
        H, W = self.shape
        depth = np.zeros((H, W), np.float32)
        plane = np.zeros((H, W, 3), np.float32)
        score = np.zeros((H, W), np.float32)
        nghbr = np.zeros((H, W), np.int32)
        self.L.ref_est_compute(self.h, mode, _P(depth, _f), _P(plane, _f), _P(score, _f),
                               _P(nghbr, _i32))
        return [depth, plane, score, nghbr]

    def compute_brute_force(self):
        return self._compute(0)

    def compute_patch_match(self):
        return self._compute(1)

    def compute_patch_match_sample(self):
        return self._compute(2)

    def score_planes(self, planes):
        H, W = self.shape
        pl = np.ascontiguousarray(planes, np.float32)
        score = np.zeros((H, W), np.float32)
        nghbr = np.zeros((H, W), np.int32)
        self.L.ref_est_score_planes(self.h, _P(pl, _f), _P(score, _f), _P(nghbr, _i32))
        return score, nghbr


def ref_clean(Ks, Rs, ts, depths, threshold=0.01, min_views=2):
    L = ref()
    h = L.ref_cleaner_new()
    keep = []
    try:
        L.ref_cleaner_set_same_depth_threshold(h, threshold)
        L.ref_cleaner_set_min_consistent_views(h, min_views)
        for K, R, t, d in zip(Ks, Rs, ts, depths):
            K = np.ascontiguousarray(K, np.float64)
            R = np.ascontiguousarray(R, np.float64)
            t = np.ascontiguousarray(t, np.float64)
            d = np.ascontiguousarray(d, np.float32)
            keep += [K, R, t, d]
            L.ref_cleaner_add_view(h, _P(K, _d), _P(R, _d), _P(t, _d), _P(d, _f), d.shape[1],
                                   d.shape[0])
        H, W = depths[0].shape
        out = np.zeros((H, W), np.float32)
        L.ref_cleaner_clean(h, _P(out, _f), W, H)
        return out
    finally:
        L.ref_cleaner_free(h)


def ref_prune(Ks, Rs, ts, depths, planes, colors, labels, threshold=0.01):
    L = ref()
    h = L.ref_pruner_new()
    keep = []
    try:
        L.ref_pruner_set_same_depth_threshold(h, threshold)
        for K, R, t, d, p, c, lb in zip(Ks, Rs, ts, depths, planes, colors, labels):
            arrs = [np.ascontiguousarray(K, np.float64), np.ascontiguousarray(R, np.float64),
                    np.ascontiguousarray(t, np.float64), np.ascontiguousarray(d, np.float32),
                    np.ascontiguousarray(p, np.float32), np.ascontiguousarray(c, np.uint8),
                    np.ascontiguousarray(lb, np.uint8)]
            keep += arrs
            L.ref_pruner_add_view(h, _P(arrs[0], _d), _P(arrs[1], _d), _P(arrs[2], _d),
                                  _P(arrs[3], _f), _P(arrs[4], _f), _P(arrs[5], _u8),
                                  _P(arrs[6], _u8), d.shape[1], d.shape[0])
        n = L.ref_pruner_prune(h)
        pts = np.zeros((n, 3), np.float32)
        nrm = np.zeros((n, 3), np.float32)
        col = np.zeros((n, 3), np.uint8)
        lab = np.zeros((n,), np.uint8)
        if n:
            L.ref_pruner_fetch(h, _P(pts, _f), _P(nrm, _f), _P(col, _u8), _P(lab, _u8))
        return pts, nrm, col, lab
    finally:
        L.ref_pruner_free(h)


def ref_median5(depth):
    d = np.ascontiguousarray(depth, np.float32)
    out = np.empty_like(d)
    ref().ref_median5(_P(d, _f), _P(out, _f), d.shape[1], d.shape[0])
    return out


# --------------------------------------------------------------------------
# float64 NCC restatement (depthmap.cc:441-487), vectorised over pixels.

def ncc_fp64(Ks, Rs, ts, images, planes, patch_size=7, pixels=None, margins=False):
    """Per-pixel max-over-views NCC in float64 for the given planes.

    Returns (score (H, W) float64, nghbr (H, W) int32); the homography, the
    affine warp, bilinear sampling, bilateral weights and the moments are all
    float64.  ``pixels``: optional boolean mask restricting the work.

    With ``margins=True`` also returns, per pixel, the distances to the
    reference's two discontinuities, minimised over views and taps: ``edge``,
    how close a tap lands to x = 0, x = W-1, y = 0 or y = H-1 (where
    LinearInterpolation switches to 0, depthmap.cc:16-18), and ``var``, how
    close var_x or var_y is to the 0.1 cut-off (depthmap.cc:68).  Float
    implementations legitimately disagree on pixels with tiny margins.
    """
    K = [np.asarray(k, np.float64) for k in Ks]
    R = [np.asarray(r, np.float64) for r in Rs]
    t = [np.asarray(x, np.float64).reshape(3) for x in ts]
    imgs = [np.asarray(im, np.float64) for im in images]
    H, W = imgs[0].shape
    hpz = (patch_size - 1) // 2
    ii, jj = np.mgrid[0:H, 0:W]
    interior = (ii >= hpz) & (ii < H - hpz) & (jj >= hpz) & (jj < W - hpz)
    if pixels is not None:
        interior &= pixels
    pi, pj = ii[interior].astype(np.float64), jj[interior].astype(np.float64)
    v = np.asarray(planes, np.float64)[interior]  # (P, 3)
    K1inv = np.linalg.inv(K[0])
    best = np.full(pi.shape, -1.0)
    bestn = np.zeros(pi.shape, np.int32)
    edge_m = np.full(pi.shape, np.inf)
    var_m = np.full(pi.shape, np.inf)
    ref = imgs[0]
    c = ref[pi.astype(int), pj.astype(int)]
    for o in range(1, len(imgs)):
        Q = R[o] @ R[0].T
        a = Q @ t[0] - t[o]
        # H = K2 (Q + a v^T) K1inv, per pixel.
        M = Q[None] + a[None, :, None] * v[:, None, :]
        Hm = K[o][None] @ M @ K1inv[None]
        u = Hm[:, 0, 0] * pj + Hm[:, 0, 1] * pi + Hm[:, 0, 2]
        vv = Hm[:, 1, 0] * pj + Hm[:, 1, 1] * pi + Hm[:, 1, 2]
        w = Hm[:, 2, 0] * pj + Hm[:, 2, 1] * pi + Hm[:, 2, 2]
        ok = w != 0
        w = np.where(ok, w, 1.0)
        dxx = (Hm[:, 0, 0] * w - Hm[:, 2, 0] * u) / (w * w)
        dxy = (Hm[:, 1, 0] * w - Hm[:, 2, 0] * vv) / (w * w)
        dyx = (Hm[:, 0, 1] * w - Hm[:, 2, 1] * u) / (w * w)
        dyy = (Hm[:, 1, 1] * w - Hm[:, 2, 1] * vv) / (w * w)
        x0, y0 = u / w, vv / w
        sx = sy = sxx = syy = sxy = sw = 0.0
        img = imgs[o]
        Ho, Wo = img.shape  # each view is sampled with its own size (depthmap.cc:16)
        for dy in range(-hpz, hpz + 1):
            for dx in range(-hpz, hpz + 1):
                x1 = ref[pi.astype(int) + dy, pj.astype(int) + dx]
                x2 = x0 + dxx * dx + dyx * dy
                y2 = y0 + dxy * dx + dyy * dy
                inside = (x2 >= 0) & (x2 < Wo - 1) & (y2 >= 0) & (y2 < Ho - 1)
                if margins:
                    e = np.minimum(np.minimum(np.abs(x2), np.abs(x2 - (Wo - 1))),
                                   np.minimum(np.abs(y2), np.abs(y2 - (Ho - 1))))
                    edge_m = np.minimum(edge_m, np.where(ok, e, np.inf))
                xs = np.where(inside, x2, 0.0)
                ys = np.where(inside, y2, 0.0)
                ix, iy = np.floor(xs).astype(int), np.floor(ys).astype(int)
                fx, fy = xs - ix, ys - iy
                s = ((1 - fy) * ((1 - fx) * img[iy, ix] + fx * img[iy, ix + 1]) +
                     fy * ((1 - fx) * img[iy + 1, ix] + fx * img[iy + 1, ix + 1]))
                y = np.where(inside, s, 0.0)
                wt = np.exp(-(x1 - c) ** 2 / (2 * 50.0 ** 2) - (dx * dx + dy * dy) / (2 * 25.0))
                sx = sx + wt * x1
                sy = sy + wt * y
                sxx = sxx + wt * x1 * x1
                syy = syy + wt * y * y
                sxy = sxy + wt * x1 * y
                sw = sw + wt
        mx, my = sx / sw, sy / sw
        vx = sxx / sw - mx * mx
        vy = syy / sw - my * my
        ncc = np.where((vx < 0.1) | (vy < 0.1) | ~ok, -1.0,
                       (sxy / sw - mx * my) / np.sqrt(np.maximum(vx * vy, 1e-300)))
        if margins:
            var_m = np.minimum(var_m, np.minimum(np.abs(vx - 0.1), np.abs(vy - 0.1)))
        upd = ncc > best
        best = np.where(upd, ncc, best)
        bestn = np.where(upd, o, bestn)
    score = np.zeros((H, W))
    nghbr = np.zeros((H, W), np.int32)
    score[interior] = best
    nghbr[interior] = bestn
    if margins:
        em = np.full((H, W), np.inf)
        vm = np.full((H, W), np.inf)
        em[interior] = edge_m
        vm[interior] = var_m
        return score, nghbr, em, vm
    return score, nghbr

def gpu_clean_fp32(Ks, Rs, ts, depths, ref, neighbor_ids, same_depth_threshold=0.01,
                   min_consistent_views=3, carving_threshold=0.2, max_carved_views=1):
    """GPUDepthmapCleaner::Clean restated in numpy FP32 (kernel
    acmmp_clean_depthmap, opencl_kernels.h:2155-2273; host cleaner.cc:56-170).

    Every operation is an FP32 operation in the kernel's order, rounded by
    itself; the source depth is sampled bilinearly with exact fractions.
    Sources must have the reference's size.  This restates the OpenCL
    kernel source: the reference cannot run it here (no OpenCL).
    """
    f32 = np.float32
    K = [np.asarray(k, np.float64).astype(f32).ravel() for k in Ks]
    R = [np.asarray(r, np.float64).astype(f32).ravel() for r in Rs]
    t = [np.asarray(x, np.float64).astype(f32).ravel() for x in ts]
    D = [np.asarray(d, f32) for d in depths]
    H, W = D[ref].shape
    ids = list(neighbor_ids)[:16]
    carving = f32(max(0.0, carving_threshold))
    max_carved = max(0, int(max_carved_views))
    eff_min = min(int(min_consistent_views), 1 + len(list(neighbor_ids)))
    thr = f32(same_depth_threshold)
    yy, xx = np.mgrid[0:H, 0:W]
    xf, yf = xx.astype(f32), yy.astype(f32)
    d = D[ref]
    valid = d > f32(0)

    def rot_t(Rm, x, y, z):
        return ((Rm[0] * x + Rm[3] * y) + Rm[6] * z, (Rm[1] * x + Rm[4] * y) + Rm[7] * z,
                (Rm[2] * x + Rm[5] * y) + Rm[8] * z)

    def rot_add(Rm, tv, p):
        x, y, z = p
        return (((Rm[0] * x + Rm[1] * y) + Rm[2] * z) + tv[0],
                ((Rm[3] * x + Rm[4] * y) + Rm[5] * z) + tv[1],
                ((Rm[6] * x + Rm[7] * y) + Rm[8] * z) + tv[2])

    def backproject(Kv, Rv, tv, u, v, dd):
        cx = (u - Kv[2]) / Kv[0] * dd
        cy = (v - Kv[5]) / Kv[4] * dd
        return rot_t(Rv, cx - tv[0], cy - tv[1], dd - tv[2])

    with np.errstate(all="ignore"):
        w = backproject(K[ref], R[ref], t[ref], xf, yf, d)
        consistent = np.ones((H, W), np.int32)
        carved = np.zeros((H, W), np.int32)
        for o in ids:
            sx, sy, sz = rot_add(R[o], t[o], w)
            ok = valid & (sz > f32(1e-6))
            su = (K[o][0] * sx) / sz + K[o][2]
            sv = (K[o][4] * sy) / sz + K[o][5]
            ok &= ~((su < f32(0)) | (sv < f32(0)) | (su >= f32(W - 1)) | (sv >= f32(H - 1)))
            ix = np.where(ok, su, f32(0)).astype(np.int64)
            iy = np.where(ok, sv, f32(0)).astype(np.int64)
            fx = np.where(ok, su, f32(0)) - ix.astype(f32)
            fy = np.where(ok, sv, f32(0)) - iy.astype(f32)
            gx, gy = f32(1) - fx, f32(1) - fy
            src = D[o]
            ix1, iy1 = np.minimum(ix + 1, W - 1), np.minimum(iy + 1, H - 1)
            top = gx * src[iy, ix] + fx * src[iy, ix1]
            bot = gx * src[iy1, ix] + fx * src[iy1, ix1]
            sd = gy * top + fy * bot
            ok &= sd > f32(0)
            carve = ok & (sd > sz * (f32(1) + carving))
            carved += carve
            ok &= ~carve
            ok &= ~(np.abs(sd - sz) >= sz * thr)
            w2 = backproject(K[o], R[o], t[o], su, sv, sd)
            rx, ry, rz = rot_add(R[ref], t[ref], w2)
            ok &= rz > f32(1e-6)
            ru = (K[ref][0] * rx) / rz + K[ref][2]
            rv = (K[ref][4] * ry) / rz + K[ref][5]
            ok &= ~((np.abs(ru - xf) + np.abs(rv - yf)) > f32(2))
            ok &= ~(np.abs(rz - d) >= d * thr)
            consistent += ok
    keep = valid & (consistent >= eff_min) & (carved < max_carved)
    return np.where(keep, d, f32(0)).astype(f32)


class _FuseView(ctypes.Structure):
    _fields_ = [("K", ctypes.c_void_p), ("R", ctypes.c_void_p), ("t", ctypes.c_void_p),
                ("W", ctypes.c_int), ("H", ctypes.c_int), ("depth", ctypes.c_void_p),
                ("normal", ctypes.c_void_p), ("color", ctypes.c_void_p),
                ("mask", ctypes.c_void_p), ("nbrs", ctypes.c_void_p), ("n_nbrs", ctypes.c_int),
                ("primary", ctypes.c_int)]


def port_fuse(views, min_num_consistent=3, max_reproj_error=2.0, max_depth_error=0.01,
              max_normal_error=10.0, border_margin=5, behind_depth_factor=0.3, sor_knn=0,
              sor_stddev_factor=2.5):
    """DepthmapFuser::Fuse (fuser.cc:115-372) in the C restatement, followed
    by the statistical outlier removal (fuser.cc:374-482, port_sor) when
    sor_knn > 0.  views: dicts with K, R, t, depth (H, W), normal (H, W, 3),
    color (H, W, 3) uint8, mask (H, W) uint8 or None, neighbor_ids, primary.
    Returns (points (N, 3) f32, normals (N, 3) f32, colors (N, 3) u8)."""
    L = port()
    if not hasattr(L, "_fuse_ready"):
        L.or_fuse.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                              ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float,
                              _f, _f, _u8, ctypes.c_long]
        L.or_fuse.restype = ctypes.c_long
        L._fuse_ready = True
    keep = []
    arr = (_FuseView * len(views))()
    cap = 0
    for k, v in enumerate(views):
        K = np.ascontiguousarray(v["K"], np.float64)
        R = np.ascontiguousarray(v["R"], np.float64)
        t = np.ascontiguousarray(v["t"], np.float64).reshape(3)
        d = np.ascontiguousarray(v["depth"], np.float32)
        n = np.ascontiguousarray(v["normal"], np.float32)
        c = np.ascontiguousarray(v["color"], np.uint8)
        m = v.get("mask")
        m = None if m is None else np.ascontiguousarray(m, np.uint8)
        nb = np.ascontiguousarray(v["neighbor_ids"], np.int32).reshape(-1)
        keep += [K, R, t, d, n, c, m, nb]
        H, W = d.shape
        arr[k] = _FuseView(K.ctypes.data, R.ctypes.data, t.ctypes.data, W, H, d.ctypes.data,
                           n.ctypes.data, c.ctypes.data, None if m is None else m.ctypes.data,
                           nb.ctypes.data if nb.size else None, int(nb.size),
                           int(bool(v.get("primary", True))))
        if v.get("primary", True):
            cap += H * W
    pts = np.zeros((max(cap, 1), 3), np.float32)
    nrm = np.zeros((max(cap, 1), 3), np.float32)
    clr = np.zeros((max(cap, 1), 3), np.uint8)
    cnt = L.or_fuse(ctypes.cast(arr, ctypes.c_void_p), len(views), int(min_num_consistent),
                    float(max_reproj_error), float(max_depth_error), float(max_normal_error),
                    int(border_margin), float(behind_depth_factor), _P(pts, _f), _P(nrm, _f),
                    _P(clr, _u8), cap)
    pts, nrm, clr = pts[:cnt].copy(), nrm[:cnt].copy(), clr[:cnt].copy()
    if sor_knn > 0:
        keep, _ = port_sor(pts, sor_knn, sor_stddev_factor)
        pts, nrm, clr = pts[keep], nrm[keep], clr[keep]
    return pts, nrm, clr


def port_sor(points, knn, stddev_factor):
    """The fuser's statistical outlier removal (fuser.cc:374-482) in the C
    restatement (or_sor: exact K nearest neighbours by brute force, so small
    inputs only).  Returns (keep (N,) bool, mean kNN distance (N,) f32)."""
    L = port()
    if not getattr(L, "_sor_ready", False):
        L.or_sor.argtypes = [_f, ctypes.c_long, ctypes.c_int, ctypes.c_float, _u8, _f]
        L.or_sor.restype = ctypes.c_long
        L._sor_ready = True
    p = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    keep = np.zeros(len(p), np.uint8)
    mk = np.zeros(len(p), np.float32)
    L.or_sor(_P(p, _f), len(p), int(knn), float(stddev_factor), _P(keep, _u8), _P(mk, _f))
    return keep.astype(bool), mk


class _SvoView(ctypes.Structure):
    _fields_ = [("K", ctypes.c_void_p), ("R", ctypes.c_void_p), ("t", ctypes.c_void_p),
                ("W", ctypes.c_int), ("H", ctypes.c_int), ("depth", ctypes.c_void_p),
                ("normal", ctypes.c_void_p), ("color", ctypes.c_void_p),
                ("mask", ctypes.c_void_p), ("weight", ctypes.c_void_p)]


def _svo_views(views):
    keep = []
    arr = (_SvoView * max(len(views), 1))()
    for k, v in enumerate(views):
        K = np.ascontiguousarray(v["K"], np.float64)
        R = np.ascontiguousarray(v["R"], np.float64)
        t = np.ascontiguousarray(v["t"], np.float64).reshape(3)
        d = np.ascontiguousarray(v["depth"], np.float32)
        H, W = d.shape

        def opt(name, dt):
            a = v.get(name)
            if a is None:
                return None
            a = np.ascontiguousarray(a, dt)
            keep.append(a)
            return a.ctypes.data

        keep += [K, R, t, d]
        arr[k] = _SvoView(K.ctypes.data, R.ctypes.data, t.ctypes.data, W, H, d.ctypes.data,
                          opt("normal", np.float32), opt("color", np.uint8),
                          opt("mask", np.uint8), opt("weight", np.float32))
    return arr, keep


def _svo_lib():
    L = port()
    if not getattr(L, "_svo_ready", False):
        fp3 = ctypes.POINTER(ctypes.c_float)
        L.or_svo_count.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                   fp3, fp3]
        L.or_svo_count.restype = ctypes.c_long
        L.or_svo_fuse.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                  ctypes.c_float, fp3, fp3, ctypes.c_long, _f, _f, _u8,
                                  ctypes.c_long]
        L.or_svo_fuse.restype = ctypes.c_long
        L._svo_ready = True
    return L


def port_svo(views, voxel_size=0.02, trunc_factor=4.0, min_weight=3.0, bbox=None):
    """SVOFuser (svo_fuser.cc:52-183 over the kernels of
    svo_opencl_kernels.h:187-651) in the C restatement.  views: dicts with K,
    R, t, depth (H, W) and optional normal (H, W, 3), color (H, W, 3) uint8,
    mask (H, W) uint8, weight (H, W) f32.  bbox: (min_world, max_world) or
    None.  The setters' clamps (svo_fuser.cc:15-21) are applied here.
    Returns (count, points (N, 3) f32, normals (N, 3) f32, colors (N, 3) u8),
    the points in ascending voxel order, +X, +Y, +Z per voxel."""
    L = _svo_lib()
    vs = max(1e-6, float(np.float32(voxel_size)))
    tf = max(1.0, float(np.float32(trunc_factor)))
    mw = max(0.0, float(np.float32(min_weight)))
    arr, keep = _svo_views(views)
    if bbox is not None:
        bmin = np.ascontiguousarray(bbox[0], np.float32).reshape(3)
        bmax = np.ascontiguousarray(bbox[1], np.float32).reshape(3)
        pb = (_P(bmin, _f), _P(bmax, _f))
    else:
        pb = (None, None)
    n_views = len(views)
    cnt = L.or_svo_count(ctypes.cast(arr, ctypes.c_void_p), n_views, vs, tf, *pb)
    if cnt < 0:
        raise MemoryError("or_svo_count")
    n = L.or_svo_fuse(ctypes.cast(arr, ctypes.c_void_p), n_views, vs, tf, mw, *pb, cnt,
                      None, None, None, 0)
    if n < 0:
        raise MemoryError("or_svo_fuse")
    pts = np.zeros((max(n, 1), 3), np.float32)
    nrm = np.zeros((max(n, 1), 3), np.float32)
    clr = np.zeros((max(n, 1), 3), np.uint8)
    L.or_svo_fuse(ctypes.cast(arr, ctypes.c_void_p), n_views, vs, tf, mw, *pb, cnt,
                  _P(pts, _f), _P(nrm, _f), _P(clr, _u8), n)
    del keep
    return int(cnt), pts[:n].copy(), nrm[:n].copy(), clr[:n].copy()


def acm_float_image(img):
    """An 8-bit image as the live estimator uploads it (cv::Mat::convertTo
    with scale 1/255: float(v) * float(1/255))."""
    return np.ascontiguousarray(img, np.float32) * np.float32(1.0 / 255.0)


def _acm_args(views):
    L = port()
    if not getattr(L, "_acm_ready", False):
        pp = ctypes.POINTER(ctypes.c_void_p)
        ip = ctypes.POINTER(ctypes.c_int)
        L.or_acmmp_run.argtypes = [pp, ip, ip, pp, pp, pp, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                   ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                   ctypes.c_float, ctypes.c_float, _f, _f, _f, _f]
        L.or_acmmp_run.restype = ctypes.c_int
        L.or_acmmp_init.argtypes = [pp, ip, ip, pp, pp, pp, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_float, _f, _f,
                                    ctypes.POINTER(ctypes.c_uint32)]
        L.or_acmmp_init.restype = ctypes.c_int
        L._acm_ready = True
    keep = []
    n = len(views)
    imgs = (ctypes.c_void_p * n)()
    Ks = (ctypes.c_void_p * n)()
    Rs = (ctypes.c_void_p * n)()
    ts = (ctypes.c_void_p * n)()
    ws = (ctypes.c_int * n)()
    hs = (ctypes.c_int * n)()
    for i, (K, R, t, img) in enumerate(views):
        f = acm_float_image(img)
        K = np.ascontiguousarray(K, np.float64)
        R = np.ascontiguousarray(R, np.float64)
        t = np.ascontiguousarray(t, np.float64).reshape(3)
        keep += [f, K, R, t]
        imgs[i], Ks[i], Rs[i], ts[i] = f.ctypes.data, K.ctypes.data, R.ctypes.data, t.ctypes.data
        hs[i], ws[i] = f.shape
    return L, keep, imgs, ws, hs, Ks, Rs, ts


def port_acmmp(views, depth_min, depth_max, iterations=3, patch_size=11, sigma_spatial=5.0,
               sigma_color=3.0 / 255.0, top_k=4, census_weight=0.3, smooth_weight=0.0,
               geom_weight=0.0):
    """The live path's PatchMatch estimator for one reference view, one
    level, no SfM prior (estimator.cc:120-243, 941-1040 over the kernels of
    opencl_kernels.h) in the C restatement.  views: [(K, R, t, image u8)],
    the reference first.  Returns (depth, normal (H, W, 3), cost,
    confidence), all float32."""
    L, keep, imgs, ws, hs, Ks, Rs, ts = _acm_args(views)
    H, W = hs[0], ws[0]
    depth = np.zeros((H, W), np.float32)
    nrm = np.zeros((H, W, 3), np.float32)
    cost = np.zeros((H, W), np.float32)
    conf = np.zeros((H, W), np.float32)
    rc = L.or_acmmp_run(imgs, ws, hs, Ks, Rs, ts, len(views), int(iterations), int(patch_size),
                        float(sigma_spatial), float(sigma_color), int(top_k),
                        float(census_weight), float(smooth_weight), float(geom_weight),
                        float(depth_min), float(depth_max), _P(depth, _f), _P(nrm, _f),
                        _P(cost, _f), _P(conf, _f))
    if rc:
        raise ValueError(f"or_acmmp_run failed ({rc})")
    del keep
    return depth, nrm, cost, conf


def port_acmmp_init(views, depth_min, depth_max, patch_size=11, sigma_spatial=5.0,
                    sigma_color=3.0 / 255.0, top_k=4, census_weight=0.3):
    """The random initialisation alone (opencl_kernels.h:1055-1124):
    (planes (H, W, 4), costs (H, W), selected views (H, W) uint32)."""
    L, keep, imgs, ws, hs, Ks, Rs, ts = _acm_args(views)
    H, W = hs[0], ws[0]
    planes = np.zeros((H, W, 4), np.float32)
    costs = np.zeros((H, W), np.float32)
    sel = np.zeros((H, W), np.uint32)
    rc = L.or_acmmp_init(imgs, ws, hs, Ks, Rs, ts, len(views), int(patch_size),
                         float(sigma_spatial), float(sigma_color), int(top_k),
                         float(census_weight), float(depth_min), float(depth_max),
                         _P(planes, _f), _P(costs, _f),
                         sel.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    if rc:
        raise ValueError(f"or_acmmp_init failed ({rc})")
    del keep
    return planes, costs, sel


def _acm_level_lib():
    L = port()
    if not getattr(L, "_acm_level_ready", False):
        pp = ctypes.POINTER(ctypes.c_void_p)
        ip = ctypes.POINTER(ctypes.c_int)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        dp = ctypes.POINTER(ctypes.c_double)
        L.or_acmmp_level.argtypes = [pp, ip, ip, pp, pp, pp, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                     ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                     ctypes.c_float, ctypes.c_float, _f, _f, ctypes.c_int,
                                     ctypes.c_int, _f, ctypes.c_uint32, _f, u32p, ctypes.c_int,
                                     _f, _f, _f, _f]
        L.or_acmmp_sfm_project.argtypes = [dp, ctypes.c_long, dp, dp, dp, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_float, ctypes.c_float, _f, _f,
                                           _f]
        L.or_acmmp_sfm_project.restype = ctypes.c_long
        L.or_acmmp_sfm_prior.argtypes = [_f, _f, _f, ctypes.c_long,
                                         ctypes.POINTER(ctypes.c_int), ctypes.c_long, dp,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                         ctypes.c_float, _f, u32p]
        L.or_acmmp_sfm_prior.restype = ctypes.c_long
        L.or_acmmp_level.restype = ctypes.c_int
        L.or_resize_area_u8.argtypes = [_u8, ctypes.c_int, ctypes.c_int, ctypes.c_int, _u8]
        L.or_resize_area_general_u8.argtypes = [_u8, ctypes.c_int, ctypes.c_int, _u8,
                                                ctypes.c_int, ctypes.c_int]
        L.or_resize_linear_f32.argtypes = [_f, ctypes.c_int, ctypes.c_int, _f, ctypes.c_int,
                                           ctypes.c_int]
        L._acm_level_ready = True
    return L


def acm_resize_area(img, k):
    """cv::resize(INTER_AREA) by an integer factor k dividing both sizes."""
    L = _acm_level_lib()
    im = np.ascontiguousarray(img, np.uint8)
    H, W = im.shape
    out = np.zeros((H // k, W // k), np.uint8)
    L.or_resize_area_u8(_P(im, _u8), W, H, int(k), _P(out, _u8))
    return out


def acm_resize_area_to(img, w, h):
    """cv::resize(INTER_AREA) of an 8-bit image to (w, h): the fast path for
    integer ratios, the general area path otherwise."""
    L = _acm_level_lib()
    im = np.ascontiguousarray(img, np.uint8)
    H, W = im.shape
    if W % w == 0 and H % h == 0 and W // w == H // h:
        return acm_resize_area(im, W // w)
    out = np.zeros((h, w), np.uint8)
    L.or_resize_area_general_u8(_P(im, _u8), W, H, _P(out, _u8), int(w), int(h))
    return out


def acm_resize_linear(depth, W, H):
    """The previous-level depth resize (OpenCV's pixel-centre bilinear in
    FP32, each operation rounded by itself)."""
    L = _acm_level_lib()
    d = np.ascontiguousarray(depth, np.float32)
    out = np.zeros((H, W), np.float32)
    L.or_resize_linear_f32(_P(d, _f), d.shape[1], d.shape[0], _P(out, _f), int(W), int(H))
    return out


def acm_delaunay(xy, W, H):
    """The prior's triangulation as cv::Subdiv2D builds it: the Delaunay
    triangles (scipy's Qhull) of the points with the virtual vertices
    (3M, 0), (0, 3M), (-3M, -3M), M = max(W, H), less those touching them;
    ascending index triples, sorted."""
    from scipy.spatial import Delaunay

    xy = np.asarray(xy, np.float64).reshape(-1, 2)
    n = len(xy)
    big = 3.0 * max(W, H)
    aug = np.concatenate([xy, [[big, 0.0], [0.0, big], [-big, -big]]])
    t = Delaunay(aug).simplices
    t = np.sort(t[(t < n).all(axis=1)], axis=1)
    return t[np.lexsort((t[:, 2], t[:, 1], t[:, 0]))].astype(np.int32).copy()


def acm_sfm_prior(points, K, R, t, W, H, depth_min, depth_max):
    """ComputeSfMPlanarPrior (estimator.cc:664-940) in the restatement: the
    projection and the per-triangle planes, rasterisation and depth check in
    C; the triangulation by acm_delaunay (scipy's Qhull over the points and
    cv::Subdiv2D's virtual vertices).  Returns (planes (H, W, 4) f32, mask
    (H, W) uint32), or
    None when fewer than 4 points project."""
    from scipy.spatial import Delaunay

    L = _acm_level_lib()
    dp = ctypes.POINTER(ctypes.c_double)
    p = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    K = np.ascontiguousarray(K, np.float64).reshape(9)
    R = np.ascontiguousarray(R, np.float64).reshape(9)
    t = np.ascontiguousarray(t, np.float64).reshape(3)
    n = len(p)
    uv = np.zeros((max(n, 1), 2), np.float32)
    dep = np.zeros(max(n, 1), np.float32)
    cam = np.zeros((max(n, 1), 3), np.float32)
    m = L.or_acmmp_sfm_project(p.ctypes.data_as(dp), n, K.ctypes.data_as(dp),
                               R.ctypes.data_as(dp), t.ctypes.data_as(dp), int(W), int(H),
                               float(depth_min), float(depth_max), _P(uv, _f), _P(dep, _f),
                               _P(cam, _f))
    if m < 4:
        return None
    tri = acm_delaunay(uv[:m].astype(np.float64), W, H)
    planes = np.zeros((H, W, 4), np.float32)
    mask = np.zeros((H, W), np.uint32)
    L.or_acmmp_sfm_prior(_P(uv, _f), _P(dep, _f), _P(cam, _f), m,
                         tri.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(tri),
                         K.ctypes.data_as(dp), int(W), int(H), float(depth_min), float(depth_max),
                         _P(planes, _f), mask.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    return planes, mask


def port_acmmp_cluster(refs, hierarchy_levels=1, iterations=3, patch_size=11, sigma_spatial=5.0,
                       sigma_color=3.0 / 255.0, top_k=4, census_weight=0.3, smooth_weight=0.0,
                       geom_weight=0.0, geom_links=()):
    """DepthmapClusterEstimator::Run (cluster_estimator.cc:82-138) over
    RunLevel (estimator.cc:159-243) in the C restatement, levels outermost:
    the pyramid (estimator.cc:562-588, OpenCV's area resize),
    upsampling from each reference's own coarser result, and previous-level
    depths of linked references for the geometric term (updated in place as
    the references of a level finish, as the reference does), and each
    level's SfM planar prior where a reference has "sfm" points.
    refs: [dict(views=[(K, R, t, image u8), ...] (reference first),
    depth_min, depth_max, optional sfm (N, 3))]; geom_links: (ref, source
    index, from ref).
    Returns [(depth, normal, cost, confidence)] per reference."""
    L = _acm_level_lib()
    N = max(1, int(hierarchy_levels))
    n_refs = len(refs)
    links = {}
    for r, s, fr in geom_links:
        links.setdefault(r, []).append((s, fr))
    prev_depths = [None] * n_refs
    coarse = [None] * n_refs
    results = [None] * n_refs
    for level in range(N):
        scale = np.float32(1.0 / 2.0 ** (N - 1 - level))
        for i, ref in enumerate(refs):
            views = []
            for K, R, t, img in ref["views"]:
                K = np.array(K, np.float64).reshape(3, 3)
                img = np.ascontiguousarray(img, np.uint8)
                if scale < np.float32(0.999):
                    h0, w0 = img.shape
                    nw = max(int(np.float32(w0) * scale), 1)
                    nh = max(int(np.float32(h0) * scale), 1)
                    img = acm_resize_area_to(img, nw, nh)
                    sx = np.float32(nw) / np.float32(w0)
                    sy = np.float32(nh) / np.float32(h0)
                    K = K.copy()
                    K[0, 0] *= np.float64(sx)
                    K[0, 2] *= np.float64(sx)
                    K[1, 1] *= np.float64(sy)
                    K[1, 2] *= np.float64(sy)
                views.append((K, R, t, img))
            _, keep, imgs, ws, hs, Ks, Rs, ts = _acm_args(views)
            H, W = hs[0], ws[0]
            entries = []
            if level > 0 and geom_weight > 0 and links.get(i):
                for s_idx, fr in links[i]:
                    if 0 <= fr < n_refs and prev_depths[fr] is not None:
                        entries.append((s_idx, prev_depths[fr]))
            pd, mask = None, 0
            if entries:
                pd = np.zeros((16, H, W), np.float32)
                for s_idx, d in entries:
                    if not 0 <= s_idx < 16:
                        continue
                    if d.shape != (H, W):
                        d = acm_resize_linear(d, W, H)
                    pd[s_idx] = d
                    mask |= 1 << s_idx
            cd = cn = None
            cw = ch = 0
            if level > 0:
                cd, cn, _, cw, ch = coarse[i]
            prior = None
            if ref.get("sfm") is not None and len(ref["sfm"]):
                K0, R0, t0, _ = views[0]
                prior = acm_sfm_prior(ref["sfm"], K0, R0, t0, W, H, ref["depth_min"],
                                      ref["depth_max"])
                if prior is not None and not prior[1].any():
                    prior = None
            depth = np.zeros((H, W), np.float32)
            nrm = np.zeros((H, W, 3), np.float32)
            cost = np.zeros((H, W), np.float32)
            conf = np.zeros((H, W), np.float32)
            rc = L.or_acmmp_level(
                imgs, ws, hs, Ks, Rs, ts, len(views), int(iterations), int(patch_size),
                float(sigma_spatial), float(sigma_color), int(top_k), float(census_weight),
                float(smooth_weight), float(geom_weight), float(ref["depth_min"]),
                float(ref["depth_max"]), None if cd is None else _P(cd, _f),
                None if cn is None else _P(cn, _f), cw, ch,
                None if pd is None else _P(pd, _f), mask,
                None if prior is None else _P(prior[0], _f),
                None if prior is None else prior[1].ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                int(level == N - 1), _P(depth, _f),
                _P(nrm, _f), _P(cost, _f), _P(conf, _f))
            if rc:
                raise ValueError(f"or_acmmp_level failed ({rc})")
            del keep
            results[i] = (depth, nrm, cost, conf)
            if level < N - 1:
                coarse[i] = (depth, nrm, cost, W, H)
                prev_depths[i] = depth
    return results
