"""OpenSfM's dense depthmap stages on the B200 library, file for file.

The live pipeline (``opensfm/dense.py``) makes raw depthmaps per cluster with
the OpenCL ``DepthmapClusterEstimator`` and cleans them with the
``GPUDepthmapCleaner``.  Two entry points stand in for those two call sites
on the library's classes of the same names, writing the same files:

- :func:`run_cluster_raw` - ``dense._run_cluster_raw`` (``dense.py:627-797``);
- :func:`clean_cluster_gpu` - the per-cluster cleaning inside
  ``dense._clean_views_batched_gpu`` (``dense.py:804-1018``).

Two more run the same two stages with the legacy ``pydense`` classes (the
API the B200 PatchMatch kernels implement):

- :func:`compute_raw_depthmaps` - the per-view raw depthmaps of
  ``dense._run_cluster_raw`` (``dense.py:627-797``): one batched PatchMatch
  run over every listed view (each against its nearest neighbours), written
  as ``<data>/depthmaps/<image>.raw.npz``.
- :func:`clean_depthmaps` - the cleaning of ``dense._clean_views_batched_gpu``
  (``dense.py:860-1018``): every view's raw depth checked against its
  neighbours' (``DepthmapCleaner``), written as ``<image>.clean.npz`` with the
  raw plane and a zero score, as ``dense.py:896-905`` writes them.

The estimator is the legacy ``pydense`` one (bilateral NCC PatchMatch,
``depthmap.cc``), not the OpenCL ACMMP estimator the live ``dense.py`` drives,
so the raw files carry its outputs: depth, plane (the ``n / d`` vector of
``depthmap.cc``), NCC score and the per-pixel best neighbour index.  Inputs
are what ``dense.py`` gathers for each shot: ``K`` in pixel coordinates of
the grey image, ``R`` and ``t`` of the pose, the grey uint8 image, the
neighbour list (the shot itself first, then the nearest views, as
``best_neighbors`` holds them) and the depth range.
"""
from __future__ import annotations

from typing import Dict, List, Mapping, Optional, Sequence, Tuple

import numpy as np

from . import dense_io, pydense

View = Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]  # K, R, t, grey image


def _cfg(config: Mapping, key: str, default):
    v = config.get(key, default) if config is not None else default
    return default if v is None else v


def compute_raw_depthmaps(data_path: str, views: Mapping[str, View],
                          best_neighbors: Mapping[str, Sequence[str]],
                          depth_ranges: Mapping[str, Tuple[float, float]],
                          shot_ids: Sequence[str], config: Optional[Mapping] = None,
                          seed: int = 1, tuning: Optional[Tuple[int, int, int]] = None
                          ) -> List[str]:
    """Raw depthmaps of ``shot_ids`` in one batched run; returns the ids.

    Config keys (OpenSfM's names): ``depthmap_num_matching_views`` (4),
    ``depthmap_patch_size`` (7), ``depthmap_min_patch_sd`` (1.0),
    ``depthmap_patchmatch_iterations`` (3).
    """
    n_match = int(_cfg(config, "depthmap_num_matching_views", 4))
    patch = int(_cfg(config, "depthmap_patch_size", 7))
    min_sd = float(_cfg(config, "depthmap_min_patch_sd", 1.0))
    iters = int(_cfg(config, "depthmap_patchmatch_iterations", 3))
    b = pydense.Batch()
    index: Dict[str, int] = {}

    def view_id(sid: str) -> int:
        if sid not in index:
            K, R, t, img = views[sid]
            index[sid] = b.add_view(K, R, t, np.ascontiguousarray(img, np.uint8))
        return index[sid]

    maps = []
    for sid in shot_ids:
        nbrs = [n for n in best_neighbors[sid] if n != sid][:n_match]
        if not nbrs:
            continue
        ref = view_id(sid)
        mn, mx = depth_ranges[sid]
        m = b.add_depthmap(ref, [view_id(n) for n in nbrs], float(mn), float(mx))
        maps.append((sid, m))
    if not maps:
        b.close()
        return []
    b.set_params(patch_size=patch, min_patch_sd=min_sd, iterations=iters, seed=seed)
    if tuning:
        b.set_tuning(*tuning)
    b.run()
    b.synchronize()
    done = []
    for sid, m in maps:
        depth, plane, score, nghbr = b.get(m)[:4]
        dense_io.save_raw_depthmap(data_path, sid, depth, plane, score, nghbr,
                                   list(best_neighbors[sid]))
        done.append(sid)
    b.close()
    return done


def clean_depthmaps(data_path: str, views: Mapping[str, View],
                    clean_neighbors: Mapping[str, Sequence[str]], shot_ids: Sequence[str],
                    config: Optional[Mapping] = None) -> List[str]:
    """Cleaned depthmaps of ``shot_ids`` from their raw files; returns the ids.

    Config keys: ``depthmap_same_depth_threshold`` (0.01),
    ``depthmap_min_consistent_views`` (3).  Neighbours without a raw file
    are left out, as ``dense.py`` only loads views that have one.
    """
    import os

    thr = float(_cfg(config, "depthmap_same_depth_threshold", 0.01))
    min_views = int(_cfg(config, "depthmap_min_consistent_views", 3))
    cache: Dict[str, tuple] = {}

    def raw(sid: str):
        if sid not in cache:
            cache[sid] = dense_io.load_raw_depthmap(data_path, sid)
        return cache[sid]

    done = []
    for sid in shot_ids:
        if not os.path.isfile(dense_io.depthmap_file(data_path, sid, "raw.npz")):
            continue
        c = pydense.DepthmapCleaner()
        c.set_same_depth_threshold(thr)
        c.set_min_consistent_views(min_views)
        K, R, t, _ = views[sid]
        depth, plane = raw(sid)[0], raw(sid)[1]
        c.add_view(K, R, t, depth)
        for n in clean_neighbors[sid]:
            if n == sid or not os.path.isfile(dense_io.depthmap_file(data_path, n, "raw.npz")):
                continue
            Kn, Rn, tn, _ = views[n]
            c.add_view(Kn, Rn, tn, raw(n)[0])
        cleaned = c.clean()
        dense_io.save_clean_depthmap(data_path, sid, cleaned, plane, np.zeros_like(cleaned))
        done.append(sid)
    return done


# ----------------------------------------------------------------------
# The live pipeline's stages: the cluster estimator and the GPU cleaner.

# OpenSfM's defaults for the keys these stages read (opensfm/config.py:375-463).
LIVE_DEFAULTS = {
    "depthmap_num_matching_views": 4, "depthmap_max_iterations": 4, "depthmap_patch_size": 5,
    "depthmap_max_image_size": 3200, "depthmap_max_cost": 0.9,
    "depthmap_same_depth_threshold": 0.01, "depthmap_min_consistent_views": 3,
    "depthmap_carving_threshold": 0.2, "depthmap_max_carved_views": 1,
    "depthmap_sigma_spatial": 5.0, "depthmap_sigma_color": 3.0 / 255.0,
    "depthmap_census_weight": 0.3, "depthmap_hierarchy_levels": 4,
    "depthmap_smooth_weight": 0.3, "depthmap_geom_consistency_weight": 0.05,
    "depthmap_sfm_planar_prior": True,
}


def _live(config: Optional[Mapping], key: str):
    return _cfg(config, key, LIVE_DEFAULTS[key])


def run_cluster_raw(data_path: str, views: Mapping[str, View],
                    best_neighbors: Mapping[str, Sequence[str]], cluster_shot_ids: Sequence[str],
                    depth_ranges: Mapping[str, Tuple[float, float]],
                    config: Optional[Mapping] = None,
                    sfm_points: Optional[Mapping[str, np.ndarray]] = None,
                    device_idx: int = 0) -> List[str]:
    """Raw depthmaps of one cluster, as ``dense._run_cluster_raw``
    (``dense.py:627-797``) makes them, on the library's
    ``DepthmapClusterEstimator``: every shot of the cluster is a reference
    with its ``depthmap_num_matching_views`` best neighbours as sources,
    references that are each other's sources are linked for geometric
    consistency, the SfM points seen by a shot (``sfm_points[shot]``, world
    coordinates) give its planar prior.  Each result is written as
    ``<image>.raw.npz`` with the live path's fields (``dense.py:741-775``):
    depth with non-finite pixels and pixels of cost > ``depthmap_max_cost``
    zeroed, ``plane`` = the normal map, ``score`` = the cost, an empty
    ``nghbr``, the neighbour ids and the confidence.  Returns the ids.

    ``views`` hold grey images no larger than ``depthmap_max_image_size``
    (``dense.py`` shrinks larger ones before this point) and ``K`` in pixel
    coordinates of that image; ``best_neighbors[shot]`` lists the shot
    itself first, as ``dense.py``'s neighbour lists do.
    """
    n_src = int(_live(config, "depthmap_num_matching_views"))
    max_size = int(_live(config, "depthmap_max_image_size"))
    cluster = pydense.DepthmapClusterEstimator()
    cluster.set_max_iterations(int(_live(config, "depthmap_max_iterations")))
    cluster.set_patch_size(int(_live(config, "depthmap_patch_size")))
    cluster.set_max_image_size(max_size)
    cluster.set_sigma_spatial(float(_live(config, "depthmap_sigma_spatial")))
    cluster.set_sigma_color(float(_live(config, "depthmap_sigma_color")))
    cluster.set_top_k(n_src)
    cluster.set_census_weight(float(_live(config, "depthmap_census_weight")))
    cluster.set_hierarchy_levels(int(_live(config, "depthmap_hierarchy_levels")))
    cluster.set_smooth_weight(float(_live(config, "depthmap_smooth_weight")))
    cluster.set_geom_consistency_weight(float(_live(config, "depthmap_geom_consistency_weight")))
    cluster.set_device(device_idx)

    def image(sid):
        K, R, t, img = views[sid]
        img = np.ascontiguousarray(img, np.uint8)
        if max(img.shape) > max_size:
            raise ValueError(f"view {sid} is larger than depthmap_max_image_size ({max_size})")
        return K, R, t, img

    ref_idx: Dict[str, int] = {}
    ref_nbrs: Dict[int, List[str]] = {}
    for sid in cluster_shot_ids:
        K, R, t, img = image(sid)
        mn, mx = depth_ranges[sid]
        idx = cluster.begin_ref_view(K, R, t, img, float(mn), float(mx))
        ref_idx[sid] = idx
        if _live(config, "depthmap_sfm_planar_prior") and sfm_points and sid in sfm_points:
            pts = np.asarray(sfm_points[sid], np.float64).reshape(-1, 3)
            if len(pts):
                cluster.set_sfm_points(pts)
        nbrs = [sid]
        for s in list(best_neighbors[sid])[1:n_src + 1]:
            Ks, Rs, ts, imgs = image(s)
            cluster.add_source_view(Ks, Rs, ts, imgs)
            nbrs.append(s)
        ref_nbrs[idx] = nbrs
    for sid, idx in ref_idx.items():
        nbrs = ref_nbrs[idx]
        for other, other_idx in ref_idx.items():
            if other != sid and other in nbrs:
                cluster.add_geom_link(idx, nbrs.index(other) - 1, other_idx)
    results = cluster.run()
    cluster.clear()
    max_cost = float(_live(config, "depthmap_max_cost"))
    done = []
    for sid, (depth, normal, cost, confidence) in zip(cluster_shot_ids, results):
        depth = np.asarray(depth, np.float32).copy()
        normal = np.asarray(normal, np.float32).copy()
        bad = ~np.isfinite(depth)
        depth[bad] = 0.0
        normal[bad] = 0.0
        if max_cost > 0:
            depth[cost > max_cost] = 0.0
        dense_io.save_raw_depthmap(data_path, sid, depth, normal, np.asarray(cost, np.float32),
                                   np.zeros((0,), np.int32), list(best_neighbors.get(sid, [])),
                                   np.asarray(confidence, np.float32))
        done.append(sid)
    cluster.close()
    return done


def clean_cluster_gpu(data_path: str, views: Mapping[str, View],
                      all_neighbors: Mapping[str, Sequence[str]], cluster_shots: Sequence[str],
                      config: Optional[Mapping] = None, max_neighbors: int = 16,
                      device_idx: int = 0) -> List[str]:
    """Cleaned depthmaps of one cluster, as ``_gpu_clean_and_save_cluster``
    inside ``dense._clean_views_batched_gpu`` (``dense.py:830-905``) makes
    them, on the library's ``GPUDepthmapCleaner``: every shot of the cluster
    against its first ``max_neighbors`` neighbours that have a raw file,
    views indexed in sorted id order; written as ``<image>.clean.npz`` with
    the raw normal as ``plane``, a zero score and the raw confidence.
    Returns the ids."""
    import os

    def has_raw(sid):
        return os.path.isfile(dense_io.depthmap_file(data_path, sid, "raw.npz"))

    cleaner = pydense.GPUDepthmapCleaner()
    cleaner.set_same_depth_threshold(float(_live(config, "depthmap_same_depth_threshold")))
    cleaner.set_min_consistent_views(int(_live(config, "depthmap_min_consistent_views")))
    cleaner.set_carving_threshold(float(_live(config, "depthmap_carving_threshold")))
    cleaner.set_max_carved_views(int(_live(config, "depthmap_max_carved_views")))
    cleaner.set_device(device_idx)
    shots = [s for s in cluster_shots if has_raw(s)]
    per_ref: Dict[str, List[str]] = {}
    needed = set(shots)
    for sid in shots:
        nbrs = [n for n in all_neighbors.get(sid, []) if n != sid and has_raw(n)][:max_neighbors]
        per_ref[sid] = nbrs
        needed.update(nbrs)
    ordered = sorted(needed)
    index = {sid: k for k, sid in enumerate(ordered)}
    raw = {}
    for sid in ordered:
        depth, normal, _, _, _, confidence = dense_io.load_raw_depthmap(data_path, sid)
        K, R, t, _ = views[sid]
        cleaner.add_view(K, R, t, depth)
        if sid in per_ref:
            raw[sid] = (normal, confidence)
    done = []
    for sid in shots:
        cleaned = cleaner.clean(index[sid], np.array([index[n] for n in per_ref[sid]], np.int32))
        normal, confidence = raw[sid]
        dense_io.save_clean_depthmap(data_path, sid, np.asarray(cleaned, np.float32), normal,
                                     np.zeros_like(cleaned, dtype=np.float32), confidence)
        done.append(sid)
    cleaner.clear()
    cleaner.close()
    return done
