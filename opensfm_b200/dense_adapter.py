"""OpenSfM's dense depthmap stages on the B200 library, file for file.

Two entry points stand in for the places where ``opensfm/dense.py`` makes
per-view depthmaps and cleans them:

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
