"""Generates ``acmmp_oracle_regression.npz``: inputs and outputs of the
cluster estimator's C restatement (``oracle/acmmp_oracle.c`` through
``oracle.port_acmmp`` and ``oracle.port_acmmp_cluster``) on two small seeded
cases.  The live estimator's OpenCL kernels cannot run here, so these are
not reference outputs: they pin the restatement itself, so that a change to
its arithmetic shows up on the CPU before any GPU comparison.

Case A: one reference, three sources, one level, patch 5, 2 iterations,
smoothness 0.2.  Case B: two references of three sources each, 2 levels,
geometric weight 0.2 with a link each way, the SfM planar prior from 120
sampled surface points per reference (those with a depth kept).

Usage: python tests/golden/make_acmmp_regression.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from opensfm_b200 import synthetic as S  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "acmmp_oracle_regression.npz")
W, H = 48, 36


def surface_points(vs, k, n, seed):
    rng = np.random.default_rng(seed)
    d, c = vs.depths[k], vs.cameras[k]
    ys, xs = rng.integers(0, H, n), rng.integers(0, W, n)
    dd = d[ys, xs]
    ray = np.stack([xs + rng.uniform(0, 1, n), ys + rng.uniform(0, 1, n), np.ones(n)], -1)
    Xc = (ray @ np.linalg.inv(c.K).T) * dd[:, None]
    return ((Xc - c.t) @ c.R)[dd > 0]


def main():
    vs = S.ring_viewset(21, 6, W, H)
    f = {"images": np.stack(vs.images), "K": np.stack([c.K for c in vs.cameras]),
         "R": np.stack([c.R for c in vs.cameras]), "t": np.stack([c.t for c in vs.cameras])}
    ranges = np.array([S.depth_range(vs.depths[i]) for i in range(2)], np.float64)
    f["ranges"] = ranges
    view = lambda i: (f["K"][i], f["R"][i], f["t"][i], f["images"][i])  # noqa: E731
    # Case A.
    a = O.port_acmmp([view(i) for i in (0, 1, 2, 5)], ranges[0, 0], ranges[0, 1], iterations=2,
                     patch_size=5, smooth_weight=0.2)
    for name, arr in zip(("depth", "normal", "cost", "conf"), a):
        f["a_" + name] = arr
    # Case B.
    f["sfm0"], f["sfm1"] = surface_points(vs, 0, 120, 7), surface_points(vs, 1, 120, 8)
    refs = [dict(views=[view(i) for i in (0, 1, 2, 5)], depth_min=ranges[0, 0],
                 depth_max=ranges[0, 1], sfm=f["sfm0"]),
            dict(views=[view(i) for i in (1, 0, 2, 3)], depth_min=ranges[1, 0],
                 depth_max=ranges[1, 1], sfm=f["sfm1"])]
    b = O.port_acmmp_cluster(refs, hierarchy_levels=2, iterations=2, patch_size=5,
                             geom_weight=0.2, geom_links=[(0, 0, 1), (1, 0, 0)])
    for r, res in enumerate(b):
        for name, arr in zip(("depth", "normal", "cost", "conf"), res):
            f[f"b{r}_" + name] = arr
    np.savez_compressed(OUT, **f)
    print(OUT, {k: v.shape for k, v in f.items()},
          "valid A", float((f["a_depth"] > 0).mean()), "B", float((f["b0_depth"] > 0).mean()),
          float((f["b1_depth"] > 0).mean()))


if __name__ == "__main__":
    main()
