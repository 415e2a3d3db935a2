"""Generates ``fusion_oracle_regression.npz``: inputs and outputs of the
restatements of the steps after the depthmaps (``oracle.gpu_clean_fp32``,
``oracle.port_fuse`` with and without the outlier removal, and
``oracle.port_svo``) on one small seeded case.  The reference's OpenCL
cleaner and SVO kernels cannot run here and its fuser needs its C++ build,
so these are not reference outputs: they pin the restatements themselves,
so that a change to their arithmetic shows up on the CPU.

Four ring views at 40x30: ray-cast depths with 0.2 % noise and 3 % holes,
tilted normals, colours from the images, a mask on two views.

Usage: python tests/golden/make_fusion_regression.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from opensfm_b200 import synthetic as S  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fusion_oracle_regression.npz")
W, H, N = 40, 30, 4
FUSE = dict(min_num_consistent=2, max_reproj_error=2.0, max_depth_error=0.02,
            max_normal_error=40.0, border_margin=2, behind_depth_factor=0.3)
SVO = dict(voxel_size=0.15, trunc_factor=3.0, min_weight=1.0)
CLEAN = dict(same_depth_threshold=0.02, min_consistent_views=2, carving_threshold=0.2,
             max_carved_views=1)


def views_from(f):
    out = []
    for k in range(N):
        out.append(dict(K=f["K"][k], R=f["R"][k], t=f["t"][k], depth=f["depth"][k],
                        normal=f["normal"][k], color=f["color"][k],
                        mask=f["mask"][k] if f["has_mask"][k] else None,
                        neighbor_ids=list(range(N)), primary=(k != N - 1)))
    return out


def outputs(f):
    """The restatements' outputs for the stored inputs, by name."""
    o = {}
    views = views_from(f)
    for ref in range(N):
        nb = [v for v in range(N) if v != ref]
        o[f"clean{ref}"] = O.gpu_clean_fp32(list(f["K"]), list(f["R"]), list(f["t"]),
                                            list(f["depth"]), ref, nb, **CLEAN)
    for name, kw in (("fuse", {}), ("fuse_sor", dict(sor_knn=6, sor_stddev_factor=2.0))):
        p, n, c = O.port_fuse(views, **FUSE, **kw)
        o[name + "_points"], o[name + "_normals"], o[name + "_colors"] = p, n, c
    svo_views = [dict(v, weight=None) for v in views]
    cnt, p, n, c = O.port_svo(svo_views, **SVO)
    o["svo_count"] = np.array(cnt, np.int64)
    o["svo_points"], o["svo_normals"], o["svo_colors"] = p, n, c
    return o


def main():
    vs = S.ring_viewset(17, N, W, H)
    rng = np.random.default_rng(4)
    depth, normal, color, mask = [], [], [], []
    for k in range(N):
        d = (vs.depths[k] * (1 + 0.002 * rng.standard_normal((H, W)))).astype(np.float32)
        d[rng.random((H, W)) < 0.03] = 0
        nr = np.zeros((H, W, 3), np.float32)
        nr[..., 2] = -1.0
        nr[..., :2] = 0.2 * rng.standard_normal((H, W, 2))
        depth.append(d)
        normal.append(nr)
        color.append(np.stack([vs.images[k], 255 - vs.images[k], vs.images[k] // 2], -1))
        m = np.ones((H, W), np.uint8)
        m[:, : W // 8] = 0
        mask.append(m)
    f = dict(K=np.stack([c.K for c in vs.cameras]), R=np.stack([c.R for c in vs.cameras]),
             t=np.stack([c.t for c in vs.cameras]), depth=np.stack(depth), normal=np.stack(normal),
             color=np.stack(color).astype(np.uint8), mask=np.stack(mask),
             has_mask=np.array([k % 2 == 1 for k in range(N)]))
    f.update(outputs(f))
    np.savez_compressed(OUT, **f)
    print(OUT, {k: v.shape for k, v in f.items()})


if __name__ == "__main__":
    main()
