"""Generates the golden vectors in this folder from the reference's own code.

Runs the reference's ``opensfm/src/lib/dense/src/depthmap.cc`` (compiled
unmodified against the project's OpenCV shim by ``oracle/Makefile`` into
``oracle/_ref/``) on small seeded synthetic scenes and stores inputs and
outputs as ``.npz``.  The reference's own tests hold no depthmap, cleaner or
pruner vectors (``opensfm/src/lib/dense/test/depthmap_test.cc`` is empty), so
these are the pinned fixtures the CPU restatement is checked against.

Usage: python tests/golden/make_golden.py   (needs oracle/_ref built)
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from opensfm_b200 import synthetic as S  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def cams(vs):
    return ([c.K for c in vs.cameras], [c.R for c in vs.cameras], [c.t for c in vs.cameras])


def estimator_case(seed, W, H, n_views, patch, planes, sd):
    vs = S.ring_viewset(seed, n_views, W, H)
    Ks, Rs, ts = cams(vs)
    mn, mx = S.depth_range(vs.depths[0])
    masks = [np.ones_like(im) for im in vs.images]
    masks[0][: H // 6, : W // 5] = 0  # a masked corner
    e = O.RefEstimator()
    for K, R, t, im, mk in zip(Ks, Rs, ts, vs.images, masks):
        e.add_view(K, R, t, im, mk)
    e.set_depth_range(mn, mx, planes)
    e.set_patch_size(patch)
    e.set_min_patch_sd(sd)
    bf = e.compute_brute_force()
    rng = np.random.default_rng(seed + 100)
    # Random planes near the brute-force ones plus wild ones.
    rand_planes = bf[1] * (1 + 0.05 * rng.standard_normal(bf[1].shape)).astype(np.float32)
    rand_planes[::7] = rng.uniform(-0.3, 0.3, size=rand_planes[::7].shape).astype(np.float32)
    rand_planes = rand_planes.astype(np.float32)
    sp_score, sp_nghbr = e.score_planes(rand_planes)
    return dict(
        K=np.stack(Ks), R=np.stack(Rs), t=np.stack(ts), images=np.stack(vs.images),
        masks=np.stack(masks), gt=np.stack(vs.depths), min_depth=mn, max_depth=mx,
        num_planes=planes, patch_size=patch, min_patch_sd=sd,
        bf_depth=bf[0], bf_plane=bf[1], bf_score=bf[2], bf_nghbr=bf[3],
        planes=rand_planes, sp_score=sp_score, sp_nghbr=sp_nghbr,
        median_in=bf[0], median_out=O.ref_median5(bf[0]),
    )


def estimator_mixed_case(seed, sizes, patch, planes, sd):
    """Views of different sizes (the reference samples every view with its
    own rows and cols, depthmap.cc:16): view k is stored as image_k etc."""
    vs = S.mixed_viewset(seed, len(sizes), "box", sizes=sizes, step_deg=10.0)
    # mixed_viewset draws the sizes from the seed; pin them to the given order.
    cams_ = [S.Camera(S.intrinsics(w, h), c.R, c.t, w, h) for c, (w, h) in zip(vs.cameras, sizes)]
    imgs, deps = [], []
    for c in cams_:
        im, de = S.render(vs.scene, c, 2)
        imgs.append(im)
        deps.append(de)
    Ks, Rs, ts = [c.K for c in cams_], [c.R for c in cams_], [c.t for c in cams_]
    mn, mx = S.depth_range(deps[0])
    e = O.RefEstimator()
    for K, R, t, im in zip(Ks, Rs, ts, imgs):
        e.add_view(K, R, t, im, np.ones_like(im))
    e.set_depth_range(mn, mx, planes)
    e.set_patch_size(patch)
    e.set_min_patch_sd(sd)
    bf = e.compute_brute_force()
    rng = np.random.default_rng(seed + 100)
    rand_planes = (bf[1] * (1 + 0.05 * rng.standard_normal(bf[1].shape))).astype(np.float32)
    sp_score, sp_nghbr = e.score_planes(rand_planes)
    out = dict(n_views=len(sizes), min_depth=mn, max_depth=mx, num_planes=planes,
               patch_size=patch, min_patch_sd=sd, bf_depth=bf[0], bf_plane=bf[1],
               bf_score=bf[2], bf_nghbr=bf[3], planes=rand_planes, sp_score=sp_score,
               sp_nghbr=sp_nghbr)
    for k in range(len(sizes)):
        out.update({f"K_{k}": Ks[k], f"R_{k}": Rs[k], f"t_{k}": ts[k], f"image_{k}": imgs[k],
                    f"gt_{k}": deps[k]})
    return out


def clean_prune_case(seed, W, H, n_views):
    vs = S.ring_viewset(seed, n_views, W, H)
    Ks, Rs, ts = cams(vs)
    rng = np.random.default_rng(seed)
    depths = []
    for d in vs.depths:
        noisy = d * (1 + 0.004 * rng.standard_normal(d.shape))
        noisy[rng.random(d.shape) < 0.05] = 0
        depths.append(noisy.astype(np.float32))
    planes = []
    for K, d in zip(Ks, depths):
        ii, jj = np.mgrid[0:H, 0:W]
        ray = np.stack([jj, ii, np.ones_like(jj)], -1) @ np.linalg.inv(K).T
        n = np.array([0.1, -0.2, -1.0]) + 0.2 * rng.standard_normal((H, W, 3))
        denom = -(n * ray * d[..., None]).sum(-1, keepdims=True)
        denom = np.where(np.abs(denom) < 1e-6, 1e-6, denom)
        planes.append((n / denom).astype(np.float32))
    colors = [np.stack([im, 255 - im, im // 2], -1).astype(np.uint8) for im in vs.images]
    labels = [(im % 7).astype(np.uint8) for im in vs.images]
    clean = O.ref_clean(Ks, Rs, ts, depths, 0.01, 3)
    clean2 = O.ref_clean(Ks, Rs, ts, depths, 0.02, 2)
    pts, nrm, col, lab = O.ref_prune(Ks, Rs, ts, depths, planes, colors, labels, 0.01)
    return dict(
        K=np.stack(Ks), R=np.stack(Rs), t=np.stack(ts), depths=np.stack(depths),
        planes=np.stack(planes), colors=np.stack(colors), labels=np.stack(labels),
        clean_t01_v3=clean, clean_t02_v2=clean2,
        prune_points=pts, prune_normals=nrm, prune_colors=col, prune_labels=lab,
    )


CASES = {
    "estimator_80x60_v3_p7.npz": lambda: estimator_case(11, 80, 60, 3, 7, 24, 1.0),
    "estimator_72x54_v4_p5.npz": lambda: estimator_case(12, 72, 54, 4, 5, 16, 2.0),
    "clean_prune_64x48_v4.npz": lambda: clean_prune_case(13, 64, 48, 4),
    "estimator_mixed_v4_p7.npz": lambda: estimator_mixed_case(
        14, [(96, 72), (72, 96), (96, 54), (64, 48)], 7, 24, 1.0),
}


def main():
    """Writes the fixtures that are missing (all of them with --force)."""
    if not O.ref_available():
        O.build()
    force = "--force" in sys.argv
    for name, make in CASES.items():
        path = os.path.join(OUT, name)
        if force or not os.path.exists(path):
            np.savez_compressed(path, **make())
    for f in sorted(os.listdir(OUT)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
