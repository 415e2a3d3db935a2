"""Generates the PatchMatch and brute-force fixtures at the benchmark sizes
from the reference's own code.

The reference's ``opensfm/src/lib/dense/src/depthmap.cc`` (compiled
unmodified by ``oracle/Makefile`` into ``oracle/_ref/``) runs on two
workloads:

``pm_config1_320x240.npz``
    Box scene (ground plane + 12 boxes), 1 reference + 4 neighbours on a
    ring of radius 15 m at 10 degree steps (the reference in the middle, so
    its neighbours sit at -20, -10, +10 and +20 degrees), 320 x 240, patch 7,
    min_patch_sd 1.0: ``ComputeBruteForce`` with 64 planes (deterministic),
    ``ComputePatchMatch`` with 3 iterations and ``ComputePatchMatchSample``
    with 3 iterations.
``pm_config2_640x480.npz``
    The benchmark's ring reconstruction (seed 2024, 24 views of 640 x 480
    at 10 degree steps): depthmaps 0, 8 and 16, each against its 6 nearest
    views, patch 7, min_patch_sd 1.0, 50 planes of depth range, 3
    iterations.

The reference's PatchMatch is random: its initialisation draws from
``rand()`` (seeded here with ``srand``) and its refinements from an
``mt19937`` seeded by ``std::random_device`` (depthmap.cc:127-141), so every
run differs.  Each PatchMatch case is run RUNS times; the fixture keeps
every run's accuracy against the ray-cast ground truth (|d - gt| / gt <=
1 %), the valid fraction, and the depth of the first run as float16 (the
agreement test compares at 1 %, and float16 keeps 0.05 %).

The same cases also run through ``oracle.port_compute_redblack``: the GPU's
red-black schedule (6 half-passes; 4 adjacent + 4 far candidates and 6
refinements per update) restated in C with the reference's arithmetic.
Its accuracies (``rb_*``) are what that schedule reaches by itself, so the
GPU is held to them, and their distance to the reference's (a raster sweep)
is the schedule's own.  Inputs are not
stored: the scenes are regenerated from their seeds by
``opensfm_b200.synthetic`` and checked against the stored SHA-256 of the
images.

Usage: python tests/golden/make_pm_configs.py   (needs oracle/_ref built;
about two minutes on 8 cores)
"""
import hashlib
import multiprocessing as mp
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.dirname(os.path.abspath(__file__))
RUNS = 3
PATCH, MIN_SD, ITERS = 7, 1.0, 3
C1 = dict(seed=31, n_views=5, W=320, H=240, ref=2, planes=64)
C2 = dict(seed=2024, n_views=24, W=640, H=480, maps=(0, 8, 16), n_match=6, planes=50)


def images_digest(images):
    h = hashlib.sha256()
    for im in images:
        h.update(np.ascontiguousarray(im, np.uint8).tobytes())
    return h.hexdigest()


def config1_views():
    """(cameras, images, depths) in the reference's order: view 0 is the reference."""
    from opensfm_b200 import synthetic as S

    vs = S.ring_viewset(C1["seed"], C1["n_views"], C1["W"], C1["H"])
    order = [C1["ref"]] + [k for k in range(C1["n_views"]) if k != C1["ref"]]
    return ([vs.cameras[k] for k in order], [vs.images[k] for k in order],
            [vs.depths[k] for k in order])


def config2_views():
    """The ring reconstruction and, per fixture map, its 6 nearest views."""
    from opensfm_b200 import synthetic as S

    vs = S.ring_viewset(C2["seed"], C2["n_views"], C2["W"], C2["H"])
    matches = {v: vs.neighbors(v, 10)[:C2["n_match"]] for v in C2["maps"]}
    return vs, matches


def _run(task):
    """One reference run: (mode, K, R, t, images, min, max, planes, seed);
    modes 3 / 4: the red-black restatement of the GPU schedule (plain /
    sample) instead."""
    import oracle as O

    mode, Ks, Rs, ts, images, mn, mx, planes, seed = task
    if mode >= 3:
        t0 = time.perf_counter()
        out = O.port_compute_redblack(Ks, Rs, ts, images, [np.ones_like(im) for im in images], PATCH,
                                      mn, mx, 2 * ITERS, MIN_SD, seed, sample=(mode == 4))
        return list(out), time.perf_counter() - t0
    O.ref().ref_srand(seed)
    e = O.RefEstimator()
    for K, R, t, im in zip(Ks, Rs, ts, images):
        e.add_view(K, R, t, im, np.ones_like(im))
    e.set_depth_range(mn, mx, planes)
    e.set_patch_size(PATCH)
    e.set_min_patch_sd(MIN_SD)
    e.set_patchmatch_iterations(ITERS)
    t0 = time.perf_counter()
    out = e._compute(mode)
    return out, time.perf_counter() - t0


def main():
    import oracle as O
    from opensfm_b200 import synthetic as S

    assert O.ref_available(), "build oracle/_ref first (oracle/Makefile)"
    ctx = mp.get_context("spawn")
    # ---------------------------------------------------------- config 1
    cams, images, depths = config1_views()
    Ks, Rs, ts = [c.K for c in cams], [c.R for c in cams], [c.t for c in cams]
    gt = depths[0]
    mn, mx = S.depth_range(gt)
    base = (Ks, Rs, ts, images, mn, mx)
    tasks = [(0, *base, C1["planes"], 1)]
    tasks += [(1, *base, C1["planes"], 1000 + r) for r in range(RUNS)]
    tasks += [(2, *base, C1["planes"], 2000 + r) for r in range(RUNS)]
    tasks += [(3, *base, C1["planes"], 4000 + r) for r in range(RUNS)]
    tasks += [(4, *base, C1["planes"], 5000 + r) for r in range(RUNS)]
    # ---------------------------------------------------------- config 2
    vs, matches = config2_views()
    c2_tasks = []
    for v in C2["maps"]:
        ids = [v] + matches[v]
        g = vs.depths[v]
        a, b = S.depth_range(g)
        for mode in (1, 3):
            for r in range(RUNS):
                c2_tasks.append((mode, [vs.cameras[k].K for k in ids],
                                 [vs.cameras[k].R for k in ids], [vs.cameras[k].t for k in ids],
                                 [vs.images[k] for k in ids], a, b, C2["planes"],
                                 (3000 if mode == 1 else 6000) + 10 * v + r))
    t0 = time.time()
    with ctx.Pool(min(len(tasks) + len(c2_tasks), os.cpu_count() or 1)) as pool:
        res = pool.map(_run, tasks + c2_tasks, chunksize=1)
    print(f"reference runs done in {time.time() - t0:.0f} s", flush=True)
    r1, r2 = res[:len(tasks)], res[len(tasks):]

    bf, bf_s = r1[0]
    pm = r1[1:1 + RUNS]
    sm = r1[1 + RUNS:1 + 2 * RUNS]
    rb = r1[1 + 2 * RUNS:1 + 3 * RUNS]
    rbs = r1[1 + 3 * RUNS:]
    np.savez_compressed(
        os.path.join(OUT, "pm_config1_320x240.npz"),
        seed=C1["seed"], n_views=C1["n_views"], W=C1["W"], H=C1["H"], ref=C1["ref"],
        images_sha256=images_digest(images), min_depth=mn, max_depth=mx,
        num_planes=C1["planes"], patch_size=PATCH, min_patch_sd=MIN_SD, iterations=ITERS,
        bf_depth=bf[0], bf_score=bf[2], bf_nghbr=bf[3].astype(np.int8), bf_seconds=bf_s,
        pm_accuracy=np.array([S.accuracy(o[0], gt) for o, _ in pm]),
        pm_valid=np.array([float((o[0] > 0).mean()) for o, _ in pm]),
        pm_depth0=pm[0][0][0].astype(np.float16), pm_seconds=np.array([s for _, s in pm]),
        sample_accuracy=np.array([S.accuracy(o[0], gt) for o, _ in sm]),
        sample_valid=np.array([float((o[0] > 0).mean()) for o, _ in sm]),
        sample_depth0=sm[0][0][0].astype(np.float16),
        sample_seconds=np.array([s for _, s in sm]),
        rb_accuracy=np.array([S.accuracy(o[0], gt) for o, _ in rb]),
        rb_valid=np.array([float((o[0] > 0).mean()) for o, _ in rb]),
        rb_sample_accuracy=np.array([S.accuracy(o[0], gt) for o, _ in rbs]),
        rb_sample_valid=np.array([float((o[0] > 0).mean()) for o, _ in rbs]),
    )
    acc = np.zeros((len(C2["maps"]), RUNS))
    val = np.zeros_like(acc)
    secs = np.zeros_like(acc)
    rb_acc = np.zeros_like(acc)
    rb_val = np.zeros_like(acc)
    d0 = []
    for i, v in enumerate(C2["maps"]):
        for r in range(RUNS):
            out, s = r2[(2 * i) * RUNS + r]
            acc[i, r] = S.accuracy(out[0], vs.depths[v])
            val[i, r] = float((out[0] > 0).mean())
            secs[i, r] = s
            if r == 0:
                d0.append(out[0].astype(np.float16))
            out, s = r2[(2 * i + 1) * RUNS + r]
            rb_acc[i, r] = S.accuracy(out[0], vs.depths[v])
            rb_val[i, r] = float((out[0] > 0).mean())
    np.savez_compressed(
        os.path.join(OUT, "pm_config2_640x480.npz"),
        seed=C2["seed"], n_views=C2["n_views"], W=C2["W"], H=C2["H"],
        maps=np.array(C2["maps"]), matches=np.array([matches[v] for v in C2["maps"]]),
        images_sha256=images_digest(vs.images), num_planes=C2["planes"], patch_size=PATCH,
        min_patch_sd=MIN_SD, iterations=ITERS, pm_accuracy=acc, pm_valid=val,
        pm_depth0=np.stack(d0), pm_seconds=secs, rb_accuracy=rb_acc, rb_valid=rb_val,
    )
    print("config 1: brute force %.1f s; PatchMatch accuracy %s; sample accuracy %s"
          % (bf_s, np.round([S.accuracy(o[0], gt) for o, _ in pm], 4),
             np.round([S.accuracy(o[0], gt) for o, _ in sm], 4)))
    print("config 1 red-black restatement: PatchMatch %s, sample %s"
          % (np.round([S.accuracy(o[0], gt) for o, _ in rb], 4),
             np.round([S.accuracy(o[0], gt) for o, _ in rbs], 4)))
    print("config 2: PatchMatch accuracy per map x run\n%s\nseconds per run %.1f"
          % (np.round(acc, 4), secs.mean()))
    print("config 2 red-black restatement:\n%s" % np.round(rb_acc, 4))


if __name__ == "__main__":
    main()
