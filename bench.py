#!/usr/bin/env python
"""Benchmark of the dense depthmap path on B200.

Workload (one "step"): a ring reconstruction of 24 reference views at
640 x 480 (box scene: ground plane + 12 boxes, 4-octave value-noise texture),
each depthmap scored against its 6 nearest matching views with patch 7,
min patch sd 1.0 and 3 PatchMatch iterations, then DepthmapCleaner
(threshold 0.01, 3 consistent views) and DepthmapPruner (threshold 0.01)
over each map's 10 candidate neighbours.  Synthetic, seeded, ray-cast in
this process.

``value``: depthmaps/s with the views resident in HBM (one batched run per
step, replayed from a CUDA graph), device-timed over K steps.  ``e2e``: the
same through the public batch API from pinned host buffers, each step
uploading every view image and reading every cleaned depth map back, the
copies pipelined beside the runs on the batch's upload and readback streams.

``--impl reference`` times the reference's own CPU depthmap code
(opensfm/src/lib/dense/src/depthmap.cc compiled as oracle/_ref) on the
host's cores over the same whole reconstruction: every map's PatchMatch,
then DepthmapCleaner and DepthmapPruner, one process per core.  The
``cpu_baseline`` of the default line is a bounded ~30 s sample of bands of
the same views.

Multi-GPU: one process per GPU (torchrun); each rank runs its own replica of
the reconstruction (the path has no exchange step), so scaling is weak and
the job value is the sum over ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "640px depthmaps/s (6 views, 3 iters): learned-init vs plain at equal accuracy"
UNIT = "depthmaps/s"
W_, H_ = 640, 480
N_VIEWS, N_CAND, N_MATCH = 24, 10, 6
PATCH, MIN_SD, ITERS = 7, 1.0, 3
SEED = 2024
FLOPS_PER_TAP = 25  # affine warp 8 + bilinear 11 + NCC sums 6 (FMA = 2)
# The plain GPU PatchMatch: the reference's random initialisation and
# red-black half-passes with every matching view scored per candidate.
PLAIN_HALF_PASSES, PLAIN_KNIGHTS = 2 * ITERS, False
# DRAM bytes per half-pass on the ring workload, from ncu captures at tuning
# 32,4,2: a tile half-pass over every pixel of a colour
# (halfpass_kernel<3, true, 2> and <3, false, 2>), and the first list
# half-pass of the learned schedule with a settled start
# (halfpass_list_kernel<3, true, 2>).
TRAFFIC_SAMPLE_TILE, TRAFFIC_PLAIN_TILE, TRAFFIC_SETTLED_LIST = 318.8e6, 318.3e6, 278.0e6
# Learned schedules (half-passes, refinements per update, active-pixel
# tolerance, candidate-view mode, settled-start score, random-initialisation
# fallback), chosen on 12 held-out 640x480 scenes (seeds 900000-900011, none
# of them a training scene) with the committed network, every one of them
# above plain's accuracy there.  Mode 2: one view per candidate from the
# initialisation on; pixels whose neighbourhood moved by less than 1 % are
# left alone.  In order:
# - the settled-start schedule, whose held-out accuracy is within 0.0005 of
#   the same schedule without it (0.9031 / 5.93 ms against 0.9034 / 6.65;
#   plain's 0.8959 / 47.5 ms);
# - the schedules without it, fastest first (0.9034 / 6.65, 0.9044 / 7.50,
#   0.9041 / 7.88, 0.9038 / 8.18, 0.9035 / 8.34, 0.9042 / 8.89 ms), the last
#   a full initialisation on every view, then one view per candidate
#   (mode 1; 0.9048 / 8.98 ms);
# - the schedules with the random-initialisation fallback, fastest first
#   (0.9024 / 8.73, 0.9023 / 9.05 ms), for views unlike the training scenes;
#   the last scores every view per candidate.
LEARNED_SCHEDULES = ((4, 2, 0.01, 2, 0.9, 0), (4, 2, 0.01, 2, 0.0, 0), (6, 3, 0.01, 2, 0.0, 0),
                     (8, 3, 0.01, 2, 0.0, 0), (10, 3, 0.01, 2, 0.0, 0), (12, 3, 0.01, 2, 0.0, 0),
                     (8, 6, 0.01, 2, 0.0, 0), (6, 6, 0.01, 1, 0.0, 0), (8, 3, 0.01, 2, 0.0, 1),
                     (10, 3, 0.01, 2, 0.0, 1), (6, 6, 0.01, 0, 0.0, 1))


# ---------------------------------------------------------------- workload
WORKLOADS = ("ring24", "mixed-box", "mixed-terrain", "aerial")


def make_workload(seed=SEED, n_views=N_VIEWS, W=W_, H=H_, kind="ring24"):
    """(views, depth ranges, cleaner neighbours, matching views) per view.

    ring24: the box scene, 24 views 640x480 on a ring, 10 cleaner neighbours
    and the 6 nearest as matching views.  mixed-box / mixed-terrain: 64 views
    whose sizes are drawn from 640x480, 480x640, 640x360 and 320x240 by the
    seed, each with U{4..10} neighbours that serve as matching and cleaner
    views (rendered by the CUDA ray caster)."""
    from opensfm_b200 import synthetic as S

    if kind == "ring24":
        vs = S.ring_viewset(seed, n_views, W, H)
        cands = [vs.neighbors(v, N_CAND) for v in range(n_views)]
        matches = [c[:N_MATCH] for c in cands]
    elif kind == "aerial":
        vs = S.aerial_viewset(seed)
        cands = [vs.neighbors_by_footprint(v, N_CAND) for v in range(len(vs.cameras))]
        matches = [c[:N_MATCH] for c in cands]
    else:
        vs = S.mixed_viewset(seed, 64, kind.split("-")[1], gpu=True)
        rng = np.random.default_rng(seed + 3)
        counts = rng.integers(4, 11, size=len(vs.cameras))
        cands = [vs.neighbors(v, int(k)) for v, k in enumerate(counts)]
        matches = cands
    ranges = [S.depth_range(d) for d in vs.depths]
    return vs, ranges, cands, matches


def schedules():
    """(plain, learned candidates): the plain GPU PatchMatch, and the learned
    schedules tried in order of cost; the first whose accuracy is no lower
    than the plain method's is the headline."""
    from opensfm_b200.learned import Schedule

    plain = Schedule("plain", "plain", PLAIN_HALF_PASSES, {}, knights=PLAIN_KNIGHTS)
    learned = [Schedule(f"learned-{hp}hp-refine{nr}-active{a:g}-views{mode}"
                        + (f"-settled{seed:g}" if seed > 0 else "") + ("-fallback" if fb else ""),
                        "learned", hp, {} if nr == 6 else {"n_refine": nr}, sample=mode, active=a,
                        seed=seed, fallback=bool(fb))
               for hp, nr, a, mode, seed, fb in LEARNED_SCHEDULES]
    return plain, learned


def timed_runs(b, steps, learned, group=None):
    """Device ms of `steps` graph replays (batch stream events)."""
    if group:
        group.barrier()
    b.synchronize()
    b.timer_record(0)
    for _ in range(steps):
        b.run(prune=True, graph=True, learned=learned)
    b.timer_record(1)
    b.synchronize()
    ms = b.timer_elapsed()
    if group:
        group.barrier()
    return ms


def map_accuracy(b, vs, n_maps):
    accs = [S_accuracy(b.get_depth(v), vs.depths[v]) for v in range(n_maps)]
    return float(np.median(accs)), float(np.mean(accs))


def S_accuracy(d, gt):
    from opensfm_b200 import synthetic as S

    return S.accuracy(d, gt)


def stage_roofline(b, sched, learned, peak):
    """One instrumented run of the schedule (per-stage launches, events per
    stage; outside the timed region): stage ms, taps and the half-pass
    kernel's algorithmic FP32 throughput."""
    b.run(prune=True, graph=False, timing=True, learned=learned)
    b.synchronize()
    stages, taps = b.timings()
    hp_ms = stages[1]
    achieved = FLOPS_PER_TAP * taps[1] / (hp_ms * 1e-3) / 1e12 if hp_ms > 0 else 0.0
    return {"stage_ms": {"proposal": stages[5], "init": stages[0], "halfpasses": stages[1],
                         "post": stages[2], "clean_and_prune": stages[3], "total": stages[4]},
            "halfpass_taps": taps[1], "achieved": achieved, "frac": achieved / peak}


def fusion_leg(b, vs, cands, n_maps, repeats=3, oracle=True):
    """DepthmapFuser over the batch's cleaned depthmaps (normals from the
    PatchMatch planes, grey colours, each view checked against itself and its
    cleaner neighbours, as dense.py lists a cluster).  Times fuse() on the
    host clock, without outlier removal (the dense pipeline's setting,
    depthmap_fusion_sor_knn = 0) and with the fuser's default removal (K = 12,
    factor 2.5).  With `oracle`, the single-thread C restatement fuses the
    same views (without removal: its exact kNN is a brute force) and the two
    point clouds are compared."""
    from opensfm_b200 import pydense

    views = []
    for v in range(n_maps):
        depth, plane, score, nghbr, clean = b.get(v, clean=True)
        img = vs.images[v]
        c = vs.cameras[v]
        views.append(dict(K=c.K, R=c.R, t=c.t, depth=clean, normal=plane,
                          color=np.stack([img, img, img], -1), mask=None,
                          neighbor_ids=sorted({v} | {o for o in cands[v] if o < n_maps}),
                          primary=True))
    f = pydense.DepthmapFuser()
    for v in views:
        f.add_view(v["K"], v["R"], v["t"], v["depth"], v["normal"], v["color"], None,
                   np.array(v["neighbor_ids"]))

    def timed():
        f.fuse()  # warm-up
        ts = []
        for _ in range(repeats):
            t0 = time.perf_counter()
            res = f.fuse()
            ts.append(time.perf_counter() - t0)
        return res, float(np.median(ts))

    got_sor, t_sor = timed()  # the fuser's defaults: removal with K = 12
    removal_ms = f.last_removal_ms()
    f.set_sor_params(0, 2.5)
    got, t_plain = timed()
    out = {"points": int(len(got[0])), "fuse_s": t_plain,
           "points_after_outlier_removal": int(len(got_sor[0])), "fuse_with_removal_s": t_sor,
           "removal_device_ms": removal_ms,
           "views": n_maps, "neighbours_per_view": float(np.mean([len(v["neighbor_ids"])
                                                                  for v in views]))}
    if oracle:
        import oracle as O

        t0 = time.perf_counter()
        want = O.port_fuse(views)
        out["oracle_1thread_s"] = time.perf_counter() - t0
        out["identical_to_oracle"] = bool(all(np.array_equal(a, w) for a, w in zip(got, want)))
    out["svo"] = svo_leg(views, repeats, oracle)
    return out


ACMMP_SETTINGS = {
    # DepthmapParams' own defaults (estimator.h:17-31), 6 sources.
    "estimator_defaults": dict(n_src=6, levels=1, iterations=3, patch_size=11, top_k=4,
                               smooth=0.0, geom=0.0, sfm=False),
    # OpenSfM's dense pipeline (config.py:379-420, dense.py:608-735): 4 matching
    # views, 4 iterations, patch 5, 4 pyramid levels, smoothness 0.3, geometric
    # consistency 0.05 between the cluster's references, the SfM planar prior.
    "pipeline_defaults": dict(n_src=4, levels=4, iterations=4, patch_size=5, top_k=4,
                              smooth=0.3, geom=0.05, sfm=True),
}


def acmmp_leg(vs, cands, n_refs=4, repeats=2, oracle=True):
    """The live path's PatchMatch estimator (DepthmapClusterEstimator) on the
    first `n_refs` ring views at full size as one cluster, under its own
    defaults and under the dense pipeline's: device time and depthmaps/s.
    The SfM points for the prior are 2000 points per reference sampled on
    the ray-cast surface (as a reconstruction's tracks would be).  With
    `oracle`, the single-thread C restatement runs the same cluster at an
    eighth of the size in each axis, the GPU runs it too, and the outputs
    are compared."""
    from opensfm_b200 import pydense
    from opensfm_b200 import synthetic as S

    def surface_points(views, k, n, seed):
        rng = np.random.default_rng(seed)
        d, c = views.depths[k], views.cameras[k]
        H, W = d.shape
        ys, xs = rng.integers(0, H, n), rng.integers(0, W, n)
        dd = d[ys, xs]
        ray = np.stack([xs + rng.uniform(0, 1, n), ys + rng.uniform(0, 1, n), np.ones(n)], -1)
        Xc = (ray @ np.linalg.inv(c.K).T) * dd[:, None]
        return ((Xc - c.t) @ c.R)[dd > 0]

    def setup(views, refs, cfg, sfm_n):
        e = pydense.DepthmapClusterEstimator()
        e.set_max_iterations(cfg["iterations"])
        e.set_patch_size(cfg["patch_size"])
        e.set_top_k(cfg["top_k"])
        e.set_hierarchy_levels(cfg["levels"])
        e.set_smooth_weight(cfg["smooth"])
        e.set_geom_consistency_weight(cfg["geom"])
        oracle_refs, links = [], []
        for ref in refs:
            dmin, dmax = S.depth_range(views.depths[ref])
            c = views.cameras[ref]
            e.begin_ref_view(c.K, c.R, c.t, views.images[ref], dmin, dmax)
            pts = surface_points(views, ref, sfm_n, 100 + ref) if cfg["sfm"] else None
            if pts is not None:
                e.set_sfm_points(pts)
            srcs = list(cands[ref][:cfg["n_src"]])
            for s_ in srcs:
                cs = views.cameras[s_]
                e.add_source_view(cs.K, cs.R, cs.t, views.images[s_])
            oracle_refs.append(dict(views=[(views.cameras[i].K, views.cameras[i].R,
                                            views.cameras[i].t, views.images[i])
                                           for i in [ref] + srcs],
                                    depth_min=dmin, depth_max=dmax, sfm=pts))
        # dense.py:718-728: a reference's sources that are references too.
        for i, ref in enumerate(refs):
            srcs = list(cands[ref][:cfg["n_src"]])
            for j, other in enumerate(refs):
                if other != ref and other in srcs:
                    links.append((i, srcs.index(other), j))
                    e.add_geom_link(i, srcs.index(other), j)
        return e, oracle_refs, links

    res = {"refs": n_refs, "size": list(vs.images[0].shape[::-1])}
    for name, cfg in ACMMP_SETTINGS.items():
        e, _, _ = setup(vs, list(range(n_refs)), cfg, 2000)
        out = e.run()  # warm-up
        ms, host = [], []
        for _ in range(repeats):
            t0 = time.perf_counter()
            out = e.run()
            host.append(time.perf_counter() - t0)
            ms.append(e.last_run_ms())
        t = float(np.median(ms))
        r = dict(cfg, device_ms=t, depthmaps_per_s=n_refs / (t * 1e-3),
                 host_s=float(np.median(host)),
                 accuracy_1pct_median=float(np.median([S.accuracy(o[0], vs.depths[i])
                                                       for i, o in enumerate(out)])))
        if oracle:
            import oracle as O

            H, W = vs.images[0].shape
            small = S.ring_viewset(SEED, len(vs.images), W // 8, H // 8)
            es, orefs, links = setup(small, list(range(n_refs)), cfg, 200)
            got = es.run()
            t0 = time.perf_counter()
            want = O.port_acmmp_cluster(orefs, hierarchy_levels=cfg["levels"],
                                        iterations=cfg["iterations"],
                                        patch_size=cfg["patch_size"], top_k=cfg["top_k"],
                                        smooth_weight=cfg["smooth"], geom_weight=cfg["geom"],
                                        geom_links=links)
            r["oracle_sample"] = f"the same {n_refs}-view cluster at {W // 8}x{H // 8}"
            r["oracle_1thread_s"] = time.perf_counter() - t0
            r["sample_device_ms"] = es.last_run_ms()
            r["identical_to_oracle"] = bool(all(np.array_equal(a, b) for g, w in zip(got, want)
                                                for a, b in zip(g, w)))
        res[name] = r
    return res


def svo_leg(views, repeats=3, oracle=True, voxel_size=0.05, trunc_factor=4.0, min_weight=3.0):
    """SVOFuser (TSDF fusion) over the same views: count_voxels() + fuse()
    timed on the host clock, the device time of the fuse, and with `oracle`
    the single-thread C restatement and an identity check."""
    from opensfm_b200 import pydense

    f = pydense.SVOFuser()
    f.set_voxel_size(voxel_size)
    f.set_trunc_factor(trunc_factor)
    f.set_min_weight(min_weight)
    for v in views:
        f.add_view(v["K"], v["R"], v["t"], v["depth"], v["normal"], v["color"], None)
    f.count_voxels()
    f.fuse()  # warm-up
    ts = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        n_vox = f.count_voxels()
        got = f.fuse()
        ts.append(time.perf_counter() - t0)
    out = {"voxel_size": voxel_size, "trunc_factor": trunc_factor, "min_weight": min_weight,
           "voxels": int(n_vox), "points": int(len(got[0])), "count_and_fuse_s": float(np.median(ts)),
           "fuse_device_ms": f.last_fuse_ms()}
    if oracle:
        import oracle as O

        t0 = time.perf_counter()
        cnt, wp, wn, wc = O.port_svo([dict(v, mask=None) for v in views], voxel_size=voxel_size,
                                     trunc_factor=trunc_factor, min_weight=min_weight)
        out["oracle_1thread_s"] = time.perf_counter() - t0
        out["identical_to_oracle"] = bool(cnt == n_vox and all(
            np.array_equal(a, w) for a, w in zip(got, (wp, wn, wc))))
    return out


# ------------------------------------------------------------------ clocks
class Clocks:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, n in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


# ------------------------------------------------------------ distributed
def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(
        os.environ.get("LOCAL_RANK", 0))


class Group:
    """Barrier + max-reduce across ranks for N > 1: torch.distributed over
    NCCL between GPUs (gloo on CPU for the multi-process tests).  The
    depthmap path itself exchanges nothing: every rank is a replica."""

    def __init__(self, world, local_rank, backend="nccl"):
        self.world = world
        self.pg = None
        self.device = "cuda" if backend == "nccl" else "cpu"
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            if backend == "nccl":
                torch.cuda.set_device(local_rank)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.torch, self.dist = torch, dist
            self.pg = True

    def barrier(self):
        if self.pg:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.dist.destroy_process_group()


def replica_throughput(world: int, maps_per_rank: int, steps: int, ms_max: float) -> float:
    """Whole-job depthmaps/s: every rank processes its own reconstruction of
    maps_per_rank depthmaps per step; the job time is the slowest rank's."""
    return world * maps_per_rank * steps / (ms_max * 1e-3)


# ------------------------------------------------------------- CPU legs
def _ref_band(task):
    """Reference PatchMatch on rows [r0, r0 + rows) of one reference view."""
    import oracle as O

    (K, R, t, img, nbrs, r0, rows, mn, mx, hpz) = task
    H, W = img.shape
    top = max(r0 - hpz, 0)
    bot = min(r0 + rows + hpz, H)
    Kc = K.copy()
    Kc[1, 2] -= top
    e = O.RefEstimator() if O.ref_available() else None
    t0 = time.perf_counter()
    if e is not None:
        crop = np.ascontiguousarray(img[top:bot])
        e.add_view(Kc, R, t, crop, np.ones_like(crop))
        for (Kn, Rn, tn, imn) in nbrs:
            # Matching views keep their full extent (the reference samples
            # each view with its own size, depthmap.cc:472).
            e.add_view(Kn, Rn, tn, imn, np.ones_like(imn))
        e.set_depth_range(mn, mx, 50)
        e.set_patch_size(PATCH)
        e.set_min_patch_sd(MIN_SD)
        e.set_patchmatch_iterations(ITERS)
        e.compute_patch_match()
        kind = "reference"
    else:
        crop = np.ascontiguousarray(img[top:bot])
        Ks = [Kc] + [n[0].copy() for n in nbrs]
        for k in Ks[1:]:
            k[1, 2] -= top
        O.port_compute(1, Ks, [R] + [n[1] for n in nbrs], [t] + [n[2] for n in nbrs],
                       [crop] + [np.ascontiguousarray(n[3][top:bot]) for n in nbrs],
                       [np.ones_like(crop)] * (1 + len(nbrs)), PATCH, mn, mx, 50, ITERS, MIN_SD, 1)
        kind = "port"
    dt = time.perf_counter() - t0
    interior = (bot - top - 2 * hpz) * (W - 2 * hpz)
    return interior, dt, kind


def cpu_model() -> str:
    """The host CPU's model name (first /proc/cpuinfo entry)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _ref_whole_map(task):
    """Reference PatchMatch (ComputePatchMatch, depthmap.cc:202-213) on one
    whole reference view with its matching views: (depth, plane, seconds,
    kind)."""
    import oracle as O

    (Ks, Rs, ts, imgs, mn, mx, seed) = task
    t0 = time.perf_counter()
    masks = [np.ones_like(im) for im in imgs]
    if O.ref_available():
        O.ref().ref_srand(seed)
        e = O.RefEstimator()
        for K, R, t, im, mk in zip(Ks, Rs, ts, imgs, masks):
            e.add_view(K, R, t, im, mk)
        e.set_depth_range(mn, mx, 50)
        e.set_patch_size(PATCH)
        e.set_min_patch_sd(MIN_SD)
        e.set_patchmatch_iterations(ITERS)
        depth, plane, _, _ = e.compute_patch_match()
        kind = "reference"
    else:
        depth, plane, _, _ = O.port_compute(1, Ks, Rs, ts, imgs, masks, PATCH, mn, mx, 50, ITERS,
                                            MIN_SD, seed)
        kind = "port"
    return depth, plane, time.perf_counter() - t0, kind


def _ref_clean_map(task):
    """Reference DepthmapCleaner::Clean (depthmap.cc:524-555) of one map."""
    import oracle as O

    Ks, Rs, ts, depths = task
    if O.ref_available():
        return O.ref_clean(Ks, Rs, ts, depths, 0.01, 3)
    return O.port_clean(Ks, Rs, ts, depths, 0.01, 3)


def _ref_prune_map(task):
    """Reference DepthmapPruner::Prune (depthmap.cc:577-637) of one map: its
    point count."""
    import oracle as O

    Ks, Rs, ts, depths, planes, colors, labels = task
    fn = O.ref_prune if O.ref_available() else O.port_prune
    return len(fn(Ks, Rs, ts, depths, planes, colors, labels, 0.01)[3])


def reference_reconstruction(work, cores=None, seed=0):
    """The reference's CPU path over the whole reconstruction: every depthmap
    (whole 640 x 480 views, ComputePatchMatch) distributed over the host's
    cores, one process per core, then DepthmapCleaner and DepthmapPruner of
    every map against its cleaner neighbours, as the GPU arm runs them.
    Returns depthmaps/s over the wall time of all three stages, the stage
    seconds, the reference's accuracy and the pruned point count."""
    from opensfm_b200 import synthetic as S

    vs, ranges, cands, matches = work
    n = len(vs.cameras)
    cores = cores or os.cpu_count() or 1
    cam = vs.cameras

    def pm_task(v):
        ids = [v] + list(matches[v])
        return ([cam[k].K for k in ids], [cam[k].R for k in ids], [cam[k].t for k in ids],
                [vs.images[k] for k in ids], ranges[v][0], ranges[v][1], 1000 + seed * 100 + v)

    ctx = mp.get_context("spawn")
    with ctx.Pool(min(cores, n)) as pool:
        pool.map(_ref_clean_map, [([cam[0].K], [cam[0].R], [cam[0].t],
                                   [np.zeros((8, 8), np.float32)])] * min(cores, n))  # start-up
        t0 = time.perf_counter()
        pm = pool.map(_ref_whole_map, [pm_task(v) for v in range(n)], chunksize=1)
        t1 = time.perf_counter()
        depth = [r[0] for r in pm]
        plane = [r[1] for r in pm]
        clean = pool.map(_ref_clean_map, [
            ([cam[k].K for k in [v] + cands[v]], [cam[k].R for k in [v] + cands[v]],
             [cam[k].t for k in [v] + cands[v]], [depth[k] for k in [v] + cands[v]])
            for v in range(n)], chunksize=1)
        t2 = time.perf_counter()
        gray3 = [np.repeat(im[..., None], 3, axis=2) for im in vs.images]
        zeros = [np.zeros_like(im) for im in vs.images]
        counts = pool.map(_ref_prune_map, [
            tuple([[x[k] for k in [v] + cands[v]] for x in (
                [c.K for c in cam], [c.R for c in cam], [c.t for c in cam], clean, plane, gray3,
                zeros)]) for v in range(n)], chunksize=1)
        t3 = time.perf_counter()
    accs = [S.accuracy(depth[v], vs.depths[v]) for v in range(n)]
    return {"value": n / (t3 - t0), "unit": UNIT, "cores": min(cores, n), "kind": pm[0][3],
            "stage_s": {"patchmatch": t1 - t0, "clean": t2 - t1, "prune": t3 - t2},
            "map_s_median": float(np.median([r[2] for r in pm])),
            "accuracy_1pct_median": float(np.median(accs)),
            "accuracy_1pct_mean": float(np.mean(accs)),
            "pruned_points": int(sum(counts)), "cpu_model": cpu_model(),
            "sample": f"the whole reconstruction: {n} depthmaps of "
                      f"{vs.images[0].shape[1]}x{vs.images[0].shape[0]} (whole views, "
                      f"{N_MATCH} matching views, PatchMatch {ITERS} iterations, raster schedule) "
                      f"over {min(cores, n)} processes, then DepthmapCleaner (0.01, 3 views) and "
                      f"DepthmapPruner (0.01) of every map against its {N_CAND} neighbours; "
                      f"{t3 - t0:.1f} s wall"}


def cpu_sample(work, seconds=20.0, cores=None, seed=0):
    """Times the reference CPU path on bands of the workload, all cores.

    Returns depthmaps/s (band pixels per second over the pixels of one
    640 x 480 depthmap's interior), cores used, kind and a description.
    """
    vs, ranges, cands, matches = work
    cores = cores or os.cpu_count() or 1
    hpz = (PATCH - 1) // 2
    H, W = vs.images[0].shape
    rng = np.random.default_rng(seed)

    def task(v, r0, rows):
        c = vs.cameras[v]
        nb = [(vs.cameras[o].K, vs.cameras[o].R, vs.cameras[o].t, vs.images[o]) for o in matches[v]]
        return (c.K, c.R, c.t, vs.images[v], nb, r0, rows, ranges[v][0], ranges[v][1], hpz)

    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        # Calibrate the per-pixel cost on one small band per worker.
        cal_rows = 4
        cal = pool.map(_ref_band, [task(int(rng.integers(N_VIEWS)), int(rng.integers(hpz, H - 40)),
                                        cal_rows) for _ in range(cores)])
        px_per_s = sum(c[0] for c in cal) / sum(c[1] for c in cal)
        rows = int(max(2, min(H - 2 * hpz, seconds * px_per_s / (W - 2 * hpz))))
        tasks = []
        for k in range(cores):
            v = int(rng.integers(N_VIEWS))
            r0 = int(rng.integers(hpz, max(hpz + 1, H - hpz - rows)))
            tasks.append(task(v, r0, rows))
        t0 = time.perf_counter()
        res = pool.map(_ref_band, tasks)
        wall = time.perf_counter() - t0
    pixels = sum(r[0] for r in res)
    per_map = (W - 2 * hpz) * (H - 2 * hpz)
    value = pixels / per_map / wall
    kind = res[0][2]
    return {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{cores} bands of {rows} rows x {W} px of the 24 reference views "
                      f"({pixels} interior px, {pixels / per_map:.3f} depthmaps) in {wall:.1f} s, "
                      f"one process per core; PatchMatch 3 iterations, 6 matching views, "
                      f"patch 7 (reference view cropped to the band, matching views whole)"}


# ----------------------------------------------------------------- our arm
def build_batch(work, seed=1, n_maps=None):
    from opensfm_b200 import pydense

    vs, ranges, cands, matches = work
    n_maps = n_maps or len(vs.cameras)
    b = pydense.Batch()
    for c, im in zip(vs.cameras, vs.images):
        b.add_view(c.K, c.R, c.t, im)
    for v in range(n_maps):
        b.add_depthmap(v, matches[v], ranges[v][0], ranges[v][1])
    for v in range(n_maps):
        b.set_clean_views(v, [o for o in cands[v] if o < n_maps])
    b.set_params(patch_size=PATCH, min_patch_sd=MIN_SD, iterations=ITERS,
                 same_depth_threshold=0.01, min_consistent_views=3, seed=seed)
    return b


def mixed_leg(kind, learned_scheds=()):
    """Config 3: 64 views of mixed sizes (box or terrain).  The plain
    schedule runs every depthmap with its cleaner and pruner in one
    persistent cooperative launch replayed from a CUDA graph.  The learned
    schedules (one view per candidate, so per-stage launches; the network
    runs once per image size in the batch) are tried in their order, and the
    first whose accuracy is no lower than plain's (median and mean) is
    reported, with every one tried.  Device-timed over 3 replays."""
    from opensfm_b200 import learned as LN

    work = make_workload(kind=kind)
    vs, ranges, cands, matches = work
    b = build_batch(work)
    b.set_tuning(32, 4, 18)  # 2 lanes per pixel, persistent launch (+16)
    plain, _ = schedules()
    out = {"views": len(vs.cameras), "sizes": {}}
    for h, w in (im.shape for im in vs.images):
        out["sizes"][f"{w}x{h}"] = out["sizes"].get(f"{w}x{h}", 0) + 1
    if learned_scheds:
        LN.install(LN.ProposalNet.load(), b)
    tried = []
    for sch in [plain] + list(learned_scheds):
        is_l = sch.init == "learned"
        sch.apply(b)
        b.run(prune=True, graph=True, learned=is_l)
        b.synchronize()
        ms = timed_runs(b, 3, is_l) / 3
        acc = map_accuracy(b, vs, len(vs.cameras))
        res = {"schedule": sch.name, "value": len(vs.cameras) / (ms * 1e-3), "ms_per_step": ms,
               "accuracy_1pct_median": acc[0], "accuracy_1pct_mean": acc[1],
               "pruned_points": b.pruned_count()}
        if not is_l:
            out["plain"] = res
            continue
        res["equal_accuracy"] = (acc[0] >= out["plain"]["accuracy_1pct_median"]
                                 and acc[1] >= out["plain"]["accuracy_1pct_mean"])
        tried.append(res)
        if res["equal_accuracy"]:
            break
    if tried:
        ok = [r for r in tried if r["equal_accuracy"]]
        out["learned"] = dict(ok[0] if ok else tried[-1])
        out["learned_over_plain"] = out["learned"]["value"] / out["plain"]["value"]
        out["learned_schedules_tried"] = [{k: r[k] for k in ("schedule", "ms_per_step",
                                           "accuracy_1pct_median", "accuracy_1pct_mean",
                                           "equal_accuracy")} for r in tried]
    b.close()
    return out


def run_ours(args):
    rank, world, local = dist_env()
    from opensfm_b200 import _lib, pydense
    from opensfm_b200 import learned as LN

    group = Group(world, local)
    _lib.check(_lib.load().dn_set_device(local))
    work = make_workload(kind=args.workload)
    vs, ranges, cands, matches = work
    n_maps = args.maps or len(vs.cameras)
    shapes = [im.shape for im in vs.images]
    ring = args.workload == "ring24"
    b = build_batch(work, n_maps=n_maps)
    plain, learned_scheds = schedules()
    plain.apply(b)
    tuning = None
    if args.tuning:
        bx, by, var = (int(x) for x in args.tuning.split(","))
        b.set_tuning(bx, by, var)
        tuning = {"choice": [bx, by, var], "source": "--tuning"}
    else:
        from opensfm_b200 import autotune

        key = autotune.workload_key(shapes[:n_maps], [len(m) for m in matches[:n_maps]], PATCH)
        tune_cands = autotune.CANDIDATES
        if args.workload == "aerial":  # a step takes seconds: the two leading choices only
            tune_cands = [(32, 4, 2), (32, 4, 18)]
        t = autotune.tune(b, key, {"prune": True, "graph": True}, candidates=tune_cands)
        tuning = {"choice": list(t["choice"]), "ms": t["ms"], "cached": t["cached"],
                  "source": "opensfm_b200.autotune"}
    choice = tuning["choice"]
    peak = pydense.fp32_peak()
    walk_ceiling = pydense.walk_ceiling()  # G taps/s of the table walk alone

    def leg(sch, learned, choice):
        """Warm-up, one instrumented run (per-stage launches), accuracy, then
        the K timed graph replays, with the launch tuning `choice`."""
        b.set_tuning(*choice)
        sch.apply(b)
        for _ in range(args.warmup):
            b.run(prune=True, graph=True, learned=learned)
        b.synchronize()
        if choice[2] & 16:  # stage events need one launch per stage
            b.set_tuning(choice[0], choice[1], choice[2] & 15)
        roof = stage_roofline(b, sch, learned, peak)
        if choice[2] & 16:
            b.set_tuning(*choice)
            b.run(prune=True, graph=True, learned=learned)
        b.synchronize()
        acc = map_accuracy(b, vs, n_maps)
        ms = group.max(timed_runs(b, args.steps, learned, group))
        return {"schedule": sch.name, "half_passes": sch.half_passes,
                "candidate_views": ["all", "one per candidate after a full initialisation",
                                    "one per candidate (ComputePatchMatchSample)"][sch.sample],
                "refinements": sch.kw.get("n_refine", 6),
                "knight_moves": sch.knights, "active_pixels": sch.active,
                "settled_start_score": sch.seed, "init_fallback": sch.fallback,
                "value": replica_throughput(world, n_maps, args.steps, ms),
                "ms_per_step": ms / args.steps, "accuracy_1pct_median": acc[0],
                "accuracy_1pct_mean": acc[1], "pruned_points": b.pruned_count(), **roof}

    # Plain GPU PatchMatch (random initialisation, every view per candidate).
    with Clocks(local) as clk_plain:
        plain_res = leg(plain, False, choice)
    head, head_learned, clk = plain_res, False, clk_plain
    learned_res, tried = None, []
    choice_l = choice
    if len({tuple(sh) for sh in shapes[:n_maps]}) == 1:  # one image size (ring24, aerial)
        LN.install(LN.ProposalNet.load(), b)
        # The cheapest learned schedule whose accuracy is no lower than plain's
        # (medians and means over the maps), from one graph replay each.
        pick = learned_scheds[-1]
        for sch in learned_scheds:
            sch.apply(b)
            b.run(prune=True, graph=True, learned=True)
            b.synchronize()
            ms = timed_runs(b, 2, True) / 2
            acc = map_accuracy(b, vs, n_maps)
            ok = acc[0] >= plain_res["accuracy_1pct_median"] and acc[1] >= plain_res["accuracy_1pct_mean"]
            tried.append({"schedule": sch.name, "ms": ms, "accuracy_1pct_median": acc[0],
                          "accuracy_1pct_mean": acc[1], "equal_accuracy": ok})
            if ok:
                pick = sch
                break
        # The learned schedule's own launch tuning (one view per candidate
        # runs shorter evaluations than the plain schedule; per-stage
        # launches, as one view per candidate is not in the persistent
        # launch).
        choice_l = choice
        if not args.tuning:
            from opensfm_b200 import autotune

            pick.apply(b)
            key_l = autotune.workload_key(shapes[:n_maps], [len(m) for m in matches[:n_maps]],
                                          PATCH) + ":learned:" + pick.name
            t_l = autotune.tune(b, key_l, {"prune": True, "graph": True, "learned": True},
                                candidates=[c for c in autotune.CANDIDATES if not c[2] & 16])
            choice_l = tuple(t_l["choice"])
            tuning["learned"] = {"choice": list(choice_l), "ms": t_l["ms"],
                                 "cached": t_l["cached"]}
        with Clocks(local) as clk_learned:
            learned_res = leg(pick, True, choice_l)
        learned_res["equal_accuracy"] = (
            learned_res["accuracy_1pct_median"] >= plain_res["accuracy_1pct_median"]
            and learned_res["accuracy_1pct_mean"] >= plain_res["accuracy_1pct_mean"])
        head, head_learned, clk = learned_res, True, clk_learned
        head_sched = pick
        # The same schedule from the reference's random initialisation: what
        # the schedule gives without the proposal network.
        from opensfm_b200.learned import Schedule

        same = Schedule("plain-init-" + pick.name, "plain", pick.half_passes, dict(pick.kw),
                        sample=pick.sample, active=pick.active, knights=pick.knights,
                        seed=pick.seed, fallback=pick.fallback)
        same.apply(b)
        b.run(prune=True, graph=True)
        b.synchronize()
        ms = timed_runs(b, max(2, args.steps // 4), False) / max(2, args.steps // 4)
        acc = map_accuracy(b, vs, n_maps)
        plain_same = {"schedule": same.name, "value": n_maps / (ms * 1e-3), "ms_per_step": ms,
                      "accuracy_1pct_median": acc[0], "accuracy_1pct_mean": acc[1]}
    else:
        head_sched = plain
        plain_same = None

    # End to end through the public batch API from pinned host buffers: every
    # step uploads the images, runs the headline schedule, and reads every
    # final depth back.
    import torch

    def pinned(a):
        t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype))).pin_memory()
        t.numpy()[...] = a
        return t

    b.set_tuning(*(choice_l if head_learned else choice))
    head_sched.apply(b)
    b.run(prune=True, graph=True, learned=head_learned)
    keep = [pinned(np.ascontiguousarray(im)) for im in vs.images[:n_maps]]
    imgs = [t.numpy() for t in keep]
    # Two sets of host outputs, alternating: a step's readback may still be
    # in flight while the next one is enqueued.
    keep += [pinned(np.zeros(sh, np.float32)) for _ in range(2) for sh in shapes[:n_maps]]
    out_sets = [[t.numpy() for t in keep[n_maps * (1 + k):n_maps * (2 + k)]] for k in range(2)]
    outs = out_sets[0]
    map_ids = list(range(n_maps))
    group.barrier()
    b.synchronize()
    # Pipelined through the batch's I/O streams: each step's uploads run while
    # the previous step's run executes, and its readback while the next run
    # executes (upload_view_image / get_depths_async keep the stream order);
    # the end timer waits for the last readback.
    b.timer_record(0)
    for step in range(args.steps):
        for v, im in enumerate(imgs):
            b.upload_view_image(v, im)
        b.run(prune=True, graph=True, learned=head_learned)
        b.get_depths_async(map_ids, out_sets[step % 2], clean=True)
    b.timer_record(1)
    b.synchronize()
    e2e_ms = group.max(b.timer_elapsed())
    group.barrier()
    e2e = replica_throughput(world, n_maps, args.steps, e2e_ms)
    # The pipelined readback of the last step is the batch's result (checked
    # after the timed region against a synchronous fetch).
    e2e_same = all(np.array_equal(o, d) for o, d in
                   zip(out_sets[(args.steps - 1) % 2], b.get_depths(map_ids, clean=True)))

    if ring:
        desc = (f"ring reconstruction, {n_maps} reference views {W_}x{H_}, "
                f"{N_MATCH} matching views, {N_CAND} cleaner neighbours, PatchMatch "
                f"{ITERS} iterations, patch {PATCH}, min_patch_sd {MIN_SD}, "
                f"cleaner 0.01 / 3 views, pruner 0.01")
    elif args.workload == "aerial":
        desc = (f"aerial block: terrain 300x300 m with 40 buildings, {n_maps} reference views "
                f"1280x960 (128 nadir + 128 at 45 deg, 60 m), {N_MATCH} matching views, "
                f"{N_CAND} cleaner neighbours (nearest footprints, similar directions), "
                f"PatchMatch {ITERS} iterations, patch {PATCH}, cleaner 0.01 / 3 views, "
                f"pruner 0.01")
    else:
        sizes = {}
        for h, w in shapes[:n_maps]:
            sizes[f"{w}x{h}"] = sizes.get(f"{w}x{h}", 0) + 1
        desc = (f"{args.workload}: {n_maps} depthmaps of mixed sizes {sizes}, "
                f"{min(len(m) for m in matches)}-{max(len(m) for m in matches)} matching "
                f"(and cleaner) views, PatchMatch {ITERS} iterations, patch {PATCH}, "
                f"min_patch_sd {MIN_SD}, cleaner 0.01 / 3 views, pruner 0.01; "
                f"{sum(h * w for h, w in shapes[:n_maps]) / 1e6:.2f} Mpx per step")
    head_choice = choice_l if head_learned else choice
    hp_gtaps = head["halfpass_taps"] / (head["stage_ms"]["halfpasses"] * 1e-3) / 1e9
    hp_variant = head_choice[2] & 15
    line = {
        "metric": METRIC if ring else (
            "1280px depthmaps/s (256-view aerial block, 6 views, 3 iters, cleaner + pruner)"
            if args.workload == "aerial" else
            "depthmaps/s (64 mixed-size views, 4-10 matching views, 3 iters, cleaner + pruner)"),
        "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {
            "workload": desc,
            "init": "learned" if head_learned else "plain",
            "global_batch": n_maps * world, "parallelism": f"replicas x{world}",
            "tuning": tuning,
            "l2": "working set larger than L2 (views, tables and state ~%.0f MB)" % (
                sum((w + 15) * (h + 15) * 8 + w * h * (16 + 4 + 4 + 4 + 4 + 2)
                    for h, w in shapes[:n_maps]) / 1e6),
            "plain": plain_res,
            "learned": learned_res,
            "learned_schedules_tried": tried,
            "plain_init_same_schedule": plain_same,
            "learned_over_plain": (learned_res["value"] / plain_res["value"]) if learned_res else None,
            "equal_accuracy": learned_res["equal_accuracy"] if learned_res else None,
        },
        "roofline": {
            "kernel": "halfpass_kernel<3,%s,%d>" % (
                "true" if head_sched.sample else "false", hp_variant),
            "bound": "fp32", "achieved": head["achieved"], "peak": peak, "unit": "TFLOP/s",
            "frac": head["frac"],
            # DRAM bytes (read + write) of one tile half-pass over every pixel
            # of a colour, from the ncu capture of this workload at tuning
            # 32,4,2 (not measured inside the bench).
            "traffic": ((TRAFFIC_SETTLED_LIST if head_sched.seed > 0 else TRAFFIC_SAMPLE_TILE)
                        if head_sched.sample else TRAFFIC_PLAIN_TILE)
            if ring and n_maps == len(vs.cameras) else None,
            "traffic_source": "ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of one "
                              "half-pass, 24 x 640x480: the first list half-pass with a settled "
                              "start, else a tile half-pass over every pixel of a colour "
                              "(profiles/halfpass_sample_and_list_ring24_640x480.md); later "
                              "list half-passes move less",
            "peak_source": "measured FP32 FMA loop on this GPU (dn_fp32_peak); "
                           "MEASURED_PEAKS.json has no FP32 figure",
            "walk_ceiling": {
                "gtaps_s": walk_ceiling,
                "halfpass_gtaps_s": hp_gtaps,
                "frac": hp_gtaps / walk_ceiling,
                "source": "dn_walk_ceiling: 7x7 affine walks through the FP16 coefficient "
                          "table with the production sampler and the three NCC sums alone, one "
                          "thread per pixel of a 1024x768 view (measured on this GPU)"},
            "algorithmic": f"{FLOPS_PER_TAP} flops per NCC tap x {head['halfpass_taps']} taps "
                           f"in {head_sched.half_passes} half-passes "
                           f"({head['stage_ms']['halfpasses']:.2f} ms)",
        },
        "e2e": {"value": e2e, "unit": UNIT,
                "h2d_bytes_per_step": int(sum(im.nbytes for im in imgs[:n_maps])),
                "d2h_bytes_per_step": int(sum(o.nbytes for o in outs)),
                "io": "pipelined (upload_view_image / get_depths_async on the batch's upload and readback streams)",
                "result_matches_sync_fetch": e2e_same},
        "gpu_launches": None,
        "clocks": {k: v for k, v in clk.summary().items()},
    }
    # Kernel launches per step: the learned proposal (sweep, 6 network
    # layers, plane install), then init + half-passes + post, one cleaner
    # launch and three pruner launches over all maps -- or, with the
    # persistent choice, one launch for all of PatchMatch, cleaner and pruner.
    # An active half-pass is five launches (the per-tile counts, their scan
    # per map, the pixel lists, the chunk offsets and the half-pass over the
    # lists): from the third on, or from the first with a settled start.
    n_groups = len({tuple(sh) for sh in shapes[:n_maps]})
    prop = (1 + 6 * n_groups + 1) if head_learned else 0
    hp = head_sched.half_passes
    first = 0 if head_sched.seed > 0 else min(hp, 2)
    hp_launches = first + 5 * (hp - first) if head_sched.active else hp
    pm = 1 if (head_choice[2] & 16 and not head_sched.sample) else (1 + hp_launches + 1 + 1 + 3)
    line["gpu_launches"] = args.steps * (prop + pm)
    if ring and not args.no_mixed:
        line["config"]["mixed_size_batches"] = {
            k: mixed_leg(k, learned_scheds if head_learned else ())
            for k in ("mixed-box", "mixed-terrain")}
    if args.fuse:
        line["config"]["fusion"] = fusion_leg(b, vs, cands, n_maps)
    if args.acmmp:
        line["config"]["acmmp"] = acmmp_leg(vs, cands)
    if rank == 0 and world == 1 and not args.no_cpu and ring:
        try:
            line["cpu_baseline"] = cpu_sample(work, seconds=args.cpu_seconds)
        except Exception as e:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    group.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    import oracle as O

    work = make_workload()
    # Warm-up: W short bands of one view (library start-up, page-in), untimed.
    for k in range(args.warmup):
        cpu_sample(work, seconds=1.0, cores=1, seed=k)
    r = reference_reconstruction(work, seed=0)
    value = r["value"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 / value if value else None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": f"ring reconstruction, {N_VIEWS} reference views {W_}x{H_}, "
                               f"{N_MATCH} matching views, PatchMatch {ITERS} iterations "
                               f"(raster), patch {PATCH}, min_patch_sd {MIN_SD}, then "
                               f"DepthmapCleaner (0.01, 3 views) and DepthmapPruner (0.01) over "
                               f"{N_CAND} neighbours; whole maps, one process per core",
                   "timed": "one whole reconstruction (all maps, cleaner and pruner); a step is "
                            "one depthmap of it",
                   "reference_code": "opensfm/src/lib/dense/src/depthmap.cc (oracle/_ref)"
                   if O.ref_available() else "C restatement (oracle/_build)",
                   "accuracy_1pct_median": r["accuracy_1pct_median"],
                   "accuracy_1pct_mean": r["accuracy_1pct_mean"],
                   "stage_s": r["stage_s"], "map_s_median": r["map_s_median"],
                   "pruned_points": r["pruned_points"], "cpu_model": r["cpu_model"],
                   "same_config": True},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                         "sample": r["sample"], "cpu_model": r["cpu_model"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--tuning", default="", help="bx,by,variant (default: library default)")
    ap.add_argument("--maps", type=int, default=0,
                    help="depthmaps per step (default: all; smaller for profiling)")
    ap.add_argument("--workload", default="ring24", choices=WORKLOADS,
                    help="ring24 (640x480, the headline configuration), 64 mixed-size views "
                         "of the box or terrain scene, or the 256-view 1280x960 aerial block")
    ap.add_argument("--fuse", action="store_true",
                    help="also time DepthmapFuser on the cleaned maps against its C oracle")
    ap.add_argument("--acmmp", action="store_true",
                    help="also time the live path's PatchMatch estimator (DepthmapClusterEstimator)")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the two 64-view mixed-size batches of the default run")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
