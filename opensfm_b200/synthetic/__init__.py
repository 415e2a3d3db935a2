"""Seeded synthetic scenes with ray-cast views and ground-truth depth.

The reference ships no rendered test data for its dense path (its synthetic
generator in ``opensfm/synthetic_data`` produces cameras and tracks only), so
this module produces the inputs every parity test and benchmark uses:

* ``box_scene``: ground plane z = 0 plus axis-aligned boxes (footprint
  U[1, 4] m, height U[0.5, 3] m) in a 20 x 20 m area;
* ``terrain_scene``: a gradient-noise heightfield (amplitude in metres over a
  square area), optionally with boxes standing on it;
* ``ring_cameras`` / ``nadir_cameras``: pinhole cameras (f = 0.85 * width) on
  a ring aimed at the centre, or on a nadir grid with given overlaps;
* ``render``: uint8 grayscale image and float32 ground-truth depth (z_cam, 0
  where the ray escapes) for one camera.

Cameras follow OpenSfM's convention ``x_cam = R X + t``, ``q ~ K x_cam``.
The ray caster is plain C (``raycast.c``) driven through ctypes; rows are
split over host threads.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "raycast.c")
_LIB_PATH = os.path.join(_HERE, "_build", "libraycast.so")
_lib = None


def build(force: bool = False) -> str:
    """Compiles the ray caster (gcc) next to its source."""
    if force or not os.path.exists(_LIB_PATH) or (
        os.path.getmtime(_LIB_PATH) < os.path.getmtime(_SRC)
    ):
        os.makedirs(os.path.dirname(_LIB_PATH), exist_ok=True)
        subprocess.check_call(
            ["gcc", "-O2", "-fPIC", "-shared", "-o", _LIB_PATH, _SRC, "-lm"]
        )
    return _LIB_PATH


_GPU_SRC = os.path.join(_HERE, "raycast_gpu.cu")
_GPU_LIB = os.path.join(_HERE, "_build", "libraycast_gpu.so")
_glib = None


def build_gpu(force: bool = False) -> str:
    """Compiles the CUDA ray caster (sm_100a) next to its source."""
    if force or not os.path.exists(_GPU_LIB) or (
        os.path.getmtime(_GPU_LIB) < os.path.getmtime(_GPU_SRC)
    ):
        os.makedirs(os.path.dirname(_GPU_LIB), exist_ok=True)
        subprocess.check_call(["/usr/local/cuda/bin/nvcc", "-gencode",
                               "arch=compute_100a,code=sm_100a", "-O3", "-Xcompiler", "-fPIC",
                               "-shared", "-o", _GPU_LIB, _GPU_SRC])
    return _GPU_LIB


def _load_gpu():
    global _glib
    if _glib is None:
        lib = ctypes.CDLL(build_gpu())
        d = ctypes.c_void_p
        lib.rcg_render.argtypes = [
            d, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double,
            ctypes.c_double, ctypes.c_uint32, ctypes.c_int, ctypes.c_uint32, ctypes.c_double,
            ctypes.c_int, ctypes.c_double, ctypes.c_double, d, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, d, d, d]
        lib.rcg_render.restype = ctypes.c_int
        _glib = lib
    return _glib


def render_gpu(scene: "Scene", cams, supersample: int = 2):
    """Ray-casts views on the current CUDA device (torch tensors on 'cuda').

    Returns (images uint8 (n, H, W), depths float32 (n, H, W)) as torch CUDA
    tensors.  All cameras must share one size.
    """
    import torch

    lib = _load_gpu()
    W, H = cams[0].width, cams[0].height
    n = len(cams)
    cam = np.concatenate([np.concatenate([c.K.ravel(), c.R.ravel(), c.t.ravel()]) for c in cams])
    dcam = torch.from_numpy(cam.astype(np.float64)).cuda()
    boxes = scene.boxes.reshape(-1) if scene.boxes.size else np.zeros(6)
    dbox = torch.from_numpy(np.ascontiguousarray(boxes, np.float64)).cuda()
    imgs = torch.empty((n, H, W), dtype=torch.uint8, device="cuda")
    deps = torch.empty((n, H, W), dtype=torch.float32, device="cuda")
    st = lib.rcg_render(dbox.data_ptr(), int(scene.boxes.shape[0]), int(scene.ground),
                        float(scene.ground_half), int(scene.terrain), scene.terrain_amp,
                        scene.terrain_scale, scene.terrain_seed, scene.terrain_octaves,
                        scene.tex_seed, scene.tex_freq, scene.tex_octaves, scene.contrast,
                        scene.sky, dcam.data_ptr(), n, W, H, supersample, imgs.data_ptr(),
                        deps.data_ptr(), torch.cuda.current_stream().cuda_stream)
    if st != 0:
        raise RuntimeError(f"rcg_render failed with CUDA error {st}")
    return imgs, deps


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(build())
        d = ctypes.POINTER(ctypes.c_double)
        lib.rc_render.argtypes = [
            d, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
            ctypes.c_uint32, ctypes.c_int, ctypes.c_uint32, ctypes.c_double, ctypes.c_int,
            ctypes.c_double, ctypes.c_double, d, d, d, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_int,
            ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(ctypes.c_float),
        ]
        lib.rc_render.restype = ctypes.c_int
        _lib = lib
    return _lib


@dataclass
class Scene:
    boxes: np.ndarray  # (n, 6) float64: xmin, ymin, zmin, xmax, ymax, zmax
    ground: bool = True
    ground_half: float = 0.0
    terrain: bool = False
    terrain_amp: float = 0.0
    terrain_scale: float = 1.0
    terrain_seed: int = 0
    terrain_octaves: int = 4
    tex_seed: int = 1
    tex_freq: float = 2.0
    tex_octaves: int = 4
    contrast: float = 1.6
    sky: float = 0.8
    center: np.ndarray = field(default_factory=lambda: np.zeros(3))
    extent: float = 20.0


@dataclass
class Camera:
    K: np.ndarray  # (3, 3) float64
    R: np.ndarray  # (3, 3) float64
    t: np.ndarray  # (3,) float64
    width: int
    height: int

    @property
    def center(self) -> np.ndarray:
        return -self.R.T @ self.t


def box_scene(seed: int, n_boxes: int = 12, area: float = 20.0) -> Scene:
    """Ground plane plus ``n_boxes`` boxes, footprint U[1,4] m, height U[0.5,3] m."""
    rng = np.random.default_rng(seed)
    boxes = np.zeros((n_boxes, 6))
    for b in range(n_boxes):
        sx, sy = rng.uniform(1.0, 4.0, size=2)
        h = rng.uniform(0.5, 3.0)
        cx, cy = rng.uniform(-area / 2 + sx / 2, area / 2 - sx / 2), rng.uniform(
            -area / 2 + sy / 2, area / 2 - sy / 2
        )
        boxes[b] = [cx - sx / 2, cy - sy / 2, 0.0, cx + sx / 2, cy + sy / 2, h]
    return Scene(
        boxes=boxes, ground=True, ground_half=area, tex_seed=int(rng.integers(1, 2**31)),
        center=np.array([0.0, 0.0, 0.5]), extent=area,
    )


def terrain_scene(seed: int, size: float = 100.0, amp: float = 8.0, n_buildings: int = 0) -> Scene:
    """Gradient-noise heightfield of the given amplitude over size x size m."""
    rng = np.random.default_rng(seed)
    boxes = np.zeros((n_buildings, 6))
    s = Scene(
        boxes=boxes, ground=False, terrain=True, terrain_amp=amp, terrain_scale=size / 4.0,
        terrain_seed=int(rng.integers(1, 2**31)), terrain_octaves=4,
        tex_seed=int(rng.integers(1, 2**31)), tex_freq=1.0, center=np.zeros(3), extent=size,
    )
    if n_buildings:
        # Buildings stand on the terrain: base at the lowest corner height.
        lib_scene_probe = s
        for b in range(n_buildings):
            sx, sy = rng.uniform(6.0, 20.0, size=2)
            h = rng.uniform(4.0, 20.0)
            cx, cy = rng.uniform(-size / 2 + 15, size / 2 - 15, size=2)
            base = -amp - 1.0
            boxes[b] = [cx - sx / 2, cy - sy / 2, base, cx + sx / 2, cy + sy / 2, h]
        lib_scene_probe.boxes = boxes
    return s


def look_at(center: np.ndarray, target: np.ndarray, up=(0.0, 0.0, 1.0)) -> Tuple[np.ndarray, np.ndarray]:
    """R, t for a camera at ``center`` looking at ``target`` (x right, y down)."""
    f = np.asarray(target, float) - np.asarray(center, float)
    f /= np.linalg.norm(f)
    up = np.asarray(up, float)
    r = np.cross(f, up)
    if np.linalg.norm(r) < 1e-9:
        r = np.cross(f, np.array([0.0, 1.0, 0.0]))
    r /= np.linalg.norm(r)
    d = np.cross(f, r)
    R = np.stack([r, d, f])
    t = -R @ np.asarray(center, float)
    return R, t


def intrinsics(width: int, height: int, focal_ratio: float = 0.85) -> np.ndarray:
    f = focal_ratio * width
    return np.array([[f, 0.0, (width - 1) / 2.0], [0.0, f, (height - 1) / 2.0], [0.0, 0.0, 1.0]])


def ring_cameras(n_views: int, width: int, height: int, radius: float = 15.0,
                 height_m: float = 6.0, step_deg: float = 10.0, start_deg: float = 0.0,
                 target=(0.0, 0.0, 0.5)) -> List[Camera]:
    cams = []
    K = intrinsics(width, height)
    for v in range(n_views):
        a = np.deg2rad(start_deg + step_deg * v)
        c = np.array([radius * np.cos(a), radius * np.sin(a), height_m])
        R, t = look_at(c, target)
        cams.append(Camera(K.copy(), R, t, width, height))
    return cams


def nadir_cameras(size: float, altitude: float, width: int, height: int,
                  forward_overlap: float = 0.7, side_overlap: float = 0.6,
                  oblique_deg: float = 0.0, max_views: Optional[int] = None,
                  yaw_deg: float = 0.0) -> List[Camera]:
    """Grid of nadir (or tilted by ``oblique_deg``) cameras over a size x size area."""
    K = intrinsics(width, height)
    f = K[0, 0]
    fw = altitude * width / f  # ground footprint width (m)
    fh = altitude * height / f
    dx = fw * (1.0 - side_overlap)
    dy = fh * (1.0 - forward_overlap)
    xs = np.arange(-size / 2 + fw / 2, size / 2 - fw / 2 + 1e-6, dx)
    ys = np.arange(-size / 2 + fh / 2, size / 2 - fh / 2 + 1e-6, dy)
    cams = []
    tilt = np.deg2rad(oblique_deg)
    yaw = np.deg2rad(yaw_deg)
    for y in ys:
        for x in xs:
            c = np.array([x, y, altitude])
            tgt = c + np.array([np.sin(tilt) * np.cos(yaw), np.sin(tilt) * np.sin(yaw), -np.cos(tilt)])
            R, t = look_at(c, tgt, up=(0.0, 1.0, 0.0))
            cams.append(Camera(K.copy(), R, t, width, height))
            if max_views and len(cams) >= max_views:
                return cams
    return cams


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def render(scene: Scene, cam: Camera, supersample: int = 2, threads: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """Ray-casts one view: (uint8 image (H, W), float32 depth (H, W))."""
    lib = _load()
    W, H = cam.width, cam.height
    img = np.zeros((H, W), np.uint8)
    dep = np.zeros((H, W), np.float32)
    boxes = np.ascontiguousarray(scene.boxes, np.float64).reshape(-1)
    if boxes.size == 0:
        boxes = np.zeros(6)
    K = np.ascontiguousarray(cam.K, np.float64)
    R = np.ascontiguousarray(cam.R, np.float64)
    t = np.ascontiguousarray(cam.t, np.float64)
    threads = threads or min(16, os.cpu_count() or 1)
    bands = np.linspace(0, H, threads + 1).astype(int)

    def run(k):
        r0, r1 = int(bands[k]), int(bands[k + 1])
        if r1 <= r0:
            return
        lib.rc_render(
            _dptr(boxes), int(scene.boxes.shape[0]), int(scene.ground), float(scene.ground_half),
            int(scene.terrain),
            scene.terrain_amp, scene.terrain_scale, scene.terrain_seed, scene.terrain_octaves,
            scene.tex_seed, scene.tex_freq, scene.tex_octaves, scene.contrast, scene.sky,
            _dptr(K), _dptr(R), _dptr(t), W, H, supersample, r0, r1,
            img.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
            dep.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
        )

    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(run, range(threads)))
    return img, dep


def depth_range(depth: np.ndarray, margin: float = 0.05) -> Tuple[float, float]:
    """Depth range of a view from its valid ground-truth depths, widened by ``margin``."""
    v = depth[depth > 0]
    return float(v.min() * (1 - margin)), float(v.max() * (1 + margin))


@dataclass
class ViewSet:
    """A rendered multi-view set: cameras, images, ground-truth depths."""
    scene: Scene
    cameras: List[Camera]
    images: List[np.ndarray]
    depths: List[np.ndarray]

    def neighbors(self, ref: int, k: int) -> List[int]:
        """The k views whose optical centres are nearest to ``ref``'s."""
        c0 = self.cameras[ref].center
        d = [(np.linalg.norm(c.center - c0), v) for v, c in enumerate(self.cameras) if v != ref]
        d.sort()
        return [v for _, v in d[:k]]

    def neighbors_by_footprint(self, ref: int, k: int, min_cos: float = 0.9,
                               ground_z: float = 0.0) -> List[int]:
        """The k views looking the most alike at the nearest ground point:
        among views whose optical axes are within acos(min_cos) of ``ref``'s,
        the ones whose axes meet the plane z = ground_z nearest to where
        ``ref``'s does (for mixed nadir and oblique sets)."""
        def axis(c):
            d = c.R[2]
            s = (ground_z - c.center[2]) / d[2] if abs(d[2]) > 1e-9 else 1e9
            return d, c.center + s * d

        d0, g0 = axis(self.cameras[ref])
        cand = []
        for v, c in enumerate(self.cameras):
            if v == ref:
                continue
            d, g = axis(c)
            if float(d @ d0) >= min_cos:
                cand.append((float(np.linalg.norm(g - g0)), v))
        cand.sort()
        return [v for _, v in cand[:k]]


def ring_viewset(seed: int, n_views: int, width: int, height: int, step_deg: float = 10.0,
                 supersample: int = 2) -> ViewSet:
    scene = box_scene(seed)
    cams = ring_cameras(n_views, width, height, step_deg=step_deg,
                        start_deg=float(np.random.default_rng(seed + 1).uniform(0, 360)))
    imgs, deps = [], []
    for c in cams:
        im, de = render(scene, c, supersample)
        imgs.append(im)
        deps.append(de)
    return ViewSet(scene, cams, imgs, deps)


MIXED_SIZES = ((640, 480), (480, 640), (640, 360), (320, 240))


def mixed_viewset(seed: int, n_views: int = 64, kind: str = "box",
                  sizes: Sequence[Tuple[int, int]] = MIXED_SIZES, supersample: int = 2,
                  scale: float = 1.0, gpu: bool = False,
                  step_deg: Optional[float] = None) -> ViewSet:
    """Views of mixed sizes, each drawn uniformly from ``sizes`` (width,
    height) by the seed, every camera with its own intrinsics.

    kind "box": the box scene seen from a ring of ``n_views`` cameras
    (radius 15 m, height 6 m), ``step_deg`` apart (default: a full circle).  kind "terrain": a heightfield of amplitude
    8 m with the feature scale of a 100 x 100 m terrain (the field extends
    beyond it), seen by nadir cameras at 60 m altitude on a grid with 70 %
    forward and 60 % side overlap (spacing from the 640 x 480 footprint).
    ``scale`` shrinks every size (for quick tests); ``gpu`` renders with the
    CUDA ray caster instead of the CPU one."""
    rng = np.random.default_rng(seed + 7)
    pick = rng.integers(len(sizes), size=n_views)
    dims = [(max(16, int(round(sizes[k][0] * scale))), max(16, int(round(sizes[k][1] * scale))))
            for k in pick]
    if kind == "box":
        scene = box_scene(seed)
        base = ring_cameras(n_views, 640, 480, step_deg=step_deg or 360.0 / n_views,
                            start_deg=float(np.random.default_rng(seed + 1).uniform(0, 360)))
    elif kind == "terrain":
        scene = terrain_scene(seed, size=100.0, amp=8.0)
        side = int(np.ceil(np.sqrt(n_views)))
        K0 = intrinsics(640, 480)
        fw, fh = 60.0 * 640 / K0[0, 0], 60.0 * 480 / K0[0, 0]
        span = max((side - 1) * fw * 0.4 + fw, (side - 1) * fh * 0.3 + fh) + 1.0
        base = nadir_cameras(span, 60.0, 640, 480, forward_overlap=0.7, side_overlap=0.6,
                             max_views=n_views)
    else:
        raise ValueError(f"unknown kind {kind!r}")
    if len(base) < n_views:
        raise ValueError(f"only {len(base)} cameras fit the {kind} layout")
    cams = [Camera(intrinsics(w, h), c.R, c.t, w, h) for c, (w, h) in zip(base, dims)]
    imgs, deps = [], []
    for c in cams:
        if gpu:
            im, de = render_gpu(scene, [c], supersample)
            im, de = im[0].cpu().numpy(), de[0].cpu().numpy()
        else:
            im, de = render(scene, c, supersample)
        imgs.append(im)
        deps.append(de)
    return ViewSet(scene, cams, imgs, deps)


def aerial_viewset(seed: int, n_nadir: int = 128, n_oblique: int = 128, width: int = 1280,
                   height: int = 960, size: float = 300.0, n_buildings: int = 40,
                   altitude: float = 60.0, oblique_deg: float = 45.0, supersample: int = 1,
                   gpu: bool = True) -> ViewSet:
    """A large aerial block: terrain of size x size m (amplitude 8 m) with
    ``n_buildings`` buildings, seen by ``n_nadir`` nadir views and
    ``n_oblique`` views tilted by ``oblique_deg`` (a quarter looking each
    way), all width x height, spread evenly over grids with 70 % forward and
    60 % side overlap at ``altitude``."""
    scene = terrain_scene(seed, size=size, amp=8.0, n_buildings=n_buildings)

    def spread(cams, n):
        if n >= len(cams):
            return cams
        idx = np.round(np.linspace(0, len(cams) - 1, n)).astype(int)
        return [cams[i] for i in idx]

    cams = spread(nadir_cameras(size, altitude, width, height), n_nadir)
    per = [n_oblique // 4 + (1 if k < n_oblique % 4 else 0) for k in range(4)]
    for k in range(4):
        if per[k]:
            grid = nadir_cameras(size, altitude, width, height, oblique_deg=oblique_deg,
                                 yaw_deg=90.0 * k)
            cams += spread(grid, per[k])
    imgs, deps = [], []
    for c in cams:
        if gpu:
            im, de = render_gpu(scene, [c], supersample)
            im, de = im[0].cpu().numpy(), de[0].cpu().numpy()
        else:
            im, de = render(scene, c, supersample)
        imgs.append(im)
        deps.append(de)
    return ViewSet(scene, cams, imgs, deps)


def accuracy(depth: np.ndarray, gt: np.ndarray, rel: float = 0.01, valid: Optional[np.ndarray] = None) -> float:
    """Fraction of valid ground-truth pixels whose depth is within ``rel`` relative error."""
    m = gt > 0
    if valid is not None:
        m &= valid
    if not m.any():
        return 0.0
    err = np.abs(depth[m] - gt[m]) / gt[m]
    return float((err <= rel).mean())
