"""Learned PatchMatch initialisation (no reference counterpart).

The reference starts PatchMatch from random planes
(``RandomInitialization``, ``opensfm/src/lib/dense/src/depthmap.cc:237-256``)
and spends three raster iterations converging.  Here a small network proposes
the initial plane of every pixel, so PatchMatch needs fewer iterations for
the same accuracy; the random initialisation stays as the fallback for any
pixel without a proposal.

Network: 6 convolutions 3 x 3 (5 x 32 channels + ReLU, then 4 outputs),
BF16 weights and activations, FP32 accumulation, run by the library's own
tensor-core kernels (``dn_nn_*`` in ``include/dense_b200.h``).  Input per
pixel: the reference intensity and the bilateral NCC of 8 swept
fronto-parallel planes against the 2 nearest matching views
(``dn_batch_sweep_features``).  Output: the inverse-depth fraction over the
depth range and the normal slopes (sx, sy), normal ~ (sx, sy, -1).

Training data: plain PatchMatch depthmaps of seeded synthetic scenes (box
and terrain), computed by this library; targets are the pixels whose score
is at least ``min_score``.  PyTorch only provides device buffers and a
stream here; every kernel is the library's.
"""
from __future__ import annotations

import ctypes
import math
import os
import time
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib, pydense
from . import synthetic as S

FEAT_C = 32
LAYERS = [(32, 32, 1)] * 5 + [(32, 4, 0)]  # (cin, cout, relu)
WEIGHTS_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights")
DEFAULT_WEIGHTS = os.path.join(WEIGHTS_DIR, "proposal_net.npz")


def _torch():
    import torch
    return torch


def _ptr(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(_torch().cuda.current_stream().cuda_stream)


class ProposalNet:
    """FP32 master weights + Adam state on the device, BF16 copies for the kernels."""

    def __init__(self, seed: int = 0, stride: int = 2, n_planes: int = 8):
        torch = _torch()
        self.stride = stride  # proposal grid the network was trained on
        self.n_planes = n_planes  # sweep planes of its input features
        self.train_dim = 0  # larger side of its training images (0: not recorded)
        g = torch.Generator().manual_seed(seed)
        self.w32, self.b32, self.w16 = [], [], []
        for cin, cout, relu in LAYERS:
            fan_in = 9 * cin
            std = math.sqrt(2.0 / fan_in) if relu else math.sqrt(1.0 / fan_in)
            w = torch.randn((cout, 9 * cin), generator=g) * std
            self.w32.append(w.cuda())
            self.b32.append(torch.zeros(cout).cuda())
        self.sync_bf16()
        self.m = [torch.zeros_like(t) for t in self.w32 + self.b32]
        self.v = [torch.zeros_like(t) for t in self.w32 + self.b32]
        self.step = 0
        self.wt_scratch = torch.empty(32 * 9 * 32, dtype=torch.bfloat16, device="cuda")

    def sync_bf16(self):
        self.w16 = [w.to(_torch().bfloat16).contiguous() for w in self.w32]

    def packed(self) -> Tuple[np.ndarray, np.ndarray]:
        """(BF16 bit patterns of every layer's [cout][288] weights one after
        the other, FP32 biases), the layout of ``Batch.set_proposal_net``."""
        torch = _torch()
        w = torch.cat([t.reshape(-1) for t in self.w16]).view(torch.int16).cpu().numpy()
        b = torch.cat([t.reshape(-1) for t in self.b32]).cpu().numpy()
        return w.view(np.uint16).copy(), b.astype(np.float32)

    # ------------------------------------------------------------ state
    def state_dict(self) -> Dict[str, np.ndarray]:
        d = {}
        for k, (w, b) in enumerate(zip(self.w32, self.b32)):
            d[f"w{k}"] = w.cpu().numpy()
            d[f"b{k}"] = b.cpu().numpy()
        d["step"] = np.array(self.step)
        d["stride"] = np.array(self.stride)
        d["planes"] = np.array(self.n_planes)
        return d

    def save(self, path: str, **extra):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        d = self.state_dict()
        d.update({k: np.asarray(v) for k, v in extra.items()})
        np.savez(path, **d)

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS) -> "ProposalNet":
        torch = _torch()
        z = np.load(path)
        net = cls.__new__(cls)
        net.w32 = [torch.from_numpy(z[f"w{k}"]).cuda() for k in range(len(LAYERS))]
        net.b32 = [torch.from_numpy(z[f"b{k}"]).cuda() for k in range(len(LAYERS))]
        net.sync_bf16()
        net.m = [torch.zeros_like(t) for t in net.w32 + net.b32]
        net.v = [torch.zeros_like(t) for t in net.w32 + net.b32]
        net.step = int(z["step"]) if "step" in z else 0
        net.stride = int(z["stride"]) if "stride" in z else 1
        net.n_planes = int(z["planes"]) if "planes" in z else 8
        net.train_dim = (max(int(z["train_W"]), int(z["train_H"])) if "train_W" in z else 0)
        net.wt_scratch = torch.empty(32 * 9 * 32, dtype=torch.bfloat16, device="cuda")
        return net

    # ---------------------------------------------------------- compute
    def forward(self, feat, n_pix: int, H: int, W: int, keep: bool = False):
        """feat: BF16 [n_pix * 32].  Returns FP32 output [n_pix, 4] and, with
        keep, the list of layer inputs for backward."""
        torch = _torch()
        L = _lib.load()
        acts = [feat]
        x = feat
        out32 = torch.empty((n_pix, 4), dtype=torch.float32, device="cuda")
        for k, (cin, cout, relu) in enumerate(LAYERS):
            last = k == len(LAYERS) - 1
            y = None if last else torch.empty(n_pix * cout, dtype=torch.bfloat16, device="cuda")
            _lib.check(L.dn_nn_conv3x3_forward(
                _ptr(x), _ptr(self.w16[k]), _ptr(self.b32[k]), n_pix, H, W, cin, cout, relu,
                _ptr(y) if y is not None else None, _ptr(out32) if last else None, _stream()))
            if not last:
                x = y
                acts.append(y)
        return (out32, acts) if keep else out32

    def backward(self, acts, dpred, n_pix: int, H: int, W: int, tensor_cores: bool = True):
        """Gradients (FP32, summed over pixels) of every layer's weights and
        biases.  tensor_cores: the tcgen05 kernels (weight gradient as a
        split-K GEMM in tensor memory, data gradient as the forward kernel on
        flipped weights); False: the mma.sync kernels."""
        torch = _torch()
        L = _lib.load()
        dws = [torch.zeros_like(w) for w in self.w32]
        dbs = [torch.zeros_like(b) for b in self.b32]
        if tensor_cores:
            need = int(L.dn_nn_backward_scratch_bytes(n_pix, LAYERS[-1][1]))
            scratch = getattr(self, "bwd_scratch", None)
            if scratch is None or scratch.numel() < need:
                scratch = self.bwd_scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
        dy = dpred
        for k in range(len(LAYERS) - 1, -1, -1):
            cin, cout, relu = LAYERS[k]
            x = acts[k]
            need_dx = k > 0
            dx = torch.empty(n_pix * cin, dtype=torch.bfloat16, device="cuda") if need_dx else None
            # dx is masked by the ReLU of the layer below (its output x > 0).
            if tensor_cores:
                _lib.check(L.dn_nn_conv3x3_backward_tc(
                    _ptr(dy), _ptr(x), _ptr(self.w16[k]), _ptr(x) if need_dx else None, n_pix, H,
                    W, cin, cout, _ptr(dx) if need_dx else None, _ptr(dws[k]), _ptr(dbs[k]),
                    _ptr(scratch), scratch.numel(), _stream()))
            else:
                _lib.check(L.dn_nn_conv3x3_backward(
                    _ptr(dy), _ptr(x), _ptr(self.w16[k]), _ptr(x) if need_dx else None, n_pix, H,
                    W, cin, cout, _ptr(dx) if need_dx else None, _ptr(dws[k]), _ptr(dbs[k]),
                    _ptr(self.wt_scratch), _stream()))
            dy = dx
        return dws, dbs

    def adam(self, dws, dbs, count, lr: float, b1=0.9, b2=0.999, eps=1e-8):
        L = _lib.load()
        self.step += 1
        bc1 = 1.0 - b1 ** self.step
        bc2 = 1.0 - b2 ** self.step
        params = self.w32 + self.b32
        grads = dws + dbs
        w16 = self.w16 + [None] * len(self.b32)
        for p, g, m, v, h in zip(params, grads, self.m, self.v, w16):
            _lib.check(L.dn_nn_adam(_ptr(p), _ptr(m), _ptr(v), _ptr(g), p.numel(), _ptr(count), lr,
                                    b1, b2, eps, bc1, bc2, _ptr(h) if h is not None else None,
                                    _stream()))


# ------------------------------------------------------------------ data
@dataclass
class SceneViews:
    cams: List[S.Camera]
    images: np.ndarray  # (n, H, W) uint8
    depths: np.ndarray  # (n, H, W) float32 ground truth
    ref: int
    matching: List[int]  # nearest first; the first two are the sweep views


def make_scene(seed: int, W: int, H: int, kind: Optional[str] = None, n_match: int = 6) -> SceneViews:
    """Box scene on a camera ring, or terrain under a nadir grid (by seed
    parity); kind "aerial": 300 x 300 m terrain with 40 buildings under a
    nadir or 45-degree oblique grid (one of four headings) at 60 m."""
    rng = np.random.default_rng(seed)
    kind = kind or ("box" if seed % 2 == 0 else "terrain")
    if kind == "aerial":
        scene = S.terrain_scene(seed, size=300.0, amp=8.0, n_buildings=40)
        tilt = 45.0 if rng.random() < 0.5 else 0.0
        grid = S.nadir_cameras(300.0, 60.0, W, H, forward_overlap=0.7, side_overlap=0.6,
                               oblique_deg=tilt, yaw_deg=90.0 * int(rng.integers(4)))
        centres = np.stack([c.center for c in grid])
        c0 = centres[int(rng.integers(len(grid)))]
        order = np.argsort(np.linalg.norm(centres - c0, axis=1))[: n_match + 1]
        cams = [grid[k] for k in order]
        ref = 0
    elif kind == "box":
        scene = S.box_scene(seed)
        n = n_match + 1
        cams = S.ring_cameras(n, W, H, step_deg=10.0, start_deg=float(rng.uniform(0, 360)))
        ref = n // 2
    else:
        scene = S.terrain_scene(seed, size=100.0, amp=8.0)
        grid = S.nadir_cameras(100.0, 60.0, W, H, forward_overlap=0.7, side_overlap=0.6)
        centres = np.stack([c.center for c in grid])
        c0 = centres[int(rng.integers(len(grid)))]
        order = np.argsort(np.linalg.norm(centres - c0, axis=1))[: n_match + 1]
        cams = [grid[k] for k in order]
        ref = 0
    imgs, deps = S.render_gpu(scene, cams)
    images = imgs.cpu().numpy()
    depths = deps.cpu().numpy()
    others = [k for k in range(len(cams)) if k != ref]
    c_ref = cams[ref].center
    others.sort(key=lambda k: float(np.linalg.norm(cams[k].center - c_ref)))
    return SceneViews(cams, images, depths, ref, others[:n_match])


def depth_range_of(sv: SceneViews) -> Tuple[float, float]:
    return S.depth_range(sv.depths[sv.ref])


def build_batch(scenes: Sequence[SceneViews], iterations: int = 3, seed: int = 1,
                patch: int = 7, min_sd: float = 1.0) -> Tuple[pydense.Batch, List[int]]:
    """One batch holding every scene's views; one depthmap per scene."""
    b = pydense.Batch()
    maps = []
    for sv in scenes:
        ids = [b.add_view(c.K, c.R, c.t, im) for c, im in zip(sv.cams, sv.images)]
        mn, mx = depth_range_of(sv)
        maps.append(b.add_depthmap(ids[sv.ref], [ids[k] for k in sv.matching], mn, mx))
    b.set_params(patch_size=patch, min_patch_sd=min_sd, iterations=iterations, seed=seed)
    return b, maps


def grid_shape(H: int, W: int, stride: int) -> Tuple[int, int]:
    """The proposal grid of an H x W map: every ``stride``-th pixel."""
    return (H + stride - 1) // stride, (W + stride - 1) // stride


def features(b: pydense.Batch, n_maps: int, H: int, W: int, n_planes: int = 8, stride: int = 1):
    torch = _torch()
    Hs, Ws = grid_shape(H, W, stride)
    per = Hs * Ws * FEAT_C
    feat = torch.zeros(n_maps * per, dtype=torch.bfloat16, device="cuda")
    _lib.check(b._L.dn_batch_sweep_features(b._h, _ptr(feat), per, n_planes, stride))
    b.synchronize()
    return feat


def targets(b: pydense.Batch, n_maps: int, H: int, W: int, min_score: float = 0.5,
            stride: int = 1):
    torch = _torch()
    Hs, Ws = grid_shape(H, W, stride)
    per = Hs * Ws * 4
    tg = torch.zeros(n_maps * per, dtype=torch.float32, device="cuda")
    _lib.check(b._L.dn_batch_targets(b._h, _ptr(tg), per, min_score, stride))
    b.synchronize()
    return tg


def make_dataset(seeds: Sequence[int], W: int = 640, H: int = 480, chunk: int = 50,
                 iterations: int = 3, stride: int = 2, n_planes: int = 8,
                 gt_filter: float = 0.0, log=None, kind: Optional[str] = None):
    """Features on the proposal grid and plain-PatchMatch targets at the same
    grid points for every seed (device tensors).  gt_filter > 0 keeps only
    the targets whose depth is within that relative error of the rendered
    ground truth (the other grid points get weight 0)."""
    torch = _torch()
    feats, tgs = [], []
    t0 = time.time()
    Hs, Ws = grid_shape(H, W, stride)
    for c0 in range(0, len(seeds), chunk):
        scenes = [make_scene(s, W, H, kind=kind) for s in seeds[c0:c0 + chunk]]
        b, maps = build_batch(scenes, iterations=iterations, seed=int(seeds[c0]) + 7)
        b.run()
        b.synchronize()
        tg = targets(b, len(maps), H, W, stride=stride)
        if gt_filter > 0:
            # The target depth from its inverse-depth fraction, against the
            # ground truth at the same pixel (grid point (ys, xs) = pixel
            # (stride ys, stride xs)).
            gt = torch.from_numpy(np.stack([sv.depths[sv.ref][::stride, ::stride]
                                            for sv in scenes]).astype(np.float32)).cuda()
            rng = np.array([depth_range_of(sv) for sv in scenes], np.float64)
            a = torch.from_numpy(1.0 / rng[:, 1]).float().cuda().view(-1, 1, 1)
            bb = torch.from_numpy(1.0 / rng[:, 0]).float().cuda().view(-1, 1, 1)
            t4 = tg.view(len(maps), Hs, Ws, 4)
            d = 1.0 / (a + (bb - a) * t4[..., 0])
            keep = (t4[..., 3] > 0) & (gt > 0) & ((d - gt).abs() <= gt_filter * gt)
            t4[..., 3] = keep.float()
        tgs.append(tg)
        feats.append(features(b, len(maps), H, W, n_planes=n_planes, stride=stride))
        b.close()
        if log:
            log(f"dataset {c0 + len(scenes)}/{len(seeds)} scenes, {time.time() - t0:.1f} s")
    return torch.cat(feats), torch.cat(tgs)


# -------------------------------------------------------------- training
def save_checkpoint(net: ProposalNet, path: str, step: int, generator) -> None:
    """Everything a training run needs to continue bit for bit where it
    stopped: FP32 master weights and biases, both Adam moments, the Adam
    step, the loop step and the state of the batch-sampling generator."""
    torch = _torch()
    d = net.state_dict()
    for k, (m, v) in enumerate(zip(net.m, net.v)):
        d[f"adam_m{k}"] = m.cpu().numpy()
        d[f"adam_v{k}"] = v.cpu().numpy()
    d["loop_step"] = np.array(step)
    d["rng_state"] = generator.get_state().numpy()
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez(path, **d)


def load_checkpoint(path: str) -> Tuple[ProposalNet, int, "object"]:
    """(network with its Adam state, next loop step, generator) from
    ``save_checkpoint``."""
    torch = _torch()
    z = np.load(path)
    net = ProposalNet.load(path)
    n = len(net.m)
    net.m = [torch.from_numpy(z[f"adam_m{k}"]).cuda() for k in range(n)]
    net.v = [torch.from_numpy(z[f"adam_v{k}"]).cuda() for k in range(n)]
    g = torch.Generator(device="cpu")
    g.set_state(torch.from_numpy(z["rng_state"]))
    return net, int(z["loop_step"]), g


def train(net: ProposalNet, feat, tgt, n_maps: int, H: int, W: int, steps: int = 1500,
          batch: int = 8, lr: float = 2e-3, normal_weight: float = 0.1, seed: int = 0, log=None,
          start_step: int = 0, generator=None, stop_step: Optional[int] = None,
          checkpoint: Optional[str] = None):
    """Adam on the L1 loss over ``steps`` steps of a cosine learning-rate
    schedule.  A run can stop early (``stop_step``; with ``checkpoint`` the
    state is saved there) and continue from ``load_checkpoint``'s state
    (``start_step``, ``generator``) with the same ``steps``."""
    return train_sets(net, [(feat, tgt, n_maps, H, W)], steps=steps, batch=batch, lr=lr,
                      normal_weight=normal_weight, seed=seed, log=log, start_step=start_step,
                      generator=generator, stop_step=stop_step, checkpoint=checkpoint)


def train_sets(net: ProposalNet, sets, steps: int = 1500, batch: int = 8, lr: float = 2e-3,
               normal_weight: float = 0.1, seed: int = 0, log=None, start_step: int = 0,
               generator=None, stop_step: Optional[int] = None,
               checkpoint: Optional[str] = None):
    """``train`` over several datasets of different grid shapes, sets =
    [(feat, tgt, n_maps, H, W), ...]: each step draws its dataset with
    probability proportional to n_maps, then its batch from that dataset
    (one dataset: the same draws as ``train``)."""
    torch = _torch()
    L = _lib.load()
    g = generator if generator is not None else torch.Generator(device="cpu").manual_seed(seed)
    loss_acc = torch.zeros(1, dtype=torch.float32, device="cuda")
    count = torch.zeros(1, dtype=torch.float32, device="cuda")
    views = [(f.view(n, H * W * FEAT_C), t.view(n, H * W * 4), n, H, W) for f, t, n, H, W in sets]
    weights = torch.tensor([float(v[2]) for v in views])
    history = []
    t0 = time.time()
    end = steps if stop_step is None else min(stop_step, steps)
    for step in range(start_step, end):
        k = 0 if len(views) == 1 else int(torch.multinomial(weights, 1, generator=g))
        fv, tv, n_maps, H, W = views[k]
        n_pix = batch * H * W
        dpred = torch.empty(n_pix * 4, dtype=torch.bfloat16, device="cuda")
        idx = torch.randint(0, n_maps, (batch,), generator=g).cuda()
        xb = fv.index_select(0, idx).reshape(-1).contiguous()
        tb = tv.index_select(0, idx).reshape(-1).contiguous()
        out, acts = net.forward(xb, n_pix, H, W, keep=True)
        loss_acc.zero_()
        count.zero_()
        _lib.check(L.dn_nn_l1_loss(_ptr(out), _ptr(tb), n_pix, normal_weight, _ptr(dpred),
                                   _ptr(loss_acc), _ptr(count), _stream()))
        dws, dbs = net.backward(acts, dpred, n_pix, H, W)
        cur_lr = lr * 0.5 * (1 + math.cos(math.pi * step / steps))
        net.adam(dws, dbs, count, cur_lr)
        if step % 100 == 0 or step == steps - 1:
            l = float(loss_acc.item() / max(count.item(), 1.0))
            history.append((step, l))
            if log:
                log(f"step {step} loss {l:.4f} lr {cur_lr:.2e} {time.time() - t0:.1f} s")
    if checkpoint:
        save_checkpoint(net, checkpoint, end, g)
    return history


# ------------------------------------------------------------- inference
def propose(net: ProposalNet, b: pydense.Batch, maps: Sequence[int], H: int, W: int):
    """Runs the sweep and the network for every depthmap of the batch at full
    resolution and installs the proposals as the batch's initial planes (the
    step-by-step form of ``run(learned=True)`` with stride 1)."""
    torch = _torch()
    n = len(maps)
    feat = features(b, n, H, W)
    out = net.forward(feat, n * H * W, H, W)
    _lib.check(_lib.load().dn_nn_synchronize(_stream()))
    for k, m in enumerate(maps):
        _lib.check(b._L.dn_batch_init_from_output(b._h, int(m), _ptr(out[k * H * W:])))
    b.synchronize()
    return out


def install(net: ProposalNet, b: pydense.Batch, stride: Optional[int] = None,
            n_planes: Optional[int] = None) -> None:
    """Hands the network to the batch: ``b.run(learned=True)`` then sweeps,
    runs the network and installs the proposals on the batch stream (by
    default on the grid and with the sweep planes it was trained with).  Maps
    of other sizes than the training images get the stride scaled to their
    size (``Batch.set_proposal_scale``), so their grid has the training
    scale."""
    w, bias = net.packed()
    b.set_proposal_net(w, bias, n_planes=n_planes or net.n_planes, stride=stride or net.stride)
    b.set_proposal_scale(getattr(net, "train_dim", 0))


def main(argv=None):
    """Trains the proposal network (python -m opensfm_b200.learned --scenes
    2000), or, with --evaluate, compares learned-init and plain PatchMatch
    on held-out scenes and prints the result as one JSON line."""
    import argparse
    import json

    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=2000)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--size", default="640x480", help="training scene size WxH")
    ap.add_argument("--stride", type=int, default=4, help="proposal grid stride (1, 2 or 4)")
    ap.add_argument("--planes", type=int, default=15, help="sweep planes (1..15)")
    ap.add_argument("--portrait", type=int, default=600,
                    help="also train on this many portrait scenes (the size transposed; "
                         "seeds 200000 and up)")
    ap.add_argument("--aerial", type=int, default=400,
                    help="also train on this many aerial scenes (terrain with buildings, nadir "
                         "or oblique) at twice the size and stride (seeds 300000 and up)")
    ap.add_argument("--gt-filter", type=float, default=0.01,
                    help="keep only targets within this relative depth error of the ground truth")
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--evaluate", action="store_true",
                    help="evaluate the weights in --out instead of training")
    ap.add_argument("--eval-seeds", default="900000:900012",
                    help="held-out scene seeds, start:stop (training uses 100000 and up)")
    ap.add_argument("--repeats", type=int, default=3)
    args = ap.parse_args(argv)
    log = lambda s: print(s, flush=True)  # noqa: E731
    if args.evaluate:
        a, b = (int(x) for x in args.eval_seeds.split(":"))
        net = ProposalNet.load(args.out)
        res = evaluate(net, list(range(a, b)), repeats=args.repeats, log=log)
        print(json.dumps(res), flush=True)
        return
    W, H = (int(x) for x in args.size.split("x"))
    seeds = list(range(100000, 100000 + args.scenes))
    feat, tgt = make_dataset(seeds, W=W, H=H, stride=args.stride, n_planes=args.planes,
                             gt_filter=args.gt_filter, log=log)
    valid = float((tgt.view(-1, 4)[:, 3] > 0).float().mean().item())
    log(f"target coverage {valid:.3f}")
    Hs, Ws = grid_shape(H, W, args.stride)
    torch = _torch()
    n_main = len(seeds)
    if args.aerial:
        # Twice the size at twice the stride: the same grid as the main scenes.
        fa, ta = make_dataset(list(range(300000, 300000 + args.aerial)), W=2 * W, H=2 * H,
                              stride=2 * args.stride, n_planes=args.planes,
                              gt_filter=args.gt_filter, log=log, kind="aerial", chunk=25)
        feat, tgt = torch.cat([feat, fa]), torch.cat([tgt, ta])
        n_main += args.aerial
    sets = [(feat, tgt, n_main, Hs, Ws)]
    if args.portrait:
        fp, tp = make_dataset(list(range(200000, 200000 + args.portrait)), W=H, H=W,
                              stride=args.stride, n_planes=args.planes,
                              gt_filter=args.gt_filter, log=log)
        sets.append((fp, tp, args.portrait, Ws, Hs))
    net = ProposalNet(seed=args.seed, stride=args.stride, n_planes=args.planes)
    hist = train_sets(net, sets, steps=args.steps, batch=args.batch, lr=args.lr, log=log)
    net.save(args.out, history=np.array(hist), scenes=np.array(args.scenes),
             seeds_start=np.array(seeds[0]), stride=np.array(args.stride),
             train_W=np.array(W), train_H=np.array(H), gt_filter=np.array(args.gt_filter),
             steps=np.array(args.steps), portrait=np.array(args.portrait),
             aerial=np.array(args.aerial))
    log(f"saved {args.out}")


# ------------------------------------------------------------ evaluation
@dataclass
class Schedule:
    """A PatchMatch schedule compared by ``evaluate``: the initialisation
    ("plain" = the reference's random initialisation, "learned" = the
    proposal network), the half-passes, the candidate sets of
    ``Batch.set_schedule``, one view per candidate (``sample``) and the
    active-pixel half-passes (``active``)."""
    name: str
    init: str
    half_passes: int
    kw: dict
    sample: int = 0  # Batch.set_candidate_views mode
    active: float = 0.0  # > 0: active pixels, a depth moves by more than this
    knights: bool = False
    seed: float = 0.0  # > 0: settled start below this initial score (Batch.set_active_seed)
    fallback: bool = False  # random plane where it scores higher (Batch.set_init_fallback)

    def apply(self, b: pydense.Batch) -> None:
        b.set_schedule(half_passes=self.half_passes, **self.kw)
        b.set_candidate_views(self.sample)
        b.set_active_pixels(self.active > 0, self.active)
        b.set_active_seed(self.seed)
        b.set_init_fallback(self.fallback)
        b.set_knight_moves(self.knights)


PLAIN_3IT = Schedule("plain-3it", "plain", 6, {})
_NEAR = dict(use_far=False, depth_range0=0.02, normal_range0=0.3)
SCHEDULES = [
    Schedule("plain-1it", "plain", 2, {}),
    Schedule("plain-2it", "plain", 4, {}),
    PLAIN_3IT,
    Schedule("plain-3it-active", "plain", 6, {}, active=0.002),
    Schedule("learned-0hp", "learned", 0, {}),
    Schedule("learned-2hp", "learned", 2, {}),
    Schedule("learned-4hp", "learned", 4, {}),
    Schedule("learned-6hp", "learned", 6, {}),
    Schedule("learned-sample-2hp", "learned", 2, {}, sample=True),
    Schedule("learned-sample-4hp", "learned", 4, {}, sample=True),
    Schedule("learned-sample-6hp", "learned", 6, {}, sample=True),
    Schedule("learned-sample-8hp", "learned", 8, {}, sample=True),
    Schedule("learned-sample-active-6hp", "learned", 6, {}, sample=True, active=0.002),
    Schedule("learned-sample-active-8hp", "learned", 8, {}, sample=True, active=0.002),
    Schedule("learned-sample-near-4hp", "learned", 4, _NEAR, sample=True),
    Schedule("learned-sample-near-6hp", "learned", 6, _NEAR, sample=True),
    Schedule("learned-sample-near3-6hp", "learned", 6, dict(_NEAR, n_refine=3), sample=True),
    Schedule("learned-active-4hp", "learned", 4, {}, active=0.002),
    Schedule("learned-active-6hp", "learned", 6, {}, active=0.002),
]


def evaluate(net: Optional[ProposalNet], seeds: Sequence[int], W: int = 640, H: int = 480,
             schedules=SCHEDULES, repeats: int = 3, stride: Optional[int] = None, log=None,
             scenes=None) -> dict:
    """Plain (random init) vs learned-init PatchMatch on held-out scenes.

    Every schedule runs as one captured CUDA graph over all the scenes'
    depthmaps (for learned schedules the feature sweep, the network and the
    plane install included, on the batch stream) and is timed with device
    events around the replay.  Accuracy: the mean over the maps of the
    fraction of valid ground-truth pixels with |d - gt| / gt <= 1 %.
    """
    scenes = scenes or [make_scene(s, W, H) for s in seeds]
    b, maps = build_batch(scenes, iterations=3, seed=int(seeds[0]) + 11)
    gts = [sv.depths[sv.ref] for sv in scenes]
    if net is not None:
        install(net, b, stride=stride or net.stride)

    def acc():
        return float(np.mean([S.accuracy(b.get_depth(m), gt) for m, gt in zip(maps, gts)]))

    out = {"scenes": len(scenes), "W": W, "H": H, "runs": [],
           "stride": (stride or net.stride) if net is not None else None}
    plain_ms = None
    for sc in schedules:
        if sc.init == "learned" and net is None:
            continue
        sc.apply(b)
        learned = sc.init == "learned"
        b.run(graph=True, learned=learned)  # capture
        b.synchronize()
        ts = []
        for _ in range(repeats):
            b.timer_record(0)
            b.run(graph=True, learned=learned)
            b.timer_record(1)
            b.synchronize()
            ts.append(b.timer_elapsed())
        t = float(np.median(ts))
        b.run(graph=False, learned=learned, timing=True)
        b.synchronize()
        stages, taps = b.timings()
        r = {"name": sc.name, "init": sc.init, "half_passes": sc.half_passes, "schedule": sc.kw,
             "sample": sc.sample, "active": sc.active, "accuracy": acc(), "ms": t,
             "stage_ms": {"proposal": stages[5], "init": stages[0], "halfpasses": stages[1],
                          "post": stages[2]},
             "halfpass_taps": taps[1]}
        if sc.name == PLAIN_3IT.name:
            plain_ms = t
        out["runs"].append(r)
        if log:
            log(f"{sc.name:28s} acc {r['accuracy']:.4f} {t:7.2f} ms  (proposal {stages[5]:.2f}, "
                f"init {stages[0]:.2f}, half-passes {stages[1]:.2f}, taps {taps[1] / 1e9:.2f}e9)")
    if plain_ms:
        for r in out["runs"]:
            r["speedup_vs_plain_3it"] = plain_ms / r["ms"]
    b.close()
    return out


if __name__ == "__main__":
    main()
