"""GPU tests of the learned-initialisation kernels: forward and backward of
the tensor-core 3x3 convolutions against a float64 PyTorch CPU oracle, the
loss / Adam kernels, and one training step of the whole network.

Tolerances: activations and weights are BF16 (8 bits of mantissa), sums are
FP32; results are compared relative to the oracle's largest magnitude:
single-layer outputs within 1e-2, gradients within 2e-2."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

if not gpu_available():
    pytest.skip("no CUDA device", allow_module_level=True)

torch = pytest.importorskip("torch")

from opensfm_b200 import _lib, learned  # noqa: E402


def _bf(t):
    return t.to(torch.bfloat16)


def _ref_conv(x_nhwc, w, b, relu):
    """float64 oracle: x (n, H, W, cin), w (cout, 9 cin) with k = tap * cin + ci."""
    n, H, W, cin = x_nhwc.shape
    cout = w.shape[0]
    wt = w.view(cout, 3, 3, cin).permute(0, 3, 1, 2)
    z = torch.nn.functional.conv2d(x_nhwc.permute(0, 3, 1, 2), wt, b, padding=1)
    y = torch.relu(z) if relu else z
    return y.permute(0, 2, 3, 1)


def _rel(a, b):
    return float((a - b).abs().max() / max(b.abs().max(), 1e-12))


@pytest.mark.parametrize("cout,relu", [(32, 1), (4, 0)])
def test_conv_forward_matches_float64(cout, relu):
    g = torch.Generator().manual_seed(cout)
    n, H, W, cin = 2, 9, 13, 32
    x = _bf(torch.randn((n, H, W, cin), generator=g))
    w = _bf(torch.randn((cout, 9 * cin), generator=g) * 0.1)
    b = torch.randn(cout, generator=g) * 0.1
    L = _lib.load()
    n_pix = n * H * W
    y32 = torch.empty((n_pix, cout), dtype=torch.float32, device="cuda")
    y16 = torch.empty((n_pix * cout,), dtype=torch.bfloat16, device="cuda")
    xd, wd, bd = x.cuda().contiguous(), w.cuda().contiguous(), b.cuda().contiguous()
    _lib.check(L.dn_nn_conv3x3_forward(learned._ptr(xd), learned._ptr(wd), learned._ptr(bd), n_pix,
                                       H, W, cin, cout, relu, learned._ptr(y16), learned._ptr(y32),
                                       None))
    _lib.check(L.dn_nn_synchronize(None))
    ref = _ref_conv(x.double(), w.double(), b.double(), relu).reshape(n_pix, cout)
    assert _rel(y32.cpu().double(), ref) < 1e-4  # FP32 accumulation of BF16 products
    assert _rel(y16.view(n_pix, cout).cpu().double(), ref) < 1e-2


@pytest.mark.parametrize("cout,relu", [(32, 1), (32, 0), (4, 0)])
def test_conv_forward_tcgen05_matches_mma_sync(cout, relu):
    """The tcgen05 forward (tensor-memory accumulators, 128-pixel tiles, CTAs
    looping over tiles) against the warp-level mma.sync forward on a batch
    large enough that every CTA takes several tiles, with a ragged last tile."""
    g = torch.Generator().manual_seed(7 + cout)
    n, H, W, cin = 2, 121, 203, 32
    n_pix = n * H * W
    x = _bf(torch.randn((n_pix, cin), generator=g)).cuda().contiguous()
    w = _bf(torch.randn((cout, 9 * cin), generator=g) * 0.1).cuda().contiguous()
    b = (torch.randn(cout, generator=g) * 0.1).cuda().contiguous()
    L = _lib.load()
    outs = []
    for fn in (L.dn_nn_conv3x3_forward, L.dn_nn_conv3x3_forward_mma_sync):
        y32 = torch.full((n_pix, cout), float("nan"), dtype=torch.float32, device="cuda")
        y16 = torch.full((n_pix * cout,), float("nan"), dtype=torch.bfloat16, device="cuda")
        _lib.check(fn(learned._ptr(x), learned._ptr(w), learned._ptr(b), n_pix, H, W, cin, cout,
                      relu, learned._ptr(y16), learned._ptr(y32), None))
        _lib.check(L.dn_nn_synchronize(None))
        outs.append((y32.cpu().double(), y16.cpu().double().view(n_pix, cout)))
    (a32, a16), (b32, b16) = outs
    assert torch.isfinite(a32).all() and torch.isfinite(a16).all()
    assert _rel(a32, b32) < 2e-6  # same BF16 products, FP32 sums in another order
    assert float((a16 - b16).abs().max()) <= float(b16.abs().max()) * 2 ** -7


@pytest.mark.parametrize("cout", [32, 4])
def test_conv_backward_matches_float64(cout):
    g = torch.Generator().manual_seed(100 + cout)
    n, H, W, cin = 2, 7, 11, 32
    x = _bf(torch.relu(torch.randn((n, H, W, cin), generator=g)))  # a ReLU output
    w = _bf(torch.randn((cout, 9 * cin), generator=g) * 0.1)
    dz = _bf(torch.randn((n, H, W, cout), generator=g))
    L = _lib.load()
    n_pix = n * H * W
    xd, wd, dzd = x.cuda().contiguous(), w.cuda().contiguous(), dz.cuda().contiguous()
    dx = torch.empty((n_pix * cin,), dtype=torch.bfloat16, device="cuda")
    dw = torch.zeros((cout, 9 * cin), dtype=torch.float32, device="cuda")
    db = torch.zeros((cout,), dtype=torch.float32, device="cuda")
    scratch = torch.empty(32 * 9 * 32, dtype=torch.bfloat16, device="cuda")
    P = learned._ptr
    _lib.check(L.dn_nn_conv3x3_backward(P(dzd), P(xd), P(wd), P(xd), n_pix, H, W, cin, cout, P(dx),
                                        P(dw), P(db), P(scratch), None))
    torch.cuda.synchronize()
    # float64 oracle via autograd: z = conv(x, w); dL/dz = dz.
    xr = x.double().requires_grad_(True)
    wr = w.double().requires_grad_(True)
    br = torch.zeros(cout, dtype=torch.float64, requires_grad=True)
    z = _ref_conv(xr, wr, br, 0)
    z.backward(dz.double())
    want_dx = xr.grad * (x.double() > 0)
    assert _rel(dw.cpu().double(), wr.grad) < 2e-2
    assert _rel(db.cpu().double(), br.grad) < 2e-2
    assert _rel(dx.view(n, H, W, cin).cpu().double(), want_dx) < 2e-2


@pytest.mark.parametrize("cout", [32, 4])
@pytest.mark.parametrize("shape", [(2, 7, 11), (3, 21, 19), (1, 48, 64)])
def test_conv_backward_tcgen05_matches_float64_and_mma_sync(cout, shape):
    """The tcgen05 backward (weight gradient in tensor memory, data gradient
    through the forward kernel on flipped weights) against float64 autograd
    and against the mma.sync backward, on tile-aligned and ragged images."""
    g = torch.Generator().manual_seed(200 + cout + shape[1])
    n, H, W = shape
    cin = 32
    x = _bf(torch.relu(torch.randn((n, H, W, cin), generator=g)))
    w = _bf(torch.randn((cout, 9 * cin), generator=g) * 0.1)
    dz = _bf(torch.randn((n, H, W, cout), generator=g))
    L = _lib.load()
    P = learned._ptr
    n_pix = n * H * W
    xd, wd, dzd = x.cuda().contiguous(), w.cuda().contiguous(), dz.cuda().contiguous()
    outs = []
    for tc in (True, False):
        dx = torch.empty((n_pix * cin,), dtype=torch.bfloat16, device="cuda")
        dw = torch.zeros((cout, 9 * cin), dtype=torch.float32, device="cuda")
        db = torch.zeros((cout,), dtype=torch.float32, device="cuda")
        if tc:
            nb = int(L.dn_nn_backward_scratch_bytes(n_pix, cout))
            scratch = torch.empty(nb, dtype=torch.uint8, device="cuda")
            _lib.check(L.dn_nn_conv3x3_backward_tc(P(dzd), P(xd), P(wd), P(xd), n_pix, H, W, cin,
                                                   cout, P(dx), P(dw), P(db), P(scratch), nb,
                                                   None))
        else:
            scratch = torch.empty(32 * 9 * 32, dtype=torch.bfloat16, device="cuda")
            _lib.check(L.dn_nn_conv3x3_backward(P(dzd), P(xd), P(wd), P(xd), n_pix, H, W, cin,
                                                cout, P(dx), P(dw), P(db), P(scratch), None))
        torch.cuda.synchronize()
        outs.append((dx.view(n, H, W, cin).cpu().double(), dw.cpu().double(), db.cpu().double()))
    xr = x.double().requires_grad_(True)
    wr = w.double().requires_grad_(True)
    br = torch.zeros(cout, dtype=torch.float64, requires_grad=True)
    _ref_conv(xr, wr, br, 0).backward(dz.double())
    want_dx = xr.grad * (x.double() > 0)
    (dx_t, dw_t, db_t), (dx_m, dw_m, db_m) = outs
    assert _rel(dw_t, wr.grad) < 2e-2 and _rel(db_t, br.grad) < 2e-2
    assert _rel(dx_t, want_dx) < 2e-2
    # Same BF16 products summed in FP32 in another order: FP32 rounding for
    # the weight gradient, one BF16 rounding step for the data gradient.
    assert _rel(dw_t, dw_m) < 1e-4 and _rel(db_t, db_m) < 1e-4
    assert float((dx_t - dx_m).abs().max()) <= float(dx_m.abs().max()) * 2 ** -7
    assert float(dx_t[x.double() <= 0].abs().max()) == 0.0


@pytest.mark.parametrize("tensor_cores", [True, False])
def test_network_gradient_matches_float64(tensor_cores):
    """Whole-network gradient of the L1 loss against float64 autograd on the
    same BF16-quantised weights and input (intermediate BF16 rounding is the
    only difference), through the tcgen05 and the mma.sync backward."""
    g = torch.Generator().manual_seed(7)
    n, H, W = 2, 10, 12
    net = learned.ProposalNet(seed=3)
    x = _bf(torch.randn((n, H, W, 32), generator=g) * 0.5)
    n_pix = n * H * W
    tgt = torch.rand((n_pix, 4), generator=g)
    tgt[:, 3] = (torch.rand(n_pix, generator=g) > 0.2).float()
    out, acts = net.forward(x.cuda().reshape(-1).contiguous(), n_pix, H, W, keep=True)
    L = _lib.load()
    P = learned._ptr
    loss = torch.zeros(1, device="cuda")
    cnt = torch.zeros(1, device="cuda")
    dpred = torch.empty(n_pix * 4, dtype=torch.bfloat16, device="cuda")
    tg = tgt.cuda().contiguous()
    _lib.check(L.dn_nn_l1_loss(P(out), P(tg), n_pix, 0.1, P(dpred), P(loss), P(cnt), None))
    dws, dbs = net.backward(acts, dpred, n_pix, H, W, tensor_cores=tensor_cores)
    torch.cuda.synchronize()
    # Oracle, rounding to BF16 where the kernels store BF16: each hidden
    # layer's output, and the gradient flowing into each layer's output.
    bf = lambda t: t.to(torch.bfloat16).double()  # noqa: E731
    ws = [w.cpu().to(torch.bfloat16).double().requires_grad_(True) for w in net.w32]
    bs = [b.cpu().double().requires_grad_(True) for b in net.b32]
    h = x.double()
    for k, (cin, cout, relu) in enumerate(learned.LAYERS):
        h = _ref_conv(h, ws[k], bs[k], relu)
        if k < len(learned.LAYERS) - 1:
            h = bf(h)
            h.register_hook(lambda g: bf(g))
    pred = h.reshape(n_pix, 4)
    pred.register_hook(lambda g: bf(g))
    wgt = tgt[:, 3].double()
    l = (wgt * ((pred[:, 0] - tgt[:, 0]).abs() + 0.1 * ((pred[:, 1] - tgt[:, 1]).abs() +
                                                        (pred[:, 2] - tgt[:, 2]).abs()))).sum()
    l.backward()
    assert abs(float(loss.item()) - float(l)) / float(l) < 2e-2
    assert abs(float(cnt.item()) - float(wgt.sum())) < 1e-3
    for k in range(len(learned.LAYERS)):
        assert _rel(dws[k].cpu().double(), ws[k].grad) < 2e-2, k
        assert _rel(dbs[k].cpu().double(), bs[k].grad) < 2e-2, k


def test_adam_step_matches_formula():
    L = _lib.load()
    P = learned._ptr
    w = torch.randn(1000, device="cuda")
    m = torch.zeros_like(w)
    v = torch.zeros_like(w)
    grad = torch.randn(1000, device="cuda")
    cnt = torch.tensor([4.0], device="cuda")
    w0 = w.clone()
    w16 = torch.empty(1000, dtype=torch.bfloat16, device="cuda")
    _lib.check(L.dn_nn_adam(P(w), P(m), P(v), P(grad), 1000, P(cnt), 0.01, 0.9, 0.999, 1e-8,
                            0.1, 0.001, P(w16), None))
    torch.cuda.synchronize()
    gr = grad / 4
    mk = 0.1 * gr
    vk = 0.001 * gr * gr
    want = w0 - 0.01 * (mk / 0.1) / (torch.sqrt(vk / 0.001) + 1e-8)
    assert torch.allclose(w, want, rtol=1e-5, atol=1e-6)
    assert torch.equal(w16, w.to(torch.bfloat16))


def test_short_training_reduces_loss():
    """Trains on 16 seeded scenes for 60 steps: the loss must drop."""
    seeds = list(range(500, 516))
    feat, tgt = learned.make_dataset(seeds, W=160, H=120, chunk=16, stride=1)
    net = learned.ProposalNet(seed=1)
    hist = learned.train(net, feat, tgt, len(seeds), 120, 160, steps=60, batch=4, lr=3e-3)
    assert hist[-1][1] < 0.8 * hist[0][1], hist


def test_trained_network_gains_over_random_initialisation():
    """The committed network (opensfm_b200/weights/proposal_net.npz) on 4
    held-out scenes at 640 x 480 (seeds beyond the training range): learned
    initialisation + k half-passes is more accurate than the reference's
    random initialisation (RandomInitialization, depthmap.cc:237-256) + the
    same k half-passes, for k = 1 and 2, with the same candidate sets.
    Accuracy = fraction of ground-truth pixels within 1 % relative depth;
    device time per run printed beside it."""
    seeds = [910000, 910001, 910002, 910003]
    scenes = [learned.make_scene(s, 640, 480) for s in seeds]
    net = learned.ProposalNet.load()
    scheds = []
    for k in (1, 2):
        scheds += [learned.Schedule(f"plain-{k}hp", "plain", k, {}),
                   learned.Schedule(f"learned-{k}hp", "learned", k, {})]
    res = learned.evaluate(net, seeds, scenes=scenes, schedules=scheds, repeats=2,
                           log=lambda s: print(s, flush=True))
    acc = {r["name"]: r["accuracy"] for r in res["runs"]}
    ms = {r["name"]: r["ms"] for r in res["runs"]}
    for k in (1, 2):
        print("k = %d: learned %.4f (%.2f ms) vs random %.4f (%.2f ms)"
              % (k, acc[f"learned-{k}hp"], ms[f"learned-{k}hp"], acc[f"plain-{k}hp"],
                 ms[f"plain-{k}hp"]))
        assert acc[f"learned-{k}hp"] > acc[f"plain-{k}hp"] + 0.05


def test_training_checkpoint_resume(tmp_path):
    """A checkpoint restores the training state exactly -- master weights,
    both Adam moments, the Adam step, the loop step and the batch sampler --
    and a run resumed from it follows the uninterrupted run: after 20 steps
    it is far closer to the uninterrupted run than a run that drew other
    batches.  (The weight gradients are summed with atomics in any order,
    and Adam divides by the root of the second moment, so two runs of the
    same batches agree closely but not bit for bit.)"""
    seeds = list(range(520, 528))
    feat, tgt = learned.make_dataset(seeds, W=160, H=120, chunk=8, stride=1)
    kw = dict(steps=20, batch=2, lr=3e-3)
    a = learned.ProposalNet(seed=3, stride=1)
    learned.train(a, feat, tgt, len(seeds), 120, 160, **kw)
    b = learned.ProposalNet(seed=3, stride=1)
    ck = str(tmp_path / "checkpoint.npz")
    learned.train(b, feat, tgt, len(seeds), 120, 160, stop_step=10, checkpoint=ck, **kw)
    c, start, g = learned.load_checkpoint(ck)
    assert start == 10 and c.step == b.step == 10 and c.stride == 1
    for x, y in zip(b.w32 + b.b32 + b.m + b.v, c.w32 + c.b32 + c.m + c.v):
        assert torch.equal(x, y)
    for x, y in zip(b.w16, c.w16):
        assert torch.equal(x, y)
    learned.train(c, feat, tgt, len(seeds), 120, 160, start_step=start, generator=g, **kw)
    assert c.step == a.step == 20
    d = learned.ProposalNet(seed=3, stride=1)
    learned.train(d, feat, tgt, len(seeds), 120, 160, seed=1, **kw)

    def dist(p, q):
        return max(float((x - y).abs().max()) for x, y in zip(p.w32, q.w32))

    assert dist(a, d) > 1e-3
    assert dist(a, c) < 0.2 * dist(a, d), (dist(a, c), dist(a, d))


def test_headline_schedule_reaches_plain_accuracy_on_unseen_scenes():
    """The bench's first learned schedule (chosen on held-out seeds
    900000-900011) on 4 other scenes at 640 x 480 (seeds 920000-920003,
    outside the training and the selection seeds): its accuracy@1 % is at
    least the plain schedule's (the reference's random initialisation,
    every view per candidate, 3 iterations), and it is several times
    faster (device time of CUDA-graph replays; printed)."""
    import bench

    seeds = [920000, 920001, 920002, 920003]
    scenes = [learned.make_scene(s, 640, 480) for s in seeds]
    plain, scheds = bench.schedules()
    res = learned.evaluate(learned.ProposalNet.load(), seeds, scenes=scenes,
                           schedules=[plain, scheds[0]], repeats=3)
    r = {x["name"]: x for x in res["runs"]}
    p, q = r[plain.name], r[scheds[0].name]
    print(f"plain {p['accuracy']:.4f} {p['ms']:.2f} ms, {q['name']} {q['accuracy']:.4f} "
          f"{q['ms']:.2f} ms, x{p['ms'] / q['ms']:.2f}")
    assert q["accuracy"] >= p["accuracy"]
    assert p["ms"] / q["ms"] >= 4.0


def test_per_map_proposal_stride_matches_a_batch_of_that_size():
    """With the training size recorded (Batch.set_proposal_scale), a 320 x 240
    map batched with a 640 x 480 map gets the stride-2 grid that the network's
    stride-4, 640 x 480 training scale asks for: its proposal (a learned run
    without half-passes) equals the same map's alone at stride 2.  Without
    the scale it shares the stride-4 grid, and differs."""
    net = learned.ProposalNet.load()
    assert net.stride == 4 and net.train_dim == 640
    small = learned.make_scene(930000, 320, 240)
    large = learned.make_scene(930001, 640, 480)
    w, bias = net.packed()

    def run(scenes, stride, scale):
        b, maps = learned.build_batch(scenes, seed=5)
        b.set_proposal_net(w, bias, n_planes=net.n_planes, stride=stride)
        b.set_proposal_scale(scale)
        b.set_schedule(half_passes=0)
        b.run(learned=True)
        b.synchronize()
        out = [b.get_depth(m) for m in maps]
        b.close()
        return out

    scaled = run([small, large], 4, 640)
    alone = run([small], 2, 0)
    assert np.array_equal(scaled[0], alone[0])
    assert (scaled[0] > 0).mean() > 0.3
    assert (scaled[1] > 0).mean() > 0.3
    one_stride = run([small, large], 4, 0)
    assert not np.array_equal(one_stride[0], scaled[0])
    assert np.array_equal(one_stride[1], scaled[1])


@pytest.mark.parametrize("mode", [0, 2])
def test_random_initialisation_fallback_keeps_the_better_plane(mode):
    """With the fallback on, the learned proposal competes with the
    reference's random plane per pixel (same view(s)): after the
    initialisation alone every pixel's score is at least its score with the
    proposal alone, and pixels that switch score strictly higher."""
    net = learned.ProposalNet.load()
    scenes = [learned.make_scene(s, 640, 480) for s in (940000, 940001)]
    out = {}
    for fb in (False, True):
        b, maps = learned.build_batch(scenes, seed=3)
        learned.install(net, b)
        learned.Schedule("init", "learned", 0, {}, sample=mode, fallback=fb).apply(b)
        b.run(learned=True)
        b.synchronize()
        out[fb] = [b.get(m) for m in maps]
        b.close()
    switched = 0
    for (d0, p0, s0, n0), (d1, p1, s1, n1) in zip(out[False], out[True]):
        valid = p0[..., 2] != 0
        assert (s1[valid] >= s0[valid]).all()
        moved = valid & (p1 != p0).any(axis=-1)
        assert (s1[moved] > s0[moved]).all()
        switched += int(moved.sum())
    assert switched > 0
