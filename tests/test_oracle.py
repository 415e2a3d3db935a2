"""CPU tests: the oracles themselves.

The C restatement (``oracle/depthmap_oracle.c``) is pinned against golden
vectors produced by the reference's own ``depthmap.cc`` (tests/golden/), and,
where the compiled reference is present, against it directly.  Bit-exact:
brute force, plane scoring, the median post-process, cleaner and pruner.
"""
import numpy as np
import pytest

import oracle as O
from opensfm_b200 import synthetic as S
from conftest import cams

EST_CASES = ["estimator_80x60_v3_p7.npz", "estimator_72x54_v4_p5.npz"]


@pytest.mark.parametrize("name", EST_CASES)
def test_port_brute_force_matches_golden(golden, name):
    g = golden(name)
    out = O.port_compute(0, list(g["K"]), list(g["R"]), list(g["t"]), list(g["images"]),
                         list(g["masks"]), int(g["patch_size"]), float(g["min_depth"]),
                         float(g["max_depth"]), int(g["num_planes"]), 3,
                         float(g["min_patch_sd"]), 1)
    for a, key in zip(out, ["bf_depth", "bf_plane", "bf_score", "bf_nghbr"]):
        assert np.array_equal(a, g[key]), key


@pytest.mark.parametrize("name", EST_CASES)
def test_port_score_planes_matches_golden(golden, name):
    g = golden(name)
    s, n = O.port_score_planes(list(g["K"]), list(g["R"]), list(g["t"]), list(g["images"]),
                               g["planes"], int(g["patch_size"]))
    assert np.array_equal(s, g["sp_score"])
    assert np.array_equal(n, g["sp_nghbr"])


@pytest.mark.parametrize("name", EST_CASES)
def test_port_median_matches_golden(golden, name):
    g = golden(name)
    assert np.array_equal(O.port_median5(g["median_in"]), g["median_out"])


def test_port_clean_prune_match_golden(golden):
    g = golden("clean_prune_64x48_v4.npz")
    K, R, t = list(g["K"]), list(g["R"]), list(g["t"])
    d = list(g["depths"])
    assert np.array_equal(O.port_clean(K, R, t, d, 0.01, 3), g["clean_t01_v3"])
    assert np.array_equal(O.port_clean(K, R, t, d, 0.02, 2), g["clean_t02_v2"])
    pts, nrm, col, lab = O.port_prune(K, R, t, d, list(g["planes"]), list(g["colors"]),
                                      list(g["labels"]), 0.01)
    assert len(lab) > 0
    assert np.array_equal(pts, g["prune_points"])
    assert np.array_equal(nrm, g["prune_normals"])
    assert np.array_equal(col, g["prune_colors"])
    assert np.array_equal(lab, g["prune_labels"])


def test_fp64_ncc_close_to_reference(golden):
    """The float64 restatement agrees with the reference's float NCC to ~1e-3
    on the median pixel (its job is to be the more exact of the two)."""
    g = golden(EST_CASES[0])
    s64, _ = O.ncc_fp64(list(g["K"]), list(g["R"]), list(g["t"]), list(g["images"]),
                        g["bf_plane"], int(g["patch_size"]))
    m = g["bf_depth"] > 0
    err = np.abs(s64[m] - g["bf_score"][m])
    assert np.median(err) < 1e-4
    assert np.mean(err < 1e-3) > 0.98


def _mixed(g):
    n = int(g["n_views"])
    return ([g[f"K_{k}"] for k in range(n)], [g[f"R_{k}"] for k in range(n)],
            [g[f"t_{k}"] for k in range(n)], [g[f"image_{k}"] for k in range(n)])


def test_fp64_ncc_mixed_sizes_close_to_reference(golden):
    """Views of different sizes: the float64 restatement samples each view
    with its own size, as the reference does (depthmap.cc:16)."""
    g = golden("estimator_mixed_v4_p7.npz")
    Ks, Rs, ts, ims = _mixed(g)
    assert len({im.shape for im in ims}) == len(ims)
    s64, n64 = O.ncc_fp64(Ks, Rs, ts, ims, g["bf_plane"], int(g["patch_size"]))
    m = g["bf_depth"] > 0
    err = np.abs(s64[m] - g["bf_score"][m])
    assert np.median(err) < 1e-4
    assert np.mean(err < 1e-3) > 0.98
    s64, n64 = O.ncc_fp64(Ks, Rs, ts, ims, g["planes"], int(g["patch_size"]))
    inner = np.zeros(m.shape, bool)
    inner[3:-3, 3:-3] = True
    err = np.abs(s64 - g["sp_score"])[inner]
    assert np.mean(err < 2e-3) > 0.98


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference not built")
def test_port_matches_compiled_reference_fresh_scene():
    vs = S.ring_viewset(21, 4, 72, 56)
    Ks, Rs, ts = cams(vs)
    mn, mx = S.depth_range(vs.depths[0])
    masks = [np.ones_like(im) for im in vs.images]
    e = O.RefEstimator()
    for K, R, t, im, mk in zip(Ks, Rs, ts, vs.images, masks):
        e.add_view(K, R, t, im, mk)
    e.set_depth_range(mn, mx, 12)
    e.set_patch_size(7)
    e.set_min_patch_sd(1.0)
    ref = e.compute_brute_force()
    port = O.port_compute(0, Ks, Rs, ts, vs.images, masks, 7, mn, mx, 12, 3, 1.0, 1)
    for a, b in zip(ref, port):
        assert np.array_equal(a, b)


def test_shim_inverse_and_median_match_cv2():
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(0)
    L = O.port()
    for _ in range(50):
        a = rng.normal(size=(3, 3))
        a[2] = [0, 0, 1] if rng.random() < 0.5 else a[2]
        out = np.zeros(9)
        aa = np.ascontiguousarray(a)
        L.or_inv3(O._P(aa, O._d), O._P(out, O._d))
        ok, inv = cv2.invert(aa, flags=cv2.DECOMP_LU)
        assert np.array_equal(out.reshape(3, 3), inv)
    d = rng.uniform(0, 10, size=(37, 23)).astype(np.float32)
    d[rng.random(d.shape) < 0.3] = 0
    assert np.array_equal(O.port_median5(d), cv2.medianBlur(d, 5))


def test_port_patchmatch_accuracy_close_to_reference():
    """The port's PatchMatch (own RNG) reaches the reference's accuracy band."""
    if not O.ref_available():
        pytest.skip("compiled reference not built")
    vs = S.ring_viewset(5, 4, 96, 72)
    Ks, Rs, ts = cams(vs)
    mn, mx = S.depth_range(vs.depths[0])
    masks = [np.ones_like(im) for im in vs.images]
    O.ref().ref_srand(3)
    e = O.RefEstimator()
    for K, R, t, im, mk in zip(Ks, Rs, ts, vs.images, masks):
        e.add_view(K, R, t, im, mk)
    e.set_depth_range(mn, mx, 32)
    e.set_patch_size(7)
    e.set_min_patch_sd(1.0)
    e.set_patchmatch_iterations(3)
    ref = e.compute_patch_match()
    port = O.port_compute(1, Ks, Rs, ts, vs.images, masks, 7, mn, mx, 32, 3, 1.0, 7)
    gt = vs.depths[0]
    a_ref = S.accuracy(ref[0], gt)
    a_port = S.accuracy(port[0], gt)
    assert abs(a_ref - a_port) < 0.1


def test_redblack_schedule_gap_to_the_raster_sweep():
    """The GPU's red-black schedule, restated with the reference's arithmetic
    (or_compute_redblack), against the reference's raster schedule with the
    same arithmetic (or_compute, bit-identical to depthmap.cc), on the
    320 x 240 benchmark scene with fixed seeds: the red-black result is
    slightly less accurate (the pinned fixture's gap) because fewer of its
    pixels survive the 5 x 5 median post-process; and the restatement
    reproduces the fixture's red-black accuracies."""
    import os
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_pm_configs as M

    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                             "pm_config1_320x240.npz"))
    cams_, images, depths = M.config1_views()
    Ks, Rs, ts = [c.K for c in cams_], [c.R for c in cams_], [c.t for c in cams_]
    masks = [np.ones_like(im) for im in images]
    mn, mx, gt = float(z["min_depth"]), float(z["max_depth"]), depths[0]
    raster = O.port_compute(1, Ks, Rs, ts, images, masks, 7, mn, mx, 64, 3, 1.0, 1)[0]
    rb = O.port_compute_redblack(Ks, Rs, ts, images, masks, 7, mn, mx, 6, 1.0, 1)[0]
    a_raster, a_rb = S.accuracy(raster, gt), S.accuracy(rb, gt)
    v_raster, v_rb = float((raster > 0).mean()), float((rb > 0).mean())
    print("raster %.4f (valid %.4f) red-black %.4f (valid %.4f); fixture: reference %.4f, "
          "red-black %.4f" % (a_raster, v_raster, a_rb, v_rb, z["pm_accuracy"].mean(),
                              z["rb_accuracy"].mean()))
    assert 0.0 < a_raster - a_rb < 0.01
    assert v_rb < v_raster
    assert abs(a_rb - z["rb_accuracy"].mean()) <= 0.003
    assert abs(a_raster - z["pm_accuracy"].mean()) <= 0.003


# ---------------------------------------------------------------- Philox
def philox_py(ctr, key):
    M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
    c = list(ctr)
    k0, k1 = key
    for r in range(10):
        if r:
            k0 = (k0 + W0) & 0xFFFFFFFF
            k1 = (k1 + W1) & 0xFFFFFFFF
        p0 = M0 * c[0]
        p1 = M1 * c[2]
        c = [((p1 >> 32) ^ c[1] ^ k0) & 0xFFFFFFFF, p1 & 0xFFFFFFFF,
             ((p0 >> 32) ^ c[3] ^ k1) & 0xFFFFFFFF, p0 & 0xFFFFFFFF]
    return c


def test_philox_known_answers():
    """Philox-4x32-10 known-answer vectors published with Random123."""
    assert philox_py([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    f = 0xFFFFFFFF
    assert philox_py([f, f, f, f], [f, f]) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert philox_py([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


# ------------------------------------------------------------------- KATs
def _fronto_setup(W=40, H=32, seed=0):
    rng = np.random.default_rng(seed)
    img = rng.integers(0, 256, size=(H, W)).astype(np.uint8)
    K = S.intrinsics(W, H)
    R = np.eye(3)
    t = np.zeros(3)
    return img, K, R, t


def test_kat_identical_views_true_plane_scores_one():
    """Same camera twice: the homography is the identity for any plane, NCC = 1.

    Patches touching the last row or column are excluded: LinearInterpolation
    returns 0 for x >= W - 1 or y >= H - 1 (depthmap.cc:16-18), so those taps
    sample 0 even under the identity warp."""
    img, K, R, t = _fronto_setup()
    H, W = img.shape
    planes = np.zeros((H, W, 3), np.float32)
    planes[..., 2] = -1.0 / 10.0
    s, n = O.port_score_planes([K, K], [R, R], [t, t], [img, img], planes, 7)
    inner = s[3:-4, 3:-4]
    assert np.allclose(inner, 1.0, atol=1e-5)
    assert (n[3:-4, 3:-4] == 1).all()
    assert (s[-4, 3:-4] < 1.0 - 1e-4).any()


def test_kat_affine_intensity_change_keeps_ncc():
    img, K, R, t = _fronto_setup(seed=1)
    H, W = img.shape
    other = np.clip(np.round(0.5 * img.astype(np.float64) + 20), 0, 255).astype(np.uint8)
    planes = np.zeros((H, W, 3), np.float32)
    planes[..., 2] = -0.1
    s, _ = O.port_score_planes([K, K], [R, R], [t, t], [img, other], planes, 7)
    # 0.5 x + 20 rounds to integers, so NCC is within rounding noise of 1.
    assert np.median(s[3:-4, 3:-4]) > 0.995


def test_kat_flat_patch_scores_minus_one():
    img, K, R, t = _fronto_setup()
    flat = np.full_like(img, 77)
    H, W = img.shape
    planes = np.zeros((H, W, 3), np.float32)
    planes[..., 2] = -0.1
    s, n = O.port_score_planes([K, K], [R, R], [t, t], [img, flat], planes, 7)
    assert (s[3:-4, 3:-4] == -1).all()
    assert (n[3:-4, 3:-4] == 0).all()


def test_kat_plane_depth_round_trip():
    """Brute-force planes are fronto-parallel: depth_of_plane(plane(d)) == d."""
    g = np.load(__import__("os").path.join(__import__("os").path.dirname(__file__), "golden",
                                           EST_CASES[0]))
    d = g["bf_depth"]
    p = g["bf_plane"]
    m = d > 0
    assert np.allclose(-1.0 / p[m][:, 2], d[m], rtol=1e-6)


def test_gpu_cleaner_oracle_known_answers():
    """GPUDepthmapCleaner restatement: a view against itself is consistent
    everywhere; a neighbour that sees farther everywhere carves every point;
    one that sees nearer (an occluder) neither confirms nor carves."""
    vs = S.ring_viewset(3, 2, 48, 36)
    Ks, Rs, ts = cams(vs)
    d = vs.depths[0].astype(np.float32)
    same = O.gpu_clean_fp32([Ks[0]] * 2, [Rs[0]] * 2, [ts[0]] * 2, [d, d], 0, [1],
                            0.01, 2, 0.2, 1)
    inner = np.zeros_like(d, bool)
    inner[1:-2, 1:-2] = True
    assert np.array_equal(same[inner], d[inner])
    far = O.gpu_clean_fp32([Ks[0]] * 2, [Rs[0]] * 2, [ts[0]] * 2, [d, d * 1.5], 0, [1],
                           0.01, 1, 0.2, 1)
    assert not far[inner].any()
    near = O.gpu_clean_fp32([Ks[0]] * 2, [Rs[0]] * 2, [ts[0]] * 2, [d, d * 0.5], 0, [1],
                            0.01, 1, 0.2, 1)
    assert np.array_equal(near, d)


def test_fuser_oracle_known_answers():
    """DepthmapFuser restatement: with two identical views each pixel of the
    first fuses with its twin (2 observations, the point it back-projects
    to), the twin's pixels are then used up, and asking for 3 observations
    fuses nothing."""
    vs = S.ring_viewset(3, 1, 40, 30)
    c = vs.cameras[0]
    d = vs.depths[0].astype(np.float32)
    H, W = d.shape
    n = np.zeros((H, W, 3), np.float32)
    n[..., 2] = -1.0
    col = np.stack([vs.images[0]] * 3, -1)
    view = dict(K=c.K, R=c.R, t=c.t, depth=d, normal=n, color=col, mask=None)
    views = [dict(view, neighbor_ids=[1]), dict(view, neighbor_ids=[0])]
    pts, nrm, clr = O.port_fuse(views, min_num_consistent=2, border_margin=2)
    inner = np.zeros((H, W), bool)
    inner[2:-2, 2:-2] = True
    assert len(pts) == int((inner & (d > 0)).sum())
    ii, jj = np.nonzero(inner & (d > 0))
    ray = np.stack([jj, ii, np.ones_like(jj)], -1) @ np.linalg.inv(c.K).T
    world = (ray * d[ii, jj][:, None] - c.t) @ c.R
    assert np.allclose(pts, world, rtol=1e-5, atol=1e-4)
    assert np.array_equal(clr, col[ii, jj])
    assert np.allclose(nrm, np.tile(-c.R[2], (len(pts), 1)), atol=1e-6)
    none = O.port_fuse(views, min_num_consistent=3, border_margin=2)
    assert len(none[0]) == 0


def test_sor_oracle_known_answers():
    """Outlier removal restatement: on a unit grid every interior point's 4
    nearest neighbours lie at distance 1 (mean exactly 1), a far point is
    removed, and with knn = 0 or too few points nothing is removed."""
    g = np.stack(np.meshgrid(np.arange(10.0), np.arange(10.0), indexing="ij"), -1).reshape(-1, 2)
    pts = np.concatenate([np.c_[g, np.zeros(len(g))], [[100.0, 100.0, 100.0]]]).astype(np.float32)
    keep, mk = O.port_sor(pts, 4, 2.5)
    interior = (g[:, 0] > 0) & (g[:, 0] < 9) & (g[:, 1] > 0) & (g[:, 1] < 9)
    assert np.all(mk[:-1][interior] == 1.0)
    corner = np.float32((np.float32(1) + np.float32(1) + np.sqrt(np.float32(2))
                         + np.float32(2)) / np.float32(4))
    assert mk[0] == corner
    assert keep[:-1].all() and not keep[-1]
    assert O.port_sor(pts, 0, 2.5)[0].all()
    assert O.port_sor(pts[:5], 4, 2.5)[0].all()  # n <= k + 1: skipped


def test_sor_oracle_matches_numpy_restatement():
    """The C brute force against a float32 numpy restatement of the same
    arithmetic (squared distance summed x, y, z; K smallest; float square
    roots summed in ascending order; double statistics)."""
    rng = np.random.default_rng(5)
    pts = rng.normal(0, 1, (600, 3)).astype(np.float32)
    pts[:20] *= 8  # a few far points
    K, fac = 6, 1.5
    keep, mk = O.port_sor(pts, K, fac)
    d = pts[:, None, :] - pts[None, :, :]
    d2 = (d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1]) + d[..., 2] * d[..., 2]
    np.fill_diagonal(d2, np.inf)
    nn = np.sort(d2, axis=1)[:, :K]
    want = np.zeros(len(pts), np.float32)
    for m in range(K):
        want = want + np.sqrt(nn[:, m])
    want = want / np.float32(K)
    assert np.array_equal(mk, want)
    s = 0.0
    s2 = 0.0
    for v in want.astype(np.float64):
        s += v
        s2 += v * v
    mean = s / len(pts)
    thr = np.float32(mean + np.float64(np.float32(fac)) * np.sqrt(max(0.0, s2 / len(pts) - mean * mean)))
    assert np.array_equal(keep, want <= thr)
    assert 0 < (~keep).sum() < 40


def _plane_view(Z=2.0, W=64, H=48, f=60.0, color=(100, 150, 200)):
    K = np.array([[f, 0, W / 2], [0, f, H / 2], [0, 0, 1.0]])
    nrm = np.zeros((H, W, 3), np.float32)
    nrm[..., 2] = -1.0
    return dict(K=K, R=np.eye(3), t=np.zeros(3), depth=np.full((H, W), Z, np.float32),
                normal=nrm, color=np.tile(np.array(color, np.uint8), (H, W, 1)))


def test_svo_oracle_known_answers():
    """SVO fusion restatement on a fronto-parallel plane seen by a camera at
    the origin: the TSDF's zero crossing lies on the plane, the normals are
    the plane's, the colour is the views' (within the truncation of the
    weighted average), and the counting pass covers every fused voxel."""
    v = _plane_view()
    cnt, pts, nrm, clr = O.port_svo([v], voxel_size=0.05, trunc_factor=4.0, min_weight=1.0)
    assert len(pts) > 100 and cnt >= len(pts) // 3
    assert np.all(np.abs(pts[:, 2] - 2.0) < 1e-3)
    assert np.allclose(nrm, [0, 0, -1], atol=1e-6)
    assert np.all(np.abs(clr.astype(int) - [100, 150, 200]) <= 1)
    # min_weight above what the view gives: nothing is extracted.
    assert len(O.port_svo([v], voxel_size=0.05, min_weight=1e4)[1]) == 0
    # The same view twice doubles every sum: the averages, the voxels and
    # the points stay the same.
    cnt2, pts2, _, _ = O.port_svo([v, v], voxel_size=0.05, min_weight=1.0)
    assert cnt2 == cnt and np.array_equal(pts2, pts)
    # A box around part of the plane keeps only its voxels.
    _, pb, _, _ = O.port_svo([v], voxel_size=0.05, min_weight=1.0,
                             bbox=([-0.5, -0.5, 1.5], [0.0, 0.5, 2.5]))
    assert 0 < len(pb) < len(pts)
    assert np.all(pb[:, 0] <= 0.0 + 0.05) and np.all(pb[:, 0] >= -0.5 - 0.05)
    # Points come in ascending voxel order.
    k = np.floor(pts / 0.05).astype(np.int64)
    order = np.lexsort((k[:, 2], k[:, 1], k[:, 0]))
    assert np.array_equal(order, np.arange(len(pts))) or len(np.unique(k, axis=0)) < len(k)


def test_acmmp_oracle_exp_log_accuracy():
    """The live estimator's own exp and log (Cody-Waite reduction, fixed
    polynomials), which the library and the oracle share by construction:
    within 2 ulp of float64 over the ranges the estimator uses."""
    import ctypes
    L = O.port()
    L.acm_exp.argtypes = [ctypes.c_float]
    L.acm_exp.restype = ctypes.c_float
    L.acm_log.argtypes = [ctypes.c_float]
    L.acm_log.restype = ctypes.c_float
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-87, 88, 3000), rng.uniform(-2, 2, 3000),
                         [0.0, -0.0, 1.0, -1.0, 88.7, -87.0]]).astype(np.float32)
    for x in xs:
        got = np.float32(L.acm_exp(float(x)))
        want = np.exp(np.float64(x))
        assert abs(float(got) - want) <= 2 * float(np.spacing(np.float32(want))), x
    ys = np.concatenate([10.0 ** rng.uniform(-6, 6, 3000), rng.uniform(0.5, 2, 2000)]).astype(np.float32)
    for y in ys:
        got = np.float32(L.acm_log(float(y)))
        want = np.log(np.float64(y))
        assert abs(float(got) - want) <= 2 * float(np.spacing(np.float32(max(abs(want), 1e-7)))) + 1e-7, y
    assert L.acm_exp(-200.0) == 0.0 and np.isinf(L.acm_exp(100.0))


def test_acmmp_oracle_known_answers():
    """The live estimator restated: with the source identical to the
    reference (same camera), every plane maps each pixel onto itself, so on
    texture the NCC is 1 and the initial cost 0 (to rounding); and on a
    textured ring scene the estimator recovers most depths within 5 %."""
    vs = S.ring_viewset(3, 4, 96, 72)
    c = vs.cameras[0]
    views = [(c.K, c.R, c.t, vs.images[0])] * 2
    dmin, dmax = S.depth_range(vs.depths[0])
    planes, costs, sel = O.port_acmmp_init(views, dmin, dmax, patch_size=5)
    assert planes.shape == (72, 96, 4) and np.isfinite(planes).all()
    assert np.all((costs >= -1e-5) & (costs <= 2)) and np.all(sel <= 1)
    textured = vs.images[0][2:-2, 2:-2].std() > 5
    assert textured and np.median(costs[4:-4, 4:-4]) < 1e-3
    d, n, cost, conf = O.port_acmmp([(cc.K, cc.R, cc.t, im) for cc, im in
                                     zip(vs.cameras, vs.images)], dmin, dmax, iterations=3,
                                    patch_size=7)
    gt = vs.depths[0]
    m = (d > 0) & (gt > 0)
    assert m.mean() > 0.3
    rel = np.abs(d[m] - gt[m]) / gt[m]
    assert np.median(rel) < 0.05
    assert np.all((conf[d > 0] > 0) & (conf[d > 0] < 1)) and np.all(conf[d == 0] == 0)
    assert np.allclose(np.linalg.norm(n[d > 0], axis=-1), 1, atol=1e-5)


def test_acmmp_pyramid_resizes_against_opencv():
    """The estimator's pyramid: cv::resize(INTER_AREA) by 2, 4 and 8 is
    reproduced exactly, on the fast path (integer ratios) and on the general
    area path (sizes that do not divide); the previous-depth bilinear resize
    follows OpenCV's
    INTER_LINEAR mapping and agrees to a few ulp (OpenCV's SIMD arithmetic
    differs in the last bits, so the library fixes its own order)."""
    cv2 = pytest.importorskip("cv2")
    rng = np.random.default_rng(7)
    for k in (2, 4, 8):
        for H, W in ((48, 64), (96, 128), (40, 56)):
            if H % k or W % k:
                continue
            im = rng.integers(0, 256, (H, W), dtype=np.uint8)
            want = cv2.resize(im, (W // k, H // k), interpolation=cv2.INTER_AREA)
            assert np.array_equal(O.acm_resize_area(im, k), want), (k, H, W)
    for _ in range(60):
        H, W = (int(v) for v in rng.integers(5, 150, 2))
        s = float(rng.choice([0.5, 0.25, 0.125]))
        h, w = max(1, int(H * s)), max(1, int(W * s))
        im = rng.integers(0, 256, (H, W), dtype=np.uint8)
        want = cv2.resize(im, (w, h), interpolation=cv2.INTER_AREA)
        assert np.array_equal(O.acm_resize_area_to(im, w, h), want), (H, W, h, w)
    d = rng.uniform(1, 30, (24, 32)).astype(np.float32)
    d[rng.random(d.shape) < 0.2] = 0
    got = O.acm_resize_linear(d, 64, 48)
    want = cv2.resize(d, (64, 48), interpolation=cv2.INTER_LINEAR)
    assert np.allclose(got, want, rtol=1e-6, atol=1e-6)


def test_acmmp_oracle_matches_its_regression_fixture():
    """The cluster estimator's C restatement reproduces, bit for bit, the
    outputs stored by tests/golden/make_acmmp_regression.py: one level with
    smoothness, and two levels with geometric links and the planar prior."""
    import os

    f = np.load(os.path.join(os.path.dirname(__file__), "golden", "acmmp_oracle_regression.npz"))
    view = lambda i: (f["K"][i], f["R"][i], f["t"][i], f["images"][i])  # noqa: E731
    rg = f["ranges"]
    a = O.port_acmmp([view(i) for i in (0, 1, 2, 5)], rg[0, 0], rg[0, 1], iterations=2,
                     patch_size=5, smooth_weight=0.2)
    for name, arr in zip(("depth", "normal", "cost", "conf"), a):
        assert np.array_equal(arr, f["a_" + name]), name
    refs = [dict(views=[view(i) for i in (0, 1, 2, 5)], depth_min=rg[0, 0], depth_max=rg[0, 1],
                 sfm=f["sfm0"]),
            dict(views=[view(i) for i in (1, 0, 2, 3)], depth_min=rg[1, 0], depth_max=rg[1, 1],
                 sfm=f["sfm1"])]
    b = O.port_acmmp_cluster(refs, hierarchy_levels=2, iterations=2, patch_size=5,
                             geom_weight=0.2, geom_links=[(0, 0, 1), (1, 0, 0)])
    for r, res in enumerate(b):
        for name, arr in zip(("depth", "normal", "cost", "conf"), res):
            assert np.array_equal(arr, f[f"b{r}_" + name]), (r, name)


def test_fusion_oracles_match_their_regression_fixture():
    """The restatements of the live cleaner, the per-pixel fuser (with and
    without outlier removal) and the SVO fuser reproduce, bit for bit, the
    outputs stored by tests/golden/make_fusion_regression.py."""
    import importlib.util
    import os

    here = os.path.join(os.path.dirname(__file__), "golden")
    spec = importlib.util.spec_from_file_location(
        "make_fusion_regression", os.path.join(here, "make_fusion_regression.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    f = dict(np.load(os.path.join(here, "fusion_oracle_regression.npz")))
    got = gen.outputs(f)
    assert set(got) <= set(f)
    for name, arr in got.items():
        assert np.array_equal(np.asarray(arr), f[name]), name
    assert 0 < len(f["fuse_sor_points"]) < len(f["fuse_points"])
    assert all(0 < (f[f"clean{r}"] > 0).sum() < (f["depth"][r] > 0).sum() for r in range(4))
