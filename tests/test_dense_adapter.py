"""GPU test of the dense.py stand-in (opensfm_b200.dense_adapter): raw and
clean depthmap files written in OpenSfM's layout must hold exactly what the
batch API and DepthmapCleaner compute for the same views."""
import numpy as np
import pytest

from conftest import gpu_available
from opensfm_b200 import synthetic as S

pytestmark = pytest.mark.gpu

if not gpu_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from opensfm_b200 import dense_adapter, dense_io, pydense  # noqa: E402


@pytest.fixture(scope="module")
def views():
    vs = S.ring_viewset(7, 5, 160, 120)
    ids = [f"img_{k:02d}.jpg" for k in range(5)]
    v = {i: (c.K, c.R, c.t, im) for i, c, im in zip(ids, vs.cameras, vs.images)}
    bn = {ids[k]: [ids[k]] + [ids[o] for o in vs.neighbors(k, 4)] for k in range(5)}
    dr = {ids[k]: S.depth_range(vs.depths[k]) for k in range(5)}
    return ids, v, bn, dr, vs


def test_raw_and_clean_files_match_the_library(tmp_path, views):
    ids, v, bn, dr, vs = views
    d = str(tmp_path)
    cfg = {"depthmap_num_matching_views": 3, "depthmap_patch_size": 7,
           "depthmap_min_consistent_views": 2}
    done = dense_adapter.compute_raw_depthmaps(d, v, bn, dr, ids, cfg, seed=4)
    assert done == ids
    # The same batch built directly.
    b = pydense.Batch()
    index = {}
    for i in ids:
        K, R, t, im = v[i]
        index[i] = b.add_view(K, R, t, im)
    for i in ids:
        b.add_depthmap(index[i], [index[n] for n in bn[i][1:4]], *dr[i])
    b.set_params(patch_size=7, min_patch_sd=1.0, iterations=3, seed=4)
    b.run()
    b.synchronize()
    for m, i in enumerate(ids):
        depth, plane, score, nghbr, nghbrs, conf = dense_io.load_raw_depthmap(d, i)
        want = b.get(m)
        for a, w in zip((depth, plane, score, nghbr), want):
            assert a.dtype == w.dtype and np.array_equal(a, w)
        assert list(nghbrs) == bn[i] and conf is None
        assert S.accuracy(depth, vs.depths[m]) > 0.3
    b.close()

    done = dense_adapter.clean_depthmaps(d, v, bn, ids, cfg)
    assert done == ids
    for i in ids:
        raw = dense_io.load_raw_depthmap(d, i)
        c = pydense.DepthmapCleaner()
        c.set_same_depth_threshold(0.01)
        c.set_min_consistent_views(2)
        K, R, t, _ = v[i]
        c.add_view(K, R, t, raw[0])
        for n in bn[i][1:]:
            Kn, Rn, tn, _ = v[n]
            c.add_view(Kn, Rn, tn, dense_io.load_raw_depthmap(d, n)[0])
        want = c.clean()
        depth, plane, score, conf = dense_io.load_clean_depthmap(d, i)
        assert np.array_equal(depth, want)
        assert np.array_equal(plane, raw[1]) and not score.any()
        assert (depth > 0).sum() < (raw[0] > 0).sum()


def test_live_stages_write_what_the_live_classes_compute(tmp_path, views):
    """run_cluster_raw / clean_cluster_gpu (the stand-ins for dense.py's
    live call sites) write exactly what DepthmapClusterEstimator and
    GPUDepthmapCleaner give when driven as dense.py drives them, in the live
    path's raw fields (dense.py:741-775) and clean fields (dense.py:896-905)."""
    ids, v, bn, dr, vs = views
    d = str(tmp_path)
    cfg = {"depthmap_num_matching_views": 3, "depthmap_hierarchy_levels": 2,
           "depthmap_max_iterations": 2, "depthmap_patch_size": 5,
           "depthmap_sfm_planar_prior": False, "depthmap_min_consistent_views": 2}
    cluster = ids[1:4]
    done = dense_adapter.run_cluster_raw(d, v, bn, cluster, dr, cfg)
    assert done == cluster
    # The same cluster, driven directly.
    c = pydense.DepthmapClusterEstimator()
    c.set_max_iterations(2)
    c.set_patch_size(5)
    c.set_max_image_size(3200)
    c.set_sigma_spatial(5.0)
    c.set_sigma_color(3.0 / 255.0)
    c.set_top_k(3)
    c.set_census_weight(0.3)
    c.set_hierarchy_levels(2)
    c.set_smooth_weight(0.3)
    c.set_geom_consistency_weight(0.05)
    idx, nb = {}, {}
    for sid in cluster:
        K, R, t, im = v[sid]
        idx[sid] = c.begin_ref_view(K, R, t, im, *dr[sid])
        nb[sid] = [sid] + bn[sid][1:4]
        for s in bn[sid][1:4]:
            Ks, Rs, ts, ims = v[s]
            c.add_source_view(Ks, Rs, ts, ims)
    for sid in cluster:
        for o in cluster:
            if o != sid and o in nb[sid]:
                c.add_geom_link(idx[sid], nb[sid].index(o) - 1, idx[o])
    want = c.run()
    for sid, (depth, normal, cost, conf) in zip(cluster, want):
        got = dense_io.load_raw_depthmap(d, sid)
        exp_depth = depth.copy()
        exp_depth[~np.isfinite(exp_depth)] = 0
        exp_depth[cost > 0.9] = 0
        assert np.array_equal(got[0], exp_depth)
        assert np.array_equal(got[1], normal) and np.array_equal(got[2], cost)
        assert got[3].shape == (0,) and list(got[4]) == bn[sid]
        assert np.array_equal(got[5], conf)
        assert (got[0] > 0).mean() > 0.3

    done = dense_adapter.clean_cluster_gpu(d, v, bn, cluster, cfg, max_neighbors=3)
    assert done == cluster
    g = pydense.GPUDepthmapCleaner()
    g.set_same_depth_threshold(0.01)
    g.set_min_consistent_views(2)
    g.set_carving_threshold(0.2)
    g.set_max_carved_views(1)
    have = set(cluster)  # only the cluster's shots have raw files
    order = sorted(have)
    for sid in order:
        K, R, t, _ = v[sid]
        g.add_view(K, R, t, dense_io.load_raw_depthmap(d, sid)[0])
    for sid in cluster:
        nbrs = [n for n in bn[sid] if n != sid and n in have][:3]
        exp = g.clean(order.index(sid), np.array([order.index(n) for n in nbrs], np.int32))
        depth, plane, score, conf = dense_io.load_clean_depthmap(d, sid)
        raw = dense_io.load_raw_depthmap(d, sid)
        assert np.array_equal(depth, exp)
        assert np.array_equal(plane, raw[1]) and not score.any()
        assert np.array_equal(conf, raw[5])
