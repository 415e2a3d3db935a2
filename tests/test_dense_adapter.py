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
