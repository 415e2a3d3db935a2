"""GPU test of dn_prune_noalloc, the pruner entry point that allocates no
device memory (for callers whose process cannot or may not allocate on the
GPU).  It is called through the C ABI with caller-owned device buffers, twice
in a row, and must reproduce the regular pruner (dn_pruner_*) bit for bit,
the tolerance the pruner tests use.  It also rejects a reference depthmap
above its static-scratch limit.  Kept in a file of its own that pytest
collects last."""
import ctypes

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

if not gpu_available():
    pytest.skip("no CUDA device", allow_module_level=True)

torch = pytest.importorskip("torch")

from opensfm_b200 import _lib, pydense  # noqa: E402


def _views(g):
    """Device copies of the golden pruner case and the dn_prune_view table."""
    keep = []
    table = (_lib.PruneView * len(g["K"]))()
    for k in range(len(g["K"])):
        d = torch.from_numpy(np.ascontiguousarray(g["depths"][k], np.float32)).cuda()
        p = torch.from_numpy(np.ascontiguousarray(g["planes"][k], np.float32)).cuda()
        c = torch.from_numpy(np.ascontiguousarray(g["colors"][k], np.uint8)).cuda()
        lb = torch.from_numpy(np.ascontiguousarray(g["labels"][k], np.uint8)).cuda()
        keep += [d, p, c, lb]
        v = table[k]
        v.K[:] = [float(x) for x in np.asarray(g["K"][k], np.float64).ravel()]
        v.R[:] = [float(x) for x in np.asarray(g["R"][k], np.float64).ravel()]
        v.t[:] = [float(x) for x in np.asarray(g["t"][k], np.float64).ravel()]
        v.depth, v.plane, v.color, v.label = d.data_ptr(), p.data_ptr(), c.data_ptr(), lb.data_ptr()
        v.height, v.width = g["depths"][k].shape
    return table, keep


def _noalloc(lib, table, n, thr, H, W):
    cap = H * W
    pts = torch.zeros((cap, 3), dtype=torch.float32, device="cuda")
    nrm = torch.zeros((cap, 3), dtype=torch.float32, device="cuda")
    col = torch.zeros((cap, 3), dtype=torch.uint8, device="cuda")
    lab = torch.zeros((cap,), dtype=torch.uint8, device="cuda")
    cnt = torch.zeros((1,), dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.dn_prune_noalloc(ctypes.cast(table, ctypes.c_void_p), n, thr, pts.data_ptr(),
                              nrm.data_ptr(), col.data_ptr(), lab.data_ptr(), cap, cnt.data_ptr(),
                              ctypes.c_void_p(stream))
    assert st == _lib.DN_OK, lib.dn_noalloc_last_error()
    torch.cuda.synchronize()
    n_out = int(cnt.item())
    return (pts[:n_out].cpu().numpy(), nrm[:n_out].cpu().numpy(), col[:n_out].cpu().numpy(),
            lab[:n_out].cpu().numpy())


def test_prune_noalloc_matches_pruner_twice(golden):
    g = golden("clean_prune_64x48_v4.npz")
    lib = _lib.load()
    p = pydense.DepthmapPruner()
    p.set_same_depth_threshold(0.01)
    for K, R, t, d, pl, c, lb in zip(g["K"], g["R"], g["t"], g["depths"], g["planes"],
                                     g["colors"], g["labels"]):
        p.add_view(K, R, t, d, pl, c, lb)
    want = p.prune()
    assert len(want[3]) > 0
    table, keep = _views(g)
    H, W = g["depths"][0].shape
    for _ in range(2):
        got = _noalloc(lib, table, len(g["K"]), 0.01, H, W)
        for a, b in zip(got, want):
            assert a.shape == b.shape
            assert np.array_equal(a, b)
    # The golden vectors from the reference's own depthmap.cc, too.
    assert np.array_equal(got[0], g["prune_points"])
    assert np.array_equal(got[3], g["prune_labels"])


def test_prune_noalloc_rejects_oversize_and_bad_args(golden):
    g = golden("clean_prune_64x48_v4.npz")
    lib = _lib.load()
    table, keep = _views(g)
    table[0].width, table[0].height = 4096, 2048  # 8 Mpx > 4 Mpx limit
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    st = lib.dn_prune_noalloc(ctypes.cast(table, ctypes.c_void_p), 4, 0.01, dummy.data_ptr(),
                              dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), 1 << 30,
                              dummy.data_ptr(), None)
    assert st == _lib.DN_INVALID_ARG
    assert b"4194304" in lib.dn_noalloc_last_error()
    table[0].height, table[0].width = g["depths"][0].shape
    st = lib.dn_prune_noalloc(ctypes.cast(table, ctypes.c_void_p), 4, 0.01, dummy.data_ptr(),
                              dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), 10,
                              dummy.data_ptr(), None)
    assert st == _lib.DN_INVALID_ARG  # capacity below width * height
