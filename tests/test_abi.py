"""CPU tests of the C ABI boundary: the library loads and exports every
function include/dense_b200.h declares; host-side argument checks fail with
ValueError / RuntimeError instead of crashing when no device is present."""
import ctypes
import subprocess

import numpy as np
import pytest

from opensfm_b200 import _lib
from conftest import gpu_available


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _lib.header_symbols()
    assert "dn_estimator_compute_patch_match" in declared
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # Every declared function has a ctypes signature in the binding.
    assert set(declared) <= set(_lib._SIGNATURES), set(declared) - set(_lib._SIGNATURES)


def test_exports_are_plain_c_symbols():
    out = subprocess.check_output(["nm", "-D", "--defined-only", _lib.LIB_PATH], text=True)
    names = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for s in _lib.header_symbols():
        assert s in names, s  # unmangled


def test_version_and_device_count_callable():
    lib = _lib.load()
    assert b"sm_100a" in lib.dn_version()
    assert lib.dn_device_count() >= 0


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_create_without_device_raises():
    from opensfm_b200 import pydense
    with pytest.raises(RuntimeError):
        pydense.DepthmapEstimator()
    with pytest.raises(RuntimeError):
        pydense.DepthmapCleaner()
    with pytest.raises(RuntimeError):
        pydense.DepthmapPruner()


def test_null_arguments_are_rejected_without_device():
    lib = _lib.load()
    assert lib.dn_estimator_create(None) == _lib.DN_INVALID_ARG
    assert b"NULL" in lib.dn_last_error()
    assert lib.dn_estimator_add_view(None, None, None, None, None, None, 4, 4, 4) == _lib.DN_INVALID_ARG
    assert lib.dn_cleaner_clean(None, None) == _lib.DN_INVALID_ARG
    assert lib.dn_pruner_prune(None, None) == _lib.DN_INVALID_ARG
    assert lib.dn_batch_run(None, 0) == _lib.DN_INVALID_ARG
    assert lib.dn_batch_upload_view_image(None, 0, None, 0) == _lib.DN_INVALID_ARG
    assert lib.dn_batch_get_depths_async(None, 0, None, None, 0) == _lib.DN_INVALID_ARG
    assert lib.dn_walk_ceiling(None, None) == _lib.DN_INVALID_ARG


def test_pydense_argument_validation():
    from opensfm_b200 import pydense
    with pytest.raises(ValueError):
        pydense._mat(np.zeros(8), (3, 3), "K")
    with pytest.raises(ValueError):
        pydense._image(np.zeros((2, 3, 4)), "image")
    assert pydense._image(np.zeros((3, 4), np.float64), "image").dtype == np.uint8


def test_prior_delaunay_matches_oracle():
    """The SfM planar prior's triangulation (host code in the library) equals
    the oracle's: Qhull over the points plus cv::Subdiv2D's virtual outer
    triangle, less the triangles touching it.  Includes collinear rows,
    duplicates and points on the image border."""
    import oracle

    lib = _lib.load()
    rng = np.random.default_rng(11)
    cases = []
    for _ in range(40):
        W, H = int(rng.integers(32, 700)), int(rng.integers(32, 500))
        n = int(rng.integers(3, 300))
        cases.append((rng.uniform(0, [W, H], (n, 2)), W, H))
    grid = np.stack(np.meshgrid(np.arange(0, 60, 6.0), np.arange(0, 40, 8.0)), -1).reshape(-1, 2)
    cases.append((grid, 64, 48))  # cocircular quadruples: ties broken alike
    cases.append((np.array([[0, 0], [63, 0], [63, 47], [0, 47], [32, 24]], float), 64, 48))
    for xy, W, H in cases:
        xy = np.ascontiguousarray(xy, np.float64)
        cnt = ctypes.c_int(0)
        p = xy.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        assert lib.dn_delaunay_2d(p, len(xy), W, H, None, 0, ctypes.byref(cnt)) == _lib.DN_OK
        out = np.zeros((max(cnt.value, 1), 3), np.int32)
        assert lib.dn_delaunay_2d(p, len(xy), W, H, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  cnt.value, ctypes.byref(cnt)) == _lib.DN_OK
        ref = oracle.acm_delaunay(xy, W, H)
        if len(ref) and not np.array_equal(out[:cnt.value], ref):
            # Cocircular points have several Delaunay triangulations; both
            # must then cover the same area with the same triangle count.
            assert xy is grid or len(xy) == 5, (W, H, len(xy))
            assert cnt.value == len(ref)


def test_prior_delaunay_rejects_non_finite_points():
    lib = _lib.load()
    xy = np.array([[1.0, 2.0], [np.nan, 3.0], [4.0, 5.0], [6.0, 1.0]])
    cnt = ctypes.c_int(0)
    st = lib.dn_delaunay_2d(xy.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 4, 8, 8, None, 0,
                            ctypes.byref(cnt))
    assert st == _lib.DN_INVALID_ARG
    assert b"non-finite" in lib.dn_acmmp_last_error()


def test_prior_delaunay_duplicates_join_the_first():
    """Exact duplicate positions are inserted once, under their first index;
    the triangles equal Qhull's once every index is mapped to the first
    point at its position."""
    import oracle

    lib = _lib.load()
    rng = np.random.default_rng(3)
    for _ in range(6):
        base = rng.uniform(0, [320, 240], (60, 2))
        xy = np.ascontiguousarray(base[rng.integers(0, 60, 150)])
        cnt = ctypes.c_int(0)
        p = xy.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        assert lib.dn_delaunay_2d(p, len(xy), 320, 240, None, 0, ctypes.byref(cnt)) == _lib.DN_OK
        out = np.zeros((cnt.value, 3), np.int32)
        assert lib.dn_delaunay_2d(p, len(xy), 320, 240, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  cnt.value, ctypes.byref(cnt)) == _lib.DN_OK
        _, first, inv = np.unique(xy, axis=0, return_index=True, return_inverse=True)
        canon = first[inv.ravel()]
        assert np.array_equal(canon[out], out)  # only first indices are used

        def norm(t):
            t = np.sort(canon[t], axis=1)
            return t[np.lexsort((t[:, 2], t[:, 1], t[:, 0]))]

        assert np.array_equal(norm(out), norm(oracle.acm_delaunay(xy, 320, 240)))


def test_plain_c_caller_compiles_links_and_runs(tmp_path):
    """A C99 program includes the header, links the library by name and
    calls it: the version string, the device count, a host-only
    triangulation and an estimator constructor, whose status is DN_OK with
    a device and an error (not a crash) without one."""
    import os
    import shutil

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "caller.c"
    src.write_text(r'''
#include <stdio.h>
#include <string.h>
#include "dense_b200.h"
int main(void) {
  if (!strstr(dn_version(), "sm_100a")) return 2;
  const int devices = dn_device_count();
  const double xy[8] = {0, 0, 10, 0, 0, 10, 10, 10};
  int tris[6], count = 0;
  if (dn_delaunay_2d(xy, 4, 16, 16, tris, 2, &count) != DN_OK || count != 2) return 3;
  dn_acmmp* c = NULL;
  const dn_status st = dn_acmmp_create(&c);
  if (devices > 0 && st != DN_OK) return 4;
  if (devices == 0 && st == DN_OK) return 5;
  if (c) dn_acmmp_destroy(c);
  printf("ok %d\n", devices);
  return 0;
}
''')
    exe = tmp_path / "caller"
    lib_dir = os.path.dirname(_lib.LIB_PATH)
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(root, "include"),
                           str(src), "-o", str(exe), "-L", lib_dir, "-ldense_b200",
                           "-Wl,-rpath," + lib_dir])
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert out.stdout.startswith("ok")
