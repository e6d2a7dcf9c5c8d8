"""The C++ drop-in shim (include/cukd/*.h): reference-style user code
(tests/cpp/shim_test.cu) built against it and linked to libcukd_b200.so; its
trees and query answers are compared with the CPU oracle bit for bit."""
import os
import subprocess

import numpy as np
import pytest

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cpp", "shim_test")


@pytest.fixture(scope="module")
def out(tmp_path_factory):
    if not os.path.exists(BIN):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "tests", "cpp")])
    d = tmp_path_factory.mktemp("shim")
    r = subprocess.run([BIN, str(d)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "shim_test OK" in r.stdout
    assert "sqrDist 2.8466301" in r.stdout
    assert "loadPoints OK" in r.stdout
    return d


def _f(d, name, dtype, cols=None):
    a = np.fromfile(os.path.join(d, name), dtype=dtype)
    return a if cols is None else a.reshape(-1, cols)


def test_payload_build_and_user_knn_kernel(out):
    pts = _f(out, "points.bin", np.float32, 3)
    q = _f(out, "queries.bin", np.float32, 3)
    perm, _, bounds = po.build(pts)
    assert np.array_equal(_f(out, "payload_order.bin", np.int32), perm.astype(np.int32))
    ri, rd, _ = po.knn(pts[perm], q, 8, po.STACK_BASED, bounds=bounds)
    assert np.array_equal(_f(out, "knn8_ids.bin", np.int32, 8), ri)
    assert np.array_equal(_f(out, "knn8_d2.bin", np.uint32, 8), rd.view(np.uint32))


def test_explicit_dim_build_and_user_kernels(out):
    pts = _f(out, "points.bin", np.float32, 3)
    q = _f(out, "queries.bin", np.float32, 3)
    perm, dims, bounds = po.build(pts, explicit_dim=True)
    tree = _f(out, "dim_tree.bin", np.int32, 4)
    assert np.array_equal(tree[:, :3].view(np.float32), pts[perm])
    assert np.array_equal(tree[:, 3], dims)
    assert np.array_equal(_f(out, "dim_bounds.bin", np.float32).reshape(2, 3), bounds)
    assert np.array_equal(_f(out, "fcp_cct.bin", np.int32),
                          po.fcp(pts[perm], q, po.CCT, dims=dims, bounds=bounds))
    ri, _, _ = po.knn(pts[perm], q, 20, po.STACK_FREE, dims=dims, bounds=bounds,
                      list_kind=po.HEAP_LIST)
    assert np.array_equal(_f(out, "knn20_heap_sf.bin", np.int32, 20), ri)


def test_spatial_tree_user_kernel(out):
    pts = _f(out, "points.bin", np.float32, 3)
    q = _f(out, "queries.bin", np.float32, 3)
    nodes, prims, b = po.spatial_build(pts)
    ri, _ = po.spatial_knn(nodes, prims, pts, b, q, 16, po.CCT, list_kind=po.HEAP_LIST)
    assert np.array_equal(_f(out, "spatial_knn16.bin", np.int32, 16), ri)


def test_vec_float8_build_and_user_knn_kernel(out):
    """cukd::buildTree<cukd::vec_float<8>> on the reference builder test's
    N = 8 inputs (unique integer coordinates,
    testing/testBuildersSameResult.cu:404-428) and a user kNN kernel
    (stackBased::knn<FixedCandidateList<8>, vec_float<8>>) over the tree."""
    pts = _f(out, "vec8_points.bin", np.float32, 8)
    q = _f(out, "vec8_queries.bin", np.float32, 8)
    perm, _, bounds = po.build(pts)
    tree = _f(out, "vec8_tree.bin", np.float32, 8)
    assert np.array_equal(tree, pts[perm])
    ri, _, _ = po.knn(pts[perm], q, 8, po.STACK_BASED, bounds=bounds)
    assert np.array_equal(_f(out, "vec8_knn8.bin", np.int32, 8), ri)
