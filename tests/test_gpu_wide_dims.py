"""Points of 5 to 8 dims (the reference's vec_float<N>, cukd-math.h:133-181).

The reference's own builder test runs N = 8 for float and int points,
point-only, with a payload, and with a payload plus an explicit split dim,
at 4, 10, 1000 and 10000 points (testing/testBuildersSameResult.cu:404-428);
its fcp / knn templates take any N.  Here: every builder name against the
oracle at those sizes and at sizes that reach the builders' global levels,
tie-heavy inputs, and FCP / kNN of the three traversals against the oracle.
The fast kNN, learned, spatial, batched and allocation-free paths take at
most 4 dims and refuse more.
"""
import ctypes as C
import math

import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from oracle import pyoracle as po
from tests.helpers import f32_bits, make_points, make_queries

pytestmark = pytest.mark.gpu

METHODS = [("stack_based", po.STACK_BASED), ("stack_free", po.STACK_FREE), ("cct", po.CCT)]


def _records(pts, kind):
    """point-only, +payload (input index), +payload+dim word (explicit)."""
    n, D = pts.shape
    raw = pts.view(np.int32)
    if kind == "point":
        return np.ascontiguousarray(raw), ck.layout_for(
            "float32" if pts.dtype == np.float32 else "int32", D)
    sc = "float32" if pts.dtype == np.float32 else "int32"
    words = D + (1 if kind == "payload" else 2)
    rec = np.zeros((n, words), np.int32)
    rec[:, :D] = raw
    rec[:, D] = np.arange(n, dtype=np.int32)
    if kind == "payload":
        return rec, ck.layout_for(sc, D, stride=4 * words)
    return rec, ck.layout_for(sc, D, stride=4 * words, dim_offset=4 * (D + 1))


@pytest.mark.parametrize("builder", ["default", "bitonic", "inplace"])
@pytest.mark.parametrize("n", [4, 10, 1000, 10000, 300000])
@pytest.mark.parametrize("D", [5, 8])
@pytest.mark.parametrize("scalar", ["float32", "int32"])
@pytest.mark.parametrize("kind", ["point", "payload", "payload_dim"])
def test_builders_same_result_wide(builder, n, D, scalar, kind):
    """Unique coordinates (the reference test's inputs): every builder name
    gives the oracle's canonical tree, explicit dims and world bounds."""
    pts = make_points(n, D, "unique", seed=n + D).astype(
        np.float32 if scalar == "float32" else np.int32)
    explicit = kind == "payload_dim"
    perm, dims, bounds = po.build(pts, explicit_dim=explicit)
    rec, lay = _records(pts, kind)
    t = torch.from_numpy(rec.copy()).cuda()
    wb = ck.build_tree(t, layout=lay, builder=builder)
    ck.build_check()
    out = t.cpu().numpy()
    assert np.array_equal(out[:, :D], rec[perm][:, :D])
    if kind != "point":
        assert np.array_equal(out[:, D], perm.astype(np.int32))
    if explicit:
        assert np.array_equal(out[:, D + 1], dims.astype(np.int32))
    assert np.array_equal(wb.cpu().numpy(), bounds)


@pytest.mark.parametrize("n", [1000, 50000, 300000])
@pytest.mark.parametrize("D", [6, 8])
def test_ties_wide(n, D):
    """Tie-heavy coordinates: default and bitonic give the canonical tree
    (ties broken like the reference's stable sorts), inplace a valid k-d tree
    of the same points."""
    pts = make_points(n, D, "tie", seed=n)
    perm, _, bounds = po.build(pts)
    for b in ("default", "bitonic"):
        t = torch.from_numpy(pts.copy()).cuda()
        ck.build_tree(t, builder=b)
        ck.build_check()
        assert np.array_equal(t.cpu().numpy(), pts[perm]), b
    t = torch.from_numpy(pts.copy()).cuda()
    wb = ck.build_tree(t, builder="inplace")
    ck.build_check()
    out = t.cpu().numpy()
    assert po.check_kd(out) == 0
    row = np.dtype((np.void, 4 * D))
    assert np.array_equal(np.sort(out.view(row).ravel()), np.sort(pts.view(row).ravel()))
    assert np.array_equal(wb.cpu().numpy(), bounds)


@pytest.mark.parametrize("mname,m", METHODS)
@pytest.mark.parametrize("D", [5, 8])
@pytest.mark.parametrize("kind", ["uniform", "tie"])
@pytest.mark.parametrize("explicit", [False, True])
def test_fcp_and_knn_wide(mname, m, D, kind, explicit):
    n, nq = 20000, 4000
    pts = make_points(n, D, kind, seed=D)
    perm, dims, bounds = po.build(pts, explicit_dim=explicit)
    tree = pts[perm]
    q = make_queries(nq, D, kind, seed=D + 1)
    if explicit:
        rec = np.zeros((n, D + 1), np.int32)
        rec[:, :D] = tree.view(np.int32)
        rec[:, D] = dims
        t = torch.from_numpy(rec).cuda()
        lay = ck.layout_for("float32", D, stride=4 * (D + 1), dim_offset=4 * D)
    else:
        t = torch.from_numpy(np.ascontiguousarray(tree)).cuda()
        lay = ck.layout_for("float32", D)
    wb = torch.from_numpy(bounds).cuda()
    dq = torch.from_numpy(q).cuda()
    d = dims if explicit else None
    ids = ck.fcp(t, dq, mname, layout=lay, world_bounds=wb)
    assert np.array_equal(ids.cpu().numpy(), po.fcp(tree, q, m, dims=d, bounds=bounds))
    for k in (1, 8, 16, 40):
        ri, rd, _ = po.knn(tree, q, k, m, dims=d, bounds=bounds)
        gi, gd = ck.knn(t, dq, k, mname, layout=lay, world_bounds=wb)
        assert np.array_equal(gi.cpu().numpy(), ri), k
        assert np.array_equal(f32_bits(gd.cpu().numpy()), f32_bits(rd)), k


@pytest.mark.parametrize("D", [5, 8])
def test_int_knn_wide(D):
    n, nq = 20000, 3000
    pts = make_points(n, D, "tie", scalar="int32", seed=D)
    perm, _, bounds = po.build(pts)
    tree = pts[perm]
    q = make_queries(nq, D, "tie", scalar="int32", seed=D)
    ri, rd, _ = po.knn(tree, q, 16, po.STACK_BASED, bounds=bounds)
    gi, gd = ck.knn(torch.from_numpy(np.ascontiguousarray(tree)).cuda(), torch.from_numpy(q).cuda(),
                    16, "stack_based", world_bounds=torch.from_numpy(bounds).cuda())
    assert np.array_equal(gi.cpu().numpy(), ri)
    assert np.array_equal(gd.cpu().numpy(), rd)


def test_paths_limited_to_four_dims_refuse_more():
    n, D = 5000, 5
    pts = torch.from_numpy(make_points(n, D, "uniform", seed=1)).cuda()
    lay = ck.layout_for("float32", D)
    L = ck.lib()
    # spatial tree
    with pytest.raises(ck.CukdError) as err:
        ck.spatial_build(pts, layout=lay)
    assert err.value.status == 5  # CUKD_ERR_UNSUPPORTED
    # allocation-free builder
    L.cukd_build_tree_noalloc.argtypes = [C.c_void_p, C.c_int64, C.POINTER(ck.Layout),
                                          C.c_void_p, C.c_void_p]
    assert L.cukd_build_tree_noalloc(C.c_void_p(pts.data_ptr()), n, C.byref(lay), None,
                                     None) == 5
    # learned radius model and batched plans
    with pytest.raises(ck.CukdError):
        ck.RadiusModel(grid_res=8, num_dims=5)
    with pytest.raises(ck.CukdError):
        ck.BatchPlan(np.array([0, n]), np.array([0, 10]), 5, k=8)
