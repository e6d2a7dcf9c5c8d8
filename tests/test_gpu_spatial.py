"""GPU parity of the spatial k-d tree (reference: cukd/spatial-kdtree.h).

The builder is deterministic (children numbered in parent order, degenerate
splits alternating by prim id) and must produce exactly the oracle's node
array and prim list; queries must match the oracle bit for bit.  Against the
reference's own GPU builder (whose numbering depends on atomics) the trees
are compared structurally: same splits, same leaves' prim sets."""
import math

import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from oracle import pyoracle as po
from tests.helpers import f32_bits, make_points, make_queries

pytestmark = pytest.mark.gpu


def _gpu_tree(pts, thr=0):
    t = torch.from_numpy(pts).cuda()
    tree = ck.spatial_build(t, leaf_threshold=thr)
    nodes = tree.nodes().cpu().numpy().copy().view(po.SPATIAL_NODE).reshape(-1)
    prims = tree.prim_ids().cpu().numpy().astype(np.uint32)
    return t, tree, nodes, prims


@pytest.mark.parametrize("n", [1, 5, 8, 9, 100, 5000, 100000])
@pytest.mark.parametrize("kind", ["uniform", "gmm", "tie", "same"])
@pytest.mark.parametrize("thr", [0, 1, 16])
def test_spatial_build_matches_oracle(n, kind, thr):
    pts = make_points(n, 3, kind, seed=n)
    on, op, ob = po.spatial_build(pts, thr or 8)
    t, tree, nodes, prims = _gpu_tree(pts, thr)
    assert tree.num_nodes == len(on)
    assert np.array_equal(nodes.view(np.uint8), on.view(np.uint8))
    assert np.array_equal(prims, op)
    assert np.array_equal(np.array(tree.bounds, np.float32), ob)
    tree.free()


@pytest.mark.parametrize("method,m", [("stack_based", po.STACK_BASED), ("cct", po.CCT)])
@pytest.mark.parametrize("kind", ["uniform", "gmm", "tie"])
@pytest.mark.parametrize("k", [1, 8, 20])
@pytest.mark.parametrize("cutoff", [math.inf, 0.05])
def test_spatial_queries_match_oracle(method, m, kind, k, cutoff):
    n, nq = 30000, 10000
    pts = make_points(n, 3, kind, seed=3)
    q = make_queries(nq, 3, kind, seed=4)
    if kind == "tie":
        cutoff = cutoff * 20
    on, op, ob = po.spatial_build(pts)
    t, tree, _, _ = _gpu_tree(pts)
    dq = torch.from_numpy(q).cuda()
    ref_f = po.spatial_fcp(on, op, pts, ob, q, m, cutoff=cutoff)
    assert np.array_equal(tree.fcp(dq, method, cutoff=cutoff).cpu().numpy(), ref_f)
    ri, rd = po.spatial_knn(on, op, pts, ob, q, k, m, cutoff=cutoff,
                            list_kind=po.HEAP_LIST if k == 20 else po.FIXED_LIST)
    ids, d2 = tree.knn(dq, k, method, cutoff=cutoff, heap_order=(k == 20))
    assert np.array_equal(ids.cpu().numpy(), ri)
    assert np.array_equal(f32_bits(d2.cpu().numpy()), f32_bits(rd))
    tree.free()


def test_spatial_queries_match_reference_traversal_code():
    """The reference's own spatial traversals (host build of its headers)
    run over this library's tree give the same answers."""
    if po.ref_host() is None:
        pytest.skip("oracle/_ref not built")
    pts = make_points(20000, 3, "gmm", seed=5)
    q = make_queries(5000, 3, "gmm", seed=6)
    t, tree, nodes, prims = _gpu_tree(pts)
    b = np.array(tree.bounds, np.float32)
    dq = torch.from_numpy(q).cuda()
    for method, m in (("stack_based", po.STACK_BASED), ("cct", po.CCT)):
        ref = po.ref_spatial_fcp_host(nodes, prims, pts, b, q, m)
        assert np.array_equal(tree.fcp(dq, method).cpu().numpy(), ref)
        ri, rd = po.ref_spatial_knn_host(nodes, prims, pts, b, q, 8, m)
        ids, d2 = tree.knn(dq, 8, method)
        assert np.array_equal(ids.cpu().numpy(), ri)


def _structure(nodes, prims, node=0):
    """Canonical form of a spatial tree: nested (dim, pos, left, right) with
    leaves as sorted prim tuples (numbering-independent)."""
    nd = nodes[node]
    if nd["count"]:
        return tuple(sorted(prims[nd["offset"]: nd["offset"] + nd["count"]].tolist()))
    return (int(nd["dim"]), float(nd["pos"]), _structure(nodes, prims, nd["offset"]),
            _structure(nodes, prims, nd["offset"] + 1))


@pytest.mark.parametrize("kind", ["uniform", "gmm"])
def test_spatial_build_matches_reference_gpu_builder(kind):
    """Same splits and leaves as the reference's GPU builder (no degenerate
    splits on these inputs, so its atomic choices only renumber nodes)."""
    L = po.ref_gpu()
    if L is None:
        pytest.skip("oracle/_ref not built")
    import ctypes as C
    import sys
    sys.setrecursionlimit(100000)
    n = 20000
    pts = make_points(n, 3, kind, seed=7)
    d = torch.from_numpy(pts).cuda()
    rn = np.zeros(2 * n + 2, po.SPATIAL_NODE)
    rp = np.zeros(n, np.uint32)
    nn = np.zeros(1, np.int32)
    rb = np.zeros((2, 3), np.float32)
    rc = L.refg_spatial_build_float3(C.c_void_p(d.data_ptr()), n, 8,
                                     rn.ctypes.data_as(C.c_void_p), rp.ctypes.data_as(C.c_void_p),
                                     nn.ctypes.data_as(C.c_void_p), rb.ctypes.data_as(C.c_void_p))
    assert rc == 0
    rn = rn[: nn[0]]
    _, tree, nodes, prims = _gpu_tree(pts)
    assert tree.num_nodes == len(rn)
    assert _structure(nodes, prims) == _structure(rn, rp)
    assert np.array_equal(np.array(tree.bounds, np.float32), rb)
