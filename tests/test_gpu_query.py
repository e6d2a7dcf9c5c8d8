"""GPU parity of the FCP / kNN traversals against the CPU oracle.

Bar: bit-exact ids AND squared-distance bits for every query, for the three
traversals (stackBased / stackFree / cct), fixed and heap candidate lists,
cut-offs, Morton reordering on and off, round-robin and explicit dims,
float and int coordinates.  The reference's own query test
(testing/floatN-knn-and-fcp.cu) only compares distances against brute force
within 1e-6; this is strictly tighter.
"""
import math

import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from oracle import pyoracle as po
from tests.helpers import f32_bits, make_points, make_queries

pytestmark = pytest.mark.gpu

METHODS = [("stack_based", po.STACK_BASED), ("stack_free", po.STACK_FREE), ("cct", po.CCT)]


def _tree(n, D, kind, explicit=False, scalar="float32", seed=0):
    pts = make_points(n, D, kind, scalar=scalar, seed=seed)
    perm, dims, bounds = po.build(pts, explicit_dim=explicit)
    return pts[perm], (dims if explicit else None), bounds


def _gpu_tree(tree, dims):
    n, D = tree.shape
    if dims is None:
        return torch.from_numpy(np.ascontiguousarray(tree)).cuda(), ck.infer_layout(
            torch.from_numpy(tree))
    rec = np.zeros((n, D + 1), np.int32)
    rec[:, :D] = tree.view(np.int32)
    rec[:, D] = dims
    sc = "float32" if tree.dtype == np.float32 else "int32"
    return torch.from_numpy(rec).cuda(), ck.layout_for(sc, D, stride=4 * (D + 1),
                                                       dim_offset=4 * D)


@pytest.mark.parametrize("mname,m", METHODS)
@pytest.mark.parametrize("kind", ["uniform", "tie", "gmm"])
@pytest.mark.parametrize("explicit", [False, True])
@pytest.mark.parametrize("cutoff", [math.inf, 0.05])
@pytest.mark.parametrize("morton", [True, False])
def test_fcp(mname, m, kind, explicit, cutoff, morton):
    n, nq = 20000, 30000
    tree, dims, bounds = _tree(n, 3, kind, explicit, seed=1)
    q = make_queries(nq, 3, kind, seed=2)
    ref, vis = po.fcp(tree, q, m, dims=dims, bounds=bounds, cutoff=cutoff, visits=True)
    t, lay = _gpu_tree(tree, dims)
    wb = torch.from_numpy(bounds).cuda()
    ids, d2 = ck.fcp(t, torch.from_numpy(q).cuda(), mname, layout=lay, world_bounds=wb,
                     cutoff=cutoff, morton=morton, with_d2=True)
    ids = ids.cpu().numpy()
    assert np.array_equal(ids, ref)
    d2 = d2.cpu().numpy()
    has = ref >= 0
    exp = ((tree[ref[has]] - q[has]) ** 2)
    # the d2 output is the traversal's own float sum; compare bits with the
    # oracle's left-to-right float evaluation
    e = np.zeros(has.sum(), np.float32)
    for d in range(3):
        e = (e + exp[:, d].astype(np.float32)).astype(np.float32)
    assert np.array_equal(f32_bits(d2[has]), f32_bits(e))


@pytest.mark.parametrize("mname,m", METHODS)
@pytest.mark.parametrize("k", [1, 4, 5, 8, 16, 20, 32, 33, 50, 64, 65, 128, 129, 200])
@pytest.mark.parametrize("kind", ["uniform", "tie"])
def test_knn(mname, m, k, kind):
    n, nq = 20000, 8000
    tree, dims, bounds = _tree(n, 3, kind, False, seed=4)
    q = make_queries(nq, 3, kind, seed=5)
    ri, rd, rr = po.knn(tree, q, k, m, bounds=bounds)
    t, lay = _gpu_tree(tree, dims)
    wb = torch.from_numpy(bounds).cuda()
    ids, d2, mx = ck.knn(t, torch.from_numpy(q).cuda(), k, mname, layout=lay, world_bounds=wb,
                         with_max=True)
    assert np.array_equal(ids.cpu().numpy(), ri)
    assert np.array_equal(f32_bits(d2.cpu().numpy()), f32_bits(rd))
    assert np.array_equal(f32_bits(mx.cpu().numpy()), f32_bits(rr))


@pytest.mark.parametrize("mname,m", METHODS)
@pytest.mark.parametrize("k", [8, 20, 64])
def test_knn_heap_order(mname, m, k):
    """HeapCandidateList returns its heap layout (knn.h:427-493)."""
    n, nq = 5000, 3000
    tree, dims, bounds = _tree(n, 3, "tie", False, seed=6)
    q = make_queries(nq, 3, "tie", seed=7)
    ri, rd, _ = po.knn(tree, q, k, m, bounds=bounds, list_kind=po.HEAP_LIST)
    t, lay = _gpu_tree(tree, dims)
    ids, d2 = ck.knn(t, torch.from_numpy(q).cuda(), k, mname, layout=lay,
                     world_bounds=torch.from_numpy(bounds).cuda(), heap_order=True)
    assert np.array_equal(ids.cpu().numpy(), ri)
    assert np.array_equal(f32_bits(d2.cpu().numpy()), f32_bits(rd))


@pytest.mark.parametrize("mname,m", METHODS)
@pytest.mark.parametrize("explicit", [False, True])
@pytest.mark.parametrize("D", [2, 4])
@pytest.mark.parametrize("cutoff", [math.inf, 0.1])
@pytest.mark.parametrize("k", [8, 64])
def test_knn_dims_cutoff(mname, m, explicit, D, cutoff, k):
    n, nq = 10000, 5000
    tree, dims, bounds = _tree(n, D, "uniform", explicit, seed=D)
    q = make_queries(nq, D, "uniform", seed=D + 1)
    ri, rd, _ = po.knn(tree, q, k, m, dims=dims, bounds=bounds, cutoff=cutoff)
    t, lay = _gpu_tree(tree, dims)
    ids, d2 = ck.knn(t, torch.from_numpy(q).cuda(), k, mname, layout=lay,
                     world_bounds=torch.from_numpy(bounds).cuda(), cutoff=cutoff)
    assert np.array_equal(ids.cpu().numpy(), ri)
    assert np.array_equal(f32_bits(d2.cpu().numpy()), f32_bits(rd))


@pytest.mark.parametrize("mname,m", METHODS)
@pytest.mark.parametrize("k", [1, 2, 8, 16, 33, 64, 128])
@pytest.mark.parametrize("explicit", [False, True])
def test_int_coordinates(mname, m, k, explicit):
    """int32 trees: exact int64 squared distances (no reference traversal
    exists for integer points; the oracle restates the same algorithm)."""
    n, nq = 20000, 6000
    tree, dims, bounds = _tree(n, 3, "uniform", explicit, scalar="int32", seed=8)
    q = make_queries(nq, 3, "uniform", scalar="int32", seed=9)
    ri, rd, _ = po.knn(tree, q, k, m, dims=dims, bounds=bounds)
    t, lay = _gpu_tree(tree, dims)
    ids, d2 = ck.knn(t, torch.from_numpy(q).cuda(), k, mname, layout=lay,
                     world_bounds=torch.from_numpy(bounds).cuda())
    assert np.array_equal(ids.cpu().numpy(), ri)
    assert np.array_equal(d2.cpu().numpy(), rd)
    fi = ck.fcp(t, torch.from_numpy(q).cuda(), mname, layout=lay,
                world_bounds=torch.from_numpy(bounds).cuda())
    assert np.array_equal(fi.cpu().numpy(), po.fcp(tree, q, m, dims=dims, bounds=bounds))


@pytest.mark.parametrize("eps", [0.0, 0.5])
def test_stack_free_eps(eps):
    """FcpSearchParams::eps, honoured by the stack-free traversal only
    (traverse-stack-free.h:37,85)."""
    tree, dims, bounds = _tree(20000, 3, "uniform", False, seed=10)
    q = make_queries(10000, 3, "uniform", seed=11)
    ref = po.fcp(tree, q, po.STACK_FREE, bounds=bounds, eps=eps)
    ids = ck.fcp(torch.from_numpy(tree).cuda(), torch.from_numpy(q).cuda(), "stack_free",
                 eps=eps)
    assert np.array_equal(ids.cpu().numpy(), ref)


@pytest.mark.parametrize("n", [0, 1, 2, 3])
@pytest.mark.parametrize("mname,m", METHODS)
def test_tiny_trees(n, mname, m):
    pts = make_points(max(n, 1), 3, "uniform", seed=12)[:n]
    if n:
        perm, _, bounds = po.build(pts)
        tree = pts[perm]
    else:
        tree, bounds = pts, np.zeros((2, 3), np.float32)
    q = make_queries(100, 3, "uniform", seed=13)
    ref = po.fcp(tree, q, m, bounds=bounds)
    t = torch.from_numpy(np.ascontiguousarray(tree)).cuda()
    ids = ck.fcp(t, torch.from_numpy(q).cuda(), mname, layout=ck.layout_for("float32", 3),
                 world_bounds=torch.from_numpy(bounds).cuda(), n=n)
    assert np.array_equal(ids.cpu().numpy(), ref)
    ri, rd, _ = po.knn(tree, q, 4, m, bounds=bounds)
    ids, d2 = ck.knn(t, torch.from_numpy(q).cuda(), 4, mname, layout=ck.layout_for("float32", 3),
                     world_bounds=torch.from_numpy(bounds).cuda(), n=n)
    assert np.array_equal(ids.cpu().numpy(), ri)


def test_visits_match_oracle():
    tree, dims, bounds = _tree(50000, 3, "gmm", False, seed=14)
    q = make_queries(20000, 3, "gmm", seed=15)
    _, _, _, vis = po.knn(tree, q, 16, po.STACK_BASED, bounds=bounds, visits=True)
    v = ck.knn_visits(torch.from_numpy(tree).cuda(), torch.from_numpy(q).cuda(), 16,
                      "stack_based")
    assert np.array_equal(v.cpu().numpy(), vis)


def test_morton_order_is_a_permutation():
    q = make_queries(100003, 3, "gmm", seed=16)
    perm = ck.morton_order(torch.from_numpy(q).cuda()).cpu().numpy()
    assert np.array_equal(np.sort(perm), np.arange(len(q)))


def _morton_codes(cells, D):
    bits = 30 // D
    code = np.zeros(len(cells), np.uint64)
    for d in range(D):
        c = cells[:, d].astype(np.uint64)
        for b in range(bits):
            code |= ((c >> np.uint64(b)) & np.uint64(1)) << np.uint64(b * D + (D - 1 - d))
    return code


@pytest.mark.parametrize("D", [2, 3, 4])
@pytest.mark.parametrize("n", [1, 4095, 4097, 1_000_003])
def test_morton_order_is_the_stable_sort_of_the_codes(D, n):
    """With bounds [0, 1] the grid scale is a power of two, so points at
    (cell + 1/2) / 2^bits fall in known cells: the permutation must be
    numpy's stable argsort of their Morton codes (sorted, equal codes in
    input order) -- half the points in a few cells, so equal codes abound,
    across many sort tiles and a partial last one."""
    bits = 30 // D
    rng = np.random.default_rng(n + D)
    cells = rng.integers(0, 1 << bits, size=(n, D))
    few = rng.random(n) < 0.5
    cells[few] = rng.integers(0, 4, size=(int(few.sum()), D))
    pts = ((cells + 0.5) / float(1 << bits)).astype(np.float32)
    bounds = torch.tensor([[0.0] * D, [1.0] * D], dtype=torch.float32, device="cuda")
    perm = ck.morton_order(torch.from_numpy(pts).cuda(), bounds=bounds).cpu().numpy()
    want = np.argsort(_morton_codes(cells, D), kind="stable")
    assert np.array_equal(perm, want.astype(np.int32))


@pytest.mark.parametrize("kind", ["uniform", "tie", "gmm"])
@pytest.mark.parametrize("explicit", [False, True])
def test_tree_path_order_same_answers(kind, explicit):
    """CUKD_QUERY_TREE_ORDER only changes the visiting order of the queries."""
    n, nq = 20000, 8000
    tree, dims, bounds = _tree(n, 3, kind, explicit, seed=11)
    q = make_queries(nq, 3, kind, seed=12)
    t, lay = _gpu_tree(tree, dims)
    wb = torch.from_numpy(bounds).cuda()
    dq = torch.from_numpy(q).cuda()
    for k in (1, 16, 40):
        ri, rd, _ = po.knn(tree, q, k, po.STACK_BASED, dims=dims, bounds=bounds)
        ids, d2 = ck.knn(t, dq, k, "stack_based", layout=lay, world_bounds=wb, tree_order=True)
        assert np.array_equal(ids.cpu().numpy(), ri)
        assert np.array_equal(f32_bits(d2.cpu().numpy()), f32_bits(rd))
    rf = po.fcp(tree, q, po.CCT, dims=dims, bounds=bounds)
    assert np.array_equal(ck.fcp(t, dq, "cct", layout=lay, world_bounds=wb,
                                 tree_order=True).cpu().numpy(), rf)


@pytest.mark.parametrize("mname,m", METHODS)
@pytest.mark.parametrize("k", [4, 16, 64])
@pytest.mark.parametrize("cutoff_d2", [2**62, 40, 0])
def test_int_tie_heavy_and_cutoff(mname, m, k, cutoff_d2):
    """Integer fast path on tie-heavy points (many equal distances at the
    k-th boundary, re-run in the reference order) with squared cut-offs,
    including a point exactly at the cut-off."""
    n, nq = 20000, 6000
    tree, dims, bounds = _tree(n, 3, "tie", False, scalar="int32", seed=13)
    q = make_queries(nq, 3, "tie", scalar="int32", seed=14)
    ri, rd, _ = po.knn(tree, q, k, m, bounds=bounds, cutoff_d2_int=cutoff_d2)
    t, lay = _gpu_tree(tree, dims)
    ids, d2 = ck.knn(t, torch.from_numpy(q).cuda(), k, mname, layout=lay,
                     world_bounds=torch.from_numpy(bounds).cuda(), cutoff_d2=cutoff_d2)
    assert np.array_equal(ids.cpu().numpy(), ri)
    assert np.array_equal(d2.cpu().numpy(), rd)


@pytest.mark.parametrize("D", [2, 3, 4])
@pytest.mark.parametrize("kind", ["uniform", "tie", "gmm"])
@pytest.mark.parametrize("k", [2, 8, 16, 32])
def test_warp_packet_traversal_identical(D, kind, k):
    """The warp-cooperative traversal (CUKD_QUERY_WARP_PACKET) returns the
    oracle's ids and distance bits, like the per-thread fast path."""
    n, nq = 40000, 5003  # a partial last warp
    pts = make_points(n, D, kind, seed=D + k)
    q = make_queries(nq, D, kind, seed=D + 2 * k)
    perm, _, bounds = po.build(pts)
    t = torch.from_numpy(pts).cuda()
    wb = ck.build_tree(t)
    for name, m in (("stack_based", po.STACK_BASED), ("stack_free", po.STACK_FREE)):
        ids, d2 = ck.knn(t, torch.from_numpy(q).cuda(), k, name, world_bounds=wb,
                         warp_packet=True)
        ri, rd, _ = po.knn(pts[perm], q, k, m, bounds=bounds)
        assert np.array_equal(ids.cpu().numpy(), ri)
        assert np.array_equal(f32_bits(d2.cpu().numpy()), f32_bits(rd))
    # with a cut-off radius (unfilled slots)
    ids, d2 = ck.knn(t, torch.from_numpy(q).cuda(), k, world_bounds=wb, cutoff=0.02,
                     warp_packet=True)
    pi, pd = ck.knn(t, torch.from_numpy(q).cuda(), k, world_bounds=wb, cutoff=0.02)
    assert torch.equal(ids, pi) and torch.equal(d2, pd)


def test_warp_packet_seeded_by_learned_radius_identical():
    n = 200000
    pts = make_points(n, 3, "gmm", seed=1)
    t = torch.from_numpy(pts).cuda()
    wb = ck.build_tree(t)
    m = ck.RadiusModel(seed=2, quantile=0.9)
    m.fit(t, torch.from_numpy(make_queries(30000, 3, "gmm", seed=3)).cuda(), 16,
          world_bounds=wb, epochs=4)
    q = torch.from_numpy(make_queries(40000, 3, "gmm", seed=4)).cuda()
    pi, pd = ck.knn(t, q, 16, world_bounds=wb)
    li, ld, fb, _ = ck.knn_learned(t, q, 16, m, world_bounds=wb, warp_packet=True)
    assert torch.equal(li, pi) and torch.equal(ld, pd)


def test_trees_beyond_32_bit_child_indices_are_refused():
    """Trees of 2^30 nodes or more would overflow the traversals' 32-bit
    child indices (2i+1): refused with CUKD_ERR_UNSUPPORTED before any
    launch (the buffer is never read)."""
    import ctypes as C
    t = torch.zeros((16, 3), dtype=torch.float32, device="cuda")
    q = torch.zeros((4, 3), dtype=torch.float32, device="cuda")
    ids = torch.empty((4, 8), dtype=torch.int32, device="cuda")
    d2 = torch.empty((4, 8), dtype=torch.float32, device="cuda")
    lay = ck.layout_for("float32", 3)
    p = ck._params("stack_based", 8)
    rc = ck.lib().cukd_knn(t.data_ptr(), 1 << 30, C.byref(lay), None, q.data_ptr(), 4,
                           C.byref(p), ids.data_ptr(), d2.data_ptr(), None, None, None)
    assert rc == 5  # CUKD_ERR_UNSUPPORTED
