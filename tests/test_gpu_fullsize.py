"""Parity at the benchmark configurations' full sizes.

Every other GPU test compares with the oracle on inputs small enough to
rebuild in a second; these run the five configurations' own workloads
(seeded generators of cudakdtree_b200.workloads) through the CUDA path and
compare byte for byte with the CPU oracle: whole trees where the oracle's
recursive build finishes in seconds (1M, 10M, 20M points), the canonical-
tree checker (oracle cko_check_tree, pinned to the reference's own
buildTree_host in test_oracle.py) for the 100M-point float4 tree, and query
answers (ids and squared-distance bits) on samples of each configuration's
queries.  Reference: builder_thrust.h:514-601 (buildTree_host),
knn.h:549-678, fcp.h:210-254.
"""
import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from cudakdtree_b200 import workloads as wl
from oracle import pyoracle as po
from tests.helpers import f32_bits

pytestmark = pytest.mark.gpu

METHODS = [("stack_based", po.STACK_BASED), ("stack_free", po.STACK_FREE), ("cct", po.CCT)]
PACKED = ck.layout_for("float32", 3, stride=16, dim_offset=12, dim_shift=30, dim_bits=2)


def _knn_equal(ids, d2, ri, rd):
    assert np.array_equal(ids.cpu().numpy(), ri)
    got = d2.cpu().numpy()
    if got.dtype == np.float32:
        assert np.array_equal(f32_bits(got), f32_bits(rd))
    else:
        assert np.array_equal(got, rd)


def test_c1_uniform_1m_round_robin():
    """Config 1: 1M uniform float3, round-robin dims; FCP and kNN k = 8 for
    all 1M uniform queries with every traversal."""
    n = nq = 1_000_000
    pts = wl.uniform_points(n, seed=1)
    q = wl.uniform_points(nq, seed=2)
    perm, _, bounds = po.build(pts)
    d = torch.from_numpy(pts).cuda()
    wb = ck.build_tree(d)
    tree = pts[perm]
    assert np.array_equal(d.cpu().numpy(), tree)
    assert np.array_equal(wb.cpu().numpy(), bounds)
    dq = torch.from_numpy(q).cuda()
    for name, m in METHODS:
        fi = ck.fcp(d, dq, name, world_bounds=wb)
        assert np.array_equal(fi.cpu().numpy(), po.fcp(tree, q, m, bounds=bounds)), name
        ids, d2 = ck.knn(d, dq, 8, name, world_bounds=wb)
        ri, rd, _ = po.knn(tree, q, 8, m, bounds=bounds)
        _knn_equal(ids, d2, ri, rd)


@pytest.fixture(scope="module")
def c2():
    """Config 2's 10M mixture points as the benchmark's packed 16-byte
    records, their oracle build and the queries."""
    n = 10_000_000
    pts = wl.gmm_points(n, seed=3)
    perm, dims, bounds = po.build(pts, explicit_dim=True)
    recs = wl.packed_records(pts).view(np.int32).reshape(n, 4).copy()
    q = wl.gmm_points(1_000_000, seed=3, sample_seed=4)
    return pts, recs, perm, dims, bounds, q


@pytest.mark.parametrize("builder", ["thrust", "bitonic"])
def test_c2_gmm_10m_build_every_builder(c2, builder):
    """The whole 10M-point tree (order and explicit dims) of the default
    and bitonic builders equals the oracle's."""
    pts, recs, perm, dims, bounds, _ = c2
    d = torch.from_numpy(recs).cuda()
    wb = ck.build_tree(d, layout=PACKED, builder=builder)
    ck.build_check()
    out = d.cpu().numpy()
    pay = out[:, 3].view(np.uint32)
    assert np.array_equal(pay & 0x3FFFFFFF, perm.astype(np.uint32))
    assert np.array_equal(pay >> 30, dims.astype(np.uint32))
    assert np.array_equal(out[:, :3].view(np.float32), pts[perm])
    assert np.array_equal(wb.cpu().numpy(), bounds)


def test_c2_gmm_10m_build_inplace(c2):
    """The in-place builder on the 10M mixture records (which share
    coordinate values): a valid k-d tree with the widest-extent dims of its
    domain boxes, holding every record once, the oracle's world bounds; and
    the same tree on a second run."""
    pts, recs, perm, dims, bounds, _ = c2
    d = torch.from_numpy(recs).cuda()
    wb = ck.build_tree(d, layout=PACKED, builder="inplace")
    ck.build_check()
    out = d.cpu().numpy()
    pay = out[:, 3].view(np.uint32)
    assert np.array_equal(np.sort(pay & 0x3FFFFFFF), np.arange(len(pts), dtype=np.uint32))
    idx = (pay & 0x3FFFFFFF).astype(np.int64)
    assert np.array_equal(out[:, :3].view(np.float32), pts[idx])
    assert np.array_equal(wb.cpu().numpy(), bounds)
    assert po.check_kd(out[:, :3].view(np.float32), (pay >> 30).astype(np.int32), bounds) == 0
    d2 = torch.from_numpy(recs).cuda()
    ck.build_tree(d2, layout=PACKED, builder="inplace")
    assert torch.equal(d2, d)


@pytest.fixture(scope="module")
def c2_tree(c2):
    pts, recs, perm, dims, bounds, q = c2
    d = torch.from_numpy(recs).cuda()
    wb = ck.build_tree(d, layout=PACKED)
    return d, wb, pts[perm], dims, bounds, q


@pytest.mark.parametrize("name,m", METHODS[:2])
def test_c2_gmm_10m_knn16(c2_tree, name, m):
    """kNN k = 16 on the 10M-point tree for 1M of the mixture queries."""
    d, wb, tree, dims, bounds, q = c2_tree
    ids, d2 = ck.knn(d, torch.from_numpy(q).cuda(), 16, name, layout=PACKED, world_bounds=wb)
    ri, rd, _ = po.knn(tree, q, 16, m, dims=dims, bounds=bounds)
    _knn_equal(ids, d2, ri, rd)


def test_c2_gmm_10m_learned_knn16(c2_tree):
    """The learned-radius path on the 10M-point tree, trained as the
    benchmark trains it, against the oracle directly (not only against the
    plain GPU path)."""
    d, wb, tree, dims, bounds, q = c2_tree
    m = ck.RadiusModel(grid_res=64, seed=1)
    qt = torch.from_numpy(wl.gmm_points(1_000_000, seed=3, sample_seed=14)).cuda()
    m.fit(d, qt, 16, layout=PACKED, world_bounds=wb, epochs=10, batch=4096)
    qs = q[:300_000]
    ids, d2, fb, _ = ck.knn_learned(d, torch.from_numpy(qs).cuda(), 16, m, "stack_based",
                                    layout=PACKED, world_bounds=wb, scale=1.2)
    ri, rd, _ = po.knn(tree, qs, 16, po.STACK_BASED, dims=dims, bounds=bounds)
    _knn_equal(ids, d2, ri, rd)
    assert int(fb[0]) < 0.1 * len(qs)


def test_c5_int3_20m_build_and_knn64():
    """Config 5, integer part: 20M int3 points in [-2^20, 2^20]^3 (round-robin
    dims), the whole tree, and kNN k = 64 (exact int64 distances) for a
    sample of 100K queries from the same distribution."""
    n = 20_000_000
    pts = wl.int3_points(n)
    perm, _, bounds = po.build(pts)
    d = torch.from_numpy(pts).cuda()
    wb = ck.build_tree(d)
    tree = pts[perm]
    assert np.array_equal(d.cpu().numpy(), tree)
    assert np.array_equal(wb.cpu().numpy(), bounds)
    q = wl.int3_points(100_000, seed=9)
    ids, d2 = ck.knn(d, torch.from_numpy(q).cuda(), 64, world_bounds=wb)
    ri, rd, _ = po.knn(tree, q, 64, po.STACK_BASED, bounds=bounds)
    _knn_equal(ids, d2, ri, rd)


# the reference's {float4 p; int dim;} record: 32 bytes (float4 is 16-byte
# aligned); the test keeps each point's input index in the padding
F4_RECORD = np.dtype({"names": ["p", "dim", "index"],
                      "formats": [(np.float32, (4,)), np.int32, np.int32],
                      "offsets": [0, 16, 20], "itemsize": 32})
F4_LAYOUT = ck.layout_for("float32", 4, stride=32, dim_offset=16, dim_bits=32)


def test_c5_float4_100m_canonical_tree_and_knn64():
    """Config 5, float part: 100M float4 points (xyz uniform, w normal) with
    widest-extent dims.  Too large to rebuild on the CPU here, so the tree
    is checked with the canonical-tree property (order against every
    ancestor under the composite key, every dim the widest extent of its
    domain box); kNN k = 64 against the oracle on 50K queries."""
    n = 100_000_000
    pts = wl.wide_float4(n)
    rec = np.zeros(n, F4_RECORD)
    rec["p"] = pts
    rec["dim"] = -1
    rec["index"] = np.arange(n, dtype=np.int32)
    del pts
    d = torch.from_numpy(rec.view(np.uint8)).cuda()
    wb = ck.build_tree(d, layout=F4_LAYOUT)
    out = d.cpu().numpy().view(F4_RECORD)
    del d
    tree = np.ascontiguousarray(out["p"])
    idx = out["index"].astype(np.int64)
    dims = np.ascontiguousarray(out["dim"])
    bounds = wb.cpu().numpy()
    assert np.array_equal(np.sort(idx), np.arange(n))
    assert np.array_equal(bounds, np.stack([tree.min(0), tree.max(0)]))
    assert po.check_tree(tree, idx, dims, bounds) == 0
    q = wl.wide_float4(50_000, seed=10)
    dt = torch.from_numpy(out.view(np.uint8)).cuda()
    ids, d2 = ck.knn(dt, torch.from_numpy(q).cuda(), 64, layout=F4_LAYOUT, world_bounds=wb)
    ri, rd, _ = po.knn(tree, q, 64, po.STACK_BASED, dims=dims, bounds=bounds)
    _knn_equal(ids, d2, ri, rd)
