"""GPU parity against the reference's OWN GPU code, compiled here from its
headers (oracle/_ref/libcukd_ref_gpu.so, -fmad=false): its three builders
(cukd::buildTree_thrust / _bitonic / _inPlace) and its fcp / knn traversals
run one thread per query (the pattern of testing/floatN-knn-and-fcp.cu).

Bar: the records our builders leave in memory are byte-identical to what
each reference builder leaves, world bounds included, for plain float2/3/4,
{float3; int payload}, {float3; int dim} and the 16-byte packed record with
the dim in payload bits; query ids and squared-distance bits are identical,
fixed lists sorted and heap lists in the reference's own heap layout.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from oracle import pyoracle as po
from tests.helpers import f32_bits, make_points, make_queries

pytestmark = pytest.mark.gpu


def _ref():
    L = po.ref_gpu()
    if L is None:
        pytest.skip("oracle/_ref not built")
    return L


# type code -> (D, our layout, explicit dims)
TYPES = {
    po.REF_F2: (2, ck.layout_for("float32", 2), False),
    po.REF_F3: (3, ck.layout_for("float32", 3), False),
    po.REF_F4: (4, ck.layout_for("float32", 4), False),
    po.REF_F3_DIM: (3, ck.layout_for("float32", 3, stride=16, dim_offset=12), True),
    po.REF_F3_PAYLOAD: (3, ck.layout_for("float32", 3, stride=16), False),
    po.REF_F3_PACKED: (3, ck.layout_for("float32", 3, stride=16, dim_offset=12, dim_shift=30,
                                        dim_bits=2), True),
}
BUILDERS = [(0, "thrust"), (1, "bitonic"), (2, "inplace")]


def _records(code, pts):
    D = TYPES[code][0]
    dt = po.ref_record_dtype(code)
    n = len(pts)
    if code in (po.REF_F2, po.REF_F3, po.REF_F4):
        return np.ascontiguousarray(pts[:, :D], np.float32)
    rec = np.zeros(n, dt)
    rec["p"] = pts[:, :D]
    if code == po.REF_F3_DIM:
        rec["dim"] = -1
    elif code == po.REF_F3_PAYLOAD:
        rec["payload"] = np.arange(n, dtype=np.int32)
    elif code == po.REF_F3_PACKED:
        rec["payload"] = np.arange(n, dtype=np.uint32)
    return rec


def _as_device(rec):
    raw = np.ascontiguousarray(rec).view(np.uint8).reshape(-1)
    return torch.from_numpy(raw.copy()).cuda()


def _ref_build(L, code, builder, rec, n, D):
    d = _as_device(rec)
    wb = torch.zeros((2, D), dtype=torch.float32, device="cuda")
    assert L.refg_build(code, builder, C.c_void_p(d.data_ptr()), n, C.c_void_p(wb.data_ptr())) == 0
    return d, wb


def _coords_dims(code, raw, n):
    """Coordinates [n, D] and split dims (None: round robin) of a built
    record array, and the records with their dim bits cleared."""
    D = TYPES[code][0]
    if code in (po.REF_F2, po.REF_F3, po.REF_F4):
        t = raw.view(np.float32).reshape(n, D)
        return t, None, t
    r = raw.view(po.ref_record_dtype(code)).copy()
    t = np.ascontiguousarray(r["p"], np.float32).reshape(n, D)
    dims = None
    if code == po.REF_F3_DIM:
        dims = r["dim"].astype(np.int32)
        r["dim"] = -1
    elif code == po.REF_F3_PACKED:
        dims = (r["payload"] >> 30).astype(np.int32)
        r["payload"] &= np.uint32(0x3FFFFFFF)
    return t, dims, r


def _check_valid_same_records(code, rec, d_ours, wb, n):
    raw = d_ours.cpu().numpy()
    t, dims, cleared = _coords_dims(code, raw, n)
    assert po.check_kd(t, dims, wb.cpu().numpy() if dims is not None else None) == 0
    a = np.ascontiguousarray(cleared).view(np.uint8).reshape(n, -1)
    b = np.ascontiguousarray(rec).view(np.uint8).reshape(n, -1)
    row = np.dtype((np.void, a.shape[1]))
    assert np.array_equal(np.sort(a.view(row).ravel()), np.sort(b.view(row).ravel()))


def _kd_violations(t, dims):
    """Nodes whose left subtree holds a larger, or right subtree a smaller,
    coordinate along the node's split dim."""
    n = len(t)
    bad = 0
    for g in range(n):
        dim = dims[g]
        for child, side in ((2 * g + 1, 0), (2 * g + 2, 1)):
            stack, vals = [child], []
            while stack:
                y = stack.pop()
                if y < n:
                    vals.append(t[y, dim])
                    stack += [2 * y + 1, 2 * y + 2]
            if vals and ((side == 0 and max(vals) > t[g, dim]) or
                         (side == 1 and min(vals) < t[g, dim])):
                bad += 1
    return bad


@pytest.mark.parametrize("code", list(TYPES))
@pytest.mark.parametrize("builder,bname", BUILDERS)
# sizes of the reference's own builder test (testing/testBuildersSameResult.cu:
# 4, 10, 1000, 10000) plus one deeper tree
@pytest.mark.parametrize("n", [4, 10, 1000, 10000, 30000])
@pytest.mark.parametrize("kind", ["uniform", "tie"])
def test_builders_match_reference_gpu_builders(code, builder, bname, n, kind):
    """Every builder name gives the tree of the reference's buildTree_thrust
    (its default, builder.h:108-122), records and world bounds byte for
    byte -- except our "inplace" builder on points that share coordinates,
    which has no storage for the input order and returns a valid k-d tree of
    the same records instead (the reference's own in-place builder promises
    no more, testing/testBuildersSameResult.cu:96-99).  The reference's
    bitonic and inPlace builders give the thrust tree when no two points
    share a coordinate -- except buildTree_inPlace on 3-D points, whose
    output is not a valid k-d tree (see the next test); with shared
    coordinates their unstable sorts may order equal keys differently."""
    L = _ref()
    D, lay, explicit = TYPES[code]
    pts = make_points(n, 4, kind, seed=n + builder)
    rec = _records(code, pts)
    d_thrust, wb_ref = _ref_build(L, code, 0, rec, n, D)
    d_ours = _as_device(rec)
    wb = ck.build_tree(d_ours, layout=lay, builder=bname, n=n)
    ck.build_check()
    distinct = all(len(np.unique(pts[:, d])) == n for d in range(D))
    if bname == "inplace" and not distinct:
        # no storage for the input order: a valid tree of the same records
        _check_valid_same_records(code, rec, d_ours, wb, n)
    else:
        assert torch.equal(d_ours, d_thrust)
    assert torch.equal(wb, wb_ref)
    if builder != 0 and distinct and not (builder == 2 and D == 3):
        d_var, wb_var = _ref_build(L, code, builder, rec, n, D)
        assert torch.equal(d_var, d_thrust)
        assert torch.equal(wb_var, wb_ref)


def test_reference_inplace_builder_breaks_the_kd_property_in_3d():
    """Why the inPlace comparison above uses the thrust tree for 3-D types:
    the reference's buildTree_inPlace<float3> (builder_inplace.h) leaves
    nodes whose subtrees cross their split plane (float2 / float4 are
    fine).  Our "inplace" builder returns the valid canonical tree."""
    L = _ref()
    n = 1000
    pts = make_points(n, 3, "uniform", seed=5)
    rr = np.arange(n)
    dims = (np.floor(np.log2(rr + 1)).astype(int)) % 3
    d_in, _ = _ref_build(L, po.REF_F3, 2, np.ascontiguousarray(pts), n, 3)
    t_in = d_in.cpu().numpy().view(np.float32).reshape(n, 3)
    assert _kd_violations(t_in, dims) > 0
    d_ours = torch.from_numpy(pts.copy()).cuda()
    ck.build_tree(d_ours, builder="inplace")
    assert _kd_violations(d_ours.cpu().numpy(), dims) == 0


def _built(code, n, kind, seed):
    D, lay, _ = TYPES[code]
    pts = make_points(n, 4, kind, seed=seed)
    d = _as_device(_records(code, pts))
    wb = ck.build_tree(d, layout=lay, n=n)
    torch.cuda.synchronize()
    return d, lay, wb


@pytest.mark.parametrize("code", [po.REF_F3, po.REF_F3_DIM, po.REF_F3_PACKED, po.REF_F2])
@pytest.mark.parametrize("method,mname", [(0, "stack_based"), (1, "stack_free"), (2, "cct")])
@pytest.mark.parametrize("kind", ["uniform", "tie"])
@pytest.mark.parametrize("cutoff", [np.inf, 0.08])
def test_queries_match_reference_gpu_traversals(code, method, mname, kind, cutoff):
    L = _ref()
    D = TYPES[code][0]
    n, nq = 20000, 6000
    d, lay, wb = _built(code, n, kind, seed=3)
    q = make_queries(nq, D, kind, seed=4)
    if kind == "tie":
        cutoff = cutoff * 20
    dq = torch.from_numpy(q).cuda()
    hb = np.ascontiguousarray(wb.cpu().numpy())
    hbp = hb.ctypes.data_as(C.c_void_p)
    # FCP
    rid = torch.empty(nq, dtype=torch.int32, device="cuda")
    assert L.refg_fcp(code, method, C.c_void_p(d.data_ptr()), n, hbp,
                      C.c_void_p(dq.data_ptr()), nq, float(cutoff), 0.0,
                      C.c_void_p(rid.data_ptr())) == 0
    ids = ck.fcp(d, dq, mname, layout=lay, world_bounds=wb, cutoff=cutoff, n=n)
    assert torch.equal(ids, rid)
    # kNN: the reference GPU arm instantiates fixed lists k = 1, 8, 16 and
    # heap lists k = 20, 32, 64
    for list_kind, k in ((0, 1), (0, 8), (0, 16), (1, 20), (1, 32), (1, 64)):
        ri = torch.empty((nq, k), dtype=torch.int32, device="cuda")
        rd = torch.empty((nq, k), dtype=torch.float32, device="cuda")
        assert L.refg_knn(code, method, list_kind, k, C.c_void_p(d.data_ptr()), n, hbp,
                          C.c_void_p(dq.data_ptr()), nq, float(cutoff),
                          C.c_void_p(ri.data_ptr()), C.c_void_p(rd.data_ptr())) == 0
        gi, gd = ck.knn(d, dq, k, mname, layout=lay, world_bounds=wb, cutoff=cutoff, n=n,
                        heap_order=bool(list_kind), force_heap=bool(list_kind))
        assert torch.equal(gi, ri), (list_kind, k)
        assert np.array_equal(f32_bits(gd.cpu().numpy()), f32_bits(rd.cpu().numpy())), (list_kind, k)
        if list_kind:
            # the default (sorted) output is the heap's content in (d2, id) order
            si, sd = ck.knn(d, dq, k, mname, layout=lay, world_bounds=wb, cutoff=cutoff, n=n)
            key_ref = (rd.cpu().numpy().view(np.uint32).astype(np.uint64) << 32) | \
                ri.cpu().numpy().view(np.uint32).astype(np.uint64)
            key = (sd.cpu().numpy().view(np.uint32).astype(np.uint64) << 32) | \
                si.cpu().numpy().view(np.uint32).astype(np.uint64)
            assert np.array_equal(np.sort(key_ref, axis=1), key)
