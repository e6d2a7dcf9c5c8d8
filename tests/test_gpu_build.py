"""GPU parity of the left-balanced builders against the CPU oracle.

Bar: bit-exact -- the same point order (ties included, broken like the
reference's chain of stable sorts), the same explicit split dims, the same
world bounds.  Behaviours ported from the reference's tests:
testBuilderEmptyInput.cu (n = 0), testBuilderSimpleInput.cu (smoke builds),
testBuildersSameResult.cu (all builders give byte-identical trees on
unique-int inputs, D = 2/3/4, float and int, point-only / payload /
payload+dim), floatN-knn-and-fcp.cu:387-470 (tree validity recursion).
"""
import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from oracle import pyoracle as po
from tests.helpers import make_points

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 4, 5, 7, 8, 10, 31, 100, 1000, 1023, 1024, 1025, 2047, 2048, 2049, 3000,
         4097, 10000, 50000, 200000]


def _gpu_build_plain(pts, builder="default"):
    t = torch.from_numpy(pts).cuda()
    wb = ck.build_tree(t, builder=builder)
    torch.cuda.synchronize()
    return t.cpu().numpy(), wb.cpu().numpy()


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("D", [2, 3, 4])
@pytest.mark.parametrize("kind", ["uniform", "tie"])
def test_round_robin_float(n, D, kind):
    pts = make_points(n, D, kind, seed=n + D)
    perm, _, bounds = po.build(pts)
    out, wb = _gpu_build_plain(pts)
    assert np.array_equal(out, pts[perm])
    assert np.array_equal(wb, bounds)


@pytest.mark.parametrize("n", [1, 5, 1000, 3000, 50000])
@pytest.mark.parametrize("D", [2, 3, 4])
@pytest.mark.parametrize("kind", ["uniform", "tie"])
def test_round_robin_int(n, D, kind):
    pts = make_points(n, D, kind, scalar="int32", seed=n)
    perm, _, bounds = po.build(pts)
    out, wb = _gpu_build_plain(pts)
    assert np.array_equal(out, pts[perm])
    assert np.array_equal(wb, bounds)


def _payload_records(pts):
    """[n, D+1] int32 records: coordinates (as bits) + input index."""
    n, D = pts.shape
    rec = np.zeros((n, D + 1), np.int32)
    rec[:, :D] = pts.view(np.int32) if pts.dtype == np.float32 else pts
    rec[:, D] = np.arange(n, dtype=np.int32)
    return rec


@pytest.mark.parametrize("n", [1, 2, 100, 1025, 2049, 20000, 100000])
@pytest.mark.parametrize("kind", ["tie", "same", "gmm"])
def test_payload_order_follows_input_index(n, kind):
    """Identical points must come out in the reference's order too: the
    payload exposes it (stable sorts keep the input order of ties)."""
    pts = make_points(n, 3, kind, seed=3)
    perm, _, _ = po.build(pts)
    rec = _payload_records(pts)
    t = torch.from_numpy(rec).cuda()
    lay = ck.layout_for("float32", 3, stride=16)
    ck.build_tree(t, layout=lay)
    out = t.cpu().numpy()
    assert np.array_equal(out[:, 3], perm.astype(np.int32))


@pytest.mark.parametrize("n", [1, 2, 3, 9, 1000, 2049, 5000, 60000, 250000])
@pytest.mark.parametrize("kind", ["uniform", "tie", "gmm"])
@pytest.mark.parametrize("packed", [False, True])
def test_explicit_dims(n, kind, packed):
    pts = make_points(n, 3, kind, seed=n)
    perm, dims, bounds = po.build(pts, explicit_dim=True)
    rec = _payload_records(pts)
    if packed:  # dim in payload bits 30..31 (the 16-byte config-2 record)
        lay = ck.layout_for("float32", 3, stride=16, dim_offset=12, dim_shift=30, dim_bits=2)
    else:       # {float3 p; int dim;} -- the payload column is the dim field
        rec[:, 3] = 0x5a5a5a5a
        lay = ck.layout_for("float32", 3, stride=16, dim_offset=12, dim_shift=0, dim_bits=32)
    t = torch.from_numpy(rec).cuda()
    wb = ck.build_tree(t, layout=lay)
    out = t.cpu().numpy()
    assert np.array_equal(out[:, :3].view(np.float32), pts[perm])
    if packed:
        assert np.array_equal(out[:, 3].view(np.uint32) & 0x3fffffff, perm.astype(np.uint32))
        assert np.array_equal(out[:, 3].view(np.uint32) >> 30, dims.astype(np.uint32))
    else:
        assert np.array_equal(out[:, 3], dims)
    assert np.array_equal(wb.cpu().numpy(), bounds)


@pytest.mark.parametrize("D", [2, 4])
@pytest.mark.parametrize("scalar", ["float32", "int32"])
def test_explicit_dims_other_types(D, scalar):
    n = 30000
    pts = make_points(n, D, "tie" if scalar == "int32" else "uniform", scalar=scalar, seed=D)
    perm, dims, bounds = po.build(pts, explicit_dim=True)
    rec = np.zeros((n, D + 1), np.int32)
    rec[:, :D] = pts.view(np.int32)
    lay = ck.layout_for(scalar, D, stride=4 * (D + 1), dim_offset=4 * D)
    t = torch.from_numpy(rec).cuda()
    ck.build_tree(t, layout=lay)
    out = t.cpu().numpy()
    assert np.array_equal(out[:, :D].view(pts.dtype), pts[perm])
    assert np.array_equal(out[:, D], dims)


@pytest.mark.parametrize("builder", ["default", "thrust", "bitonic", "inplace"])
@pytest.mark.parametrize("n", [4, 10, 1000, 10000])
@pytest.mark.parametrize("D", [2, 3, 4])
def test_builders_same_result(builder, n, D):
    pts = make_points(n, D, "unique", seed=D)
    perm, _, _ = po.build(pts)
    out, _ = _gpu_build_plain(pts, builder=builder)
    assert np.array_equal(out, pts[perm])


def test_empty_input_is_a_noop():
    t = torch.empty((0, 3), dtype=torch.float32, device="cuda")
    ck.build_tree(t)
    lay = ck.layout_for("float32", 3, stride=16, dim_offset=12)
    t2 = torch.empty((0, 4), dtype=torch.int32, device="cuda")
    ck.build_tree(t2, layout=lay)


def test_explicit_dims_without_bounds_is_an_error():
    """builder_thrust.h:469-473 throws; the C ABI returns status 2."""
    lay = ck.layout_for("float32", 3, stride=16, dim_offset=12)
    t = torch.zeros((10, 4), dtype=torch.int32, device="cuda")
    n = 10
    import ctypes as C
    rc = ck.lib().cukd_build_tree(C.c_void_p(t.data_ptr()), n, C.byref(lay), None, 0, None,
                                  None)
    assert rc == 2


def _check_rec(tree, dims, n, lo, hi, node):
    """floatN-knn-and-fcp.cu:387-470 checkRec: every node inside the box
    its ancestors' planes carve out."""
    stack = [(0, lo.copy(), hi.copy())]
    while stack:
        node, l, h = stack.pop()
        if node >= n:
            continue
        p = tree[node]
        assert np.all(p >= l) and np.all(p <= h), node
        d = dims[node]
        lh = h.copy()
        lh[d] = p[d]
        rl = l.copy()
        rl[d] = p[d]
        stack.append((2 * node + 1, l, lh))
        stack.append((2 * node + 2, rl, h))


@pytest.mark.parametrize("explicit", [False, True])
def test_tree_validity(explicit):
    n = 100000
    pts = make_points(n, 3, "gmm", seed=9)
    rec = _payload_records(pts)
    if explicit:
        lay = ck.layout_for("float32", 3, stride=16, dim_offset=12, dim_shift=30, dim_bits=2)
    else:
        lay = ck.layout_for("float32", 3, stride=16)
    t = torch.from_numpy(rec).cuda()
    ck.build_tree(t, layout=lay)
    out = t.cpu().numpy()
    tree = out[:, :3].view(np.float32)
    if explicit:
        dims = (out[:, 3].view(np.uint32) >> 30).astype(np.int64)
    else:
        dims = np.array([int(np.floor(np.log2(i + 1))) % 3 for i in range(n)])
    inf = np.full(3, np.inf, np.float32)
    _check_rec(tree, dims, n, -inf, inf, 0)


def test_partition_staging_waits_never_give_up():
    """The partition pass stages each chunk with bulk copies and waits on a
    barrier with a bounded poll count; after builds whose chunks start and
    end at every 16-byte phase (sizes 4097..4100 and a 10^6-point build)
    no wait has given up."""
    before = ck.async_wait_timeouts()  # other tests make waits run out on purpose
    for n in (4097, 4098, 4099, 4100, 1_000_000):
        t = torch.from_numpy(make_points(n, 3, "gmm", seed=n)).cuda()
        ck.build_tree(t)
    torch.cuda.synchronize()
    assert ck.async_wait_timeouts() == before


@pytest.mark.parametrize("offset", [4, 8, 12])
def test_memory_resource_with_any_alignment_builds_the_same_tree(offset):
    """A caller memory resource whose blocks are only 4-byte aligned (the
    reference's GpuMemoryResource makes no alignment promise,
    helpers.h:31-34): the builder aligns each block up itself, builds the
    oracle's tree, and hands every block back with the pointer it got."""
    import ctypes as C
    live = {}
    released = []

    def alloc(ctx, out, nbytes, stream):
        t = torch.empty(int(nbytes) + 64, dtype=torch.uint8, device="cuda")
        p = t.data_ptr() + offset
        live[p] = t
        out[0] = p
        return 0

    def release(ctx, ptr, stream):
        released.append(ptr)
        live.pop(ptr, None)
        return 0

    a_fn = ck._ALLOC_FN(alloc)
    r_fn = ck._RELEASE_FN(release)
    mr = ck.MemResource(None, C.cast(a_fn, C.c_void_p), C.cast(r_fn, C.c_void_p))
    n = 50000
    pts = make_points(n, 3, "tie", seed=11)
    t = torch.from_numpy(pts).cuda()
    lay = ck.layout_for("float32", 3)
    rc = ck.lib().cukd_build_tree(t.data_ptr(), n, C.byref(lay), None, 0, None, C.byref(mr))
    torch.cuda.synchronize()
    assert rc == 0
    perm, _, _ = po.build(pts)
    assert np.array_equal(t.cpu().numpy(), pts[perm])
    assert released and not live  # every block came back, by its own pointer


def test_wait_that_runs_out_leaves_the_points_and_reports_timeout():
    """The partition pass's bounded bulk-copy wait, made to give up at once
    (poll bound 0 through the test hook; the copies still land before the
    CTAs leave): the build stops, every later kernel of it returns at once,
    the caller's records are left exactly as they were, and cukd_build_check
    reports CUKD_ERR_TIMEOUT.  With the default bound restored the next
    build is the oracle's tree again."""
    n = 300000
    pts = make_points(n, 3, "gmm", seed=5)
    ck.build_check()  # clean slate
    before = ck.async_wait_timeouts()
    ck.set_async_wait_polls(0)
    try:
        t = torch.from_numpy(pts).cuda()
        ck.build_tree(t)
        with pytest.raises(ck.CukdError) as err:
            ck.build_check()
        assert err.value.status == 6  # CUKD_ERR_TIMEOUT
        assert np.array_equal(t.cpu().numpy(), pts)
        assert ck.async_wait_timeouts() > before
    finally:
        ck.set_async_wait_polls()
    t = torch.from_numpy(pts).cuda()
    ck.build_tree(t)
    ck.build_check()
    perm, _, _ = po.build(pts)
    assert np.array_equal(t.cpu().numpy(), pts[perm])
