"""The bounded-memory builders behind the reference's buildTree_bitonic and
buildTree_inPlace names (cukd/builder_bitonic.h, cukd/builder_inplace.h).

- bitonic: the canonical tree (the oracle's, ties included), with at most
  4 bytes per point of temporary memory plus a fixed amount;
- inplace: the canonical tree whenever the coordinates decide every split
  (unique coordinates: the reference's own same-result test,
  testing/testBuildersSameResult.cu:96-128), otherwise a valid
  left-balanced k-d tree (checkRec, floatN-knn-and-fcp.cu:387-470) over the
  same records, the same every time; temporary memory independent of n.

Sizes cover trees finished by the shared-memory subtree phase alone
(n <= 1024), by levels spread over all CTAs (up to 128 subtrees) and by
levels with one CTA per subtree (n > 2^18).
"""
import ctypes as C

import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from oracle import pyoracle as po
from tests.helpers import make_points

pytestmark = pytest.mark.gpu

SIZES = [1, 2, 3, 7, 1000, 1024, 1025, 4097, 50000, 300000, 1_200_000]


def _rr_dims(n, D):
    lv = np.floor(np.log2(np.arange(n, dtype=np.float64) + 1)).astype(np.int64)
    return lv % D


def _sorted_rows(a):
    a = np.ascontiguousarray(a)
    v = a.view(np.dtype((np.void, a.dtype.itemsize * a.shape[1])))
    return np.sort(v.ravel())


def _build(arr, builder, layout=None):
    t = torch.from_numpy(arr).cuda()
    wb = ck.build_tree(t, layout=layout, builder=builder)
    ck.build_check()
    return t.cpu().numpy(), wb.cpu().numpy()


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("D", [2, 3, 4])
@pytest.mark.parametrize("kind", ["uniform", "tie", "gmm"])
def test_bitonic_is_the_canonical_tree(n, D, kind):
    pts = make_points(n, D, kind, seed=n + D)
    perm, _, bounds = po.build(pts)
    out, wb = _build(pts, "bitonic")
    assert np.array_equal(out, pts[perm])
    assert np.array_equal(wb, bounds)


@pytest.mark.parametrize("n", [5, 1000, 50000, 300000])
@pytest.mark.parametrize("D", [2, 3])
def test_bitonic_int_and_explicit_dims(n, D):
    """int32 coordinates with ties, payload = input index, explicit split dims
    in the top bits of the payload word: order and dims are the oracle's."""
    pts = make_points(n, D, "tie", scalar="int32", seed=n)
    perm, dims, bounds = po.build(pts, explicit_dim=True)
    rec = np.zeros((n, D + 1), np.int32)
    rec[:, :D] = pts
    rec[:, D] = np.arange(n, dtype=np.int32)
    lay = ck.layout_for("int32", D, stride=4 * (D + 1), dim_offset=4 * D, dim_shift=30, dim_bits=2)
    out, wb = _build(rec, "bitonic", lay)
    pay = out[:, D].view(np.uint32)
    assert np.array_equal(pay & 0x3FFFFFFF, perm.astype(np.uint32))
    assert np.array_equal(pay >> 30, dims.astype(np.uint32))
    assert np.array_equal(wb, bounds)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("D", [2, 3, 4])
@pytest.mark.parametrize("scalar", ["float32", "int32"])
def test_inplace_unique_coordinates_give_the_canonical_tree(n, D, scalar):
    pts = make_points(n, D, "unique", seed=n + 3 * D)
    if scalar == "float32":
        pts = pts.astype(np.float32)
    else:
        pts = pts.astype(np.int32)
    perm, _, bounds = po.build(pts)
    out, wb = _build(pts, "inplace")
    assert np.array_equal(out, pts[perm])
    assert np.array_equal(wb, bounds)


@pytest.mark.parametrize("n", [1000, 50000, 300000, 1_200_000])
def test_inplace_unique_coordinates_explicit_dims(n):
    """Payload records with explicit dims: on unique coordinates the order
    and the dims are the oracle's."""
    D = 3
    pts = make_points(n, D, "unique", seed=n).astype(np.float32)
    perm, dims, bounds = po.build(pts, explicit_dim=True)
    rec = np.zeros((n, 4), np.int32)
    rec[:, :3] = pts.view(np.int32)
    rec[:, 3] = np.arange(n, dtype=np.int32)
    lay = ck.layout_for("float32", 3, stride=16, dim_offset=12, dim_shift=30, dim_bits=2)
    out, wb = _build(rec, "inplace", lay)
    pay = out[:, 3].view(np.uint32)
    assert np.array_equal(pay & 0x3FFFFFFF, perm.astype(np.uint32))
    assert np.array_equal(pay >> 30, dims.astype(np.uint32))
    assert np.array_equal(wb, bounds)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("D", [2, 3, 4])
@pytest.mark.parametrize("kind", ["tie", "gmm", "same"])
def test_inplace_with_ties_is_a_valid_tree_of_the_same_points(n, D, kind):
    pts = make_points(n, D, kind, seed=n + 5 * D)
    out, wb = _build(pts, "inplace")
    assert np.array_equal(_sorted_rows(out), _sorted_rows(pts))
    assert po.check_kd(out) == 0
    assert np.array_equal(wb, np.stack([pts.min(0), pts.max(0)]))
    again, _ = _build(pts, "inplace")
    assert np.array_equal(again, out)  # a function of the input array


@pytest.mark.parametrize("n", [1000, 50000, 300000, 1_200_000])
@pytest.mark.parametrize("scalar", ["float32", "int32"])
def test_inplace_with_ties_explicit_dims_and_duplicate_records(n, scalar):
    """Tie-heavy coordinates, every record present three times byte for byte
    (the split must move exactly as many twins of the pivot as its rank
    asks), explicit dims in a payload word: a valid tree with the dims of
    its domain boxes, the same records, the oracle's world bounds."""
    D = 3
    base = make_points(n // 3 + 1, D, "tie", scalar=scalar, seed=n)
    pts = np.concatenate([base, base, base])[:n]
    rec = np.zeros((n, 4), np.int32)
    rec[:, :3] = pts.view(np.int32)
    rec[:, 3] = (np.arange(n) % (n // 3 + 1)).astype(np.int32)  # payload repeats too
    lay = ck.layout_for(scalar, 3, stride=16, dim_offset=12, dim_shift=30, dim_bits=2)
    out, wb = _build(rec, "inplace", lay)
    pay = out[:, 3].view(np.uint32)
    dims = (pay >> 30).astype(np.int32)
    back = out.copy()
    back[:, 3] = (pay & 0x3FFFFFFF).view(np.int32)
    assert np.array_equal(_sorted_rows(back), _sorted_rows(rec))
    tree = out[:, :3].view(pts.dtype)
    assert np.array_equal(wb, np.stack([pts.min(0), pts.max(0)]))
    assert po.check_kd(tree, dims, wb) == 0


@pytest.mark.parametrize("builder", ["bitonic", "inplace"])
@pytest.mark.parametrize("stride", [12, 20, 64])
def test_record_strides(builder, stride):
    """float3 points at offset 4 of records of 12, 20 and 64 bytes (the
    64-byte one with explicit dims in its last word), the rest payload."""
    n = 300000
    pts = make_points(n, 3, "unique", seed=stride).astype(np.float32)
    words = stride // 4
    rec = np.zeros((n, words), np.int32)
    off = 0 if stride == 12 else 1
    rec[:, off:off + 3] = pts.view(np.int32)
    for w in range(words):
        if not off <= w < off + 3:
            rec[:, w] = np.arange(n, dtype=np.int32) * (w + 1)
    explicit = stride == 64
    perm, dims, bounds = po.build(pts, explicit_dim=explicit)
    lay = ck.layout_for("float32", 3, stride=stride, point_offset=4 * off,
                        dim_offset=stride - 4 if explicit else -1, dim_bits=32)
    out, wb = _build(rec, builder, lay)
    want = rec[perm].copy()
    if explicit:
        want[:, words - 1] = dims
    assert np.array_equal(out, want)
    assert np.array_equal(wb, bounds)


class _CountingResource:
    """A cukd_mem_resource that records the peak of its live bytes."""

    def __init__(self):
        self.live, self.peak, self.blocks = 0, 0, {}

        def alloc(ctx, out, nbytes, stream):
            t = torch.empty(int(nbytes), dtype=torch.uint8, device="cuda")
            self.blocks[t.data_ptr()] = t
            self.live += int(nbytes)
            self.peak = max(self.peak, self.live)
            out[0] = t.data_ptr()
            return 0

        def release(ctx, ptr, stream):
            t = self.blocks.pop(ptr)
            self.live -= t.numel()
            return 0

        self._a = ck._ALLOC_FN(alloc)
        self._r = ck._RELEASE_FN(release)
        self.mr = ck.MemResource(None, C.cast(self._a, C.c_void_p), C.cast(self._r, C.c_void_p))


def _peak_bytes(n, builder):
    pts = make_points(n, 3, "gmm", seed=n)
    t = torch.from_numpy(pts).cuda()
    lay = ck.layout_for("float32", 3)
    res = _CountingResource()
    code = ck.BUILDERS[builder]
    rc = ck.lib().cukd_build_tree(t.data_ptr(), n, C.byref(lay), None, code, None, C.byref(res.mr))
    torch.cuda.synchronize()
    assert rc == 0
    ck.build_check()
    assert res.live == 0 and not res.blocks
    assert po.check_kd(t.cpu().numpy()) == 0
    return res.peak


def test_temporary_memory_budgets():
    """inplace: the same fixed amount at 300K and 3M points, under 8 MiB
    (the reference's in-place builder takes none, builder_inplace.h:441-480;
    this one keeps a few MB of fixed scratch); bitonic: 4 bytes per point
    (the reference's uint32 tags, builder_bitonic.h:263-266) plus that fixed
    amount; the default builder, for contrast, about 65 bytes per point."""
    small, large = 300000, 3_000_000
    ip_s, ip_l = _peak_bytes(small, "inplace"), _peak_bytes(large, "inplace")
    assert ip_s == ip_l and ip_l < 8 << 20
    bt_l = _peak_bytes(large, "bitonic")
    assert bt_l <= 4 * large + 1024 + ip_l
    assert _peak_bytes(large, "default") > 40 * large


def test_barrier_wait_that_runs_out_reports_timeout():
    """The top levels' grid barriers poll a bounded number of times; made to
    give up at once (poll bound 0), the build stops, cukd_build_check
    reports CUKD_ERR_TIMEOUT, and the caller's array still holds every
    record once (swaps only ever exchange records).  With the default bound
    back the next build is right again."""
    n = 300000
    pts = make_points(n, 3, "gmm", seed=21)
    ck.build_check()
    ck.set_async_wait_polls(0)
    try:
        t = torch.from_numpy(pts).cuda()
        ck.build_tree(t, builder="inplace")
        with pytest.raises(ck.CukdError) as err:
            ck.build_check()
        assert err.value.status == 6
        assert np.array_equal(_sorted_rows(t.cpu().numpy()), _sorted_rows(pts))
    finally:
        ck.set_async_wait_polls()
    out, _ = _build(pts, "inplace")
    assert po.check_kd(out) == 0
