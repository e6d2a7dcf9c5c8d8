"""The allocation-free builder, cukd_build_tree_noalloc.

It exists for callers that cannot allocate device memory when they build a
tree (their device memory belongs to another framework's pool, or they run
in a loop that cannot risk an allocation's latency or failure): all of its
scratch lives in one fixed device array inside the library.  It must build
exactly the tree that the allocating entry point builds, call after call,
since every call reuses (and must re-initialise) the same array.

This file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from tests.helpers import make_points

pytestmark = pytest.mark.gpu


def _noalloc(t, layout, n, wb):
    L = ck.lib()
    L.cukd_build_tree_noalloc.argtypes = [C.c_void_p, C.c_int64, C.POINTER(ck.Layout),
                                          C.c_void_p, C.c_void_p]
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return L.cukd_build_tree_noalloc(C.c_void_p(t.data_ptr()), n, C.byref(layout),
                                     C.c_void_p(wb.data_ptr()) if wb is not None else None,
                                     stream)


def _records(pts, n, D):
    rec = np.zeros((n, D + 1), np.int32)
    rec[:, :D] = pts.view(np.int32)
    rec[:, D] = np.arange(n, dtype=np.int32)
    return rec


CASES = [  # (n, D, kind, explicit) -- two calls in a row, different shapes
    (200000, 3, "gmm", True),
    (5000, 3, "tie", False),
]


def test_noalloc_matches_allocating_builder_on_consecutive_calls():
    for n, D, kind, explicit in CASES:
        pts = make_points(n, D, kind, seed=n)
        rec = _records(pts, n, D)
        if explicit:
            lay = ck.layout_for("float32", D, stride=4 * (D + 1), dim_offset=4 * D,
                                dim_shift=30, dim_bits=2)
        else:
            lay = ck.layout_for("float32", D, stride=4 * (D + 1))
        ref = torch.from_numpy(rec).cuda()
        wb_ref = ck.build_tree(ref, layout=lay)
        got = torch.from_numpy(rec).cuda()
        wb = torch.empty((2, D), dtype=torch.float32, device="cuda")
        assert _noalloc(got, lay, n, wb) == 0
        torch.cuda.synchronize()
        assert torch.equal(got, ref), f"tree differs (n={n})"
        assert torch.equal(wb, wb_ref)


@pytest.mark.parametrize("scalar", ["float32", "int32"])
def test_noalloc_at_its_documented_limit(scalar):
    """The largest input the fixed scratch is documented to take: 262144
    records of 64 bytes with D = 4 and explicit dims, float and int, twice
    in a row, each equal to the allocating builder's tree."""
    n, D, stride = 262144, 4, 64
    words = stride // 4
    for seed in (1, 2):
        pts = make_points(n, D, "uniform", scalar=scalar, seed=seed)
        rec = np.zeros((n, words), np.int32)
        rec[:, :D] = pts.view(np.int32)
        rec[:, D + 1] = np.arange(n, dtype=np.int32)
        lay = ck.layout_for(scalar, D, stride=stride, dim_offset=4 * D, dim_bits=32)
        ref = torch.from_numpy(rec).cuda()
        wb_ref = ck.build_tree(ref, layout=lay)
        got = torch.from_numpy(rec).cuda()
        wb = torch.empty((2, D), dtype=wb_ref.dtype, device="cuda")
        assert _noalloc(got, lay, n, wb) == 0
        torch.cuda.synchronize()
        assert torch.equal(got, ref), f"tree differs ({scalar}, call {seed})"
        assert torch.equal(wb, wb_ref)


def test_noalloc_rejects_inputs_beyond_its_scratch():
    n = 262145
    t = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    assert _noalloc(t, ck.layout_for("float32", 3), n, None) == 8  # CUKD_ERR_TOO_LARGE
    wide = torch.zeros((16, 20), dtype=torch.float32, device="cuda")
    assert _noalloc(wide, ck.layout_for("float32", 3, stride=80), 16, None) == 8
