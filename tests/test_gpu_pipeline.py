"""cukd_knn_host / cukd_knn_to_host: kNN with host-resident results (and
host- or device-resident queries), chunked over overlapping streams -- their
answers must equal cukd_knn's bit for bit, for pinned and pageable host
memory and chunk sizes that do and do not divide the query count."""
import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from tests.helpers import f32_bits, make_points, make_queries

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scalar", ["float32", "int32"])
@pytest.mark.parametrize("k", [8, 40])
@pytest.mark.parametrize("chunk", [0, 1000, 7777, 50000])
@pytest.mark.parametrize("pinned", [True, False])
def test_knn_host_equals_knn(scalar, k, chunk, pinned):
    n, nq = 30000, 23456
    pts = make_points(n, 3, "uniform", scalar=scalar, seed=3)
    q = make_queries(nq, 3, "uniform", scalar=scalar, seed=4)
    t = torch.from_numpy(pts).cuda()
    lay = ck.layout_for(scalar, 3)
    wb = ck.build_tree(t, layout=lay)
    ri, rd = ck.knn(t, torch.from_numpy(q).cuda(), k, "stack_based", layout=lay, world_bounds=wb)
    hq = torch.from_numpy(q)
    if pinned:
        hq = hq.pin_memory()
    ids, d2 = ck.knn_host(t, hq, k, "stack_based", layout=lay, world_bounds=wb, chunk=chunk)
    torch.cuda.synchronize()
    assert not ids.is_cuda and ids.is_pinned() == pinned
    assert np.array_equal(ids.numpy(), ri.cpu().numpy())
    if scalar == "float32":
        assert np.array_equal(f32_bits(d2.numpy()), f32_bits(rd.cpu().numpy()))
    else:
        assert np.array_equal(d2.numpy(), rd.cpu().numpy())


def test_knn_host_rejects_device_queries():
    t = torch.from_numpy(make_points(100, 3, "uniform", seed=1)).cuda()
    with pytest.raises(ValueError):
        ck.knn_host(t, t[:4], 4)


@pytest.mark.parametrize("scalar", ["float32", "int32"])
@pytest.mark.parametrize("k", [8, 40])
@pytest.mark.parametrize("chunk", [0, 1000, 7777, 50000])
def test_knn_to_host_equals_knn(scalar, k, chunk):
    n, nq = 30000, 23456
    pts = make_points(n, 3, "uniform", scalar=scalar, seed=5)
    q = make_queries(nq, 3, "uniform", scalar=scalar, seed=6)
    t = torch.from_numpy(pts).cuda()
    lay = ck.layout_for(scalar, 3)
    wb = ck.build_tree(t, layout=lay)
    dq = torch.from_numpy(q).cuda()
    ri, rd = ck.knn(t, dq, k, "stack_free", layout=lay, world_bounds=wb)
    for _ in range(2):  # twice: buffers and streams of the first call are gone
        ids, d2 = ck.knn_to_host(t, dq, k, "stack_free", layout=lay, world_bounds=wb, chunk=chunk)
        torch.cuda.synchronize()
        assert not ids.is_cuda and ids.is_pinned()
        assert np.array_equal(ids.numpy(), ri.cpu().numpy())
        if scalar == "float32":
            assert np.array_equal(f32_bits(d2.numpy()), f32_bits(rd.cpu().numpy()))
        else:
            assert np.array_equal(d2.numpy(), rd.cpu().numpy())


def test_knn_to_host_rejects_host_queries():
    t = torch.from_numpy(make_points(100, 3, "uniform", seed=1)).cuda()
    with pytest.raises(ValueError):
        ck.knn_to_host(t, t[:4].cpu(), 4)


@pytest.mark.parametrize("chunk", [1000, 7777, 50000])
def test_knn_host_async_back_to_back_batches(chunk):
    """cukd_knn_host_async: several trees built and searched back to back on
    one stream, each batch's answers landing behind its own event while the
    next batch builds and searches (the host buffers of a batch reused two
    batches later, after waiting for its event); every batch's answers equal
    cukd_knn's."""
    n, nq, k = 30000, 23456, 8
    lay = ck.layout_for("float32", 3)
    hq = torch.from_numpy(make_queries(nq, 3, "uniform", seed=4)).pin_memory()
    slots = [{"ids": torch.empty((nq, k), dtype=torch.int32).pin_memory(),
              "d2": torch.empty((nq, k), dtype=torch.float32).pin_memory(),
              "done": torch.cuda.Event(), "used": False} for _ in range(2)]
    trees, want = [], []
    for b in range(5):
        t = torch.from_numpy(make_points(n, 3, "uniform", seed=10 + b)).cuda()
        wb = ck.build_tree(t, layout=lay)
        ri, rd = ck.knn(t, hq.cuda(), k, "stack_based", layout=lay, world_bounds=wb)
        trees.append((t, wb))
        want.append((ri.cpu().numpy(), f32_bits(rd.cpu().numpy())))
    torch.cuda.synchronize()
    main = torch.cuda.current_stream()
    for b, (t, wb) in enumerate(trees):
        sl = slots[b % 2]
        if sl["used"]:
            sl["done"].synchronize()  # the batch two back has landed: check it
            ri, rb = want[b - 2]
            assert np.array_equal(sl["ids"].numpy(), ri)
            assert np.array_equal(f32_bits(sl["d2"].numpy()), rb)
        ck.knn_host(t, hq, k, "stack_based", layout=lay, world_bounds=wb, out_ids=sl["ids"],
                    out_d2=sl["d2"], chunk=chunk, done=sl["done"])
        sl["used"] = True
    for b in (3, 4):
        sl = slots[b % 2]
        sl["done"].synchronize()
        assert np.array_equal(sl["ids"].numpy(), want[b][0])
        assert np.array_equal(f32_bits(sl["d2"].numpy()), want[b][1])
    main.synchronize()


@pytest.mark.parametrize("chunk", [0, 2000, 5000])
def test_knn_to_host_async_back_to_back_batches(chunk):
    """cukd_knn_to_host_async: device-resident queries, several trees
    searched back to back on one stream with each batch's answers behind its
    own event; every batch's answers equal cukd_knn's -- in one slice (the
    default), in 12 slices (the eight result sets reused) and in 5."""
    n, nq, k = 30000, 23456, 16
    lay = ck.layout_for("float32", 3)
    dq = torch.from_numpy(make_queries(nq, 3, "uniform", seed=6)).cuda()
    slots = [{"ids": torch.empty((nq, k), dtype=torch.int32).pin_memory(),
              "d2": torch.empty((nq, k), dtype=torch.float32).pin_memory(),
              "done": torch.cuda.Event(), "used": False} for _ in range(2)]
    trees, want = [], []
    for b in range(5):
        t = torch.from_numpy(make_points(n, 3, "gmm", seed=20 + b)).cuda()
        wb = ck.build_tree(t, layout=lay)
        ri, rd = ck.knn(t, dq, k, "stack_based", layout=lay, world_bounds=wb)
        trees.append((t, wb))
        want.append((ri.cpu().numpy(), f32_bits(rd.cpu().numpy())))
    for b, (t, wb) in enumerate(trees):
        sl = slots[b % 2]
        if sl["used"]:
            sl["done"].synchronize()
            assert np.array_equal(sl["ids"].numpy(), want[b - 2][0])
            assert np.array_equal(f32_bits(sl["d2"].numpy()), want[b - 2][1])
        ck.knn_to_host(t, dq, k, "stack_based", layout=lay, world_bounds=wb, out_ids=sl["ids"],
                       out_d2=sl["d2"], chunk=chunk, done=sl["done"])
        sl["used"] = True
    for b in (3, 4):
        sl = slots[b % 2]
        sl["done"].synchronize()
        assert np.array_equal(sl["ids"].numpy(), want[b][0])
        assert np.array_equal(f32_bits(sl["d2"].numpy()), want[b][1])


def test_knn_to_host_async_with_a_caller_memory_resource():
    """With the caller's memory resource the result buffers come from it
    (taken and released on the copy stream) instead of the library's pool:
    once `done` has completed every block is back, and the answers equal
    cukd_knn's."""
    import ctypes as C
    n, nq, k = 30000, 23456, 16
    lay = ck.layout_for("float32", 3)
    t = torch.from_numpy(make_points(n, 3, "gmm", seed=8)).cuda()
    wb = ck.build_tree(t, layout=lay)
    dq = torch.from_numpy(make_queries(nq, 3, "gmm", seed=9)).cuda()
    ri, rd = ck.knn(t, dq, k, "stack_based", layout=lay, world_bounds=wb)
    blocks, taken = {}, [0]

    def alloc(ctx, out, nbytes, stream):
        buf = torch.empty(int(nbytes), dtype=torch.uint8, device="cuda")
        blocks[buf.data_ptr()] = buf
        taken[0] += 1
        out[0] = buf.data_ptr()
        return 0

    def release(ctx, ptr, stream):
        blocks.pop(ptr)
        return 0

    a_fn, r_fn = ck._ALLOC_FN(alloc), ck._RELEASE_FN(release)
    mr = ck.MemResource(None, C.cast(a_fn, C.c_void_p), C.cast(r_fn, C.c_void_p))
    ids = torch.empty((nq, k), dtype=torch.int32).pin_memory()
    d2 = torch.empty((nq, k), dtype=torch.float32).pin_memory()
    p = ck.QueryParams()
    ck.lib().cukd_query_params_init(p)
    p.k = k
    done = torch.cuda.Event()
    ck._init_event(done, torch.cuda.current_stream())
    rc = ck.lib().cukd_knn_to_host_async(t.data_ptr(), n, C.byref(lay), wb.data_ptr(),
                                         dq.data_ptr(), nq, C.byref(p), ids.data_ptr(),
                                         d2.data_ptr(), 4000, C.c_void_p(done.cuda_event),
                                         C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                         C.byref(mr))
    assert rc == 0
    done.synchronize()
    torch.cuda.synchronize()
    assert taken[0] > 0 and not blocks
    assert np.array_equal(ids.numpy(), ri.cpu().numpy())
    assert np.array_equal(f32_bits(d2.numpy()), f32_bits(rd.cpu().numpy()))
