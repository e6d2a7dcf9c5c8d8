"""GPU parity of the batched-clouds path (cukd_batch_*) against a per-cloud
loop of the oracle's build and traversals.

Bar: every cloud's slice of the built array is bit-identical to the
oracle's tree for that cloud alone, every per-cloud box equals the
oracle's bounds, and every query's ids and squared-distance bits equal the
oracle's answer against its own cloud (ids local to the cloud) -- for all
three subtree tiles, every query tuning, the CUDA-graph replay, and after
the autotuner.
"""
import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from cudakdtree_b200 import workloads as wl
from oracle import pyoracle as po
from tests.helpers import f32_bits

pytestmark = pytest.mark.gpu

METHODS = {"stack_based": po.STACK_BASED, "stack_free": po.STACK_FREE, "cct": po.CCT}

# sizes around every tile boundary, empty and tiny clouds, and clouds deep
# enough for several top-down levels
EDGE_SIZES = [0, 1, 2, 3, 7, 100, 255, 256, 511, 512, 513, 1000, 1023, 1024, 1025, 2047,
              2048, 2049, 3000, 4097, 9000, 20000, 0, 5]


def _clouds(sizes, D=3, kind="uniform", nq_max=300, seed=0):
    rng = np.random.Generator(np.random.MT19937(seed + 17))
    sizes = np.asarray(sizes, np.int64)
    nqs = rng.integers(0, nq_max + 1, size=sizes.size)
    nqs[::7] = 0
    total = int(sizes.sum())
    if kind == "tie":
        pts = rng.integers(0, 6, size=(total, D)).astype(np.float32)
        qs = rng.integers(-1, 7, size=(int(nqs.sum()), D)).astype(np.float32)
    else:
        pts = rng.random((total, D), dtype=np.float64).astype(np.float32)
        qs = (rng.random((int(nqs.sum()), D)) * 1.2 - 0.1).astype(np.float32)
    po_ = np.zeros(sizes.size + 1, np.int64)
    po_[1:] = np.cumsum(sizes)
    qo = np.zeros(sizes.size + 1, np.int64)
    qo[1:] = np.cumsum(nqs)
    return pts, po_, qs, qo


def _oracle(pts, poff, qs, qoff, k, method, list_kind=po.FIXED_LIST, cutoff=np.inf):
    """Per-cloud loop: build, then query against that cloud alone."""
    D = pts.shape[1]
    B = poff.size - 1
    tree = np.empty_like(pts)
    bounds = np.zeros((B, 2, D), np.float32)
    kk = max(k, 1)
    ids = np.full((qs.shape[0], kk), -7, np.int32)
    d2 = np.zeros((qs.shape[0], kk), np.float32)
    for c in range(B):
        p = pts[poff[c]:poff[c + 1]]
        q = qs[qoff[c]:qoff[c + 1]]
        if p.shape[0]:
            perm, _, bnd = po.build(p)
            t = p[perm]
            bounds[c] = bnd
        else:
            t = p
            bnd = np.zeros((2, D), np.float32)
        tree[poff[c]:poff[c + 1]] = t
        if q.shape[0] == 0:
            continue
        if k == 0:
            ids[qoff[c]:qoff[c + 1], 0] = po.fcp(t, q, method, bounds=bnd, cutoff=cutoff)
        else:
            i, d, _ = po.knn(t, q, k, method, bounds=bnd, cutoff=cutoff, list_kind=list_kind)
            ids[qoff[c]:qoff[c + 1]] = i
            d2[qoff[c]:qoff[c + 1]] = d
    return tree, bounds, ids, d2


def _check(plan, pts, poff, qs, qoff, ref, bounds_dev=None, built=None, got=None):
    tree, bounds, ids, d2 = ref
    B = poff.size - 1
    if built is not None:
        assert np.array_equal(f32_bits(built), f32_bits(tree))
    if bounds_dev is not None:
        b = bounds_dev.cpu().numpy()
        ne = np.diff(poff) > 0
        assert np.array_equal(b[ne], bounds[ne])
        assert np.all(np.isposinf(b[~ne][:, 0])) and np.all(np.isneginf(b[~ne][:, 1]))
    if got is not None:
        gi, gd = got
        gi = gi.cpu().numpy().reshape(qs.shape[0], -1)
        assert np.array_equal(gi, ids[:, :gi.shape[1]])
        if plan.k > 0:
            gd = gd.cpu().numpy().reshape(qs.shape[0], -1)
            assert np.array_equal(f32_bits(gd), f32_bits(d2))


def _run_build_query(plan, pts, qs):
    P = torch.from_numpy(pts).cuda()
    Q = torch.from_numpy(qs).cuda()
    bnd = plan.bounds_tensor(P.device)
    plan.build(P, bnd)
    got = plan.query(P, Q, bnd)
    torch.cuda.synchronize()
    return P.cpu().numpy(), bnd, got


@pytest.mark.parametrize("kind", ["uniform", "tie"])
@pytest.mark.parametrize("tile", [512, 1024, 2048])
def test_build_and_knn_every_tile(kind, tile):
    pts, poff, qs, qoff = _clouds(EDGE_SIZES, 3, kind, seed=tile)
    ref = _oracle(pts, poff, qs, qoff, 8, po.STACK_BASED)
    plan = ck.BatchPlan(poff, qoff, 3, k=8)
    plan.set_tuning(build_tile=tile)
    built, bnd, got = _run_build_query(plan, pts, qs)
    _check(plan, pts, poff, qs, qoff, ref, bnd, built, got)


@pytest.mark.parametrize("D", [2, 4])
def test_other_dimensions(D):
    pts, poff, qs, qoff = _clouds(EDGE_SIZES[:18], D, "uniform", seed=D)
    ref = _oracle(pts, poff, qs, qoff, 5, po.STACK_BASED)
    plan = ck.BatchPlan(poff, qoff, D, k=5)
    plan.set_tuning(build_tile=512)
    built, bnd, got = _run_build_query(plan, pts, qs)
    _check(plan, pts, poff, qs, qoff, ref, bnd, built, got)


@pytest.mark.parametrize("method", ["stack_based", "stack_free", "cct"])
@pytest.mark.parametrize("k", [0, 1, 4, 16, 32, 40])
def test_methods_and_k(method, k):
    pts, poff, qs, qoff = _clouds(EDGE_SIZES, 3, "tie" if k in (1, 16) else "uniform", seed=k)
    # k > 32 runs the heap list; its output is sorted like the fixed list's
    ref = _oracle(pts, poff, qs, qoff, k, METHODS[method])
    plan = ck.BatchPlan(poff, qoff, 3, k=k, method=method)
    built, bnd, got = _run_build_query(plan, pts, qs)
    _check(plan, pts, poff, qs, qoff, ref, bnd, built, got)


@pytest.mark.parametrize("k", [0, 1, 40])
def test_512_thread_blocks_where_other_kernels_answer(k):
    """A 512-thread block tuning also where the heap kernel (k > 32) and the
    reference-order kernels (FCP, k = 1, the exact fallbacks of tie-heavy
    points) answer: those take at most 256 threads and are launched so."""
    pts, poff, qs, qoff = _clouds(EDGE_SIZES, 3, "tie", seed=40 + k)
    ref = _oracle(pts, poff, qs, qoff, k, po.STACK_BASED)
    plan = ck.BatchPlan(poff, qoff, 3, k=k)
    plan.set_tuning(block_size=512, queries_per_thread=2)
    built, bnd, got = _run_build_query(plan, pts, qs)
    _check(plan, pts, poff, qs, qoff, ref, bnd, built, got)


def test_cutoff_radius():
    pts, poff, qs, qoff = _clouds(EDGE_SIZES, 3, "uniform", seed=3)
    ref = _oracle(pts, poff, qs, qoff, 8, po.STACK_BASED, cutoff=0.05)
    plan = ck.BatchPlan(poff, qoff, 3, k=8, cutoff=0.05)
    built, bnd, got = _run_build_query(plan, pts, qs)
    _check(plan, pts, poff, qs, qoff, ref, bnd, built, got)


@pytest.mark.parametrize("block,qpt,morton", [(32, 1, 1), (64, 4, 0), (256, 2, 1), (128, 1, 0),
                                             (512, 1, 1), (512, 4, 0)])
def test_query_tunings_same_answers(block, qpt, morton):
    pts, poff, qs, qoff = _clouds(EDGE_SIZES, 3, "uniform", seed=9)
    ref = _oracle(pts, poff, qs, qoff, 8, po.STACK_BASED)
    plan = ck.BatchPlan(poff, qoff, 3, k=8)
    plan.set_tuning(block_size=block, queries_per_thread=qpt, morton=morton)
    built, bnd, got = _run_build_query(plan, pts, qs)
    _check(plan, pts, poff, qs, qoff, ref, bnd, built, got)


def test_graph_replay_follows_new_inputs():
    pts, poff, qs, qoff = _clouds(EDGE_SIZES, 3, "uniform", seed=21)
    plan = ck.BatchPlan(poff, qoff, 3, k=8)
    P = torch.from_numpy(pts).cuda()
    Q = torch.from_numpy(qs).cuda()
    out = plan._outputs(P.device)
    bnd = plan.bounds_tensor(P.device)
    before = ck.launch_count()
    for rep in range(3):
        # same buffers, new contents: the recorded graph must read them afresh
        rng = np.random.Generator(np.random.MT19937(100 + rep))
        p2 = rng.random(pts.shape).astype(np.float32)
        q2 = rng.random(qs.shape).astype(np.float32)
        P.copy_(torch.from_numpy(p2))
        Q.copy_(torch.from_numpy(q2))
        plan.run(P, Q, bnd, out=out)
        torch.cuda.synchronize()
        ref = _oracle(p2, poff, q2, qoff, 8, po.STACK_BASED)
        _check(plan, p2, poff, q2, qoff, ref, bnd, P.cpu().numpy(), out)
    assert ck.launch_count() > before


def test_autotune_keeps_points_and_answers():
    pts, poff, qs, qoff = _clouds(EDGE_SIZES, 3, "uniform", seed=33)
    ref = _oracle(pts, poff, qs, qoff, 8, po.STACK_BASED)
    plan = ck.BatchPlan(poff, qoff, 3, k=8)
    P = torch.from_numpy(pts).cuda()
    Q = torch.from_numpy(qs).cuda()
    t = plan.autotune(P, Q, reps=3)
    torch.cuda.synchronize()
    assert np.array_equal(f32_bits(P.cpu().numpy()), f32_bits(pts))
    assert t.build_tile in (512, 1024, 2048)
    assert t.block_size in (64, 128, 256, 512) and t.queries_per_thread in (1, 2, 4)
    assert t.morton in (0, 1) and t.build_ms > 0 and t.query_ms > 0
    assert plan.tuning.as_dict() == t.as_dict()
    bnd = plan.bounds_tensor(P.device)
    got = plan.run(P, Q, bnd)
    torch.cuda.synchronize()
    _check(plan, pts, poff, qs, qoff, ref, bnd, P.cpu().numpy(), got)


def test_invalid_arguments():
    poff = np.array([0, 10, 5], np.int64)  # decreasing
    qoff = np.array([0, 1, 2], np.int64)
    with pytest.raises(ck.CukdError):
        ck.BatchPlan(poff, qoff, 3, k=8)
    plan = ck.BatchPlan(np.array([0, 10]), np.array([0, 4]), 3, k=8)
    with pytest.raises(ck.CukdError):
        plan.set_tuning(build_tile=4096)
    with pytest.raises(ck.CukdError):
        plan.set_tuning(block_size=48)
    with pytest.raises(ck.CukdError):
        plan.set_tuning(block_size=544)
    with pytest.raises(ck.CukdError):
        ck.BatchPlan(np.array([0, 10]), np.array([0, 4]), 5, k=8)


def test_config3_shape_sampled_parity():
    """The workload of the batched benchmark at full size (4096 clouds,
    sizes log-uniform in [256, 65536], 1024 queries each, k = 8): every
    cloud's slice keeps its points (per-cloud coordinate sums), and a sample
    of clouds, the largest and smallest included, matches the oracle."""
    pts, poff, qs, qoff = wl.batched_clouds()
    plan = ck.BatchPlan(poff, qoff, 3, k=8)
    P = torch.from_numpy(pts).cuda()
    Q = torch.from_numpy(qs).cuda()
    bnd = plan.bounds_tensor(P.device)
    ids, d2 = plan.run(P, Q, bnd)
    torch.cuda.synchronize()
    built = P.cpu().numpy()
    ids = ids.cpu().numpy()
    d2 = d2.cpu().numpy()
    sizes = np.diff(poff)
    seg = np.repeat(np.arange(sizes.size), sizes)
    for d in range(3):
        a = np.bincount(seg, weights=pts[:, d].astype(np.float64), minlength=sizes.size)
        b = np.bincount(seg, weights=built[:, d].astype(np.float64), minlength=sizes.size)
        assert np.allclose(a, b, rtol=0, atol=1e-6)
    sample = sorted({int(np.argmax(sizes)), int(np.argmin(sizes)), 0, sizes.size - 1,
                     *np.random.Generator(np.random.MT19937(4)).choice(sizes.size, 8).tolist()})
    bb = bnd.cpu().numpy()
    for c in sample:
        p = pts[poff[c]:poff[c + 1]]
        q = qs[qoff[c]:qoff[c + 1]]
        perm, _, b0 = po.build(p)
        t = p[perm]
        assert np.array_equal(f32_bits(built[poff[c]:poff[c + 1]]), f32_bits(t)), c
        assert np.array_equal(bb[c], b0)
        i, d, _ = po.knn(t, q, 8, po.STACK_BASED, bounds=b0)
        assert np.array_equal(ids[qoff[c]:qoff[c + 1]], i), c
        assert np.array_equal(f32_bits(d2[qoff[c]:qoff[c + 1]]), f32_bits(d)), c


def test_large_query_cloud_takes_global_morton_sort():
    """A cloud with more queries than the per-cloud shared-memory sort holds
    sends the whole batch through the global radix sort: same answers."""
    rng = np.random.Generator(np.random.MT19937(71))
    sizes = np.array([5000, 300, 0, 2500], np.int64)
    nqs = np.array([9000, 50, 10, 0], np.int64)
    pts = rng.random((int(sizes.sum()), 3)).astype(np.float32)
    qs = rng.random((int(nqs.sum()), 3)).astype(np.float32)
    poff = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    qoff = np.concatenate([[0], np.cumsum(nqs)]).astype(np.int64)
    ref = _oracle(pts, poff, qs, qoff, 8, po.STACK_BASED)
    plan = ck.BatchPlan(poff, qoff, 3, k=8)
    built, bnd, got = _run_build_query(plan, pts, qs)
    _check(plan, pts, poff, qs, qoff, ref, bnd, built, got)
