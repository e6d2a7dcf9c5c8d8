"""GPU parity of the sharded kNN (cukd_knn_accumulate / cukd_knn_lists_extract,
the device step of the reference's samples/mpiHugeQuery.cu ring) against the
ring oracle: candidate lists bit-identical to the k smallest (d2, global id)
keys over every shard folded in, in any shard order, and k-th distances
bit-identical to what the reference writes."""
import math

import numpy as np
import pytest
import torch

import cudakdtree_b200 as ck
from cudakdtree_b200 import io as kio
from cudakdtree_b200 import shard
from oracle import ring_oracle as ro

pytestmark = pytest.mark.gpu


def _points(n, D, seed, tie=False):
    rng = np.random.Generator(np.random.MT19937(seed))
    if tie:
        return rng.integers(0, 5, size=(n, D)).astype(np.float32)
    return rng.random((n, D), dtype=np.float64).astype(np.float32)


def _check(lists, keys, k):
    got = lists.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, keys)
    ids, d2, kth = shard.lists_extract(lists, k)
    wids, wd2, wkth = ro.extract(keys)
    assert np.array_equal(ids.cpu().numpy(), wids)
    assert np.array_equal(d2.cpu().numpy().view(np.uint32), wd2.view(np.uint32))
    assert np.array_equal(kth.cpu().numpy().view(np.uint32), wkth.view(np.uint32))


@pytest.mark.parametrize("D", [2, 3, 4])
@pytest.mark.parametrize("k", [1, 8, 16, 32, 33, 64, 128])
@pytest.mark.parametrize("tie", [False, True])
@pytest.mark.parametrize("radius", [math.inf, 0.08])
def test_accumulate_matches_oracle(D, k, tie, radius):
    sizes = [1200, 0, 37, 2500]
    shards = [_points(n, D, seed=10 * D + i, tie=tie) for i, n in enumerate(sizes)]
    q = _points(3000, D, seed=99 + D, tie=tie)
    if tie:
        radius = radius * 20
    dq = torch.from_numpy(q).cuda()
    lists = shard.new_lists(len(q), k, dq.device)
    keys = ro.init_keys(len(q), k, radius)
    order = ck.morton_order(dq)
    off = 0
    for i, s in enumerate(shards):
        t = torch.from_numpy(s.copy()).cuda()
        wb = ck.build_tree(t) if len(s) else None
        tree = t.cpu().numpy()
        shard.knn_accumulate(t, dq, k, lists, id_offset=off, init=(i == 0), max_radius=radius,
                             layout=ck.layout_for("float32", D), world_bounds=wb,
                             order=order if i % 2 else None, n=len(s))
        keys = ro.fold(keys, q, tree, off)
        off += len(s)
        torch.cuda.synchronize()
        _check(lists, keys, k)


def test_accumulate_explicit_dim_records():
    """Shards stored as {float3; int dim} records with widest-extent dims."""
    k = 16
    pts = [_points(n, 3, seed=n) for n in (3000, 1700)]
    q = _points(2000, 3, seed=5)
    dq = torch.from_numpy(q).cuda()
    lay = ck.layout_for("float32", 3, stride=16, dim_offset=12)
    lists = shard.new_lists(len(q), k, dq.device)
    keys = ro.init_keys(len(q), k, math.inf)
    off = 0
    for i, s in enumerate(pts):
        rec = np.zeros((len(s), 4), np.float32)
        rec[:, :3] = s
        t = torch.from_numpy(rec).cuda()
        wb = ck.build_tree(t, layout=lay)
        shard.knn_accumulate(t, dq, k, lists, id_offset=off, init=(i == 0), layout=lay,
                             world_bounds=wb)
        keys = ro.fold(keys, q, t.cpu().numpy()[:, :3].copy(), off)
        off += len(s)
    torch.cuda.synchronize()
    _check(lists, keys, k)


@pytest.mark.parametrize("num_shards", [1, 3, 4])
def test_sharded_all_points_knn_like_mpi_huge_query(tmp_path, num_shards):
    """The mpiHugeQuery workload on one GPU: a raw float3 file split into
    rank portions, every portion's points queried against every portion, the
    k-th distances appended in rank order -- equal to the oracle's."""
    k = 10
    pts = _points(6007, 3, seed=num_shards)
    path = tmp_path / "in.float3s"
    path.write_bytes(pts.tobytes())
    parts = [kio.read_file_portion(path, r, num_shards)[0].reshape(-1, 3)
             for r in range(num_shards)]
    res, trees = shard.sharded_knn([torch.from_numpy(p.copy()).cuda() for p in parts], k)
    out = tmp_path / "out.dat"
    kio.write_rank_ordered(out, np.concatenate([r[2].cpu().numpy() for r in res]))
    built = np.concatenate([t.cpu().numpy() for t in trees])
    want = ro.fold(ro.init_keys(len(pts), k, math.inf), pts, built, 0)
    wids, _, wkth = ro.extract(want)
    got = np.fromfile(out, np.float32)
    assert np.array_equal(got.view(np.uint32), wkth.view(np.uint32))
    ids = np.concatenate([r[0].cpu().numpy() for r in res])
    assert np.array_equal(ids, wids)


def test_invalid_arguments():
    t = torch.zeros((10, 3), device="cuda")
    q = torch.zeros((4, 3), device="cuda")
    lists = shard.new_lists(4, 8, q.device)
    for kw in ({"k": 0}, {"k": 129}):
        with pytest.raises(ck.CukdError):
            shard.knn_accumulate(t, q, kw["k"], lists, init=True)
    with pytest.raises(ck.CukdError):
        shard.knn_accumulate(t, q, 8, lists, init=True, id_offset=(1 << 32) - 5)
