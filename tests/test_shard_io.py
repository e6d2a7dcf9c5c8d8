"""CPU tests of the sharded-kNN ring's host side and of the reference's file
formats: the ring oracle pinned to the reference's own host traversal, the
file readers/writers against the reference's layouts, and the ring schedule
(exchange, id offsets, round order) run by two and three gloo ranks with the
oracle's fold standing in for the GPU step."""
import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from cudakdtree_b200 import io as kio
from oracle import pyoracle as po
from oracle import ring_oracle as ro

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _points(n, D=3, seed=0, tie=False):
    rng = np.random.Generator(np.random.MT19937(seed))
    if tie:
        return rng.integers(0, 5, size=(n, D)).astype(np.float32)
    return rng.random((n, D), dtype=np.float64).astype(np.float32)


# ---------------------------------------------------------------------------
# the oracle against the reference
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("k", [8, 16, 64])
@pytest.mark.parametrize("tie", [False, True])
def test_ring_oracle_kth_matches_reference_knn(k, tie):
    """The k-th distance over all shards equals the reference's knn()
    return value over one tree of all points (a property of the point set)."""
    if po.ref_host() is None:
        pytest.skip("oracle/_ref not built")
    pts = _points(3000, seed=k + tie, tie=tie)
    shards = [pts[:700], pts[700:1900], pts[1900:]]
    keys = ro.init_keys(len(pts), k, math.inf)
    off = 0
    for s in shards:
        keys = ro.fold(keys, pts, s, off)
        off += len(s)
    _, _, kth = ro.extract(keys)
    perm, _, bounds = po.build(pts)
    tree = pts[perm]
    _, _, ret = po.ref_knn_host(po.REF_F3, tree, bounds, pts, k, po.STACK_FREE)
    want = np.where(np.isinf(ret), ret, np.sqrt(ret).astype(np.float32))
    assert np.array_equal(kth.view(np.uint32), want.view(np.uint32))


# ---------------------------------------------------------------------------
# file formats
# ---------------------------------------------------------------------------
def test_load_save_points_round_trip(tmp_path):
    """cukd::loadPoints layout: uint64 count, then raw records."""
    pts = _points(1234, 3, seed=1)
    p = tmp_path / "pts.bin"
    kio.save_points(p, pts)
    raw = p.read_bytes()
    assert np.frombuffer(raw[:8], "<u8")[0] == 1234 and len(raw) == 8 + 1234 * 12
    back = kio.load_points(p, kio.FLOAT3)
    assert np.array_equal(back.reshape(-1, 3), pts)
    rec = np.dtype([("p", np.float32, (3,)), ("payload", np.int32)])
    r = np.zeros(10, rec)
    r["payload"] = np.arange(10)
    kio.save_points(tmp_path / "r.bin", r)
    assert np.array_equal(kio.load_points(tmp_path / "r.bin", rec)["payload"], np.arange(10))


def test_load_points_rejects_truncated_files(tmp_path):
    p = tmp_path / "bad.bin"
    p.write_bytes(np.array([5], "<u8").tobytes() + b"\0" * 12)
    with pytest.raises(ValueError):
        kio.load_points(p, kio.FLOAT3)


@pytest.mark.parametrize("total", [0, 1, 7, 100, 1001])
@pytest.mark.parametrize("size", [1, 2, 3, 5])
def test_file_portions_partition_the_file(tmp_path, total, size):
    """mpiHugeQuery.cu:41-63: rank r reads [N*r/s, N*(r+1)/s)."""
    pts = _points(total, 3, seed=total)
    p = tmp_path / "raw.float3s"
    p.write_bytes(pts.tobytes())
    parts = []
    for r in range(size):
        data, begin, n = kio.read_file_portion(p, r, size)
        assert n == total and begin == total * r // size
        parts.append(data.view(np.float32).reshape(-1, 3))
    assert np.array_equal(np.concatenate(parts), pts)


def test_write_rank_ordered_single_process(tmp_path):
    p = tmp_path / "out.dat"
    kio.write_rank_ordered(p, np.array([1.5, 2.5], np.float32))
    assert np.array_equal(np.fromfile(p, np.float32), [1.5, 2.5])


# ---------------------------------------------------------------------------
# the ring on gloo ranks
# ---------------------------------------------------------------------------
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, path, outdir, k):
    import sys
    from datetime import timedelta
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from cudakdtree_b200 import io as kio
    from cudakdtree_b200 import shard
    from oracle import ring_oracle as ro
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        data, begin, total = kio.read_file_portion(path, rank, world)
        local = torch.from_numpy(data.view(np.float32).reshape(-1, 3).copy())

        def build(points):
            p = points.numpy()
            b = np.stack([p.min(0), p.max(0)]) if len(p) else np.zeros((2, 3), np.float32)
            return points.clone(), torch.from_numpy(b.astype(np.float32))

        def step(tree, n, bounds, off, queries, lists, init):
            q = queries.numpy()
            keys = ro.init_keys(len(q), k, math.inf) if init else lists.numpy().view(np.uint64)
            keys = ro.fold(keys, q, tree.numpy()[:n], off)
            lists.copy_(torch.from_numpy(keys.view(np.int64)))

        def extract(lists):
            return ro.extract(lists.numpy().view(np.uint64))

        ids, d2, kth, _ = shard.ring_knn(local, k, build=build, step=step, extract=extract)
        np.save(os.path.join(outdir, f"ids{rank}.npy"), ids)
        kio.write_rank_ordered(os.path.join(outdir, "kth.dat"), kth, rank, world)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ring_schedule_on_gloo_ranks(tmp_path, world):
    """Every rank's points against every shard, ids global, the k-th
    distances written in rank order -- equal to one fold over all points."""
    k = 8
    pts = _points(2000 + world, 3, seed=world)
    path = tmp_path / "in.float3s"
    path.write_bytes(pts.tobytes())
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, str(path), str(tmp_path), k))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    want = ro.fold(ro.init_keys(len(pts), k, math.inf), pts, pts, 0)
    wids, _, wkth = ro.extract(want)
    got = np.fromfile(tmp_path / "kth.dat", np.float32)
    assert np.array_equal(got.view(np.uint32), wkth.view(np.uint32))
    ids = np.concatenate([np.load(tmp_path / f"ids{r}.npy") for r in range(world)])
    assert np.array_equal(ids, wids)
