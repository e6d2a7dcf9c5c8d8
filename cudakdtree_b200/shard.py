"""Sharded kNN: the all-points k-nearest-neighbour ring of the reference's
samples/mpiHugeQuery.cu, B200-style.

Each rank holds one shard of the points (``io.read_file_portion``), builds a
tree over it, and uses its own points as queries.  In P rounds the trees
travel around the ring (rank r sends to r+1, receives from r-1) while every
rank folds the tree it holds into its queries' candidate lists
(``cukd_knn_accumulate``).  The reference does this with MPI and one
blocking exchange per round (mpiHugeQuery.cu:173-205); here the exchange is
torch.distributed point-to-point (NCCL over NVLink between GPUs), posted
before the round's traversal so that the next shard travels while the
current one is searched.  Candidate ids are global point indices (the
reference keeps shard-local ids, :84-86, which cannot tell shards apart);
the k-th distances are the reference's output bit for bit.

``sharded_knn`` runs the same rounds over shards that one process holds (a
single GPU) with no collective.
"""
from __future__ import annotations

import ctypes as C
import math

import torch

from . import _check, _ptr, _stream, build_tree, infer_layout, layout_for, lib, morton_order


def new_lists(num_queries, k, device):
    """Device storage for candidate lists (uint64 keys kept in an int64 tensor)."""
    return torch.empty((num_queries, k), dtype=torch.int64, device=device)


def knn_accumulate(tree, queries, k, lists, id_offset=0, init=False, max_radius=math.inf,
                   layout=None, world_bounds=None, order=None, n=None, stream=None):
    """Folds the built tree ``tree`` (a shard) into ``lists`` [nq, k]."""
    layout = layout or infer_layout(tree)
    if n is None:
        n = tree.numel() * tree.element_size() // layout.stride
    nq = queries.shape[0]
    _check(lib().cukd_knn_accumulate(_ptr(tree), n, C.byref(layout), _ptr(world_bounds),
                                     int(id_offset), _ptr(queries.contiguous()), nq, _ptr(order),
                                     k, float(max_radius), int(bool(init)), _ptr(lists),
                                     _stream(stream)), "cukd_knn_accumulate")
    return lists


def lists_extract(lists, k, stream=None):
    """(ids [nq,k] int32, -1 = unfilled; d2 [nq,k]; k-th distance [nq])."""
    nq = lists.shape[0]
    dev = lists.device
    ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
    d2 = torch.empty((nq, k), dtype=torch.float32, device=dev)
    kth = torch.empty(nq, dtype=torch.float32, device=dev)
    _check(lib().cukd_knn_lists_extract(_ptr(lists), nq, k, _ptr(ids), _ptr(d2), _ptr(kth),
                                        _stream(stream)), "cukd_knn_lists_extract")
    return ids, d2, kth


def _build(points):
    tree = points.clone()
    bounds = build_tree(tree, layout=layout_for("float32", points.shape[1]))
    return tree, bounds


def sharded_knn(shards, k, max_radius=math.inf, morton=True):
    """Every shard's points against all shards (one process, no collective).
    ``shards``: list of float [n_i, D] CUDA tensors.  Returns (results,
    trees): per shard (ids, d2, kth) for its points in input order, and the
    built shards; an id indexes the concatenation of the built shards."""
    P = len(shards)
    D = shards[0].shape[1]
    lay = layout_for("float32", D)
    begins = [0]
    for s in shards:
        begins.append(begins[-1] + s.shape[0])
    trees = [_build(s) for s in shards]
    out = []
    for i in range(P):
        q = shards[i].contiguous()
        order = morton_order(q) if (morton and q.shape[0] > 1) else None
        lists = new_lists(q.shape[0], k, q.device)
        for r in range(P):
            j = (i - r) % P
            tree, bounds = trees[j]
            knn_accumulate(tree, q, k, lists, id_offset=begins[j], init=(r == 0),
                           max_radius=max_radius, layout=lay, world_bounds=bounds, order=order,
                           n=shards[j].shape[0])
        out.append(lists_extract(lists, k))
    return out, [t for t, _ in trees]


def ring_knn(local_points, k, max_radius=math.inf, group=None, morton=True, build=None,
             step=None, extract=None):
    """All-points kNN over the ring of ranks of ``group``: this rank's points
    (float [n, D]) are its shard and its queries.  Returns (ids, d2, kth, tree)
    for this rank's points in input order, with ``tree`` this rank's built
    shard; an id indexes the rank-ordered concatenation of the built shards.

    ``build(points) -> (tree, bounds)``, ``step(tree, n, bounds, id_offset,
    queries, lists, init)`` and ``extract(lists) -> (ids, d2, kth)`` default
    to the GPU library; they are parameters so that the ring itself can be
    exercised with host stand-ins on CPU process groups."""
    import torch.distributed as dist
    P = dist.get_world_size(group)
    r = dist.get_rank(group)
    dev = local_points.device
    D = local_points.shape[1]
    lay = layout_for("float32", D)
    build = build or _build
    library_step = step is None
    if library_step:
        def step(tree, n, bounds, off, queries, lists, init, order=None):
            knn_accumulate(tree, queries, k, lists, id_offset=off, init=init,
                           max_radius=max_radius, layout=lay, world_bounds=bounds, order=order,
                           n=n)
    extract = extract or (lambda L: lists_extract(L, k))
    n_local = torch.tensor([local_points.shape[0]], dtype=torch.int64, device=dev)
    counts = [torch.zeros_like(n_local) for _ in range(P)]
    dist.all_gather(counts, n_local, group=group)
    counts = [int(c.item()) for c in counts]
    begins = [sum(counts[:i]) for i in range(P)]
    cap = max(counts) if counts else 0
    queries = local_points.contiguous()
    order = None
    if morton and library_step and queries.shape[0] > 1:
        order = morton_order(queries)
    lists = new_lists(queries.shape[0], k, dev)
    tree, bounds = build(queries)
    if bounds is None:
        raise ValueError("build() must return the shard's world bounds")
    cur = torch.zeros((cap, D), dtype=local_points.dtype, device=dev)
    cur[:counts[r]] = tree
    cur_b = bounds.clone().to(dev)
    nxt = torch.empty_like(cur)
    nxt_b = torch.empty_like(cur_b)
    nxt_rank, prv_rank = (r + 1) % P, (r - 1) % P
    for rnd in range(P):
        origin = (r - rnd) % P
        reqs = None
        if rnd + 1 < P:
            # post the next round's exchange before searching this shard
            ops = [dist.P2POp(dist.isend, cur, nxt_rank, group),
                   dist.P2POp(dist.irecv, nxt, prv_rank, group),
                   dist.P2POp(dist.isend, cur_b, nxt_rank, group),
                   dist.P2POp(dist.irecv, nxt_b, prv_rank, group)]
            reqs = dist.batch_isend_irecv(ops)
        kwargs = {"order": order} if order is not None else {}
        step(cur[:counts[origin]], counts[origin], cur_b, begins[origin], queries, lists,
             rnd == 0, **kwargs)
        if reqs is not None:
            for q in reqs:
                q.wait()
            cur, nxt = nxt, cur
            cur_b, nxt_b = nxt_b, cur_b
    return (*extract(lists), tree)
