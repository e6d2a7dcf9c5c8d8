"""cudakdtree_b200 -- B200-native k-d trees behind the C ABI of libcukd_b200.so.

Python mirror of the reference's host API (ingowald/cudaKDTree):

=======================  ==================================================
reference (C++ template)  here
=======================  ==================================================
cukd::buildTree           build_tree(points, ...)           (builder.h:108)
buildTree_thrust/...      build_tree(..., builder="thrust") (builder_*.h)
cukd::computeBounds       compute_bounds(points)            (builder_common.h:151)
stackBased/stackFree/cct  fcp(tree, queries, method=...)    (fcp.h:54-163)
  ::fcp
... ::knn                 knn(tree, queries, k, method=...) (knn.h:83-199)
=======================  ==================================================

Device memory is handled with torch CUDA tensors; every call goes through
the compiled library (there is no CPU fallback: importing works without a
GPU, but calling without the built library or a GPU raises).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import torch

__all__ = [
    "lib", "Layout", "layout_for", "build_tree", "compute_bounds", "fcp", "knn",
    "knn_visits", "knn_host", "knn_to_host", "morton_order", "CukdError", "STACK_BASED",
    "STACK_FREE", "CCT", "BatchPlan",
]

HERE = os.path.dirname(os.path.abspath(__file__))
# the in-tree build; CUKD_B200_LIBRARY names another build of the same library
LIB_PATH = os.environ.get("CUKD_B200_LIBRARY") or os.path.join(HERE, "lib", "libcukd_b200.so")

FLOAT32, INT32 = 0, 1
STACK_BASED, STACK_FREE, CCT = 0, 1, 2
METHODS = {"stack_based": STACK_BASED, "stackBased": STACK_BASED, "stack_free": STACK_FREE,
           "stackFree": STACK_FREE, "cct": CCT}
BUILDERS = {"default": 0, "thrust": 1, "bitonic": 2, "inplace": 3, "inPlace": 3}
QUERY_MORTON, QUERY_HEAP_ORDER, QUERY_FORCE_HEAP, QUERY_REFERENCE_ORDER = 1, 2, 4, 8
QUERY_TREE_ORDER = 16
QUERY_WARP_PACKET = 32
INT64_MAX = (1 << 63) - 1
ASYNC_WAIT_POLLS_DEFAULT = 4194304  # CUKD_ASYNC_WAIT_POLLS_DEFAULT


class CukdError(RuntimeError):
    def __init__(self, status, what):
        self.status = status
        msg = _status_string(status)
        if status == 4:
            msg += f" ({lib().cukd_last_cuda_error().decode()})"
        super().__init__(f"{what}: {msg} [status {status}]")


class Layout(C.Structure):
    """cukd_layout: the C-ABI form of the reference's data_traits."""
    _fields_ = [("scalar_type", C.c_int32), ("num_dims", C.c_int32), ("stride", C.c_int32),
                ("point_offset", C.c_int32), ("dim_offset", C.c_int32),
                ("dim_shift", C.c_int32), ("dim_bits", C.c_int32)]

    @property
    def explicit_dim(self):
        return self.dim_offset >= 0

    def __repr__(self):
        return (f"Layout(scalar={self.scalar_type}, D={self.num_dims}, stride={self.stride}, "
                f"poff={self.point_offset}, doff={self.dim_offset}, "
                f"dshift={self.dim_shift}, dbits={self.dim_bits})")


class SpatialTreeC(C.Structure):
    """cukd_spatial_tree."""
    _fields_ = [("nodes", C.c_void_p), ("prim_ids", C.c_void_p), ("data", C.c_void_p),
                ("num_prims", C.c_int32), ("num_nodes", C.c_int32), ("num_dims", C.c_int32),
                ("bounds", C.c_float * 8)]


class QueryParams(C.Structure):
    _fields_ = [("method", C.c_int32), ("k", C.c_int32), ("cutoff_radius", C.c_float),
                ("eps", C.c_float), ("cutoff_d2", C.c_int64), ("flags", C.c_int32),
                ("block_size", C.c_int32), ("d_reordered_count", C.c_void_p)]


class BatchTuning(C.Structure):
    """cukd_batch_tuning."""
    _fields_ = [("build_tile", C.c_int32), ("block_size", C.c_int32),
                ("queries_per_thread", C.c_int32), ("morton", C.c_int32),
                ("build_ms", C.c_float), ("query_ms", C.c_float)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def layout_for(scalar="float32", num_dims=3, stride=None, point_offset=0, dim_offset=-1,
               dim_shift=0, dim_bits=32):
    sc = {"float32": FLOAT32, "float": FLOAT32, "int32": INT32, "int": INT32,
          FLOAT32: FLOAT32, INT32: INT32}[scalar]
    if stride is None:
        stride = 4 * num_dims
    return Layout(sc, num_dims, stride, point_offset, dim_offset, dim_shift, dim_bits)


class MemResource(C.Structure):
    """cukd_mem_resource (the reference's GpuMemoryResource, helpers.h:30-70)."""
    _fields_ = [("ctx", C.c_void_p), ("alloc", C.c_void_p), ("release", C.c_void_p)]


_ALLOC_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_void_p), C.c_size_t, C.c_void_p)
_RELEASE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)


class TorchMemoryResource:
    """A cukd_mem_resource that allocates through torch's caching allocator,
    so library-owned arrays (e.g. spatial-tree nodes) are visible as torch
    tensors."""

    def __init__(self, device=None):
        self.device = torch.device("cuda" if device is None else device)
        self.live = {}
        self._alloc = _ALLOC_FN(self._do_alloc)
        self._release = _RELEASE_FN(self._do_release)
        self.struct = MemResource(None, C.cast(self._alloc, C.c_void_p),
                                  C.cast(self._release, C.c_void_p))

    def _do_alloc(self, ctx, out, nbytes, stream):
        try:
            t = torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=self.device)
        except RuntimeError:
            return 1
        self.live[t.data_ptr()] = t
        out[0] = t.data_ptr()
        return 0

    def _do_release(self, ctx, ptr, stream):
        self.live.pop(ptr, None)
        return 0

    def tensor(self, ptr, dtype, count):
        """The torch tensor viewing `count` elements of an allocation."""
        base = self.live[ptr]
        return base[: count * torch.empty((), dtype=dtype).element_size()].view(dtype)


_lib = None


def lib():
    """The compiled library.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} not built; run `make -C cudakdtree_b200/csrc` "
                "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        P, I64 = C.c_void_p, C.c_int64
        L.cukd_build_tree.argtypes = [P, I64, C.POINTER(Layout), P, C.c_int, P, P]
        L.cukd_compute_bounds.argtypes = [P, I64, C.POINTER(Layout), P, P]
        L.cukd_fcp.argtypes = [P, I64, C.POINTER(Layout), P, P, I64, C.POINTER(QueryParams), P,
                               P, P, P]
        L.cukd_knn.argtypes = [P, I64, C.POINTER(Layout), P, P, I64, C.POINTER(QueryParams), P,
                               P, P, P, P]
        L.cukd_knn_visits.argtypes = [P, I64, C.POINTER(Layout), P, P, I64,
                                      C.POINTER(QueryParams), P, P, P]
        L.cukd_morton_order.argtypes = [P, I64, C.c_int, P, P, P, P]
        L.cukd_query_params_init.argtypes = [C.POINTER(QueryParams)]
        L.cukd_status_string.argtypes = [C.c_int]
        L.cukd_status_string.restype = C.c_char_p
        L.cukd_last_cuda_error.restype = C.c_char_p
        L.cukd_launch_count.restype = C.c_ulonglong
        L.cukd_build_check.argtypes = [P]
        L.cukd_set_async_wait_polls.argtypes = [C.c_uint32]
        L.cukd_async_wait_timeouts.argtypes = [C.POINTER(C.c_uint)]
        L.cukd_spatial_build.argtypes = [P, I64, C.POINTER(Layout), C.c_int,
                                         C.POINTER(SpatialTreeC), P, C.POINTER(MemResource)]
        L.cukd_spatial_free.argtypes = [C.POINTER(SpatialTreeC), P, C.POINTER(MemResource)]
        L.cukd_spatial_fcp.argtypes = [C.POINTER(SpatialTreeC), C.POINTER(Layout), P, I64,
                                       C.POINTER(QueryParams), P, P, P, P]
        L.cukd_spatial_knn.argtypes = [C.POINTER(SpatialTreeC), C.POINTER(Layout), P, I64,
                                       C.POINTER(QueryParams), P, P, P, P]
        L.cukd_radius_model_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_uint64]
        L.cukd_radius_model_create_nd.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int,
                                                  C.c_uint64]
        L.cukd_radius_model_destroy.argtypes = [C.c_void_p]
        L.cukd_radius_model_set_loss.argtypes = [C.c_void_p, C.c_float]
        L.cukd_radius_model_set_grid.argtypes = [C.c_void_p, P, I64, C.POINTER(Layout), P, P]
        L.cukd_radius_model_train.argtypes = [C.c_void_p, P, P, I64, C.c_int, C.c_int,
                                              C.c_float, P, P]
        L.cukd_radius_model_predict.argtypes = [C.c_void_p, P, I64, P, P]
        L.cukd_radius_model_features.argtypes = [C.c_void_p, P, I64, P, P]
        L.cukd_radius_model_gradients.argtypes = [C.c_void_p, P, P, I64, P, P, P, P]
        L.cukd_knn_learned.argtypes = [P, I64, C.POINTER(Layout), P, P, I64,
                                       C.POINTER(QueryParams), C.c_void_p, C.c_float, P, P, P,
                                       P, P, P, P]
        L.cukd_batch_plan_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, I64, P, P,
                                             C.POINTER(QueryParams)]
        L.cukd_batch_plan_destroy.argtypes = [C.c_void_p]
        L.cukd_batch_get_tuning.argtypes = [C.c_void_p, C.POINTER(BatchTuning)]
        L.cukd_batch_set_tuning.argtypes = [C.c_void_p, C.POINTER(BatchTuning)]
        L.cukd_batch_build.argtypes = [C.c_void_p, P, P, P]
        L.cukd_batch_query.argtypes = [C.c_void_p, P, P, P, P, P, P]
        L.cukd_batch_run.argtypes = [C.c_void_p, P, P, P, P, P, P]
        L.cukd_batch_autotune.argtypes = [C.c_void_p, P, P, C.c_int, C.POINTER(BatchTuning), P]
        L.cukd_knn_host.argtypes = [P, I64, C.POINTER(Layout), P, P, I64,
                                    C.POINTER(QueryParams), P, P, I64, P, P]
        L.cukd_knn_to_host.argtypes = [P, I64, C.POINTER(Layout), P, P, I64,
                                       C.POINTER(QueryParams), P, P, I64, P, P]
        L.cukd_knn_host_async.argtypes = [P, I64, C.POINTER(Layout), P, P, I64,
                                          C.POINTER(QueryParams), P, P, I64, P, P, P]
        L.cukd_knn_to_host_async.argtypes = [P, I64, C.POINTER(Layout), P, P, I64,
                                             C.POINTER(QueryParams), P, P, I64, P, P, P]
        L.cukd_knn_accumulate.argtypes = [P, I64, C.POINTER(Layout), P, I64, P, I64, P, C.c_int,
                                          C.c_float, C.c_int, P, P]
        L.cukd_knn_lists_extract.argtypes = [P, I64, C.c_int, P, P, P, P]
        for name in ("cukd_build_float2", "cukd_build_float3", "cukd_build_float4",
                     "cukd_build_int2", "cukd_build_int3", "cukd_build_int4"):
            getattr(L, name).argtypes = [P, I64, P, P, P]
        _lib = L
    return _lib


def _status_string(status):
    try:
        return lib().cukd_status_string(status).decode()
    except Exception:  # pragma: no cover
        return "status"


def _check(status, what):
    if status != 0:
        raise CukdError(status, what)


def _stream(stream):
    if stream is None:
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, torch.cuda.Stream):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(stream)


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def infer_layout(points: torch.Tensor) -> Layout:
    """Layout of a plain [n, D] float32/int32 tensor (default_data_traits)."""
    if points.dim() != 2:
        raise ValueError("points must be [n, D] for an inferred layout")
    sc = {torch.float32: FLOAT32, torch.int32: INT32}[points.dtype]
    return layout_for(sc, points.shape[1])


def _num_records(points, layout):
    return points.numel() * points.element_size() // layout.stride


def _bounds_dtype(layout):
    return torch.float32 if layout.scalar_type == FLOAT32 else torch.int32


def compute_bounds(points, layout=None, stream=None):
    layout = layout or infer_layout(points)
    n = _num_records(points, layout)
    wb = torch.empty((2, layout.num_dims), dtype=_bounds_dtype(layout), device=points.device)
    _check(lib().cukd_compute_bounds(_ptr(points), n, C.byref(layout), _ptr(wb),
                                     _stream(stream)), "cukd_compute_bounds")
    return wb


def build_tree(points, layout=None, world_bounds=None, builder="default", stream=None,
               n=None, want_bounds=True):
    """Builds a left-balanced k-d tree IN PLACE over `points` (a contiguous
    CUDA tensor holding n records of `layout`).  Returns the world bounds
    tensor [2, D] (or None when want_bounds is False and the layout has no
    explicit dims)."""
    layout = layout or infer_layout(points)
    if not points.is_cuda or not points.is_contiguous():
        raise ValueError("points must be a contiguous CUDA tensor")
    if n is None:
        n = _num_records(points, layout)
    if world_bounds is None and (want_bounds or layout.explicit_dim):
        world_bounds = torch.empty((2, layout.num_dims), dtype=_bounds_dtype(layout),
                                   device=points.device)
    b = BUILDERS[builder] if isinstance(builder, str) else int(builder)
    _check(lib().cukd_build_tree(_ptr(points), n, C.byref(layout), _ptr(world_bounds), b,
                                 _stream(stream), None), "cukd_build_tree")
    return world_bounds


def _params(method, k=1, cutoff=math.inf, eps=0.0, cutoff_d2=INT64_MAX, morton=True,
            heap_order=False, force_heap=False, block_size=0, reference_order=False,
            tree_order=False, warp_packet=False):
    p = QueryParams()
    p.method = METHODS[method] if isinstance(method, str) else int(method)
    p.k = k
    p.cutoff_radius = cutoff
    p.eps = eps
    p.cutoff_d2 = cutoff_d2
    p.flags = ((QUERY_MORTON if morton else 0) | (QUERY_HEAP_ORDER if heap_order else 0)
               | (QUERY_FORCE_HEAP if force_heap else 0)
               | (QUERY_REFERENCE_ORDER if reference_order else 0)
               | (QUERY_TREE_ORDER if tree_order else 0)
               | (QUERY_WARP_PACKET if warp_packet else 0))
    p.block_size = block_size
    return p


def fcp(tree, queries, method="stack_based", layout=None, world_bounds=None, n=None,
        cutoff=math.inf, eps=0.0, cutoff_d2=INT64_MAX, morton=True, with_d2=False,
        stream=None, block_size=0, reference_order=False, tree_order=False):
    """Find-closest-point for each query ([nq, D] tensor of the tree's scalar
    type).  Returns int32 node indices (-1 = none within the cut-off)."""
    layout = layout or infer_layout(tree)
    if n is None:
        n = _num_records(tree, layout)
    nq = queries.shape[0]
    ids = torch.empty(nq, dtype=torch.int32, device=queries.device)
    d2 = None
    if with_d2:
        d2 = torch.empty(nq, dtype=torch.float32 if layout.scalar_type == FLOAT32
                         else torch.int64, device=queries.device)
    p = _params(method, 1, cutoff, eps, cutoff_d2, morton, block_size=block_size,
                reference_order=reference_order, tree_order=tree_order)
    _check(lib().cukd_fcp(_ptr(tree), n, C.byref(layout), _ptr(world_bounds),
                          _ptr(queries.contiguous()), nq, C.byref(p), _ptr(ids), _ptr(d2),
                          _stream(stream), None), "cukd_fcp")
    return (ids, d2) if with_d2 else ids


def knn(tree, queries, k, method="stack_based", layout=None, world_bounds=None, n=None,
        cutoff=math.inf, cutoff_d2=INT64_MAX, morton=True, heap_order=False,
        force_heap=False, with_max=False, stream=None, block_size=0, out_ids=None,
        out_d2=None, reference_order=False, reordered_count=None, tree_order=False,
        warp_packet=False):
    """k nearest neighbours.  Returns (ids [nq,k] int32, d2 [nq,k]) with the
    reference's candidate-list semantics; ascending unless heap_order.
    warp_packet: the warp-cooperative traversal (float, k <= 32)."""
    layout = layout or infer_layout(tree)
    if n is None:
        n = _num_records(tree, layout)
    nq = queries.shape[0]
    dev = queries.device
    dt = torch.float32 if layout.scalar_type == FLOAT32 else torch.int64
    ids = out_ids if out_ids is not None else torch.empty((nq, k), dtype=torch.int32, device=dev)
    d2 = out_d2 if out_d2 is not None else torch.empty((nq, k), dtype=dt, device=dev)
    mx = torch.empty(nq, dtype=dt, device=dev) if with_max else None
    p = _params(method, k, cutoff, 0.0, cutoff_d2, morton, heap_order, force_heap, block_size,
                reference_order, tree_order, warp_packet)
    if reordered_count is not None:  # int32 CUDA tensor of one element
        p.d_reordered_count = reordered_count.data_ptr()
    _check(lib().cukd_knn(_ptr(tree), n, C.byref(layout), _ptr(world_bounds),
                          _ptr(queries.contiguous()), nq, C.byref(p), _ptr(ids), _ptr(d2),
                          _ptr(mx), _stream(stream), None), "cukd_knn")
    return (ids, d2, mx) if with_max else (ids, d2)


def _init_event(ev, stream):
    """torch creates a CUDA event at its first record: record it once."""
    if not ev.cuda_event:
        ev.record(stream if isinstance(stream, torch.cuda.Stream) else torch.cuda.current_stream())


def knn_host(tree, queries, k, method="stack_based", layout=None, world_bounds=None, n=None,
             cutoff=math.inf, cutoff_d2=INT64_MAX, morton=True, out_ids=None, out_d2=None,
             chunk=0, stream=None, done=None):
    """knn() with host-resident queries and results (CPU tensors; pin them
    for the copies to overlap the search).  Returns (ids, d2) CPU tensors,
    complete once ``stream`` (default: the current stream) is synchronised --
    or, with ``done`` (a torch.cuda.Event), once that event has completed,
    the stream being free as soon as the searches are queued
    (cukd_knn_host_async)."""
    layout = layout or infer_layout(tree)
    if n is None:
        n = _num_records(tree, layout)
    if queries.is_cuda:
        raise ValueError("queries must be host memory (use knn() for device queries)")
    nq = queries.shape[0]
    queries = queries.contiguous()
    dt = torch.float32 if layout.scalar_type == FLOAT32 else torch.int64
    pin = queries.is_pinned()
    ids = out_ids if out_ids is not None else torch.empty((nq, k), dtype=torch.int32,
                                                          pin_memory=pin)
    d2 = out_d2 if out_d2 is not None else torch.empty((nq, k), dtype=dt, pin_memory=pin)
    p = _params(method, k, cutoff, 0.0, cutoff_d2, morton)
    if done is not None:
        _init_event(done, stream)
        _check(lib().cukd_knn_host_async(_ptr(tree), n, C.byref(layout), _ptr(world_bounds),
                                         _ptr(queries), nq, C.byref(p), _ptr(ids), _ptr(d2),
                                         int(chunk), C.c_void_p(done.cuda_event),
                                         _stream(stream), None), "cukd_knn_host_async")
        return ids, d2
    _check(lib().cukd_knn_host(_ptr(tree), n, C.byref(layout), _ptr(world_bounds), _ptr(queries),
                               nq, C.byref(p), _ptr(ids), _ptr(d2), int(chunk), _stream(stream),
                               None), "cukd_knn_host")
    return ids, d2


def knn_to_host(tree, queries, k, method="stack_based", layout=None, world_bounds=None, n=None,
                cutoff=math.inf, cutoff_d2=INT64_MAX, morton=True, out_ids=None, out_d2=None,
                chunk=0, stream=None, done=None):
    """knn() of device-resident queries with the answers written to host
    memory (pinned CPU tensors by default), searches of query slices
    overlapping the copies of earlier answers.  Returns (ids, d2) CPU
    tensors, complete once ``stream`` (default: the current stream) is
    synchronised -- or, with ``done`` (a torch.cuda.Event), once that event
    has completed, the stream being free as soon as the searches are queued
    (cukd_knn_to_host_async)."""
    layout = layout or infer_layout(tree)
    if n is None:
        n = _num_records(tree, layout)
    if not queries.is_cuda:
        raise ValueError("queries must be device memory (use knn_host() for host queries)")
    nq = queries.shape[0]
    queries = queries.contiguous()
    dt = torch.float32 if layout.scalar_type == FLOAT32 else torch.int64
    ids = out_ids if out_ids is not None else torch.empty((nq, k), dtype=torch.int32,
                                                          pin_memory=True)
    d2 = out_d2 if out_d2 is not None else torch.empty((nq, k), dtype=dt, pin_memory=True)
    if ids.is_cuda or d2.is_cuda:
        raise ValueError("out_ids / out_d2 must be host memory")
    p = _params(method, k, cutoff, 0.0, cutoff_d2, morton)
    if done is not None:
        _init_event(done, stream)
        _check(lib().cukd_knn_to_host_async(_ptr(tree), n, C.byref(layout),
                                            _ptr(world_bounds), _ptr(queries), nq, C.byref(p),
                                            _ptr(ids), _ptr(d2), int(chunk),
                                            C.c_void_p(done.cuda_event), _stream(stream),
                                            None), "cukd_knn_to_host_async")
        return ids, d2
    _check(lib().cukd_knn_to_host(_ptr(tree), n, C.byref(layout), _ptr(world_bounds),
                                  _ptr(queries), nq, C.byref(p), _ptr(ids), _ptr(d2), int(chunk),
                                  _stream(stream), None), "cukd_knn_to_host")
    return ids, d2


def knn_visits(tree, queries, k, method="stack_based", layout=None, world_bounds=None, n=None,
               cutoff=math.inf, morton=True, stream=None):
    """Per-query visited-node counts (k=0: FCP traversal)."""
    layout = layout or infer_layout(tree)
    if n is None:
        n = _num_records(tree, layout)
    nq = queries.shape[0]
    v = torch.empty(nq, dtype=torch.int64, device=queries.device)
    p = _params(method, k, cutoff, 0.0, INT64_MAX, morton)
    _check(lib().cukd_knn_visits(_ptr(tree), n, C.byref(layout), _ptr(world_bounds),
                                 _ptr(queries.contiguous()), nq, C.byref(p), _ptr(v),
                                 _stream(stream), None), "cukd_knn_visits")
    return v


def build_check(stream=None):
    """Waits for the stream and raises CukdError(CUKD_ERR_TIMEOUT) if a
    build's bounded device-side wait gave up since the last check (that
    build left its records unchanged) -- cukd_build_check."""
    _check(lib().cukd_build_check(_stream(stream)), "cukd_build_check")


def set_async_wait_polls(polls=None):
    """Test hook: polls of the builder's first bulk-copy wait (None = the
    default; 0 gives up at once) -- cukd_set_async_wait_polls."""
    _check(lib().cukd_set_async_wait_polls(ASYNC_WAIT_POLLS_DEFAULT if polls is None
                                           else int(polls)), "cukd_set_async_wait_polls")


def async_wait_timeouts():
    """Bulk-copy waits that gave up on this device so far (synchronises)."""
    c = C.c_uint()
    _check(lib().cukd_async_wait_timeouts(C.byref(c)), "cukd_async_wait_timeouts")
    return c.value


def launch_count():
    """Kernels launched by the library so far in this process."""
    return int(lib().cukd_launch_count())


def morton_order(points, bounds=None, stream=None):
    n, D = points.shape
    perm = torch.empty(n, dtype=torch.int32, device=points.device)
    _check(lib().cukd_morton_order(_ptr(points.contiguous()), n, D, _ptr(bounds), _ptr(perm),
                                   _stream(stream), None), "cukd_morton_order")
    return perm


# ---------------------------------------------------------------------------
# spatial k-d tree (reference: cukd/spatial-kdtree.h)
# ---------------------------------------------------------------------------
SPATIAL_NODE_BYTES = 12


class SpatialKDTree:
    """A spatial k-d tree whose node and prim-id arrays live in torch memory.
    `nodes` is a [num_nodes, 3] int32 view of the 12-byte node records
    ({float pos; u32 offset; u16 count; i16 dim}); `prim_ids` is int32."""

    def __init__(self, points, layout, leaf_threshold=0, stream=None):
        self.layout = layout
        self.points = points
        self.mr = TorchMemoryResource(points.device)
        self.c = SpatialTreeC()
        n = _num_records(points, layout)
        _check(lib().cukd_spatial_build(_ptr(points), n, C.byref(layout), leaf_threshold,
                                        C.byref(self.c), _stream(stream),
                                        C.byref(self.mr.struct)), "cukd_spatial_build")

    @property
    def num_nodes(self):
        return self.c.num_nodes

    @property
    def bounds(self):
        D = self.c.num_dims
        return [list(self.c.bounds[:D]), list(self.c.bounds[4:4 + D])]

    def nodes(self):
        return self.mr.tensor(self.c.nodes, torch.int32, 3 * self.c.num_nodes).view(-1, 3)

    def prim_ids(self):
        return self.mr.tensor(self.c.prim_ids, torch.int32, self.c.num_prims)

    def free(self, stream=None):
        if self.c.nodes:
            _check(lib().cukd_spatial_free(C.byref(self.c), _stream(stream),
                                           C.byref(self.mr.struct)), "cukd_spatial_free")

    def _query(self, fn, queries, p, k, with_d2, stream):
        nq = queries.shape[0]
        shape = (nq,) if k is None else (nq, k)
        ids = torch.empty(shape, dtype=torch.int32, device=queries.device)
        d2 = torch.empty(shape, dtype=torch.float32, device=queries.device) if with_d2 else None
        _check(fn(C.byref(self.c), C.byref(self.layout), _ptr(queries.contiguous()), nq,
                  C.byref(p), _ptr(ids), _ptr(d2), _stream(stream), None), fn.__name__)
        return (ids, d2) if with_d2 else ids

    def fcp(self, queries, method="cct", cutoff=math.inf, morton=True, stream=None):
        p = _params(method, 1, cutoff, 0.0, INT64_MAX, morton)
        return self._query(lib().cukd_spatial_fcp, queries, p, None, False, stream)

    def knn(self, queries, k, method="cct", cutoff=math.inf, morton=True, heap_order=False,
            stream=None):
        p = _params(method, k, cutoff, 0.0, INT64_MAX, morton, heap_order)
        return self._query(lib().cukd_spatial_knn, queries, p, k, True, stream)


def spatial_build(points, layout=None, leaf_threshold=0, stream=None):
    """Spatial k-d tree over `points` (not reordered)."""
    return SpatialKDTree(points, layout or infer_layout(points), leaf_threshold, stream)


# ---------------------------------------------------------------------------
# learned kNN-radius proposal
# ---------------------------------------------------------------------------
class RadiusModel:
    """MLP radius proposal (cukd_radius_model_*): xyz + log occupancy-grid
    density -> 64 -> 64 -> 1, BF16 weights, trained on the GPU by the
    library's own kernels on exact k-th distances."""

    NUM_PARAMS = 4801
    NUM_INPUTS = 8

    def __init__(self, grid_res=64, seed=0, quantile=0.0, num_dims=3):
        """num_dims: dimension of the tree's points (2..4).  quantile: 0
        trains with mean squared error (the network predicts the conditional
        mean of the log k-th distance); 0 < q < 1 with the pinball loss (it
        predicts that quantile)."""
        self.h = C.c_void_p()
        _check(lib().cukd_radius_model_create_nd(C.byref(self.h), grid_res, num_dims, seed),
               "cukd_radius_model_create_nd")
        _check(lib().cukd_radius_model_set_loss(self.h, float(quantile)),
               "cukd_radius_model_set_loss")
        self.final_loss = None

    def __del__(self):
        try:
            if self.h:
                lib().cukd_radius_model_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    def set_grid(self, tree, layout, world_bounds, n=None, stream=None):
        n = _num_records(tree, layout) if n is None else n
        vals = [float(v) for v in world_bounds.detach().cpu().reshape(-1)]
        wb = (C.c_float * len(vals))(*vals)
        _check(lib().cukd_radius_model_set_grid(self.h, _ptr(tree), n, C.byref(layout),
                                                C.cast(wb, C.c_void_p), _stream(stream)),
               "cukd_radius_model_set_grid")

    def train(self, queries, kth_d2, epochs=10, batch=4096, lr=2e-3, stream=None):
        loss = C.c_float()
        _check(lib().cukd_radius_model_train(self.h, _ptr(queries.contiguous()),
                                             _ptr(kth_d2.contiguous()), queries.shape[0],
                                             epochs, batch, lr, C.byref(loss), _stream(stream)),
               "cukd_radius_model_train")
        self.final_loss = loss.value
        return loss.value

    def fit(self, tree, train_queries, k, layout=None, world_bounds=None, epochs=10,
            batch=4096, lr=2e-3, stream=None):
        # train_queries should follow the distribution the model will serve
        """Occupancy grid from the tree, exact k-th distances of the training
        queries from the plain traversal, then training."""
        layout = layout or infer_layout(tree)
        if world_bounds is None:
            world_bounds = compute_bounds(tree, layout)
        self.set_grid(tree, layout, world_bounds, stream=stream)
        _, _, kth = knn(tree, train_queries, k, "cct", layout=layout, world_bounds=world_bounds,
                        with_max=True, stream=stream)
        return self.train(train_queries, kth, epochs, batch, lr, stream)

    def predict(self, queries, stream=None):
        r = torch.empty(queries.shape[0], dtype=torch.float32, device=queries.device)
        _check(lib().cukd_radius_model_predict(self.h, _ptr(queries.contiguous()),
                                               queries.shape[0], _ptr(r), _stream(stream)),
               "cukd_radius_model_predict")
        return r

    def features(self, queries, stream=None):
        f = torch.empty((queries.shape[0], self.NUM_INPUTS), dtype=torch.float32,
                        device=queries.device)
        _check(lib().cukd_radius_model_features(self.h, _ptr(queries.contiguous()),
                                                queries.shape[0], _ptr(f), _stream(stream)),
               "cukd_radius_model_features")
        return f

    def gradients(self, features, targets, stream=None):
        import numpy as np
        g = np.zeros(self.NUM_PARAMS, np.float32)
        p = np.zeros(self.NUM_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        _check(lib().cukd_radius_model_gradients(
            self.h, _ptr(features.contiguous()), _ptr(targets.contiguous()), features.shape[0],
            g.ctypes.data_as(C.c_void_p), p.ctypes.data_as(C.c_void_p),
            loss.ctypes.data_as(C.c_void_p), _stream(stream)), "cukd_radius_model_gradients")
        return g, p, float(loss[0])


def knn_learned(tree, queries, k, model, method="stack_based", layout=None, world_bounds=None,
                n=None, scale=1.2, morton=True, visits=False, status=False, stream=None,
                out_ids=None, out_d2=None, warp_packet=False):
    """kNN seeded by the learned radius: same results as knn().  Returns
    (ids, d2, fallback[2] int32 tensor, visits or None[, status]).
    warp_packet: seed the warp-cooperative traversal instead."""
    layout = layout or infer_layout(tree)
    n = _num_records(tree, layout) if n is None else n
    nq = queries.shape[0]
    dev = queries.device
    ids = out_ids if out_ids is not None else torch.empty((nq, k), dtype=torch.int32, device=dev)
    dt = torch.float32 if layout.scalar_type == FLOAT32 else torch.int64
    d2 = out_d2 if out_d2 is not None else torch.empty((nq, k), dtype=dt, device=dev)
    fb = torch.zeros(2, dtype=torch.int32, device=dev)
    v = torch.zeros(nq, dtype=torch.int64, device=dev) if visits else None
    st = torch.zeros(nq, dtype=torch.int32, device=dev) if status else None
    p = _params(method, k, math.inf, 0.0, INT64_MAX, morton, warp_packet=warp_packet)
    _check(lib().cukd_knn_learned(_ptr(tree), n, C.byref(layout), _ptr(world_bounds),
                                  _ptr(queries.contiguous()), nq, C.byref(p), model.h, scale,
                                  _ptr(ids), _ptr(d2), _ptr(fb), _ptr(st), _ptr(v),
                                  _stream(stream), None),
           "cukd_knn_learned")
    return (ids, d2, fb, v, st) if status else (ids, d2, fb, v)


# ---------------------------------------------------------------------------
# batched clouds (no reference counterpart)
# ---------------------------------------------------------------------------
class BatchPlan:
    """Many independent float clouds (CSR offsets over one [total, D] array)
    built into their own left-balanced trees in place and queried with
    their own query sets (cukd_batch_*).  Results equal a per-cloud loop of
    build_tree + knn / fcp, ids local to each cloud.  k = 0 means FCP."""

    def __init__(self, point_offsets, query_offsets, num_dims=3, k=8, method="stack_based",
                 cutoff=math.inf, eps=0.0, heap_order=False, force_heap=False,
                 reference_order=False):
        import numpy as np
        po = np.ascontiguousarray(np.asarray(point_offsets, dtype=np.int64))
        qo = np.ascontiguousarray(np.asarray(query_offsets, dtype=np.int64))
        if po.ndim != 1 or qo.shape != po.shape or po.size < 1:
            raise ValueError("point_offsets and query_offsets: int64[B + 1]")
        self.num_clouds = po.size - 1
        self.point_offsets, self.query_offsets = po, qo
        self.num_dims, self.k = num_dims, k
        self.total, self.nq = int(po[-1]), int(qo[-1])
        m = METHODS[method] if isinstance(method, str) else int(method)
        p = _params(m, k, cutoff, eps, INT64_MAX, True, heap_order=heap_order,
                    force_heap=force_heap, reference_order=reference_order)
        self.h = C.c_void_p()
        _check(lib().cukd_batch_plan_create(C.byref(self.h), num_dims, self.num_clouds,
                                            po.ctypes.data_as(C.c_void_p),
                                            qo.ctypes.data_as(C.c_void_p), C.byref(p)),
               "cukd_batch_plan_create")

    def __del__(self):
        try:
            if self.h:
                lib().cukd_batch_plan_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    def close(self):
        self.__del__()

    @property
    def tuning(self):
        t = BatchTuning()
        _check(lib().cukd_batch_get_tuning(self.h, C.byref(t)), "cukd_batch_get_tuning")
        return t

    def set_tuning(self, build_tile=None, block_size=None, queries_per_thread=None, morton=None):
        t = self.tuning
        for name, v in (("build_tile", build_tile), ("block_size", block_size),
                        ("queries_per_thread", queries_per_thread), ("morton", morton)):
            if v is not None:
                setattr(t, name, int(v))
        _check(lib().cukd_batch_set_tuning(self.h, C.byref(t)), "cukd_batch_set_tuning")

    def _outputs(self, dev):
        kk = max(self.k, 1)
        shape = (self.nq, kk) if self.k > 0 else (self.nq,)
        return (torch.empty(shape, dtype=torch.int32, device=dev),
                torch.empty(shape, dtype=torch.float32, device=dev))

    def bounds_tensor(self, dev):
        return torch.empty((self.num_clouds, 2, self.num_dims), dtype=torch.float32, device=dev)

    def build(self, points, bounds=None, stream=None):
        """Builds every cloud of `points` (float32 [total, D], in place)."""
        _check(lib().cukd_batch_build(self.h, _ptr(points), _ptr(bounds), _stream(stream)),
               "cukd_batch_build")
        return points

    def query(self, points, queries, bounds=None, out=None, stream=None):
        ids, d2 = out if out is not None else self._outputs(queries.device)
        _check(lib().cukd_batch_query(self.h, _ptr(points), _ptr(bounds),
                                      _ptr(queries.contiguous()), _ptr(ids), _ptr(d2),
                                      _stream(stream)), "cukd_batch_query")
        return ids, d2

    def run(self, points, queries, bounds=None, out=None, stream=None):
        """Build + query as one replayed CUDA graph."""
        ids, d2 = out if out is not None else self._outputs(queries.device)
        _check(lib().cukd_batch_run(self.h, _ptr(points), _ptr(bounds),
                                    _ptr(queries.contiguous()), _ptr(ids), _ptr(d2),
                                    _stream(stream)), "cukd_batch_run")
        return ids, d2

    def autotune(self, points, queries, reps=3, stream=None):
        t = BatchTuning()
        _check(lib().cukd_batch_autotune(self.h, _ptr(points), _ptr(queries.contiguous()), reps,
                                         C.byref(t), _stream(stream)), "cukd_batch_autotune")
        return t
