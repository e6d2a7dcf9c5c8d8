"""ctypes bindings for the CPU oracles (test infrastructure only).

Two oracles live under ``oracle/``:

* ``liboracle.so`` -- this project's C restatement of the reference
  algorithms (``cukd_oracle.c``; every routine cites the reference
  file:line it follows).
* ``_ref/libcukd_ref_host.so`` -- the UNMODIFIED reference library compiled
  from its own headers (``ref_host.cu``): ``cukd::buildTree_host`` and the
  reference's host-callable traversals in OpenMP loops.  It pins the
  restatement and serves as the timed CPU baseline.
* ``_ref/libcukd_ref_gpu.so`` -- the reference's GPU builders and query
  functions compiled with ``-fmad=false`` (``ref_gpu.cu``), used by GPU
  parity tests only.

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

STACK_BASED, STACK_FREE, CCT = 0, 1, 2
FIXED_LIST, HEAP_LIST = 0, 1

# reference-oracle type codes (oracle/ref_types.h)
REF_F2, REF_F3, REF_F4 = 0, 1, 2
REF_F2_DIM, REF_F3_DIM, REF_F4_DIM = 3, 4, 5
REF_F3_PAYLOAD, REF_F3_PACKED = 6, 7

_P = C.c_void_p
_I64 = C.c_int64


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


_lib = None
_ref_host = None
_ref_gpu = None


def lib():
    """The C restatement (builds it on first use if missing)."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
        L = C.CDLL(path)
        L.cko_build.argtypes = [C.c_int, C.c_int, _P, _I64, C.c_int, _P, _P, _P]
        L.cko_check_tree.argtypes = [C.c_int, C.c_int, _P, _P, _P, _I64, _P, C.c_int]
        L.cko_check_tree.restype = _I64
        L.cko_check_kd.argtypes = [C.c_int, C.c_int, _P, _P, _I64, _P, C.c_int]
        L.cko_check_kd.restype = _I64
        L.cko_subtree_size.argtypes = [_I64, _I64]
        L.cko_subtree_size.restype = _I64
        L.cko_fcp.argtypes = [C.c_int, C.c_int, C.c_int, _P, _P, _I64, _P, _P, _I64, C.c_float,
                              C.c_float, _I64, _P, _P, C.c_int]
        L.cko_knn.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _I64, _P, _P,
                              _I64, C.c_float, _I64, _P, _P, _P, _P, C.c_int]
        L.cko_spatial_build.argtypes = [C.c_int, _P, _I64, C.c_int, _P, _P, _P, _P]
        L.cko_spatial_fcp.argtypes = [C.c_int, C.c_int, _P, _P, _P, _P, _P, _I64, C.c_float, _P,
                                      C.c_int]
        L.cko_spatial_knn.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P,
                                      _I64, C.c_float, _P, _P, C.c_int]
        _lib = L
    return _lib


def ref_host():
    """The reference's own host code, or None when it was not built."""
    global _ref_host
    if _ref_host is None:
        path = os.path.join(HERE, "_ref", "libcukd_ref_host.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.refh_build.argtypes = [C.c_int, _P, C.c_int, _P]
        L.refh_fcp.argtypes = [C.c_int, C.c_int, _P, C.c_int, _P, _P, C.c_long, C.c_float,
                               C.c_float, _P, C.c_int]
        L.refh_knn.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _P, C.c_int, _P, _P,
                               C.c_long, C.c_float, _P, _P, _P, C.c_int]
        L.refh_spatial_fcp.argtypes = [C.c_int, C.c_int, _P, _P, _P, C.c_int, C.c_int, _P, _P,
                                       C.c_long, C.c_float, _P, C.c_int]
        L.refh_spatial_knn.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P, C.c_int,
                                       C.c_int, _P, _P, C.c_long, C.c_float, _P, _P, C.c_int]
        _ref_host = L
    return _ref_host


def ref_gpu():
    """The reference's own GPU code (needs a GPU to call), or None."""
    global _ref_gpu
    if _ref_gpu is None:
        path = os.path.join(HERE, "_ref", "libcukd_ref_gpu.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.refg_build.argtypes = [C.c_int, C.c_int, _P, C.c_int, _P]
        L.refg_fcp.argtypes = [C.c_int, C.c_int, _P, C.c_int, _P, _P, C.c_int, C.c_float,
                               C.c_float, _P]
        L.refg_knn.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _P, C.c_int, _P, _P, C.c_int,
                               C.c_float, _P, _P]
        L.refg_spatial_build_float3.argtypes = [_P, C.c_int, C.c_int, _P, _P, _P, _P]
        L.refg_spatial_build_ms_float3.argtypes = [_P, C.c_int, C.c_int, _P]
        _ref_gpu = L
    return _ref_gpu


def nthreads():
    return os.cpu_count() or 1


# ----------------------------------------------------------------------------
# restatement wrappers (numpy in, numpy out)
# ----------------------------------------------------------------------------

def _scalar(a):
    if a.dtype == np.float32:
        return 0
    if a.dtype == np.int32:
        return 1
    raise TypeError(a.dtype)


def build(coords, explicit_dim=False):
    """Left-balanced build.  coords: [n, D] float32/int32.
    Returns (perm, dims, bounds): perm[node] = input index at `node`."""
    coords = np.ascontiguousarray(coords)
    n, D = coords.shape
    perm = np.zeros(n, np.int64)
    dims = np.zeros(n, np.int32)
    bounds = np.zeros((2, D), coords.dtype)
    rc = lib().cko_build(_scalar(coords), D, _ptr(coords), n, int(explicit_dim), _ptr(perm),
                         _ptr(dims), _ptr(bounds))
    if rc:
        raise RuntimeError(f"cko_build failed: {rc}")
    return perm, dims, bounds


def check_tree(tree, index, dims=None, bounds=None, threads=None):
    """Violations of the canonical-tree property (0 = the tree build()
    returns for these points): tree [n, D] coordinates in node order,
    index[node] = input index of the point there, dims per node for
    explicit-dim trees (with the world bounds they were built in)."""
    tree = np.ascontiguousarray(tree)
    n, D = tree.shape
    index = np.ascontiguousarray(index, np.int64)
    d = None if dims is None else np.ascontiguousarray(dims, np.int32)
    b = None if bounds is None else np.ascontiguousarray(bounds, dtype=tree.dtype)
    r = lib().cko_check_tree(_scalar(tree), D, _ptr(tree), _ptr(index), _ptr(d), n, _ptr(b),
                             threads or nthreads())
    if r < 0:
        raise ValueError("cko_check_tree: bad arguments")
    return int(r)


def check_kd(tree, dims=None, bounds=None, threads=None):
    """Violations of the k-d property alone (0 = a valid left-balanced k-d
    tree; points equal to a split coordinate may sit on either side):
    tree [n, D] coordinates in node order, dims per node for explicit-dim
    trees (with the world bounds they were built in)."""
    tree = np.ascontiguousarray(tree)
    n, D = tree.shape
    d = None if dims is None else np.ascontiguousarray(dims, np.int32)
    b = None if bounds is None else np.ascontiguousarray(bounds, dtype=tree.dtype)
    r = lib().cko_check_kd(_scalar(tree), D, _ptr(tree), _ptr(d), n, _ptr(b), threads or nthreads())
    if r < 0:
        raise ValueError("cko_check_kd: bad arguments")
    return int(r)


def subtree_size(node, n):
    return lib().cko_subtree_size(node, n)


def fcp(tree, queries, method, dims=None, bounds=None, cutoff=np.inf, eps=0.0,
        cutoff_d2_int=np.iinfo(np.int64).max, visits=False, threads=None):
    tree = np.ascontiguousarray(tree)
    queries = np.ascontiguousarray(queries, dtype=tree.dtype)
    n, D = tree.shape
    nq = queries.shape[0]
    if bounds is None:
        bounds = np.stack([tree.min(0), tree.max(0)]) if n else np.zeros((2, D), tree.dtype)
    bounds = np.ascontiguousarray(bounds, dtype=tree.dtype)
    out = np.zeros(nq, np.int32)
    vis = np.zeros(nq, np.int64) if visits else None
    d = None if dims is None else np.ascontiguousarray(dims, np.int32)
    lib().cko_fcp(_scalar(tree), D, method, _ptr(tree), _ptr(d), n, _ptr(bounds), _ptr(queries),
                  nq, float(cutoff), float(eps), int(cutoff_d2_int), _ptr(out), _ptr(vis),
                  threads or nthreads())
    return (out, vis) if visits else out


def knn(tree, queries, k, method, dims=None, bounds=None, cutoff=np.inf, list_kind=FIXED_LIST,
        cutoff_d2_int=np.iinfo(np.int64).max, visits=False, threads=None):
    tree = np.ascontiguousarray(tree)
    queries = np.ascontiguousarray(queries, dtype=tree.dtype)
    n, D = tree.shape
    nq = queries.shape[0]
    if bounds is None:
        bounds = np.stack([tree.min(0), tree.max(0)]) if n else np.zeros((2, D), tree.dtype)
    bounds = np.ascontiguousarray(bounds, dtype=tree.dtype)
    ids = np.zeros((nq, k), np.int32)
    isint = tree.dtype == np.int32
    d2 = np.zeros((nq, k), np.int64 if isint else np.float32)
    ret = np.zeros(nq, np.int64 if isint else np.float32)
    vis = np.zeros(nq, np.int64) if visits else None
    d = None if dims is None else np.ascontiguousarray(dims, np.int32)
    rc = lib().cko_knn(_scalar(tree), D, method, list_kind, k, _ptr(tree), _ptr(d), n,
                       _ptr(bounds), _ptr(queries), nq, float(cutoff), int(cutoff_d2_int),
                       _ptr(ids), _ptr(d2), _ptr(ret), _ptr(vis), threads or nthreads())
    if rc:
        raise RuntimeError(f"cko_knn failed: {rc}")
    if visits:
        return ids, d2, ret, vis
    return ids, d2, ret


SPATIAL_NODE = np.dtype([("pos", np.float32), ("offset", np.uint32), ("count", np.uint16),
                         ("dim", np.int16)])


def spatial_build(coords, leaf_threshold=8):
    coords = np.ascontiguousarray(coords, np.float32)
    n, D = coords.shape
    nodes = np.zeros(2 * n + 2, SPATIAL_NODE)
    nn = np.zeros(1, np.int64)
    prims = np.zeros(max(n, 1), np.uint32)
    bounds = np.zeros((2, D), np.float32)
    lib().cko_spatial_build(D, _ptr(coords), n, leaf_threshold, _ptr(nodes), _ptr(nn),
                            _ptr(prims), _ptr(bounds))
    return nodes[: int(nn[0])].copy(), prims[:n].copy(), bounds


def spatial_fcp(nodes, prims, coords, bounds, queries, method, cutoff=np.inf, threads=None):
    coords = np.ascontiguousarray(coords, np.float32)
    queries = np.ascontiguousarray(queries, np.float32)
    D = coords.shape[1]
    out = np.zeros(len(queries), np.int32)
    lib().cko_spatial_fcp(D, method, _ptr(nodes), _ptr(prims), _ptr(coords),
                          _ptr(np.ascontiguousarray(bounds, np.float32)), _ptr(queries),
                          len(queries), float(cutoff), _ptr(out), threads or nthreads())
    return out


def spatial_knn(nodes, prims, coords, bounds, queries, k, method, cutoff=np.inf,
                list_kind=FIXED_LIST, threads=None):
    coords = np.ascontiguousarray(coords, np.float32)
    queries = np.ascontiguousarray(queries, np.float32)
    D = coords.shape[1]
    ids = np.zeros((len(queries), k), np.int32)
    d2 = np.zeros((len(queries), k), np.float32)
    lib().cko_spatial_knn(D, method, list_kind, k, _ptr(nodes), _ptr(prims), _ptr(coords),
                          _ptr(np.ascontiguousarray(bounds, np.float32)), _ptr(queries),
                          len(queries), float(cutoff), _ptr(ids), _ptr(d2),
                          threads or nthreads())
    return ids, d2


# ----------------------------------------------------------------------------
# reference wrappers (host)
# ----------------------------------------------------------------------------

def ref_record_dtype(type_code, D=3):
    """numpy dtype with the byte layout of the reference oracle's data_t."""
    if type_code in (REF_F2, REF_F3, REF_F4):
        return np.dtype((np.float32, (type_code + 2,)))
    if type_code in (REF_F2_DIM, REF_F3_DIM, REF_F4_DIM):
        # C++ layout: float2 is 8-byte and float4 16-byte aligned, so
        # {float2,int} is 16 bytes and {float4,int} is 32 bytes.
        D = type_code - 1
        size = {2: 16, 3: 16, 4: 32}[D]
        return np.dtype({"names": ["p", "dim"], "formats": [(np.float32, (D,)), np.int32],
                         "offsets": [0, 4 * D], "itemsize": size})
    if type_code == REF_F3_PAYLOAD:
        return np.dtype([("p", np.float32, (3,)), ("payload", np.int32)])
    if type_code == REF_F3_PACKED:
        return np.dtype([("p", np.float32, (3,)), ("payload", np.uint32)])
    raise ValueError(type_code)


def ref_build_host(type_code, records):
    """Runs cukd::buildTree_host in place on a copy of `records` (a numpy
    structured or [n,D] float32 array with the reference data_t layout).
    Returns (tree_records, bounds[2,D])."""
    L = ref_host()
    if L is None:
        raise RuntimeError("reference oracle not built (oracle/_ref)")
    recs = np.ascontiguousarray(records).copy()
    D = {REF_F2: 2, REF_F3: 3, REF_F4: 4, REF_F2_DIM: 2, REF_F3_DIM: 3, REF_F4_DIM: 4,
         REF_F3_PAYLOAD: 3, REF_F3_PACKED: 3}[type_code]
    bounds = np.zeros((2, D), np.float32)
    rc = L.refh_build(type_code, _ptr(recs), len(recs), _ptr(bounds))
    if rc:
        raise RuntimeError(f"refh_build failed: {rc}")
    return recs, bounds


def ref_fcp_host(type_code, tree_records, bounds, queries, method, cutoff=np.inf, eps=0.0,
                 threads=None):
    L = ref_host()
    q = np.ascontiguousarray(queries, np.float32)
    out = np.zeros(len(q), np.int32)
    L.refh_fcp(type_code, method, _ptr(tree_records), len(tree_records),
               _ptr(np.ascontiguousarray(bounds, np.float32)), _ptr(q), len(q), float(cutoff),
               float(eps), _ptr(out), threads or nthreads())
    return out


def ref_knn_host(type_code, tree_records, bounds, queries, k, method, list_kind=FIXED_LIST,
                 cutoff=np.inf, threads=None):
    L = ref_host()
    q = np.ascontiguousarray(queries, np.float32)
    ids = np.zeros((len(q), k), np.int32)
    d2 = np.zeros((len(q), k), np.float32)
    ret = np.zeros(len(q), np.float32)
    rc = L.refh_knn(type_code, method, list_kind, k, _ptr(tree_records), len(tree_records),
                    _ptr(np.ascontiguousarray(bounds, np.float32)), _ptr(q), len(q),
                    float(cutoff), _ptr(ids), _ptr(d2), _ptr(ret), threads or nthreads())
    if rc:
        raise RuntimeError(f"refh_knn failed: {rc} (k={k} list={list_kind} not instantiated?)")
    return ids, d2, ret


def ref_spatial_fcp_host(nodes, prims, coords, bounds, queries, method, cutoff=np.inf,
                         threads=None):
    L = ref_host()
    coords = np.ascontiguousarray(coords, np.float32)
    q = np.ascontiguousarray(queries, np.float32)
    out = np.zeros(len(q), np.int32)
    L.refh_spatial_fcp(REF_F3, method, _ptr(nodes), _ptr(prims), _ptr(coords), len(coords),
                       len(nodes), _ptr(np.ascontiguousarray(bounds, np.float32)), _ptr(q),
                       len(q), float(cutoff), _ptr(out), threads or nthreads())
    return out


def ref_spatial_knn_host(nodes, prims, coords, bounds, queries, k, method,
                         list_kind=FIXED_LIST, cutoff=np.inf, threads=None):
    L = ref_host()
    coords = np.ascontiguousarray(coords, np.float32)
    q = np.ascontiguousarray(queries, np.float32)
    ids = np.zeros((len(q), k), np.int32)
    d2 = np.zeros((len(q), k), np.float32)
    rc = L.refh_spatial_knn(REF_F3, method, list_kind, k, _ptr(nodes), _ptr(prims),
                            _ptr(coords), len(coords), len(nodes),
                            _ptr(np.ascontiguousarray(bounds, np.float32)), _ptr(q), len(q),
                            float(cutoff), _ptr(ids), _ptr(d2), threads or nthreads())
    if rc:
        raise RuntimeError(f"refh_spatial_knn failed: {rc}")
    return ids, d2
