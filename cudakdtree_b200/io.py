"""The reference's on-disk point formats, for the callers on either side of
the hot path.

* ``load_points`` / ``save_points``: ``cukd::loadPoints<T>`` (cukd/common.h:
  245-267) -- a uint64 record count, then the raw records.
* ``read_file_portion``: the input of samples/mpiHugeQuery.cu -- raw float3
  records with no header; rank r of s reads records [N*r/s, N*(r+1)/s)
  (``readFilePortion``, mpiHugeQuery.cu:41-63, size_t arithmetic).
* ``write_rank_ordered``: its output -- one float32 per point (the k-th
  neighbour distance), each rank appending its block in rank order
  (mpiHugeQuery.cu:207-223).

Records are numpy dtypes (e.g. ``np.dtype((np.float32, 3))`` for float3, or a
structured dtype for records with payloads).
"""
from __future__ import annotations

import os

import numpy as np

FLOAT3 = np.dtype((np.float32, 3))


def load_points(path, dtype=FLOAT3):
    """Records written by ``save_points`` / read by ``cukd::loadPoints``."""
    dtype = np.dtype(dtype)
    with open(path, "rb") as f:
        head = f.read(8)
        if len(head) != 8:
            raise ValueError(f"{path}: missing the 8-byte record count")
        count = int(np.frombuffer(head, dtype="<u8")[0])
        data = np.fromfile(f, dtype=dtype, count=count)
    if data.shape[0] != count:
        raise ValueError(f"{path}: header says {count} records, file holds {data.shape[0]}")
    return data


def save_points(path, records):
    """Writes the uint64 count then the raw records (cukd::loadPoints's format)."""
    records = np.ascontiguousarray(records)
    with open(path, "wb") as f:
        f.write(np.array([records.shape[0]], dtype="<u8").tobytes())
        f.write(records.tobytes())


def portion_range(num_records, rank, size):
    """[begin, end) of rank's share: num*rank/size .. num*(rank+1)/size."""
    if size < 1 or not 0 <= rank < size:
        raise ValueError("rank must be in [0, size)")
    return (num_records * rank) // size, (num_records * (rank + 1)) // size


def read_file_portion(path, rank, size, dtype=FLOAT3):
    """(records, begin, total) of rank's share of a headerless record file."""
    dtype = np.dtype(dtype)
    total = os.path.getsize(path) // dtype.itemsize
    begin, end = portion_range(total, rank, size)
    with open(path, "rb") as f:
        f.seek(begin * dtype.itemsize)
        data = np.fromfile(f, dtype=dtype, count=end - begin)
    return data, begin, total


def write_rank_ordered(path, values, rank=0, size=1, group=None):
    """Rank 0 creates the file, every rank then appends its block in rank
    order (barriers between ranks, as the reference does).  ``group`` is a
    torch.distributed process group (None with size 1)."""
    values = np.ascontiguousarray(values, dtype=np.float32)
    if size > 1:
        import torch.distributed as dist
        dist.barrier(group=group)
    for i in range(size):
        if i == rank:
            with open(path, "wb" if i == 0 else "ab") as f:
                f.write(values.tobytes())
        if size > 1:
            dist.barrier(group=group)
