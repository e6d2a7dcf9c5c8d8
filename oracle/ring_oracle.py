"""Oracle for the sharded kNN ring (test infrastructure only: tests import
it; the library never does).  Brute-force restatement of what the
reference's samples/mpiHugeQuery.cu computes: per query the k smallest
(d2, id) candidate keys over every shard (its FlexHeapCandidateList keys,
knn.h:343-353, with ids made global), d2 summed left to right in float32 as
the reference's distance (cukd-math.h:107-112), and the k-th distance as its
extractFinalResult writes it (sqrtf unless infinite, mpiHugeQuery.cu:77-90).
The k-th distance is a property of the point set, so it is pinned to the
reference independently of visiting order."""
import numpy as np


def d2_f32(q, p):
    """[nq, n] float32 squared distances, ((dx*dx + dy*dy) + dz*dz) + ..."""
    acc = None
    for d in range(q.shape[1]):
        diff = (q[:, None, d].astype(np.float32) - p[None, :, d].astype(np.float32)).astype(np.float32)
        sq = (diff * diff).astype(np.float32)
        acc = sq if acc is None else (acc + sq).astype(np.float32)
    return acc


def init_keys(nq, k, max_radius):
    r2 = np.float32(max_radius) * np.float32(max_radius)
    key = (np.uint64(np.float32(r2).view(np.uint32)) << np.uint64(32)) | np.uint64(0xFFFFFFFF)
    return np.full((nq, k), key, dtype=np.uint64)


def fold(keys, q, pts, id_offset, chunk=512):
    """keys [nq, k] uint64 ascending: merge in every point of pts."""
    k = keys.shape[1]
    out = np.empty_like(keys)
    for a in range(0, q.shape[0], chunk):
        d2 = d2_f32(q[a:a + chunk], pts)
        kk = (d2.view(np.uint32).astype(np.uint64) << np.uint64(32)) | \
            (np.arange(pts.shape[0], dtype=np.uint64) + np.uint64(id_offset))[None, :]
        allk = np.concatenate([keys[a:a + chunk], kk], axis=1)
        allk.sort(axis=1)
        out[a:a + chunk] = allk[:, :k]
    return out


def extract(keys):
    ids = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    ids = np.where(ids == 0xFFFFFFFF, -1, ids.astype(np.int64)).astype(np.int32)
    d2 = (keys >> np.uint64(32)).astype(np.uint32).view(np.float32)
    kth = d2[:, -1].copy()
    fin = ~np.isinf(kth)
    kth[fin] = np.sqrt(kth[fin]).astype(np.float32)
    return ids, d2, kth
