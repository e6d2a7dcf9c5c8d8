/*
 * cukd_b200.h -- C ABI of the B200 (sm_100a) k-d tree library.
 *
 * A drop-in for the hot path of ingowald/cudaKDTree.  The reference is a
 * header-only C++ template library with no ABI; every entry point below is
 * the plain-C, status-returning counterpart of one of its host templates
 * (cited per declaration, paths relative to the reference project).  The
 * C++ shim in include/cukd/ keeps the reference's template API and forwards
 * here; Python reaches the same entry points through ctypes
 * (cudakdtree_b200/__init__.py).
 *
 * Conventions
 *   - All pointers named d_* are device pointers (cudaMalloc'd or managed).
 *   - No entry point throws; each returns a cukd_status.  The C++ shim turns
 *     non-zero statuses into std::runtime_error, like the reference.
 *   - All work is enqueued on `stream`; entry points do not synchronise the
 *     stream unless stated (the reference builder_thrust syncs every level).
 *   - Temporary memory comes from `mem` (NULL = cudaMallocAsync /
 *     cudaFreeAsync on `stream`), the counterpart of the reference's
 *     GpuMemoryResource (cukd/helpers.h:30-70).
 */
#ifndef CUKD_B200_H
#define CUKD_B200_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime_api.h>

#if defined(_WIN32)
#define CUKD_API __declspec(dllexport)
#else
#define CUKD_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CUKD_B200_VERSION 1

typedef enum cukd_status {
  CUKD_OK = 0,
  CUKD_ERR_INVALID_ARGUMENT = 1,
  /* explicit split dims requested but no world-bounds buffer given
   * (cukd/builder_thrust.h:469-473, builder_bitonic.h:367-372) */
  CUKD_ERR_MISSING_WORLD_BOUNDS = 2,
  CUKD_ERR_OUT_OF_MEMORY = 3,
  CUKD_ERR_CUDA = 4,
  CUKD_ERR_UNSUPPORTED = 5,
  /* a bounded device-side wait gave up (batched persistent path) */
  CUKD_ERR_TIMEOUT = 6,
  /* a spatial-tree traversal exceeded its 50-entry stack
   * (cukd/knn.h:620-623 prints "STACK OVERFLOW") */
  CUKD_ERR_STACK_OVERFLOW = 7,
  /* input exceeds the fixed scratch of cukd_build_tree_noalloc */
  CUKD_ERR_TOO_LARGE = 8,
  /* a consistency check inside a builder failed (reported by
   * cukd_build_check; the records hold a permutation of the input) */
  CUKD_ERR_INTERNAL = 9
} cukd_status;

/* ------------------------------------------------------------------------
 * Data description: the C-ABI form of the reference's data_traits
 * (cukd/data.h:56-112).  A data item is a record of `stride` bytes holding
 * `num_dims` contiguous 32-bit coordinates at `point_offset`, and -- for
 * trees with explicit split dimensions (data_traits::has_explicit_dim) -- a
 * split dimension stored in bits [dim_shift, dim_shift+dim_bits) of the
 * 32-bit word at `dim_offset` (dim_offset = -1: round-robin dims).
 *
 *   float3                         {CUKD_FLOAT32, 3, 12, 0, -1, 0, 0}
 *   struct {float3 p; int dim;}    {CUKD_FLOAT32, 3, 16, 0, 12, 0, 32}
 *   struct {float3 p; int payload;} with the dim in payload bits 30..31
 *                                  {CUKD_FLOAT32, 3, 16, 0, 12, 30, 2}
 * ------------------------------------------------------------------------ */
typedef enum cukd_scalar_type { CUKD_FLOAT32 = 0, CUKD_INT32 = 1 } cukd_scalar_type;

typedef struct cukd_layout {
  int32_t scalar_type;  /* cukd_scalar_type */
  int32_t num_dims;     /* 2..8 (the reference's float2/3/4, int2/3/4 and
                         * vec_float<N>); every builder and the reference-order
                         * FCP / kNN take up to 8, the fast kNN, learned radius,
                         * spatial tree, batched plans, Morton order and the
                         * allocation-free builder up to 4 (else
                         * CUKD_ERR_UNSUPPORTED / INVALID_ARGUMENT) */
  int32_t stride;       /* bytes per record, multiple of 4 */
  int32_t point_offset; /* byte offset of coordinate 0, multiple of 4 */
  int32_t dim_offset;   /* byte offset of the dim word, multiple of 4; -1 = none */
  int32_t dim_shift;    /* dim = (word >> dim_shift) & ((1 << dim_bits) - 1) */
  int32_t dim_bits;     /* 1..32 */
} cukd_layout;

/* world bounds: box_t<point_t> (cukd/box.h:35-82) = lower[num_dims] then
 * upper[num_dims], of the scalar type. */

/* Memory resource: reference GpuMemoryResource (cukd/helpers.h:30-33).
 * Any alignment works: each request asks for 16 bytes more than it uses and
 * aligns the block up itself (the builder stages its arrays with 16-byte
 * bulk copies); release receives the pointer alloc returned. */
typedef struct cukd_mem_resource {
  void *ctx;
  int (*alloc)(void *ctx, void **ptr, size_t bytes, cudaStream_t stream); /* 0 = ok */
  int (*release)(void *ctx, void *ptr, cudaStream_t stream);
} cukd_mem_resource;

/* ------------------------------------------------------------------------
 * Left-balanced k-d tree builders
 * ------------------------------------------------------------------------ */
typedef enum cukd_builder {
  /* reference default: builder_thrust (cukd/builder.h:108-152) */
  CUKD_BUILDER_DEFAULT = 0,
  CUKD_BUILDER_THRUST = 1,
  CUKD_BUILDER_BITONIC = 2,
  CUKD_BUILDER_INPLACE = 3
} cukd_builder;

/* Builds a left-balanced k-d tree in place: reorders the n records at
 * d_points so that record i is node i of the implicit tree (children 2i+1,
 * 2i+2), and -- for explicit-dim layouts -- writes each node's split dim
 * (the widest extent of its domain).  Writes the world bounds to
 * d_world_bounds when non-NULL (mandatory for explicit-dim layouts).
 * Temporary memory (through `mem`) and output by builder:
 *   DEFAULT, THRUST  ~65 bytes per point of float3; the reference's
 *                    canonical order (buildTree_host / buildTree_thrust),
 *                    ties included;
 *   BITONIC          4 bytes per point (one uint32 tag, like the
 *                    reference's) plus ~5.5 MB; the same canonical order;
 *   INPLACE          ~5.5 MB whatever n (the reference's takes none); the
 *                    canonical order whenever the coordinates decide every
 *                    split (e.g. no two points share a coordinate value),
 *                    otherwise a valid left-balanced k-d tree of the same
 *                    records that depends only on the input array (the
 *                    reference's builders promise no more with ties,
 *                    testing/testBuildersSameResult.cu:96-99).
 * BITONIC and INPLACE run one cooperative launch for the top levels; a
 * bounded grid-barrier wait that gives up, or a failed consistency check,
 * stops the build (cukd_build_check reports CUKD_ERR_TIMEOUT /
 * CUKD_ERR_INTERNAL; the array then holds a permutation of its records).
 * Replaces cukd::buildTree (cukd/builder.h:108-152),
 * buildTree_thrust (cukd/builder_thrust.h:90-110),
 * buildTree_bitonic (cukd/builder_bitonic.h:83-94),
 * buildTree_inPlace (cukd/builder_inplace.h:82-102, 474-480).
 * n < 1 returns CUKD_OK without touching anything (builder_thrust.h:441). */
CUKD_API int cukd_build_tree(void *d_points, int64_t n, const cukd_layout *layout,
                    void *d_world_bounds, int builder, cudaStream_t stream,
                    const cukd_mem_resource *mem);

/* Allocation-free build: the same tree as cukd_build_tree (same order, same
 * explicit dims, same world bounds), for callers that cannot allocate device
 * memory when they build -- code whose device memory is owned by another
 * framework's pool, real-time loops that cannot risk cudaMalloc's latency or
 * failure, deployments with a footprint fixed at load time.  No counterpart
 * in the reference (its builders always allocate through a
 * GpuMemoryResource).
 *
 * All scratch comes from one fixed 40 MiB device array inside this library
 * (held on every GPU that loads it, until the process exits); the call
 * allocates and frees nothing.  Limits: n <= 262144 records, stride <= 64
 * bytes; larger inputs return CUKD_ERR_TOO_LARGE.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress); make
 * that first call before any stream capture on that device.  All calls
 * share the array: calls that may run concurrently on the GPU race and must
 * be ordered by the caller (one stream, or events).  Each call resets the
 * parts of the array it needs initialised. */
CUKD_API int cukd_build_tree_noalloc(void *d_points, int64_t n, const cukd_layout *layout,
                                     void *d_world_bounds, cudaStream_t stream);

/* Computes the world bounds of n records into d_world_bounds.
 * Replaces cukd::computeBounds (cukd/builder_common.h:151-162). */
CUKD_API int cukd_compute_bounds(const void *d_points, int64_t n, const cukd_layout *layout,
                        void *d_world_bounds, cudaStream_t stream);

/* Typed convenience forms of cukd_build_tree for the reference's default
 * data types (cukd/cukd-math.h:42-59: float2/3/4, int2/3/4). */
CUKD_API int cukd_build_float2(void *d_points, int64_t n, void *d_world_bounds, cudaStream_t stream,
                      const cukd_mem_resource *mem);
CUKD_API int cukd_build_float3(void *d_points, int64_t n, void *d_world_bounds, cudaStream_t stream,
                      const cukd_mem_resource *mem);
CUKD_API int cukd_build_float4(void *d_points, int64_t n, void *d_world_bounds, cudaStream_t stream,
                      const cukd_mem_resource *mem);
CUKD_API int cukd_build_int2(void *d_points, int64_t n, void *d_world_bounds, cudaStream_t stream,
                    const cukd_mem_resource *mem);
CUKD_API int cukd_build_int3(void *d_points, int64_t n, void *d_world_bounds, cudaStream_t stream,
                    const cukd_mem_resource *mem);
CUKD_API int cukd_build_int4(void *d_points, int64_t n, void *d_world_bounds, cudaStream_t stream,
                    const cukd_mem_resource *mem);

/* ------------------------------------------------------------------------
 * Queries over a left-balanced tree (whole-batch launches)
 * ------------------------------------------------------------------------ */
typedef enum cukd_method {
  CUKD_STACK_BASED = 0, /* cukd::stackBased (traverse-default-stack-based.h) */
  CUKD_STACK_FREE = 1,  /* cukd::stackFree  (traverse-stack-free.h) */
  CUKD_CCT = 2          /* cukd::cct        (traverse-cct.h) */
} cukd_method;

enum {
  /* sort queries along a 30-bit Morton curve before traversal and scatter
   * results back to the caller's order (results are unchanged) */
  CUKD_QUERY_MORTON = 1,
  /* kNN: return the candidate list in the reference HeapCandidateList's
   * heap order instead of ascending (d2, id) order */
  CUKD_QUERY_HEAP_ORDER = 2,
  /* kNN: use the heap candidate list even for small k */
  CUKD_QUERY_FORCE_HEAP = 4,
  /* run every query with the reference's own visiting order (by default
   * queries whose answer cannot depend on the order -- no distance tie at
   * the k-th boundary -- take a faster traversal; the answers are the same
   * bits either way) */
  CUKD_QUERY_REFERENCE_ORDER = 8,
  /* sort queries by the path a closest-side descent takes down this tree
   * (left / right bits, root first) instead of by Morton code: an order
   * adapted to the tree's own splits; results are unchanged.  Takes
   * precedence over CUKD_QUERY_MORTON. */
  CUKD_QUERY_TREE_ORDER = 16,
  /* float kNN with k = 2..32: the warp-cooperative traversal (the 32
   * lanes of a warp walk one node stream for 32 consecutive queries of
   * the visiting order, entering a subtree when any lane's box distance is
   * within that lane's bound) instead of one traversal per thread; the
   * same answers (cukd_knn and cukd_knn_learned) */
  CUKD_QUERY_WARP_PACKET = 32
};

typedef struct cukd_query_params {
  int32_t method;        /* cukd_method */
  int32_t k;             /* kNN only, 1..1024 */
  float cutoff_radius;   /* float trees: FcpSearchParams::cutOffRadius (INFINITY = none) */
  float eps;             /* FcpSearchParams::eps, honoured by CUKD_STACK_FREE */
  int64_t cutoff_d2;     /* int trees: squared cut-off radius (INT64_MAX = none) */
  int32_t flags;         /* CUKD_QUERY_* */
  int32_t block_size;    /* 0 = default (128); else threads per block, 32..256 */
  /* optional device int: receives how many queries were re-run in the
   * reference's visiting order (distance ties at the k-th boundary) */
  int32_t *d_reordered_count;
} cukd_query_params;

/* Default parameters: stack-based, k = 8, no cut-off, Morton on. */
CUKD_API void cukd_query_params_init(cukd_query_params *p);

/* Every query entry point below takes trees of at most 2^30 - 1 nodes and
 * returns CUKD_ERR_UNSUPPORTED for larger ones: node indices are 32-bit ints
 * (as in the reference's traversals) and a node's children 2i+1, 2i+2 must
 * fit one. */

/* Find-closest-point for nq queries (point_t[nq]: num_dims contiguous
 * scalars each).  d_out_ids[i] = node index of the closest point within the
 * cut-off, -1 if none (cukd/fcp.h:54-163, FCPResult :179-207).  For float
 * trees d_out_d2 (optional) receives the squared distance as float, for
 * int trees as int64.  d_world_bounds is required for CUKD_CCT. */
CUKD_API int cukd_fcp(const void *d_tree, int64_t n, const cukd_layout *layout,
             const void *d_world_bounds, const void *d_queries, int64_t nq,
             const cukd_query_params *params, int32_t *d_out_ids, void *d_out_d2,
             cudaStream_t stream, const cukd_mem_resource *mem);

/* k nearest neighbours (cukd/knn.h:83-199 with FixedCandidateList /
 * HeapCandidateList semantics, knn.h:214-287).  d_out_ids / d_out_d2 are
 * [nq][k]; unfilled slots hold id -1 and d2 = cutoff^2 (knn.h:505-511).
 * d_out_max_d2 (optional, [nq]) receives knn()'s return value.  float trees
 * write float d2, int trees int64 d2. */
CUKD_API int cukd_knn(const void *d_tree, int64_t n, const cukd_layout *layout,
             const void *d_world_bounds, const void *d_queries, int64_t nq,
             const cukd_query_params *params, int32_t *d_out_ids, void *d_out_d2,
             void *d_out_max_d2, cudaStream_t stream, const cukd_mem_resource *mem);

/* cukd_knn with the queries and results in host memory: the queries are
 * processed in chunks of `chunk` (0 = 2^20) whose host->device copies,
 * searches and device->host copies overlap on three streams; device
 * memory: three sets of chunk-sized query and result buffers.  Results are
 * cukd_knn's.  Use page-locked host buffers (cudaHostAlloc) for the copies
 * to overlap.  Returns once the work is queued; `stream` completes after the
 * last result copy.  No reference counterpart as one call (the reference's
 * samples copy whole arrays around one query launch, sample.cu:121-160). */
CUKD_API int cukd_knn_host(const void *d_tree, int64_t n, const cukd_layout *layout,
                           const void *d_world_bounds, const void *h_queries, int64_t nq,
                           const cukd_query_params *params, int32_t *h_out_ids, void *h_out_d2,
                           int64_t chunk, cudaStream_t stream, const cukd_mem_resource *mem);

/* cukd_knn_host that leaves `stream` free once the searches are queued: the
 * answers are complete in h_out_ids / h_out_d2 once the caller's event
 * `done` (created by the caller) has completed -- wait for it
 * (cudaEventSynchronize, or cudaStreamWaitEvent before reusing those host
 * buffers).  A caller can thus queue the next batch's build and search on
 * the same stream while these answers are still being copied.  `chunk`
 * 0 = 2^24: consecutive calls overlap each other's copies, so a batch is
 * best searched in one slice (10M queries, k = 16, back to back: 23.8 ms a
 * batch in one slice, 26.8 ms in 2^21-query slices).  Up to eight device
 * result sets per call (released on the copy stream, after the copies),
 * taken from a device memory pool of the library's own when `mem` is NULL.
 * No reference counterpart. */
CUKD_API int cukd_knn_host_async(const void *d_tree, int64_t n, const cukd_layout *layout,
                        const void *d_world_bounds, const void *h_queries, int64_t nq,
                        const cukd_query_params *params, int32_t *h_out_ids, void *h_out_d2,
                        int64_t chunk, cudaEvent_t done, cudaStream_t stream,
                        const cukd_mem_resource *mem);

/* cukd_knn_host for queries already in device memory: the searches of
 * `chunk`-query slices of d_queries overlap the device->host copies of the
 * answers of the previous slices (two streams; three sets of chunk-sized
 * result buffers).  For callers that upload the queries themselves, e.g. on
 * their own stream while the tree builds.  Results are cukd_knn's; `stream`
 * completes after the last result copy.  No reference counterpart as one
 * call (see cukd_knn_host). */
CUKD_API int cukd_knn_to_host(const void *d_tree, int64_t n, const cukd_layout *layout,
                              const void *d_world_bounds, const void *d_queries, int64_t nq,
                              const cukd_query_params *params, int32_t *h_out_ids,
                              void *h_out_d2, int64_t chunk, cudaStream_t stream,
                              const cukd_mem_resource *mem);

/* cukd_knn_to_host with the answers landing behind the caller's event `done`
 * and `stream` free once the searches are queued (see cukd_knn_host_async).
 * No reference counterpart. */
CUKD_API int cukd_knn_to_host_async(const void *d_tree, int64_t n, const cukd_layout *layout,
                           const void *d_world_bounds, const void *d_queries, int64_t nq,
                           const cukd_query_params *params, int32_t *h_out_ids,
                           void *h_out_d2, int64_t chunk, cudaEvent_t done,
                           cudaStream_t stream, const cukd_mem_resource *mem);

/* Per-query visited-node counts of the same traversal (the reference's
 * CUKD_ENABLE_STATS counter, cukd/common.h:345-360, per query). */
CUKD_API int cukd_knn_visits(const void *d_tree, int64_t n, const cukd_layout *layout,
                    const void *d_world_bounds, const void *d_queries, int64_t nq,
                    const cukd_query_params *params, int64_t *d_out_visits,
                    cudaStream_t stream, const cukd_mem_resource *mem);

/* Morton-order permutation of nq float points (30-bit codes inside the
 * given bounds): d_out_perm[i] = index of the i-th query along the curve. */
CUKD_API int cukd_morton_order(const float *d_points, int64_t n, int num_dims,
                      const float *d_bounds, int32_t *d_out_perm, cudaStream_t stream,
                      const cukd_mem_resource *mem);

/* ------------------------------------------------------------------------
 * Sharded kNN (reference: the ring of samples/mpiHugeQuery.cu:105-225, whose
 * per-round kernel resumes a FlexHeapCandidateList, cukd/knn.h:360-371)
 * ------------------------------------------------------------------------ */
/* Folds one float tree shard (built by cukd_build_tree) into per-query
 * candidate lists d_lists (device uint64[nq][k], ascending keys
 * d2-float-bits << 32 | global id) that persist across calls; global id =
 * node index + id_offset.  init != 0 starts each list as k slots of
 * (max_radius^2, id 0xffffffff), the reference's round-0 list; otherwise the
 * lists continue from the previous call.  After any sequence of calls a list
 * holds the k smallest (d2, global id) keys over all points folded in, in any
 * shard order.  d_order (optional) is a visiting order of the queries (for
 * example cukd_morton_order's).  k = 1..128. */
CUKD_API int cukd_knn_accumulate(const void *d_tree, int64_t n, const cukd_layout *layout,
                                 const void *d_world_bounds, int64_t id_offset,
                                 const void *d_queries, int64_t nq, const int32_t *d_order,
                                 int k, float max_radius, int init, uint64_t *d_lists,
                                 cudaStream_t stream);

/* Splits lists into ids (-1 = unfilled), d2 ([nq][k] each, optional) and the
 * k-th distance per query (optional; sqrt of the k-th d2 unless infinite,
 * what mpiHugeQuery.cu's extractFinalResult writes, :77-90). */
CUKD_API int cukd_knn_lists_extract(const uint64_t *d_lists, int64_t nq, int k,
                                    int32_t *d_out_ids, float *d_out_d2, float *d_out_kth_dist,
                                    cudaStream_t stream);

/* ------------------------------------------------------------------------
 * Spatial k-d tree (reference: cukd/spatial-kdtree.h)
 * ------------------------------------------------------------------------ */
/* Node record, byte-identical to SpatialKDTree<>::Node
 * (cukd/spatial-kdtree.h:69-98): inner nodes have count 0 and their
 * children at offset / offset+1; leaves list `count` prim ids from
 * prim_ids[offset]. */
typedef struct cukd_spatial_node {
  float pos;
  uint32_t offset;
  uint16_t count;
  int16_t dim;
} cukd_spatial_node;

typedef struct cukd_spatial_tree {
  cukd_spatial_node *nodes; /* device, num_nodes entries (owned) */
  uint32_t *prim_ids;       /* device, num_prims entries (owned) */
  const void *data;         /* the caller's records, not reordered (borrowed) */
  int32_t num_prims;
  int32_t num_nodes;
  int32_t num_dims;
  float bounds[8];          /* lower[0..D) at [0], upper[0..D) at [4] */
} cukd_spatial_tree;

/* Builds a spatial k-d tree over n float records (leaves of at most
 * leaf_threshold prims; 0 = the reference's default of 8).  Allocates the
 * node and prim-id arrays through `mem` (free them with cukd_spatial_free);
 * the records are only read.  Children are numbered in parent order and
 * degenerate splits alternate prims by prim id, where the reference uses
 * atomic order; the tree is otherwise the reference's.
 * Replaces cukd::buildTree(SpatialKDTree&, ...) (cukd/spatial-kdtree.h:113-126,
 * 632-645).  Synchronises `stream` once per tree level. */
CUKD_API int cukd_spatial_build(const void *d_points, int64_t n, const cukd_layout *layout,
                                int leaf_threshold, cukd_spatial_tree *out_tree,
                                cudaStream_t stream, const cukd_mem_resource *mem);

/* Replaces cukd::free(SpatialKDTree&, ...) (cukd/spatial-kdtree.h:618-630). */
CUKD_API int cukd_spatial_free(cukd_spatial_tree *tree, cudaStream_t stream,
                               const cukd_mem_resource *mem);

/* FCP / kNN over a spatial tree, CUKD_STACK_BASED or CUKD_CCT
 * (cukd/fcp.h:256-427, cukd/knn.h:566-646, 680-752).  Ids are the caller's
 * record indices.  A query that overflows the reference's 50-entry stack
 * returns what the reference returns (FCP -1). */
CUKD_API int cukd_spatial_fcp(const cukd_spatial_tree *tree, const cukd_layout *layout,
                              const void *d_queries, int64_t nq,
                              const cukd_query_params *params, int32_t *d_out_ids,
                              void *d_out_d2, cudaStream_t stream, const cukd_mem_resource *mem);
CUKD_API int cukd_spatial_knn(const cukd_spatial_tree *tree, const cukd_layout *layout,
                              const void *d_queries, int64_t nq,
                              const cukd_query_params *params, int32_t *d_out_ids,
                              void *d_out_d2, cudaStream_t stream, const cukd_mem_resource *mem);

/* ------------------------------------------------------------------------
 * Learned kNN-radius proposal (no reference counterpart)
 *
 * A small MLP (the query's D coordinates + log density of a res^D occupancy
 * grid, padded to 8 inputs -> 64 -> 64 -> 1, BF16 weights and activations,
 * FP32 accumulation, run on the tensor cores) predicts each query's k-th-
 * neighbour distance.  cukd_knn_learned seeds every query's cull radius with
 * the prediction times a safety scale; queries that find fewer than k
 * points inside it (or hit an exact distance tie at the k-th boundary) are
 * re-run by the plain traversal, so its results equal cukd_knn's bit for
 * bit.  Trees of float or int32 points, D = 2..4 (a model is made for one
 * D and learns on one coordinate type).
 * ------------------------------------------------------------------------ */
typedef struct cukd_radius_model_s cukd_radius_model;

/* Creates an untrained model for num_dims-dimensional points (2..4; at most
 * 2^24 grid cells) with a seeded initialisation on the current device. */
CUKD_API int cukd_radius_model_create_nd(cukd_radius_model **out, int grid_res, int num_dims,
                                         uint64_t seed);
/* The same for 3-D points. */
CUKD_API int cukd_radius_model_create(cukd_radius_model **out, int grid_res, uint64_t seed);
CUKD_API int cukd_radius_model_destroy(cukd_radius_model *model);

/* Builds the occupancy grid from the tree's points inside the world bounds
 * (h_world_bounds: host float[2 * D], lower then upper; int trees pass their
 * bounds as floats).  The layout's D must be the model's; its coordinate
 * type becomes the type of the queries the model takes. */
CUKD_API int cukd_radius_model_set_grid(cukd_radius_model *model, const void *d_points,
                                        int64_t n, const cukd_layout *layout,
                                        const float *h_world_bounds, cudaStream_t stream);

/* Training loss of later cukd_radius_model_train / _gradients calls on the
 * standardised log distance: quantile 0 (the default) = mean squared error,
 * so the network predicts the conditional mean; 0 < quantile < 1 = pinball
 * loss, so it predicts that quantile of the k-th distance given the
 * features -- a larger safety margin where the features say less, fewer
 * fallbacks to the plain traversal at the same radius scale. */
CUKD_API int cukd_radius_model_set_loss(cukd_radius_model *model, float quantile);

/* Trains on nq queries (device point_t[nq] of the grid's coordinate type)
 * and their exact k-th squared distances (float[nq] for float trees,
 * int64[nq] for int trees; for example the knn() return values of
 * cukd_knn): Adam on minibatches, `epochs` passes; *h_final_loss receives
 * the last epoch's mean squared error on the standardised log distance (or
 * the pinball loss, cukd_radius_model_set_loss). */
CUKD_API int cukd_radius_model_train(cukd_radius_model *model, const void *d_queries,
                                     const void *d_kth_d2, int64_t nq, int epochs, int batch,
                                     float lr, float *h_final_loss, cudaStream_t stream);

/* Predicted k-th-neighbour distance per query (not squared, not scaled). */
CUKD_API int cukd_radius_model_predict(const cukd_radius_model *model, const void *d_queries,
                                       int64_t nq, float *d_out_radius, cudaStream_t stream);

/* The model's 8 input features per query (device float[nq][8]: D
 * coordinates in [-1, 1], the density feature, zeros). */
CUKD_API int cukd_radius_model_features(const cukd_radius_model *model, const void *d_queries,
                                        int64_t nq, float *d_out_features, cudaStream_t stream);

/* Loss gradient over n (features [n][8], standardised target) pairs at the
 * model's current BF16 weights, without updating them; also returns those
 * weights as floats and the loss (host buffers of 4801 floats).  For
 * checking the hand-written backward pass against a CPU oracle. */
CUKD_API int cukd_radius_model_gradients(cukd_radius_model *model, const float *d_features,
                                         const float *d_targets, int64_t n, float *h_grad,
                                         float *h_params_bf16, float *h_loss,
                                         cudaStream_t stream);

/* kNN (k = 2..128) seeded with the learned radius times radius_scale: the
 * queries are put in Morton order (float trees), the network predicts their
 * radii on the tensor cores -- inside the search kernel for float trees and
 * k <= 32, in a pass of its own otherwise -- and the fast traversal starts
 * each query's cull radius at its prediction.
 * d_out_fallback (optional, device int[2]): queries re-run by the plain
 * traversal, and by the reference's own visiting order.  d_status
 * (optional, device int[nq]): 0 if the learned pass answered the query, 1 if
 * it was re-run.  d_visits (optional, device int64[nq], zeroed by the
 * caller): visited nodes per query, all passes together. */
CUKD_API int cukd_knn_learned(const void *d_tree, int64_t n, const cukd_layout *layout,
                              const void *d_world_bounds, const void *d_queries, int64_t nq,
                              const cukd_query_params *params, const cukd_radius_model *model,
                              float radius_scale, int32_t *d_out_ids, void *d_out_d2,
                              int32_t *d_out_fallback, int32_t *d_status, int64_t *d_visits,
                              cudaStream_t stream, const cukd_mem_resource *mem);

/* ------------------------------------------------------------------------
 * Batched clouds (no reference counterpart: the reference builds and
 * queries one tree per call, cukd/builder.h:108-122, and its samples loop
 * over calls)
 *
 * B independent float clouds (num_dims = 2..4) stored one after another in
 * one array, with CSR offsets h_point_offsets[B + 1]; B query sets, CSR
 * offsets h_query_offsets[B + 1], each answered against its own cloud.
 * Every cloud becomes the same left-balanced tree (round-robin dims) that
 * cukd_build_tree gives it alone, in place in its slice; query results are
 * the per-cloud cukd_knn / cukd_fcp results with ids local to the cloud.
 * The plan derives all per-level work lists from the sizes once and owns
 * every temporary, so a run allocates nothing and a build + query can be
 * recorded as one CUDA graph (cukd_batch_run) and replayed.
 * ------------------------------------------------------------------------ */
typedef struct cukd_batch_plan_s cukd_batch_plan;

typedef struct cukd_batch_tuning {
  int32_t build_tile;          /* subtree-phase tile: 512, 1024 or 2048 points */
  int32_t block_size;          /* query threads per block: 32..512, multiple of 32
                                * (above 256 only for k = 2..32 fixed lists) */
  int32_t queries_per_thread;  /* 1, 2 or 4 */
  int32_t morton;              /* 1: visit each cloud's queries in Morton order */
  float build_ms, query_ms;    /* cukd_batch_autotune: best times measured */
} cukd_batch_tuning;

/* params: method, k (1..1024; 0 = FCP), cutoff_radius, eps, flags as for
 * cukd_knn (CUKD_QUERY_MORTON is replaced by the tuning's `morton`).  The
 * offsets are host arrays, non-decreasing, starting at 0.  Allocates the
 * plan's device memory on the current device. */
CUKD_API int cukd_batch_plan_create(cukd_batch_plan **out, int num_dims, int64_t num_clouds,
                                    const int64_t *h_point_offsets,
                                    const int64_t *h_query_offsets,
                                    const cukd_query_params *params);
CUKD_API int cukd_batch_plan_destroy(cukd_batch_plan *plan);
CUKD_API int cukd_batch_get_tuning(const cukd_batch_plan *plan, cukd_batch_tuning *out);
/* Validates and installs a tuning (drops a recorded graph). */
CUKD_API int cukd_batch_set_tuning(cukd_batch_plan *plan, const cukd_batch_tuning *tuning);

/* Builds every cloud of d_points (float[total][D]) in place; per-cloud
 * boxes into d_cloud_bounds (optional, float[B][2][D]: lower then upper,
 * +inf/-inf for an empty cloud). */
CUKD_API int cukd_batch_build(cukd_batch_plan *plan, float *d_points, float *d_cloud_bounds,
                              cudaStream_t stream);
/* Queries of all clouds against built clouds: kNN writes d_out_ids /
 * d_out_d2 as [nq][k], FCP as [nq] (d_out_d2 optional).  d_cloud_bounds
 * (from cukd_batch_build) is required for CUKD_CCT and for Morton order. */
CUKD_API int cukd_batch_query(cukd_batch_plan *plan, const float *d_points,
                              const float *d_cloud_bounds, const float *d_queries,
                              int32_t *d_out_ids, float *d_out_d2, cudaStream_t stream);
/* Build + query as one CUDA graph: recorded on the first call with a set of
 * pointers (and after a tuning change), replayed on the caller's stream
 * afterwards.  d_cloud_bounds may be null (the plan keeps its own). */
CUKD_API int cukd_batch_run(cukd_batch_plan *plan, float *d_points, float *d_cloud_bounds,
                            const float *d_queries, int32_t *d_out_ids, float *d_out_d2,
                            cudaStream_t stream);
/* Times candidate tunings on the caller's data (build tiles, then query
 * block size x queries per thread x Morton, `reps` runs each, median) and
 * installs the fastest; d_points is copied, never modified.  *out
 * (optional) receives the chosen tuning and its times.  Synchronises. */
CUKD_API int cukd_batch_autotune(cukd_batch_plan *plan, const float *d_points,
                                 const float *d_queries, int reps, cukd_batch_tuning *out,
                                 cudaStream_t stream);

/* ------------------------------------------------------------------------
 * Error strings
 * ------------------------------------------------------------------------ */
CUKD_API const char *cukd_status_string(int status);
/* the CUDA error behind the last CUKD_ERR_CUDA on this thread */
CUKD_API const char *cukd_last_cuda_error(void);
/* running count of kernels launched by this library in this process (an
 * observability counter, like the reference's CUKD_ENABLE_STATS hook,
 * cukd/common.h:345-360) */
CUKD_API unsigned long long cukd_launch_count(void);
/* number of bounded waits on bulk-copy barriers (the builder's partition
 * pass) that gave up on the current device since the library was loaded;
 * 0 unless something is badly wrong -- a kernel ends instead of hanging,
 * and that build stops, leaving the caller's records unchanged.
 * Synchronises the device.  No reference counterpart. */
CUKD_API int cukd_async_wait_timeouts(unsigned int *count);

/* Synchronises `stream` and returns CUKD_ERR_TIMEOUT if a bounded wait of
 * a build on the current device gave up since the previous check (that
 * build stopped; the default builder leaves the caller's records exactly as
 * they were, the bitonic / in-place ones a permutation of them),
 * CUKD_ERR_INTERNAL if a bitonic / in-place build's consistency check
 * failed, else CUKD_OK.  The reference's builders synchronise and throw on failure
 * (builder_thrust.h:479-511, common.h:276-285); the C++ shim's buildTree
 * calls this after the build to do the same. */
CUKD_API int cukd_build_check(cudaStream_t stream);

/* Test hook: how many times the builder's first bulk-copy wait, and the
 * bitonic / in-place builders' grid barriers, poll before giving up, on the
 * current device (default
 * CUKD_ASYNC_WAIT_POLLS_DEFAULT; 0 gives up at once, so that a test can make
 * the wait run out without any fault).  Synchronous. */
#define CUKD_ASYNC_WAIT_POLLS_DEFAULT 4194304u
CUKD_API int cukd_set_async_wait_polls(uint32_t polls);

#ifdef __cplusplus
}
#endif
#endif /* CUKD_B200_H */
