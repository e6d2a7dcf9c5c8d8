/*
 * cukd_oracle.h -- CPU restatement of the reference k-d tree algorithms.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the tests,
 * the smoke check and the benchmark's CPU-baseline leg compare the CUDA
 * product library against.  Nothing in the product links it.
 *
 * Parity: pinned against the reference itself (oracle/_ref, built from the
 * reference headers by oracle/Makefile) and against the reference's golden
 * vectors (testing/issue5.cu) -- see tests/test_oracle.py.
 *
 * Conventions
 *   scalar : 0 = float32 coordinates, 1 = int32 coordinates
 *   D      : number of dimensions, 1..8
 *   coords : array-of-structs [n][D] of the scalar type
 *   bounds : 2*D scalars, lower[D] then upper[D]
 *   dims   : per-node split dimension (int32) for explicit-dim trees, or
 *            NULL for round-robin trees
 */
#ifndef CUKD_ORACLE_H
#define CUKD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* traversal methods */
enum { CKO_STACK_BASED = 0, CKO_STACK_FREE = 1, CKO_CCT = 2 };
/* candidate lists */
enum { CKO_FIXED_LIST = 0, CKO_HEAP_LIST = 1 };

/* Left-balanced k-d tree build.  perm_out[node] = input index of the point
 * that ends up at array position `node`; dims_out[node] = its split dim
 * (explicit-dim builds only; may be NULL otherwise); bounds_out receives the
 * world bounds (may be NULL unless explicit_dim).  Returns 0, or 2 when
 * explicit_dim is set without bounds_out (the reference's runtime_error). */
int cko_build(int scalar, int D, const void *coords, int64_t n, int explicit_dim,
              int64_t *perm_out, int32_t *dims_out, void *bounds_out);

/* Checks, without rebuilding, that `tree` ([n][D] coordinates in node order,
 * index[node] = the point's input index) is the canonical tree cko_build
 * returns: every node's left subtree below it and right subtree above it
 * in the composite stable-sort key, and -- when dims is given -- every
 * split dim the widest extent of the node's domain box inside `bounds`.
 * Returns the number of violations (0 = canonical), -1 on bad arguments. */
int64_t cko_check_tree(int scalar, int D, const void *tree, const int64_t *index,
                       const int32_t *dims, int64_t n, const void *bounds, int nthreads);
/* violations of the k-d property alone (ties on either side allowed) */
int64_t cko_check_kd(int scalar, int D, const void *tree, const int32_t *dims, int64_t n,
                     const void *bounds, int nthreads);

/* Number of nodes in the subtree under `node` of a left-balanced tree of n
 * nodes. */
int64_t cko_subtree_size(int64_t node, int64_t n);

/* Find-closest-point.  For float trees `cutoff` is the cut-off radius and
 * eps the stack-free far-side factor; for int trees cutoff_d2_int is the
 * squared cut-off (INT64_MAX = none).  out_ids[q] = node index or -1. */
int cko_fcp(int scalar, int D, int method, const void *tree, const int32_t *dims, int64_t n,
            const void *bounds, const void *queries, int64_t nq, float cutoff, float eps,
            int64_t cutoff_d2_int, int32_t *out_ids, int64_t *visits_out, int nthreads);

/* k nearest neighbours.  out_ids/out_d2 are [nq][k]; out_d2 is float32 for
 * float trees and int64 for int trees.  Fixed lists return ascending
 * entries, heap lists return the reference's heap order.  out_ret[q] (may
 * be NULL) receives the knn() return value (max radius^2). */
int cko_knn(int scalar, int D, int method, int list_kind, int k, const void *tree,
            const int32_t *dims, int64_t n, const void *bounds, const void *queries, int64_t nq,
            float cutoff, int64_t cutoff_d2_int, int32_t *out_ids, void *out_d2, void *out_ret,
            int64_t *visits_out, int nthreads);

/* Spatial k-d tree node, byte-identical to the reference's
 * SpatialKDTree<..>::Node (cukd/spatial-kdtree.h:69-98). */
typedef struct {
  float pos;
  uint32_t offset;
  uint16_t count;
  int16_t dim;
} cko_spatial_node;

/* Deterministic spatial k-d tree build over float points.  nodes_out needs
 * room for 2*n+2 nodes, prim_ids_out for n ids.  Returns 0. */
int cko_spatial_build(int D, const float *coords, int64_t n, int leaf_threshold,
                      cko_spatial_node *nodes_out, int64_t *num_nodes, uint32_t *prim_ids_out,
                      float *bounds_out);

int cko_spatial_fcp(int D, int method, const cko_spatial_node *nodes, const uint32_t *prim_ids,
                    const float *coords, const float *bounds, const float *queries, int64_t nq,
                    float cutoff, int32_t *out_ids, int nthreads);

int cko_spatial_knn(int D, int method, int list_kind, int k, const cko_spatial_node *nodes,
                    const uint32_t *prim_ids, const float *coords, const float *bounds,
                    const float *queries, int64_t nq, float cutoff, int32_t *out_ids,
                    float *out_d2, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
