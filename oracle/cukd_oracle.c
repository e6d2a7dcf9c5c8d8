/*
 * cukd_oracle.c -- CPU restatement of the reference k-d tree algorithms.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product library (see
 * cukd_oracle.h).  Compiled with -ffp-contract=off so float expressions
 * round exactly as the reference's non-contracted code does.
 *
 * Restated reference routines (paths relative to the reference project):
 *   left-balanced build    cukd/builder_thrust.h:414-512 (device) and
 *                          :514-601 (buildTree_host): L rounds of a stable
 *                          sort of (tag, coordinate) pairs followed by the
 *                          tag update of :175-235 / :238-345.  Because every
 *                          round is a STABLE sort, round L orders a subtree's
 *                          points by the coordinate of its split dim and
 *                          keeps the order of the previous round for ties;
 *                          the recursion below sorts each subtree's segment
 *                          stably and passes the two halves down in that
 *                          order, which reproduces the same permutation.
 *   split dims             round robin: level % D (traverse-*.h); explicit:
 *                          widest extent of the node's domain box
 *                          (box.h:112-125, ties to the higher dim), the box
 *                          being the world bounds clipped by the ancestors'
 *                          split planes (builder_common.h:180-218,
 *                          builder_thrust.h:238-306).
 *   subtree sizes          helpers.h:161-177 (ArbitraryBinaryTree).
 *   traversals             cukd_oracle_trav.inc.
 *   spatial k-d tree       cukd/spatial-kdtree.h:133-612, made deterministic
 *                          (see cko_spatial_build).
 */
#include "cukd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* floor(log2(node+1)) -- BinaryTree::levelOf (helpers.h:83-95) */
static inline int level_of(int64_t node)
{
  int l = 0;
  uint64_t v = (uint64_t)node + 1;
  while (v >>= 1) l++;
  return l;
}

int64_t cko_subtree_size(int64_t node, int64_t n)
{
  /* count the nodes of each level under `node` that exist in a tree of n */
  int64_t cnt = 0, lo = node, hi = node;
  while (lo < n) {
    int64_t last = hi < n - 1 ? hi : n - 1;
    cnt += last - lo + 1;
    lo = 2 * lo + 1;
    hi = 2 * hi + 2;
  }
  return cnt;
}

/* ===================================================================== */
/* build                                                                  */
/* ===================================================================== */

typedef struct {
  int scalar, D, explicit_dim;
  int64_t n;
  const float *cf;
  const int32_t *ci;
  int64_t *perm;
  int32_t *dims;
  int64_t *tmp; /* merge-sort scratch, n entries */
  int64_t *seg_base;
} build_ctx;

static inline int coord_less(const build_ctx *c, int64_t a, int64_t b, int dim)
{
  if (c->scalar == 0) return c->cf[a * c->D + dim] < c->cf[b * c->D + dim];
  return c->ci[a * c->D + dim] < c->ci[b * c->D + dim];
}

/* stable bottom-up merge sort of idx[0..cnt) by coordinate `dim` */
static void stable_sort(const build_ctx *c, int64_t *idx, int64_t *tmp, int64_t cnt, int dim)
{
  int64_t *src = idx, *dst = tmp;
  for (int64_t w = 1; w < cnt; w *= 2) {
    for (int64_t lo = 0; lo < cnt; lo += 2 * w) {
      int64_t mid = lo + w < cnt ? lo + w : cnt;
      int64_t hi = lo + 2 * w < cnt ? lo + 2 * w : cnt;
      int64_t i = lo, j = mid, o = lo;
      while (i < mid && j < hi) dst[o++] = coord_less(c, src[j], src[i], dim) ? src[j++] : src[i++];
      while (i < mid) dst[o++] = src[i++];
      while (j < hi) dst[o++] = src[j++];
    }
    int64_t *t = src;
    src = dst;
    dst = t;
  }
  if (src != idx) memcpy(idx, src, sizeof(int64_t) * cnt);
}

/* widest dimension of a box, ties to the higher dim (box.h:112-125) */
static int widest_f(const float *lo, const float *hi, int D)
{
  int best = 0;
  float wbest = 0.f;
  for (int d = 0; d < D; d++) {
    float w = hi[d] - lo[d];
    if (w < wbest) continue;
    wbest = w;
    best = d;
  }
  return best;
}

static int widest_i(const int32_t *lo, const int32_t *hi, int D)
{
  int best = 0;
  int32_t wbest = 0;
  for (int d = 0; d < D; d++) {
    int32_t w = (int32_t)((uint32_t)hi[d] - (uint32_t)lo[d]);
    if (w < wbest) continue;
    wbest = w;
    best = d;
  }
  return best;
}

typedef union {
  float f[16];
  int32_t i[16];
} box_u; /* lower[0..D), upper[D..2D) */

static void build_rec(const build_ctx *c, int64_t node, int64_t *seg, int64_t cnt, box_u box,
                      int level)
{
  if (cnt <= 0) return;
  const int D = c->D;
  int dim;
  if (c->explicit_dim)
    dim = c->scalar == 0 ? widest_f(box.f, box.f + D, D) : widest_i(box.i, box.i + D, D);
  else
    dim = level % D;
  int64_t *tmp = c->tmp + (seg - c->seg_base);
  stable_sort(c, seg, tmp, cnt, dim);
  const int64_t lchild = 2 * node + 1;
  const int64_t L = lchild < c->n ? cko_subtree_size(lchild, c->n) : 0;
  const int64_t pivot = seg[L];
  c->perm[node] = pivot;
  if (c->dims) c->dims[node] = dim;
  box_u lbox = box, rbox = box;
  if (c->scalar == 0) {
    lbox.f[D + dim] = c->cf[pivot * D + dim];
    rbox.f[dim] = c->cf[pivot * D + dim];
  } else {
    lbox.i[D + dim] = c->ci[pivot * D + dim];
    rbox.i[dim] = c->ci[pivot * D + dim];
  }
  if (cnt > 65536) {
#pragma omp task firstprivate(lbox)
    build_rec(c, lchild, seg, L, lbox, level + 1);
#pragma omp task firstprivate(rbox)
    build_rec(c, lchild + 1, seg + L + 1, cnt - L - 1, rbox, level + 1);
#pragma omp taskwait
  } else {
    build_rec(c, lchild, seg, L, lbox, level + 1);
    build_rec(c, lchild + 1, seg + L + 1, cnt - L - 1, rbox, level + 1);
  }
}

int cko_build(int scalar, int D, const void *coords, int64_t n, int explicit_dim,
              int64_t *perm_out, int32_t *dims_out, void *bounds_out)
{
  if (D < 1 || D > 8) return 1;
  if (explicit_dim && !bounds_out) return 2;
  if (n < 1) return 0;
  build_ctx c;
  c.scalar = scalar;
  c.D = D;
  c.explicit_dim = explicit_dim;
  c.n = n;
  c.cf = (const float *)coords;
  c.ci = (const int32_t *)coords;
  c.perm = perm_out;
  c.dims = dims_out;
  /* world bounds (builder_common.h:166-173) */
  box_u box;
  for (int d = 0; d < D; d++) {
    if (scalar == 0) {
      float lo = c.cf[d], hi = c.cf[d];
      for (int64_t i = 1; i < n; i++) {
        float v = c.cf[i * D + d];
        lo = v < lo ? v : lo;
        hi = hi < v ? v : hi;
      }
      box.f[d] = lo;
      box.f[D + d] = hi;
    } else {
      int32_t lo = c.ci[d], hi = c.ci[d];
      for (int64_t i = 1; i < n; i++) {
        int32_t v = c.ci[i * D + d];
        lo = v < lo ? v : lo;
        hi = hi < v ? v : hi;
      }
      box.i[d] = lo;
      box.i[D + d] = hi;
    }
  }
  if (bounds_out) memcpy(bounds_out, box.f, sizeof(float) * 2 * D);
  int64_t *seg = (int64_t *)malloc(sizeof(int64_t) * n);
  c.tmp = (int64_t *)malloc(sizeof(int64_t) * n);
  c.seg_base = seg;
  for (int64_t i = 0; i < n; i++) seg[i] = i;
#pragma omp parallel
#pragma omp single
  build_rec(&c, 0, seg, n, box, 0);
  free(seg);
  free(c.tmp);
  return 0;
}

/* ===================================================================== */
/* canonical-tree check (the build's defining property, at any size)      */
/* ===================================================================== */

/* The reference's builders (builder_thrust.h:414-512, :514-601) stable-sort
 * every subtree's points by the split coordinate, so inside the subtree of
 * node a they are ordered by the composite key
 *     (c[dim(a)], c[dim(parent(a))], ..., c[dim(root)], input index)
 * and a holds the point of rank leftSize(a).  With the left-balanced sizes
 * fixed, a tree is the canonical one exactly when, for every node a, every
 * point of its left subtree has a smaller composite key than a's point and
 * every point of its right subtree a larger one; with explicit dims each
 * node's dim must also be the widest extent of its domain box (the world
 * bounds clipped by the ancestors' planes, box.h:112-125).  Checking this
 * costs O(n log n) and no sort, so it scales to trees the recursive build
 * above is too slow for. */
typedef struct {
  int scalar, D;
  const float *cf;
  const int32_t *ci;
  const int64_t *index;
  const int32_t *dims;
} check_ctx;

static inline int node_dim(const check_ctx *c, int64_t a)
{
  return c->dims ? c->dims[a] : level_of(a) % c->D;
}

static inline int coord_cmp(const check_ctx *c, int64_t i, int64_t a, int d)
{
  if (c->scalar == 0) {
    const float x = c->cf[i * c->D + d], y = c->cf[a * c->D + d];
    return x < y ? -1 : (y < x ? 1 : 0);
  }
  const int32_t x = c->ci[i * c->D + d], y = c->ci[a * c->D + d];
  return x < y ? -1 : (y < x ? 1 : 0);
}

/* sign of key(i) - key(a) in node a's composite order */
static int composite_cmp(const check_ctx *c, int64_t i, int64_t a)
{
  for (int64_t anc = a;; anc = (anc - 1) / 2) {
    const int r = coord_cmp(c, i, a, node_dim(c, anc));
    if (r) return r;
    if (anc == 0) break;
  }
  return c->index[i] < c->index[a] ? -1 : (c->index[a] < c->index[i] ? 1 : 0);
}

static int64_t check_tree_impl(int scalar, int D, const void *tree, const int64_t *index,
                               const int32_t *dims, int64_t n, const void *bounds, int nthreads)
{
  if (D < 1 || D > 8 || (dims && !bounds)) return -1;
  check_ctx c = {scalar, D, (const float *)tree, (const int32_t *)tree, index, dims};
  int64_t bad = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(+ : bad) num_threads(nthreads)
  for (int64_t i = 0; i < n; i++) {
    /* ordering against every ancestor: the canonical composite order, or
       (no index) only the k-d property, ties on either side */
    int64_t path[64];
    int depth = 0;
    for (int64_t child = i; child > 0;) {
      const int64_t a = (child - 1) / 2;
      const int inLeft = child == 2 * a + 1;
      if (index) {
        const int r = composite_cmp(&c, i, a);
        if (inLeft ? r >= 0 : r <= 0) bad++;
      } else {
        const int r = coord_cmp(&c, i, a, node_dim(&c, a));
        if (inLeft ? r > 0 : r < 0) bad++;
      }
      path[depth++] = child;
      child = a;
    }
    /* explicit dims: widest extent of the domain box */
    if (dims) {
      box_u box;
      memcpy(box.f, bounds, sizeof(float) * 2 * D);
      int64_t a = 0;
      for (int l = depth - 1; l >= 0; l--) {
        const int64_t child = path[l];
        const int d = dims[a];
        if (d < 0 || d >= D) {
          bad++;
          break;
        }
        if (scalar == 0) {
          if (child == 2 * a + 1) box.f[D + d] = c.cf[a * D + d];
          else box.f[d] = c.cf[a * D + d];
        } else {
          if (child == 2 * a + 1) box.i[D + d] = c.ci[a * D + d];
          else box.i[d] = c.ci[a * D + d];
        }
        a = child;
      }
      const int want = scalar == 0 ? widest_f(box.f, box.f + D, D) : widest_i(box.i, box.i + D, D);
      if (dims[i] != want) bad++;
    }
  }
  return bad;
}

/* Violations of the canonical tree (reference buildTree_host order,
   builder_host.h): every point is on the correct side of every ancestor in
   the ancestor's composite order (its split coordinate, then its
   ancestors' split coordinates, then the input index), and explicit dims
   are the widest extent of each node's domain box. */
int64_t cko_check_tree(int scalar, int D, const void *tree, const int64_t *index,
                       const int32_t *dims, int64_t n, const void *bounds, int nthreads)
{
  if (!index) return -1;
  return check_tree_impl(scalar, D, tree, index, dims, n, bounds, nthreads);
}

/* Violations of the k-d property alone (any valid left-balanced k-d tree,
   the guarantee of the reference's builders when points share coordinates,
   testing/testBuildersSameResult.cu:96-99; checkRec of
   floatN-knn-and-fcp.cu:387-470): every point of a node's left subtree has
   split coordinate <= the node's, of its right subtree >=; explicit dims as
   above. */
int64_t cko_check_kd(int scalar, int D, const void *tree, const int32_t *dims, int64_t n,
                     const void *bounds, int nthreads)
{
  return check_tree_impl(scalar, D, tree, NULL, dims, n, bounds, nthreads);
}

/* ===================================================================== */
/* traversals                                                             */
/* ===================================================================== */

static inline uint64_t dist_bits_float(float d)
{
  uint32_t u;
  memcpy(&u, &d, 4);
  return u;
}
static inline float bits_dist_float(uint64_t b)
{
  uint32_t u = (uint32_t)b;
  float f;
  memcpy(&f, &u, 4);
  return f;
}
static inline int far_ok_float(float dimDist, float epsErr, float cullDist)
{
  return dimDist * dimDist * epsErr < cullDist;
}
static inline uint64_t dist_bits_int(int64_t d) { return (uint64_t)d; }
static inline int64_t bits_dist_int(uint64_t b) { return (int64_t)b; }
static inline int far_ok_int(int64_t dimDist, float epsErr, int64_t cullDist)
{
  (void)epsErr;
  return dimDist * dimDist < cullDist;
}

#define SFX _f
#define T float
#define DT float
#define dist_bits_f dist_bits_float
#define bits_dist_f bits_dist_float
#define far_ok_f far_ok_float
#include "cukd_oracle_trav.inc"
#undef SFX
#undef T
#undef DT

#define SFX _i
#define T int32_t
#define DT int64_t
#define dist_bits_i dist_bits_int
#define bits_dist_i bits_dist_int
#define far_ok_i far_ok_int
#include "cukd_oracle_trav.inc"
#undef SFX
#undef T
#undef DT

int cko_fcp(int scalar, int D, int method, const void *tree, const int32_t *dims, int64_t n,
            const void *bounds, const void *queries, int64_t nq, float cutoff, float eps,
            int64_t cutoff_d2_int, int32_t *out_ids, int64_t *visits_out, int nthreads)
{
  if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 256)
  for (int64_t i = 0; i < nq; i++) {
    if (scalar == 0) {
      res_f r;
      r.is_knn = 0;
      r.f.best = cutoff * cutoff; /* FCPResult::clear(sqr(cutOffRadius)) */
      r.f.id = -1;
      r.f.visits = 0;
      run_query_f(&r, method, (const float *)queries + i * D, (const float *)tree, dims, n, D,
                  (const float *)bounds, eps);
      out_ids[i] = r.f.id;
      if (visits_out) visits_out[i] = r.f.visits;
    } else {
      res_i r;
      r.is_knn = 0;
      r.f.best = cutoff_d2_int;
      r.f.id = -1;
      r.f.visits = 0;
      run_query_i(&r, method, (const int32_t *)queries + i * D, (const int32_t *)tree, dims, n,
                  D, (const int32_t *)bounds, eps);
      out_ids[i] = r.f.id;
      if (visits_out) visits_out[i] = r.f.visits;
    }
  }
  return 0;
}

int cko_knn(int scalar, int D, int method, int list_kind, int k, const void *tree,
            const int32_t *dims, int64_t n, const void *bounds, const void *queries, int64_t nq,
            float cutoff, int64_t cutoff_d2_int, int32_t *out_ids, void *out_d2, void *out_ret,
            int64_t *visits_out, int nthreads)
{
  if (k < 1 || k > 4096) return 1;
  if (nthreads <= 0) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
  {
    key_f *mf = (key_f *)malloc(sizeof(key_f) * k);
    key_i *mi = (key_i *)malloc(sizeof(key_i) * k);
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < nq; i++) {
      if (scalar == 0) {
        res_f r;
        r.is_knn = 1;
        knn_init_f(&r.kn, list_kind, k, mf, cutoff * cutoff);
        run_query_f(&r, method, (const float *)queries + i * D, (const float *)tree, dims, n, D,
                    (const float *)bounds, 0.f);
        for (int j = 0; j < k; j++) {
          out_ids[i * k + j] = (int32_t)mf[j].lo;
          ((float *)out_d2)[i * k + j] = bits_dist_float(mf[j].hi);
        }
        if (out_ret) ((float *)out_ret)[i] = knn_max_f(&r.kn);
        if (visits_out) visits_out[i] = r.kn.visits;
      } else {
        res_i r;
        r.is_knn = 1;
        knn_init_i(&r.kn, list_kind, k, mi, cutoff_d2_int);
        run_query_i(&r, method, (const int32_t *)queries + i * D, (const int32_t *)tree, dims,
                    n, D, (const int32_t *)bounds, 0.f);
        for (int j = 0; j < k; j++) {
          out_ids[i * k + j] = (int32_t)mi[j].lo;
          ((int64_t *)out_d2)[i * k + j] = (int64_t)mi[j].hi;
        }
        if (out_ret) ((int64_t *)out_ret)[i] = knn_max_i(&r.kn);
        if (visits_out) visits_out[i] = r.kn.visits;
      }
    }
    free(mf);
    free(mi);
  }
  return 0;
}

/* ===================================================================== */
/* spatial k-d tree                                                       */
/* ===================================================================== */

/* AtomicBox float encoding (spatial-kdtree.h:177-192): a monotone map of
 * floats onto int32 so that min/max can be taken on integers. */
static inline int32_t abox_encode(float f)
{
  int32_t bits;
  memcpy(&bits, &f, 4);
  if (bits & (int32_t)0x80000000) bits ^= 0x7fffffff;
  return bits;
}
static inline float abox_decode(int32_t bits)
{
  if (bits & (int32_t)0x80000000) bits ^= 0x7fffffff;
  float f;
  memcpy(&f, &bits, 4);
  return f;
}

/*
 * Level-synchronous build of spatial-kdtree.h:496-612 with its two
 * sources of nondeterminism replaced by a canonical choice:
 *   - child pairs are numbered in increasing order of their parent's node
 *     id within a pass (the reference takes them from an atomicAdd, :385);
 *   - a degenerate split (dim -1, :424-427) sends the i-th of its prims, in
 *     prim-id order, to side i&1 (the reference counts with an atomicAdd on
 *     an uninitialised counter).
 * Everything else -- the split rule, leaf rule, node 1 as an empty dummy,
 * prim ids ordered by node id and then prim id -- is the reference's.
 */
enum { NS_OPEN_BRANCH = 0, NS_OPEN_NODE = 1, NS_DONE = 2 };

typedef struct {
  int32_t lo[8], hi[8];
  uint32_t count;
  /* split */
  uint32_t offset;
  int dim;
  float pos;
  uint32_t tie;
} sp_tmp;

int cko_spatial_build(int D, const float *coords, int64_t n, int leaf_threshold,
                      cko_spatial_node *nodes_out, int64_t *num_nodes, uint32_t *prim_ids_out,
                      float *bounds_out)
{
  if (leaf_threshold == 0) leaf_threshold = 8;
  const int64_t cap = 2 * n + 2;
  sp_tmp *tn = (sp_tmp *)calloc(cap, sizeof(sp_tmp));
  uint8_t *ns = (uint8_t *)calloc(cap, 1);
  int64_t *pnode = (int64_t *)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
  uint8_t *pdone = (uint8_t *)calloc(n > 0 ? n : 1, 1);
  /* initState */
  int64_t numNodes = 2;
  ns[0] = NS_OPEN_BRANCH;
  for (int d = 0; d < D; d++) {
    tn[0].lo[d] = abox_encode(+FLT_MAX);
    tn[0].hi[d] = abox_encode(-FLT_MAX);
  }
  ns[1] = NS_DONE;
  tn[1].offset = 0;
  tn[1].count = 0;
  tn[1].dim = 0;
  tn[1].pos = 0.f;
  /* initPrims */
  for (int64_t i = 0; i < n; i++) {
    pnode[i] = 0;
    tn[0].count++;
    for (int d = 0; d < D; d++) {
      int32_t e = abox_encode(coords[i * D + d]);
      if (e < tn[0].lo[d]) tn[0].lo[d] = e;
      if (e > tn[0].hi[d]) tn[0].hi[d] = e;
    }
  }
  for (int d = 0; d < D; d++) {
    bounds_out[d] = abox_decode(tn[0].lo[d]);
    bounds_out[D + d] = abox_decode(tn[0].hi[d]);
  }
  int64_t numDone = 0;
  for (;;) {
    const int64_t nn = numNodes;
    if (nn == numDone) break;
    /* selectSplits (:316-396) */
    for (int64_t id = 0; id < nn; id++) {
      if (ns[id] == NS_DONE) continue;
      if (ns[id] == NS_OPEN_NODE) {
        ns[id] = NS_DONE;
        tn[id].count = 0;
        continue;
      }
      sp_tmp *in = &tn[id];
      if ((int)in->count <= leaf_threshold) {
        ns[id] = NS_DONE;
        in->offset = UINT32_MAX;
        in->dim = 0;
        in->pos = 0.f;
        continue;
      }
      float widestWidth = 0.f;
      int widestDim = -1;
      for (int d = 0; d < D; d++) {
        float width = abox_decode(in->hi[d]) - abox_decode(in->lo[d]);
        if (width <= widestWidth) continue;
        widestWidth = width;
        widestDim = d;
      }
      float pos = 0.f;
      if (widestDim >= 0) {
        pos = 0.5f * (abox_decode(in->lo[widestDim]) + abox_decode(in->hi[widestDim]));
        if (pos == abox_decode(in->lo[widestDim]) || pos == abox_decode(in->hi[widestDim]))
          widestDim = -1;
      }
      if (widestDim < 0) pos = abox_decode(in->lo[0]);
      in->dim = widestDim;
      in->pos = pos;
      in->tie = 0;
      in->offset = (uint32_t)numNodes;
      numNodes += 2;
      for (int side = 0; side < 2; side++) {
        sp_tmp *ch = &tn[in->offset + side];
        for (int d = 0; d < D; d++) {
          ch->lo[d] = abox_encode(+FLT_MAX);
          ch->hi[d] = abox_encode(-FLT_MAX);
        }
        ch->count = 0;
        ns[in->offset + side] = NS_OPEN_BRANCH;
      }
      ns[id] = NS_OPEN_NODE;
    }
    numDone = nn;
    /* updatePrims (:398-436), prims in id order */
    for (int64_t i = 0; i < n; i++) {
      if (pdone[i]) continue;
      const int64_t nid = pnode[i];
      if (ns[nid] == NS_DONE) {
        pdone[i] = 1;
        continue;
      }
      sp_tmp *split = &tn[nid];
      int side;
      if (split->dim == -1)
        side = (int)(split->tie++ & 1);
      else
        side = coords[i * D + split->dim] >= split->pos;
      const int64_t child = split->offset + side;
      tn[child].count++;
      for (int d = 0; d < D; d++) {
        int32_t e = abox_encode(coords[i * D + d]);
        if (e < tn[child].lo[d]) tn[child].lo[d] = e;
        if (e > tn[child].hi[d]) tn[child].hi[d] = e;
      }
      pnode[i] = child;
    }
  }
  /* stable grouping of prims by node id (:577-585), leaf offsets (:442-461) */
  int64_t *cnt = (int64_t *)calloc(numNodes + 1, sizeof(int64_t));
  for (int64_t i = 0; i < n; i++) cnt[pnode[i] + 1]++;
  for (int64_t j = 0; j < numNodes; j++) cnt[j + 1] += cnt[j];
  for (int64_t i = 0; i < n; i++) {
    int64_t at = cnt[pnode[i]]++;
    prim_ids_out[at] = (uint32_t)i;
    if ((uint32_t)at < tn[pnode[i]].offset) tn[pnode[i]].offset = (uint32_t)at;
  }
  for (int64_t j = 0; j < numNodes; j++) {
    nodes_out[j].pos = tn[j].pos;
    nodes_out[j].offset = tn[j].offset;
    nodes_out[j].count = (uint16_t)(ns[j] == NS_DONE && j != 1 ? tn[j].count : 0);
    nodes_out[j].dim = (int16_t)(tn[j].dim < 0 ? 0 : tn[j].dim);
  }
  *num_nodes = numNodes;
  free(cnt);
  free(tn);
  free(ns);
  free(pnode);
  free(pdone);
  return 0;
}

/* spatial traversals: fcp.h:256-427 and knn.h:566-646, 680-752 */
static void spatial_query(res_f *r, int method, const float *q, const cko_spatial_node *nodes,
                          const uint32_t *prim_ids, const float *coords, const float *bounds,
                          int D)
{
  float cullDist = res_init_cull_f(r);
  struct {
    int32_t node;
    float d;
    float corner[8];
  } stack[64];
  int sp = 0;
  float closest[8];
  if (method == CKO_CCT) {
    for (int d = 0; d < D; d++) {
      float v = q[d];
      v = (v < bounds[d]) ? bounds[d] : v;
      v = (bounds[D + d] < v) ? bounds[D + d] : v;
      closest[d] = v;
    }
    if (sqr_dist_f(q, closest, D) > cullDist) return;
  }
  int32_t nodeID = 0;
  cko_spatial_node node;
  for (;;) {
    for (;;) {
      node = nodes[nodeID];
      if (node.count) break;
      const float query_coord = q[node.dim];
      const int leftIsClose = query_coord < node.pos;
      const int32_t lChild = (int32_t)node.offset, rChild = lChild + 1;
      const int32_t closeChild = leftIsClose ? lChild : rChild;
      const int32_t farChild = leftIsClose ? rChild : lChild;
      if (method == CKO_CCT) {
        float farCorner[8];
        memcpy(farCorner, closest, sizeof(float) * D);
        farCorner[node.dim] = node.pos;
        if (sqr_dist_f(farCorner, q, D) < cullDist) {
          memcpy(stack[sp].corner, farCorner, sizeof(float) * D);
          stack[sp].node = farChild;
          sp++;
          if (sp >= 50) {
            if (r->is_knn) return; /* reference prints STACK OVERFLOW and returns */
            r->f.id = -1;
            return;
          }
        }
      } else {
        const float diff = query_coord - node.pos;
        const float sqrDistToPlane = diff * diff;
        if (sqrDistToPlane < cullDist) {
          stack[sp].node = farChild;
          stack[sp].d = sqrDistToPlane;
          sp++;
          if (sp >= 50) {
            if (r->is_knn) return;
            r->f.id = -1;
            return;
          }
        }
      }
      nodeID = closeChild;
    }
    for (int i = 0; i < node.count; i++) {
      const uint32_t primID = prim_ids[node.offset + i];
      const float d2 = sqr_dist_f(coords + (int64_t)primID * D, q, D);
      cullDist = res_process_f(r, (int32_t)primID, d2);
    }
    for (;;) {
      if (sp == 0) return;
      --sp;
      if (method == CKO_CCT) {
        memcpy(closest, stack[sp].corner, sizeof(float) * D);
        if (sqr_dist_f(closest, q, D) >= cullDist) continue;
      } else {
        if (stack[sp].d >= cullDist) continue;
      }
      nodeID = stack[sp].node;
      break;
    }
  }
}

int cko_spatial_fcp(int D, int method, const cko_spatial_node *nodes, const uint32_t *prim_ids,
                    const float *coords, const float *bounds, const float *queries, int64_t nq,
                    float cutoff, int32_t *out_ids, int nthreads)
{
  if (nthreads <= 0) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 256)
  for (int64_t i = 0; i < nq; i++) {
    res_f r;
    r.is_knn = 0;
    r.f.best = cutoff * cutoff;
    r.f.id = -1;
    r.f.visits = 0;
    spatial_query(&r, method, queries + i * D, nodes, prim_ids, coords, bounds, D);
    out_ids[i] = r.f.id;
  }
  return 0;
}

int cko_spatial_knn(int D, int method, int list_kind, int k, const cko_spatial_node *nodes,
                    const uint32_t *prim_ids, const float *coords, const float *bounds,
                    const float *queries, int64_t nq, float cutoff, int32_t *out_ids,
                    float *out_d2, int nthreads)
{
  if (nthreads <= 0) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
  {
    key_f *mf = (key_f *)malloc(sizeof(key_f) * k);
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < nq; i++) {
      res_f r;
      r.is_knn = 1;
      knn_init_f(&r.kn, list_kind, k, mf, cutoff * cutoff);
      spatial_query(&r, method, queries + i * D, nodes, prim_ids, coords, bounds, D);
      for (int j = 0; j < k; j++) {
        out_ids[i * k + j] = (int32_t)mf[j].lo;
        out_d2[i * k + j] = bits_dist_float(mf[j].hi);
      }
    }
    free(mf);
  }
  return 0;
}
