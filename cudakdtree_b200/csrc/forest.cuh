// Forest builds: many independent clouds stored one after another in one
// record array, each built into its own left-balanced tree in place (float
// coordinates, round-robin split dims).  The host plans the work once from
// the cloud sizes (batched.cu); the device side (build.cu) runs the same
// selection builder as a single tree, with every level's kernels and the
// subtree phase covering all clouds at once.
#pragma once

#include "common.cuh"

namespace ckb {

// one tile class of the subtree phase: work items (cloud, subtree index on
// level `level`), largest first, taken from `counter` by persistent CTAs
struct ForestSubtrees {
  int items;
  const int32_t *cloud, *local;
  const int8_t *level;
  const int64_t *cloudBase, *cloudN;
  int *counter;
};

// one top-down level: per work item its cloud, its subtree index on the
// level and its first child's work item on the next level (-1 when the
// children go to the subtree phase)
struct ForestLevel {
  int items, nb, chunksPerSeg;
  int64_t maxSeg;  // points of the level's largest subtree
  const int32_t *cloud, *local, *child;
};

// geometry of the global (top-down) levels, shared by the single-tree
// builder and the forest plan: points per CTA of the level kernels, and the
// histogram bins of a level whose largest subtree holds maxSeg points
constexpr int kLevelChunk = 4096;
int level_bins(int64_t maxSeg);

constexpr int kForestMaxLevels = 32;
constexpr int kForestTiles[3] = {512, 1024, 2048};

struct ForestBuild {
  int D = 3;
  int64_t total = 0;      // records over all clouds
  int64_t numClouds = 0;
  const int64_t *cloudBase = nullptr, *cloudN = nullptr;  // device, [numClouds]
  const int32_t *rootItem = nullptr;  // device, [numClouds]: level-0 work item or -1
  int numLevels = 0;
  ForestLevel level[kForestMaxLevels];
  ForestSubtrees sub[3];  // tile classes kForestTiles[0..2]
  int subGrid[3] = {0, 0, 0};
  void *ws = nullptr;     // device workspace (forest_workspace_create)
};

// sizes of the workspace: records, largest level, largest histogram
int forest_workspace_create(ForestBuild *f, int64_t maxItems, int64_t histCap);
void forest_workspace_destroy(ForestBuild *f);
// resident CTAs per SM of the subtree kernel of tile class c
int forest_subtree_occupancy(int D, int c);
// builds every cloud of `pts` (float[total][D]) in place; per-cloud boxes
// (float[numClouds][2][D], lower then upper) into `boundsOut` when given.
// With `side` streams the tile classes run as concurrent branches.
int forest_build(const ForestBuild &f, float *pts, float *boundsOut, cudaStream_t st,
                 cudaStream_t side[3], cudaEvent_t ev[4]);

}  // namespace ckb
