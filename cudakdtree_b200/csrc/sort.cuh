// Stable LSD radix sort of (uint32 key, uint32 value) pairs.
#pragma once

#include "common.cuh"

namespace ckb {

// Sorts keys/vals (n pairs) by the low `bits` bits of the keys, stably.
// keys2/vals2 are scratch of n entries; the result ends in keys/vals.
int radix_sort_pairs(uint32_t *keys, uint32_t *vals, uint32_t *keys2, uint32_t *vals2,
                     int64_t n, int bits, cudaStream_t st, TempArena *arena);

// Same with caller-provided scratch of radix_sort_counts(n) entries (no
// allocation: usable inside CUDA graph capture).
int64_t radix_sort_counts(int64_t n);
int radix_sort_pairs_ws(uint32_t *keys, uint32_t *vals, uint32_t *keys2, uint32_t *vals2,
                        int64_t n, int bits, uint32_t *counts, cudaStream_t st);

}  // namespace ckb
