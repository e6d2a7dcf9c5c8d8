// Device-wide exclusive scan of uint32 values (three launches: per-block
// totals, scan of the totals, per-block scan with carry-in).
#pragma once

#include "common.cuh"

namespace ckb {

// out[i] = sum(in[0..i)); *total (optional, device) = sum(in[0..n)).
// in and out may alias.  Temporaries come from `arena`.
int exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total,
                       cudaStream_t st, TempArena *arena);

}  // namespace ckb
