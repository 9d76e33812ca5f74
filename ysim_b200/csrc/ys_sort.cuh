// ys_sort.cuh -- stable LSD radix sort of (key, value) uint32 pairs.
#pragma once
#include "ys_common.cuh"

namespace ys {
// Bytes of scratch radix_sort_pairs needs for n pairs.
size_t sort_scratch_bytes(u32 n);
// Stable sort by key bits [beginBit, endBit) in 8-bit passes; in place.
cudaError_t radix_sort_pairs(u32* keys, u32* vals, u32 n, void* scratch, int beginBit, int endBit, cudaStream_t s);
}  // namespace ys
