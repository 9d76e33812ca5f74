// ys_scan.cuh -- device-wide exclusive prefix sum of uint32.
#pragma once
#include "ys_common.cuh"

namespace ys {
size_t scan_scratch_bytes(u32 n);
// In-place exclusive scan of data[0, n); scratch of scan_scratch_bytes(n).
cudaError_t exclusive_scan(u32* data, u32 n, void* scratch, cudaStream_t s);
}  // namespace ys
