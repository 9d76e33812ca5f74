// ys_scan.cu -- device-wide exclusive prefix sum of uint32 (CSR offsets).
#include "ys_common.cuh"
#include "ys_scan.cuh"

namespace ys {

static constexpr int SCAN_THREADS = 1024;
static constexpr int SCAN_ITEMS = 4;
static constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile(u32* __restrict__ data, u32 n, u32* __restrict__ sums) {
    __shared__ u32 warpSums[32];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const u32 base = blockIdx.x * (u32)SCAN_TILE + (u32)tid * SCAN_ITEMS;
    u32 v[SCAN_ITEMS];
    u32 s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) { v[k] = (base + k < n) ? data[base + k] : 0u; s += v[k]; }
    u32 x = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) { u32 y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) warpSums[w] = x;
    __syncthreads();
    if (w == 0) {
        u32 t = warpSums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) { u32 y = __shfl_up_sync(0xffffffffu, t, o); if (lane >= o) t += y; }
        warpSums[lane] = t;
    }
    __syncthreads();
    u32 run = x - s + (w > 0 ? warpSums[w - 1] : 0u);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) data[base + k] = run;
        run += v[k];
    }
    if (tid == SCAN_THREADS - 1 && sums) sums[blockIdx.x] = run;
}

__global__ void k_scan_add(u32* __restrict__ data, u32 n, const u32* __restrict__ offs) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) data[i] += offs[i / SCAN_TILE];
}

size_t scan_scratch_bytes(u32 n) {
    size_t total = 0;
    while (n > (u32)SCAN_TILE) {
        n = (u32)ceil_div(n, SCAN_TILE);
        total += (size_t)n * 4 + 256;
    }
    return total + 256;
}

cudaError_t exclusive_scan(u32* data, u32 n, void* scratch, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    u32 tiles = (u32)ceil_div(n, SCAN_TILE);
    if (tiles == 1) {
        k_scan_tile<<<1, SCAN_THREADS, 0, s>>>(data, n, nullptr);
        return cudaGetLastError();
    }
    u32* sums = (u32*)scratch;
    char* next = (char*)scratch + (((size_t)tiles * 4 + 255) / 256) * 256;
    k_scan_tile<<<tiles, SCAN_THREADS, 0, s>>>(data, n, sums);
    cudaError_t e = exclusive_scan(sums, tiles, next, s);
    if (e != cudaSuccess) return e;
    k_scan_add<<<ceil_div(n, 256), 256, 0, s>>>(data, n, sums);
    return cudaGetLastError();
}

}  // namespace ys
