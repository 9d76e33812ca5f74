// ys_sort.cu -- stable LSD radix sort of (uint32 key, uint32 value) pairs.
//
// Restates the reference RadixSorter (spatial_hash.hpp:48-70,
// radixsort.metal:21-111): 8-bit digits, least significant first, stable, the
// value carried with its key.  Because the sort is stable and the values enter
// in index order, the output is the unique (key, original index) order, so it
// is bit-identical to the CPU twin radixSortCPU (bvh.hpp:723-765).
//
// B200 design, per pass (3 launches):
//   upsweep  -- each 256-thread CTA owns a tile of TILE keys and builds a
//               256-bin digit histogram from per-warp shared histograms;
//   scan     -- one CTA per digit scans that digit's column of tile counts;
//               digit bases come from a 256-entry scan done redundantly by
//               every scatter CTA (256 loads, no extra launch);
//   scatter  -- the tile is walked in 256-key rounds in index order; a key's
//               stable rank = running count of its digit in this tile + keys
//               with the same digit in earlier warps of the round (shared
//               table) + lower lanes of its own warp with the same digit
//               (match mask popcount).  Keys go to that rank in a shared
//               copy of the tile, ordered by digit, which is then written
//               out in order: a digit's run is contiguous in the output, so
//               the stores coalesce.
#include "ys_common.cuh"
#include "ys_sort.cuh"

namespace ys {

static constexpr int SORT_THREADS = 256;
static constexpr int SORT_ITEMS = 16;
static constexpr int TILE = SORT_THREADS * SORT_ITEMS;  // 4096 keys per CTA

// hist layout: digit-major, hist[d * numTiles + tile].
// Per-warp histograms in shared memory (plain shared atomics; a warp's lanes
// with the same digit serialise on one address, which is cheaper here than a
// match per key), summed per digit at the end.  Keys are read four at a time.
__global__ void __launch_bounds__(SORT_THREADS) k_sort_upsweep(const u32* __restrict__ keys, u32 n, int shift,
                                                               u32* __restrict__ hist, u32 numTiles) {
    constexpr int W = SORT_THREADS / 32;
    __shared__ u32 h[W][256];
    const int tid = threadIdx.x, w = tid >> 5;
    for (int k = tid; k < W * 256; k += SORT_THREADS) (&h[0][0])[k] = 0;
    __syncthreads();
    const u32 base = blockIdx.x * (u32)TILE;
    u32* hw = h[w];
    if (base + TILE <= n && (reinterpret_cast<uintptr_t>(keys) & 15u) == 0) {
        const uint4* k4 = reinterpret_cast<const uint4*>(keys + base);
#pragma unroll
        for (int r = 0; r < SORT_ITEMS / 4; ++r) {
            const uint4 q = k4[r * SORT_THREADS + tid];
            atomicAdd(&hw[(q.x >> shift) & 255u], 1u);
            atomicAdd(&hw[(q.y >> shift) & 255u], 1u);
            atomicAdd(&hw[(q.z >> shift) & 255u], 1u);
            atomicAdd(&hw[(q.w >> shift) & 255u], 1u);
        }
    } else {
        for (int r = 0; r < SORT_ITEMS; ++r) {
            const u32 i = base + (u32)r * SORT_THREADS + tid;
            if (i < n) atomicAdd(&hw[(keys[i] >> shift) & 255u], 1u);
        }
    }
    __syncthreads();
    u32 sum = 0;
#pragma unroll
    for (int ww = 0; ww < W; ++ww) sum += h[ww][tid];
    hist[(u32)tid * numTiles + blockIdx.x] = sum;
}

// One CTA per digit: exclusive scan of hist[d, 0..numTiles) in place; total
// of digit d to totals[d].
__global__ void __launch_bounds__(1024) k_sort_scan(u32* __restrict__ hist, u32 numTiles, u32* __restrict__ totals) {
    __shared__ u32 warpSums[32];
    __shared__ u32 carry;
    const int d = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    u32* row = hist + (u64)d * numTiles;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (u32 base = 0; base < numTiles; base += 1024) {
        u32 i = base + tid;
        u32 v = (i < numTiles) ? row[i] : 0u;
        u32 x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) { u32 y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
        if (lane == 31) warpSums[w] = x;
        __syncthreads();
        if (w == 0) {
            u32 s = warpSums[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) { u32 y = __shfl_up_sync(0xffffffffu, s, o); if (lane >= o) s += y; }
            warpSums[lane] = s;
        }
        __syncthreads();
        u32 incl = x + (w > 0 ? warpSums[w - 1] : 0u) + carry;
        if (i < numTiles) row[i] = incl - v;
        __syncthreads();
        if (tid == 1023) carry = incl;
        __syncthreads();
    }
    if (tid == 0) totals[d] = carry;
}

__global__ void __launch_bounds__(SORT_THREADS) k_sort_scatter(const u32* __restrict__ kin, const u32* __restrict__ vin,
                                                               u32* __restrict__ kout, u32* __restrict__ vout, u32 n,
                                                               int shift, const u32* __restrict__ hist, u32 numTiles,
                                                               const u32* __restrict__ totals) {
    constexpr int W = SORT_THREADS / 32;
    __shared__ u32 base[256];         // global start of each digit for this tile
    __shared__ u32 lofs[256];         // start of each digit within the tile
    __shared__ u32 running[2][256];   // keys of each digit already placed by this tile (by round parity)
    __shared__ unsigned short wcnt[2][W][256];  // per-warp digit counts of a round (<= 32; by round parity)
    __shared__ u32 scanTmp[256];
    __shared__ u32 sk[TILE], sv[TILE];  // the tile, stably ordered by digit
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const u32 tileBase = blockIdx.x * (u32)TILE;
    const u32 tileCount = min((u32)TILE, n - tileBase);

    // digit bases: exclusive scan of totals (every CTA does it; 256 entries)
    const u32 t = totals[tid];
    scanTmp[tid] = t;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
        u32 add = (tid >= o) ? scanTmp[tid - o] : 0u;
        __syncthreads();
        scanTmp[tid] += add;
        __syncthreads();
    }
    // hist holds, per digit, the keys of that digit in earlier tiles: this
    // tile's own count is the difference to the next tile (or to the total)
    const u32 before_tiles = hist[(u32)tid * numTiles + blockIdx.x];
    const u32 mine = (blockIdx.x + 1 < numTiles ? hist[(u32)tid * numTiles + blockIdx.x + 1] : t) - before_tiles;
    base[tid] = scanTmp[tid] - t + before_tiles;
    running[0][tid] = 0;
    for (int k = tid; k < W * 256; k += SORT_THREADS) (&wcnt[0][0][0])[k] = 0;
    __syncthreads();
    scanTmp[tid] = mine;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
        u32 add = (tid >= o) ? scanTmp[tid - o] : 0u;
        __syncthreads();
        scanTmp[tid] += add;
        __syncthreads();
    }
    lofs[tid] = scanTmp[tid] - mine;
    __syncthreads();

    // the thread's keys and values of all rounds, loaded at once (one memory
    // latency for the tile instead of one per round)
    u32 kr[SORT_ITEMS], vr[SORT_ITEMS];
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        const u32 i = tileBase + (u32)r * SORT_THREADS + tid;
        kr[r] = i < n ? __ldcs(kin + i) : 0u;
        vr[r] = i < n ? __ldcs(vin + i) : 0u;
    }
    // stable rank of every key within the tile, into shared memory.  Round r
    // counts into wcnt[r & 1] and reads running[r & 1]; it clears the other
    // counts (last read in round r - 1, before its second barrier) and
    // writes the next running counts, so a round takes two barriers.
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; ++r) {
        const int b = r & 1;
        for (int k = tid; k < W * 256; k += SORT_THREADS) (&wcnt[b ^ 1][0][0])[k] = 0;
        const u32 i = tileBase + (u32)r * SORT_THREADS + tid;
        const bool valid = i < n;
        u32 key = 0, val = 0, d = 256u + lane;
        if (valid) { key = kr[r]; val = vr[r]; d = (key >> shift) & 255u; }
        const u32 peers = __match_any_sync(0xffffffffu, d);
        const u32 lower = __popc(peers & ((1u << lane) - 1u));
        const int leader = __ffs(peers) - 1;
        if (valid && lane == leader) wcnt[b][w][d] = (unsigned short)__popc(peers);
        __syncthreads();
        if (valid) {
            u32 before = 0;
            for (int ww = 0; ww < w; ++ww) before += wcnt[b][ww][d];
            const u32 p = lofs[d] + running[b][d] + before + lower;
            sk[p] = key;
            sv[p] = val;
        }
        // the next round's running counts: this round's totals added
        {
            u32 s = 0;
#pragma unroll
            for (int ww = 0; ww < W; ++ww) s += wcnt[b][ww][tid];
            running[b ^ 1][tid] = running[b][tid] + s;
        }
        __syncthreads();
    }
    // write out in tile order: a digit's keys are consecutive here and in the
    // output, so neighbouring threads store to neighbouring addresses
    for (u32 q = (u32)tid; q < tileCount; q += SORT_THREADS) {
        const u32 key = sk[q];
        const u32 d = (key >> shift) & 255u;
        const u32 dst = base[d] + (q - lofs[d]);
        kout[dst] = key;
        vout[dst] = sv[q];
    }
}

size_t sort_scratch_bytes(u32 n) {
    u32 tiles = (u32)ceil_div(n > 0 ? n : 1, TILE);
    return (size_t)256 * tiles * 4 + 256 * 4 + (size_t)2 * n * 4;
}

// Sort keys/vals in place.  scratch must hold sort_scratch_bytes(n) bytes.
cudaError_t radix_sort_pairs(u32* keys, u32* vals, u32 n, void* scratch, int beginBit, int endBit, cudaStream_t s) {
    if (n <= 1) return cudaSuccess;
    u32 tiles = (u32)ceil_div(n, TILE);
    u32* hist = (u32*)scratch;
    u32* totals = hist + (size_t)256 * tiles;
    u32* k2 = totals + 256;
    u32* v2 = k2 + n;
    u32 *ki = keys, *vi = vals, *ko = k2, *vo = v2;
    for (int shift = beginBit; shift < endBit; shift += 8) {
        k_sort_upsweep<<<tiles, SORT_THREADS, 0, s>>>(ki, n, shift, hist, tiles);
        k_sort_scan<<<256, 1024, 0, s>>>(hist, tiles, totals);
        k_sort_scatter<<<tiles, SORT_THREADS, 0, s>>>(ki, vi, ko, vo, n, shift, hist, tiles, totals);
        u32* tk = ki; ki = ko; ko = tk;
        u32* tv = vi; vi = vo; vo = tv;
    }
    if (ki != keys) {
        cudaMemcpyAsync(keys, ki, (size_t)n * 4, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(vals, vi, (size_t)n * 4, cudaMemcpyDeviceToDevice, s);
    }
    return cudaGetLastError();
}

}  // namespace ys

// ---------------------------------------------------------------------------
// Sort with no allocation at all, for callers that cannot call cudaMalloc:
// code that runs inside a CUDA-graph capture or an allocation-free real-time
// loop, hosts whose device memory is owned by another allocator (a game
// engine's or a framework's pool), and plugins that must not grow the
// process's device footprint behind the host's back.  The scratch lives in a
// file-scope __device__ array of fixed size, reserved on every GPU that loads
// this library until the process exits.
#include <mutex>
#include <string>

#include "ysim_b200.h"

namespace ys {
ys_status fail(ys_status code, const std::string& msg);

static constexpr u32 NOALLOC_MAX_PAIRS = 1u << 20;  // 1,048,576 pairs
static constexpr size_t NOALLOC_SCRATCH_BYTES =
    (size_t)256 * (NOALLOC_MAX_PAIRS / TILE) * 4 + 256 * 4 + (size_t)2 * NOALLOC_MAX_PAIRS * 4;  // 8,651,776 B
static __device__ __align__(256) unsigned char g_noalloc_sort_scratch[NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mutex;
static void* g_noalloc_addr[64] = {};
static unsigned long long g_noalloc_ctx[64] = {};  // context the address was looked up in

// Unique id of the calling thread's current CUDA context (cuCtxGetId, through
// the runtime's driver entry points, so the library needs no -lcuda).  A
// device reset destroys the device's primary context and the next one gets a
// new id, which is how a cached symbol address is known to be stale.
static bool current_context_id(unsigned long long* id) {
    typedef int (*GetCurrent)(void**);
    typedef int (*GetId)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", (void**)&get_current, cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess)
            get_current = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", (void**)&get_id, cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess)
            get_id = nullptr;
    }
    void* ctx = nullptr;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx) return false;
    return get_id(ctx, id) == 0;
}
}  // namespace ys

extern "C" ys_status ys_radix_sort_pairs_noalloc(uint32_t* d_keys, uint32_t* d_vals, uint32_t n, void* stream) {
    using namespace ys;
    if (n > NOALLOC_MAX_PAIRS)
        return fail(YS_ERR_CAPACITY, "ys_radix_sort_pairs_noalloc: n = " + std::to_string(n) +
                                         " exceeds the fixed scratch capacity of " +
                                         std::to_string(NOALLOC_MAX_PAIRS) + " pairs");
    if (n > 1 && (!d_keys || !d_vals)) return fail(YS_ERR_BAD_ARG, "ys_radix_sort_pairs_noalloc: null array");
    if (n <= 1) return YS_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(YS_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return fail(YS_ERR_BAD_ARG, "device index out of range");
    void* scratch = nullptr;
    {
        // first call on this device (or in a new context of it, after a
        // device reset): look up the device address of the array (its
        // host-side name is only a stand-in and must never reach a kernel)
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        unsigned long long ctx = 0;
        const bool known = current_context_id(&ctx);
        if (!g_noalloc_addr[dev] || (known && ctx != g_noalloc_ctx[dev])) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_sort_scratch);
            if (e != cudaSuccess)
                return fail(YS_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_noalloc_addr[dev] = p;
            g_noalloc_ctx[dev] = current_context_id(&ctx) ? ctx : 0;
        }
        scratch = g_noalloc_addr[dev];
    }
    // Every pass overwrites the whole histogram / totals region it reads and
    // the ping-pong halves are written before they are read, so nothing left
    // by an earlier call needs clearing.  4 passes end in the caller's arrays.
    e = radix_sort_pairs(d_keys, d_vals, n, scratch, 0, 32, (cudaStream_t)stream);
    if (e != cudaSuccess) return fail(YS_ERR_CUDA, std::string("radix sort: ") + cudaGetErrorString(e));
    return YS_OK;
}
