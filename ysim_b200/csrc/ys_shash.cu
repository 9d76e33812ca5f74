// ys_shash.cu -- uniform-grid spatial-hash broad phase, point vs triangle.
//
// The reference's spatial-hash broad phases (SpatialHashing<METAL>,
// spatial_hash.hpp:880-960; CpuSpatialHash, spatial_hash.hpp:1547-2016) bin
// primitives into grid cells, probe the cells a query overlaps, and keep the
// candidates that pass an AABB precull.  This is the B200 form for the
// collision microbenchmark: triangles are binned by their AABB into every
// cell it overlaps (cell edge = 2h by default), a radix sort of (bucket,
// triangle) groups the entries by hash bucket, and each query point probes
// the <= 8 cells its box [p - h, p + h] overlaps.  A bucket may hold entries
// of other cells (hash collisions): an entry counts for a probed cell only
// when the cell lies in its triangle's cell range, and the (stable) sort
// keeps the entries of one triangle in one bucket side by side, so a
// triangle with two cells in the bucket is seen once.  A pair (p, t) is
// emitted only from the cell that is the component-wise max of the two cell
// ranges' lower corners, so each overlapping pair comes out exactly once,
// and the candidate set equals the LBVH point query's (queryPoints,
// bvh.metal:1394-1412) under the same inclusive AABB test.
//
// The bucket of a cell is its Morton code within its block of 1024^3 cells
// (xor a hash of the block), so cells near each other have buckets near each
// other: queries taken in Morton order of their points read the bucket
// table, the sorted keys and the triangle list in nearly sequential runs
// instead of one random sector per probed cell.
//
// Build: k_sh_bound (tri boxes, order keys) -> radix sort (the internal
// order) -> k_sh_order (boxes in that order, entry counts) -> exclusive scan
// -> k_sh_emit (bucket, internal triangle) -> radix sort -> k_sh_mark (first
// slot of each bucket).  Triangles spanning more than MAX_CELLS cells go to a short
// overflow list that every query tests directly.
#include <algorithm>
#include <string>

#include "ys_common.cuh"
#include "ys_lbvh.cuh"
#include "ys_scan.cuh"
#include "ys_sort.cuh"
#include "ysim_b200.h"

namespace ys {
ys_status fail(ys_status code, const std::string& msg);

static constexpr u32 MAX_CELLS = 4096;  // larger boxes go to the overflow list, tested by every query

__device__ __forceinline__ u32 cell_bucket(int x, int y, int z, u32 mask) {
    const u32 m = (expand_bits((u32)x & 1023u) << 2) | (expand_bits((u32)y & 1023u) << 1) | expand_bits((u32)z & 1023u);
    // the block (floor division by 1024), hashed with Teschner et al. 2003's
    // spatial-hash primes
    const u32 blk = ((u32)(x >> 10) * 73856093u) ^ ((u32)(y >> 10) * 19349663u) ^ ((u32)(z >> 10) * 83492791u);
    return (m ^ blk) & mask;
}

struct ShBox { float4 mn, mx; };  // a triangle's box (w unused): 32 B, one sector

__device__ __forceinline__ void cell_range(const ShBox& r, float inv, int lo[3], int hi[3]) {
    lo[0] = (int)floorf(r.mn.x * inv); lo[1] = (int)floorf(r.mn.y * inv); lo[2] = (int)floorf(r.mn.z * inv);
    hi[0] = (int)floorf(r.mx.x * inv); hi[1] = (int)floorf(r.mx.y * inv); hi[2] = (int)floorf(r.mx.z * inv);
}

// Triangle boxes, and the key that orders the triangles internally: the
// bucket code of the first cell of each box (unmasked), so that the
// triangles of one cell and of neighbouring cells sit side by side.
__global__ void k_sh_bound(const float* __restrict__ x, const u32* __restrict__ F, u32 nF, float inv,
                           ShBox* __restrict__ tris, u32* __restrict__ key, u32* __restrict__ idx) {
    u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nF) return;
    f3 a = ldp(x, F[3 * t]), b = ldp(x, F[3 * t + 1]), c = ldp(x, F[3 * t + 2]);
    f3 lo = vmin(vmin(a, b), c), hi = vmax(vmax(a, b), c);  // leaf box (buildLeaf_Tri)
    ShBox r;
    r.mn = make_float4(lo.x, lo.y, lo.z, 0.f);
    r.mx = make_float4(hi.x, hi.y, hi.z, 0.f);
    int l[3], h[3];
    cell_range(r, inv, l, h);
    tris[t] = r;
    key[t] = cell_bucket(l[0], l[1], l[2], 0xFFFFFFFFu);
    idx[t] = t;
}

// Internal triangle i is triangle idx[i] (after the sort by key): its box in
// internal order and its entry count (0: spans more than MAX_CELLS cells).
__global__ void k_sh_order(const ShBox* __restrict__ tris, const u32* __restrict__ idx, u32 nF, float inv,
                           ShBox* __restrict__ sbox, u32* __restrict__ counts) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nF) return;
    const ShBox r = tris[idx[i]];
    int l[3], h[3];
    cell_range(r, inv, l, h);
    unsigned long long cells = 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) cells *= (unsigned long long)(h[k] - l[k] + 1);
    sbox[i] = r;
    counts[i] = cells <= MAX_CELLS ? (u32)cells : 0u;
}

// Entries of 32 triangles per warp: the warp walks their concatenated
// entries (contiguous in the output, the counts being scanned), lane by
// entry, each lane finding its triangle by a search over the lanes' first
// entries; cell ordinal o of a triangle is cell (x, y, z) with x fastest.
// A triangle's loop of 1 to MAX_CELLS cells no longer holds its warp.
__global__ void k_sh_emit(const ShBox* __restrict__ tris, const u32* __restrict__ off, u32 nF, float inv, u32 mask,
                          u32* __restrict__ ebucket, u32* __restrict__ etri, u32* __restrict__ big,
                          u32* __restrict__ nbig) {
    const u32 lane = threadIdx.x & 31u;
    const u32 t0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
    if (t0 >= nF) return;  // whole warps
    const u32 t = t0 + lane;
    const u32 tEnd = min(t0 + 32u, nF);
    const u32 start = off[t0], total = off[tEnd] - start;
    int lo[3] = {0, 0, 0}, hi[3] = {-1, -1, -1};
    u32 rel = total;  // this lane's first entry, relative to the warp's
    if (t < nF) {
        const u32 base = off[t], end = off[t + 1];
        rel = base - start;
        if (base == end) {  // oversized: tested by every query
            const u32 i = atomicAdd(nbig, 1u);
            big[i] = t;
        } else {
            cell_range(tris[t], inv, lo, hi);
        }
    }
    for (u32 e0 = 0; e0 < total; e0 += 32u) {
        const u32 e = e0 + lane;
        // the last lane whose first entry is <= e (first entries are non-decreasing)
        u32 j = 0;
#pragma unroll
        for (u32 step = 16; step >= 1; step >>= 1) {
            const u32 r = __shfl_sync(0xFFFFFFFFu, rel, (int)(j + step));
            if (r <= e) j += step;
        }
        const u32 rj = __shfl_sync(0xFFFFFFFFu, rel, (int)j);
        const int lx = __shfl_sync(0xFFFFFFFFu, lo[0], (int)j), ly = __shfl_sync(0xFFFFFFFFu, lo[1], (int)j),
                  lz = __shfl_sync(0xFFFFFFFFu, lo[2], (int)j);
        const int hx = __shfl_sync(0xFFFFFFFFu, hi[0], (int)j), hy = __shfl_sync(0xFFFFFFFFu, hi[1], (int)j);
        if (e < total) {
            const u32 o = e - rj, nx = (u32)(hx - lx + 1), ny = (u32)(hy - ly + 1);
            const u32 q = o / nx;
            ebucket[start + e] = cell_bucket(lx + (int)(o - q * nx), ly + (int)(q % ny), lz + (int)(q / ny), mask);
            etri[start + e] = t0 + j;
        }
    }
}

// Each bucket's run in the sorted keys as one word: first slot << 4 | run
// length, the length saturating at RUN_LONG (a query then finds the end
// where the key changes).  Buckets with no entry keep 0xFFFFFFFF; first
// slots stay below 2^28 - 1 (MAX_ENTRIES).
static constexpr u32 RUN_LONG = 15;
static constexpr u32 MAX_ENTRIES = (1u << 28) - 2;
__global__ void k_sh_mark(const u32* __restrict__ skey, u32 nE, u32* __restrict__ bstart) {
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nE) return;
    const u32 b = skey[k];
    if (k != 0 && skey[k - 1] == b) return;
    u32 c = 1;
    while (c < RUN_LONG && k + c < nE && skey[k + c] == b) ++c;
    bstart[b] = (k << 4) | c;
}

__device__ __forceinline__ bool box_hit(f3 qmn, f3 qmx, const ShBox& r) {
    if (qmx.x < r.mn.x || qmn.x > r.mx.x) return false;
    if (qmx.y < r.mn.y || qmn.y > r.mx.y) return false;
    if (qmx.z < r.mn.z || qmn.z > r.mx.z) return false;
    return true;
}

__global__ void __launch_bounds__(128) k_sh_query(const float* __restrict__ qx, u32 nQ, float m, float inv, u32 mask,
                                                  const ShBox* __restrict__ tris, const u32* __restrict__ tid,
                                                  const u32* __restrict__ bstart, const u32* __restrict__ skey, u32 nE,
                                                  const u32* __restrict__ sorted, const u32* __restrict__ big,
                                                  const u32* __restrict__ nbig, const u32* __restrict__ order,
                                                  u32* __restrict__ pairs, u64 cap, unsigned long long* count) {
    const u32 k0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (k0 >= nQ) return;
    const u32 p = order ? order[k0] : k0;  // the point of this thread (Morton order for large query sets)
    const f3 q = ldp(qx, p);
    const f3 qmn = q - mk(m, m, m), qmx = q + mk(m, m, m);  // queryPoints box
    const float a3[3] = {qmn.x, qmn.y, qmn.z}, b3[3] = {qmx.x, qmx.y, qmx.z};
    int lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo[k] = (int)floorf(a3[k] * inv);
        hi[k] = (int)floorf(b3[k] * inv);
    }
    // the lanes appending together reserve their slots with one atomic
    auto emit = [&](u32 t) {
        const unsigned act = __activemask();
        const u32 lane = threadIdx.x & 31u, leader = (u32)__ffs(act) - 1u;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(act));
        base = __shfl_sync(act, base, (int)leader);
        const unsigned long long i = base + (u32)__popc(act & ((1u << lane) - 1u));
        if (i < cap) { pairs[2 * i] = p; pairs[2 * i + 1] = tid[t]; }
    };
    for (int z = lo[2]; z <= hi[2]; ++z)
        for (int y = lo[1]; y <= hi[1]; ++y)
            for (int xx = lo[0]; xx <= hi[0]; ++xx) {
                const u32 b = cell_bucket(xx, y, z, mask);
                const u32 e = bstart[b];
                if (e == 0xFFFFFFFFu) continue;  // empty bucket
                // a short run is read by its length, a long one up to where the key changes
                const u32 k0 = e >> 4, len = e & 15u;
                u32 prev = 0xFFFFFFFFu;
                for (u32 k = k0; k < nE && (len < RUN_LONG ? k < k0 + len : skey[k] == b); ++k) {
                    const u32 t = sorted[k];
                    if (t == prev) continue;  // the same triangle, for another of its cells
                    prev = t;
                    const ShBox r = tris[t];
                    int rl[3], rh[3];
                    cell_range(r, inv, rl, rh);
                    // this cell is one of the triangle's (not another cell
                    // hashing to the same bucket)
                    if (xx < rl[0] || xx > rh[0] || y < rl[1] || y > rh[1] || z < rl[2] || z > rh[2]) continue;
                    // emit from the first common cell only
                    if (xx != max(lo[0], rl[0]) || y != max(lo[1], rl[1]) || z != max(lo[2], rl[2])) continue;
                    if (box_hit(qmn, qmx, r)) emit(t);
                }
            }
    const u32 nb = *nbig;
    for (u32 k = 0; k < nb; ++k) {
        const u32 t = big[k];
        if (box_hit(qmn, qmx, tris[t])) emit(t);
    }
}

}  // namespace ys

using namespace ys;

struct ys_shash {
    int device = 0;
    cudaStream_t stream = nullptr;
    u32 maxTris = 0, maxEntries = 0, nF = 0, mask = 0, nE = 0;
    u32 tableCap = 0;  // buckets allocated (power of two); each build uses 2 nE rounded up, at most this
    float cell = 0.f, inv = 0.f;
    // triangle boxes in the caller's order and in the internal order (by the
    // bucket code of each box's first cell), the key of that order and the
    // caller's id of each internal triangle
    ShBox *tris = nullptr, *sbox = nullptr;
    u32 *tkey = nullptr, *tid = nullptr;
    // entries: bucket and internal triangle, sorted in place by the build
    // into the key and the triangle of each sorted slot
    u32 *counts = nullptr, *ebucket = nullptr, *etri = nullptr, *bstart = nullptr, *big = nullptr, *nbig = nullptr;
    void* sortScratch = nullptr;
    void* scan = nullptr;
    QueryOrder qorder;  // Morton order of large query sets
};

#define YS_CK3(call)                                                                                   \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(YS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

extern "C" {

ys_status ys_shash_create(ys_shash** out, uint32_t max_tris, uint32_t max_entries, int device, void* stream) {
    if (!out || max_tris == 0 || max_entries == 0) return fail(YS_ERR_BAD_ARG, "bad argument");
    max_entries = std::min(max_entries, MAX_ENTRIES);  // the bucket words hold first slots below 2^28 - 1
    YS_CK3(cudaSetDevice(device));
    ys_shash* h = new ys_shash();
    h->device = device;
    h->stream = (cudaStream_t)stream;
    h->maxTris = max_tris;
    h->maxEntries = max_entries;
    u32 T = 1;
    while (T < 2u * max_entries && T < (1u << 31)) T <<= 1;
    h->mask = T - 1;
    h->tableCap = T;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->tris, sizeof(ShBox) * (size_t)max_tris);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->sbox, sizeof(ShBox) * (size_t)max_tris);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->tkey, 4 * (size_t)max_tris);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->tid, 4 * (size_t)max_tris);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->counts, 4 * ((size_t)max_tris + 1));
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->ebucket, 4 * (size_t)max_entries);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->etri, 4 * (size_t)max_entries);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->bstart, 4 * ((size_t)T + 1));
    if (e == cudaSuccess) e = cudaMalloc(&h->sortScratch, sort_scratch_bytes(std::max(max_entries, max_tris)));
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->big, 4 * (size_t)max_tris);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->nbig, 4);
    size_t sb = scan_scratch_bytes(max_tris + 1);
    if (e == cudaSuccess) e = cudaMalloc(&h->scan, sb);
    if (e != cudaSuccess) {
        ys_shash_destroy(h);
        return fail(YS_ERR_CUDA, cudaGetErrorString(e));
    }
    *out = h;
    return YS_OK;
}

ys_status ys_shash_destroy(ys_shash* h) {
    if (!h) return YS_OK;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    cudaFree(h->tris); cudaFree(h->sbox); cudaFree(h->tkey); cudaFree(h->tid);
    cudaFree(h->counts); cudaFree(h->ebucket); cudaFree(h->etri);
    cudaFree(h->bstart); cudaFree(h->sortScratch); cudaFree(h->big); cudaFree(h->nbig);
    cudaFree(h->scan);
    query_order_free(h->qorder);
    delete h;
    return YS_OK;
}

ys_status ys_shash_build(ys_shash* h, const float* d_x, const uint32_t* d_facets, uint32_t nF, float cell) {
    if (!h || !d_x || !d_facets || nF == 0 || !(cell > 0.f)) return fail(YS_ERR_BAD_ARG, "bad argument");
    if (nF > h->maxTris) return fail(YS_ERR_CAPACITY, "more triangles than the hash was created for");
    cudaStream_t s = h->stream;
    h->nF = nF;
    h->cell = cell;
    h->inv = 1.0f / cell;
    k_sh_bound<<<ceil_div(nF, 256), 256, 0, s>>>(d_x, d_facets, nF, h->inv, h->tris, h->tkey, h->tid);
    // internal order: neighbouring cells' triangles side by side, so a query's
    // box reads are local
    YS_CK3(radix_sort_pairs(h->tkey, h->tid, nF, h->sortScratch, 0, 32, s));
    k_sh_order<<<ceil_div(nF, 256), 256, 0, s>>>(h->tris, h->tid, nF, h->inv, h->sbox, h->counts);
    YS_CK3(cudaMemsetAsync(h->counts + nF, 0, 4, s));
    YS_CK3(exclusive_scan(h->counts, nF + 1, h->scan, s));
    u32 nE = 0;
    YS_CK3(cudaMemcpyAsync(&nE, h->counts + nF, 4, cudaMemcpyDeviceToHost, s));
    YS_CK3(cudaStreamSynchronize(s));
    if (nE > h->maxEntries) return fail(YS_ERR_CAPACITY, "cell entries exceed the hash capacity");
    h->nE = nE;
    // buckets for this build's entries (load factor at most 1/2): clearing
    // and scanning a table sized for the capacity cost more than the build
    u32 T = 1;
    while (T < 2u * std::max(nE, 1u) && T < h->tableCap) T <<= 1;
    h->mask = T - 1;
    int bits = 0;
    while ((1u << bits) < T) ++bits;
    YS_CK3(cudaMemsetAsync(h->bstart, 0xFF, 4 * ((size_t)T + 1), s));
    YS_CK3(cudaMemsetAsync(h->nbig, 0, 4, s));
    k_sh_emit<<<ceil_div(nF, 256), 256, 0, s>>>(h->sbox, h->counts, nF, h->inv, h->mask, h->ebucket, h->etri,
                                                 h->big, h->nbig);
    // entries grouped by bucket with a stable radix sort of (bucket,
    // triangle) in place of per-entry atomics on bucket counters (random
    // atomics into a table of up to 2^31 buckets); the triangle rides along
    // as the value, so no gather follows
    if (nE) {
        YS_CK3(radix_sort_pairs(h->ebucket, h->etri, nE, h->sortScratch, 0, bits, s));
        k_sh_mark<<<ceil_div(nE, 256), 256, 0, s>>>(h->ebucket, nE, h->bstart);
    }
    YS_CK3(cudaGetLastError());
    YS_CK3(cudaStreamSynchronize(s));
    return YS_OK;
}

ys_status ys_shash_query(ys_shash* h, const float* d_qx, uint32_t nQ, float margin, uint32_t* d_pairs, uint64_t cap,
                         unsigned long long* d_count) {
    if (!h || !d_qx || !d_count || h->nF == 0) return fail(YS_ERR_BAD_ARG, "bad argument / hash not built");
    if (!(2.0f * margin <= h->cell)) return fail(YS_ERR_BAD_ARG, "cell must be at least 2 * margin");
    cudaStream_t s = h->stream;
    YS_CK3(cudaMemsetAsync(d_count, 0, 8, s));
    const u32* order = nullptr;
    if (nQ >= QUERY_ORDER_MIN_HASH) {
        YS_CK3(query_order(h->qorder, d_qx, nQ, s));
        order = h->qorder.idx;
    }
    if (nQ) k_sh_query<<<ceil_div(nQ, 128), 128, 0, s>>>(d_qx, nQ, margin, h->inv, h->mask, h->sbox, h->tid, h->bstart,
                                                          h->ebucket, h->nE, h->etri, h->big, h->nbig,
                                                          order, d_pairs, cap, d_count);
    YS_CK3(cudaGetLastError());
    YS_CK3(cudaStreamSynchronize(s));
    return YS_OK;
}

ys_status ys_shash_entries(ys_shash* h, uint32_t* n_entries, uint32_t* n_oversized) {
    if (!h) return fail(YS_ERR_BAD_ARG, "null hash");
    if (n_entries) *n_entries = h->nE;
    if (n_oversized) YS_CK3(cudaMemcpy(n_oversized, h->nbig, 4, cudaMemcpyDeviceToHost));
    return YS_OK;
}

}  // extern "C"
