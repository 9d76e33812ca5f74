// ys_shash.cu -- uniform-grid spatial-hash broad phase, point vs triangle.
//
// The reference's spatial-hash broad phases (SpatialHashing<METAL>,
// spatial_hash.hpp:880-960; CpuSpatialHash, spatial_hash.hpp:1547-2016) bin
// primitives into grid cells, probe the cells a query overlaps, and keep the
// candidates that pass an AABB precull.  This is the B200 form for the
// collision microbenchmark: triangles are binned by their AABB into every
// cell it overlaps (cell edge = 2h by default), a counting sort groups the
// entries by hash bucket, and each query point probes the <= 8 cells its box
// [p - h, p + h] overlaps.  Every entry keeps the ordinal of the cell it was
// binned for, so a bucket shared by two cells (a hash collision, possibly of
// two cells of the same triangle) never passes an entry off as another
// cell's.  A pair (p, t) is emitted only from the cell that is the
// component-wise max of the two cell ranges' lower corners, so each
// overlapping pair comes out exactly once, and the candidate set equals the
// LBVH point query's (queryPoints, bvh.metal:1394-1412) under the same
// inclusive AABB test.
//
// Build: k_sh_bound (tri boxes + cell ranges + entry counts) -> exclusive
// scan -> k_sh_emit (bucket ids) -> bucket histogram -> scan -> scatter.
// Triangles spanning more than MAX_CELLS cells go to a short overflow list
// that every query tests directly.
#include <algorithm>
#include <string>

#include "ys_common.cuh"
#include "ys_lbvh.cuh"
#include "ys_scan.cuh"
#include "ys_sort.cuh"
#include "ysim_b200.h"

namespace ys {
ys_status fail(ys_status code, const std::string& msg);

static constexpr u32 MAX_CELLS = 512;

__device__ __forceinline__ u32 cell_hash(int x, int y, int z, u32 mask) {
    // Teschner et al. 2003 spatial-hash primes
    return (((u32)x * 73856093u) ^ ((u32)y * 19349663u) ^ ((u32)z * 83492791u)) & mask;
}

struct ShTri { float mn[3]; int lo[3]; float mx[3]; int hi[3]; };  // 48 B

__global__ void k_sh_bound(const float* __restrict__ x, const u32* __restrict__ F, u32 nF, float inv,
                           ShTri* __restrict__ tris, u32* __restrict__ counts) {
    u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nF) return;
    f3 a = ldp(x, F[3 * t]), b = ldp(x, F[3 * t + 1]), c = ldp(x, F[3 * t + 2]);
    f3 lo = vmin(vmin(a, b), c), hi = vmax(vmax(a, b), c);  // leaf box (buildLeaf_Tri)
    ShTri r;
    const float l3[3] = {lo.x, lo.y, lo.z}, h3[3] = {hi.x, hi.y, hi.z};
    unsigned long long cells = 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r.mn[k] = l3[k];
        r.mx[k] = h3[k];
        r.lo[k] = (int)floorf(l3[k] * inv);
        r.hi[k] = (int)floorf(h3[k] * inv);
        cells *= (unsigned long long)(r.hi[k] - r.lo[k] + 1);
    }
    tris[t] = r;
    counts[t] = cells <= MAX_CELLS ? (u32)cells : 0u;
}

__global__ void k_sh_emit(const ShTri* __restrict__ tris, const u32* __restrict__ off, u32 nF, u32 mask,
                          u32* __restrict__ ebucket, u32* __restrict__ etri, unsigned short* __restrict__ eord,
                          u32* __restrict__ eidx, u32* __restrict__ big, u32* __restrict__ nbig) {
    u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nF) return;
    const ShTri r = tris[t];
    const u32 base = off[t], end = off[t + 1];
    if (base == end) {  // oversized: tested by every query
        u32 i = atomicAdd(nbig, 1u);
        big[i] = t;
        return;
    }
    u32 k = base;
    for (int z = r.lo[2]; z <= r.hi[2]; ++z)
        for (int y = r.lo[1]; y <= r.hi[1]; ++y)
            for (int xx = r.lo[0]; xx <= r.hi[0]; ++xx) {
                u32 b = cell_hash(xx, y, z, mask);
                ebucket[k] = b;
                etri[k] = t;
                eord[k] = (unsigned short)(k - base);  // < MAX_CELLS
                eidx[k] = k;
                ++k;
            }
}

// After the entries are sorted by bucket (radix sort of (bucket, entry)):
// the triangle and cell ordinal of each sorted slot.
__global__ void k_sh_gather(const u32* __restrict__ eidx, const u32* __restrict__ etri,
                            const unsigned short* __restrict__ eord, u32 nE, u32* __restrict__ sorted,
                            unsigned short* __restrict__ sord) {
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nE) return;
    const u32 e = eidx[k];
    sorted[k] = etri[e];
    sord[k] = eord[e];
}

// First slot of each bucket's run in the sorted keys (buckets with no entry
// keep 0xFFFFFFFF); a bucket's run ends where the key changes.
__global__ void k_sh_mark(const u32* __restrict__ skey, u32 nE, u32* __restrict__ bstart) {
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nE) return;
    const u32 b = skey[k];
    if (k == 0 || skey[k - 1] != b) bstart[b] = k;
}

__device__ __forceinline__ bool box_hit(f3 qmn, f3 qmx, const ShTri& r) {
    if (qmx.x < r.mn[0] || qmn.x > r.mx[0]) return false;
    if (qmx.y < r.mn[1] || qmn.y > r.mx[1]) return false;
    if (qmx.z < r.mn[2] || qmn.z > r.mx[2]) return false;
    return true;
}

__global__ void __launch_bounds__(128) k_sh_query(const float* __restrict__ qx, u32 nQ, float m, float inv, u32 mask,
                                                  const ShTri* __restrict__ tris, const u32* __restrict__ bstart,
                                                  const u32* __restrict__ skey, u32 nE,
                                                  const u32* __restrict__ sorted,
                                                  const unsigned short* __restrict__ sord, const u32* __restrict__ big,
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
    auto emit = [&](u32 t) {
        unsigned long long i = atomicAdd(count, 1ull);
        if (i < cap) { pairs[2 * i] = p; pairs[2 * i + 1] = t; }
    };
    for (int z = lo[2]; z <= hi[2]; ++z)
        for (int y = lo[1]; y <= hi[1]; ++y)
            for (int xx = lo[0]; xx <= hi[0]; ++xx) {
                const u32 b = cell_hash(xx, y, z, mask);
                for (u32 k = bstart[b]; k < nE && skey[k] == b; ++k) {
                    const u32 t = sorted[k];
                    const ShTri r = tris[t];
                    // the entry was binned for this very cell (not for another
                    // cell hashing to the same bucket)
                    if (xx < r.lo[0] || xx > r.hi[0] || y < r.lo[1] || y > r.hi[1] || z < r.lo[2] || z > r.hi[2])
                        continue;
                    const int nx = r.hi[0] - r.lo[0] + 1, ny = r.hi[1] - r.lo[1] + 1;
                    if ((int)sord[k] != ((z - r.lo[2]) * ny + (y - r.lo[1])) * nx + (xx - r.lo[0])) continue;
                    // emit from the first common cell only
                    if (xx != max(lo[0], r.lo[0]) || y != max(lo[1], r.lo[1]) || z != max(lo[2], r.lo[2])) continue;
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
    ShTri* tris = nullptr;
    // entries: bucket (sorted in place by the build: the key of each sorted
    // slot), triangle, cell ordinal and entry index (the sort's values)
    u32 *counts = nullptr, *ebucket = nullptr, *etri = nullptr, *eidx = nullptr, *bstart = nullptr, *sorted = nullptr,
        *big = nullptr, *nbig = nullptr;
    void* sortScratch = nullptr;
    unsigned short *eord = nullptr, *sord = nullptr;  // cell ordinal of each entry within its triangle's range
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
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->tris, sizeof(ShTri) * (size_t)max_tris);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->counts, 4 * ((size_t)max_tris + 1));
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->ebucket, 4 * (size_t)max_entries);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->etri, 4 * (size_t)max_entries);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->sorted, 4 * (size_t)max_entries);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->eord, 2 * (size_t)max_entries);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->sord, 2 * (size_t)max_entries);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->bstart, 4 * ((size_t)T + 1));
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->eidx, 4 * (size_t)max_entries);
    if (e == cudaSuccess) e = cudaMalloc(&h->sortScratch, sort_scratch_bytes(max_entries));
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
    cudaFree(h->tris); cudaFree(h->counts); cudaFree(h->ebucket); cudaFree(h->etri); cudaFree(h->sorted); cudaFree(h->eord); cudaFree(h->sord);
    cudaFree(h->bstart); cudaFree(h->eidx); cudaFree(h->sortScratch); cudaFree(h->big); cudaFree(h->nbig);
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
    k_sh_bound<<<ceil_div(nF, 256), 256, 0, s>>>(d_x, d_facets, nF, h->inv, h->tris, h->counts);
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
    k_sh_emit<<<ceil_div(nF, 256), 256, 0, s>>>(h->tris, h->counts, nF, h->mask, h->ebucket, h->etri, h->eord,
                                                 h->eidx, h->big, h->nbig);
    // entries grouped by bucket with a radix sort of (bucket, entry) in place
    // of per-entry atomics on bucket counters: those are random atomics into
    // a table of up to 2^31 buckets, and two passes of them were most of the
    // build
    if (nE) {
        YS_CK3(radix_sort_pairs(h->ebucket, h->eidx, nE, h->sortScratch, 0, bits, s));
        k_sh_gather<<<ceil_div(nE, 256), 256, 0, s>>>(h->eidx, h->etri, h->eord, nE, h->sorted, h->sord);
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
    if (nQ) k_sh_query<<<ceil_div(nQ, 128), 128, 0, s>>>(d_qx, nQ, margin, h->inv, h->mask, h->tris, h->bstart,
                                                          h->ebucket, h->nE, h->sorted, h->sord, h->big, h->nbig,
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
