// ys_shff.cu -- the face-face spatial-hash broad phase (Pabst): the reference's
// SpatialHashing<METAL>::detectCollisions (spatial_hash.hpp:880-960, kernels
// spatialhashing.metal:64-478) with its rows, B200 form.
//
// Semantics (identical rows as a multiset):
//   * bounding sphere per face: centroid ((v0+v1)+v2)*(1/3), radius |c - v0|
//     (sh_buildBV takes v0 only);
//   * grid: box over all vertices, cell = 2*maxR*1 + margin, resolution
//     ceil(extent / cell) >= 1 per axis (computeGrid);
//   * home cell (floor, clamped) plus the octant's phantom cells whose wall is
//     within r; the face's type mask holds the parity types of its cells
//     (sh_assignCells);
//   * per cell, home-home and home-phantom pairs (sh_computePairCount), kept
//     unless self pairs are off and the faces share a mesh, both meshes are
//     Float, the type masks share a type below the cell's (marking dedup), or
//     the centroids are farther apart than rA + rB + margin; then 6 rows
//     (sh_broadPhase).
//
// B200 form: the reference's four host round trips (max radius, numValid,
// cell-start scan, pair-prefix scan) become device scans and device-side
// counts; the broad kernel is a grid-stride loop over the pair count read from
// device memory, so a detect is one stream of launches with no host sync.
#include <string>

#include "ys_common.cuh"
#include "ys_lbvh.cuh"
#include "ys_scan.cuh"
#include "ys_sort.cuh"
#include "ysim_b200.h"

namespace ys {
ys_status fail(ys_status code, const std::string& msg);

static constexpr u32 SH_SENT = 0xFFFFFFFFu;  // empty slot; sorts to the tail

__device__ __forceinline__ float sh_unord(u32 u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

struct ShffParams {
    float cell, margin;
    float o[3];
    int res[3];
    u32 numValid, numCells, numPairs;
};

__device__ __forceinline__ u32 face_obj(const u32* __restrict__ facetOff, u32 nM, u32 f) {
    u32 lo = 0, hi = nM;  // largest m with facetOff[m] <= f
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) >> 1;
        if (facetOff[mid] <= f) lo = mid; else hi = mid;
    }
    return lo;
}

// Face spheres (float4: centroid, radius) and the largest radius.
__global__ void __launch_bounds__(256) k_ff_bv(const float* __restrict__ x, const u32* __restrict__ stateOff,
                                               const u32* __restrict__ F, const u32* __restrict__ facetOff, u32 nM,
                                               u32 nF, float4* __restrict__ sph, u32* __restrict__ maxR) {
    const u32 f = blockIdx.x * blockDim.x + threadIdx.x;
    float r = 0.f;
    if (f < nF) {
        const u32 vb = stateOff[face_obj(facetOff, nM, f)];
        const f3 a = ldp(x, vb + F[3 * f]), b = ldp(x, vb + F[3 * f + 1]), c3 = ldp(x, vb + F[3 * f + 2]);
        const f3 c = (a + b + c3) * (1.0f / 3.0f);
        const f3 e = c - a;
        r = sqrtf(dot(e, e));
        sph[f] = make_float4(c.x, c.y, c.z, r);
    }
    // radii are >= 0: their float bits order as unsigned ints; one atomic per block
    __shared__ u32 red[8];
    const u32 m = __reduce_max_sync(0xFFFFFFFFu, __float_as_uint(r));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 b = 0;
        for (u32 w = 0; w < (blockDim.x >> 5); ++w) b = max(b, red[w]);
        if (b) atomicMax(maxR, b);
    }
}

// computeGrid from the device-side box and radius.
__global__ void k_ff_grid(const u32* __restrict__ box, const u32* __restrict__ maxR, float margin,
                          ShffParams* __restrict__ P) {
    float cell = 2.0f * __uint_as_float(*maxR) * 1.0f + margin;
    if (cell <= 0.f) cell = fmaxf(margin, 1e-6f);
    P->cell = cell;
    P->margin = margin;
    for (int k = 0; k < 3; ++k) {
        const float lo = sh_unord(box[k]), hi = sh_unord(box[3 + k]);
        P->o[k] = lo;
        const u32 r = (u32)ceilf((hi - lo) / cell);
        P->res[k] = (int)(r == 0 ? 1 : r);
    }
}

// Home + phantom cells of each face into its 8 slots: key = cell id (or
// SH_SENT), value = face << 1 | phantom; type mask per face.
__global__ void __launch_bounds__(256) k_ff_assign(const float4* __restrict__ sph, u32 nF,
                                                   const ShffParams* __restrict__ P, u32* __restrict__ keys,
                                                   u32* __restrict__ vals, u32* __restrict__ mask) {
    const u32 f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const float4 s = sph[f];
    const float cell = P->cell, hcs = cell * 0.5f;
    const float cc[3] = {s.x, s.y, s.z};
    int g[3], sg[3];
    float dist[3];
    int res[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        res[k] = P->res[k];
        const float o = P->o[k];
        int q = (int)floorf((cc[k] - o) / cell);
        q = min(max(q, 0), res[k] - 1);
        g[k] = q;
        const float local = cc[k] - (o + (float)q * cell);
        sg[k] = local > hcs ? 1 : -1;
        dist[k] = sg[k] > 0 ? cell - local : local;
    }
    u32 cb = 0, slot = 0;
    const u32 base = 8 * f;
    for (int i = 0; i <= 1; ++i) {
        if (i && dist[0] > s.w) continue;
        for (int j = 0; j <= 1; ++j) {
            if (j && dist[1] > s.w) continue;
            for (int k = 0; k <= 1; ++k) {
                if (k && dist[2] > s.w) continue;
                const int p0 = g[0] + i * sg[0], p1 = g[1] + j * sg[1], p2 = g[2] + k * sg[2];
                if (p0 < 0 || p0 >= res[0] || p1 < 0 || p1 >= res[1] || p2 < 0 || p2 >= res[2]) continue;
                cb |= 1u << ((p0 & 1) | ((p1 & 1) << 1) | ((p2 & 1) << 2));
                keys[base + slot] = ((u32)p2 * (u32)res[1] + (u32)p1) * (u32)res[0] + (u32)p0;
                vals[base + slot] = (f << 1) | ((i | j | k) ? 1u : 0u);
                ++slot;
            }
        }
    }
    for (u32 k = slot; k < 8; ++k) { keys[base + k] = SH_SENT; vals[base + k] = SH_SENT; }
    mask[f] = cb;
}

// flag[i] = entry i starts a cell (valid and a new key).
__global__ void __launch_bounds__(256) k_ff_flags(const u32* __restrict__ keys, u32 n, u32* __restrict__ flag) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 k = keys[i];
    flag[i] = (k != SH_SENT && (i == 0 || keys[i - 1] != k)) ? 1u : 0u;
}

// Per entry: its cell (scan + flag - 1), home / phantom counts, the cell's
// start and parity type; the last valid entry records the counts.
__global__ void __launch_bounds__(256) k_ff_cells(const u32* __restrict__ keys, const u32* __restrict__ vals,
                                                  u32* __restrict__ flag, const u32* __restrict__ scan, u32 n,
                                                  ShffParams* __restrict__ P, u32* __restrict__ cstart,
                                                  u32* __restrict__ nh, u32* __restrict__ np, u32* __restrict__ ctype) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 k = keys[i];
    if (k == SH_SENT) return;
    const u32 c = scan[i] + flag[i] - 1;
    atomicAdd((vals[i] & 1u) ? &np[c] : &nh[c], 1u);
    if (flag[i]) {
        cstart[c] = i;
        const u32 rx = (u32)P->res[0], ry = (u32)P->res[1];
        const u32 gx = k % rx, gy = (k / rx) % ry, gz = k / (rx * ry);
        ctype[c] = (gx & 1u) | ((gy & 1u) << 1) | ((gz & 1u) << 2);
    }
    if (i + 1 == n || keys[i + 1] == SH_SENT) {
        P->numValid = i + 1;
        P->numCells = c + 1;
    }
    flag[i] = c;  // from here on: the entry's cell
}

// Candidate pairs per cell (zero past the last cell, for the scan).
__global__ void __launch_bounds__(256) k_ff_paircount(const u32* __restrict__ nh, const u32* __restrict__ np, u32 n,
                                                      const ShffParams* __restrict__ P, u32* __restrict__ pc) {
    const u32 c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    if (c >= P->numCells) { pc[c] = 0; return; }
    const u32 h = nh[c], p = np[c];
    pc[c] = (h * (h - 1u)) / 2u + h * p;
}

__global__ void k_ff_total(const u32* __restrict__ pc, const u32* __restrict__ prefix, ShffParams* __restrict__ P) {
    const u32 c = P->numCells;
    P->numPairs = c ? prefix[c - 1] + pc[c - 1] : 0u;
}

// Candidate pairs, one warp per home entry (grid-stride over the cell-sorted
// entries, so that a crowded cell spreads over many warps): the entry against
// every later entry of its cell and every earlier phantom entry, the lanes
// taking the partners in step.  Per cell these are the h (h - 1) / 2 + h p
// pairs of the reference's unranking (spatialhashing.metal), each once.  The
// lanes that accept a pair together reserve their 6 rows with one atomic,
// stage them in shared memory, and the warp writes the run out in 16-byte
// lane stores (a scattered 32-byte row store per lane kept the load-store
// queue full).
static constexpr int FF_WARPS = 4;  // 128-thread blocks
__global__ void __launch_bounds__(128) k_ff_broad(const u32* __restrict__ vals, const u32* __restrict__ ecell,
                                                  const u32* __restrict__ cstart, const u32* __restrict__ nh,
                                                  const u32* __restrict__ np, const u32* __restrict__ ctype,
                                                  const ShffParams* __restrict__ P, const u32* __restrict__ mask,
                                                  const float4* __restrict__ sph, const u32* __restrict__ F,
                                                  const u32* __restrict__ facetOff, const u32* __restrict__ beh,
                                                  const u32* __restrict__ shape, u32 nM, int self,
                                                  Row* __restrict__ out, u64 cap,
                                                  unsigned long long* __restrict__ count) {
    __shared__ uint4 stage[FF_WARPS][32 * 6 * 2];  // 32 pairs x 6 rows x 32 bytes per warp
    uint4* st = stage[threadIdx.x >> 5];
    const u32 numValid = P->numValid;
    const float margin = P->margin;
    const u32 lane = threadIdx.x & 31u;
    const u32 warps = (gridDim.x * blockDim.x) >> 5;
    for (u32 e = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < numValid; e += warps) {
        const u32 va = vals[e];
        if (va & 1u) continue;  // a phantom entry pairs only with homes, from their side
        const u32 c = ecell[e];
        const u32 start = cstart[c], end = start + nh[c] + np[c], cbit = (1u << ctype[c]) - 1u;
        const u32 A = va >> 1;
        const u32 oA = face_obj(facetOff, nM, A);
        const u32 mA = mask[A];
        const float4 sA = sph[A];
        for (u32 j0 = start; j0 < end; j0 += 32u) {
            const u32 j = j0 + lane;
            bool ok = false;
            u32 B = 0, oB = 0;
            if (j < end) {
                const u32 vb = vals[j];
                if ((vb & 1u) || j > e) {  // later entries, and earlier phantoms
                    B = vb >> 1;
                    oB = face_obj(facetOff, nM, B);
                    ok = (self || oA != oB) && !(beh[oA] == YS_FLOAT && beh[oB] == YS_FLOAT) && !(mA & mask[B] & cbit);
                    if (ok) {
                        const float4 sB = sph[B];
                        const f3 d = mk(sA.x, sA.y, sA.z) - mk(sB.x, sB.y, sB.z);
                        ok = !(sqrtf(dot(d, d)) > sA.w + sB.w + margin);
                    }
                }
            }
            const unsigned acc = __ballot_sync(0xFFFFFFFFu, ok);
            if (!acc) continue;
            const u32 cnt = (u32)__popc(acc);
            unsigned long long wbase = 0;
            if (lane == 0) wbase = atomicAdd(count, 6ull * cnt);
            wbase = __shfl_sync(0xFFFFFFFFu, wbase, 0);
            if (ok) {
                const u32 r = 6u * (u32)__popc(acc & ((1u << lane) - 1u));  // this pair's first staged row
                const u32 fA = A - facetOff[oA], fB = B - facetOff[oB];
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    const bool second = q >= 3;
                    const u32 Pf = second ? B : A, oP = second ? oB : oA, oT = second ? oA : oB;
                    st[2 * (r + q)] = make_uint4(F[3 * Pf + (q % 3)], second ? fA : fB, oP, oT);
                    st[2 * (r + q) + 1] = make_uint4(beh[oP], beh[oT], shape[oP], shape[oT]);
                }
            }
            __syncwarp();
            // the warp's rows [wbase, wbase + 6 cnt), as far as the capacity goes
            const unsigned long long room = wbase < cap ? cap - wbase : 0ull;
            const u32 rows = (u32)min((unsigned long long)(6u * cnt), room);
            uint4* dst = reinterpret_cast<uint4*>(out + wbase);
            for (u32 i = lane; i < 2u * rows; i += 32u) dst[i] = st[i];
            __syncwarp();
        }
    }
}

}  // namespace ys

using namespace ys;

struct ys_shff {
    int device = 0;
    cudaStream_t stream = nullptr;
    u32 maxFaces = 0;
    float4* sph = nullptr;
    u32 *maxR = nullptr, *box = nullptr, *keys = nullptr, *vals = nullptr, *mask = nullptr, *flag = nullptr,
        *scan = nullptr, *cstart = nullptr, *nh = nullptr, *np = nullptr, *ctype = nullptr, *pc = nullptr;
    ShffParams* params = nullptr;
    void* sortScratch = nullptr;
    void* scanScratch = nullptr;
};

#define YS_CK4(call)                                                                                   \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(YS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

extern "C" {

ys_status ys_shff_create(ys_shff** out, uint32_t max_faces, int device, void* stream) {
    if (!out || max_faces == 0 || max_faces >= (1u << 28)) return fail(YS_ERR_BAD_ARG, "bad argument");
    YS_CK4(cudaSetDevice(device));
    ys_shff* h = new ys_shff();
    h->device = device;
    h->stream = (cudaStream_t)stream;
    h->maxFaces = max_faces;
    const size_t E = 8 * (size_t)max_faces;
    cudaError_t e = cudaSuccess;
    auto al = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, bytes); };
    al((void**)&h->sph, sizeof(float4) * (size_t)max_faces);
    al((void**)&h->maxR, 4);
    al((void**)&h->box, 32);
    al((void**)&h->params, sizeof(ShffParams));
    for (u32** p : {&h->keys, &h->vals, &h->flag, &h->scan, &h->cstart, &h->nh, &h->np, &h->ctype, &h->pc})
        al((void**)p, 4 * E);
    al((void**)&h->mask, 4 * (size_t)max_faces);
    al(&h->sortScratch, sort_scratch_bytes((u32)E));
    al(&h->scanScratch, scan_scratch_bytes((u32)E));
    if (e != cudaSuccess) {
        ys_shff_destroy(h);
        return fail(YS_ERR_CUDA, cudaGetErrorString(e));
    }
    *out = h;
    return YS_OK;
}

ys_status ys_shff_destroy(ys_shff* h) {
    if (!h) return YS_OK;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    for (void* p : {(void*)h->sph, (void*)h->maxR, (void*)h->box, (void*)h->params, (void*)h->keys, (void*)h->vals,
                    (void*)h->flag, (void*)h->scan, (void*)h->cstart, (void*)h->nh, (void*)h->np, (void*)h->ctype,
                    (void*)h->pc, (void*)h->mask, h->sortScratch, h->scanScratch})
        cudaFree(p);
    delete h;
    return YS_OK;
}

ys_status ys_shff_detect(ys_shff* h, const float* d_x, uint32_t num_vertices, const uint32_t* d_state_off,
                         const uint32_t* d_facets, const uint32_t* d_facet_off, uint32_t num_faces,
                         const uint32_t* d_behaviors, const uint32_t* d_shapes, uint32_t num_meshes, float margin,
                         int enable_self, void* d_rows, uint64_t cap, unsigned long long* d_count) {
    if (!h || !d_x || !d_state_off || !d_facets || !d_facet_off || !d_behaviors || !d_shapes || !d_count ||
        num_meshes == 0 || num_vertices == 0 || (cap && !d_rows))
        return fail(YS_ERR_BAD_ARG, "bad argument");
    if (num_faces > h->maxFaces) return fail(YS_ERR_CAPACITY, "more faces than the hash was created for");
    if (reinterpret_cast<uintptr_t>(d_rows) & 15u) return fail(YS_ERR_BAD_ARG, "rows must be 16-byte aligned");
    cudaStream_t s = h->stream;
    YS_CK4(cudaMemsetAsync(d_count, 0, 8, s));
    if (num_faces == 0) return YS_OK;
    const u32 nF = num_faces, E = 8 * nF;
    YS_CK4(cudaMemsetAsync(h->maxR, 0, 4, s));
    YS_CK4(cudaMemsetAsync(h->params, 0, sizeof(ShffParams), s));
    launch_box_init(h->box, s);
    launch_box(nullptr, d_x, 0, num_vertices, h->box, s);
    k_ff_bv<<<ceil_div(nF, 256), 256, 0, s>>>(d_x, d_state_off, d_facets, d_facet_off, num_meshes, nF, h->sph,
                                             h->maxR);
    k_ff_grid<<<1, 1, 0, s>>>(h->box, h->maxR, margin, h->params);
    k_ff_assign<<<ceil_div(nF, 256), 256, 0, s>>>(h->sph, nF, h->params, h->keys, h->vals, h->mask);
    YS_CK4(radix_sort_pairs(h->keys, h->vals, E, h->sortScratch, 0, 32, s));
    k_ff_flags<<<ceil_div(E, 256), 256, 0, s>>>(h->keys, E, h->flag);
    YS_CK4(cudaMemcpyAsync(h->scan, h->flag, 4 * (size_t)E, cudaMemcpyDeviceToDevice, s));
    YS_CK4(exclusive_scan(h->scan, E, h->scanScratch, s));
    YS_CK4(cudaMemsetAsync(h->nh, 0, 4 * (size_t)E, s));
    YS_CK4(cudaMemsetAsync(h->np, 0, 4 * (size_t)E, s));
    k_ff_cells<<<ceil_div(E, 256), 256, 0, s>>>(h->keys, h->vals, h->flag, h->scan, E, h->params, h->cstart, h->nh,
                                               h->np, h->ctype);
    k_ff_paircount<<<ceil_div(E, 256), 256, 0, s>>>(h->nh, h->np, E, h->params, h->pc);
    // prefix over pair counts (reuses the cell-scan buffer)
    YS_CK4(cudaMemcpyAsync(h->scan, h->pc, 4 * (size_t)E, cudaMemcpyDeviceToDevice, s));
    YS_CK4(exclusive_scan(h->scan, E, h->scanScratch, s));
    k_ff_total<<<1, 1, 0, s>>>(h->pc, h->scan, h->params);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_ff_broad<<<sms * 16, 128, 0, s>>>(h->vals, h->flag, h->cstart, h->nh, h->np, h->ctype, h->params, h->mask, h->sph,
                                       d_facets, d_facet_off, d_behaviors, d_shapes, num_meshes,
                                       enable_self ? 1 : 0, (Row*)d_rows, cap, d_count);
    YS_CK4(cudaGetLastError());
    return YS_OK;
}

ys_status ys_shff_stats(ys_shff* h, uint32_t out6[6]) {
    if (!h || !out6) return fail(YS_ERR_BAD_ARG, "bad argument");
    YS_CK4(cudaStreamSynchronize(h->stream));
    ShffParams P;
    YS_CK4(cudaMemcpy(&P, h->params, sizeof(P), cudaMemcpyDeviceToHost));
    out6[0] = P.numValid; out6[1] = P.numCells; out6[2] = P.numPairs;
    out6[3] = (u32)P.res[0]; out6[4] = (u32)P.res[1]; out6[5] = (u32)P.res[2];
    return YS_OK;
}

}  // extern "C"
