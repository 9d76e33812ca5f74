// ys_lbvh.cu -- Morton codes, Karras LBVH topology and the fused swept refit.
#include "ys_lbvh.cuh"

namespace ys {

// ------------------------------------------------------------------ scene box
// Order-preserving float <-> uint map so atomicMin/atomicMax on uints give
// float min/max (the min/max of a set does not depend on order).
__device__ __forceinline__ u32 ford(float f) {
    u32 u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float funord(u32 u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
#else
    u32 r = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
    float f; memcpy(&f, &r, 4); return f;
#endif
}

__global__ void k_box_init(u32* box) {
    int t = threadIdx.x;
    if (t < 3) box[t] = 0xFFFFFFFFu;  // min slots
    else if (t < 6) box[t] = 0u;      // max slots
}

__device__ __forceinline__ f3 load_pos(const float4* x4, const float* x3, u32 i) {
    return x4 ? ld(x4, i) : ldp(x3, i);
}

// bvh.hpp:1229-1231: box over every vertex of the mesh.
__global__ void __launch_bounds__(256) k_box(const float4* x4, const float* x3, u32 voff, u32 nV, u32* box) {
    u32 mn[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, mx[3] = {0u, 0u, 0u};
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < nV; i += gridDim.x * blockDim.x) {
        f3 p = load_pos(x4, x3, voff + i);
        u32 a = ford(p.x), b = ford(p.y), c = ford(p.z);
        mn[0] = min(mn[0], a); mn[1] = min(mn[1], b); mn[2] = min(mn[2], c);
        mx[0] = max(mx[0], a); mx[1] = max(mx[1], b); mx[2] = max(mx[2], c);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        mn[k] = __reduce_min_sync(0xffffffffu, mn[k]);
        mx[k] = __reduce_max_sync(0xffffffffu, mx[k]);
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) { atomicMin(&box[k], mn[k]); atomicMax(&box[3 + k], mx[k]); }
    }
}

void launch_box_init(u32* box, cudaStream_t s) { k_box_init<<<1, 32, 0, s>>>(box); }
void launch_box(const float4* x4, const float* x3, u32 voff, u32 nV, u32* box, cudaStream_t s) {
    if (nV == 0) return;
    int blocks = ceil_div(nV, 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_box<<<blocks, 256, 0, s>>>(x4, x3, voff, nV, box);
}

// ------------------------------------------------------------------ Morton
__device__ __forceinline__ u32 expand_bits(u32 v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
__device__ __forceinline__ float clamp01023(float v) { return fminf(fmaxf(v, 0.f), 1023.f); }

// fillMortons_Tri (bvh.metal:42-63): centroid ((x0+x1)+x2)/3, normalised by
// the scene box (width clamped to >= 1e-8), 10 bits per axis, code = x*4+y*2+z.
// cube != 0 normalises all three axes by the box's largest width instead of
// each axis by its own: a flat sheet's thin axis then keeps its few high bits
// constant rather than spreading its jitter over all ten, which would split the
// tree on that axis at every third level into siblings covering the same area.
__global__ void __launch_bounds__(256) k_morton(const float4* x4, const float* x3, u32 voff, const u32* __restrict__ F,
                                                u32 nF, const u32* __restrict__ box, u32* __restrict__ codes,
                                                u32* __restrict__ idx, int cube) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nF) return;
    f3 bmin = mk(funord(box[0]), funord(box[1]), funord(box[2]));
    f3 bmax = mk(funord(box[3]), funord(box[4]), funord(box[5]));
    f3 w = bmax - bmin;
    w = mk(fmaxf(w.x, 1e-8f), fmaxf(w.y, 1e-8f), fmaxf(w.z, 1e-8f));
    if (cube) {
        const float W = fmaxf(w.x, fmaxf(w.y, w.z));
        w = mk(W, W, W);
    }
    f3 c = (load_pos(x4, x3, voff + F[3 * i]) + load_pos(x4, x3, voff + F[3 * i + 1]) +
            load_pos(x4, x3, voff + F[3 * i + 2])) / 3.0f;
    c = (c - bmin) / w;
    f3 p = c * 1024.f;
    codes[i] = expand_bits((u32)clamp01023(p.x)) * 4 + expand_bits((u32)clamp01023(p.y)) * 2 +
               expand_bits((u32)clamp01023(p.z));
    idx[i] = i;
}

void launch_morton(const float4* x4, const float* x3, u32 voff, const u32* facets, u32 nF, const u32* box, u32* codes,
                   u32* idx, cudaStream_t s, bool cube) {
    if (nF == 0) return;
    k_morton<<<ceil_div(nF, 256), 256, 0, s>>>(x4, x3, voff, facets, nF, box, codes, idx, cube ? 1 : 0);
}

// ------------------------------------------------------------------ Karras
// delta / determineRange / findSplit (bvh.metal:197-258).
struct KarrasView {
    const u32* __restrict__ c;
    const u32* __restrict__ ix;
    int n;
    __device__ __forceinline__ int delta(int i, int j) const {
        if (j < 0 || j >= n) return -1;
        u32 ci = c[i], cj = c[j];
        if (ci != cj) return clz32(ci ^ cj);
        return 32 + clz32(ix[i] ^ ix[j]);
    }
};

__global__ void k_parent_init(i32* __restrict__ parent, i32* __restrict__ parent2, u32 numNodes) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < numNodes) { parent[i] = -1; parent2[i] = 0x7FFFFFFF; }
}

__global__ void __launch_bounds__(256) k_karras(const u32* __restrict__ codes, const u32* __restrict__ idx, u32 n,
                                                Node* __restrict__ nodes, i32* __restrict__ parent,
                                                i32* __restrict__ parent2, u32* __restrict__ visits) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int)n) return;
    KarrasView K{codes, idx, (int)n};
    Node* L = nodes + (n - 1 + i);
    L->a = -1;
    L->b = (i32)idx[i];
    if (i + 1 >= (int)n) return;
    visits[i] = 0;
    int d = (K.delta(i, i + 1) - K.delta(i, i - 1) >= 0) ? 1 : -1;
    int dmin = K.delta(i, i - d);
    int lmax = 2;
    while (K.delta(i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (K.delta(i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int first = d < 0 ? j : i, last = d < 0 ? i : j;
    // findSplit
    u32 c0 = codes[first], c1 = codes[last];
    u32 split;
    if (c0 == c1) {
        split = (u32)((first + last) >> 1);
    } else {
        int prefix = clz32(c0 ^ c1);
        u32 sp = (u32)first, step = (u32)(last - first);
        do {
            step = (step + 1) >> 1;
            u32 ns = sp + step;
            if (ns < (u32)last && clz32(c0 ^ codes[ns]) > prefix) sp = ns;
        } while (step > 1);
        split = sp;
    }
    int s = (int)split;
    int ca = (s == first) ? s + (int)n - 1 : s;
    int cb = (s + 1 == last) ? s + (int)n : s + 1;
    nodes[i].a = ca;
    nodes[i].b = cb;
    atomicMax(&parent[ca], i);
    atomicMin(&parent2[ca], i);
    atomicMax(&parent[cb], i);
    atomicMin(&parent2[cb], i);
}

void launch_karras(const u32* codes, const u32* idx, u32 n, Node* nodes, i32* parent, i32* parent2, u32* visits,
                   cudaStream_t s) {
    if (n == 0) return;
    k_parent_init<<<ceil_div(2 * n - 1, 256), 256, 0, s>>>(parent, parent2, 2 * n - 1);
    k_karras<<<ceil_div(n, 256), 256, 0, s>>>(codes, idx, n, nodes, parent, parent2, visits);
}

// ------------------------------------------------------------------ refit
// buildSweptLeaf_Tri / buildLeaf_Tri (bvh.metal:260-351) + bottomUpBoxes
// (bvh.metal:510-586).  One thread per leaf writes its box, then climbs: the
// first thread to arrive at a parent stops, the second combines both children
// and continues.  Arrival counters are never reset between refits: every
// internal node receives exactly two arrivals per refit (one per child it
// lists), so an even old value means "first", odd means "second".  Karras
// zeroes them at build.
// Memory order: box store -> __threadfence -> atomicAdd (release); atomicAdd
// -> __threadfence -> L1-bypassing loads of the children (acquire).
__device__ __forceinline__ void store_box(Node* nd, f3 lo, f3 hi) {
    float4* p = reinterpret_cast<float4*>(nd);
    float4 a = __ldcg(p), b = __ldcg(p + 1);
    a.x = lo.x; a.y = lo.y; a.z = lo.z;
    b.x = hi.x; b.y = hi.y; b.z = hi.z;
    __stcg(p, a);
    __stcg(p + 1, b);
}

__global__ void __launch_bounds__(256) k_refit(const RefitJob* __restrict__ jobs, u32 numJobs, u32 totalLeaves,
                                               u32* status) {
    u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= totalLeaves) return;
    // find the job owning leaf g (few jobs; linear scan is fine up to a few
    // hundred and stays uniform within a warp most of the time)
    u32 j = 0;
    {
        u32 lo = 0, hi = numJobs;  // largest j with leafBase <= g
        while (hi - lo > 1) {
            u32 mid = (lo + hi) >> 1;
            if (jobs[mid].leafBase <= g) lo = mid; else hi = mid;
        }
        j = lo;
    }
    const RefitJob J = jobs[j];
    const u32 n = J.n;
    const u32 i = g - J.leafBase;
    Node* nodes = J.nodes;
    const u32 leaf = n - 1 + i;
    const u32 f = (u32)__ldcg(&nodes[leaf].b);
    const u32 vid[3] = {J.facets[3 * f], J.facets[3 * f + 1], J.facets[3 * f + 2]};
    f3 lo, hi;
    float ext = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        u32 gv = J.voff + vid[k];
        f3 p = J.x4 ? ld(J.x4, gv) : ldp(J.x3, gv);
        f3 a = p, b = p;
        if (J.swept) {
            f3 vv = J.v4 ? ld(J.v4, gv) : ldp(J.v3, gv);
            f3 sp = p + vv * J.dt;
            a = vmin(p, sp);
            b = vmax(p, sp);
        }
        if (k == 0) { lo = a; hi = b; } else { lo = vmin(lo, a); hi = vmax(hi, b); }
    }
    if (J.selfMargin > 0.f) {
        // H1 grid extent: largest axis extent of the tri AABB inflated by m
        // (collectFaceBoxes, spatial_hash.hpp:1613-1655), finite faces only.
        float m = J.selfMargin;
        bool ok = true;
        float e = 0.f;
        f3 P0, P1, P2;
        {
            u32 g0 = J.voff + vid[0], g1 = J.voff + vid[1], g2 = J.voff + vid[2];
            P0 = J.x4 ? ld(J.x4, g0) : ldp(J.x3, g0);
            P1 = J.x4 ? ld(J.x4, g1) : ldp(J.x3, g1);
            P2 = J.x4 ? ld(J.x4, g2) : ldp(J.x3, g2);
        }
        float pa[3][3] = {{P0.x, P1.x, P2.x}, {P0.y, P1.y, P2.y}, {P0.z, P1.z, P2.z}};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (!isfinite(pa[a][0]) || !isfinite(pa[a][1]) || !isfinite(pa[a][2])) ok = false;
            float l = tmin(pa[a][0], tmin(pa[a][1], pa[a][2]));
            float h = tmax(pa[a][0], tmax(pa[a][1], pa[a][2]));
            float bmn = l - m, bmx = h + m;
            e = fmaxf(e, bmx - bmn);
        }
        if (ok) ext = e;
    }
    {
        // one atomic per warp and job: group lanes by their target slot
        const unsigned act = __activemask();
        const unsigned peers = __match_any_sync(act, (unsigned long long)J.maxExt);
        const u32 e = __reduce_max_sync(peers, __float_as_uint(ext));
        if (J.selfMargin > 0.f && (threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicMax(J.maxExt, e);
    }
    store_box(&nodes[leaf], lo, hi);
    if (n == 1) return;
    const u32 numInner = n - 1;
    // Climb: deliver this node's arrival to every internal node that claims
    // it as a child (one claimant in a consistent tree); the second arrival
    // at a claimant combines it and climbs on from there.  Extra climbs (a
    // node with two claimants) wait in a small pending list.
    u32 pending[4];
    int np = 0;
    u32 child = leaf;
    __threadfence();
    for (u32 step = 0; step < 2 * n; ++step) {
        const i32 p1 = __ldcg(&J.parent[child]);
        const i32 p2 = __ldcg(&J.parent2[child]);
        i32 claim[2] = {p1, (p2 != p1 && p2 != 0x7FFFFFFF) ? p2 : -1};
        i32 next = -1;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const i32 par = claim[c];
            if (par < 0) continue;
            if ((u32)par >= numInner) { atomicOr(status, ST_ITER_CAP); continue; }
            u32 old = atomicAdd(&J.visits[par], 1u);
            if ((old & 1u) == 0u) continue;  // first arrival: the sibling's thread combines
            __threadfence();
            const float4* pn = reinterpret_cast<const float4*>(&nodes[par]);
            const float4 h0 = __ldcg(pn), h1 = __ldcg(pn + 1);
            const i32 ca = __float_as_int(h0.w), cb = __float_as_int(h1.w);
            if (ca < 0 || (u32)ca >= 2 * n - 1 || cb < 0 || (u32)cb >= 2 * n - 1) {
                atomicOr(status, ST_ITER_CAP);
                continue;
            }
            const float4* A = reinterpret_cast<const float4*>(&nodes[ca]);
            const float4* B = reinterpret_cast<const float4*>(&nodes[cb]);
            float4 a0 = __ldcg(A), a1 = __ldcg(A + 1), b0 = __ldcg(B), b1 = __ldcg(B + 1);
            f3 plo = vmin(mk(a0.x, a0.y, a0.z), mk(b0.x, b0.y, b0.z));
            f3 phi = vmax(mk(a1.x, a1.y, a1.z), mk(b1.x, b1.y, b1.z));
            store_box(&nodes[par], plo, phi);
            __threadfence();
            if (next < 0) next = par;
            else if (np < 4) pending[np++] = (u32)par;
            else atomicOr(status, ST_ITER_CAP);
        }
        if (next < 0) {
            if (np == 0) return;  // root reached, first arrival, or an unclaimed node
            next = (i32)pending[--np];
        }
        child = (u32)next;
    }
    atomicOr(status, ST_ITER_CAP);
}

void launch_refit(const RefitJob* jobsDev, u32 numJobs, u32 totalLeaves, u32* status, cudaStream_t s) {
    if (totalLeaves == 0) return;
    k_refit<<<ceil_div(totalLeaves, 256), 256, 0, s>>>(jobsDev, numJobs, totalLeaves, status);
}

}  // namespace ys
