// ys_lbvh.cu -- Morton codes, Karras LBVH topology and the fused swept refit.
#include <utility>

#include "ys_lbvh.cuh"
#include "ys_sort.cuh"

namespace ys {

// ------------------------------------------------------------------ scene box

__global__ void k_box_init(u32* box) {
    int t = threadIdx.x;
    if (t < 3) box[t] = 0xFFFFFFFFu;  // min slots
    else if (t < 6) box[t] = 0u;      // max slots
}

__device__ __forceinline__ f3 load_pos(const float4* x4, const float* x3, u32 i) {
    return x4 ? ld(x4, i) : ldp(x3, i);
}

// bvh.hpp:1229-1231: box over every vertex of the mesh.  Grid-stride
// threads, a warp reduction, a block reduction through shared memory, and
// one atomic per block and slot (min / max on the order-preserving integer
// form of the floats, exact).
__global__ void __launch_bounds__(256) k_box(const float4* x4, const float* x3, u32 voff, u32 nV, u32* box) {
    __shared__ u32 sh[6][8];
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
    const u32 w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) { sh[k][w] = mn[k]; sh[3 + k][w] = mx[k]; }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const u32 k = threadIdx.x;
        u32 v = sh[k][0];
        for (u32 j = 1; j < nw; ++j) v = k < 3 ? min(v, sh[k][j]) : max(v, sh[k][j]);
        if (k < 3) atomicMin(&box[k], v);
        else atomicMax(&box[k], v);
    }
}

void launch_box_init(u32* box, cudaStream_t s) { k_box_init<<<1, 32, 0, s>>>(box); }
void launch_box(const float4* x4, const float* x3, u32 voff, u32 nV, u32* box, cudaStream_t s) {
    if (nV == 0) return;
    // up to full occupancy (8 blocks of 256 per SM): the reduction is a
    // stream over the vertices, and with fewer threads in flight a 48M-vertex
    // box ran at a quarter of the bandwidth
    int blocks = ceil_div(nV, 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_box<<<blocks, 256, 0, s>>>(x4, x3, voff, nV, box);
}

// ------------------------------------------------------------------ Morton
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

// ------------------------------------------------------------------ query order
// Morton code of each query point over the points' own box (10 bits per
// axis), paired with its index for the sort.
__global__ void k_point_codes(const float* __restrict__ qx, u32 n, const u32* __restrict__ box, u32* __restrict__ codes,
                              u32* __restrict__ idx) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const f3 p = ldp(qx, i);
    const float c[3] = {p.x, p.y, p.z};
    u32 q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float lo = funord(box[a]), w = funord(box[3 + a]) - lo;
        const float t = w > 0.f ? (c[a] - lo) / w : 0.f;
        const int v = (int)(t * 1024.f);  // NaN converts to 0
        q[a] = (u32)min(max(v, 0), 1023);
    }
    codes[i] = (expand_bits(q[0]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[2]);
    idx[i] = i;
}

void query_order_free(QueryOrder& o) {
    cudaFree(o.codes); cudaFree(o.idx); cudaFree(o.scratch); cudaFree(o.box);
    o = QueryOrder();
}

cudaError_t query_order(QueryOrder& o, const float* qx, u32 n, cudaStream_t s) {
    if (n > o.cap) {
        cudaStreamSynchronize(s);
        query_order_free(o);
        cudaError_t e;
        if ((e = cudaMalloc((void**)&o.codes, 4 * (size_t)n)) || (e = cudaMalloc((void**)&o.idx, 4 * (size_t)n)) ||
            (e = cudaMalloc(&o.scratch, sort_scratch_bytes(n))) || (e = cudaMalloc((void**)&o.box, 32))) {
            query_order_free(o);
            return e;
        }
        o.cap = n;
    }
    launch_box_init(o.box, s);
    launch_box(nullptr, qx, 0, n, o.box, s);
    k_point_codes<<<ceil_div(n, 256), 256, 0, s>>>(qx, n, o.box, o.codes, o.idx);
    return radix_sort_pairs(o.codes, o.idx, n, o.scratch, 0, 32, s);
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

__global__ void k_parent_init(i32* __restrict__ parent, u32* __restrict__ claimOff, u32 numNodes) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < numNodes) parent[i] = -1;
    if (i <= numNodes) claimOff[i] = 0;
}
// After the exclusive scan of the claim counts: every internal node enters
// itself in its two children's claimant lists.  The cursor is the list start
// itself, so afterwards claimOff[c] is the end of c's list and the start is
// claimOff[c - 1] (0 for c = 0).
__global__ void k_claim_fill(const Node* __restrict__ nodes, u32 nInner, u32* __restrict__ claimOff,
                             i32* __restrict__ claims) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nInner) return;
    const i32 a = nodes[i].a, b = nodes[i].b, nn = 2 * (i32)nInner + 1;
    if (a >= 0 && a < nn) claims[atomicAdd(&claimOff[a], 1u)] = (i32)i;
    if (b >= 0 && b < nn) claims[atomicAdd(&claimOff[b], 1u)] = (i32)i;
}

__global__ void __launch_bounds__(256) k_karras(const u32* __restrict__ codes, const u32* __restrict__ idx, u32 n,
                                                Node* __restrict__ nodes, i32* __restrict__ parent,
                                                u32* __restrict__ claimCount, u32* __restrict__ visits,
                                                int consistent, BinRanges R) {
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
    if (consistent) {
        // largest s in [first, last) sharing more key bits with first than last does
        const int dnode = K.delta(first, last);
        int sp = first, step = last - first;
        do {
            step = (step + 1) >> 1;
            const int ns = sp + step;
            if (ns < last && K.delta(first, ns) > dnode) sp = ns;
        } while (step > 1);
        split = (u32)sp;
    } else if (c0 == c1) {
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
    atomicAdd(&claimCount[ca], 1u);
    atomicMax(&parent[cb], i);
    atomicAdd(&claimCount[cb], 1u);
    if (R.range) {
        // sorted-leaf range of node i (one end is leaf i); nodes whose range
        // leaves i's 256-leaf block go to the big / huge lists
        R.range[i] = make_uint2((u32)first, (u32)last);
        const bool out = ((u32)first >> 8) != ((u32)last >> 8);
        const bool huge = out && (u32)(last - first) >= BIN_RANGE_HUGE;
        const unsigned act = __activemask();
        const unsigned mb = __ballot_sync(act, out && !huge), mh = __ballot_sync(act, huge);
        const u32 lane = threadIdx.x & 31u, lead = (u32)__ffs(act) - 1u;
        u32 bb = 0, bh = 0;
        if (lane == lead) {
            if (mb) bb = atomicAdd(&R.count[0], (u32)__popc(mb));
            if (mh) bh = atomicAdd(&R.count[1], (u32)__popc(mh));
        }
        bb = __shfl_sync(act, bb, (int)lead);
        bh = __shfl_sync(act, bh, (int)lead);
        const unsigned below = (1u << lane) - 1u;
        if (out && !huge) R.big[bb + (u32)__popc(mb & below)] = (u32)i;
        if (huge) R.huge[bh + (u32)__popc(mh & below)] = (u32)i;
    }
}

size_t karras_scratch_bytes(u32 n) { return scan_scratch_bytes(n ? 2 * n : 1); }

cudaError_t launch_karras(const u32* codes, const u32* idx, u32 n, Node* nodes, i32* parent, u32* claimOff,
                          i32* claims, u32* visits, void* scratch, cudaStream_t s, bool consistent, BinRanges R) {
    if (n == 0) return cudaSuccess;
    k_parent_init<<<ceil_div(2 * n, 256), 256, 0, s>>>(parent, claimOff, 2 * n - 1);
    if (R.range) {
        cudaError_t e0 = cudaMemsetAsync(R.count, 0, 8, s);
        if (e0 != cudaSuccess) return e0;
    }
    k_karras<<<ceil_div(n, 256), 256, 0, s>>>(codes, idx, n, nodes, parent, claimOff, visits, consistent ? 1 : 0, R);
    cudaError_t e = exclusive_scan(claimOff, 2 * n, scratch, s);
    if (e != cudaSuccess) return e;
    if (n > 1) k_claim_fill<<<ceil_div(n - 1, 256), 256, 0, s>>>(nodes, n - 1, claimOff, claims);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ 4-wide
// Depth of every binary node by pointer jumping: after round r, anc[i] is the
// 2^r-th ancestor (or -1) and dep[i] the distance to it.
__global__ void k_depth_init(const i32* __restrict__ parent, u32 m, i32* __restrict__ anc, i32* __restrict__ dep) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const i32 p = parent[i];
    anc[i] = p;
    dep[i] = p >= 0 ? 1 : 0;
}
__global__ void k_depth_jump(const i32* __restrict__ anc, const i32* __restrict__ dep, i32* __restrict__ anc2,
                             i32* __restrict__ dep2, u32 m) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const i32 a = anc[i];
    if (a >= 0 && (u32)a < m) {
        dep2[i] = dep[i] + dep[a];
        anc2[i] = anc[a];
    } else {
        dep2[i] = dep[i];
        anc2[i] = -1;
    }
}
__global__ void k_wide_flag(const i32* __restrict__ dep, u32 nInner, u32* __restrict__ flag) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nInner) flag[i] = (dep[i] & 1) == 0 ? 1u : 0u;
}
__device__ __forceinline__ void w4_empty_boxes(Wide4& o) {
    const float inf = __int_as_float(0x7f800000);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        o.lox[k] = inf; o.loy[k] = inf; o.loz[k] = inf;
        o.hix[k] = -inf; o.hiy[k] = -inf; o.hiz[k] = -inf;
        o.child[k] = W4_EMPTY;
    }
}
// One thread per even-depth internal node i: wide node widx[i] takes i's
// children, each internal child replaced by its own two children.
__global__ void k_wide_fill(const Node* __restrict__ nodes, const i32* __restrict__ dep, const u32* __restrict__ widx,
                            u32 n, Wide4* __restrict__ w4, int2* __restrict__ leafW, int2* __restrict__ leafWf,
                            u32* __restrict__ warrive) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 nInner = n - 1;
    if (i >= nInner || (dep[i] & 1)) return;
    const u32 W = widx[i];
    i32 kids[4];
    int nk = 0;
    const i32 ab[2] = {nodes[i].a, nodes[i].b};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const i32 x = ab[c];
        if (x >= 0 && (u32)x < nInner) {
            kids[nk++] = nodes[x].a;
            kids[nk++] = nodes[x].b;
        } else {
            kids[nk++] = x;
        }
    }
    Wide4 o;
    w4_empty_boxes(o);
    for (int k = 0; k < nk; ++k) {
        const i32 x = kids[k];
        if (x >= 0 && (u32)x < nInner) {
            const u32 cw = widx[x];
            o.child[k] = (i32)cw;
            w4[cw].parent = (i32)W;  // the child's own thread never writes these two words
            w4[cw].slot = (u32)k;
        } else {
            o.child[k] = ~nodes[x].b;
            leafW[(u32)x - nInner] = make_int2((i32)W, k);
            leafWf[nodes[x].b] = make_int2((i32)W, k);
        }
    }
    float4* dst = reinterpret_cast<float4*>(&w4[W]);
    const float4* src = reinterpret_cast<const float4*>(&o);
#pragma unroll
    for (int k = 0; k < 7; ++k) dst[k] = src[k];  // boxes + child words
    w4[W].nchild = (u32)nk;
    if (i == 0) { w4[W].parent = -1; w4[W].slot = 0; }
    warrive[W] = 0;
}
// A tree of one leaf (binary node 0 is the leaf): one wide node, one slot.
__global__ void k_wide_single(const Node* __restrict__ nodes, Wide4* __restrict__ w4, int2* __restrict__ leafW,
                              int2* __restrict__ leafWf, u32* __restrict__ warrive, u32* __restrict__ wcount) {
    Wide4 o;
    w4_empty_boxes(o);
    o.child[0] = ~nodes[0].b;
    o.nchild = 1;
    o.parent = -1;
    o.slot = 0;
    o.pad = 0;
    w4[0] = o;
    leafW[0] = make_int2(0, 0);
    leafWf[nodes[0].b] = make_int2(0, 0);
    warrive[0] = 0;
    *wcount = 1;
}
// Number of wide nodes: the scan's last entry plus the last flag.
__global__ void k_wide_count(const i32* __restrict__ dep, const u32* __restrict__ widx, u32 nInner, u32* wcount) {
    *wcount = widx[nInner - 1] + ((dep[nInner - 1] & 1) == 0 ? 1u : 0u);
}

size_t wide_build_scratch_bytes(u32 n) {
    const size_t m = n ? 2 * (size_t)n - 1 : 1;
    return 4 * m * sizeof(i32) + 256 + (size_t)n * sizeof(u32) + 256 + scan_scratch_bytes(n ? n : 1);
}

cudaError_t launch_wide_build(const Node* nodes, const i32* parent, u32 n, Wide4* w4, int2* leafW, int2* leafWf,
                              u32* warrive, u32* wcount, void* scratch, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    if (n == 1) {
        k_wide_single<<<1, 1, 0, s>>>(nodes, w4, leafW, leafWf, warrive, wcount);
        return cudaGetLastError();
    }
    const u32 m = 2 * n - 1;
    char* base = static_cast<char*>(scratch);
    i32* anc = reinterpret_cast<i32*>(base);
    i32* dep = anc + m;
    i32* anc2 = dep + m;
    i32* dep2 = anc2 + m;
    size_t off = ((4 * (size_t)m * sizeof(i32)) + 255) & ~(size_t)255;
    u32* widx = reinterpret_cast<u32*>(base + off);
    off = (off + (size_t)n * sizeof(u32) + 255) & ~(size_t)255;
    void* scanScratch = base + off;
    k_depth_init<<<ceil_div(m, 256), 256, 0, s>>>(parent, m, anc, dep);
    // enough rounds for any depth below m
    int rounds = 1;
    while ((1u << rounds) < m && rounds < 31) ++rounds;
    for (int r = 0; r < rounds; ++r) {
        k_depth_jump<<<ceil_div(m, 256), 256, 0, s>>>(anc, dep, anc2, dep2, m);
        std::swap(anc, anc2);
        std::swap(dep, dep2);
    }
    k_wide_flag<<<ceil_div(n - 1, 256), 256, 0, s>>>(dep, n - 1, widx);
    cudaError_t e = exclusive_scan(widx, n - 1, scanScratch, s);
    if (e != cudaSuccess) return e;
    k_wide_fill<<<ceil_div(n - 1, 256), 256, 0, s>>>(nodes, dep, widx, n, w4, leafW, leafWf, warrive);
    k_wide_count<<<1, 1, 0, s>>>(dep, widx, n - 1, wcount);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ refit
// buildSweptLeaf_Tri / buildLeaf_Tri (bvh.metal:260-351) + bottomUpBoxes
// (bvh.metal:510-586).  One thread per leaf writes its box, then climbs: the
// first thread to arrive at a parent stops, the second combines both children
// and continues.  Arrival counters are never reset between refits: every
// internal node receives exactly two arrivals per refit (one per child it
// lists), so an even old value means "first", odd means "second".  Karras
// zeroes them at build.
// Memory order: the arrival is an acq_rel atomic at GPU scope: it releases
// this thread's box stores and acquires the sibling's; the children are then
// read with L1-bypassing loads.
// Box coordinates only: the child / face words (w) are left alone, so no
// read-modify-write is needed.
__device__ __forceinline__ void store_box(Node* nd, f3 lo, f3 hi) {
    float* p = reinterpret_cast<float*>(nd);
    __stcg(reinterpret_cast<float2*>(p), make_float2(lo.x, lo.y));
    __stcg(p + 2, lo.z);
    __stcg(reinterpret_cast<float2*>(p + 4), make_float2(hi.x, hi.y));
    __stcg(p + 6, hi.z);
}

__device__ __forceinline__ u32 arrive_acq_rel(u32* counter) {
    u32 old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(counter) : "memory");
    return old;
}

// Arrival at a wide node: counts 0 .. wrap, then back to 0 (no reset needed
// between refits); acq_rel as arrive_acq_rel.
__device__ __forceinline__ u32 arrive_inc_acq_rel(u32* counter, u32 wrap) {
    u32 old;
    asm volatile("atom.inc.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(counter), "r"(wrap) : "memory");
    return old;
}

// Wide climb: write this box into the parent's slot; the last of the node's
// children to arrive takes the union of its slots (in slot order) to the
// grandparent, and the root's union becomes the binary root box.
__device__ __forceinline__ void climb_wide(const RefitJob& J, u32 i, f3 lo, f3 hi, u32* status) {
    const int2 ws = J.leafW[i];
    i32 w = ws.x;
    u32 s = (u32)ws.y;
    const u32 cap = J.n > 1 ? J.n - 1 : 1;
    for (u32 step = 0; step < 128; ++step) {
        if (w < 0 || (u32)w >= cap || s > 3) break;
        Wide4* W = J.w4 + w;
        __stcg(&W->lox[s], lo.x); __stcg(&W->loy[s], lo.y); __stcg(&W->loz[s], lo.z);
        __stcg(&W->hix[s], hi.x); __stcg(&W->hiy[s], hi.y); __stcg(&W->hiz[s], hi.z);
        const u32 nc = __ldcg(&W->nchild);
        const i32 par = __ldcg(&W->parent);
        const u32 ps = __ldcg(&W->slot);
        if (nc == 0 || nc > 4) break;
        if (arrive_inc_acq_rel(&J.warrive[w], nc - 1) != nc - 1) return;
        const float4* p = reinterpret_cast<const float4*>(W);
        const float4 lx = __ldcg(p), ly = __ldcg(p + 1), lz = __ldcg(p + 2);
        const float4 hx = __ldcg(p + 3), hy = __ldcg(p + 4), hz = __ldcg(p + 5);
        lo = mk(lx.x, ly.x, lz.x);
        hi = mk(hx.x, hy.x, hz.x);
        if (nc > 1) { lo = vmin(lo, mk(lx.y, ly.y, lz.y)); hi = vmax(hi, mk(hx.y, hy.y, hz.y)); }
        if (nc > 2) { lo = vmin(lo, mk(lx.z, ly.z, lz.z)); hi = vmax(hi, mk(hx.z, hy.z, hz.z)); }
        if (nc > 3) { lo = vmin(lo, mk(lx.w, ly.w, lz.w)); hi = vmax(hi, mk(hx.w, hy.w, hz.w)); }
        if (par < 0) {
            store_box(&J.nodes[0], lo, hi);
            return;
        }
        w = par;
        s = ps;
    }
    atomicOr(status, ST_ITER_CAP);
}

__device__ __forceinline__ u32 job_of(const RefitJob* __restrict__ jobs, u32 numJobs, u32 g) {
    u32 lo = 0, hi = numJobs;  // largest j with leafBase <= g
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) >> 1;
        if (jobs[mid].leafBase <= g) lo = mid; else hi = mid;
    }
    return lo;
}

// Range mode, leaf pass: the boxes of this block's 16-leaf groups and of the
// whole block (256 consecutive sorted leaves i0 .. i0 + 255 of job J, i the
// thread's leaf), and the slot boxes of the wide nodes whose range lies in
// the block, from the leaf boxes in shared memory.  Every thread of the block
// calls this.  Min and max of a set do not depend on the order they are taken
// in, so the unions below equal the bottom-up ones.
__device__ __forceinline__ void range_block_boxes(const RefitJob& J, u32 i, bool has, f3 lo, f3 hi) {
    __shared__ float sh_box[8][6];
    __shared__ float sh_leaf[6][256];
    __shared__ float sh_g16[6][16];  // boxes of the block's 16-leaf groups
    const float inf = __int_as_float(0x7F800000);
    float v[6] = {has ? lo.x : inf, has ? lo.y : inf, has ? lo.z : inf,
                  has ? hi.x : -inf, has ? hi.y : -inf, has ? hi.z : -inf};
#pragma unroll
    for (int k = 0; k < 6; ++k) sh_leaf[k][threadIdx.x] = v[k];
    const u32 lane = threadIdx.x & 31u;
#pragma unroll
    for (int off = 8; off >= 1; off >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            v[k] = fminf(v[k], __shfl_xor_sync(0xFFFFFFFFu, v[k], off));
            v[3 + k] = fmaxf(v[3 + k], __shfl_xor_sync(0xFFFFFFFFu, v[3 + k], off));
        }
    }
    if ((lane & 15u) == 0) {
        store_box(J.bb16 + ((J.leafBase + i) >> 4), mk(v[0], v[1], v[2]), mk(v[3], v[4], v[5]));
#pragma unroll
        for (int k = 0; k < 6; ++k) sh_g16[k][threadIdx.x >> 4] = v[k];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v[k] = fminf(v[k], __shfl_xor_sync(0xFFFFFFFFu, v[k], 16));
        v[3 + k] = fmaxf(v[3 + k], __shfl_xor_sync(0xFFFFFFFFu, v[3 + k], 16));
    }
    if (lane == 0)
        for (int k = 0; k < 6; ++k) sh_box[threadIdx.x >> 5][k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (u32 w = 1; w < (blockDim.x >> 5); ++w)
            for (int k = 0; k < 3; ++k) {
                v[k] = fminf(v[k], sh_box[w][k]);
                v[3 + k] = fmaxf(v[3 + k], sh_box[w][3 + k]);
            }
        store_box(J.bb256 + ((J.leafBase + i) >> 8), mk(v[0], v[1], v[2]), mk(v[3], v[4], v[5]));
    }
    // the wide nodes inside this block: their parents' slots
    const u32 gb = (J.leafBase + i) >> 8, i0 = i & ~255u;
    const u32 eb = J.blkOff[gb], ee = J.blkOff[gb + 1];
    for (u32 q = eb + threadIdx.x; q < ee; q += blockDim.x) {
        const uint4 r = J.blkEnt[q];  // (parent, slot, first, last)
        if (r.z < i0 || r.w > i0 + 255u || r.z > r.w || r.y > 3u) continue;
        float b[6] = {inf, inf, inf, -inf, -inf, -inf};
        // single leaves up to a 16-leaf boundary, whole groups, single leaves
        const u32 L = r.z - i0, e = r.w - i0 + 1;
        u32 s16 = (L + 15u) & ~15u, e16 = e & ~15u;
        if (s16 >= e16) { s16 = e; e16 = e; }
        auto take = [&](const float (*src)[256], u32 l) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                b[k] = fminf(b[k], src[k][l]);
                b[3 + k] = fmaxf(b[3 + k], src[3 + k][l]);
            }
        };
        for (u32 l = L; l < s16; ++l) take(sh_leaf, l);
        for (u32 gq = s16 >> 4; gq < (e16 >> 4); ++gq) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                b[k] = fminf(b[k], sh_g16[k][gq]);
                b[3 + k] = fmaxf(b[3 + k], sh_g16[3 + k][gq]);
            }
        }
        for (u32 l = e16; l < e; ++l) take(sh_leaf, l);
        Wide4* W = J.w4 + r.x;
        W->lox[r.y] = b[0]; W->loy[r.y] = b[1]; W->loz[r.y] = b[2];
        W->hix[r.y] = b[3]; W->hiy[r.y] = b[4]; W->hiz[r.y] = b[5];
    }
}

__device__ __forceinline__ void box_union(f3& lo, f3& hi, const Node* nd) {
    const float4* p = reinterpret_cast<const float4*>(nd);
    const float4 a = __ldcg(p), b = __ldcg(p + 1);
    lo = mk(fminf(lo.x, a.x), fminf(lo.y, a.y), fminf(lo.z, a.z));
    hi = mk(fmaxf(hi.x, b.x), fmaxf(hi.y, b.y), fmaxf(hi.z, b.z));
}

// Union of the leaf boxes of sorted leaves [L, R] of job J by a group of G
// threads (thread g of the group, g < G), reduced over groups of RED lanes
// (RED divides 32, groups aligned; RED = G up to a warp): the range
// splits into single leaves up to a 16-leaf boundary, 16-leaf blocks up to a
// 256-leaf boundary, 256-leaf blocks, then 16-leaf blocks and single leaves
// again; the lanes take those pieces in turn (four loads in flight per lane)
// and the group reduces.  Every lane of the group gets the union.
template <int G, int RED = G>
__device__ __forceinline__ void range_union_group(const RefitJob& J, u32 L, u32 R, u32 g, f3& lo, f3& hi) {
    const float inf = __int_as_float(0x7F800000);
    const Node* leaves = J.nodes + (J.n - 1);
    const u32 b = J.leafBase;  // a multiple of 256
    const u32 e = R + 1;
    u32 s16 = (L + 15u) & ~15u, e16 = e & ~15u;
    if (s16 >= e16) { s16 = e; e16 = e; }
    u32 s256 = (s16 + 255u) & ~255u, e256 = e16 & ~255u;
    if (s256 >= e256) { s256 = e16; e256 = e16; }
    const u32 n0 = s16 - L, n1 = (s256 - s16) >> 4, n2 = (e256 - s256) >> 8, n3 = (e16 - e256) >> 4;
    const u32 total = n0 + n1 + n2 + n3 + (e - e16);
    auto piece = [&](u32 r) -> const Node* {
        if (r < n0) return leaves + L + r;
        if ((r -= n0) < n1) return J.bb16 + ((b + s16) >> 4) + r;
        if ((r -= n1) < n2) return J.bb256 + ((b + s256) >> 8) + r;
        if ((r -= n2) < n3) return J.bb16 + ((b + e256) >> 4) + r;
        return leaves + e16 + (r - n3);
    };
    float v[6] = {inf, inf, inf, -inf, -inf, -inf};
    u32 q = g;
    for (; q + 3 * G < total; q += 4 * G) {
        float4 a[4], c[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float4* p = reinterpret_cast<const float4*>(piece(q + u * G));
            a[u] = __ldcg(p);
            c[u] = __ldcg(p + 1);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            v[0] = fminf(v[0], a[u].x); v[1] = fminf(v[1], a[u].y); v[2] = fminf(v[2], a[u].z);
            v[3] = fmaxf(v[3], c[u].x); v[4] = fmaxf(v[4], c[u].y); v[5] = fmaxf(v[5], c[u].z);
        }
    }
    for (; q < total; q += G) {
        const float4* p = reinterpret_cast<const float4*>(piece(q));
        const float4 a = __ldcg(p), c = __ldcg(p + 1);
        v[0] = fminf(v[0], a.x); v[1] = fminf(v[1], a.y); v[2] = fminf(v[2], a.z);
        v[3] = fmaxf(v[3], c.x); v[4] = fmaxf(v[4], c.y); v[5] = fmaxf(v[5], c.z);
    }
#pragma unroll
    for (int off = RED / 2; off >= 1; off >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            v[k] = fminf(v[k], __shfl_xor_sync(0xFFFFFFFFu, v[k], off));
            v[3 + k] = fmaxf(v[3 + k], __shfl_xor_sync(0xFFFFFFFFu, v[3 + k], off));
        }
    }
    lo = mk(v[0], v[1], v[2]);
    hi = mk(v[3], v[4], v[5]);
}

// Union of the leaf boxes of sorted leaves [L, R] of job J by a whole block
// (every thread calls this; each gets the union).
__device__ __forceinline__ void range_union_block(const RefitJob& J, u32 L, u32 R, f3& lo, f3& hi) {
    __shared__ float sh_red[8][6];
    range_union_group<256, 32>(J, L, R, threadIdx.x, lo, hi);  // pieces over the block, reduced per warp
    // then across the warps
    if ((threadIdx.x & 31u) == 0) {
        sh_red[threadIdx.x >> 5][0] = lo.x; sh_red[threadIdx.x >> 5][1] = lo.y; sh_red[threadIdx.x >> 5][2] = lo.z;
        sh_red[threadIdx.x >> 5][3] = hi.x; sh_red[threadIdx.x >> 5][4] = hi.y; sh_red[threadIdx.x >> 5][5] = hi.z;
    }
    __syncthreads();
    for (u32 w = 0; w < (blockDim.x >> 5); ++w) {
        lo = mk(fminf(lo.x, sh_red[w][0]), fminf(lo.y, sh_red[w][1]), fminf(lo.z, sh_red[w][2]));
        hi = mk(fmaxf(hi.x, sh_red[w][3]), fmaxf(hi.y, sh_red[w][4]), fmaxf(hi.z, sh_red[w][5]));
    }
    __syncthreads();
}

// Second pass of the range refit.  Blocks [0, nmed): 8 lanes per record of
// the medium list (wide nodes whose range spans more than one 256-leaf
// block); then one block per record of the huge list (ranges of more than
// RANGE_HUGE leaves); then one block per job for the tree's root box (its
// whole range).  A record sets its parent's slot from its sorted-leaf range.
static constexpr u32 RANGE_HUGE = 16384;

__device__ __forceinline__ void put_slot(const RefitJob& J, uint4 r, f3 lo, f3 hi) {
    Wide4* W = J.w4 + r.x;
    const u32 k = r.y & 3u;
    W->lox[k] = lo.x; W->loy[k] = lo.y; W->loz[k] = lo.z;
    W->hix[k] = hi.x; W->hiy[k] = hi.y; W->hiz[k] = hi.z;
}

__global__ void __launch_bounds__(256) k_refit_ranges(const RefitJob* __restrict__ jobs, u32 numJobs,
                                                      const uint4* __restrict__ med, u32 nmed,
                                                      const uint4* __restrict__ huge, u32 nhuge) {
    const u32 medBlocks = (nmed + 31) / 32;  // 32 records of 8 lanes per block
    const u32 lane = threadIdx.x & 31u;
    if (blockIdx.x < medBlocks) {
        const u32 grp = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
        uint4 r = make_uint4(0u, 0u, 1u, 0u);  // empty: no pieces
        const RefitJob* J = jobs;
        if (grp < nmed) {
            r = med[grp];
            const u32 j = r.y >> 2;
            if (j < numJobs && jobs[j].ranges && r.z <= r.w && r.w < jobs[j].n) J = jobs + j;
            else r = make_uint4(0u, 0u, 1u, 0u);
        }
        f3 lo, hi;
        range_union_group<8>(*J, r.z, r.w, lane & 7u, lo, hi);
        if ((lane & 7u) == 0 && r.z <= r.w) put_slot(*J, r, lo, hi);
        return;
    }
    u32 b = blockIdx.x - medBlocks;
    if (b < nhuge) {
        uint4 r = huge[b];
        const u32 j = r.y >> 2;
        const bool ok = j < numJobs && jobs[j].ranges && r.z <= r.w && r.w < jobs[j].n;  // uniform
        if (!ok) return;
        f3 lo, hi;
        range_union_block(jobs[j], r.z, r.w, lo, hi);
        if (threadIdx.x == 0) put_slot(jobs[j], r, lo, hi);
        return;
    }
    b -= nhuge;
    if (b >= numJobs || !jobs[b].ranges || jobs[b].n == 0) return;
    f3 lo, hi;
    range_union_block(jobs[b], 0u, jobs[b].n - 1, lo, hi);
    if (threadIdx.x == 0) store_box(jobs[b].nodes, lo, hi);
}

// Range-refit records of the wide nodes (see launch_range_lists).
__global__ void __launch_bounds__(256) k_range_records(const RefitJob* __restrict__ jobs, u32 numJobs,
                                                       u32 totalLeaves, u32* __restrict__ blkCnt,
                                                       const u32* __restrict__ blkOff, uint4* __restrict__ blkEnt,
                                                       uint4* __restrict__ big, u32 bigCap, u32* __restrict__ bigCnt,
                                                       int fill) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= totalLeaves) return;
    const u32 j = job_of(jobs, numJobs, g);
    const RefitJob& J = jobs[j];
    if (!J.ranges) return;
    const u32 c = g - J.leafBase;
    if (c >= *J.wcount) return;
    const Wide4& W = J.w4[c];
    if (W.parent < 0 || W.slot > 3u) return;  // the root: its box is the job's root pass
    const uint2 r = J.wrange[c];
    if (r.x > r.y || r.y >= J.n) return;
    const uint4 rec = make_uint4((u32)W.parent, W.slot, r.x, r.y);
    if ((r.x >> 8) == (r.y >> 8)) {
        const u32 b = (J.leafBase + r.x) >> 8;
        const u32 at = atomicAdd(&blkCnt[b], 1u);
        if (fill) blkEnt[blkOff[b] + at] = rec;
    } else {
        // medium records from the front of `big`, huge ones from its back
        const bool huge = r.y - r.x >= RANGE_HUGE;
        const u32 at = atomicAdd(&bigCnt[huge ? 1 : 0], 1u);
        if (fill) big[huge ? bigCap - 1 - at : at] = make_uint4(rec.x, rec.y | (j << 2), rec.z, rec.w);
    }
}

cudaError_t launch_range_lists(const RefitJob* jobsDev, u32 numJobs, u32 totalLeaves, u32* blkCnt, u32* blkOff,
                               uint4* blkEnt, uint4* big, u32 bigCap, u32* bigCnt, void* scanScratch,
                               cudaStream_t s) {
    const u32 nb = totalLeaves / 256 + 1;
    cudaError_t e = cudaMemsetAsync(blkCnt, 0, 4 * (size_t)(nb + 1), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(bigCnt, 0, 8, s);
    if (e != cudaSuccess || totalLeaves == 0) return e;
    const int grid = ceil_div(totalLeaves, 256);
    k_range_records<<<grid, 256, 0, s>>>(jobsDev, numJobs, totalLeaves, blkCnt, blkOff, blkEnt, big, bigCap, bigCnt,
                                         0);
    e = cudaMemcpyAsync(blkOff, blkCnt, 4 * (size_t)(nb + 1), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = exclusive_scan(blkOff, nb + 1, scanScratch, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(blkCnt, 0, 4 * (size_t)(nb + 1), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(bigCnt, 0, 8, s);
    if (e != cudaSuccess) return e;
    k_range_records<<<grid, 256, 0, s>>>(jobsDev, numJobs, totalLeaves, blkCnt, blkOff, blkEnt, big, bigCap, bigCnt,
                                         1);
    return cudaGetLastError();
}

// ---- range refit of a consistent binary tree (the standalone LBVH)
// The swept or static box of face f (buildLeaf_Tri / buildSweptLeaf_Tri).
__device__ __forceinline__ void face_box(const RefitJob& J, u32 f, f3& lo, f3& hi) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const u32 gv = J.voff + J.facets[3 * f + k];
        const f3 p = J.x4 ? ld(J.x4, gv) : ldp(J.x3, gv);
        f3 a = p, b = p;
        if (J.swept) {
            const f3 vv = J.v4 ? ld(J.v4, gv) : ldp(J.v3, gv);
            const f3 sp = p + vv * J.dt;
            a = vmin(p, sp);
            b = vmax(p, sp);
        }
        if (k == 0) { lo = a; hi = b; } else { lo = vmin(lo, a); hi = vmax(hi, b); }
    }
}

// Face pass: thread f is face f, so the facet and vertex reads stream in the
// caller's order; its box goes to its sorted slot rank[f] of lbox (one full
// 32-byte sector).  In sorted-leaf order these reads were random gathers,
// several sectors per leaf.
__global__ void __launch_bounds__(256) k_refit_bin_faces(RefitJob J, const u32* __restrict__ rank,
                                                         float4* __restrict__ lbox) {
    const u32 f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= J.n) return;
    f3 lo, hi;
    face_box(J, f, lo, hi);
    const u32 r = rank[f];
    __stcg(lbox + 2 * (size_t)r, make_float4(lo.x, lo.y, lo.z, __int_as_float(-1)));  // the leaf node's a
    __stcg(lbox + 2 * (size_t)r + 1, make_float4(hi.x, hi.y, hi.z, __uint_as_float(f)));  // and b (its face)
}

// Leaf pass: thread i is sorted leaf i (leaf node n - 1 + i, face in .b);
// its box (from lbox when the face pass ran, else gathered here) goes to the
// leaf node, the block's 16- and 256-leaf boxes to bb16 / bb256, and
// internal node i (whose range has leaf i at one end) gets its box here when
// its range stays in the block.
__global__ void __launch_bounds__(256) k_refit_bin_leaves(RefitJob J, const uint2* __restrict__ range,
                                                          const float4* __restrict__ lbox) {
    __shared__ float sh_leaf[6][256];
    __shared__ float sh_g16[6][16];
    __shared__ float sh_box[8][6];
    const u32 n = J.n;
    const u32 i0 = blockIdx.x * 256u, i = i0 + threadIdx.x;
    const bool has = i < n;
    const u32 li = has ? i : n - 1;
    Node* nodes = J.nodes;
    f3 lo, hi;
    if (lbox) {
        // the whole leaf node (box, a = -1, b = face) in two 16-byte stores:
        // no read of the node to merge a partial write
        const float4 a = __ldcs(lbox + 2 * (size_t)li), b = __ldcs(lbox + 2 * (size_t)li + 1);
        lo = mk(a.x, a.y, a.z);
        hi = mk(b.x, b.y, b.z);
        if (has) {
            float4* nd = reinterpret_cast<float4*>(&nodes[n - 1 + i]);
            __stcg(nd, a);
            __stcg(nd + 1, b);
        }
    } else {
        face_box(J, (u32)__ldcg(&nodes[n - 1 + li].b), lo, hi);
        if (has) store_box(&nodes[n - 1 + i], lo, hi);
    }
    const float inf = __int_as_float(0x7F800000);
    float v[6] = {has ? lo.x : inf, has ? lo.y : inf, has ? lo.z : inf,
                  has ? hi.x : -inf, has ? hi.y : -inf, has ? hi.z : -inf};
#pragma unroll
    for (int k = 0; k < 6; ++k) sh_leaf[k][threadIdx.x] = v[k];
    const u32 lane = threadIdx.x & 31u;
#pragma unroll
    for (int off = 8; off >= 1; off >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            v[k] = fminf(v[k], __shfl_xor_sync(0xFFFFFFFFu, v[k], off));
            v[3 + k] = fmaxf(v[3 + k], __shfl_xor_sync(0xFFFFFFFFu, v[3 + k], off));
        }
    }
    if ((lane & 15u) == 0) {
        store_box(J.bb16 + (i >> 4), mk(v[0], v[1], v[2]), mk(v[3], v[4], v[5]));
#pragma unroll
        for (int k = 0; k < 6; ++k) sh_g16[k][threadIdx.x >> 4] = v[k];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v[k] = fminf(v[k], __shfl_xor_sync(0xFFFFFFFFu, v[k], 16));
        v[3 + k] = fmaxf(v[3 + k], __shfl_xor_sync(0xFFFFFFFFu, v[3 + k], 16));
    }
    if (lane == 0)
        for (int k = 0; k < 6; ++k) sh_box[threadIdx.x >> 5][k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (u32 w = 1; w < 8; ++w)
            for (int k = 0; k < 3; ++k) {
                v[k] = fminf(v[k], sh_box[w][k]);
                v[3 + k] = fmaxf(v[3 + k], sh_box[w][3 + k]);
            }
        store_box(J.bb256 + (i0 >> 8), mk(v[0], v[1], v[2]), mk(v[3], v[4], v[5]));
    }
    if (i + 1 >= n) return;  // no internal node i
    const uint2 r = range[i];
    if ((r.x >> 8) != (i0 >> 8) || (r.y >> 8) != (i0 >> 8) || r.x > r.y) return;  // a big node
    float b[6] = {inf, inf, inf, -inf, -inf, -inf};
    const u32 L = r.x - i0, e = r.y - i0 + 1;
    u32 s16 = (L + 15u) & ~15u, e16 = e & ~15u;
    if (s16 >= e16) { s16 = e; e16 = e; }
    for (u32 l = L; l < s16; ++l)
#pragma unroll
        for (int k = 0; k < 3; ++k) { b[k] = fminf(b[k], sh_leaf[k][l]); b[3 + k] = fmaxf(b[3 + k], sh_leaf[3 + k][l]); }
    for (u32 q = s16 >> 4; q < (e16 >> 4); ++q)
#pragma unroll
        for (int k = 0; k < 3; ++k) { b[k] = fminf(b[k], sh_g16[k][q]); b[3 + k] = fmaxf(b[3 + k], sh_g16[3 + k][q]); }
    for (u32 l = e16; l < e; ++l)
#pragma unroll
        for (int k = 0; k < 3; ++k) { b[k] = fminf(b[k], sh_leaf[k][l]); b[3 + k] = fmaxf(b[3 + k], sh_leaf[3 + k][l]); }
    store_box(&nodes[i], mk(b[0], b[1], b[2]), mk(b[3], b[4], b[5]));
}

// Big nodes (ranges across blocks): 8 lanes per node of big, then a block
// per node of huge (ranges of BIN_RANGE_HUGE leaves or more).
__global__ void __launch_bounds__(256) k_refit_bin_ranges(RefitJob J, const uint2* __restrict__ range,
                                                          const u32* __restrict__ big, u32 nbig,
                                                          const u32* __restrict__ huge, u32 nhuge) {
    const u32 medBlocks = (nbig + 31) / 32;
    if (blockIdx.x < medBlocks) {
        const u32 grp = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
        u32 node = 0;
        uint2 r = make_uint2(1u, 0u);  // empty
        if (grp < nbig) {
            node = big[grp];
            r = range[node];
        }
        f3 lo, hi;
        range_union_group<8>(J, r.x, r.y, threadIdx.x & 7u, lo, hi);
        if ((threadIdx.x & 7u) == 0 && r.x <= r.y) store_box(&J.nodes[node], lo, hi);
        return;
    }
    const u32 b = blockIdx.x - medBlocks;
    if (b >= nhuge) return;
    const u32 node = huge[b];
    const uint2 r = range[node];
    if (r.x > r.y || r.y >= J.n) return;  // uniform over the block
    f3 lo, hi;
    range_union_block(J, r.x, r.y, lo, hi);
    if (threadIdx.x == 0) store_box(&J.nodes[node], lo, hi);
}

__global__ void k_leaf_vids(const u32* __restrict__ idx, const u32* __restrict__ facets, u32 n,
                            uint4* __restrict__ lvid) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u32 f = idx[i];
    lvid[i] = make_uint4(facets[3 * f], facets[3 * f + 1], facets[3 * f + 2], f);
}

void launch_leaf_vids(const u32* idx, const u32* facets, u32 n, uint4* lvid, cudaStream_t s) {
    if (n) k_leaf_vids<<<ceil_div(n, 256), 256, 0, s>>>(idx, facets, n, lvid);
}

// Sorted-leaf rank of each face: rank[idx[i]] = i.
__global__ void k_leaf_rank(const u32* __restrict__ idx, u32 n, u32* __restrict__ rank) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rank[idx[i]] = i;
}

void launch_leaf_rank(const u32* idx, u32 n, u32* rank, cudaStream_t s) {
    if (n) k_leaf_rank<<<ceil_div(n, 256), 256, 0, s>>>(idx, n, rank);
}

void launch_refit_bin(const RefitJob& J, const uint2* range, const u32* big, u32 nbig, const u32* huge, u32 nhuge,
                      const u32* rank, float4* lbox, cudaStream_t s) {
    if (J.n == 0) return;
    if (rank && lbox) k_refit_bin_faces<<<ceil_div(J.n, 256), 256, 0, s>>>(J, rank, lbox);
    k_refit_bin_leaves<<<ceil_div(J.n, 256), 256, 0, s>>>(J, range, rank && lbox ? lbox : nullptr);
    const u32 blocks = (nbig + 31) / 32 + nhuge;
    if (blocks) k_refit_bin_ranges<<<blocks, 256, 0, s>>>(J, range, big, nbig, huge, nhuge);
}

void launch_refit_ranges(const RefitJob* jobsDev, u32 numJobs, const uint4* big, u32 bigCap, u32 nmed, u32 nhuge,
                         cudaStream_t s) {
    const u32 blocks = (nmed + 31) / 32 + nhuge + numJobs;
    if (blocks) k_refit_ranges<<<blocks, 256, 0, s>>>(jobsDev, numJobs, big, nmed, big + (bigCap - nhuge), nhuge);
}

__global__ void __launch_bounds__(256) k_refit(const RefitJob* __restrict__ jobs, u32 numJobs, u32 totalLeaves,
                                               u32* status) {
    __shared__ u32 sh_ext[8];
    __shared__ u32 sh_j0;
    // threads past the last leaf do the work of the last leaf and drop it:
    // every thread reaches the block reduction below
    const u32 g0 = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = g0 < totalLeaves;
    const u32 g = valid ? g0 : totalLeaves - 1;
    const u32 j = job_of(jobs, numJobs, g);  // the job owning leaf g
    if (threadIdx.x == 0) sh_j0 = j;
    const RefitJob J = jobs[j];
    const u32 n = J.n;
    const u32 i = g - J.leafBase;
    Node* nodes = J.nodes;
    // jobs' leaves may be padded to a multiple of 256 (range mode): the
    // padding threads take the job's last leaf and drop it
    const bool pad = i >= n;
    const u32 li = pad ? n - 1 : i;
    const u32 leaf = n - 1 + li;
    // root only: the tree is not built; levels: thread i is face i (its slot
    // comes from leafWf); ranges: thread i is sorted leaf i
    u32 f, vid[3];
    if (J.ranges && J.lvid) {
        const uint4 q = J.lvid[li];
        f = q.w; vid[0] = q.x; vid[1] = q.y; vid[2] = q.z;
    } else {
        f = J.ranges ? J.idx[li] : ((J.rootOnly || J.levels) ? li : (u32)__ldcg(&nodes[leaf].b));
        vid[0] = J.facets[3 * f]; vid[1] = J.facets[3 * f + 1]; vid[2] = J.facets[3 * f + 2];
    }
    f3 lo, hi;
    float ext = 0.f;
    f3 P[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const u32 gv = J.voff + vid[k];
        P[k] = J.x4 ? ld(J.x4, gv) : ldp(J.x3, gv);
    }
    if (J.fpos && valid && !pad) {
        float4* o = J.fpos + 3 * (size_t)f;
#pragma unroll
        for (int k = 0; k < 3; ++k) o[k] = make_float4(P[k].x, P[k].y, P[k].z, __uint_as_float(vid[k]));
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        u32 gv = J.voff + vid[k];
        f3 p = P[k];
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
        const f3 P0 = P[0], P1 = P[1], P2 = P[2];
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
        // H1 extent: one atomic per block for the block's first job (most
        // blocks hold one job), per warp and job for the others
        __syncthreads();
        const u32 j0 = sh_j0;
        const u32 eb = (valid && !pad) ? __float_as_uint(ext) : 0u;  // positive floats order as ints
        const u32 e0 = __reduce_max_sync(0xFFFFFFFFu, j == j0 ? eb : 0u);
        if ((threadIdx.x & 31) == 0) sh_ext[threadIdx.x >> 5] = e0;
        if (valid && j != j0 && J.selfMargin > 0.f) {
            const unsigned act = __activemask();
            const unsigned peers = __match_any_sync(act, (unsigned long long)J.maxExt);
            const u32 e = __reduce_max_sync(peers, eb);
            if ((threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) atomicMax(J.maxExt, e);
        }
        __syncthreads();
        if (threadIdx.x == 0 && jobs[j0].selfMargin > 0.f) {
            u32 e = 0;
            for (u32 w = 0; w < (blockDim.x >> 5); ++w) e = max(e, sh_ext[w]);
            atomicMax(jobs[j0].maxExt, e);
        }
        // range mode: a block holds 256 consecutive sorted leaves of one job
        if (jobs[j0].ranges) range_block_boxes(J, i, valid && !pad, lo, hi);
        if (!valid || pad) return;
    }
    if (J.ranges) {
        store_box(&nodes[leaf], lo, hi);
        const int2 ws = J.leafW[i];
        if (ws.x < 0 || (u32)ws.x >= (n > 1 ? n - 1 : 1u) || ws.y < 0 || ws.y > 3) {
            atomicOr(status, ST_ITER_CAP);
            return;
        }
        Wide4* W = J.w4 + ws.x;
        const int k = ws.y;
        W->lox[k] = lo.x; W->loy[k] = lo.y; W->loz[k] = lo.z;
        W->hix[k] = hi.x; W->hiy[k] = hi.y; W->hiz[k] = hi.z;
        return;
    }
    if (J.rootOnly) {
        // union of the leaf boxes, one atomic per warp and job
        const unsigned act = __activemask();
        const unsigned peers = __match_any_sync(act, (unsigned long long)J.rootAcc);
        const u32 v[6] = {ford(lo.x), ford(lo.y), ford(lo.z), ford(hi.x), ford(hi.y), ford(hi.z)};
        u32 r[6];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            r[k] = __reduce_min_sync(peers, v[k]);
            r[3 + k] = __reduce_max_sync(peers, v[3 + k]);
        }
        if ((threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                atomicMin(&J.rootAcc[k], r[k]);
                atomicMax(&J.rootAcc[3 + k], r[3 + k]);
            }
        }
        return;
    }
    if (J.w4 && J.levels) {
        const int2 ws = J.leafWf[f];
        if (ws.x < 0 || (u32)ws.x >= (n > 1 ? n - 1 : 1u) || ws.y < 0 || ws.y > 3) {
            atomicOr(status, ST_ITER_CAP);
            return;
        }
        Wide4* W = J.w4 + ws.x;
        const int k = ws.y;
        W->lox[k] = lo.x; W->loy[k] = lo.y; W->loz[k] = lo.z;
        W->hix[k] = hi.x; W->hiy[k] = hi.y; W->hiz[k] = hi.z;
        return;
    }
    if (J.w4) {
        climb_wide(J, i, lo, hi, status);
        return;
    }
    store_box(&nodes[leaf], lo, hi);
    if (n == 1) return;
    const u32 numInner = n - 1;
    // Climb: deliver this node's arrival to every internal node that claims
    // it as a child (one claimant in a consistent tree, any number in the
    // reference's tree over runs of equal codes); the second arrival at a
    // claimant combines it and climbs on from there.  Further completed
    // claimants wait in a bounded pending list.  The climbing thread keeps
    // the box of the node it carries in registers and, at a claimant, loads
    // only the other child's box.
    constexpr int PENDING = 16;
    u32 pending[PENDING];
    int np = 0;
    u32 child = leaf;
    f3 clo = lo, chi = hi;
    bool have_box = true;  // clo/chi hold child's box (false for a resumed pending node)
    const u32 nClaims = 2 * (n - 1);
    for (u32 step = 0; step < 2 * n; ++step) {
        const u32 cs = child ? __ldcg(&J.claimOff[child - 1]) : 0u;
        const u32 ce = __ldcg(&J.claimOff[child]);
        i32 next = -1;
        f3 nlo = clo, nhi = chi;
        if (ce < cs || ce > nClaims) { atomicOr(status, ST_ITER_CAP); return; }
        for (u32 k = cs; k < ce; ++k) {
            const i32 par = __ldcg(&J.claims[k]);
            if (par < 0 || (u32)par >= numInner) { atomicOr(status, ST_ITER_CAP); continue; }
            const i32 ca = __ldcg(&nodes[par].a), cb = __ldcg(&nodes[par].b);
            u32 old = arrive_acq_rel(&J.visits[par]);
            if ((old & 1u) == 0u) continue;  // first arrival: the sibling's thread combines
            if (ca < 0 || (u32)ca >= 2 * n - 1 || cb < 0 || (u32)cb >= 2 * n - 1) {
                atomicOr(status, ST_ITER_CAP);
                continue;
            }
            f3 plo, phi;
            const bool mineA = have_box && (u32)ca == child, mineB = have_box && (u32)cb == child;
            if (mineA || mineB) {
                const float4* O = reinterpret_cast<const float4*>(&nodes[mineA ? cb : ca]);
                const float4 o0 = __ldcg(O), o1 = __ldcg(O + 1);
                const f3 olo = mk(o0.x, o0.y, o0.z), ohi = mk(o1.x, o1.y, o1.z);
                // operands in (a, b) order, as the combine of two loaded boxes
                plo = mineA ? vmin(clo, olo) : vmin(olo, clo);
                phi = mineA ? vmax(chi, ohi) : vmax(ohi, chi);
            } else {
                const float4* A = reinterpret_cast<const float4*>(&nodes[ca]);
                const float4* B = reinterpret_cast<const float4*>(&nodes[cb]);
                float4 a0 = __ldcg(A), a1 = __ldcg(A + 1), b0 = __ldcg(B), b1 = __ldcg(B + 1);
                plo = vmin(mk(a0.x, a0.y, a0.z), mk(b0.x, b0.y, b0.z));
                phi = vmax(mk(a1.x, a1.y, a1.z), mk(b1.x, b1.y, b1.z));
            }
            store_box(&nodes[par], plo, phi);
            if (next < 0) { next = par; nlo = plo; nhi = phi; }
            else if (np < PENDING) pending[np++] = (u32)par;
            else atomicOr(status, ST_ITER_CAP);
        }
        if (next < 0) {
            if (np == 0) return;  // root reached, first arrival, or an unclaimed node
            next = (i32)pending[--np];
            have_box = false;     // its box is in memory (stored above)
        } else {
            have_box = true;
            clo = nlo;
            chi = nhi;
        }
        child = (u32)next;
    }
    atomicOr(status, ST_ITER_CAP);
}

__global__ void k_refit_roots(const RefitJob* __restrict__ jobs, u32 numJobs) {
    const u32 j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= numJobs || !jobs[j].rootOnly || jobs[j].n == 0) return;
    u32* a = jobs[j].rootAcc;
    store_box(jobs[j].nodes, mk(funord(a[0]), funord(a[1]), funord(a[2])), mk(funord(a[3]), funord(a[4]), funord(a[5])));
    // ready for the next refit
    a[0] = a[1] = a[2] = 0xFFFFFFFFu;
    a[3] = a[4] = a[5] = 0u;
}

void launch_refit_roots(const RefitJob* jobsDev, u32 numJobs, cudaStream_t s) {
    if (numJobs) k_refit_roots<<<ceil_div(numJobs, 128), 128, 0, s>>>(jobsDev, numJobs);
}

__global__ void __launch_bounds__(256) k_root_boxes(const RefitJob* __restrict__ jobs, const uint2* __restrict__ chunks) {
    __shared__ u32 red[8][6];
    const uint2 c = chunks[blockIdx.x];
    const RefitJob& J = jobs[c.x];
    const u32 end = min(c.y + ROOT_CHUNK, J.nVert);
    u32 r[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
    for (u32 i = c.y + threadIdx.x; i < end; i += blockDim.x) {
        const f3 p = ld(J.x4, J.voff + i);
        f3 a = p, b = p;
        if (J.swept) {
            const f3 sp = p + ld(J.v4, J.voff + i) * J.dt;  // the swept leaf's x + v dt
            a = vmin(p, sp);
            b = vmax(p, sp);
        }
        r[0] = min(r[0], ford(a.x)); r[1] = min(r[1], ford(a.y)); r[2] = min(r[2], ford(a.z));
        r[3] = max(r[3], ford(b.x)); r[4] = max(r[4], ford(b.y)); r[5] = max(r[5], ford(b.z));
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r[k] = __reduce_min_sync(0xFFFFFFFFu, r[k]);
        r[3 + k] = __reduce_max_sync(0xFFFFFFFFu, r[3 + k]);
    }
    const u32 w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 6; ++k) red[w][k] = r[k];
    __syncthreads();
    if (threadIdx.x < 6) {
        const u32 k = threadIdx.x;
        u32 v = red[0][k];
        for (u32 q = 1; q < (blockDim.x >> 5); ++q) v = k < 3 ? min(v, red[q][k]) : max(v, red[q][k]);
        if (k < 3) atomicMin(&J.rootAcc[k], v);
        else atomicMax(&J.rootAcc[k], v);
    }
}

void launch_root_boxes(const RefitJob* jobsDev, u32 numJobs, const uint2* chunks, u32 numChunks, cudaStream_t s) {
    if (!numJobs || !numChunks) return;
    k_root_boxes<<<numChunks, 256, 0, s>>>(jobsDev, chunks);
    k_refit_roots<<<ceil_div(numJobs, 128), 128, 0, s>>>(jobsDev, numJobs);
}

// ---- level-synchronous 4-wide refit

// Heights: every leaf climbs carrying the height of the node it leaves; the
// last child to arrive at a wide node reads the node's height (the max over
// its children + 1) and climbs on.
__global__ void __launch_bounds__(256) k_wide_heights(const RefitJob* __restrict__ jobs, u32 numJobs,
                                                      u32 totalLeaves, u32* status) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= totalLeaves) return;
    const RefitJob& J = jobs[job_of(jobs, numJobs, g)];
    if (!J.w4 || !J.levels) return;
    const u32 i = g - J.leafBase;
    if (i >= J.n) return;  // padding
    const u32 cap = J.n > 1 ? J.n - 1 : 1;
    i32 w = J.leafW[i].x;
    u32 h = 0, rlo = i, rhi = i;  // height and sorted-leaf range of the node carried up
    for (u32 step = 0; step < 128; ++step) {
        if (w < 0 || (u32)w >= cap) break;
        const u32 nc = __ldcg(&J.w4[w].nchild);
        if (nc == 0 || nc > 4) break;
        atomicMax(&J.hacc[w], h + 1);
        if (J.wrange) {
            atomicMin(&J.wrange[w].x, rlo);
            atomicMax(&J.wrange[w].y, rhi);
        }
        if (arrive_inc_acq_rel(&J.warrive[w], nc - 1) != nc - 1) return;
        h = __ldcg(&J.hacc[w]);
        if (J.wrange) {
            rlo = __ldcg(&J.wrange[w].x);
            rhi = __ldcg(&J.wrange[w].y);
        }
        w = __ldcg(&J.w4[w].parent);
        if (w < 0) return;
    }
    atomicOr(status, ST_ITER_CAP);
}

__global__ void __launch_bounds__(256) k_level_count(const RefitJob* __restrict__ jobs, u32 numJobs,
                                                     u32 totalLeaves, u32* __restrict__ hcount, u32* status) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= totalLeaves) return;
    const RefitJob& J = jobs[job_of(jobs, numJobs, g)];
    if (!J.w4 || !J.levels) return;
    const u32 local = g - J.leafBase;
    if (local >= *J.wcount) return;
    const u32 h = J.hacc[local];
    if (h == 0 || h > MAX_LEVELS) {
        atomicOr(status, ST_ITER_CAP);
        atomicAdd(&hcount[0], 1u);  // marks the level lists unusable
        return;
    }
    atomicAdd(&hcount[h], 1u);
}

__global__ void __launch_bounds__(256) k_level_fill(const RefitJob* __restrict__ jobs, u32 numJobs, u32 totalLeaves,
                                                    const u32* __restrict__ hoff, u32* __restrict__ hcursor,
                                                    uint2* __restrict__ list) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= totalLeaves) return;
    const u32 j = job_of(jobs, numJobs, g);
    const RefitJob& J = jobs[j];
    if (!J.w4 || !J.levels) return;
    const u32 local = g - J.leafBase;
    if (local >= *J.wcount) return;
    const u32 h = J.hacc[local];
    if (h == 0 || h > MAX_LEVELS) return;
    list[hoff[h] + atomicAdd(&hcursor[h], 1u)] = make_uint2(local, j);
}

void launch_wide_heights(const RefitJob* jobsDev, u32 numJobs, u32 totalLeaves, u32* status, cudaStream_t s) {
    if (totalLeaves) k_wide_heights<<<ceil_div(totalLeaves, 256), 256, 0, s>>>(jobsDev, numJobs, totalLeaves, status);
}
void launch_level_count(const RefitJob* jobsDev, u32 numJobs, u32 totalLeaves, u32* hcount, u32* status,
                        cudaStream_t s) {
    if (totalLeaves)
        k_level_count<<<ceil_div(totalLeaves, 256), 256, 0, s>>>(jobsDev, numJobs, totalLeaves, hcount, status);
}
void launch_level_fill(const RefitJob* jobsDev, u32 numJobs, u32 totalLeaves, const u32* hoff, u32* hcursor,
                       uint2* list, cudaStream_t s) {
    if (totalLeaves)
        k_level_fill<<<ceil_div(totalLeaves, 256), 256, 0, s>>>(jobsDev, numJobs, totalLeaves, hoff, hcursor, list);
}

// One wide node: the union of its slots (in slot order) into its parent's
// slot, or into the binary root node at the top.
// Box of wide node `local` (the union of its nc child slots) into its slot
// `ps` of parent `par`, or into the binary root node when par < 0.
__device__ __forceinline__ void refit_wide_box(const RefitJob& J, u32 local, i32 par, u32 ps, u32 nc) {
    const float4* p = reinterpret_cast<const float4*>(J.w4 + local);
    const float4 lx = p[0], ly = p[1], lz = p[2], hx = p[3], hy = p[4], hz = p[5];
    f3 lo = mk(lx.x, ly.x, lz.x), hi = mk(hx.x, hy.x, hz.x);
    if (nc > 1) { lo = vmin(lo, mk(lx.y, ly.y, lz.y)); hi = vmax(hi, mk(hx.y, hy.y, hz.y)); }
    if (nc > 2) { lo = vmin(lo, mk(lx.z, ly.z, lz.z)); hi = vmax(hi, mk(hx.z, hy.z, hz.z)); }
    if (nc > 3) { lo = vmin(lo, mk(lx.w, ly.w, lz.w)); hi = vmax(hi, mk(hx.w, hy.w, hz.w)); }
    if (par < 0) {
        store_box(J.nodes, lo, hi);
        return;
    }
    Wide4* P = J.w4 + par;
    P->lox[ps] = lo.x; P->loy[ps] = lo.y; P->loz[ps] = lo.z;
    P->hix[ps] = hi.x; P->hiy[ps] = hi.y; P->hiz[ps] = hi.z;
}

__device__ __forceinline__ void refit_wide_node(const RefitJob& J, u32 local) {
    const Wide4* W = J.w4 + local;
    refit_wide_box(J, local, W->parent, W->slot, W->nchild);
}

__global__ void __launch_bounds__(256) k_refit_level(const RefitJob* __restrict__ jobs, const uint2* __restrict__ list,
                                                     u32 count) {
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint2 e = list[t];
    refit_wide_node(jobs[e.y], e.x);
}

// Levels from..top in one block.  A node's list entry, parent link, slot and
// child count do not change between refits; they are staged in shared memory
// first, so that a level costs one dependent round trip (its children's
// boxes, written by this block before the preceding __syncthreads) instead of
// three.  Up to REFIT_TOP_NODES nodes (16 B of shared memory each).
static constexpr u32 REFIT_TOP_NODES = 8192;
static constexpr u32 REFIT_TOP_THREADS = 1024;

__global__ void __launch_bounds__(REFIT_TOP_THREADS) k_refit_top(const RefitJob* __restrict__ jobs,
                                                                const uint2* __restrict__ list,
                                                                const u32* __restrict__ hoff, u32 from, u32 top) {
    extern __shared__ uint4 sh_top[];  // (node, job, parent, slot << 8 | nchild)
    const u32 b0 = hoff[from], e0 = hoff[top + 1];
    for (u32 t = b0 + threadIdx.x; t < e0 && t - b0 < REFIT_TOP_NODES; t += blockDim.x) {
        const uint2 q = list[t];
        const Wide4* W = jobs[q.y].w4 + q.x;
        sh_top[t - b0] = make_uint4(q.x, q.y, (u32)W->parent, (W->slot << 8) | (W->nchild & 0xFFu));
    }
    __syncthreads();
    for (u32 h = from; h <= top; ++h) {
        const u32 b = hoff[h], e = hoff[h + 1];
        for (u32 t = b + threadIdx.x; t < e && t - b0 < REFIT_TOP_NODES; t += blockDim.x) {
            const uint4 it = sh_top[t - b0];
            refit_wide_box(jobs[it.y], it.x, (i32)it.z, it.w >> 8, it.w & 0xFFu);
        }
        __syncthreads();
    }
}

cudaError_t refit_levels_prepare() {
    return cudaFuncSetAttribute(k_refit_top, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(REFIT_TOP_NODES * sizeof(uint4)));
}

void launch_refit_levels(const RefitJob* jobsDev, const uint2* list, const u32* hoffDev, const u32* hostOff,
                         u32 top, cudaStream_t s) {
    // one launch per level down to the first level of fewer than 2048 nodes
    // (or until the rest no longer fits the top kernel's staging), then the
    // top kernel: one block is the faster form only for small levels
    u32 h = 1;
    for (; h <= top; ++h) {
        const u32 cnt = hostOff[h + 1] - hostOff[h];
        if (cnt < 2048 && hostOff[top + 1] - hostOff[h] <= REFIT_TOP_NODES) break;
        if (cnt) k_refit_level<<<ceil_div(cnt, 256), 256, 0, s>>>(jobsDev, list + hostOff[h], cnt);
    }
    if (h <= top) {
        const u32 nodes = hostOff[top + 1] - hostOff[h];
        k_refit_top<<<1, REFIT_TOP_THREADS, nodes * sizeof(uint4), s>>>(jobsDev, list, hoffDev, h, top);
    }
}

void launch_refit(const RefitJob* jobsDev, u32 numJobs, u32 totalLeaves, u32* status, cudaStream_t s) {
    if (totalLeaves == 0) return;
    k_refit<<<ceil_div(totalLeaves, 256), 256, 0, s>>>(jobsDev, numJobs, totalLeaves, status);
}

// ------------------------------------------------------------------ Apetrei
// agglomerativeBuild_Tri + agglomerativeSwapRoot (bvh.metal:884-1199): the
// topology and every box in one pass, one thread per leaf.
__global__ void k_apetrei_init(Node* __restrict__ nodes, u32* __restrict__ flags, u32 nInner) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nInner) return;
    nodes[i].a = -1;
    nodes[i].b = -1;
    flags[i] = 0u;
}

// Leaf i (sorted order) at slot n-1+i with its triangle's box; then the climb:
// at range [L, R] join the side whose neighbouring key differs less (code XOR,
// ties by index XOR; an end forces the other side).  Going right the parent is
// slot R and this node its left child; going left, slot L-1 and the right
// child.  The arrival (acq_rel) releases the child link, the range end and
// the box; the first arrival stops, the second combines and climbs on with
// the node's range.  A valid climb widens the range every step, so 2n steps
// bound it; indices are checked before use.
__global__ void __launch_bounds__(256) k_apetrei(const float4* x4, const float* x3, u32 voff, const u32* __restrict__ F,
                                                 const u32* __restrict__ codes, const u32* __restrict__ idx, u32 n,
                                                 Node* __restrict__ nodes, i32* __restrict__ parent,
                                                 u32* __restrict__ flags, i32* __restrict__ rangeL,
                                                 i32* __restrict__ rangeR, i32* __restrict__ root, u32* status) {
    const int N = (int)n;
    const int id = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (id >= N) return;
    const u32 f = idx[id];
    const f3 p0 = load_pos(x4, x3, voff + F[3 * f]), p1 = load_pos(x4, x3, voff + F[3 * f + 1]),
             p2 = load_pos(x4, x3, voff + F[3 * f + 2]);
    f3 lo = vmin(vmin(p0, p1), p2), hi = vmax(vmax(p0, p1), p2);
    const int leaf = N - 1 + id;
    nodes[leaf].a = -1;
    nodes[leaf].b = (i32)f;
    store_box(&nodes[leaf], lo, hi);
    if (N == 1) {
        *root = leaf;
        return;
    }
    int node = leaf, L = id, R = id;
    for (int step = 0; step < 2 * N; ++step) {
        if (L == 0 && R == N - 1) {
            *root = node;
            return;
        }
        bool right;
        if (L == 0) right = true;
        else if (R == N - 1) right = false;
        else {
            const u32 dr = codes[R] ^ codes[R + 1], dl = codes[L - 1] ^ codes[L];
            right = dr != dl ? dr < dl : (idx[R] ^ idx[R + 1]) < (idx[L - 1] ^ idx[L]);
        }
        const int p = right ? R : L - 1;
        if (right) {
            __stcg(&nodes[p].a, node);
            __stcg(&rangeL[p], L);
        } else {
            __stcg(&nodes[p].b, node);
            __stcg(&rangeR[p], R);
        }
        __stcg(&parent[node], p);
        if (arrive_acq_rel(&flags[p]) == 0u) return;
        const i32 ca = __ldcg(&nodes[p].a), cb = __ldcg(&nodes[p].b);
        if (ca < 0 || ca >= 2 * N - 1 || cb < 0 || cb >= 2 * N - 1) {
            atomicOr(status, ST_ITER_CAP);
            return;
        }
        const float4* A = reinterpret_cast<const float4*>(&nodes[ca]);
        const float4* B = reinterpret_cast<const float4*>(&nodes[cb]);
        const float4 a0 = __ldcg(A), a1 = __ldcg(A + 1), b0 = __ldcg(B), b1 = __ldcg(B + 1);
        lo = vmin(mk(a0.x, a0.y, a0.z), mk(b0.x, b0.y, b0.z));
        hi = vmax(mk(a1.x, a1.y, a1.z), mk(b1.x, b1.y, b1.z));
        store_box(&nodes[p], lo, hi);
        node = p;
        L = __ldcg(&rangeL[p]);
        R = __ldcg(&rangeR[p]);
        if (L < 0 || R >= N || L > R) {
            atomicOr(status, ST_ITER_CAP);
            return;
        }
    }
    atomicOr(status, ST_ITER_CAP);
}

// agglomerativeSwapRoot (bvh.metal:1131-1199): the root (built in slot k)
// moves to slot 0 and the node that was there to slot k, with the children's
// parent links, the displaced node's parent's child link and the root's own
// links to slot 0 patched.  One thread.
__global__ void k_apetrei_swap(Node* __restrict__ nodes, i32* __restrict__ parent, const i32* __restrict__ root,
                               u32 n, u32* status) {
    if (blockIdx.x || threadIdx.x || n <= 1) return;
    const i32 k = *root;
    if (k == 0) return;
    const i32 nInner = (i32)n - 1, nn = 2 * (i32)n - 1;
    if (k < 0 || k >= nInner) {  // the root must be an internal slot
        atomicOr(status, ST_ITER_CAP);
        return;
    }
    const Node Rn = nodes[k], O = nodes[0];
    const i32 p0 = parent[0];
    const i32 ra = Rn.a == 0 ? k : Rn.a, rb = Rn.b == 0 ? k : Rn.b;
    if (O.a < 0 || O.a >= nn || O.b < 0 || O.b >= nn || ra < 0 || ra >= nn || rb < 0 || rb >= nn ||
        (p0 != k && (p0 < 0 || p0 >= nInner))) {
        atomicOr(status, ST_ITER_CAP);
        return;
    }
    Node r0 = Rn;
    r0.a = ra;
    r0.b = rb;
    nodes[0] = r0;
    nodes[k] = O;
    parent[O.a] = k;
    parent[O.b] = k;
    parent[ra] = 0;
    parent[rb] = 0;
    if (p0 != k) {
        if (nodes[p0].a == 0) nodes[p0].a = k;
        else nodes[p0].b = k;
        parent[k] = p0;
    }
    parent[0] = -1;
}

// Claimant counts of a built tree (one per child link; leaves and the root's
// absent parent included by their zero).
__global__ void k_claim_count(const Node* __restrict__ nodes, u32 nInner, u32* __restrict__ claimCount) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nInner) return;
    const i32 a = nodes[i].a, b = nodes[i].b, nn = 2 * (i32)nInner + 1;
    if (a >= 0 && a < nn) atomicAdd(&claimCount[a], 1u);
    if (b >= 0 && b < nn) atomicAdd(&claimCount[b], 1u);
}

size_t apetrei_scratch_bytes(u32 n) { return 8 * (size_t)(n ? n : 1) + 256; }

cudaError_t launch_apetrei(const float4* x4, const float* x3, u32 voff, const u32* facets, const u32* codes,
                           const u32* idx, u32 n, Node* nodes, i32* parent, u32* claimOff, i32* claims, u32* visits,
                           void* scanScratch, void* aggScratch, u32* status, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const u32 nInner = n > 1 ? n - 1 : 0;
    i32* rangeL = reinterpret_cast<i32*>(aggScratch);
    i32* rangeR = rangeL + (n ? n : 1);
    i32* root = reinterpret_cast<i32*>(reinterpret_cast<char*>(aggScratch) + 8 * (size_t)(n ? n : 1));
    k_parent_init<<<ceil_div(2 * n, 256), 256, 0, s>>>(parent, claimOff, 2 * n - 1);
    if (nInner) k_apetrei_init<<<ceil_div(nInner, 256), 256, 0, s>>>(nodes, visits, nInner);
    k_apetrei<<<ceil_div(n, 256), 256, 0, s>>>(x4, x3, voff, facets, codes, idx, n, nodes, parent, visits, rangeL,
                                                rangeR, root, status);
    if (n > 1) {
        k_apetrei_swap<<<1, 32, 0, s>>>(nodes, parent, root, n, status);
        k_claim_count<<<ceil_div(nInner, 256), 256, 0, s>>>(nodes, nInner, claimOff);
    }
    cudaError_t e = exclusive_scan(claimOff, 2 * n, scanScratch, s);
    if (e != cudaSuccess) return e;
    if (n > 1) k_claim_fill<<<ceil_div(nInner, 256), 256, 0, s>>>(nodes, nInner, claimOff, claims);
    return cudaGetLastError();
}

}  // namespace ys
