// ys_api.cu -- C ABI of the standalone LBVH (one triangle soup) and of the
// build primitives (Morton codes, radix sort).  BVH<CUDA,PR,LINEAR,TRIANGLE>
// surface: build (bvh.hpp:1194-1301), refit / refitSwept (bvh.hpp:1555-1606,
// 1100-1115), queryPoints (bvh.hpp:1803-1841).
#include <string>

#include "ys_collide.cuh"
#include "ys_common.cuh"
#include "ys_lbvh.cuh"
#include "ys_sort.cuh"
#include "ysim_b200.h"

namespace ys {
ys_status fail(ys_status code, const std::string& msg);

// queryPoints (bvh.metal:1394-1412): one thread per query point; pairs are
// (point, triangle).  The lanes that reach a leaf together (the converged
// lanes at the append) reserve their slots with one atomic, made by the
// lowest of them; the reference appends with one atomic per pair
// (bvh.metal:1372-1381).
__global__ void __launch_bounds__(128) k_query_points(const Node* __restrict__ nodes, u32 numNodes,
                                                      const u32* __restrict__ F, const float* __restrict__ qx, u32 nQ,
                                                      const u32* __restrict__ order, float m, int self,
                                                      u32* __restrict__ pairs, u64 cap, unsigned long long* count,
                                                      u32* status) {
    const u32 k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nQ) return;
    const u32 p = order ? order[k] : k;  // the point of this thread (Morton order for large query sets)
    const f3 q = ldp(qx, p);
    const f3 qmn = q - mk(m, m, m), qmx = q + mk(m, m, m);
    u32 st = traverse(nodes, numNodes, qmn, qmx, [&](u32 f) {
        if (self && (F[3 * f] == p || F[3 * f + 1] == p || F[3 * f + 2] == p)) return;
        const unsigned act = __activemask();
        const u32 lane = threadIdx.x & 31u, leader = (u32)__ffs(act) - 1u;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(act));
        base = __shfl_sync(act, base, (int)leader);
        const unsigned long long i = base + (u32)__popc(act & ((1u << lane) - 1u));
        if (i < cap) { pairs[2 * i] = p; pairs[2 * i + 1] = f; }
    });
    if (st) atomicOr(status, st);
}

}  // namespace ys

using namespace ys;

struct ys_lbvh {
    int device = 0;
    cudaStream_t stream = nullptr;
    u32 maxPrims = 0, n = 0;
    Node* nodes = nullptr;
    i32* parent = nullptr;
    u32* claimOff = nullptr;  // claimant lists (2N + 1 entries) and ids (2N)
    i32* claims = nullptr;
    void* karrasScratch = nullptr;
    u32 *codes = nullptr, *idx = nullptr, *visits = nullptr, *box = nullptr, *status = nullptr;
    void* scratch = nullptr;
    RefitJob* job = nullptr;
    const u32* facets = nullptr;
    bool consistent = false;  // Karras split of runs of equal codes (ys_lbvh_set_split)
    QueryOrder qorder;        // Morton order of large query sets
    int builder = YS_BUILD_KARRAS;  // ys_lbvh_set_builder
    void* aggScratch = nullptr;     // Apetrei range ends and root slot
    // range refit of a consistent Karras tree: per internal node its
    // sorted-leaf range, the nodes whose range leaves their block, block boxes
    uint2* range = nullptr;
    u32 *big = nullptr, *huge = nullptr, *bcount = nullptr;
    Node *bb16 = nullptr, *bb256 = nullptr;
    u32* rank = nullptr;      // sorted-leaf position of each face
    float4* lbox = nullptr;   // leaf boxes in sorted order (face-order pass of the refit)
    u32 nbig = 0, nhuge = 0;
    bool ranged = false;            // the last build recorded ranges (consistent Karras split)
};

#define YS_CK2(call)                                                                                   \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(YS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

extern "C" {

ys_status ys_lbvh_create(ys_lbvh** out, uint32_t maxPrims, int device, void* stream) {
    if (!out || maxPrims == 0) return fail(YS_ERR_BAD_ARG, "bad argument");
    YS_CK2(cudaSetDevice(device));
    ys_lbvh* t = new ys_lbvh();
    t->device = device;
    t->stream = (cudaStream_t)stream;
    t->maxPrims = maxPrims;
    size_t nn = 2 * (size_t)maxPrims - 1;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->nodes, nn * sizeof(Node));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->parent, nn * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->claimOff, (nn + 2) * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->claims, (nn + 1) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&t->karrasScratch, karras_scratch_bytes(maxPrims));
    if (e == cudaSuccess) e = cudaMalloc(&t->aggScratch, apetrei_scratch_bytes(maxPrims));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->codes, (size_t)maxPrims * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->idx, (size_t)maxPrims * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->visits, (size_t)maxPrims * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->box, 32);
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->status, 4);
    if (e == cudaSuccess) e = cudaMalloc(&t->scratch, sort_scratch_bytes(maxPrims));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->job, sizeof(RefitJob));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->range, (size_t)maxPrims * sizeof(uint2));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->big, (size_t)maxPrims * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->huge, (size_t)maxPrims * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->bcount, 8);
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->bb16, ((size_t)maxPrims / 16 + 1) * sizeof(Node));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->bb256, ((size_t)maxPrims / 256 + 1) * sizeof(Node));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->rank, (size_t)maxPrims * 4);
    if (e == cudaSuccess) e = cudaMalloc((void**)&t->lbox, (size_t)maxPrims * 2 * sizeof(float4));
    // completed before this returns: later launches may go to any stream,
    // including non-blocking ones that do not wait for the legacy stream
    if (e == cudaSuccess) e = cudaMemsetAsync(t->status, 0, 4, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        ys_lbvh_destroy(t);
        return fail(YS_ERR_CUDA, cudaGetErrorString(e));
    }
    *out = t;
    return YS_OK;
}

ys_status ys_lbvh_destroy(ys_lbvh* t) {
    if (!t) return YS_OK;
    cudaSetDevice(t->device);
    cudaStreamSynchronize(t->stream);
    cudaFree(t->nodes); cudaFree(t->parent); cudaFree(t->claimOff); cudaFree(t->claims); cudaFree(t->karrasScratch); cudaFree(t->aggScratch); cudaFree(t->codes); cudaFree(t->idx); cudaFree(t->visits);
    cudaFree(t->box); cudaFree(t->status); cudaFree(t->scratch); cudaFree(t->job);
    cudaFree(t->range); cudaFree(t->big); cudaFree(t->huge); cudaFree(t->bcount); cudaFree(t->bb16); cudaFree(t->bb256);
    cudaFree(t->rank); cudaFree(t->lbox);
    query_order_free(t->qorder);
    delete t;
    return YS_OK;
}

static ys_status run_refit(ys_lbvh* t, const float* x, const float* v, float dt, int swept) {
    RefitJob J;
    memset(&J, 0, sizeof(J));
    J.nodes = t->nodes; J.parent = t->parent; J.claimOff = t->claimOff; J.claims = t->claims; J.visits = t->visits; J.facets = t->facets;
    J.x3 = x; J.v3 = v; J.voff = 0; J.n = t->n; J.leafBase = 0; J.dt = dt; J.swept = swept ? 1u : 0u;
    J.selfMargin = 0.f; J.maxExt = t->box;
    if (t->ranged) {
        // consistent tree: every internal box is the union of its sorted-leaf
        // range, from the leaf pass's block boxes (no climb)
        J.bb16 = t->bb16;
        J.bb256 = t->bb256;
        launch_refit_bin(J, t->range, t->big, t->nbig, t->huge, t->nhuge, t->rank, t->lbox, t->stream);
        YS_CK2(cudaGetLastError());
        YS_CK2(cudaStreamSynchronize(t->stream));
        return YS_OK;
    }
    YS_CK2(cudaMemcpyAsync(t->job, &J, sizeof(J), cudaMemcpyHostToDevice, t->stream));
    launch_refit(t->job, 1, t->n, t->status, t->stream);
    YS_CK2(cudaGetLastError());
    YS_CK2(cudaStreamSynchronize(t->stream));
    return YS_OK;
}

ys_status ys_lbvh_set_split(ys_lbvh* t, int consistent) {
    if (!t) return fail(YS_ERR_BAD_ARG, "null tree");
    t->consistent = consistent != 0;
    return YS_OK;
}

ys_status ys_lbvh_set_builder(ys_lbvh* t, int builder) {
    if (!t) return fail(YS_ERR_BAD_ARG, "null tree");
    if (builder != YS_BUILD_KARRAS && builder != YS_BUILD_APETREI) return fail(YS_ERR_BAD_ARG, "unknown tree builder");
    t->builder = builder;
    return YS_OK;
}

ys_status ys_lbvh_build(ys_lbvh* t, const float* x, uint32_t nV, const uint32_t* F, uint32_t nF) {
    if (!t || !x || !F || nF == 0 || nV == 0) return fail(YS_ERR_BAD_ARG, "bad argument");
    if (nF > t->maxPrims) return fail(YS_ERR_CAPACITY, "more primitives than the tree was created for");
    t->n = nF;
    t->facets = F;
    launch_box_init(t->box, t->stream);
    launch_box(nullptr, x, 0, nV, t->box, t->stream);
    launch_morton(nullptr, x, 0, F, nF, t->box, t->codes, t->idx, t->stream);
    YS_CK2(radix_sort_pairs(t->codes, t->idx, nF, t->scratch, 0, 32, t->stream));
    t->ranged = false;
    if (t->builder == YS_BUILD_APETREI) {
        // topology and boxes in one pass: no refit afterwards
        YS_CK2(launch_apetrei(nullptr, x, 0, F, t->codes, t->idx, nF, t->nodes, t->parent, t->claimOff, t->claims,
                              t->visits, t->karrasScratch, t->aggScratch, t->status, t->stream));
        YS_CK2(cudaStreamSynchronize(t->stream));
        return YS_OK;
    }
    BinRanges R;
    if (t->consistent) {  // one parent per node: boxes are unions of contiguous sorted-leaf ranges
        R.range = t->range; R.big = t->big; R.huge = t->huge; R.count = t->bcount;
    }
    YS_CK2(launch_karras(t->codes, t->idx, nF, t->nodes, t->parent, t->claimOff, t->claims, t->visits,
                         t->karrasScratch, t->stream, t->consistent, R));
    YS_CK2(cudaGetLastError());
    if (t->consistent) {
        u32 cnt[2] = {0, 0};
        YS_CK2(cudaMemcpyAsync(cnt, t->bcount, 8, cudaMemcpyDeviceToHost, t->stream));
        YS_CK2(cudaStreamSynchronize(t->stream));
        t->nbig = cnt[0];
        t->nhuge = cnt[1];
        t->ranged = true;
        launch_leaf_rank(t->idx, nF, t->rank, t->stream);
    }
    return run_refit(t, x, nullptr, 0.f, 0);
}

ys_status ys_lbvh_refit(ys_lbvh* t, const float* x, const float* v, float dt, int swept) {
    if (!t || !x || t->n == 0) return fail(YS_ERR_BAD_ARG, "bad argument / tree not built");
    if (swept && !v) return fail(YS_ERR_BAD_ARG, "swept refit needs velocities");
    return run_refit(t, x, v, dt, swept);
}

ys_status ys_lbvh_query(ys_lbvh* t, const float* qx, uint32_t nQ, float margin, int self, uint32_t* pairs, uint64_t cap,
                        unsigned long long* count) {
    if (!t || !qx || !count || t->n == 0) return fail(YS_ERR_BAD_ARG, "bad argument / tree not built");
    YS_CK2(cudaMemsetAsync(count, 0, 8, t->stream));
    const u32* order = nullptr;
    if (nQ >= QUERY_ORDER_MIN_LBVH) {
        YS_CK2(query_order(t->qorder, qx, nQ, t->stream));
        order = t->qorder.idx;
    }
    if (nQ) k_query_points<<<ceil_div(nQ, 128), 128, 0, t->stream>>>(t->nodes, 2 * t->n - 1, t->facets, qx, nQ, order,
                                                                      margin, self, pairs, cap, count, t->status);
    YS_CK2(cudaGetLastError());
    YS_CK2(cudaStreamSynchronize(t->stream));
    return YS_OK;
}

ys_status ys_lbvh_arrays(ys_lbvh* t, void** nodes, int32_t** parent, uint32_t** codes, uint32_t** idx, uint32_t* n) {
    if (!t) return fail(YS_ERR_BAD_ARG, "null tree");
    if (nodes) *nodes = t->nodes;
    if (parent) *parent = t->parent;
    if (codes) *codes = t->codes;
    if (idx) *idx = t->idx;
    if (n) *n = t->n;
    return YS_OK;
}

ys_status ys_morton_codes(const float* x, uint32_t nV, const uint32_t* F, uint32_t nF, uint32_t* codes, uint32_t* idx,
                          void* stream) {
    if (!x || !F || !codes || !idx || nV == 0) return fail(YS_ERR_BAD_ARG, "bad argument");
    cudaStream_t s = (cudaStream_t)stream;
    u32* box = nullptr;
    YS_CK2(cudaMallocAsync((void**)&box, 32, s));
    launch_box_init(box, s);
    launch_box(nullptr, x, 0, nV, box, s);
    launch_morton(nullptr, x, 0, F, nF, box, codes, idx, s);
    YS_CK2(cudaFreeAsync(box, s));
    YS_CK2(cudaStreamSynchronize(s));
    return YS_OK;
}

size_t ys_radix_sort_scratch_bytes(uint32_t n) { return sort_scratch_bytes(n); }

ys_status ys_radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, void* scratch, void* stream) {
    if ((!keys || !vals || !scratch) && n > 1) return fail(YS_ERR_BAD_ARG, "bad argument");
    YS_CK2(radix_sort_pairs(keys, vals, n, scratch, 0, 32, (cudaStream_t)stream));
    YS_CK2(cudaStreamSynchronize((cudaStream_t)stream));
    return YS_OK;
}

}  // extern "C"
