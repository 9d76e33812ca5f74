// ref_harness.cpp -- runs the reference's own Metal compute kernels on the host.
//
// TEST INFRASTRUCTURE ONLY.  oracle/build_ref.py compiles this file once per
// shader (YS_REF_BVH / YS_REF_NARROW / YS_REF_PHYSICS selects which), with the
// shader file included from the reference checkout in place (nothing is
// copied) and oracle/ref_shim standing in for <metal_stdlib>.  Each extern "C"
// function below dispatches one kernel over its thread ids, the way
// MetalGlobalContext::dispatchThreads does (core_types.hpp:120-149), so the
// oracle restatement (ys_oracle.cpp) can be compared with the reference's
// kernel code on the same inputs.
//
// Kernels with no threadgroup cooperation run with OpenMP over ids (their
// device atomics are std::atomic); bottomUpBoxes runs concurrently as
// designed (its arrival counters and fences are real).
#include <cstdint>
#include <cstring>
#include <vector>

#include "metal_shim.h"
using namespace metal;

#define YS_STR2(x) #x
#define YS_STR(x) YS_STR2(x)

#if defined(YS_REF_BVH)
#include YS_STR(YS_REF_SRC)

static_assert(sizeof(BVHNode) == 32, "BVHNode");
static_assert(sizeof(MortonNode) == 8, "MortonNode");
static_assert(sizeof(AABB4) == 32, "AABB4");
static_assert(sizeof(BroadCollision) == 32, "BroadCollision");

static AABB4 box_of(const float* box6, uint n) {
    AABB4 b;
    b.min = packed_float3(box6[0], box6[1], box6[2]);
    b.max = packed_float3(box6[3], box6[4], box6[5]);
    b._pad0 = (int)n;
    b._pad1 = 0;
    return b;
}

extern "C" {

// fillMortons_Tri over every face; mortons = (code, index) pairs.
void yref_fill_mortons(const float* x, const uint32_t* F, uint32_t n, const float* box6, uint32_t* mortons) {
    AABB4 b = box_of(box6, n);
#pragma omp parallel for
    for (long long i = 0; i < (long long)n; ++i)
        fillMortons_Tri((const packed_float3*)x, (const packed_uint3*)F, b, (MortonNode*)mortons, (uint)i);
}

// buildTree_Tri over every leaf (sorted mortons in), then zeroVisitCounts +
// bottomUpBoxes (BVH::buildTreeGPU + bottomUpBoxesGPU, bvh.hpp:499-517, 709-721).
void yref_build_tree(const float* x, const uint32_t* F, uint32_t n, const uint32_t* mortons, void* nodes,
                     int32_t* parent) {
    const int np = (int)n;
#pragma omp parallel for
    for (long long i = 0; i < (long long)n; ++i)
        buildTree_Tri((const packed_float3*)x, (const packed_uint3*)F, np, (const MortonNode*)mortons,
                      (BVHNode*)nodes, (int*)parent, (uint)i);
}

void yref_leaves(const float* x, const uint32_t* F, uint32_t n, const uint32_t* mortons, void* nodes) {
    const int np = (int)n;
#pragma omp parallel for
    for (long long i = 0; i < (long long)n; ++i)
        buildLeaf_Tri((const packed_float3*)x, (const packed_uint3*)F, np, (const MortonNode*)mortons,
                      (BVHNode*)nodes, (uint)i);
}

void yref_swept_leaves(const float* x, const float* v, const uint32_t* F, uint32_t n, float dt,
                       const uint32_t* mortons, void* nodes) {
    const int np = (int)n;
#pragma omp parallel for
    for (long long i = 0; i < (long long)n; ++i)
        buildSweptLeaf_Tri((const packed_float3*)x, (const packed_float3*)v, (const packed_uint3*)F, np, dt,
                           (const MortonNode*)mortons, (BVHNode*)nodes, (uint)i);
}

// zeroVisitCounts over the N-1 flags + agglomerativeBuild_Tri (one thread per
// leaf, run one after another: a node's second arrival always comes from a
// later thread) + agglomerativeSwapRoot (BVH::agglomerativeBuildGPU /
// agglomerativeSwapRootGPU, bvh.hpp:649-694).  Returns the pre-swap root slot.
int32_t yref_agglomerative(const float* x, const uint32_t* F, uint32_t n, const uint32_t* mortons, void* nodes,
                           int32_t* parent) {
    const int np = (int)n;
    const uint ni = n > 1 ? n - 1 : 1;
    std::vector<uint32_t> flags(ni, 0u);
    std::vector<int> rl(ni, 0), rr(ni, 0);
    atomic_int root;
    root.v.store(-1);
    for (uint i = 0; i < n; ++i)
        agglomerativeBuild_Tri((const packed_float3*)x, (const packed_uint3*)F, np, (const MortonNode*)mortons,
                               (BVHNode*)nodes, (int*)parent, (atomic_uint*)flags.data(), rl.data(), rr.data(), &root,
                               i);
    const int k = root.v.load();
    agglomerativeSwapRoot((BVHNode*)nodes, (int*)parent, &k, np, 0u);
    return k;
}

// zeroVisitCounts + bottomUpBoxes, leaf threads concurrent.
void yref_bottom_up(void* nodes, const int32_t* parent, uint32_t n, uint32_t* visits) {
    static const float zero6[6] = {0, 0, 0, 0, 0, 0};
    AABB4 b = box_of(zero6, n);  // bottomUpBoxes reads only the count (_pad0)
    const uint nn = n ? 2 * n - 1 : 0;
#pragma omp parallel for
    for (long long i = 0; i < (long long)nn; ++i) zeroVisitCounts(visits, nn, (uint)i);
#pragma omp parallel for schedule(dynamic, 256)
    for (long long i = 0; i < (long long)n; ++i)
        bottomUpBoxes(b, (BVHNode*)nodes, (const int*)parent, (atomic_uint*)visits, (uint)i);
}

// queryPoints for nQ query points against one tree; rows appended through
// the kernel's own atomic counter.
uint32_t yref_query_points(const float* qx, uint32_t nQ, const uint32_t* F, const void* nodes, uint32_t numNodes,
                           float margin, uint32_t qObj, uint32_t tObj, void* rows, uint32_t cap, uint32_t* flags) {
    QueryPointsParams p;
    std::memset(&p, 0, sizeof(p));
    p.queryMargin = margin; p.numPoints = nQ; p.qObjId = qObj; p.tObjId = tObj; p.maxNumCollisions = cap;
    p.numNodes = numNodes; p.entryRoot = 0;
    atomic_uint count; count.v.store(0);
    QueryFlag qf = {0u, 0u};
#pragma omp parallel for schedule(dynamic, 64)
    for (long long i = 0; i < (long long)nQ; ++i)
        queryPoints((const packed_float3*)qx, (const packed_uint3*)F, (const BVHNode*)nodes, p, (BroadCollision*)rows,
                    &count, &qf, (uint)i);
    if (flags) { flags[0] = qf.stackOverflow; flags[1] = qf.collisionOverflow; }
    return count.v.load();
}

}  // extern "C"

#elif defined(YS_REF_NARROW)
#include YS_STR(YS_REF_SRC)

static_assert(sizeof(BroadCollision) == 32, "BroadCollision");
static_assert(sizeof(NarrowCollision) == 48, "NarrowCollision");

extern "C" {

// narrow_pt_tri over nrows broad rows of a packed scene.
uint32_t yref_narrow(const void* rows, uint32_t nrows, const float* x, const uint32_t* voff, const uint32_t* F,
                     const uint32_t* foff, const uint32_t* vaf, const uint32_t* vaf_off, float radius, float thickness,
                     const float* xprev, void* out, uint32_t cap) {
    NarrowParams p;
    std::memset(&p, 0, sizeof(p));
    p.numBroadCollisions = nrows; p.maxNumCollisions = cap; p.radius = radius; p.thickness = thickness;
    p.skipAnalytic = 0u;
    atomic_uint count; count.v.store(0);
    uint nb = nrows;
#pragma omp parallel for schedule(dynamic, 1024)
    for (long long i = 0; i < (long long)nrows; ++i)
        narrow_pt_tri((const BroadCollision*)rows, &count, (NarrowCollision*)out, (const packed_float3*)x, voff,
                      (const packed_uint3*)F, foff, vaf, vaf_off, p, (const packed_float3*)xprev, &nb, (uint)i);
    return count.v.load();
}

static_assert(sizeof(AnalyticShape) == 96, "AnalyticShape");

// narrow_pt_analytic for every vertex of cloth mesh `oid` against
// shapes[shape_index], one thread at a time (appends in vertex order).
uint32_t yref_narrow_analytic(const float* x, const float* xprev, const uint32_t* voff, const void* shapes,
                              uint32_t oid, uint32_t nverts, uint32_t shape_index, uint32_t cloth_beh, float radius,
                              float thickness, float rot_margin, void* out, uint32_t cap) {
    AnalyticNarrowParams p;
    std::memset(&p, 0, sizeof(p));
    p.oid = oid; p.numVerts = nverts; p.shapeIndex = shape_index; p.maxNumCollisions = cap;
    p.clothBehavior = cloth_beh; p.radius = radius; p.thickness = thickness; p.rotMargin = rot_margin;
    atomic_uint count; count.v.store(0);
    for (uint i = 0; i < nverts; ++i)
        narrow_pt_analytic(&count, (NarrowCollision*)out, (const packed_float3*)x, voff, (const AnalyticShape*)shapes,
                           p, (const packed_float3*)xprev, i);
    return count.v.load();
}

}  // extern "C"

#elif defined(YS_REF_PHYSICS)
#include YS_STR(YS_REF_SRC)

static_assert(sizeof(NarrowCollision) == 48, "NarrowCollision");
static_assert(sizeof(SimParams) == 24, "SimParams");
static_assert(sizeof(ClothGridParams) == 44, "ClothGridParams");
static_assert(sizeof(ClothParams) == 16, "ClothParams");

static SimParams sim(float subh, float kair, float kd, uint32_t nV) {
    SimParams p;
    p.subh = subh; p.G = -9.81f; p.kair = kair; p.kd = kd; p.vertexNum = nV; p.acctime = 0.f;
    return p;
}

extern "C" {

// compute_tri_spring_forces over one mesh (mesh-local arrays).
void yref_tri_forces(const float* x, const float* v, float* f, const float* m3, const float* mask, const float* ext,
                     float subh, float kair, float kd, const float* cp4, const uint32_t* edges, const uint32_t* F,
                     const uint32_t* vae, const uint32_t* vae_off, const float* rest_edge, const uint32_t* opp,
                     const uint32_t* opp_off, const float* rest_opp, uint32_t nV) {
    SimParams sp = sim(subh, kair, kd, nV);
    ClothParams cp;
    std::memcpy(&cp, cp4, sizeof(cp));
#pragma omp parallel for
    for (long long i = 0; i < (long long)nV; ++i)
        compute_tri_spring_forces((const packed_float3*)x, (const packed_float3*)v, (packed_float3*)f, m3, mask,
                                  (const packed_float3*)ext, sp, cp, (const uint2*)edges, F, vae, vae_off, rest_edge,
                                  opp, opp_off, rest_opp, (uint)i);
}

void yref_integrate_tri(float* x, float* v, const float* f, const float* m3, const float* mask, const void* csr,
                        const uint32_t* csr_off, const uint32_t* voff, uint32_t oid, float subh, const float* cp4,
                        uint32_t nV, uint32_t* anomaly) {
    SimParams sp = sim(subh, 0.f, 0.f, nV);
    ClothParams cp;
    std::memcpy(&cp, cp4, sizeof(cp));
#pragma omp parallel for
    for (long long i = 0; i < (long long)nV; ++i)
        integrate_cloth((packed_float3*)x, (packed_float3*)v, (const packed_float3*)f, m3, mask,
                        (const NarrowCollision*)csr, csr_off, sp, cp, voff, oid, anomaly, (uint)i);
}

// compute_cloth_grid_forces_fast; gp11 = ClothGridParams field by field.
void yref_grid_forces(const float* x, const float* v, float* f, const float* m3, const float* ext, float subh,
                      float kair, float kd, const uint32_t* gp11, uint32_t nV) {
    SimParams sp = sim(subh, kair, kd, nV);
    ClothGridParams gp;
    std::memcpy(&gp, gp11, sizeof(gp));
#pragma omp parallel for
    for (long long i = 0; i < (long long)nV; ++i)
        compute_cloth_grid_forces_fast((const packed_float3*)x, (const packed_float3*)v, (packed_float3*)f, m3,
                                       (const packed_float3*)ext, sp, gp, (uint)i);
}

void yref_integrate_grid(float* x, float* v, const float* f, const float* m3, const float* mask, const void* csr,
                         const uint32_t* csr_off, const uint32_t* voff, uint32_t oid, float subh,
                         const uint32_t* gp11, uint32_t nV, uint32_t* anomaly) {
    SimParams sp = sim(subh, 0.f, 0.f, nV);
    ClothGridParams gp;
    std::memcpy(&gp, gp11, sizeof(gp));
#pragma omp parallel for
    for (long long i = 0; i < (long long)nV; ++i)
        integrate_cloth_grid((packed_float3*)x, (packed_float3*)v, (const packed_float3*)f, m3, mask,
                             (const NarrowCollision*)csr, csr_off, sp, gp, voff, oid, anomaly, (uint)i);
}

// narrow_bucket_zero / count / scan / scatter (physics.metal:555-616).
void yref_bucket(const void* contacts, uint32_t n, const uint32_t* voff, uint32_t nOffsets, uint32_t* offsets,
                 uint32_t* counter, void* out) {
    uint nOff = nOffsets, maxN = n, cnt = n;
    for (uint i = 0; i < nOff; ++i) narrow_bucket_zero(offsets, counter, nOff, i);
#pragma omp parallel for
    for (long long i = 0; i < (long long)n; ++i)
        narrow_bucket_count((const NarrowCollision*)contacts, &cnt, voff, (atomic_uint*)offsets, maxN, (uint)i);
    narrow_bucket_scan(offsets, nOff, 0u);
#pragma omp parallel for
    for (long long i = 0; i < (long long)n; ++i)
        narrow_bucket_scatter((const NarrowCollision*)contacts, &cnt, voff, offsets, (atomic_uint*)counter,
                              (NarrowCollision*)out, maxN, (uint)i);
}

}  // extern "C"
#elif defined(YS_REF_SH)
#include <algorithm>
#include <vector>
#include YS_STR(YS_REF_SRC)

static_assert(sizeof(SHEntry) == 8, "SHEntry");
static_assert(sizeof(CellProp) == 20, "CellProp");
static_assert(sizeof(BroadCollision) == 32, "BroadCollision");

extern "C" {

// SpatialHashing<METAL>::detectCollisions (spatial_hash.hpp:880-960) over a
// packed scene: the reference's kernels sh_buildBV, sh_assignCells,
// sh_markStarts, sh_fillCellProp, sh_computePairCount and sh_broadPhase, in
// that order, with the host steps between them restated from
// spatial_hash.hpp: faceObj (:255-267), the max-radius reduction (the
// maximum of the radii, :308-341), computeGrid (:343-400), the stable
// 4-pass radix sort by cellID (:409-412, RadixSorter), findNumValid
// (:414-426), hostScanCellStarts (:439-449) and hostScanPairPrefix
// (:590-602).  Returns the number of rows the kernel counted (rows past cap
// are dropped by the kernel).  out6: numValid, numCells, numPairs, gridRes.
uint32_t yref_sh_detect(const float* x, const uint32_t* stateOff, const uint32_t* F, const uint32_t* facetOff,
                        const uint32_t* behaviors, const uint32_t* shapes, uint32_t numMeshes, float margin,
                        uint32_t enableSelf, void* rows, uint32_t cap, uint32_t* out6) {
    const uint32_t nV = stateOff[numMeshes], nF = facetOff[numMeshes];
    for (int k = 0; k < 6; ++k) out6[k] = 0;
    if (nF == 0 || nV == 0) return 0;
    std::vector<uint32_t> faceObj(nF);
    for (uint32_t m = 0; m < numMeshes; ++m)
        for (uint32_t f = facetOff[m]; f < facetOff[m + 1]; ++f) faceObj[f] = m;
    SHParams params;
    std::memset(&params, 0, sizeof(params));
    params.numFaces = nF;
    std::vector<float> centroid(3 * (size_t)nF), radius(nF);
    for (uint32_t i = 0; i < nF; ++i)
        sh_buildBV((const packed_float3*)x, stateOff, (const packed_uint3*)F, faceObj.data(), params,
                   (packed_float3*)centroid.data(), radius.data(), i);
    float maxR = 0.0f;
    for (uint32_t i = 0; i < nF; ++i) maxR = max(maxR, radius[i]);
    float3 mn(x[0], x[1], x[2]), mx = mn;
    for (uint32_t v = 0; v < nV; ++v) {
        float3 p(x[3 * v], x[3 * v + 1], x[3 * v + 2]);
        mn = float3(std::min(mn.x, p.x), std::min(mn.y, p.y), std::min(mn.z, p.z));
        mx = float3(std::max(mx.x, p.x), std::max(mx.y, p.y), std::max(mx.z, p.z));
    }
    float cellSize = 2.0f * maxR * 1.0f + margin;
    if (cellSize <= 0.f) cellSize = std::max(margin, 1e-6f);
    params.cellSize = cellSize;
    params.epsilon = margin;
    params.originMin = packed_float3(mn.x, mn.y, mn.z);
    for (int k = 0; k < 3; ++k) {
        float extent = mx[k] - mn[k];
        uint32_t r = (uint32_t)std::ceil(extent / cellSize);
        params.gridRes[k] = r == 0 ? 1 : r;
    }
    std::vector<SHEntry> entries(8 * (size_t)nF);
    std::vector<uchar> faceCB(nF);
    for (uint32_t i = 0; i < nF; ++i)
        sh_assignCells((const packed_float3*)centroid.data(), radius.data(), params, entries.data(), faceCB.data(), i);
    std::stable_sort(entries.begin(), entries.end(),
                     [](const SHEntry& a, const SHEntry& b) { return a.cellID < b.cellID; });
    uint32_t numValid = 0;
    while (numValid < entries.size() && entries[numValid].cellID != 0xFFFFFFFFu) ++numValid;
    std::vector<uint32_t> flag(numValid + 1), cellIdxOf(numValid + 1);
    for (uint32_t i = 0; i < numValid; ++i) sh_markStarts(entries.data(), numValid, flag.data(), i);
    uint32_t numCells = 0;
    for (uint32_t i = 0; i < numValid; ++i) {
        numCells += flag[i];
        cellIdxOf[i] = numCells - 1;
    }
    std::vector<uint32_t> cpRaw(5 * (size_t)std::max(numCells, 1u), 0u);  // CellProp: 5 words, zeroed
    CellProp* cp = reinterpret_cast<CellProp*>(cpRaw.data());
    for (uint32_t i = 0; i < numValid; ++i)
        sh_fillCellProp(entries.data(), flag.data(), cellIdxOf.data(), numValid, params, cp, i);
    for (uint32_t c = 0; c < numCells; ++c) sh_computePairCount(cp, numCells, c);
    std::vector<uint32_t> pairPrefix(numCells + 1, 0);
    uint64_t running = 0;
    for (uint32_t c = 0; c < numCells; ++c) {
        pairPrefix[c] = (uint32_t)running;
        running += cpRaw[5 * (size_t)c + 3];  // pairCnt
    }
    pairPrefix[numCells] = (uint32_t)running;
    SHBroadParams bp;
    bp.numCandidatePairs = (uint32_t)running;
    bp.numCells = numCells;
    bp.maxNumCollisions = cap;
    bp.enableSelfCollisions = enableSelf ? 1u : 0u;
    bp.epsilon = margin;
    atomic_uint counter;
    counter.v.store(0);
    for (uint32_t id = 0; id < bp.numCandidatePairs; ++id)
        sh_broadPhase(entries.data(), cp, pairPrefix.data(), faceCB.data(), faceObj.data(), (const packed_uint3*)F,
                      facetOff, (const packed_float3*)centroid.data(), radius.data(), behaviors, shapes, bp, &counter,
                      (BroadCollision*)rows, id);
    out6[0] = numValid; out6[1] = numCells; out6[2] = bp.numCandidatePairs;
    out6[3] = params.gridRes[0]; out6[4] = params.gridRes[1]; out6[5] = params.gridRes[2];
    return counter.v.load();
}

}  // extern "C"
#else
#error "select YS_REF_BVH, YS_REF_NARROW, YS_REF_PHYSICS or YS_REF_SH"
#endif
