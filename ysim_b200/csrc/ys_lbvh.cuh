// ys_lbvh.cuh -- linear BVH over triangles: Morton codes, Karras topology,
// swept refit.  Node layout and slot numbering follow the reference
// (bvh.hpp:148-177, bvh.metal:260-393): internal nodes [0, N-2] with the root
// at slot 0, leaves at [N-1, 2N-2].
#pragma once
#include <cstring>

#include "ys_common.cuh"
#include "ys_scan.cuh"

namespace ys {

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

// expandBits (bvh.metal:26-32): the 10 low bits of v spread to every third bit.
__device__ __forceinline__ u32 expand_bits(u32 v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// One tree to refit: leaves are recomputed from positions (optionally swept by
// v*dt) and combined bottom-up.  Positions/velocities are float4 (padded) or
// packed float3 (reference layout) depending on which pointer is set.
struct RefitJob {
    Node* nodes;            // 2N-1 nodes
    const i32* parent;      // 2N-1: largest internal node claiming the node as a child (-1: none)
    const u32* claimOff;    // claimant lists: node c's are claims[claimOff[c-1] (0 for c = 0) .. claimOff[c])
    const i32* claims;      // 2N-2 internal node ids
    u32* visits;            // N-1 per-internal-node arrival counters
    const u32* facets;      // 3 local vertex ids per face (packed)
    const float4* x4;       // positions (float4) or nullptr
    const float4* v4;
    const float* x3;        // positions (packed xyz) or nullptr
    const float* v3;
    u32 voff;               // vertex offset of this mesh in x4/v4
    u32 n;                  // leaves
    u32 leafBase;           // prefix of leaves over jobs
    float dt;
    u32 swept;
    float selfMargin;       // > 0: also reduce the H1 grid extent into *maxExt
    u32* maxExt;            // float bits, atomicMax (positive floats order as ints)
    // 4-wide form (cube layout): when set the refit fills the wide nodes'
    // child slots and the binary root box instead of the binary nodes
    Wide4* w4;
    const int2* leafW;      // per leaf: (wide node, slot)
    u32* warrive;           // per wide node: arrivals this refit (self-resetting)
    // root only: no query descends this tree, only its root box is used (the
    // inter-object cull); the leaves (face i for thread i, the tree need not
    // be built) are reduced straight into rootAcc (3 ordered-int minima, then
    // 3 maxima) and launch_refit_roots writes the root node and resets
    // rootAcc to (~0, ~0, ~0, 0, 0, 0) for the next refit.
    u32 rootOnly;
    u32* rootAcc;
    u32 nVert;              // vertices of the mesh (vertex form of the root box)
    // level-synchronous 4-wide refit: the leaf kernel (face order) only
    // writes each leaf box into its slot (leafWf); launch_refit_levels then
    // combines the wide nodes height by height
    u32 levels;
    const int2* leafWf;     // per face: (wide node, slot)
    const u32* wcount;      // number of wide nodes of this tree
    u32* hacc;              // per wide node: height (1 = leaf children only)
    // face positions (or null): per face its three vertices' current
    // positions, each float4 carrying the mesh-local vertex id in w, written
    // by the leaf pass for the queries that test the face
    float4* fpos;
    // range refit of the 4-wide form (with levels; leafBase a multiple of
    // 256): the leaf pass runs in sorted-leaf order (idx: the face of each
    // sorted leaf), writes each leaf box into its binary leaf node and its
    // wide slot (leafW) and the boxes of every 16- and 256-leaf block (bb16 /
    // bb256, indexed by (leafBase + leaf) / 16 and / 256);
    // launch_refit_ranges then gives every internal wide child its slot box,
    // and the tree its root box, as the union of the leaves of a sorted-leaf
    // range (wrange), from the block boxes.
    u32 ranges;
    const u32* idx;
    // range mode, optional: per sorted leaf its face's three vertex ids and
    // the face id (w), written at the build (one coalesced load in place of
    // the face index and the facet)
    const uint4* lvid;
    Node* bb16;
    Node* bb256;
    uint2* wrange;          // per wide node: (first, last) sorted leaf under it
    // the wide nodes whose range lies in one 256-leaf block, per block (index
    // (leafBase + leaf) / 256): (parent, slot, first, last) records
    // blkEnt[blkOff[b] .. blkOff[b + 1]); the leaf pass's block fills their
    // slots from its leaf boxes in shared memory
    const uint4* blkEnt;
    const u32* blkOff;
};

// Scene box of a mesh (min/max over all its vertices) into box[6] (float
// bits stored via ordered-int atomics; call box_init first).
void launch_box_init(u32* box, cudaStream_t s);
void launch_box(const float4* x4, const float* x3, u32 voff, u32 nV, u32* box, cudaStream_t s);
// Morton code per face from the scene box (fillMortons_Tri, bvh.metal:42-63);
// cube = one scale for all axes (the box's largest width) instead of per axis.
void launch_morton(const float4* x4, const float* x3, u32 voff, const u32* facets, u32 nF, const u32* box, u32* codes,
                   u32* idx, cudaStream_t s, bool cube = false);
// Karras topology (buildTree_Tri, bvh.metal:352-393); zeroes visit counters.
// Runs of three or more equal Morton codes make the reference's topology
// inconsistent (findSplit splits them at the midpoint, bvh.metal:204, while
// determineRange orders them by index): a node can then be claimed as a child
// by several internal nodes, or by none.  Child arrays stay exactly the
// reference's; parent keeps the largest claimant (what a serial build loop
// leaves behind) and the claimant lists (claimOff, 2N entries; claims, 2N - 2)
// hold every claimant, so the refit reaches all of them.
// consistent = true splits runs of equal codes by the (code, index) key that
// determineRange already orders them by, so every node has one parent (the
// cube layout); false keeps the reference's midpoint split.
size_t karras_scratch_bytes(u32 n);
// Optional outputs of a Karras build for the range refit of a consistent
// tree: per internal node its sorted-leaf range, and the nodes whose range
// leaves the 256-leaf block of their own index, in big (ranges under
// BIN_RANGE_HUGE leaves, count[0]) or huge (count[1]); both lists need n
// entries.  range = null: none.
static constexpr u32 BIN_RANGE_HUGE = 16384;
struct BinRanges {
    uint2* range = nullptr;
    u32* big = nullptr;
    u32* huge = nullptr;
    u32* count = nullptr;
};
cudaError_t launch_karras(const u32* codes, const u32* idx, u32 n, Node* nodes, i32* parent, u32* claimOff,
                          i32* claims, u32* visits, void* scratch, cudaStream_t s, bool consistent = false,
                          BinRanges R = BinRanges());
// Range refit of a consistent binary tree built with BinRanges (J: nodes,
// facets, positions (and velocities when swept), n; bb16 / bb256 with
// n / 16 + 1 and n / 256 + 1 boxes): leaf pass, then the big and huge nodes.
// With rank (each face's sorted-leaf position) and lbox (2 float4 per leaf) a
// face-order pass computes the leaf boxes first, so the leaf pass reads them
// in order instead of gathering facets and vertices.
void launch_refit_bin(const RefitJob& J, const uint2* range, const u32* big, u32 nbig, const u32* huge, u32 nhuge,
                      const u32* rank, float4* lbox, cudaStream_t s);
// lvid[i] = (facet of idx[i], idx[i]) for the sorted faces of a build.
void launch_leaf_vids(const u32* idx, const u32* facets, u32 n, uint4* lvid, cudaStream_t s);
// rank[idx[i]] = i for the sorted face indices of a build.
void launch_leaf_rank(const u32* idx, u32 n, u32* rank, cudaStream_t s);
// Apetrei build (agglomerativeBuild_Tri + agglomerativeSwapRoot,
// bvh.metal:884-1199) of sorted (code, index) pairs: topology, leaf boxes
// from the current positions and every internal box in one pass, the root
// moved to slot 0, claimant lists filled as launch_karras does, visit
// counters left even.  Its tree is consistent for any input (runs of equal
// codes split by index).  aggScratch holds apetrei_scratch_bytes(n).
size_t apetrei_scratch_bytes(u32 n);
cudaError_t launch_apetrei(const float4* x4, const float* x3, u32 voff, const u32* facets, const u32* codes,
                           const u32* idx, u32 n, Node* nodes, i32* parent, u32* claimOff, i32* claims, u32* visits,
                           void* scanScratch, void* aggScratch, u32* status, cudaStream_t s);
// 4-wide form of a consistent binary tree of n leaves: internal nodes at even
// depth become wide nodes (numbered by an exclusive scan), their children and
// grandchildren their slots.  w4 and warrive need max(n - 1, 1) entries,
// leafW n, scratch wide_build_scratch_bytes(n).  Boxes are filled by a refit.
size_t wide_build_scratch_bytes(u32 n);
cudaError_t launch_wide_build(const Node* nodes, const i32* parent, u32 n, Wide4* w4, int2* leafW, int2* leafWf,
                              u32* warrive, u32* wcount, void* scratch, cudaStream_t s);

// Level lists of the 4-wide trees of a job table (jobs with w4 and levels):
// heights by a climb, then every wide node into the list of its height as
// (node, job).  hcount / hoff: MAX_LEVELS + 1 entries; the host reads hcount
// to size the level launches.
static constexpr u32 MAX_LEVELS = 64;
void launch_wide_heights(const RefitJob* jobsDev, u32 numJobs, u32 totalLeaves, u32* status, cudaStream_t s);
void launch_level_count(const RefitJob* jobsDev, u32 numJobs, u32 totalLeaves, u32* hcount, u32* status,
                        cudaStream_t s);
void launch_level_fill(const RefitJob* jobsDev, u32 numJobs, u32 totalLeaves, const u32* hoff, u32* hcursor,
                       uint2* list, cudaStream_t s);
// Per substep, after launch_refit wrote the leaf slots: levels 1 .. split-1
// one launch each (hostOff[h] .. hostOff[h+1] of list), then levels split ..
// top in one block, level by level.
// Query points in Morton order (over their own box): idx[k] is the point of
// sorted slot k.  The standalone point queries run one thread per sorted
// slot, so neighbouring threads query neighbouring points and share the tree
// nodes / hash buckets they read.  Buffers grow on demand.
struct QueryOrder {
    u32* codes = nullptr;
    u32* idx = nullptr;
    void* scratch = nullptr;
    u32* box = nullptr;
    u32 cap = 0;
};
// From these sizes on the order pays for its sort (measured on uniform
// points: LBVH query at 4M 1.64 -> 1.38 ms and 16M 18.3 -> 11.4 ms, at 1M
// 0.32 -> 0.37 ms; hash query at 16M 44.0 -> 40.2 ms, at 4M 3.48 -> 3.60 ms)
static constexpr u32 QUERY_ORDER_MIN_LBVH = 1u << 21;
static constexpr u32 QUERY_ORDER_MIN_HASH = 1u << 23;
cudaError_t query_order(QueryOrder& o, const float* qx, u32 n, cudaStream_t s);
void query_order_free(QueryOrder& o);

// The range refit's second pass (after launch_refit) over the records
// (parent, slot | job << 2, first, last) of the wide nodes whose range spans
// more than one 256-leaf block: nmed at the front of big (8 lanes each), nhuge
// at its back (ranges over 16384 leaves, a block each), then a block per job
// for its root box.
void launch_refit_ranges(const RefitJob* jobsDev, u32 numJobs, const uint4* big, u32 bigCap, u32 nmed, u32 nhuge,
                         cudaStream_t s);
// The range refit's node records after launch_wide_heights: each non-root
// wide node of the range jobs goes to the list of the 256-leaf block holding
// its range, or to big (bigCap records: medium ones from the front, huge
// ones from the back).  blkCnt (numBlocks + 1 entries) is used as scratch;
// blkOff gets the per-block offsets; bigCnt[0] / [1] the medium and huge
// counts.  Scratch of scan_scratch_bytes(numBlocks + 1).
cudaError_t launch_range_lists(const RefitJob* jobsDev, u32 numJobs, u32 totalLeaves, u32* blkCnt, u32* blkOff,
                               uint4* blkEnt, uint4* big, u32 bigCap, u32* bigCnt, void* scanScratch,
                               cudaStream_t s);
// Allow the top-levels refit kernel its staging shared memory (once, before
// the first launch_refit_levels; not during a stream capture).
cudaError_t refit_levels_prepare();
void launch_refit_levels(const RefitJob* jobsDev, const uint2* list, const u32* hoffDev, const u32* hostOff,
                         u32 top, cudaStream_t s);
// Leaves + bottom-up for every job (jobs in device memory, jobsHost mirrors
// them for the launch size).
void launch_refit(const RefitJob* jobsDev, u32 numJobs, u32 totalLeaves, u32* status, cudaStream_t s);
// Root boxes of the root-only jobs from their accumulators (after launch_refit).
void launch_refit_roots(const RefitJob* jobsDev, u32 numJobs, cudaStream_t s);
// Root boxes from vertices, for meshes whose every vertex belongs to a face
// (then the union of the swept leaf boxes is the union of {x, x + v dt} over
// the vertices): one block per chunk (job, first vertex) of ROOT_CHUNK
// vertices, then launch_refit_roots on the same jobs.
static constexpr u32 ROOT_CHUNK = 512;
void launch_root_boxes(const RefitJob* jobsDev, u32 numJobs, const uint2* chunks, u32 numChunks, cudaStream_t s);

}  // namespace ys
