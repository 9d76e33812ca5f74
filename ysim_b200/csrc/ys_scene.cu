// ys_scene.cu -- the packed scene, the per-substep kernels and the C ABI.
//
// Host side restates Scene<BE,PR>::pack (scene.hpp:783-1180),
// MeshAdjacencyInitializer (mesh_state.hpp:236-411) and the substep order of
// Simulator::update (simulator.hpp:3512-3815).  Device side has two paths
// with identical results:
//   staged -- one kernel group per reference stage: swept refit, broad rows,
//             narrow contacts, per-vertex CSR, forces, integrate;
//   fused  -- swept refit, then ONE kernel per substep in which the thread of
//             a vertex traverses the trees, runs the narrow test on every
//             candidate, keeps its contacts in canonical order in local
//             memory, gathers its spring forces and integrates.  Broad rows,
//             contacts and forces never touch HBM.
// xPrev is not copied: positions live in three rotating buffers (current,
// previous, next), so SymplecticSystem::snapshotXPrev becomes a pointer
// rotation.
#include <cuda.h>  // CUtensorMap and the cuTensorMapEncodeTiled prototype (the entry point comes from the runtime)

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "ys_analytic.cuh"
#include "ys_collide.cuh"
#include "ys_common.cuh"
#include "ys_lbvh.cuh"
#include "ys_scan.cuh"
#include "ys_sort.cuh"
#include "ysim_b200.h"

namespace ys {

thread_local std::string g_err;
ys_status fail(ys_status code, const std::string& msg) {
    g_err = msg;
    return code;
}
#define YS_CK(call)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return fail(YS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

enum : u32 {
    MF_STATIC = 1, MF_COLLIDABLE = 2, MF_SELF = 4, MF_QUERY = 8, MF_CLOTH = 16, MF_TREE = 32, MF_GRID = 64,
    MF_ANALYTIC = 128,  // analytic collider: tested against its shape, its triangles unused
};
static constexpr int MAXC = 32;  // per-vertex contact buffer of the fused kernel

struct MeshDev {
    u32 voff, nV, foff, nF;
    u32 node_off, behavior, flags, grid_n;
    float kstretch, kshear, kbend, thickness;
    float rest[6];
    u32 tgt_begin, tgt_end;
    u32 gspr;  // FastGridCloth: offset of this mesh's per-spring k / L arrays, or NO_SPRINGS
    u32 w4_off, w4_cap;  // wide nodes of this mesh's tree (cube layout)
    u32 shape;           // analytic collider: slot in the shape table
    u32 tmap;            // FastGridCloth: first of its 5 tensor maps (X[0..2], V[0..1]) or NO_PAIR
    u32 pad[2];
};
static constexpr u32 NO_SPRINGS = 0xFFFFFFFFu;
static constexpr u32 NO_PAIR = 0xFFFFFFFFu;

struct StepArgs {
    const float4* x;
    const float4* xp;
    const float4* v;
    float4* xn;
    float4* vn;
    const float* mass;
    const float* mask;
    const u32* vobj;
    const MeshDev* meshes;
    const u32* targets;
    const uint4* F;
    // per face (global face index): its three vertices' positions at the
    // start of the substep, the mesh-local vertex id in w (written by the
    // refit's leaf pass, or at the build of a tree that is never refit)
    const float4* fpos;
    // per vertex, its own faces (the faces holding it) as two windows of 8
    // face ids: x = first id of window A, y = (B - A) << 16 | mask B << 8 |
    // mask A; a vertex whose faces do not fit has both masks 0
    const uint2* own;
    const Node* nodes;
    const Wide4* w4;  // 4-wide form of the trees (wide != 0)
    u32 wide;
    const u32* spr_off;
    const u32* spr_split;
    const u32* spr_nbr;
    const float* spr_rest;
    const u32* vaf_off;
    const u32* vaf;
    const u32* maxext;
    const float4* ext;  // external forces (applyEnvironmentForces) or null: g * m
    const float* gk;    // per-spring stiffness / rest length of grid cloths (MeshDev::gspr)
    const float* gL;
    // analytic colliders: shape table, marker pair of each target entry (or
    // NO_PAIR), marker pairs (cloth, collider, slot, first thread), and the
    // marker flags of this detect (written) and of the previous one (read)
    const DShape* shapes;
    const u32* tpair;
    const uint4* apairs;
    u32* mk_fresh;
    const u32* mk_held;
    u32 npairs, apair_total;
    u32 analytic;  // the scene has analytic colliders
    float subh, kair, kd, gx, gy, gz, margin, band, radius;
    u32 nV, self_mode, record, cap;
    // fused kernel: thread t of a launch works on vertex vorder[tbase + t]
    // (the working vertices: static non-query vertices are left out) while
    // tbase + t < tend.  vorder lists the meshes of one size class after
    // another, each mesh's vertices in Morton or vertex order; a launch covers
    // one class.
    const u32* vorder;
    u32 tbase, tend;
    // tile thread order (a launch over a class in that order): each CTA of a
    // FastGridCloth is one 16 x 8 tile, whose positions and velocities with a
    // 2-vertex halo come into shared memory by two TMA loads through the
    // mesh's tensor maps (tmaps[tmap + xbuf], tmaps[tmap + 3 + vbuf])
    u32 tiles, xbuf, vbuf;
    const CUtensorMap* tmaps;
    u32* status;
    unsigned long long* counters;  // [0] broad rows, [1] contacts, [2] pool fill, [3] [4] running totals of 0, 1
    // fused record pool
    VContact* pool;
    u32* vstart;
    u32* vcount;
    // staged path
    Row* rows;
    Contact* contacts;
    float4* f;
    u32* bucket;    // per-vertex counts / fill (V + 1)
    u32* csr_off;   // V + 1
    VContact* csr;
};

// ------------------------------------------------------------------ query
// BroadPhase::detectCollisions for one query vertex (bvh.hpp:2853-2949 and
// the hybrid self pass, simulator.hpp:3678-3701): self rows first, then every
// target mesh whose root box overlaps this mesh's root box.
// Leaves of mesh t's tree overlapping [qmn, qmx], binary or 4-wide form.
template <class Fn>
__device__ __forceinline__ u32 descend(const StepArgs& A, const MeshDev& T, f3 qmn, f3 qmx, Fn&& fn) {
    if (A.wide) return traverse_wide(A.nodes + T.node_off, A.w4 + T.w4_off, T.w4_cap, qmn, qmx, fn);
    return traverse(A.nodes + T.node_off, 2 * T.nF - 1, qmn, qmx, fn);
}

template <class Sink>
__device__ __forceinline__ u32 query_vertex(const StepArgs& A, u32 g, u32 m, const MeshDev& M, f3 xc, f3 xpv,
                                            Sink&& sink) {
    u32 st = 0;
    if (!(M.flags & MF_QUERY) || !(M.flags & MF_TREE)) return 0;
    const u32 lid = g - M.voff;
    const float mg = A.margin;
    if (A.self_mode == YS_SELF_HASH && (M.flags & MF_CLOTH) && (M.flags & MF_SELF)) {
        float mx = __uint_as_float(A.maxext[m]);
        float cs = (mx > 1e-5f) ? mx : 1e-5f;
        float inv = 1.f / cs;
        H1Vertex h;
        if (h1_vertex(xc, xpv, inv, h)) {
            f3 qmn, qmx;
            h1_query_box(h, mg, qmn, qmx);
            st |= descend(A, M, qmn, qmx, [&](u32 f) {
                uint4 tri = A.F[M.foff + f];
                if (h1_face(A.x, M.voff, tri, lid, mg, inv, h)) sink(m, f, tri, M.voff);
            });
        }
    } else if (A.self_mode == YS_SELF_BVH && !(M.flags & MF_ANALYTIC)) {
        f3 qmn = xc - mk(mg, mg, mg), qmx = xc + mk(mg, mg, mg);
        st |= descend(A, M, qmn, qmx, [&](u32 f) {
            uint4 tri = A.F[M.foff + f];
            if (tri.x == lid || tri.y == lid || tri.z == lid) return;
            sink(m, f, tri, M.voff);
        });
    }
    for (u32 k = M.tgt_begin; k < M.tgt_end; ++k) {
        const u32 t = A.targets[k];
        const MeshDev T = A.meshes[t];
        // an analytic collider has no live tree and queries none (its pairs
        // are markers)
        if ((T.flags & MF_ANALYTIC) || (M.flags & MF_ANALYTIC) || T.nF == 0) continue;
        if (!root_overlap(A.nodes + M.node_off, A.nodes + T.node_off)) continue;
        f3 qmn = xc - mk(mg, mg, mg), qmx = xc + mk(mg, mg, mg);
        st |= descend(A, T, qmn, qmx, [&](u32 f) {
            uint4 tri = A.F[T.foff + f];
            sink(t, f, tri, T.voff);
        });
    }
    return st;
}

__device__ __forceinline__ bool key_less(u32 t1, u32 f1, u32 t2, u32 f2) { return t1 < t2 || (t1 == t2 && f1 < f2); }

// The 12 stencil springs of grid vertex (row, col) in the order of
// compute_cloth_grid_forces_fast (physics.metal:197-218): fn(r, c, family,
// spring id).  Families 0..5 = stretch x, stretch y, shear "\\", shear "/",
// bend x, bend y (rest[family]; k = kstretch, kstretch, kshear, kshear,
// kbend, kbend); spring ids number each family row-major, families
// concatenated in that order.
template <class Fn>
__device__ __forceinline__ void grid_stencil(int N, int row, int col, Fn&& fn) {
    const u32 n = (u32)N;
    const u32 bSY = n * (n - 1), bHA = bSY + (n - 1) * n, bHB = bHA + (n - 1) * (n - 1), bBX = bHB + (n - 1) * (n - 1),
              bBY = bBX + n * (n - 2);
    const u32 r = (u32)row, c = (u32)col;
    if (col > 0) fn(row, col - 1, 0, r * (n - 1) + c - 1);
    if (col < N - 1) fn(row, col + 1, 0, r * (n - 1) + c);
    if (row > 0) fn(row - 1, col, 1, bSY + (r - 1) * n + c);
    if (row < N - 1) fn(row + 1, col, 1, bSY + r * n + c);
    if (col > 0 && row > 0) fn(row - 1, col - 1, 2, bHA + (r - 1) * (n - 1) + c - 1);
    if (col < N - 1 && row > 0) fn(row - 1, col + 1, 3, bHB + (r - 1) * (n - 1) + c);
    if (col > 0 && row < N - 1) fn(row + 1, col - 1, 3, bHB + r * (n - 1) + c - 1);
    if (col < N - 1 && row < N - 1) fn(row + 1, col + 1, 2, bHA + r * (n - 1) + c);
    if (col > 1) fn(row, col - 2, 4, bBX + r * (n - 2) + c - 2);
    if (col < N - 2) fn(row, col + 2, 4, bBX + r * (n - 2) + c);
    if (row > 1) fn(row - 2, col, 5, bBY + (r - 2) * n + c);
    if (row < N - 2) fn(row + 2, col, 5, bBY + r * n + c);
}

__device__ __forceinline__ void grid_spring_kL(const StepArgs& A, const MeshDev& M, int fam, u32 sid, float& k,
                                               float& rest) {
    if (M.gspr != NO_SPRINGS) {
        k = A.gk[M.gspr + sid];
        rest = A.gL[M.gspr + sid];
    } else {
        k = fam < 2 ? M.kstretch : (fam < 4 ? M.kshear : M.kbend);
        rest = M.rest[fam];
    }
}

// Spring forces of one cloth vertex from the old state:
// compute_cloth_grid_forces_fast (physics.metal:171-224) or
// compute_tri_spring_forces (physics.metal:319-378).
// The force before the springs: environment (g * m, or the external-force
// buffer) plus air drag.
__device__ __forceinline__ f3 base_force(const StepArgs& A, u32 g, f3 vel, float mass) {
    return (A.ext ? ld(A.ext, g) : mk(A.gx * mass, A.gy * mass, A.gz * mass)) + vel * A.kair;
}

__device__ __forceinline__ f3 vertex_force(const StepArgs& A, const MeshDev& M, u32 g, f3 pos, f3 vel, float mass) {
    f3 force = base_force(A, g, vel, mass);
    const float kd = A.kd;
    if (M.flags & MF_GRID) {
        const int N = (int)M.grid_n;
        const u32 lid = g - M.voff;
        const int row = (int)(lid / (u32)N), col = (int)(lid % (u32)N);
        grid_stencil(N, row, col, [&](int r, int c, int fam, u32 sid) {
            float k, rest;
            grid_spring_kL(A, M, fam, sid, k, rest);
            u32 j = M.voff + (u32)(r * N + c);
            force = force + spring(pos, vel, ld(A.x, j), ld(A.v, j), rest, k, kd);
        });
    } else {
        const u32 b = A.spr_off[g], s = A.spr_split[g], e = A.spr_off[g + 1];
        for (u32 i = b; i < s; ++i) {
            u32 j = A.spr_nbr[i];
            force = force + spring(pos, vel, ld(A.x, j), ld(A.v, j), A.spr_rest[i], M.kstretch, kd);
        }
        for (u32 i = s; i < e; ++i) {
            u32 j = A.spr_nbr[i];
            force = force + spring(pos, vel, ld(A.x, j), ld(A.v, j), A.spr_rest[i], M.kbend, kd);
        }
    }
    return force;
}

// ---------------------------------------------------------- grid-cloth tiles
// In tile thread order a CTA's 128 threads are one 16 x 8 tile of a
// FastGridCloth (tile-row-major, 16 vertices per tile row).  Each spring with
// an end in the tile is evaluated once, as the force on its first end a from
// its second end b.  Seen from b the force is its negation, bit for bit (dx,
// dv and the unit vector change sign exactly, the length and the scalar
// factor do not change), except where both ends compute the same value: a
// component whose dx is exactly zero (+0 in the unit vector from either end)
// and a degenerate spring (+0 from both ends).  The table keeps those cases
// in a flag byte per spring, so each vertex sums its 12 stencil springs in
// the reference's order from the table and gets the per-vertex loop's result
// exactly, signed zeros included.  890 evaluations per full tile instead of
// 1536.
//
// Springs of the tile, by family (first end a, second end b = a + (dr, dc)),
// a's rows and columns relative to the tile origin:
//   0 stretch x  rows 0..7,  cols -1..15  b = a + (0, 1)
//   1 stretch y  rows -1..7, cols 0..15   b = a + (1, 0)
//   2 shear "\\" rows -1..7, cols -1..15  b = a + (1, 1)
//   3 shear "/"  rows -1..7, cols 0..16   b = a + (1, -1)
//   4 bend x     rows 0..7,  cols -2..15  b = a + (0, 2)
//   5 bend y     rows -2..7, cols 0..15   b = a + (2, 0)
static constexpr int TILE_W = 16, TILE_H = 8;
static constexpr int HALO_W = TILE_W + 4, HALO_H = TILE_H + 4;  // the stencil reaches 2 vertices out
static constexpr u32 TILE_BOX_BYTES = HALO_W * HALO_H * 16;      // one float4 buffer's tile
static constexpr u32 TILE_FLAG_BYTES = 896;                      // one flag byte per tile spring
// x and v tiles, then the spring flags; 128-byte aligned
static constexpr size_t TILE_SMEM = 2 * TILE_BOX_BYTES + TILE_FLAG_BYTES + 128;
// first spring of each family in the tile's table
static constexpr u32 TS_SX = 0, TS_SY = 136, TS_HA = 280, TS_HB = 433, TS_BX = 586, TS_BY = 730;
static constexpr u32 TILE_SPRINGS = 890;

__device__ __forceinline__ u32 smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void tile_load(float4* xs, const CUtensorMap* mx, const CUtensorMap* mv, int r0, int c0,
                                          unsigned long long* bar) {
    const u32 b = smem_u32(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    // the maps were written by a host copy: acquire them for the tensor-map proxy
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(mx) : "memory");
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(mv) : "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(2u * TILE_BOX_BYTES) : "memory");
    // box {4 floats, HALO_W columns, HALO_H rows} from (0, c0 - 2, r0 - 2):
    // the innermost coordinate is always 0; rows or columns outside the
    // mesh read zeros (their springs are never used)
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(xs)), "l"(mx), "r"(0), "r"(c0 - 2), "r"(r0 - 2), "r"(b) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(xs + HALO_W * HALO_H)), "l"(mv), "r"(0), "r"(c0 - 2), "r"(r0 - 2), "r"(b) : "memory");
}

// Bounded wait for the tile's two loads (phase 0 of the barrier).
__device__ __forceinline__ bool tile_wait(unsigned long long* bar) {
    const u32 b = smem_u32(bar);
    for (u32 i = 0; i < (1u << 22); ++i) {
        u32 done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done) : "r"(b) : "memory");
        if (done) return true;
    }
    return false;
}

// The springs of one family of the tile at origin (r0, c0) of a grid mesh of
// side N: force on a from b into sf[0..2][base + i] (zeros for springs off
// the mesh).  Thread t starts at (t + 32 * FAM) mod 128, so that each
// family's remainder past 128 springs falls to another warp.  k and rest are
// the family's values, or per spring from gk / gL at gspr (not NO_SPRINGS).
template <int FAM>
__device__ __forceinline__ void tile_family(const StepArgs& A, u32 gspr, u32 n, int r0, int c0, float kf, float restf,
                                            const float4* xs, const float4* vs, float* sf, unsigned char* flags) {
    constexpr u32 W = FAM == 4 ? 18u : ((FAM == 1 || FAM == 5) ? 16u : 17u);
    constexpr u32 H = FAM == 5 ? 10u : ((FAM >= 1 && FAM <= 3) ? 9u : 8u);
    constexpr u32 BASE = FAM == 0 ? TS_SX : FAM == 1 ? TS_SY : FAM == 2 ? TS_HA : FAM == 3 ? TS_HB : FAM == 4 ? TS_BX : TS_BY;
    constexpr int AR = FAM == 5 ? -2 : ((FAM >= 1 && FAM <= 3) ? -1 : 0);
    constexpr int AC = FAM == 4 ? -2 : ((FAM == 0 || FAM == 2) ? -1 : 0);
    constexpr int DR = FAM == 5 ? 2 : ((FAM >= 1 && FAM <= 3) ? 1 : 0);
    constexpr int DC = FAM == 4 ? 2 : ((FAM == 0 || FAM == 2) ? 1 : (FAM == 3 ? -1 : 0));
    static_assert(BASE + W * H <= TILE_SPRINGS, "tile table");
    for (u32 i = (threadIdx.x + 32u * FAM) & 127u; i < W * H; i += 128u) {
        const int rr = (int)(i / W), cc = (int)(i % W);
        const int ar = r0 + AR + rr, ac = c0 + AC + cc, br = ar + DR, bc = ac + DC;
        f3 F = mk(0.f, 0.f, 0.f);
        u32 fl = 0;
        if ((u32)ar < n && (u32)ac < n && (u32)br < n && (u32)bc < n) {
            const int ia = (AR + 2 + rr) * HALO_W + (AC + 2 + cc), ib = ia + DR * HALO_W + DC;
            float k = kf, rest = restf;
            if (gspr != NO_SPRINGS) {
                const u32 R = (u32)ar, C = (u32)ac;
                const u32 bSY = n * (n - 1), bHA = bSY + (n - 1) * n, bHB = bHA + (n - 1) * (n - 1),
                          bBX = bHB + (n - 1) * (n - 1), bBY = bBX + n * (n - 2);
                const u32 sid = FAM == 0 ? R * (n - 1) + C
                              : FAM == 1 ? bSY + R * n + C
                              : FAM == 2 ? bHA + R * (n - 1) + C
                              : FAM == 3 ? bHB + R * (n - 1) + C - 1
                              : FAM == 4 ? bBX + R * (n - 2) + C
                                         : bBY + R * n + C;
                k = A.gk[gspr + sid];
                rest = A.gL[gspr + sid];
            }
            const float4 pa = xs[ia], va = vs[ia], pb = xs[ib], vb = vs[ib];
            const f3 P0 = mk(pa.x, pa.y, pa.z), P1 = mk(pb.x, pb.y, pb.z);
            F = spring(P0, mk(va.x, va.y, va.z), P1, mk(vb.x, vb.y, vb.z), rest, k, A.kd);
            // the cases where b computes the same value as a (see above)
            const f3 dx = P1 - P0;
            fl = (dx.x == 0.f ? 1u : 0u) | (dx.y == 0.f ? 2u : 0u) | (dx.z == 0.f ? 4u : 0u) |
                 (sqrtf(dot(dx, dx)) < 1e-7f ? 7u : 0u);
        }
        flags[BASE + i] = (unsigned char)fl;
        sf[BASE + i] = F.x;
        sf[TILE_SPRINGS + BASE + i] = F.y;
        sf[2 * TILE_SPRINGS + BASE + i] = F.z;
    }
}

// Every spring of the tile at origin (r0, c0) of grid mesh M.
__device__ __forceinline__ void tile_springs(const StepArgs& A, const MeshDev& M, int r0, int c0, const float4* xs,
                                             const float4* vs, float* sf, unsigned char* flags) {
    const u32 n = M.grid_n, gspr = M.gspr;
    const float ks = M.kstretch, kh = M.kshear, kb = M.kbend;
    const float r[6] = {M.rest[0], M.rest[1], M.rest[2], M.rest[3], M.rest[4], M.rest[5]};
    tile_family<0>(A, gspr, n, r0, c0, ks, r[0], xs, vs, sf, flags);
    tile_family<1>(A, gspr, n, r0, c0, ks, r[1], xs, vs, sf, flags);
    tile_family<2>(A, gspr, n, r0, c0, kh, r[2], xs, vs, sf, flags);
    tile_family<3>(A, gspr, n, r0, c0, kh, r[3], xs, vs, sf, flags);
    tile_family<4>(A, gspr, n, r0, c0, kb, r[4], xs, vs, sf, flags);
    tile_family<5>(A, gspr, n, r0, c0, kb, r[5], xs, vs, sf, flags);
}

// The 12 stencil springs of vertex (row, col) at (ty, tx) in its tile, in
// grid_stencil's order, from the tile's table: the table's force for the
// springs whose first end is the vertex, its negation for the others (but
// for the components the flags keep).
__device__ __forceinline__ f3 tile_force(f3 force, int N, int row, int col, int ty, int tx, const float* sf,
                                         const unsigned char* flags) {
    auto add = [&](u32 i, bool neg) {
        f3 F = mk(sf[i], sf[TILE_SPRINGS + i], sf[2 * TILE_SPRINGS + i]);
        if (neg) {
            const u32 fl = flags[i];
            F = mk((fl & 1u) ? F.x : -F.x, (fl & 2u) ? F.y : -F.y, (fl & 4u) ? F.z : -F.z);
        }
        force = force + F;
    };
    const u32 y = (u32)ty, x = (u32)tx;
    if (col > 0) add(TS_SX + y * 17 + x, true);
    if (col < N - 1) add(TS_SX + y * 17 + x + 1, false);
    if (row > 0) add(TS_SY + y * 16 + x, true);
    if (row < N - 1) add(TS_SY + (y + 1) * 16 + x, false);
    if (col > 0 && row > 0) add(TS_HA + y * 17 + x, true);
    if (col < N - 1 && row > 0) add(TS_HB + y * 17 + x + 1, true);
    if (col > 0 && row < N - 1) add(TS_HB + (y + 1) * 17 + x, false);
    if (col < N - 1 && row < N - 1) add(TS_HA + (y + 1) * 17 + x + 1, false);
    if (col > 1) add(TS_BX + y * 18 + x, true);
    if (col < N - 2) add(TS_BX + y * 18 + x + 2, false);
    if (row > 1) add(TS_BY + y * 16 + x, true);
    if (row < N - 2) add(TS_BY + (y + 2) * 16 + x, false);
    return force;
}

// Warp-aggregated add of v into ctr[0] and the running total ctr[3].
__device__ __forceinline__ void warp_count(unsigned long long* ctr, u32 v) {
    const unsigned act = __activemask();
    u32 s = __reduce_add_sync(act, v);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(act) - 1) && s) {
        atomicAdd(ctr, (unsigned long long)s);
        atomicAdd(ctr + 3, (unsigned long long)s);
    }
}

// ------------------------------------------------------------------ fused
// One thread per vertex, but the per-candidate work (the H1 face test with its
// two point-triangle distances, and the narrow test) is not done inside the
// thread's own tree descent, where a warp would run it with the few lanes that
// reached a leaf on that iteration.  Descents only push (owner lane, mesh,
// face) into a per-warp queue in shared memory; whenever 32 candidates wait,
// the whole warp takes one each, fetching the owner's positions by shuffle.
// Contacts go back to their owner through a per-warp buffer and are inserted
// into the owner's sorted list, which keeps the MAXC smallest (mesh, face)
// keys whatever the arrival order -- so results are those of a per-vertex
// loop over candidates in descent order.
static constexpr int FUSED_WARPS = 4;  // 128-thread blocks
static constexpr u32 WQ_CAP = 160;     // candidate queue: < 32 left over + up to 4 leaves per lane
static constexpr u32 WC_CAP = 64;      // contact buffer between flushes
static constexpr u32 KEY_SELF = 32u;   // queue key: (mesh << 6) | KEY_SELF? | owner lane
static constexpr unsigned FULL_MASK = 0xFFFFFFFFu;

struct WarpWork {
    u32 qf[WQ_CAP];
    u32 qk[WQ_CAP];
    VContact cb[WC_CAP];
    unsigned char co[WC_CAP];
};

__device__ __forceinline__ void insert_contact(VContact (&buf)[MAXC], int& nc, u32& st, const VContact& c) {
    if (nc == MAXC) {
        st |= ST_CONTACT_OVF;
        if (!key_less(c.tobj, c.tri, buf[MAXC - 1].tobj, buf[MAXC - 1].tri)) return;
        --nc;
    }
    int i = nc;
    while (i > 0 && key_less(c.tobj, c.tri, buf[i - 1].tobj, buf[i - 1].tri)) { buf[i] = buf[i - 1]; --i; }
    buf[i] = c;
    ++nc;
}

// Analytic marker of one detect (BroadPhase::detectCollisions,
// bvh.hpp:2886-2941): the cloth's root box against the collider's broad box
// (AABB4::intersect; a half-space always overlaps).  A pair is live when it
// is marked at this detect or was at the previous one
// (PackedCollisionData::endAnalyticPairs, scene.hpp:485-530).  The cloth's
// first vertex records this detect's mark for the next; the flags of the two
// detects alternate between two slots by substep parity.
__device__ __forceinline__ bool analytic_live(const StepArgs& A, const DShape& S, const Node* root, u32 p, bool writer) {
    bool fresh = true;
    if (S.lo.w != 0.f) {
        const Node r = *root;
        fresh = !(S.hi.x < r.mnx || S.lo.x > r.mxx || S.hi.y < r.mny || S.lo.y > r.mxy || S.hi.z < r.mnz ||
                  S.lo.z > r.mxz);
    }
    if (writer) A.mk_fresh[p] = fresh ? 1u : 0u;
    return fresh || A.mk_held[p] != 0u;
}

// The analytic test out of line, so that the fused kernel's descent keeps its
// register allocation (the call is taken only for live collider pairs).
__device__ __noinline__ bool analytic_contact(const DShape* S, f3 pcur, f3 pprev, float radius, float thickness,
                                              VContact* c) {
    f3 n;
    float d;
    if (!analytic_narrow(S->s, pcur, pprev, radius, thickness, S->rot_margin, n, d)) return false;
    c->tobj = S->s.obj;
    c->tri = 0u;
    c->nx = n.x; c->ny = n.y; c->nz = n.z; c->d = d;
    return true;
}

// WIDE: descend the 4-wide form of the trees (cube layout), else the binary one.
// MINB: CTAs per SM the registers are capped for (8: 64 registers, 7: 72,
// 4: no cap); the results do not depend on it (ys_scene_autotune picks one).
// ANA: the scene has analytic colliders (without them the kernel carries no
// analytic branch).
static constexpr u32 NO_VERTEX = 0xFFFFFFFFu;  // a padding slot of the thread order
static_assert(sizeof(WarpWork) * FUSED_WARPS >= 3 * TILE_SPRINGS * sizeof(float),
              "the tile's spring table reuses the warps' queues");

template <bool WIDE, int MINB, bool ANA>
__global__ void __launch_bounds__(128, MINB) k_fused(StepArgs A) {
    __shared__ WarpWork wq[FUSED_WARPS];
    __shared__ unsigned long long tile_bar;
    extern __shared__ unsigned char fused_dyn[];  // TILE_SMEM bytes in tile order, else none
    const u32 lane = threadIdx.x & 31u;
    WarpWork& Q = wq[threadIdx.x >> 5];
    const u32 t = A.tbase + blockIdx.x * blockDim.x + threadIdx.x;
    u32 g = t < A.tend ? A.vorder[t] : NO_VERTEX;
    const bool valid = g != NO_VERTEX;
    if (!valid) g = 0u;
    // tile order: this CTA is one tile of a grid cloth when its first slot
    // (a tile's origin, never padding) is a vertex of one (block-uniform)
    bool tile = false;
    int tr0 = 0, tc0 = 0;
    const MeshDev* TM = A.meshes;
    // 128-byte aligned, kept a shared-memory pointer (an offset into fused_dyn)
    float4* xs = reinterpret_cast<float4*>(fused_dyn + ((128u - (smem_u32(fused_dyn) & 127u)) & 127u));
    if (A.tiles) {
        const u32 g0 = A.vorder[A.tbase + blockIdx.x * blockDim.x];
        if (g0 != NO_VERTEX) {
            TM = A.meshes + A.vobj[g0];
            if ((TM->flags & MF_GRID) && (TM->flags & MF_CLOTH) && TM->tmap != NO_PAIR) {
                const u32 N = TM->grid_n, l0 = g0 - TM->voff;
                tile = true;
                tr0 = (int)(l0 / N);
                tc0 = (int)(l0 % N);
                if (threadIdx.x == 0)
                    tile_load(xs, A.tmaps + TM->tmap + A.xbuf, A.tmaps + TM->tmap + 3 + A.vbuf, tr0, tc0, &tile_bar);
            }
        }
    }
    const u32 m = valid ? A.vobj[g] : 0u;
    const MeshDev* __restrict__ Mp = A.meshes + m;
    const u32 mflags = Mp->flags;
    const f3 xc = valid ? ld(A.x, g) : mk(0.f, 0.f, 0.f);
    const bool query = valid && (mflags & MF_QUERY) && (mflags & MF_TREE);
    const f3 xpv = query ? ld(A.xp, g) : xc;
    const float mg = A.margin;
    u32 st = 0, rows = 0;
    // own faces of this vertex: never a self row, dropped before the queue
    const uint2 ownw = (query && A.own) ? A.own[g] : make_uint2(0u, 0u);
    auto own_face = [&](u32 f) -> bool {
        const u32 da = f - ownw.x, db = da - (ownw.y >> 16);
        return (da < 8u && ((ownw.y >> da) & 1u)) || (db < 8u && ((ownw.y >> (8u + db)) & 1u));
    };

    // ---- descent state: the own tree first (set up here), then the targets
    int stack[STACK_DEPTH];
    int sp = 0;
    auto push = [&](int v) -> bool {
        if (sp >= STACK_DEPTH) return false;
        stack[sp++] = v;
        return true;
    };
    auto pop = [&]() -> int { return stack[--sp]; };
    u32 visited = 0, nn = 0, key = 0;
    const Node* nodes = A.nodes;  // binary form
    const Wide4* wn = A.w4;       // wide form
    f3 qmn = xc, qmx = xc;
    float inv = 0.f;
    // start a descent of mesh t's tree unless the query misses its root box
    auto start = [&](u32 t, u32 k) {
        const MeshDev* T = A.meshes + t;
        key = k;
        visited = 0;
        if (WIDE) {
            const float4* r = reinterpret_cast<const float4*>(A.nodes + T->node_off);
            if (!overlap(qmn, qmx, __ldg(r), __ldg(r + 1))) return;
            wn = A.w4 + T->w4_off;
            nn = T->w4_cap;
        } else {
            nodes = A.nodes + T->node_off;
            nn = 2 * T->nF - 1;
        }
        sp = 0;
        push(0);
    };
    if (query && Mp->nF) {
        bool selfOK = false;
        if (A.self_mode == YS_SELF_HASH && (mflags & MF_CLOTH) && (mflags & MF_SELF)) {
            float mx = __uint_as_float(A.maxext[m]);
            float cs = (mx > 1e-5f) ? mx : 1e-5f;
            inv = 1.f / cs;
            H1Vertex h;
            if (h1_vertex(xc, xpv, inv, h)) { selfOK = true; h1_query_box(h, mg, qmn, qmx); }
        } else if (A.self_mode == YS_SELF_BVH && !(mflags & MF_ANALYTIC)) {
            selfOK = true;
            qmn = xc - mk(mg, mg, mg);
            qmx = xc + mk(mg, mg, mg);
        }
        if (selfOK) start(m, (m << 6) | KEY_SELF | lane);
    }
    VContact buf[MAXC];
    int nc = 0;
    const u32 te = query ? Mp->tgt_end : 0u;
    u32 tk = query ? Mp->tgt_begin : 0u;  // next target
    auto next_tree = [&]() -> bool {
        while (tk < te) {
            const u32 k = tk++;
            const u32 t = A.targets[k];
            if (ANA && (A.meshes[t].flags & MF_ANALYTIC)) {
                // narrowAnalytic for a marked (cloth, collider) pair: this
                // vertex against the shape, no descent
                const u32 p = A.tpair[k];
                if (p == NO_PAIR) continue;
                const DShape* S = A.shapes + A.meshes[t].shape;
                VContact c;
                if (analytic_live(A, *S, A.nodes + Mp->node_off, p, g == Mp->voff) &&
                    analytic_contact(S, xc, xpv, A.radius, mg, &c))
                    insert_contact(buf, nc, st, c);
                continue;
            }
            if (ANA && (mflags & MF_ANALYTIC)) continue;  // no queries from an analytic collider
            const u32 tno = A.meshes[t].node_off, tnf = A.meshes[t].nF;
            if (tnf == 0 || !root_overlap(A.nodes + Mp->node_off, A.nodes + tno)) continue;
            qmn = xc - mk(mg, mg, mg);
            qmx = xc + mk(mg, mg, mg);
            start(t, (t << 6) | lane);
            if (sp) return true;
        }
        return false;
    };

    u32 qn = 0, cn = 0;  // warp-uniform fill of the queue and of the contact buffer

    auto flush = [&]() {
        __syncwarp();
        for (u32 i = 0; i < cn; ++i)
            if (Q.co[i] == lane) insert_contact(buf, nc, st, Q.cb[i]);
        __syncwarp();
        cn = 0;
    };
    // Process queue entries [base, base + cnt), cnt <= 32: lane i takes entry base + i.
    auto drain = [&](u32 base, u32 cnt) {
        __syncwarp();
        const bool has = lane < cnt;
        u32 f = 0, k = 0;
        if (has) { f = Q.qf[base + lane]; k = Q.qk[base + lane]; }
        __syncwarp();
        const int owner = (int)(k & 31u);
        const f3 oxc = mk(__shfl_sync(FULL_MASK, xc.x, owner), __shfl_sync(FULL_MASK, xc.y, owner),
                          __shfl_sync(FULL_MASK, xc.z, owner));
        const f3 oxp = mk(__shfl_sync(FULL_MASK, xpv.x, owner), __shfl_sync(FULL_MASK, xpv.y, owner),
                          __shfl_sync(FULL_MASK, xpv.z, owner));
        const u32 og = __shfl_sync(FULL_MASK, g, owner);
        const float oinv = __shfl_sync(FULL_MASK, inv, owner);
        bool hit = false;
        VContact c;
        if (has) {
            const u32 t = k >> 6;
            // the face's vertices in one 48-byte record (ids in w)
            const float4* fp = A.fpos + 3 * (size_t)(A.meshes[t].foff + f);
            const float4 q0 = __ldg(fp), q1 = __ldg(fp + 1), q2 = __ldg(fp + 2);
            const f3 P0 = mk(q0.x, q0.y, q0.z), P1 = mk(q1.x, q1.y, q1.z), P2 = mk(q2.x, q2.y, q2.z);
            bool row = true;
            if (k & KEY_SELF) {
                const u32 lid = og - A.meshes[t].voff;
                row = !(__float_as_uint(q0.w) == lid || __float_as_uint(q1.w) == lid || __float_as_uint(q2.w) == lid);
                if (row && A.self_mode == YS_SELF_HASH) {
                    // the owner passed its 64-cell check; the cell size is the
                    // extent the refit just took from these positions
                    H1Vertex h;
                    h1_vertex_box(oxc, oxp, h);
                    row = h1_face_at(P0, P1, P2, mg, oinv, h, false);
                }
            }
            if (row) {
                ++rows;
                f3 n;
                float d;
                if (narrow_one(oxc, oxp, P0, P1, P2, A.band, n, d)) {
                    hit = true;
                    c = VContact{t, f, n.x, n.y, n.z, d};
                }
            }
        }
        const unsigned hm = __ballot_sync(FULL_MASK, hit);
        if (hm) {
            if (cn + (u32)__popc(hm) > WC_CAP) flush();
            if (hit) {
                const u32 slot = cn + (u32)__popc(hm & ((1u << lane) - 1u));
                Q.cb[slot] = c;
                Q.co[slot] = (unsigned char)owner;
            }
            cn += (u32)__popc(hm);
        }
        __syncwarp();
    };
    // warp-aggregated append of this lane's leaf (face >= 0) to the queue
    auto enqueue = [&](int face) {
        const unsigned lm = __ballot_sync(FULL_MASK, face >= 0);
        if (lm) {
            if (face >= 0) {
                const u32 slot = qn + (u32)__popc(lm & ((1u << lane) - 1u));
                Q.qf[slot] = (u32)face;
                Q.qk[slot] = key;
            }
            qn += (u32)__popc(lm);
        }
    };

    bool active = sp > 0 || next_tree();
    while (true) {
        if (active && sp == 0) active = next_tree();
        if (!__ballot_sync(FULL_MASK, active)) break;
        if (WIDE) {
            int lf[4] = {-1, -1, -1, -1};
            if (active) {
                if (++visited > VISIT_CAP) {
                    st |= ST_STACK_OVF;
                    sp = 0;
                } else {
                    const int w = pop();
                    if (w >= 0 && (u32)w < nn) {
                        const bool selfTree = (key & KEY_SELF) != 0;
                        st |= wide_step_p(wn, w, qmn, qmx, push, [&](int s, u32 f) {
                            if (!(selfTree && own_face(f))) lf[s] = (int)f;
                        });
                    }
                }
            }
#pragma unroll
            for (int s = 0; s < 4; ++s) enqueue(lf[s]);
        } else {
            int leaf = -1;
            if (active) {
                if (++visited > VISIT_CAP) {
                    st |= ST_STACK_OVF;
                    sp = 0;
                } else {
                    const int id = pop();
                    if (id >= 0 && (u32)id < nn) {
                        const float4* p = reinterpret_cast<const float4*>(nodes + id);
                        const float4 n0 = __ldg(p), n1 = __ldg(p + 1);
                        if (overlap(qmn, qmx, n0, n1)) {
                            const int a = __float_as_int(n0.w), b = __float_as_int(n1.w);
                            if (a < 0) {
                                if (!((key & KEY_SELF) && own_face((u32)b))) leaf = b;
                            } else if (sp + 2 > STACK_DEPTH) {
                                st |= ST_STACK_OVF;
                            } else {
                                push(a);
                                push(b);
                            }
                        }
                    }
                }
            }
            enqueue(leaf);
        }
        while (qn >= 32) {
            drain(qn - 32, 32);
            qn -= 32;
        }
    }
    if (qn) drain(0, qn);
    if (cn) flush();

    // The tile's springs, once every warp is done with its queue (the table
    // takes the queues' memory); the TMA loads ran during the descents.
    float* sf = reinterpret_cast<float*>(wq);
    if (tile) {
        __syncthreads();  // also orders the barrier's initialisation before the waits
        if (!tile_wait(&tile_bar)) st |= ST_ITER_CAP;
        tile_springs(A, *TM, tr0, tc0, xs, xs + HALO_W * HALO_H, sf,
                     reinterpret_cast<unsigned char*>(xs + 2 * HALO_W * HALO_H));
        __syncthreads();
    }
    if (valid && (mflags & MF_CLOTH)) {
        f3 vel = ld(A.v, g);
        const float mass = A.mass[g], mask = A.mask[g];
        f3 force;
        // by the tile layout every vertex of a tile CTA is in its tile; the
        // test keeps any other vertex on the per-vertex stencil
        const u32 N = TM->grid_n, lid = g - TM->voff;
        const bool in = tile && Mp == TM;
        const int row = in ? (int)(lid / N) : 0, col = in ? (int)(lid % N) : 0;
        if (in && row >= tr0 && row < tr0 + TILE_H && col >= tc0 && col < tc0 + TILE_W)
            force = tile_force(base_force(A, g, vel, mass), (int)N, row, col, row - tr0, col - tc0, sf,
                               reinterpret_cast<const unsigned char*>(xs + 2 * HALO_W * HALO_H));
        else
            force = vertex_force(A, *Mp, g, xc, vel, mass);
        f3 pos = xc;
        vel = vel + ((force * A.subh) / mass) * mask;
        contact_response(pos, vel, nc, Mp->thickness, [&](int i) { return buf[i]; });
        pos = pos + (vel * A.subh) * mask;
        if (sanitize(pos, vel, xc)) st |= ST_NONFINITE;
        A.xn[g] = make_float4(pos.x, pos.y, pos.z, 0.f);
        A.vn[g] = make_float4(vel.x, vel.y, vel.z, 0.f);
    } else if (valid && !(mflags & MF_STATIC)) {
        // not integrated (Rigid / Float / Kinematic): carry the state over
        A.xn[g] = A.x[g];
        A.vn[g] = A.v[g];
    }
    if (A.record) {
        // pool slots: one atomic per warp (every lane of the block reaches
        // this point), the lanes' runs in lane order after the warp's base
        const u32 mine = valid ? (u32)nc : 0u;
        u32 incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 y = __shfl_up_sync(FULL_MASK, incl, o);
            if ((int)lane >= o) incl += y;
        }
        const u32 total = __shfl_sync(FULL_MASK, incl, 31);
        u32 wbase = 0;
        if (lane == 31 && total) wbase = (u32)atomicAdd(&A.counters[2], (unsigned long long)total);
        wbase = __shfl_sync(FULL_MASK, wbase, 31);
        const u32 base = wbase + (incl - mine);
        if (!valid) {
        } else if (base + (u32)nc > A.cap) {
            st |= ST_PAIR_OVF;
            A.vstart[g] = 0;
            A.vcount[g] = 0;
        } else {
            for (int i = 0; i < nc; ++i) A.pool[base + i] = buf[i];
            A.vstart[g] = base;
            A.vcount[g] = (u32)nc;
        }
    }
    // rows and contacts: one atomic per block and counter (every thread of
    // the block gets here)
    {
        __shared__ u32 sh_cnt[2][FUSED_WARPS];
        const u32 r = __reduce_add_sync(FULL_MASK, rows), c = __reduce_add_sync(FULL_MASK, (u32)nc);
        if (lane == 0) { sh_cnt[0][threadIdx.x >> 5] = r; sh_cnt[1][threadIdx.x >> 5] = c; }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned long long R = 0, Cn = 0;
            for (int w = 0; w < FUSED_WARPS; ++w) { R += sh_cnt[0][w]; Cn += sh_cnt[1][w]; }
            if (R) { atomicAdd(&A.counters[0], R); atomicAdd(&A.counters[3], R); }
            if (Cn) { atomicAdd(&A.counters[1], Cn); atomicAdd(&A.counters[4], Cn); }
        }
    }
    if (st) atomicOr(A.status, st);
}

static constexpr int FUSED_VARIANTS[3] = {8, 7, 4};  // register caps, as CTAs per SM
// Size classes of the working meshes: at most 64^2, 128^2, 256^2 vertices, larger.
static constexpr int NCLASS = 4;
enum : int { ORDER_VERTEX = 0, ORDER_MORTON = 1, ORDER_TILE = 2 };  // a class's thread order
static constexpr u32 CLASS_MAX[NCLASS] = {4096u, 16384u, 65536u, 0xFFFFFFFFu};

template <bool ANA>
void launch_fused_t(const StepArgs& A, dim3 g, dim3 b, cudaStream_t st, int minBlocks, size_t smem) {
    switch ((A.wide ? 0 : 10) + minBlocks) {
        case 8: k_fused<true, 8, ANA><<<g, b, smem, st>>>(A); break;
        case 7: k_fused<true, 7, ANA><<<g, b, smem, st>>>(A); break;
        case 4: k_fused<true, 4, ANA><<<g, b, smem, st>>>(A); break;
        case 18: k_fused<false, 8, ANA><<<g, b, smem, st>>>(A); break;
        case 17: k_fused<false, 7, ANA><<<g, b, smem, st>>>(A); break;
        default: k_fused<false, 4, ANA><<<g, b, smem, st>>>(A); break;
    }
}

void launch_fused(const StepArgs& A, cudaStream_t st, int minBlocks) {
    if (A.tend <= A.tbase) return;
    const dim3 g(ceil_div(A.tend - A.tbase, 128)), b(128);
    const size_t smem = A.tiles ? TILE_SMEM : 0;
    if (A.analytic) launch_fused_t<true>(A, g, b, st, minBlocks, smem);
    else launch_fused_t<false>(A, g, b, st, minBlocks, smem);
}

// ------------------------------------------------------------------ staged
// queryPoints append (bvh.metal:1372-1381) / CPU-hash row append.
__global__ void __launch_bounds__(128) k_detect_rows(StepArgs A) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= A.nV) return;
    const u32 m = A.vobj[g];
    const MeshDev M = A.meshes[m];
    if (!(M.flags & MF_QUERY)) return;
    const f3 xc = ld(A.x, g), xpv = ld(A.xp, g);
    const u32 lid = g - M.voff;
    u32 st = query_vertex(A, g, m, M, xc, xpv, [&](u32 t, u32 f, uint4, u32) {
        unsigned long long idx = atomicAdd(&A.counters[0], 1ull);
        if (idx >= A.cap) { atomicOr(A.status, ST_PAIR_OVF); return; }
        A.rows[idx] = Row{lid, f, m, t, M.behavior, A.meshes[t].behavior, 0u, 0u};
    });
    if (st) atomicOr(A.status, st);
}

// narrow_pt_tri over the broad rows (bruteforce.metal:41-178).
__global__ void __launch_bounds__(128) k_narrow_rows(StepArgs A, u32 nrows) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    const Row r = A.rows[i];
    const MeshDev& T = A.meshes[r.tobj];
    const uint4 tri = A.F[T.foff + r.tri];
    if (r.qobj == r.tobj) {
        u32 gp = r.point + T.voff;
        for (u32 k = A.vaf_off[gp]; k < A.vaf_off[gp + 1]; ++k)
            if (A.vaf[k] == r.tri) return;
    }
    const u32 qo = A.meshes[r.qobj].voff, to = T.voff;
    f3 n;
    float d;
    if (!narrow_one(ld(A.x, r.point + qo), ld(A.xp, r.point + qo), ld(A.x, to + tri.x), ld(A.x, to + tri.y),
                    ld(A.x, to + tri.z), A.band, n, d))
        return;
    unsigned long long o = atomicAdd(&A.counters[1], 1ull);
    if (o >= A.cap) { atomicOr(A.status, ST_PAIR_OVF); return; }
    Contact c;
    c.point = r.point; c.tri = r.tri; c.qobj = r.qobj; c.tobj = r.tobj;
    c.nx = n.x; c.ny = n.y; c.nz = n.z; c.d = d;
    c.qbeh = r.qbeh; c.tbeh = r.tbeh; c.qshape = r.qshape; c.tshape = r.tshape;
    A.contacts[o] = c;
}

// narrow_pt_analytic over every vertex of every live (cloth, collider) marker
// pair (BruteForce::narrowAnalytic, bruteforce.hpp:245-309), appended to the
// contacts after the triangle rows: (vertex, 0), (cloth, collider).
__global__ void __launch_bounds__(128) k_narrow_analytic_scene(StepArgs A) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.apair_total) return;
    u32 lo = 0, hi = A.npairs;  // the pair whose thread range holds i
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) >> 1;
        if (A.apairs[mid].w <= i) lo = mid;
        else hi = mid;
    }
    const uint4 P = A.apairs[lo];
    const MeshDev& Q = A.meshes[P.x];
    const u32 id = i - P.w, g = Q.voff + id;
    const DShape& S = A.shapes[P.z];
    if (!analytic_live(A, S, A.nodes + Q.node_off, lo, id == 0)) return;
    f3 n;
    float d;
    if (!analytic_narrow(S.s, ld(A.x, g), ld(A.xp, g), A.radius, A.margin, S.rot_margin, n, d)) return;
    unsigned long long o = atomicAdd(&A.counters[1], 1ull);
    if (o >= A.cap) { atomicOr(A.status, ST_PAIR_OVF); return; }
    Contact c;
    c.point = id; c.tri = 0u; c.qobj = P.x; c.tobj = P.y;
    c.nx = n.x; c.ny = n.y; c.nz = n.z; c.d = d;
    c.qbeh = Q.behavior; c.tbeh = S.s.beh; c.qshape = COL_MESH; c.tshape = S.s.kind;
    A.contacts[o] = c;
}

// Per-vertex CSR of the contacts (narrow_bucket_count/scan/scatter,
// physics.metal:566-616), then canonical (tobj, tri) order per vertex.
__global__ void k_bucket_count(StepArgs A, u32 nc) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    const Contact& c = A.contacts[i];
    atomicAdd(&A.bucket[A.meshes[c.qobj].voff + c.point], 1u);
}
__global__ void k_bucket_scatter(StepArgs A, u32 nc) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nc) return;
    const Contact c = A.contacts[i];
    const u32 g = A.meshes[c.qobj].voff + c.point;
    const u32 slot = A.csr_off[g] + atomicAdd(&A.bucket[g], 1u);
    A.csr[slot] = VContact{c.tobj, c.tri, c.nx, c.ny, c.nz, c.d};
}
__global__ void k_bucket_sort(StepArgs A) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= A.nV) return;
    const u32 b = A.csr_off[g], e = A.csr_off[g + 1];
    for (u32 i = b + 1; i < e; ++i) {
        VContact c = A.csr[i];
        u32 j = i;
        while (j > b && key_less(c.tobj, c.tri, A.csr[j - 1].tobj, A.csr[j - 1].tri)) { A.csr[j] = A.csr[j - 1]; --j; }
        A.csr[j] = c;
    }
}
// Pass 1 of SymplecticSystem::update: forces of every cloth vertex.
__global__ void __launch_bounds__(128) k_forces(StepArgs A) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= A.nV) return;
    const MeshDev M = A.meshes[A.vobj[g]];
    if (!(M.flags & MF_CLOTH)) return;
    f3 f = vertex_force(A, M, g, ld(A.x, g), ld(A.v, g), A.mass[g]);
    A.f[g] = make_float4(f.x, f.y, f.z, 0.f);
}
// Pass 2: integrate_cloth / integrate_cloth_grid (physics.metal:226-312, 380-466).
__global__ void __launch_bounds__(128) k_integrate(StepArgs A) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= A.nV) return;
    const MeshDev M = A.meshes[A.vobj[g]];
    if (!(M.flags & MF_CLOTH)) {
        if (!(M.flags & MF_STATIC)) { A.xn[g] = A.x[g]; A.vn[g] = A.v[g]; }
        return;
    }
    const f3 xc = ld(A.x, g);
    f3 vel = ld(A.v, g), pos = xc;
    const f3 force = ld(A.f, g);
    const float mass = A.mass[g], mask = A.mask[g];
    vel = vel + ((force * A.subh) / mass) * mask;
    const u32 b = A.csr_off[g];
    contact_response(pos, vel, (int)(A.csr_off[g + 1] - b), M.thickness, [&](int i) { return A.csr[b + i]; });
    pos = pos + (vel * A.subh) * mask;
    if (sanitize(pos, vel, xc)) atomicOr(A.status, ST_NONFINITE);
    A.xn[g] = make_float4(pos.x, pos.y, pos.z, 0.f);
    A.vn[g] = make_float4(vel.x, vel.y, vel.z, 0.f);
}

__global__ void k_pack4(const float* __restrict__ in, float4* __restrict__ out, u32 n) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_float4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0.f);
}
__global__ void k_unpack4(const float4* __restrict__ in, float* __restrict__ out, u32 n) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { float4 q = in[i]; out[3 * i] = q.x; out[3 * i + 1] = q.y; out[3 * i + 2] = q.z; }
}

// Sorted-leaf ranges of the wide nodes before a height pass: empty.
__global__ void k_range_init(uint2* __restrict__ r, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = make_uint2(0xFFFFFFFFu, 0u);
}

// Face positions of one mesh (the layout of RefitJob::fpos) from x.
__global__ void k_face_pos(const float4* __restrict__ x, u32 voff, const u32* __restrict__ F3, u32 n,
                           float4* __restrict__ fpos) {
    const u32 f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= n) return;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const u32 v = F3[3 * f + k];
        const float4 p = x[voff + v];
        fpos[3 * (size_t)f + k] = make_float4(p.x, p.y, p.z, __uint_as_float(v));
    }
}

// ------------------------------------------------------------------ thread order
// The fused kernel's threads take the scene's working vertices in Morton
// order within each mesh, so the 32 vertices of a warp are a compact patch of
// the mesh (an 8 x 4 tile of a grid cloth instead of 32 vertices of one row):
// their tree descents share nodes and their candidate faces, which the L1
// then serves.  Results do not depend on the order.  Mesh boxes first (one
// atomic per warp and mesh), then keys (active-mesh rank in the high bits,
// the Morton code of the vertex in its mesh box, all axes scaled by the
// largest extent, below), then a radix sort of (key, vertex).
__global__ void k_order_box(const float4* __restrict__ x, const u32* __restrict__ vobj,
                            const u32* __restrict__ aoff, u32 nV, u32* __restrict__ mbox) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nV) return;
    const u32 m = vobj[g];
    if (aoff[m] == NO_PAIR) return;
    const f3 p = ld(x, g);
    const unsigned act = __activemask();
    const unsigned peers = __match_any_sync(act, m);
    const u32 v[6] = {ford(p.x), ford(p.y), ford(p.z), ford(p.x), ford(p.y), ford(p.z)};
    u32 r[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r[k] = __reduce_min_sync(peers, v[k]);
        r[3 + k] = __reduce_max_sync(peers, v[3 + k]);
    }
    if ((threadIdx.x & 31) == (unsigned)(__ffs(peers) - 1)) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicMin(&mbox[6 * m + k], r[k]);
            atomicMax(&mbox[6 * m + 3 + k], r[3 + k]);
        }
    }
}

__global__ void k_order_keys(const float4* __restrict__ x, const u32* __restrict__ vobj,
                             const u32* __restrict__ aoff, const u32* __restrict__ arank,
                             const u32* __restrict__ morton, const MeshDev* __restrict__ meshes,
                             const u32* __restrict__ mbox, u32 nV, u32 kbits, u32* __restrict__ keys,
                             u32* __restrict__ vals) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nV) return;
    const u32 m = vobj[g];
    if (aoff[m] == NO_PAIR) return;
    const u32 rank = arank[m];
    const u32 local = g - meshes[m].voff;
    if (morton[m] == 2u) {
        // tile order: a grid cloth's vertex goes to its slot in its 16 x 8
        // tile (tiles row-major, 16 vertices per tile row); any other mesh
        // keeps vertex order
        u32 i = aoff[m] + local;
        if (meshes[m].flags & MF_GRID) {
            const u32 n = meshes[m].grid_n, r = local / n, c = local % n;
            const u32 ntx = (n + TILE_W - 1) / TILE_W;
            i = aoff[m] + ((r / TILE_H) * ntx + c / TILE_W) * (TILE_W * TILE_H) + (r % TILE_H) * TILE_W + c % TILE_W;
        }
        vals[i] = g;
        return;
    }
    const u32 i = aoff[m] + local;
    vals[i] = g;
    if (!morton[m]) {
        // vertex order: the vertex's index in its mesh (clamped: the sort is
        // stable, so equal keys keep vertex order)
        const u32 cap = kbits >= 32 ? 0xFFFFFFFFu : (1u << kbits) - 1u;
        keys[i] = (kbits >= 32 ? 0u : (rank << kbits)) | min(local, cap);
        return;
    }
    const f3 p = ld(x, g);
    const float lo[3] = {funord(mbox[6 * m]), funord(mbox[6 * m + 1]), funord(mbox[6 * m + 2])};
    const float c[3] = {p.x, p.y, p.z};
    float w = 0.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) w = fmaxf(w, funord(mbox[6 * m + 3 + a]) - lo[a]);
    u32 q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float t = w > 0.f ? (c[a] - lo[a]) / w : 0.f;
        const int v = (int)(t * 1024.f);  // NaN converts to 0
        q[a] = (u32)min(max(v, 0), 1023);
    }
    u32 code = (expand_bits(q[0]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[2]);  // 30 bits
    if (kbits < 30) code >>= (30 - kbits);
    keys[i] = (kbits >= 32 ? 0u : (rank << kbits)) | code;
}

// ------------------------------------------------------------------ host
struct HostMesh {
    ys_mesh_desc d;
    std::vector<float> x, v, mass, mask;
    std::vector<u32> F;
    u32 voff = 0, foff = 0, node_off = 0, flags = 0;
    u32 w4_off = 0, w4_cap = 0;
    bool built = false;
    // the tree is descended by some query (a target of a query mesh, or
    // self-queried), or is a static query mesh's (root box for the cull)
    bool needs_tree = true;
    // TriangularCloth springs (mesh-local ids)
    std::vector<u32> spr_off, spr_split, spr_nbr, vaf_off, vaf;
    std::vector<float> spr_rest;
    bool grid_springs_on = false;  // per-spring parameters set (ys_scene_set_grid_springs)
    // analytic collider (GeneralMesh::colliderKind) and its pose: centre,
    // local half extents, orientation (w, x, y, z)
    u32 collider = COL_MESH;
    float pose[10] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f};
};

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count) {
        if (p) { cudaFree(p); p = nullptr; }
        n = count;
        if (count == 0) return cudaSuccess;
        return cudaMalloc((void**)&p, count * sizeof(T));
    }
    void free() { if (p) cudaFree(p); p = nullptr; n = 0; }
};

// MeshAdjacencyInitializer::initialize (mesh_state.hpp:236-411) restricted to
// what the path consumes: vertexAdjFacets CSR, unique edges with rest
// lengths, vertexAdjEdges and vertexOppVertices with rest lengths; merged
// into one per-vertex spring list (stretch entries, then bend entries).
static void build_adjacency(HostMesh& H) {
    const u32 nV = H.d.num_vertices, nF = H.d.num_facets;
    const u32* F = H.F.data();
    const float* x = H.x.data();
    H.vaf_off.assign(nV + 1, 0);
    for (u32 f = 0; f < nF; ++f) for (int k = 0; k < 3; ++k) H.vaf_off[F[3 * f + k] + 1]++;
    for (u32 v = 0; v < nV; ++v) H.vaf_off[v + 1] += H.vaf_off[v];
    H.vaf.assign(H.vaf_off[nV], 0);
    {
        std::vector<u32> o(nV, 0);
        for (u32 f = 0; f < nF; ++f)
            for (int k = 0; k < 3; ++k) { u32 v = F[3 * f + k]; H.vaf[H.vaf_off[v] + o[v]++] = f; }
    }
    struct E { u32 v0, v1; i32 o0, o1; };
    std::vector<E> tmp;
    tmp.reserve(3 * (size_t)nF);
    for (u32 f = 0; f < nF; ++f) {
        u32 a = F[3 * f], b = F[3 * f + 1], c = F[3 * f + 2];
        u32 tri[3][3] = {{a, b, c}, {b, c, a}, {c, a, b}};
        for (auto& t : tri) {
            u32 p = t[0], q = t[1];
            if (p > q) std::swap(p, q);
            tmp.push_back(E{p, q, (i32)t[2], -1});
        }
    }
    std::stable_sort(tmp.begin(), tmp.end(), [](const E& p, const E& q) { return p.v0 < q.v0 || (p.v0 == q.v0 && p.v1 < q.v1); });
    std::vector<E> edges;
    for (const E& e : tmp) {
        if (edges.empty() || edges.back().v0 != e.v0 || edges.back().v1 != e.v1) edges.push_back(e);
        else edges.back().o1 = e.o0;
    }
    auto len = [&](u32 a, u32 b) {
        float dx = x[3 * b] - x[3 * a], dy = x[3 * b + 1] - x[3 * a + 1], dz = x[3 * b + 2] - x[3 * a + 2];
        return sqrtf(dx * dx + dy * dy + dz * dz);
    };
    std::vector<u32> ne(nV, 0), no(nV, 0);
    for (const E& e : edges) {
        ne[e.v0]++; ne[e.v1]++;
        if (e.o1 != -1) { no[(u32)e.o0]++; no[(u32)e.o1]++; }
    }
    H.spr_off.assign(nV + 1, 0);
    H.spr_split.assign(nV, 0);
    for (u32 v = 0; v < nV; ++v) H.spr_off[v + 1] = H.spr_off[v] + ne[v] + no[v];
    for (u32 v = 0; v < nV; ++v) H.spr_split[v] = H.spr_off[v] + ne[v];
    H.spr_nbr.assign(H.spr_off[nV], 0);
    H.spr_rest.assign(H.spr_off[nV], 0.f);
    std::vector<u32> fe(nV, 0), fo(nV, 0);
    for (const E& e : edges) {
        // vertexOppVertices entries (bend), in edge order
        if (e.o1 != -1) {
            u32 o0 = (u32)e.o0, o1 = (u32)e.o1;
            float r = len(o0, o1);
            u32 s0 = H.spr_split[o0] + fo[o0]++, s1 = H.spr_split[o1] + fo[o1]++;
            H.spr_nbr[s0] = o1; H.spr_rest[s0] = r;
            H.spr_nbr[s1] = o0; H.spr_rest[s1] = r;
        }
        // vertexAdjEdges entries (stretch), in edge order
        float r = len(e.v0, e.v1);
        u32 a = H.spr_off[e.v0] + fe[e.v0]++, b = H.spr_off[e.v1] + fe[e.v1]++;
        H.spr_nbr[a] = e.v1; H.spr_rest[a] = r;
        H.spr_nbr[b] = e.v0; H.spr_rest[b] = r;
    }
}

}  // namespace ys

using namespace ys;

struct ys_scene {
    int device = 0;
    cudaStream_t stream = nullptr;
    ys_sim_params P{};
    std::vector<HostMesh> meshes;
    bool packed = false;
    u32 nV = 0, nF = 0, nNodes = 0;
    // device state
    DBuf<float4> X[3], V[2], Fbuf;
    int cur = 0, prev = 1, cv = 0;
    bool snapshot_pending = false;
    DBuf<float> mass, mask;
    DBuf<u32> vobj, targets, spr_off, spr_split, spr_nbr, vaf_off, vaf, maxext, status, codes, idx, visits, box;
    DBuf<float> spr_rest, scratch3;
    DBuf<uint4> F4;
    DBuf<u32> F3;  // packed facets (3 per face) for the refit kernel
    DBuf<float4> fpos;  // per face: its three vertex positions (id in w), for the fused kernel's tests
    DBuf<uint4> lvid;   // per sorted leaf: its face's vertex ids and the face id (range refit)
    DBuf<uint2> own;    // per vertex: its own faces as two 8-face windows (StepArgs::own)
    DBuf<Node> nodes;
    DBuf<i32> parent, claims;        // largest claimant per node; claimant lists (offset node_off)
    DBuf<u32> claimOff;              // per mesh 2N entries at node_off + mesh index
    DBuf<u32> rootAcc;               // 32 per refit job (root-only jobs' leaf-box union, one line each)
    u32 nRootOnly = 0;
    // root-only jobs of meshes whose every vertex is on a face: root box by a
    // chunked vertex reduction (6 tables (cur x cv) of nrjobs, like jobs)
    DBuf<RefitJob> rjobs;
    DBuf<uint2> rchunks;
    u32 nrjobs = 0, nrchunks = 0;
    DBuf<char> karrasScratch;
    DBuf<Wide4> w4;                  // cube layout: 4-wide trees used by every query and refit
    DBuf<int2> leafW, leafWf;        // per leaf / per face: (wide node, slot)
    DBuf<u32> warrive, wcount, hacc; // arrivals, wide nodes per mesh, heights
    DBuf<char> wideScratch;
    // level-synchronous refit of the wide trees: nodes listed by height
    DBuf<uint2> wlist;
    DBuf<u32> hcount, hoff, hcursor;
    std::vector<u32> lvl_off;        // host copy of hoff (MAX_LEVELS + 2)
    u32 lvl_top = 0;
    bool use_levels = false;
    // range refit (RefitJob::ranges): block boxes of 16 / 256 sorted leaves,
    // per wide node its sorted-leaf range
    bool use_ranges = true;
    DBuf<Node> bb16, bb256;
    DBuf<uint2> wrange;
    DBuf<uint4> blkEnt, bigEnt;      // wide-node records: inside one 256-leaf block / spanning several
    DBuf<u32> blkCnt, blkOff, bigCnt;
    DBuf<char> rangeScratch;
    u32 nbig = 0, nhuge = 0;
    DBuf<MeshDev> dmeshes;
    DBuf<RefitJob> jobs;            // 6 tables (cur x cv) of njobs, then one build slot
    std::vector<RefitJob> hjobs;
    u32 njobs = 0;
    u32 refitLeaves = 0;
    DBuf<unsigned long long> counters;
    DBuf<float4> ext;
    bool use_ext = false;
    DBuf<float> gk, gL;              // per-spring grid-cloth parameters
    // analytic colliders: compact shape table (mesh of each slot), marker
    // pairs, per-target pair ids, marker flags of two detects (2 x np, by
    // substep parity)
    std::vector<int> shape_mesh;
    std::vector<DShape> hshapes;
    bool analytic_primed = false, shapes_uploaded = false;
    DBuf<DShape> dshapes;
    DBuf<uint4> apairs;
    DBuf<u32> tpair, markers;
    u32 npairs = 0, apair_total = 0;
    std::vector<MeshDev> hmeshes;    // host copy of the device mesh table
    // per-kernel CUDA-event timing of the fused path
    bool timing = false;
    std::vector<cudaEvent_t> evPool;
    size_t evUsed = 0;
    std::vector<size_t> evRefit, evFused;  // indices of (begin, end) event pairs
    // one executable graph per buffer-rotation state (cur, prev, cv): the
    // refit + fused substep replayed without host launch overhead
    bool use_graphs = true;
    cudaGraphExec_t graphs[18] = {};
    int fused_min_blocks = 8;        // k_fused register cap (ys_scene_set_fused_variant / ys_scene_autotune)
    // fused-kernel thread order (ys_scene_set_thread_order): working vertices
    // in Morton order per mesh, recomputed at every tree rebuild
    u32 nact = 0, order_kbits = 0;   // working vertices; key bits below the mesh rank
    DBuf<u32> vorder, okeys, oaoff, orank, obox, omorton;
    // size classes of the working meshes (by vertex count, bounds CLASS_MAX):
    // each class is one k_fused launch over its contiguous part of vorder,
    // with its own register-cap variant and thread order
    std::vector<u32> cls_off;        // NCLASS + 1 offsets into vorder
    std::vector<u32> cls_meshes;     // working meshes per class
    std::vector<int> cls_variant;    // CTAs per SM of each class's launch
    std::vector<int> cls_order;      // per class: ORDER_VERTEX, ORDER_MORTON or ORDER_TILE
    std::vector<u32> act_aoff;       // per mesh: first slot in vorder, or NO_PAIR (not working)
    DBuf<CUtensorMap> tmaps;         // 5 per grid cloth: X[0..2], V[0..1] (tile order)
    std::vector<int> mesh_class;     // per mesh, or -1 (not working)
    DBuf<char> oscratch;
    int tree_layout = YS_TREE_CUBE;  // Morton normalisation of the scene trees
    int tree_builder = YS_BUILD_KARRAS;
    DBuf<char> aggScratch;           // Apetrei range ends and root slot
    DBuf<char> sortScratch, scanScratch;
    // staged / record buffers
    u32 cap = 0;
    DBuf<Row> rows;
    DBuf<Contact> contacts;
    DBuf<VContact> csr, pool;
    DBuf<u32> bucket, csr_off, vstart, vcount;
    bool staged_ready = false, record = false, record_ready = false;
    int last_contacts = 0;  // 0 none, 1 staged csr, 2 fused pool
    // progress
    uint64_t frame = 0, substeps_run = 0;
    u32 cursor = 0;
    uint64_t last_rows = 0, last_contacts_n = 0;
};

namespace {

ys_status check_scene(ys_scene* s) {
    if (!s) return fail(YS_ERR_BAD_ARG, "null scene");
    if (!s->packed) return fail(YS_ERR_STATE, "scene not packed");
    return YS_OK;
}

StepArgs make_args(ys_scene* s) {
    StepArgs A;
    memset(&A, 0, sizeof(A));
    const int nxt = 3 - s->cur - s->prev;
    A.x = s->X[s->cur].p;
    A.xp = s->X[s->prev].p;
    A.xn = s->X[nxt].p;
    A.v = s->V[s->cv].p;
    A.vn = s->V[1 - s->cv].p;
    A.mass = s->mass.p;
    A.mask = s->mask.p;
    A.vobj = s->vobj.p;
    A.meshes = s->dmeshes.p;
    A.targets = s->targets.p;
    A.F = s->F4.p;
    A.fpos = s->fpos.p;
    A.own = s->own.p;
    A.nodes = s->nodes.p;
    A.w4 = s->w4.p;
    A.wide = s->tree_layout == YS_TREE_CUBE ? 1u : 0u;
    A.spr_off = s->spr_off.p;
    A.spr_split = s->spr_split.p;
    A.spr_nbr = s->spr_nbr.p;
    A.spr_rest = s->spr_rest.p;
    A.vaf_off = s->vaf_off.p;
    A.vaf = s->vaf.p;
    A.maxext = s->maxext.p;
    A.ext = s->use_ext ? s->ext.p : nullptr;
    A.gk = s->gk.p;
    A.gL = s->gL.p;
    A.shapes = s->dshapes.p;
    A.tpair = s->tpair.p;
    A.apairs = s->apairs.p;
    A.mk_fresh = s->markers.p ? s->markers.p + (size_t)s->cv * s->npairs : nullptr;
    A.mk_held = s->markers.p ? s->markers.p + (size_t)(1 - s->cv) * s->npairs : nullptr;
    A.npairs = s->npairs;
    A.apair_total = s->apair_total;
    A.analytic = s->shape_mesh.empty() ? 0u : 1u;
    A.radius = s->P.radius;
    A.subh = s->P.subh; A.kair = s->P.kair; A.kd = s->P.kd;
    A.gx = s->P.gravity[0]; A.gy = s->P.gravity[1]; A.gz = s->P.gravity[2];
    A.margin = s->P.margin;
    A.band = s->P.radius + s->P.margin;
    A.nV = s->nV;
    A.vorder = s->vorder.p;
    A.tmaps = s->tmaps.p;
    A.xbuf = (u32)s->cur;
    A.vbuf = (u32)s->cv;
    A.tbase = 0;
    A.tend = s->nact;
    A.self_mode = s->P.self_mode;
    A.record = s->record ? 1u : 0u;
    A.cap = s->cap;
    A.status = s->status.p;
    A.counters = s->counters.p;
    A.pool = s->pool.p; A.vstart = s->vstart.p; A.vcount = s->vcount.p;
    A.rows = s->rows.p; A.contacts = s->contacts.p; A.f = s->Fbuf.p;
    A.bucket = s->bucket.p; A.csr_off = s->csr_off.p; A.csr = s->csr.p;
    return A;
}

// Rotate the position / velocity buffers after an integrate:
// prev <- cur when xPrev was snapshotted, cur <- next.
void rotate(ys_scene* s) {
    const int nxt = 3 - s->cur - s->prev;
    if (s->snapshot_pending) s->prev = s->cur;
    s->cur = nxt;
    if (s->prev == s->cur) s->prev = 3 - s->cur - nxt;  // unreachable guard
    s->cv = 1 - s->cv;
    s->snapshot_pending = false;
    s->substeps_run++;
    if (++s->cursor >= s->P.substeps) { s->cursor = 0; s->frame++; }
}

// BVH<..,LINEAR,TRIANGLE>::build for one mesh on the current positions.
// Claimant-list offsets of mesh H's tree (2N entries after its nodes' offset,
// one extra slot per earlier mesh).
u32* claim_off(ys_scene* s, const HostMesh& H) {
    return s->claimOff.p + H.node_off + (size_t)(&H - s->meshes.data());
}

ys_status build_tree(ys_scene* s, HostMesh& H) {
    const u32 n = H.d.num_facets;
    if (n == 0) return YS_OK;
    cudaStream_t st = s->stream;
    u32* codes = s->codes.p + H.foff;
    u32* idx = s->idx.p + H.foff;
    launch_box_init(s->box.p, st);
    launch_box(s->X[s->cur].p, nullptr, H.voff, H.d.num_vertices, s->box.p, st);
    launch_morton(s->X[s->cur].p, nullptr, H.voff, s->F3.p + 3 * (size_t)H.foff, n, s->box.p, codes, idx, st,
                  s->tree_layout == YS_TREE_CUBE);
    YS_CK(radix_sort_pairs(codes, idx, n, s->sortScratch.p, 0, 32, st));
    launch_leaf_vids(idx, s->F3.p + 3 * (size_t)H.foff, n, s->lvid.p + H.foff, st);  // for the range refit
    const bool cube = s->tree_layout == YS_TREE_CUBE;
    const bool agg = s->tree_builder == YS_BUILD_APETREI;
    if (agg)
        YS_CK(launch_apetrei(s->X[s->cur].p, nullptr, H.voff, s->F3.p + 3 * (size_t)H.foff, codes, idx, n,
                             s->nodes.p + H.node_off, s->parent.p + H.node_off, claim_off(s, H),
                             s->claims.p + H.node_off, s->visits.p + H.foff, s->karrasScratch.p, s->aggScratch.p,
                             s->status.p, st));
    else
        YS_CK(launch_karras(codes, idx, n, s->nodes.p + H.node_off, s->parent.p + H.node_off, claim_off(s, H),
                            s->claims.p + H.node_off, s->visits.p + H.foff, s->karrasScratch.p, st, cube));
    if (cube)
        YS_CK(launch_wide_build(s->nodes.p + H.node_off, s->parent.p + H.node_off, n, s->w4.p + H.w4_off,
                                s->leafW.p + H.foff, s->leafWf.p + H.foff, s->warrive.p + H.w4_off,
                                s->wcount.p + (&H - s->meshes.data()), s->wideScratch.p, st));
    k_face_pos<<<ceil_div(n, 256), 256, 0, st>>>(s->X[s->cur].p, H.voff, s->F3.p + 3 * (size_t)H.foff, n,
                                                  s->fpos.p + 3 * (size_t)H.foff);
    RefitJob J;
    memset(&J, 0, sizeof(J));
    J.nodes = s->nodes.p + H.node_off;
    J.parent = s->parent.p + H.node_off;
    J.claimOff = claim_off(s, H);
    J.claims = s->claims.p + H.node_off;
    J.visits = s->visits.p + H.foff;
    J.facets = s->F3.p + 3 * (size_t)H.foff;
    J.x4 = s->X[s->cur].p;
    J.voff = H.voff;
    J.n = n;
    J.leafBase = 0;
    J.swept = 0;
    J.selfMargin = 0.f;
    J.maxExt = s->maxext.p;  // unused (selfMargin == 0)
    RefitJob* slot = s->jobs.p + 6 * (size_t)s->njobs;
    if (!agg) {  // the Apetrei build wrote every box already
        YS_CK(cudaMemcpyAsync(slot, &J, sizeof(J), cudaMemcpyHostToDevice, st));
        launch_refit(slot, 1, n, s->status.p, st);
    }
    RefitJob JW = J;  // the wide boxes (and the root box) from the same positions
    if (cube) {
        JW.w4 = s->w4.p + H.w4_off;
        JW.leafW = s->leafW.p + H.foff;
        JW.warrive = s->warrive.p + H.w4_off;
        YS_CK(cudaMemcpyAsync(slot + 1, &JW, sizeof(JW), cudaMemcpyHostToDevice, st));
        launch_refit(slot + 1, 1, n, s->status.p, st);
    }
    YS_CK(cudaStreamSynchronize(st));  // J, JW live on the host stack
    H.built = true;
    return YS_OK;
}

void drop_graphs(ys_scene* s);

// Upload the 6 job tables (cur x cv) with the level-mode flag of the 4-wide jobs.
ys_status upload_jobs(ys_scene* s, bool levels) {
    for (int c = 0; c < 3; ++c)
        for (int w = 0; w < 2; ++w) {
            std::vector<RefitJob> t = s->hjobs;
            for (auto& J : t) {
                J.x4 = s->X[c].p;
                J.v4 = s->V[w].p;
                J.levels = (levels && J.w4) ? 1u : 0u;
                J.ranges = (J.levels && s->use_ranges) ? 1u : 0u;
            }
            if (!t.empty())
                YS_CK(cudaMemcpyAsync(s->jobs.p + (size_t)(c * 2 + w) * s->njobs, t.data(), t.size() * sizeof(RefitJob), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
        }
    return YS_OK;
}

// Level lists of the 4-wide trees after a build: heights, counts per height,
// the lists.  Falls back to the climb refit when a tree is taller than
// MAX_LEVELS.  Level sizes change with every build, so captured substeps
// are dropped.
ys_status build_levels(ys_scene* s) {
    if (s->tree_layout != YS_TREE_CUBE || s->njobs == 0) return YS_OK;
    bool any = false;
    for (auto& J : s->hjobs) any = any || J.w4;
    if (!any) return YS_OK;
    cudaStream_t st = s->stream;
    YS_CK(refit_levels_prepare());
    ys_status r = upload_jobs(s, true);
    if (r) return r;
    const RefitJob* table = s->jobs.p;
    YS_CK(cudaMemsetAsync(s->hacc.p, 0, 4 * s->hacc.n, st));
    if (s->wrange.p) k_range_init<<<ceil_div(s->wrange.n, 256), 256, 0, st>>>(s->wrange.p, (u32)s->wrange.n);
    launch_wide_heights(table, s->njobs, s->refitLeaves, s->status.p, st);
    if (s->use_ranges) {
        // range refit: the node records replace the level lists
        YS_CK(launch_range_lists(table, s->njobs, s->refitLeaves, s->blkCnt.p, s->blkOff.p, s->blkEnt.p,
                                 s->bigEnt.p, (u32)s->bigEnt.n, s->bigCnt.p, s->rangeScratch.p, st));
        u32 nbig[2] = {0, 0};
        YS_CK(cudaMemcpyAsync(nbig, s->bigCnt.p, 8, cudaMemcpyDeviceToHost, st));
        YS_CK(cudaStreamSynchronize(st));
        drop_graphs(s);
        s->nbig = nbig[0];
        s->nhuge = nbig[1];
        s->use_levels = true;
        return YS_OK;
    }
    YS_CK(cudaMemsetAsync(s->hcount.p, 0, 4 * (MAX_LEVELS + 2), st));
    launch_level_count(table, s->njobs, s->refitLeaves, s->hcount.p, s->status.p, st);
    std::vector<u32> cnt(MAX_LEVELS + 2);
    YS_CK(cudaMemcpyAsync(cnt.data(), s->hcount.p, 4 * cnt.size(), cudaMemcpyDeviceToHost, st));
    YS_CK(cudaStreamSynchronize(st));
    drop_graphs(s);
    if (cnt[0] != 0) {  // a tree taller than MAX_LEVELS: climb instead
        s->use_levels = false;
        return upload_jobs(s, false);
    }
    s->lvl_off.assign(MAX_LEVELS + 2, 0);
    s->lvl_top = 0;
    for (u32 h = 1; h <= MAX_LEVELS; ++h) {
        s->lvl_off[h + 1] = s->lvl_off[h] + cnt[h];
        if (cnt[h]) s->lvl_top = h;
    }
    YS_CK(cudaMemcpyAsync(s->hoff.p, s->lvl_off.data(), 4 * s->lvl_off.size(), cudaMemcpyHostToDevice, st));
    YS_CK(cudaMemsetAsync(s->hcursor.p, 0, 4 * (MAX_LEVELS + 2), st));
    launch_level_fill(table, s->njobs, s->refitLeaves, s->hoff.p, s->hcursor.p, s->wlist.p, st);
    YS_CK(cudaStreamSynchronize(st));  // the host copy of the offsets stays valid
    s->use_levels = true;
    return YS_OK;
}

// Scene::refreshAnalyticShapes (scene.hpp:659-745): the shape of each
// collider from its pose (sphere: semi-axes h, radius h.x; box: half extents
// h; cylinder: radius max(h.x, h.z), half height h.y; plane: centre and
// orientation only); after the first refresh the previous centre and
// orientation roll into the prev slots.  Each entry also carries its broad
// box (inflated by radius + margin, BVH::analyticInflate) and the narrow
// rotation margin.  The device table is rewritten only when it changed.
ys_status refresh_shapes(ys_scene* s) {
    const size_t ns = s->shape_mesh.size();
    if (ns == 0) return YS_OK;
    std::vector<DShape> t(ns);
    for (size_t k = 0; k < ns; ++k) {
        const HostMesh& H = s->meshes[s->shape_mesh[k]];
        const float *c = H.pose, *h = H.pose + 3, *q = H.pose + 6;
        AShape a;
        memset(&a, 0, sizeof(a));
        a.rq = make_float4(q[0], q[1], q[2], q[3]);
        if (s->analytic_primed) {
            const AShape& o = s->hshapes[k].s;
            a.pc = make_float4(o.cr.x, o.cr.y, o.cr.z, 0.f);
            a.prq = o.rq;
        } else {
            a.pc = make_float4(c[0], c[1], c[2], 0.f);
            a.prq = a.rq;
        }
        a.kind = H.collider;
        a.obj = (u32)s->shape_mesh[k];
        a.beh = H.d.behavior;
        a.flags = (H.d.flags & YS_MESH_COLLIDABLE) ? 1u : 0u;
        if (H.collider == COL_SPHERE) {
            a.cr = make_float4(c[0], c[1], c[2], h[0]);
            a.he = make_float4(h[0], h[1], h[2], h[1]);
        } else if (H.collider == COL_BOX) {
            a.cr = make_float4(c[0], c[1], c[2], 0.f);
            a.he = make_float4(h[0], h[1], h[2], 0.f);
        } else if (H.collider == COL_CYLINDER) {
            a.cr = make_float4(c[0], c[1], c[2], std::max(h[0], h[2]));
            a.he = make_float4(h[0], h[1], h[2], h[1]);
        } else {  // plane
            a.cr = make_float4(c[0], c[1], c[2], 0.f);
            a.he = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        DShape& D = t[k];
        memset(&D, 0, sizeof(D));
        D.s = a;
        f3 lo, hi;
        const float inflate = s->P.radius + s->P.margin;
        const bool finite = analytic_broad_box(a, inflate, lo, hi);
        D.lo = make_float4(lo.x, lo.y, lo.z, finite ? 1.f : 0.f);
        D.hi = make_float4(hi.x, hi.y, hi.z, 0.f);
        D.rot_margin = analytic_rot_margin(a, s->P.radius, s->P.margin);
    }
    s->analytic_primed = true;
    if (s->shapes_uploaded && memcmp(t.data(), s->hshapes.data(), ns * sizeof(DShape)) == 0) return YS_OK;
    s->hshapes = t;
    // pageable source: the call returns once the table is staged
    YS_CK(cudaMemcpyAsync(s->dshapes.p, s->hshapes.data(), ns * sizeof(DShape), cudaMemcpyHostToDevice, s->stream));
    s->shapes_uploaded = true;
    return YS_OK;
}

// Slots of mesh m in the thread order of its class: its vertices, or in tile
// order whole 16 x 8 tiles (a grid cloth) or whole 128-thread CTAs (any other
// mesh), so that every CTA of the class lies in one mesh.
static u32 order_slots(const ys_scene* s, size_t m, int order) {
    const u32 nv = s->meshes[m].d.num_vertices;
    if (order != ORDER_TILE) return nv;
    if (s->meshes[m].flags & MF_GRID) {
        const u32 n = s->meshes[m].d.grid_n;
        return (u32)ceil_div(n, TILE_H) * (u32)ceil_div(n, TILE_W) * (u32)(TILE_W * TILE_H);
    }
    return (u32)ceil_div(nv, 128) * 128u;
}

// Offsets of the classes and meshes in vorder for the classes' thread orders.
ys_status order_layout(ys_scene* s) {
    const size_t nm = s->meshes.size();
    std::vector<u32> aoff(nm, NO_PAIR), rank(nm, 0);
    u32 na = 0, nmesh = 0;
    s->cls_off.assign(NCLASS + 1, 0);
    for (int c = 0; c < NCLASS; ++c) {
        s->cls_off[c] = na;
        for (size_t m = 0; m < nm; ++m) {
            if (s->mesh_class[m] != c) continue;
            aoff[m] = na;
            rank[m] = nmesh++;
            na += order_slots(s, m, s->cls_order[c]);
        }
    }
    s->cls_off[NCLASS] = na;
    s->nact = na;
    s->act_aoff = aoff;
    if (s->vorder.n < std::max(na, 1u)) {
        YS_CK(s->vorder.alloc(std::max(na, 1u)));
        YS_CK(s->okeys.alloc(std::max(na, 1u)));
        YS_CK(s->oscratch.alloc(sort_scratch_bytes(std::max(na, 1u))));
    }
    YS_CK(cudaMemcpyAsync(s->oaoff.p, aoff.data(), 4 * nm, cudaMemcpyHostToDevice, s->stream));
    YS_CK(cudaMemcpyAsync(s->orank.p, rank.data(), 4 * nm, cudaMemcpyHostToDevice, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));  // aoff and rank live on the host stack
    return YS_OK;
}

// Fused-kernel thread order from the current positions (see k_order_keys):
// Morton and vertex order by one radix sort per class, tile order written in
// place (padding slots hold NO_VERTEX).
ys_status compute_order(ys_scene* s) {
    if (s->nact == 0) return YS_OK;
    cudaStream_t st = s->stream;
    const size_t nm = s->meshes.size();
    std::vector<u32> init(6 * nm);
    for (size_t m = 0; m < nm; ++m)
        for (int k = 0; k < 6; ++k) init[6 * m + k] = k < 3 ? 0xFFFFFFFFu : 0u;
    YS_CK(cudaMemcpyAsync(s->obox.p, init.data(), 4 * init.size(), cudaMemcpyHostToDevice, st));
    k_order_box<<<ceil_div(s->nV, 256), 256, 0, st>>>(s->X[s->cur].p, s->vobj.p, s->oaoff.p, s->nV, s->obox.p);
    std::vector<u32> mode(nm, (u32)ORDER_VERTEX);
    for (size_t m = 0; m < nm; ++m)
        if (s->mesh_class[m] >= 0) mode[m] = (u32)s->cls_order[s->mesh_class[m]];
    YS_CK(cudaMemcpyAsync(s->omorton.p, mode.data(), 4 * nm, cudaMemcpyHostToDevice, st));
    for (int c = 0; c < NCLASS; ++c)
        if (s->cls_order[c] == ORDER_TILE && s->cls_off[c + 1] > s->cls_off[c])
            YS_CK(cudaMemsetAsync(s->vorder.p + s->cls_off[c], 0xFF, 4 * (size_t)(s->cls_off[c + 1] - s->cls_off[c]), st));
    k_order_keys<<<ceil_div(s->nV, 256), 256, 0, st>>>(s->X[s->cur].p, s->vobj.p, s->oaoff.p, s->orank.p,
                                                       s->omorton.p, s->dmeshes.p, s->obox.p, s->nV, s->order_kbits,
                                                       s->okeys.p, s->vorder.p);
    YS_CK(cudaGetLastError());
    for (int c = 0; c < NCLASS; ++c) {
        const u32 b = s->cls_off[c], e = s->cls_off[c + 1];
        if (s->cls_order[c] == ORDER_TILE || e <= b) continue;
        YS_CK(radix_sort_pairs(s->okeys.p + b, s->vorder.p + b, e - b, s->oscratch.p, 0, 32, st));
    }
    YS_CK(cudaStreamSynchronize(st));  // init and mode live on the host stack
    return YS_OK;
}

// Tensor maps of the tile order: per grid cloth, each of X[0..2] and V[0..1]
// as a 3-D float array {4 components, N columns, N rows} with a box of
// {4, HALO_W, HALO_H}.  Without the driver's encoder the grid cloths keep no
// maps, and their tile-order CTAs gather the stencil per vertex instead.
ys_status encode_tile_maps(ys_scene* s) {
    using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    EncodeFn encode = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", (void**)&encode, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
        encode = nullptr;
    std::vector<MeshDev> md = s->hmeshes;
    std::vector<CUtensorMap> maps;
    for (size_t m = 0; m < md.size(); ++m) {
        md[m].tmap = NO_PAIR;
        const HostMesh& H = s->meshes[m];
        if (!encode || !(H.flags & MF_GRID) || !(H.flags & MF_CLOTH)) continue;
        const u32 n = H.d.grid_n;
        const cuuint64_t dims[3] = {4, n, n};
        const cuuint64_t strides[2] = {16, 16 * (cuuint64_t)n};  // bytes, dims 1 and 2
        const cuuint32_t box[3] = {4, (cuuint32_t)HALO_W, (cuuint32_t)HALO_H};
        const cuuint32_t estr[3] = {1, 1, 1};
        const u32 first = (u32)maps.size();
        bool ok = true;
        for (int b = 0; b < 5 && ok; ++b) {
            float4* base = (b < 3 ? s->X[b].p : s->V[b - 3].p) + H.voff;
            CUtensorMap tm;
            ok = encode(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
            if (ok) maps.push_back(tm);
        }
        if (!ok) { maps.resize(first); continue; }
        md[m].tmap = first;
    }
    if (!maps.empty()) {
        YS_CK(s->tmaps.alloc(maps.size()));
        YS_CK(cudaMemcpyAsync(s->tmaps.p, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice,
                              s->stream));
    }
    YS_CK(cudaMemcpyAsync(s->dmeshes.p, md.data(), sizeof(MeshDev) * md.size(), cudaMemcpyHostToDevice, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));  // md and maps live on the host stack
    s->hmeshes = md;
    return YS_OK;
}

// One k_fused launch per non-empty size class (classes do not interact:
// each launch writes only its own vertices' next state).
void launch_fused_classes(ys_scene* s, StepArgs A) {
    for (size_t c = 0; c + 1 < s->cls_off.size(); ++c) {
        A.tbase = s->cls_off[c];
        A.tend = s->cls_off[c + 1];
        A.tiles = s->cls_order[c] == ORDER_TILE ? 1u : 0u;
        launch_fused(A, s->stream, s->cls_variant[c]);
    }
}

ys_status preamble(ys_scene* s) {
    if (s->cursor != 0) return YS_OK;
    {
        ys_status r = refresh_shapes(s);
        if (r) return r;
    }
    if (s->P.rebuild_frames && s->frame % s->P.rebuild_frames == 0) {
        bool rebuilt = false;
        for (auto& H : s->meshes) {
            if (H.built && H.d.behavior == YS_FLOAT) continue;
            if (!H.needs_tree) continue;  // its root box comes from the root-only refit
            ys_status r = build_tree(s, H);
            if (r) return r;
            rebuilt = true;
        }
        if (rebuilt) {
            ys_status r = build_levels(s);
            if (r) return r;
            if ((r = compute_order(s))) return r;
        }
    }
    // environment forces (ext = g * m) are evaluated inside the force kernels
    return YS_OK;
}

// Refit of every live tree (the analytic markers are taken from the new root
// boxes by the kernels that consume them).
ys_status refit(ys_scene* s) {
    if (s->nrjobs)
        launch_root_boxes(s->rjobs.p + (size_t)(s->cur * 2 + s->cv) * s->nrjobs, s->nrjobs, s->rchunks.p,
                          s->nrchunks, s->stream);
    if (s->njobs) {
        // the job table for the current (position, velocity) buffer pair
        const RefitJob* table = s->jobs.p + (size_t)(s->cur * 2 + s->cv) * s->njobs;
        YS_CK(cudaMemsetAsync(s->maxext.p, 0, s->maxext.n * 4, s->stream));
        launch_refit(table, s->njobs, s->refitLeaves, s->status.p, s->stream);
        if (s->use_levels && s->use_ranges) {
            launch_refit_ranges(table, s->njobs, s->bigEnt.p, (u32)s->bigEnt.n, s->nbig, s->nhuge, s->stream);
        } else if (s->use_levels) {
            launch_refit_levels(table, s->wlist.p, s->hoff.p, s->lvl_off.data(), s->lvl_top, s->stream);
        }
        if (s->nRootOnly) launch_refit_roots(table, s->njobs, s->stream);
    }
    return YS_OK;
}

ys_status ensure_staged(ys_scene* s) {
    if (s->staged_ready) return YS_OK;
    YS_CK(s->rows.alloc(s->cap));
    YS_CK(s->contacts.alloc(s->cap));
    YS_CK(s->csr.alloc(s->cap));
    YS_CK(s->bucket.alloc(s->nV + 1));
    YS_CK(s->csr_off.alloc(s->nV + 1));
    YS_CK(s->Fbuf.alloc(s->nV));
    YS_CK(cudaMemsetAsync(s->Fbuf.p, 0, s->nV * sizeof(float4), s->stream));
    YS_CK(s->scanScratch.alloc(scan_scratch_bytes(s->nV + 1)));
    s->staged_ready = true;
    return YS_OK;
}

ys_status ensure_record(ys_scene* s) {
    if (s->record_ready) return YS_OK;
    YS_CK(s->pool.alloc(s->cap));
    YS_CK(s->vstart.alloc(s->nV));
    YS_CK(s->vcount.alloc(s->nV));
    YS_CK(cudaMemsetAsync(s->vcount.p, 0, s->nV * 4, s->stream));
    YS_CK(cudaMemsetAsync(s->vstart.p, 0, s->nV * 4, s->stream));
    s->record_ready = true;
    return YS_OK;
}

ys_status detect(ys_scene* s) {
    ys_status r = ensure_staged(s);
    if (r) return r;
    YS_CK(cudaMemsetAsync(s->counters.p, 0, 8, s->stream));
    StepArgs A = make_args(s);
    k_detect_rows<<<ceil_div(s->nV, 128), 128, 0, s->stream>>>(A);
    YS_CK(cudaGetLastError());
    return YS_OK;
}

ys_status narrow_and_sort(ys_scene* s) {
    ys_status r = ensure_staged(s);
    if (r) return r;
    unsigned long long cnt[2];
    YS_CK(cudaMemcpyAsync(cnt, s->counters.p, 16, cudaMemcpyDeviceToHost, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));
    u32 nrows = (u32)std::min<unsigned long long>(cnt[0], s->cap);
    s->last_rows = cnt[0];
    YS_CK(cudaMemsetAsync(s->counters.p + 1, 0, 8, s->stream));
    StepArgs A = make_args(s);
    if (nrows) k_narrow_rows<<<ceil_div(nrows, 128), 128, 0, s->stream>>>(A, nrows);
    if (s->apair_total) k_narrow_analytic_scene<<<ceil_div(s->apair_total, 128), 128, 0, s->stream>>>(A);
    YS_CK(cudaMemcpyAsync(cnt, s->counters.p, 16, cudaMemcpyDeviceToHost, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));
    u32 nc = (u32)std::min<unsigned long long>(cnt[1], s->cap);
    s->last_contacts_n = cnt[1];
    YS_CK(cudaMemsetAsync(s->bucket.p, 0, (s->nV + 1) * 4, s->stream));
    if (nc) k_bucket_count<<<ceil_div(nc, 256), 256, 0, s->stream>>>(A, nc);
    YS_CK(cudaMemcpyAsync(s->csr_off.p, s->bucket.p, (s->nV + 1) * 4, cudaMemcpyDeviceToDevice, s->stream));
    YS_CK(exclusive_scan(s->csr_off.p, s->nV + 1, s->scanScratch.p, s->stream));
    YS_CK(cudaMemsetAsync(s->bucket.p, 0, (s->nV + 1) * 4, s->stream));
    if (nc) k_bucket_scatter<<<ceil_div(nc, 256), 256, 0, s->stream>>>(A, nc);
    k_bucket_sort<<<ceil_div(s->nV, 256), 256, 0, s->stream>>>(A);
    YS_CK(cudaGetLastError());
    s->last_contacts = 1;
    return YS_OK;
}

ys_status system_update(ys_scene* s) {
    ys_status r = ensure_staged(s);
    if (r) return r;
    StepArgs A = make_args(s);
    k_forces<<<ceil_div(s->nV, 128), 128, 0, s->stream>>>(A);
    k_integrate<<<ceil_div(s->nV, 128), 128, 0, s->stream>>>(A);
    YS_CK(cudaGetLastError());
    // non-cloth vertices are never written: keep every buffer equal for them
    rotate(s);
    return YS_OK;
}

void drop_graphs(ys_scene* s) {
    for (auto& g : s->graphs)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

// Enqueue the device work of one fused substep (no preamble, no rotation).
ys_status enqueue_fused(ys_scene* s) {
    ys_status r = refit(s);
    if (r) return r;
    YS_CK(cudaMemsetAsync(s->counters.p, 0, s->record ? 24 : 16, s->stream));
    StepArgs A = make_args(s);
    launch_fused_classes(s, A);
    YS_CK(cudaGetLastError());
    return YS_OK;
}

cudaEvent_t next_event(ys_scene* s) {
    if (s->evUsed == s->evPool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        s->evPool.push_back(e);
    }
    return s->evPool[s->evUsed++];
}

ys_status fused_substep(ys_scene* s) {
    ys_status r = preamble(s);
    if (r) return r;
    if (s->use_graphs && !s->timing && !s->record) {
        const int key = (s->cur * 3 + s->prev) * 2 + s->cv;
        if (!s->graphs[key]) {
            cudaGraph_t g = nullptr;
            YS_CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
            ys_status er = enqueue_fused(s);
            cudaError_t ce = cudaStreamEndCapture(s->stream, &g);
            if (er) { if (g) cudaGraphDestroy(g); return er; }
            if (ce != cudaSuccess) return fail(YS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
            ce = cudaGraphInstantiate(&s->graphs[key], g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) return fail(YS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
        }
        YS_CK(cudaGraphLaunch(s->graphs[key], s->stream));
        s->snapshot_pending = true;
        rotate(s);
        return YS_OK;
    }
    if (s->timing) {
        s->evRefit.push_back(s->evUsed);
        YS_CK(cudaEventRecord(next_event(s), s->stream));
    }
    r = refit(s);
    if (r) return r;
    if (s->timing) {
        YS_CK(cudaEventRecord(next_event(s), s->stream));
    }
    if (s->record) {
        r = ensure_record(s);
        if (r) return r;
        YS_CK(cudaMemsetAsync(s->counters.p, 0, 24, s->stream));
    } else {
        // counters [0] [1] only; [3] [4] keep running totals
        YS_CK(cudaMemsetAsync(s->counters.p, 0, 16, s->stream));
    }
    StepArgs A = make_args(s);
    if (s->timing) {
        s->evFused.push_back(s->evUsed);
        YS_CK(cudaEventRecord(next_event(s), s->stream));
    }
    launch_fused_classes(s, A);
    YS_CK(cudaGetLastError());
    if (s->timing) YS_CK(cudaEventRecord(next_event(s), s->stream));
    s->snapshot_pending = true;
    rotate(s);
    if (s->record) s->last_contacts = 2;
    return YS_OK;
}

}  // namespace

extern "C" {

const char* ys_last_error(void) { return g_err.c_str(); }
const char* ys_version(void) { return "ysim_b200 0.1 (sm_100a)"; }

ys_status ys_scene_create(ys_scene** out, const ys_sim_params* p, int device) {
    if (!out || !p) return fail(YS_ERR_BAD_ARG, "null argument");
    if (p->substeps == 0) return fail(YS_ERR_BAD_ARG, "substeps must be > 0");
    if (p->self_mode > YS_SELF_BVH) return fail(YS_ERR_BAD_ARG, "bad self_mode");
    YS_CK(cudaSetDevice(device));
    ys_scene* s = new ys_scene();
    s->device = device;
    s->P = *p;
    if (s->P.cols_per_point == 0) s->P.cols_per_point = 15;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete s; return fail(YS_ERR_CUDA, cudaGetErrorString(e)); }
    *out = s;
    return YS_OK;
}

ys_status ys_scene_destroy(ys_scene* s) {
    if (!s) return YS_OK;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    for (auto& b : s->X) b.free();
    for (auto& b : s->V) b.free();
    s->Fbuf.free(); s->mass.free(); s->mask.free(); s->vobj.free(); s->targets.free(); s->spr_off.free();
    s->spr_split.free(); s->spr_nbr.free(); s->vaf_off.free(); s->vaf.free(); s->maxext.free(); s->status.free();
    s->codes.free(); s->idx.free(); s->lvid.free(); s->visits.free(); s->box.free(); s->spr_rest.free(); s->scratch3.free(); s->gk.free(); s->gL.free(); s->F4.free(); s->F3.free();
    s->nodes.free(); s->parent.free(); s->claims.free(); s->claimOff.free(); s->karrasScratch.free(); s->aggScratch.free(); s->rootAcc.free();
    s->rjobs.free(); s->rchunks.free(); s->dmeshes.free(); s->jobs.free(); s->counters.free(); s->sortScratch.free();
    s->w4.free(); s->leafW.free(); s->warrive.free(); s->wideScratch.free();
    s->leafWf.free(); s->wcount.free(); s->hacc.free(); s->wlist.free(); s->hcount.free(); s->hoff.free();
    s->hcursor.free();
    s->dshapes.free(); s->apairs.free(); s->tpair.free(); s->markers.free();
    s->scanScratch.free(); s->rows.free(); s->contacts.free(); s->csr.free(); s->pool.free(); s->bucket.free();
    drop_graphs(s);
    s->csr_off.free(); s->vstart.free(); s->vcount.free(); s->ext.free();
    s->fpos.free(); s->own.free(); s->bb16.free(); s->bb256.free(); s->wrange.free(); s->blkEnt.free(); s->bigEnt.free();
    s->blkCnt.free(); s->blkOff.free(); s->bigCnt.free(); s->rangeScratch.free(); s->vorder.free(); s->okeys.free(); s->oaoff.free(); s->orank.free(); s->obox.free(); s->oscratch.free(); s->omorton.free();
    for (auto e : s->evPool) cudaEventDestroy(e);
    cudaStreamDestroy(s->stream);
    delete s;
    return YS_OK;
}

ys_status ys_scene_add_mesh(ys_scene* s, const ys_mesh_desc* d, int* index_out) {
    if (!s || !d) return fail(YS_ERR_BAD_ARG, "null argument");
    if (s->packed) return fail(YS_ERR_STATE, "scene already packed");
    if (d->num_vertices == 0 || !d->x) return fail(YS_ERR_BAD_ARG, "mesh needs vertices");
    if (d->num_facets && !d->facets) return fail(YS_ERR_BAD_ARG, "facets missing");
    const bool cloth = d->behavior == YS_TRIANGULAR_CLOTH || d->behavior == YS_FAST_GRID_CLOTH;
    if (cloth && (!d->mass || !d->mask)) return fail(YS_ERR_BAD_ARG, "cloth needs mass and mask");
    if (d->behavior == YS_FAST_GRID_CLOTH && (d->grid_n < 3 || d->grid_n * d->grid_n != d->num_vertices))
        return fail(YS_ERR_BAD_ARG, "FastGridCloth needs grid_n^2 vertices, grid_n >= 3");
    for (u32 i = 0; i < 3 * d->num_facets; ++i)
        if (d->facets[i] >= d->num_vertices) return fail(YS_ERR_BAD_ARG, "facet index out of range");
    HostMesh H;
    H.d = *d;
    const u32 nV = d->num_vertices;
    H.x.assign(d->x, d->x + 3 * (size_t)nV);
    if (d->v) H.v.assign(d->v, d->v + 3 * (size_t)nV); else H.v.assign(3 * (size_t)nV, 0.f);
    if (d->mass) H.mass.assign(d->mass, d->mass + nV); else H.mass.assign(nV, 1.f);
    if (d->mask) H.mask.assign(d->mask, d->mask + nV); else H.mask.assign(nV, 1.f);
    H.F.assign(d->facets, d->facets + 3 * (size_t)d->num_facets);
    H.d.x = H.d.v = H.d.mass = H.d.mask = nullptr;
    H.d.facets = nullptr;
    s->meshes.push_back(std::move(H));
    if (index_out) *index_out = (int)s->meshes.size() - 1;
    return YS_OK;
}

ys_status ys_scene_pack(ys_scene* s) {
    if (!s) return fail(YS_ERR_BAD_ARG, "null scene");
    if (s->packed) return fail(YS_ERR_STATE, "already packed");
    if (s->meshes.empty()) return fail(YS_ERR_BAD_ARG, "empty scene");
    YS_CK(cudaSetDevice(s->device));
    u32 nV = 0, nF = 0, nNodes = 0, maxF = 1, nW4 = 0;
    for (auto& H : s->meshes) {
        H.voff = nV; H.foff = nF; H.node_off = nNodes;
        H.w4_off = nW4;
        H.w4_cap = H.d.num_facets ? std::max(H.d.num_facets - 1, 1u) : 0u;
        nW4 += H.w4_cap;
        nV += H.d.num_vertices;
        nF += H.d.num_facets;
        nNodes += H.d.num_facets ? 2 * H.d.num_facets - 1 : 0;
        maxF = std::max(maxF, H.d.num_facets);
        const bool cloth = H.d.behavior == YS_TRIANGULAR_CLOTH || H.d.behavior == YS_FAST_GRID_CLOTH;
        u32 f = 0;
        if (H.d.flags & YS_MESH_STATIC) f |= MF_STATIC;
        if (H.d.flags & YS_MESH_COLLIDABLE) f |= MF_COLLIDABLE;
        if (H.d.flags & YS_MESH_SELF_COLLIDE) f |= MF_SELF;
        if ((H.d.flags & YS_MESH_COLLIDABLE) && H.d.behavior != YS_FLOAT && H.d.behavior != YS_KINEMATIC) f |= MF_QUERY;
        if (cloth) f |= MF_CLOTH;
        if (H.d.num_facets) f |= MF_TREE;
        if (H.d.behavior == YS_FAST_GRID_CLOTH) f |= MF_GRID;
        // an analytic collider descends no tree: as a query it only marks
        // pairs with analytic targets (when it is cloth) and keeps the CPU-hash
        // self rows (BroadPhase::detectCollisions, bvh.hpp:2886-2937;
        // simulator.hpp:3678-3701)
        if (H.collider != COL_MESH) f |= MF_ANALYTIC;
        H.flags = f;
        build_adjacency(H);
    }
    s->nV = nV; s->nF = nF; s->nNodes = nNodes;
    s->cap = s->P.cols_per_point * nV;
    // host staging of packed arrays
    std::vector<float> x3(3 * (size_t)nV), v3(3 * (size_t)nV), mass(nV), mask(nV);
    std::vector<u32> vobj(nV), F3(3 * (size_t)nF), spr_off(nV + 1, 0), spr_split(nV, 0), vaf_off(nV + 1, 0);
    std::vector<uint4> F4(nF);
    std::vector<u32> spr_nbr, vaf;
    std::vector<float> spr_rest;
    std::vector<MeshDev> md(s->meshes.size());
    std::vector<u32> targets;
    for (size_t m = 0; m < s->meshes.size(); ++m) {
        HostMesh& H = s->meshes[m];
        const u32 n = H.d.num_vertices;
        std::copy(H.x.begin(), H.x.end(), x3.begin() + 3 * (size_t)H.voff);
        std::copy(H.v.begin(), H.v.end(), v3.begin() + 3 * (size_t)H.voff);
        std::copy(H.mass.begin(), H.mass.end(), mass.begin() + H.voff);
        std::copy(H.mask.begin(), H.mask.end(), mask.begin() + H.voff);
        for (u32 i = 0; i < n; ++i) vobj[H.voff + i] = (u32)m;
        for (u32 f = 0; f < H.d.num_facets; ++f) {
            F4[H.foff + f] = make_uint4(H.F[3 * f], H.F[3 * f + 1], H.F[3 * f + 2], 0u);
            for (int k = 0; k < 3; ++k) F3[3 * ((size_t)H.foff + f) + k] = H.F[3 * f + k];
        }
        // springs: global neighbour ids
        const u32 sbase = (u32)spr_nbr.size();
        for (u32 i = 0; i < n; ++i) {
            spr_off[H.voff + i] = sbase + H.spr_off[i];
            spr_split[H.voff + i] = sbase + H.spr_split[i];
        }
        for (u32 j : H.spr_nbr) spr_nbr.push_back(H.voff + j);
        spr_rest.insert(spr_rest.end(), H.spr_rest.begin(), H.spr_rest.end());
        const u32 abase = (u32)vaf.size();
        for (u32 i = 0; i < n; ++i) vaf_off[H.voff + i] = abase + H.vaf_off[i];
        vaf.insert(vaf.end(), H.vaf.begin(), H.vaf.end());
        MeshDev D;
        memset(&D, 0, sizeof(D));
        D.voff = H.voff; D.nV = n; D.foff = H.foff; D.nF = H.d.num_facets; D.node_off = H.node_off;
        D.behavior = H.d.behavior; D.flags = H.flags; D.grid_n = H.d.grid_n;
        D.kstretch = H.d.kstretch; D.kshear = H.d.kshear; D.kbend = H.d.kbend; D.thickness = H.d.thickness;
        for (int k = 0; k < 6; ++k) D.rest[k] = H.d.grid_rest[k];
        // inter-object targets, in mesh order (bvh.hpp:2884-2941)
        D.tgt_begin = (u32)targets.size();
        if (H.flags & MF_QUERY)
            for (size_t t = 0; t < s->meshes.size(); ++t) {
                if (t == m) continue;
                const HostMesh& T = s->meshes[t];
                if (!(T.d.flags & YS_MESH_COLLIDABLE)) continue;
                if (T.d.num_facets == 0 && T.collider == COL_MESH) continue;
                if (T.d.group != H.d.group) continue;
                targets.push_back((u32)t);
            }
        D.tgt_end = (u32)targets.size();
        D.gspr = NO_SPRINGS;
        D.w4_off = H.w4_off;
        D.w4_cap = H.w4_cap;
        D.shape = NO_PAIR;
        if (H.collider != COL_MESH) {
            D.shape = (u32)s->shape_mesh.size();
            s->shape_mesh.push_back((int)m);
        }
        md[m] = D;
    }
    spr_off[nV] = (u32)spr_nbr.size();
    vaf_off[nV] = (u32)vaf.size();
    // own-face windows: a vertex's faces, sorted, in at most two runs of 8
    // ids each (a grid cloth's vertex: the two cell rows around it)
    std::vector<uint2> ownw(nV, make_uint2(0u, 0u));
    for (u32 gv = 0; gv < nV; ++gv) {
        std::vector<u32> fs(vaf.begin() + vaf_off[gv], vaf.begin() + vaf_off[gv + 1]);
        if (fs.empty()) continue;
        std::sort(fs.begin(), fs.end());
        const u32 a = fs[0];
        size_t k = 0;
        u32 ma = 0, mb = 0, b = a;
        while (k < fs.size() && fs[k] - a < 8u) ma |= 1u << (fs[k++] - a);
        if (k < fs.size()) {
            b = fs[k];
            while (k < fs.size() && fs[k] - b < 8u) mb |= 1u << (fs[k++] - b);
        }
        if (k < fs.size() || b - a >= 65536u) continue;  // does not fit: no filtering for this vertex
        ownw[gv] = make_uint2(a, ((b - a) << 16) | (mb << 8) | ma);
    }
    cudaStream_t st = s->stream;
    // device allocations
    for (auto& b : s->X) YS_CK(b.alloc(nV));
    for (auto& b : s->V) YS_CK(b.alloc(nV));
    YS_CK(s->mass.alloc(nV)); YS_CK(s->mask.alloc(nV)); YS_CK(s->vobj.alloc(nV));
    YS_CK(s->targets.alloc(std::max<size_t>(targets.size(), 1)));
    YS_CK(s->spr_off.alloc(nV + 1)); YS_CK(s->spr_split.alloc(nV));
    YS_CK(s->spr_nbr.alloc(std::max<size_t>(spr_nbr.size(), 1))); YS_CK(s->spr_rest.alloc(std::max<size_t>(spr_rest.size(), 1)));
    YS_CK(s->vaf_off.alloc(nV + 1)); YS_CK(s->vaf.alloc(std::max<size_t>(vaf.size(), 1)));
    YS_CK(s->maxext.alloc(s->meshes.size())); YS_CK(s->status.alloc(1)); YS_CK(s->box.alloc(8));
    YS_CK(s->codes.alloc(std::max(nF, 1u))); YS_CK(s->idx.alloc(std::max(nF, 1u))); YS_CK(s->lvid.alloc(std::max(nF, 1u))); YS_CK(s->visits.alloc(std::max(nF, 1u)));
    YS_CK(s->F4.alloc(std::max(nF, 1u))); YS_CK(s->F3.alloc(3 * (size_t)std::max(nF, 1u)));
    YS_CK(s->fpos.alloc(3 * (size_t)std::max(nF, 1u)));
    YS_CK(s->own.alloc(std::max(nV, 1u)));
    YS_CK(s->nodes.alloc(std::max(nNodes, 1u))); YS_CK(s->parent.alloc(std::max(nNodes, 1u)));
    YS_CK(s->claims.alloc(std::max(nNodes, 1u)));
    YS_CK(s->claimOff.alloc((size_t)nNodes + s->meshes.size() + 1));
    YS_CK(s->karrasScratch.alloc(karras_scratch_bytes(maxF)));
    if (s->tree_builder == YS_BUILD_APETREI) YS_CK(s->aggScratch.alloc(apetrei_scratch_bytes(maxF)));
    YS_CK(s->dmeshes.alloc(md.size())); YS_CK(s->jobs.alloc(6 * s->meshes.size() + 2));
    if (s->tree_layout == YS_TREE_CUBE) {
        YS_CK(s->w4.alloc(std::max(nW4, 1u))); YS_CK(s->leafW.alloc(std::max(nF, 1u)));
        YS_CK(s->leafWf.alloc(std::max(nF, 1u)));
        YS_CK(s->warrive.alloc(std::max(nW4, 1u))); YS_CK(s->wideScratch.alloc(wide_build_scratch_bytes(maxF)));
        YS_CK(cudaMemsetAsync(s->warrive.p, 0, 4 * s->warrive.n, s->stream));
        YS_CK(s->wcount.alloc(s->meshes.size())); YS_CK(cudaMemsetAsync(s->wcount.p, 0, 4 * s->meshes.size(), s->stream));
        YS_CK(s->hacc.alloc(std::max(nW4, 1u))); YS_CK(s->wlist.alloc(std::max(nW4, 1u)));
        YS_CK(s->wrange.alloc(std::max(nW4, 1u)));
        YS_CK(s->hcount.alloc(MAX_LEVELS + 2)); YS_CK(s->hoff.alloc(MAX_LEVELS + 2));
        YS_CK(s->hcursor.alloc(MAX_LEVELS + 2));
    }
    YS_CK(s->counters.alloc(8));
    YS_CK(s->sortScratch.alloc(sort_scratch_bytes(maxF)));
    // uploads
    DBuf<float> tmp3;
    YS_CK(tmp3.alloc(3 * (size_t)nV));
    YS_CK(cudaMemcpyAsync(tmp3.p, x3.data(), 12 * (size_t)nV, cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    for (auto& b : s->X) k_pack4<<<ceil_div(nV, 256), 256, 0, st>>>(tmp3.p, b.p, nV);
    YS_CK(cudaStreamSynchronize(st));
    YS_CK(cudaMemcpyAsync(tmp3.p, v3.data(), 12 * (size_t)nV, cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    for (auto& b : s->V) k_pack4<<<ceil_div(nV, 256), 256, 0, st>>>(tmp3.p, b.p, nV);
    YS_CK(cudaStreamSynchronize(st));
    tmp3.free();
    YS_CK(cudaMemcpyAsync(s->mass.p, mass.data(), 4 * (size_t)nV, cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    YS_CK(cudaMemcpyAsync(s->mask.p, mask.data(), 4 * (size_t)nV, cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    YS_CK(cudaMemcpyAsync(s->vobj.p, vobj.data(), 4 * (size_t)nV, cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    if (!targets.empty()) YS_CK(cudaMemcpyAsync(s->targets.p, targets.data(), 4 * targets.size(), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    YS_CK(cudaMemcpyAsync(s->spr_off.p, spr_off.data(), 4 * (size_t)(nV + 1), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    YS_CK(cudaMemcpyAsync(s->spr_split.p, spr_split.data(), 4 * (size_t)nV, cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    if (!spr_nbr.empty()) {
        YS_CK(cudaMemcpyAsync(s->spr_nbr.p, spr_nbr.data(), 4 * spr_nbr.size(), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
        YS_CK(cudaMemcpyAsync(s->spr_rest.p, spr_rest.data(), 4 * spr_rest.size(), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    }
    YS_CK(cudaMemcpyAsync(s->vaf_off.p, vaf_off.data(), 4 * (size_t)(nV + 1), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    YS_CK(cudaMemcpyAsync(s->own.p, ownw.data(), sizeof(uint2) * (size_t)nV, cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    if (!vaf.empty()) YS_CK(cudaMemcpyAsync(s->vaf.p, vaf.data(), 4 * vaf.size(), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    if (nF) {
        YS_CK(cudaMemcpyAsync(s->F4.p, F4.data(), 16 * (size_t)nF, cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
        YS_CK(cudaMemcpyAsync(s->F3.p, F3.data(), 12 * (size_t)nF, cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    }
    YS_CK(cudaMemcpyAsync(s->dmeshes.p, md.data(), sizeof(MeshDev) * md.size(), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
    s->hmeshes = md;
    // Analytic marker pairs: every (cloth query mesh with a tree, analytic
    // target), in target order; pair p owns threads [w, w + nV) of the staged
    // analytic kernel.
    {
        std::vector<uint4> ap;
        std::vector<u32> tp(std::max<size_t>(targets.size(), 1), NO_PAIR);
        u32 vb = 0;
        for (size_t m = 0; m < md.size(); ++m) {
            const u32 f = md[m].flags;
            if (!(f & MF_QUERY) || !(f & MF_CLOTH) || !(f & MF_TREE) || md[m].nV == 0) continue;
            for (u32 k = md[m].tgt_begin; k < md[m].tgt_end; ++k) {
                const u32 t = targets[k];
                if (!(md[t].flags & MF_ANALYTIC)) continue;
                tp[k] = (u32)ap.size();
                ap.push_back(make_uint4((u32)m, t, md[t].shape, vb));
                vb += md[m].nV;
            }
        }
        s->npairs = (u32)ap.size();
        s->apair_total = vb;
        YS_CK(s->tpair.alloc(tp.size()));
        YS_CK(cudaMemcpyAsync(s->tpair.p, tp.data(), 4 * tp.size(), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
        if (!ap.empty()) {
            YS_CK(s->apairs.alloc(ap.size()));
            YS_CK(cudaMemcpyAsync(s->apairs.p, ap.data(), sizeof(uint4) * ap.size(), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
            YS_CK(s->markers.alloc(2 * ap.size()));
            YS_CK(cudaMemsetAsync(s->markers.p, 0, 4 * 2 * ap.size(), s->stream));
        }
        if (!s->shape_mesh.empty()) {
            // seeded at pack (Scene::packAnalyticShapes, scene.hpp:762-781):
            // the first frame's refresh still takes prev = cur
            YS_CK(s->dshapes.alloc(s->shape_mesh.size()));
            DShape z;
            memset(&z, 0, sizeof(z));
            s->hshapes.assign(s->shape_mesh.size(), z);
            s->analytic_primed = false;
            s->shapes_uploaded = false;
            ys_status r = refresh_shapes(s);
            if (r) return r;
            s->analytic_primed = false;
            YS_CK(cudaStreamSynchronize(s->stream));
        }
    }
    YS_CK(cudaMemsetAsync(s->status.p, 0, 4, s->stream));
    YS_CK(cudaMemsetAsync(s->maxext.p, 0, 4 * s->meshes.size(), s->stream));
    YS_CK(cudaMemsetAsync(s->counters.p, 0, 8 * s->counters.n, s->stream));
    // Which trees a query descends: the targets of every query mesh, and the
    // self-queried meshes.  A query mesh whose own tree nothing descends
    // still needs that tree's root box (the inter-object cull): a root-only
    // refit (or, for a static mesh, the one build) provides it.
    std::vector<char> descended(s->meshes.size(), 0), rootUsed(s->meshes.size(), 0);
    for (size_t m = 0; m < s->meshes.size(); ++m) {
        const HostMesh& H = s->meshes[m];
        if (!(H.flags & MF_QUERY) || !(H.flags & MF_TREE)) continue;
        const bool selfQ = s->P.self_mode == YS_SELF_BVH ||
                           (s->P.self_mode == YS_SELF_HASH && (H.flags & MF_CLOTH) && (H.flags & MF_SELF));
        if (selfQ) descended[m] = 1;
        for (u32 k = md[m].tgt_begin; k < md[m].tgt_end; ++k)
            if (!(md[targets[k]].flags & MF_ANALYTIC) && !(H.flags & MF_ANALYTIC)) descended[targets[k]] = 1;
        if (md[m].tgt_end > md[m].tgt_begin) rootUsed[m] = 1;
    }
    for (size_t m = 0; m < s->meshes.size(); ++m) {
        HostMesh& H = s->meshes[m];
        H.needs_tree = H.d.num_facets && (descended[m] || ((H.flags & MF_STATIC) && rootUsed[m]));
    }
    // refit jobs: every non-static tree a query descends, plus static cloth
    // that needs the self-hash grid extent; root-only jobs for the rest whose
    // root box the cull reads
    s->hjobs.clear();
    std::vector<RefitJob> hr;        // vertex-form root-only jobs
    std::vector<uint2> chunks;
    u32 leaves = 0;
    s->nRootOnly = 0;
    for (size_t m = 0; m < s->meshes.size(); ++m) {
        HostMesh& H = s->meshes[m];
        if (!H.d.num_facets) continue;
        const bool selfHash = s->P.self_mode == YS_SELF_HASH && (H.flags & MF_CLOTH) && (H.flags & MF_SELF) &&
                              (H.flags & MF_QUERY);
        if ((H.flags & MF_STATIC) && !selfHash) continue;
        if (!descended[m] && !rootUsed[m] && !selfHash) continue;
        const bool rootOnly = !descended[m] && !selfHash;
        RefitJob J;
        memset(&J, 0, sizeof(J));
        J.nodes = s->nodes.p + H.node_off;
        J.parent = s->parent.p + H.node_off;
        J.claimOff = claim_off(s, H);
    J.claims = s->claims.p + H.node_off;
        J.visits = s->visits.p + H.foff;
        J.facets = s->F3.p + 3 * (size_t)H.foff;
        J.voff = H.voff;
        J.n = H.d.num_facets;
        J.leafBase = leaves;
        J.dt = s->P.subh;
        J.swept = (H.flags & MF_STATIC) ? 0u : 1u;
        J.selfMargin = selfHash ? s->P.margin : 0.f;
        J.maxExt = s->maxext.p + m;
        if (rootOnly) {
            J.rootOnly = 1;
            J.nVert = H.d.num_vertices;
            std::vector<char> onFace(H.d.num_vertices, 0);
            for (u32 v : H.F) onFace[v] = 1;
            if (std::all_of(onFace.begin(), onFace.end(), [](char c) { return c != 0; })) {
                for (u32 c0 = 0; c0 < J.nVert; c0 += ROOT_CHUNK) chunks.push_back(make_uint2((u32)hr.size(), c0));
                hr.push_back(J);
                continue;
            }
            ++s->nRootOnly;
        } else if (s->tree_layout == YS_TREE_CUBE) {
            J.w4 = s->w4.p + H.w4_off;
            J.leafW = s->leafW.p + H.foff;
            J.warrive = s->warrive.p + H.w4_off;
            J.leafWf = s->leafWf.p + H.foff;
            J.wcount = s->wcount.p + m;
            J.hacc = s->hacc.p + H.w4_off;
        }
        if (!J.rootOnly) J.fpos = s->fpos.p + 3 * (size_t)H.foff;  // faces the fused kernel tests
        if (J.w4) { J.wrange = s->wrange.p + H.w4_off; J.idx = s->idx.p + H.foff; J.lvid = s->lvid.p + H.foff; }
        s->hjobs.push_back(J);
        // every job's leaves start on a 256-leaf boundary (the range refit's
        // blocks then never hold two jobs)
        leaves = (leaves + J.n + 255u) & ~255u;
    }
    s->refitLeaves = leaves;
    YS_CK(s->bb16.alloc(std::max<size_t>(leaves / 16, 1)));
    YS_CK(s->bb256.alloc(std::max<size_t>(leaves / 256, 1)));
    {
        const u32 nb = leaves / 256 + 1;
        YS_CK(s->blkCnt.alloc(nb + 1)); YS_CK(s->blkOff.alloc(nb + 1)); YS_CK(s->bigCnt.alloc(2));
        YS_CK(s->blkEnt.alloc(std::max(nW4, 1u))); YS_CK(s->bigEnt.alloc(std::max(nW4, 1u)));
        YS_CK(s->rangeScratch.alloc(scan_scratch_bytes(nb + 1)));
        YS_CK(cudaMemsetAsync(s->blkOff.p, 0, 4 * (size_t)(nb + 1), s->stream));
    }
    for (auto& J : s->hjobs) {
        J.bb16 = s->bb16.p; J.bb256 = s->bb256.p;
        J.blkEnt = s->blkEnt.p; J.blkOff = s->blkOff.p;
    }
    s->njobs = (u32)s->hjobs.size();
    s->nrjobs = (u32)hr.size();
    s->nrchunks = (u32)chunks.size();
    {
        const size_t nacc = std::max<size_t>(s->njobs + s->nrjobs, 1);
        std::vector<u32> acc(32 * nacc, 0u);
        for (size_t j = 0; j < nacc; ++j)
            for (int k = 0; k < 3; ++k) acc[32 * j + k] = 0xFFFFFFFFu;
        YS_CK(s->rootAcc.alloc(acc.size()));
        YS_CK(cudaMemcpyAsync(s->rootAcc.p, acc.data(), 4 * acc.size(), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
        for (size_t j = 0; j < s->hjobs.size(); ++j)
            s->hjobs[j].rootAcc = s->rootAcc.p + 32 * j;
        for (size_t j = 0; j < hr.size(); ++j) hr[j].rootAcc = s->rootAcc.p + 32 * (s->njobs + j);
    }
    if (s->nrjobs) {
        YS_CK(s->rjobs.alloc(6 * (size_t)s->nrjobs));
        YS_CK(s->rchunks.alloc(chunks.size()));
        YS_CK(cudaMemcpyAsync(s->rchunks.p, chunks.data(), chunks.size() * sizeof(uint2), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
        for (int c = 0; c < 3; ++c)
            for (int w = 0; w < 2; ++w) {
                std::vector<RefitJob> t = hr;
                for (auto& J : t) { J.x4 = s->X[c].p; J.v4 = s->V[w].p; }
                YS_CK(cudaMemcpyAsync(s->rjobs.p + (size_t)(c * 2 + w) * s->nrjobs, t.data(),
                                 t.size() * sizeof(RefitJob), cudaMemcpyHostToDevice, s->stream)); YS_CK(cudaStreamSynchronize(s->stream));
            }
    }
    {
        ys_status r = upload_jobs(s, false);
        if (r) return r;
    }
    s->packed = true;
    s->cur = 0; s->prev = 1; s->cv = 0;
    // BroadPhase::build at initialize (Simulator::initialize -> build)
    for (auto& H : s->meshes) {
        if (!H.needs_tree) continue;
        ys_status r = build_tree(s, H);
        if (r) return r;
    }
    {
        ys_status r = build_levels(s);
        if (r) return r;
    }
    {
        // working vertices of the fused kernel (cloth, moving, or querying),
        // mesh by mesh in size-class order
        const size_t nm = s->meshes.size();
        s->mesh_class.assign(nm, -1);
        s->cls_meshes.assign(NCLASS, 0);
        for (size_t m = 0; m < nm; ++m) {
            const u32 f = s->meshes[m].flags;
            if (!(f & MF_CLOTH) && (f & MF_STATIC) && !(f & MF_QUERY)) continue;
            const u32 nv = s->meshes[m].d.num_vertices;
            if (nv == 0) continue;
            int c = 0;
            while (c + 1 < NCLASS && nv > CLASS_MAX[c]) ++c;
            s->mesh_class[m] = c;
            s->cls_meshes[c]++;
        }
        u32 nmesh = 0;
        for (size_t m = 0; m < nm; ++m) nmesh += s->mesh_class[m] >= 0 ? 1u : 0u;
        s->cls_variant.assign(NCLASS, s->fused_min_blocks);
        s->cls_order.assign(NCLASS, ORDER_MORTON);
        u32 mbits = 0;
        while (mbits < 32 && (1ull << mbits) < nmesh) ++mbits;
        s->order_kbits = 32 - mbits;
        YS_CK(s->oaoff.alloc(nm));
        YS_CK(s->orank.alloc(nm));
        YS_CK(s->obox.alloc(6 * nm));
        YS_CK(s->omorton.alloc(nm));
        ys_status r = encode_tile_maps(s);
        if (r) return r;
        if ((r = order_layout(s))) return r;
        if ((r = compute_order(s))) return r;
    }
    YS_CK(cudaStreamSynchronize(st));
    return YS_OK;
}

ys_status ys_frame_preamble(ys_scene* s) { ys_status r = check_scene(s); return r ? r : preamble(s); }
ys_status ys_broad_refit(ys_scene* s) { ys_status r = check_scene(s); return r ? r : refit(s); }
ys_status ys_broad_detect(ys_scene* s) { ys_status r = check_scene(s); return r ? r : detect(s); }
ys_status ys_narrow_and_sort(ys_scene* s) { ys_status r = check_scene(s); return r ? r : narrow_and_sort(s); }
ys_status ys_snapshot_xprev(ys_scene* s) {
    ys_status r = check_scene(s);
    if (r) return r;
    s->snapshot_pending = true;
    return YS_OK;
}
ys_status ys_system_update(ys_scene* s) { ys_status r = check_scene(s); return r ? r : system_update(s); }

ys_status ys_scene_step_staged(ys_scene* s, uint32_t n) {
    ys_status r = check_scene(s);
    if (r) return r;
    for (u32 i = 0; i < n; ++i) {
        if ((r = preamble(s)) || (r = refit(s)) || (r = detect(s)) || (r = narrow_and_sort(s))) return r;
        s->snapshot_pending = true;
        if ((r = system_update(s))) return r;
    }
    return YS_OK;
}

ys_status ys_scene_step(ys_scene* s, uint32_t n) {
    ys_status r = check_scene(s);
    if (r) return r;
    for (u32 i = 0; i < n; ++i)
        if ((r = fused_substep(s))) return r;
    return YS_OK;
}

ys_status ys_scene_set_record(ys_scene* s, int record) {
    if (!s) return fail(YS_ERR_BAD_ARG, "null scene");
    s->record = record != 0;
    return YS_OK;
}

ys_status ys_scene_set_tree_layout(ys_scene* s, int layout) {
    if (!s) return fail(YS_ERR_BAD_ARG, "null scene");
    if (s->packed) return fail(YS_ERR_STATE, "ys_scene_set_tree_layout: call before ys_scene_pack");
    if (layout != YS_TREE_REFERENCE && layout != YS_TREE_CUBE) return fail(YS_ERR_BAD_ARG, "unknown tree layout");
    s->tree_layout = layout;
    return YS_OK;
}

ys_status ys_scene_set_collider(ys_scene* s, int mesh, uint32_t kind, const float center[3], const float half[3],
                                const float rot_wxyz[4]) {
    if (!s) return fail(YS_ERR_BAD_ARG, "null scene");
    if (mesh < 0 || (size_t)mesh >= s->meshes.size()) return fail(YS_ERR_BAD_ARG, "ys_scene_set_collider: bad mesh");
    if (kind > COL_PLANE) return fail(YS_ERR_BAD_ARG, "ys_scene_set_collider: unknown collider kind");
    if (!center || !rot_wxyz || (!half && kind != COL_PLANE && kind != COL_MESH))
        return fail(YS_ERR_BAD_ARG, "ys_scene_set_collider: null pose");
    HostMesh& H = s->meshes[mesh];
    if (s->packed && kind != H.collider)
        return fail(YS_ERR_STATE, "ys_scene_set_collider: the collider kind is fixed at ys_scene_pack");
    H.collider = kind;
    for (int k = 0; k < 3; ++k) H.pose[k] = center[k];
    for (int k = 0; k < 3; ++k) H.pose[3 + k] = half ? half[k] : 0.f;
    for (int k = 0; k < 4; ++k) H.pose[6 + k] = rot_wxyz[k];
    return YS_OK;
}

ys_status ys_scene_colliders(ys_scene* s, ys_analytic_shape* out, uint32_t cap, uint32_t* num_out) {
    if (!s) return fail(YS_ERR_BAD_ARG, "null scene");
    const u32 n = (u32)s->hshapes.size();
    if (num_out) *num_out = n;
    if (out) {
        static_assert(sizeof(ys_analytic_shape) == sizeof(AShape), "ys_analytic_shape layout");
        for (u32 k = 0; k < n && k < cap; ++k) memcpy(&out[k], &s->hshapes[k].s, sizeof(AShape));
    }
    return YS_OK;
}

ys_status ys_scene_set_tree_builder(ys_scene* s, int builder) {
    if (!s) return fail(YS_ERR_BAD_ARG, "null scene");
    if (s->packed) return fail(YS_ERR_STATE, "ys_scene_set_tree_builder: call before ys_scene_pack");
    if (builder != YS_BUILD_KARRAS && builder != YS_BUILD_APETREI) return fail(YS_ERR_BAD_ARG, "unknown tree builder");
    s->tree_builder = builder;
    return YS_OK;
}

ys_status ys_scene_set_fused_variant(ys_scene* s, int min_blocks) {
    if (!s) return fail(YS_ERR_BAD_ARG, "null scene");
    if (min_blocks != 8 && min_blocks != 7 && min_blocks != 4)
        return fail(YS_ERR_BAD_ARG, "fused variant: CTAs per SM must be 8, 7 or 4");
    s->fused_min_blocks = min_blocks;
    for (auto& v : s->cls_variant) v = min_blocks;
    drop_graphs(s);
    return YS_OK;
}

ys_status ys_scene_set_thread_order(ys_scene* s, int order) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (order < ORDER_VERTEX || order > ORDER_TILE) return fail(YS_ERR_BAD_ARG, "thread order must be 0, 1 or 2");
    for (auto& o : s->cls_order) o = order;
    drop_graphs(s);
    if ((r = order_layout(s))) return r;
    return compute_order(s);
}

// Time every k_fused variant on the current state (the kernel only writes the
// next-state buffers, which the next substep overwrites; the running totals
// are restored) and keep the fastest.  The scene does not advance.
ys_status ys_scene_autotune(ys_scene* s, uint32_t reps, int* chosen, float* ms_out) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (reps == 0) reps = 5;
    cudaStream_t st = s->stream;
    const bool rec = s->record;
    s->record = false;
    r = refit(s);  // trees of the current positions
    if (r) { s->record = rec; return r; }
    unsigned long long saved[8];
    YS_CK(cudaMemcpyAsync(saved, s->counters.p, sizeof(saved), cudaMemcpyDeviceToHost, st));
    YS_CK(cudaStreamSynchronize(st));
    cudaEvent_t e0, e1;
    YS_CK(cudaEventCreate(&e0));
    YS_CK(cudaEventCreate(&e1));
    const StepArgs A = make_args(s);
    float best = 1e30f;
    int bestV = s->fused_min_blocks;
    for (int i = 0; i < 3; ++i) {
        const int v = FUSED_VARIANTS[i];
        launch_fused(A, st, v);  // warm-up
        float t = 0.f;
        for (u32 k = 0; k < reps; ++k) {
            cudaEventRecord(e0, st);
            launch_fused(A, st, v);
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            t += ms;
        }
        t /= (float)reps;
        if (ms_out) ms_out[i] = t;
        if (t < best) { best = t; bestV = v; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    YS_CK(cudaGetLastError());
    YS_CK(cudaMemcpyAsync(s->counters.p, saved, sizeof(saved), cudaMemcpyHostToDevice, st));
    YS_CK(cudaStreamSynchronize(st));
    s->record = rec;
    s->fused_min_blocks = bestV;
    for (auto& v : s->cls_variant) v = bestV;
    drop_graphs(s);
    if (chosen) *chosen = bestV;
    return YS_OK;
}

// Per size class: time each register-cap variant under each thread order on
// the current state (the kernel writes only the next-state buffers; the
// running totals are restored) and keep the fastest pair for the class.
ys_status ys_scene_autotune_classes(ys_scene* s, uint32_t reps, ys_fused_class* out, uint32_t cap,
                                    uint32_t* nclasses) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (reps == 0) reps = 5;
    cudaStream_t st = s->stream;
    const bool rec = s->record;
    s->record = false;
    r = refit(s);
    if (r) { s->record = rec; return r; }
    unsigned long long saved[8];
    YS_CK(cudaMemcpyAsync(saved, s->counters.p, sizeof(saved), cudaMemcpyDeviceToHost, st));
    YS_CK(cudaStreamSynchronize(st));
    cudaEvent_t e0, e1;
    YS_CK(cudaEventCreate(&e0));
    YS_CK(cudaEventCreate(&e1));
    float ms[NCLASS][3][3] = {};
    for (int order = ORDER_VERTEX; order <= ORDER_TILE && !r; ++order) {
        for (auto& o : s->cls_order) o = order;
        if ((r = order_layout(s)) || (r = compute_order(s))) break;
        StepArgs A = make_args(s);
        A.tiles = order == ORDER_TILE ? 1u : 0u;
        for (int c = 0; c < NCLASS; ++c) {
            A.tbase = s->cls_off[c];
            A.tend = s->cls_off[c + 1];
            if (A.tend <= A.tbase) continue;
            for (int i = 0; i < 3; ++i) {
                launch_fused(A, st, FUSED_VARIANTS[i]);  // warm-up
                float t = 0.f;
                for (u32 k = 0; k < reps; ++k) {
                    cudaEventRecord(e0, st);
                    launch_fused(A, st, FUSED_VARIANTS[i]);
                    cudaEventRecord(e1, st);
                    cudaEventSynchronize(e1);
                    float m = 0.f;
                    cudaEventElapsedTime(&m, e0, e1);
                    t += m;
                }
                ms[c][order][i] = t / (float)reps;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!r) {
        for (int c = 0; c < NCLASS; ++c) {
            if (s->cls_off[c + 1] <= s->cls_off[c]) continue;
            int bo = ORDER_MORTON, bi = 0;
            for (int o = ORDER_VERTEX; o <= ORDER_TILE; ++o)
                for (int i = 0; i < 3; ++i)
                    if (ms[c][o][i] < ms[c][bo][bi]) { bo = o; bi = i; }
            s->cls_order[c] = bo;
            s->cls_variant[c] = FUSED_VARIANTS[bi];
        }
        if (!(r = order_layout(s))) r = compute_order(s);
    }
    YS_CK(cudaGetLastError());
    YS_CK(cudaMemcpyAsync(s->counters.p, saved, sizeof(saved), cudaMemcpyHostToDevice, st));
    YS_CK(cudaStreamSynchronize(st));
    s->record = rec;
    drop_graphs(s);
    if (r) return r;
    if (nclasses) *nclasses = NCLASS;
    for (int c = 0; c < NCLASS && out && (u32)c < cap; ++c) {
        ys_fused_class& o = out[c];
        memset(&o, 0, sizeof(o));
        o.max_mesh_vertices = CLASS_MAX[c];
        o.meshes = s->cls_meshes[c];
        for (size_t m = 0; m < s->meshes.size(); ++m)
            if (s->mesh_class[m] == c) o.vertices += s->meshes[m].d.num_vertices;
        o.ctas_per_sm = s->cls_variant[c];
        o.thread_order = s->cls_order[c];
        for (int k = 0; k < 3; ++k)
            for (int i = 0; i < 3; ++i) o.ms[k][i] = ms[c][k][i];
    }
    return YS_OK;
}

ys_status ys_scene_set_graphs(ys_scene* s, int on) {
    if (!s) return fail(YS_ERR_BAD_ARG, "null scene");
    s->use_graphs = on != 0;
    if (!s->use_graphs) drop_graphs(s);
    return YS_OK;
}

ys_status ys_scene_sync(ys_scene* s) {
    if (!s) return fail(YS_ERR_BAD_ARG, "null scene");
    YS_CK(cudaStreamSynchronize(s->stream));
    return YS_OK;
}

ys_status ys_scene_stream(ys_scene* s, void** out) {
    if (!s || !out) return fail(YS_ERR_BAD_ARG, "null argument");
    *out = (void*)s->stream;
    return YS_OK;
}

ys_status ys_scene_get_state(ys_scene* s, int which, float* out) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (!out) return fail(YS_ERR_BAD_ARG, "null output");
    const float4* src = nullptr;
    if (which == 0) src = s->X[s->cur].p;
    else if (which == 1) src = s->V[s->cv].p;
    else if (which == 2) src = s->snapshot_pending ? s->X[s->cur].p : s->X[s->prev].p;
    else if (which == 3) { r = ensure_staged(s); if (r) return r; src = s->Fbuf.p; }
    else return fail(YS_ERR_BAD_ARG, "bad state id");
    DBuf<float> tmp;
    YS_CK(tmp.alloc(3 * (size_t)s->nV));
    k_unpack4<<<ceil_div(s->nV, 256), 256, 0, s->stream>>>(src, tmp.p, s->nV);
    YS_CK(cudaMemcpyAsync(out, tmp.p, 12 * (size_t)s->nV, cudaMemcpyDeviceToHost, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));
    tmp.free();
    return YS_OK;
}

ys_status ys_scene_set_state(ys_scene* s, int which, const float* in) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (!in) return fail(YS_ERR_BAD_ARG, "null input");
    DBuf<float> tmp;
    YS_CK(tmp.alloc(3 * (size_t)s->nV));
    YS_CK(cudaMemcpyAsync(tmp.p, in, 12 * (size_t)s->nV, cudaMemcpyHostToDevice, s->stream));
    if (which == 0) k_pack4<<<ceil_div(s->nV, 256), 256, 0, s->stream>>>(tmp.p, s->X[s->cur].p, s->nV);
    else if (which == 1) k_pack4<<<ceil_div(s->nV, 256), 256, 0, s->stream>>>(tmp.p, s->V[s->cv].p, s->nV);
    else if (which == 2) k_pack4<<<ceil_div(s->nV, 256), 256, 0, s->stream>>>(tmp.p, s->X[s->prev].p, s->nV);
    else { tmp.free(); return fail(YS_ERR_BAD_ARG, "bad state id"); }
    // vertices of static meshes are never rewritten by a substep, so every
    // rotating buffer must hold the same values for them
    if (which == 0 || which == 1)
        for (auto& H : s->meshes) {
            if (!(H.flags & MF_STATIC)) continue;
            const size_t bytes = sizeof(float4) * H.d.num_vertices;
            if (which == 0) {
                for (int b = 0; b < 3; ++b)
                    if (b != s->cur)
                        YS_CK(cudaMemcpyAsync(s->X[b].p + H.voff, s->X[s->cur].p + H.voff, bytes,
                                              cudaMemcpyDeviceToDevice, s->stream));
            } else {
                YS_CK(cudaMemcpyAsync(s->V[1 - s->cv].p + H.voff, s->V[s->cv].p + H.voff, bytes,
                                      cudaMemcpyDeviceToDevice, s->stream));
            }
        }
    YS_CK(cudaStreamSynchronize(s->stream));
    tmp.free();
    return YS_OK;
}

ys_status ys_scene_stats(ys_scene* s, uint64_t out[8]) {
    ys_status r = check_scene(s);
    if (r) return r;
    unsigned long long cnt[3];
    u32 st;
    YS_CK(cudaMemcpyAsync(cnt, s->counters.p, 24, cudaMemcpyDeviceToHost, s->stream));
    YS_CK(cudaMemcpyAsync(&st, s->status.p, 4, cudaMemcpyDeviceToHost, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));
    out[0] = s->frame;
    out[1] = s->cursor;
    out[2] = cnt[0];
    out[3] = cnt[1];
    out[4] = (st & ST_NONFINITE) ? 1 : 0;
    if (cnt[0] > s->cap || cnt[1] > s->cap) st |= ST_PAIR_OVF;
    out[5] = st;
    out[6] = s->nV;
    out[7] = s->substeps_run;
    return YS_OK;
}

ys_status ys_scene_set_external_forces(ys_scene* s, const float* host_ext) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (!host_ext) {
        if (s->use_ext) drop_graphs(s);
        s->use_ext = false;
        return YS_OK;
    }
    if (!s->use_ext) drop_graphs(s);  // captured graphs read g * m, not the buffer
    if (!s->ext.p) {
        YS_CK(s->ext.alloc(s->nV));
        YS_CK(s->scratch3.alloc(3 * (size_t)s->nV));
    }
    YS_CK(cudaMemcpyAsync(s->scratch3.p, host_ext, 12 * (size_t)s->nV, cudaMemcpyHostToDevice, s->stream));
    k_pack4<<<ceil_div(s->nV, 256), 256, 0, s->stream>>>(s->scratch3.p, s->ext.p, s->nV);
    YS_CK(cudaGetLastError());
    s->use_ext = true;
    return YS_OK;
}

ys_status ys_scene_read_positions_async(ys_scene* s, float* host_out) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (!host_out) return fail(YS_ERR_BAD_ARG, "null output");
    if (!s->scratch3.p) YS_CK(s->scratch3.alloc(3 * (size_t)s->nV));
    k_unpack4<<<ceil_div(s->nV, 256), 256, 0, s->stream>>>(s->X[s->cur].p, s->scratch3.p, s->nV);
    YS_CK(cudaMemcpyAsync(host_out, s->scratch3.p, 12 * (size_t)s->nV, cudaMemcpyDeviceToHost, s->stream));
    return YS_OK;
}

ys_status ys_scene_set_timing(ys_scene* s, int on) {
    ys_status r = check_scene(s);
    if (r) return r;
    YS_CK(cudaStreamSynchronize(s->stream));
    s->timing = on != 0;
    s->evUsed = 0;
    s->evRefit.clear();
    s->evFused.clear();
    return YS_OK;
}

ys_status ys_scene_kernel_times(ys_scene* s, double out[4]) {
    ys_status r = check_scene(s);
    if (r) return r;
    YS_CK(cudaStreamSynchronize(s->stream));
    double tr = 0, tf = 0;
    for (size_t i : s->evRefit) { float ms; YS_CK(cudaEventElapsedTime(&ms, s->evPool[i], s->evPool[i + 1])); tr += ms; }
    for (size_t i : s->evFused) { float ms; YS_CK(cudaEventElapsedTime(&ms, s->evPool[i], s->evPool[i + 1])); tf += ms; }
    out[0] = tr; out[1] = (double)s->evRefit.size(); out[2] = tf; out[3] = (double)s->evFused.size();
    return YS_OK;
}

ys_status ys_scene_totals(ys_scene* s, uint64_t out[2]) {
    ys_status r = check_scene(s);
    if (r) return r;
    unsigned long long c[2];
    YS_CK(cudaMemcpyAsync(c, s->counters.p + 3, 16, cudaMemcpyDeviceToHost, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));
    out[0] = c[0]; out[1] = c[1];
    return YS_OK;
}

ys_status ys_scene_clear_flags(ys_scene* s) {
    ys_status r = check_scene(s);
    if (r) return r;
    YS_CK(cudaMemsetAsync(s->status.p, 0, 4, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));
    return YS_OK;
}

ys_status ys_scene_rows(ys_scene* s, void* out, uint64_t cap, uint64_t* n_out) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (!s->staged_ready) { if (n_out) *n_out = 0; return YS_OK; }
    unsigned long long cnt;
    YS_CK(cudaMemcpyAsync(&cnt, s->counters.p, 8, cudaMemcpyDeviceToHost, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));
    uint64_t n = std::min<uint64_t>(cnt, s->cap);
    if (n_out) *n_out = n;
    if (out && n) YS_CK(cudaMemcpy(out, s->rows.p, sizeof(Row) * std::min(n, cap), cudaMemcpyDeviceToHost));
    return YS_OK;
}

ys_status ys_scene_contacts(ys_scene* s, uint32_t* off, void* out, uint64_t cap, uint64_t* n_out) {
    ys_status r = check_scene(s);
    if (r) return r;
    YS_CK(cudaStreamSynchronize(s->stream));
    if (s->last_contacts == 1) {
        std::vector<u32> o(s->nV + 1);
        YS_CK(cudaMemcpy(o.data(), s->csr_off.p, 4 * (size_t)(s->nV + 1), cudaMemcpyDeviceToHost));
        uint64_t n = o[s->nV];
        if (n_out) *n_out = n;
        if (off) memcpy(off, o.data(), 4 * (size_t)(s->nV + 1));
        if (out && n) YS_CK(cudaMemcpy(out, s->csr.p, sizeof(VContact) * std::min(n, cap), cudaMemcpyDeviceToHost));
        return YS_OK;
    }
    if (s->last_contacts == 2) {
        std::vector<u32> vs(s->nV), vc(s->nV);
        YS_CK(cudaMemcpy(vs.data(), s->vstart.p, 4 * (size_t)s->nV, cudaMemcpyDeviceToHost));
        YS_CK(cudaMemcpy(vc.data(), s->vcount.p, 4 * (size_t)s->nV, cudaMemcpyDeviceToHost));
        unsigned long long fill;
        YS_CK(cudaMemcpy(&fill, s->counters.p + 2, 8, cudaMemcpyDeviceToHost));
        std::vector<VContact> pool(std::min<unsigned long long>(fill, s->cap));
        if (!pool.empty()) YS_CK(cudaMemcpy(pool.data(), s->pool.p, sizeof(VContact) * pool.size(), cudaMemcpyDeviceToHost));
        std::vector<u32> o(s->nV + 1, 0);
        for (u32 g = 0; g < s->nV; ++g) o[g + 1] = o[g] + vc[g];
        uint64_t n = o[s->nV];
        if (n_out) *n_out = n;
        if (off) memcpy(off, o.data(), 4 * (size_t)(s->nV + 1));
        if (out) {
            VContact* dst = (VContact*)out;
            for (u32 g = 0; g < s->nV; ++g)
                for (u32 k = 0; k < vc[g]; ++k)
                    if (o[g] + k < cap) dst[o[g] + k] = pool[vs[g] + k];
        }
        return YS_OK;
    }
    if (n_out) *n_out = 0;
    if (off) memset(off, 0, 4 * (size_t)(s->nV + 1));
    return YS_OK;
}

ys_status ys_scene_wide_tree(ys_scene* s, int mesh, void* out, uint32_t cap, uint32_t* count) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (mesh < 0 || (size_t)mesh >= s->meshes.size()) return fail(YS_ERR_BAD_ARG, "bad mesh index");
    if (!count) return fail(YS_ERR_BAD_ARG, "null count");
    *count = 0;
    HostMesh& H = s->meshes[mesh];
    if (s->tree_layout != YS_TREE_CUBE || !H.built || H.d.num_facets == 0) return YS_OK;
    u32 n = 0;
    YS_CK(cudaMemcpyAsync(&n, s->wcount.p + mesh, 4, cudaMemcpyDeviceToHost, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));
    *count = n;
    if (out && cap)
        YS_CK(cudaMemcpyAsync(out, s->w4.p + H.w4_off, sizeof(Wide4) * std::min(n, cap), cudaMemcpyDeviceToHost,
                              s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));
    return YS_OK;
}

ys_status ys_scene_tree(ys_scene* s, int mesh, void* nodes, int32_t* parent, uint32_t* codes, uint32_t* idx,
                        uint32_t* nprims) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (mesh < 0 || (size_t)mesh >= s->meshes.size()) return fail(YS_ERR_BAD_ARG, "bad mesh index");
    HostMesh& H = s->meshes[mesh];
    const u32 n = H.d.num_facets;
    if (nprims) *nprims = n;
    YS_CK(cudaStreamSynchronize(s->stream));
    if (n == 0) return YS_OK;
    if (!H.built) {  // a tree no query descends is built only when inspected
        r = build_tree(s, H);
        if (r) return r;
    }
    const size_t nn = 2 * (size_t)n - 1;
    if (nodes && s->tree_layout == YS_TREE_CUBE) {
        // the cube layout refits the wide form only; give the binary form the
        // boxes of a refit from the current state (swept for moving meshes)
        RefitJob J;
        memset(&J, 0, sizeof(J));
        J.nodes = s->nodes.p + H.node_off;
        J.parent = s->parent.p + H.node_off;
        J.claimOff = claim_off(s, H);
    J.claims = s->claims.p + H.node_off;
        J.visits = s->visits.p + H.foff;
        J.facets = s->F3.p + 3 * (size_t)H.foff;
        J.x4 = s->X[s->cur].p;
        J.v4 = s->V[s->cv].p;
        J.voff = H.voff;
        J.n = n;
        J.dt = s->P.subh;
        J.swept = (H.flags & MF_STATIC) ? 0u : 1u;
        J.maxExt = s->maxext.p;  // unused (selfMargin == 0)
        RefitJob* slot = s->jobs.p + 6 * (size_t)s->njobs;
        YS_CK(cudaMemcpyAsync(slot, &J, sizeof(J), cudaMemcpyHostToDevice, s->stream));
        launch_refit(slot, 1, n, s->status.p, s->stream);
        YS_CK(cudaStreamSynchronize(s->stream));
    }
    if (nodes) YS_CK(cudaMemcpy(nodes, s->nodes.p + H.node_off, 32 * nn, cudaMemcpyDeviceToHost));
    if (parent) YS_CK(cudaMemcpy(parent, s->parent.p + H.node_off, 4 * nn, cudaMemcpyDeviceToHost));
    if (codes) YS_CK(cudaMemcpy(codes, s->codes.p + H.foff, 4 * (size_t)n, cudaMemcpyDeviceToHost));
    if (idx) YS_CK(cudaMemcpy(idx, s->idx.p + H.foff, 4 * (size_t)n, cudaMemcpyDeviceToHost));
    return YS_OK;
}

}  // extern "C"

// =====================================================================
// Adjoint of the substep for one FastGridCloth (differentiable rollouts).
//
// Forward step of the cloth (the fused substep's arithmetic):
//   f_i = ext_i + kair v_i + sum_s (k_s (l - L_s) + kd (dv . n)) n
//   v'  = v + (subh f / m) mask;  for each contact (n_c, d_c) with d_c < thickness:
//         { if v'.n_c < 0: v' -= (v'.n_c) n_c;  x += (thickness - d_c) n_c }
//   x'  = x + subh v' mask
// Reverse step with the forward's active set frozen (which contacts exist,
// push and project): the contact push is x -> x + (t - n.(x - t0)) n, so its
// transpose removes the normal component; the projections are symmetric and
// are undone in reverse order; the spring force's Jacobian is
//   dF/d(dx)^T g = (k n + kd (I - nn^T) dv / l)(n.g) + a/l (I - nn^T) g,
//   dF/d(dv)^T g = kd n (n.g),  dF/dk = (l - L) n,  dF/dL = -k n.
// Checkpoints of the whole scene state every K steps; the backward pass
// replays one segment at a time (recording its contacts and states) and
// reverses it.
namespace ys {

struct AdjArgs {
    const float4* x;   // scene positions at step t (all vertices)
    const float4* v;   // velocities at step t
    const u32* vstart; const u32* vcount; const VContact* pool;  // contacts recorded at step t
    const float4* ax;  // dL/dx_{t+1} (all vertices; only the mesh's are used)
    const float4* av;  // dL/dv_{t+1}
    float4* xbar; float4* vbar; float4* fbar;
    float4* ax_out; float4* av_out;
    float* gk; float* gL;  // per-spring accumulators (this mesh's arrays)
    u32 voff, nV, N;
};

__global__ void __launch_bounds__(128) k_adj_vertex(StepArgs A, AdjArgs J, u32 m) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= J.nV) return;
    const u32 g = J.voff + i;
    const MeshDev M = A.meshes[m];
    const f3 x = ld(J.x, g);
    f3 vel = ld(J.v, g);
    const float mass = A.mass[g], mask = A.mask[g];
    const f3 force = vertex_force(A, M, g, x, vel, mass);
    vel = vel + ((force * A.subh) / mass) * mask;
    // replay the contact loop of contact_response to freeze its active set
    const u32 b = J.vstart[g], nc = J.vcount[g];
    u32 proj = 0, push = 0;  // bit c: contact c projected the velocity / pushed the position
    for (u32 c = 0; c < nc && c < 32; ++c) {
        const VContact ci = J.pool[b + c];
        bool dup = false;
        for (u32 d = 0; d < c; ++d) {
            const VContact cd = J.pool[b + d];
            if (cd.tobj == ci.tobj && cd.tri == ci.tri) { dup = true; break; }
        }
        if (dup) continue;
        f3 n = mk(ci.nx, ci.ny, ci.nz);
        float nl2 = dot(n, n);
        if (nl2 < 1e-12f) continue;
        n = n * (1.0f / sqrtf(nl2));
        float vn = dot(vel, n);
        if (ci.d < M.thickness) {
            if (vn < 0.0f) { vel = vel - n * vn; proj |= 1u << c; }
            push |= 1u << c;
        }
    }
    const f3 axi = ld(J.ax, g);
    f3 vb = ld(J.av, g) + axi * (A.subh * mask);
    for (int c = (int)(nc < 32 ? nc : 32) - 1; c >= 0; --c) {
        if (!(proj >> c & 1u)) continue;
        const VContact ci = J.pool[b + c];
        f3 n = mk(ci.nx, ci.ny, ci.nz);
        n = n * (1.0f / sqrtf(dot(n, n)));
        vb = vb - n * dot(n, vb);
    }
    f3 xb = axi;
    for (u32 c = 0; c < nc && c < 32; ++c) {
        if (!(push >> c & 1u)) continue;
        const VContact ci = J.pool[b + c];
        f3 n = mk(ci.nx, ci.ny, ci.nz);
        n = n * (1.0f / sqrtf(dot(n, n)));
        xb = xb - n * dot(n, axi);
    }
    const f3 fb = vb * ((A.subh / mass) * mask);
    J.xbar[g] = make_float4(xb.x, xb.y, xb.z, 0.f);
    J.vbar[g] = make_float4(vb.x, vb.y, vb.z, 0.f);
    J.fbar[g] = make_float4(fb.x, fb.y, fb.z, 0.f);
}

__global__ void __launch_bounds__(128) k_adj_springs(StepArgs A, AdjArgs J, u32 m) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= J.nV) return;
    const u32 g = J.voff + i;
    const MeshDev M = A.meshes[m];
    const int N = (int)J.N, row = (int)(i / J.N), col = (int)(i % J.N);
    const f3 p = ld(J.x, g), w = ld(J.v, g), fi = ld(J.fbar, g);
    const float kd = A.kd;
    f3 dxb = mk(0.f, 0.f, 0.f), dvb = mk(0.f, 0.f, 0.f);
    grid_stencil(N, row, col, [&](int r, int c, int fam, u32 sid) {
        float k, rest;
        grid_spring_kL(A, M, fam, sid, k, rest);
        const u32 jl = (u32)(r * N + c), j = J.voff + jl;
        const f3 dx = ld(J.x, j) - p, dv = ld(J.v, j) - w;
        const float l = sqrtf(dot(dx, dx));
        if (l < 1e-7f) return;
        const f3 nd = dx / l;
        const float a = k * (l - rest) + kd * dot(dv, nd);
        const f3 gdir = fi - ld(J.fbar, j);
        const float ng = dot(nd, gdir);
        const f3 dvp = dv - nd * dot(nd, dv), gp = gdir - nd * ng;
        const f3 ddx = nd * (k * ng) + dvp * (kd * ng / l) + gp * (a / l);
        dxb = dxb - ddx;
        dvb = dvb - nd * (kd * ng);
        if (i < jl) {  // one owner per spring: no race on the accumulators
            J.gk[sid] += (l - rest) * ng;
            J.gL[sid] += -k * ng;
        }
    });
    const f3 xb = ld(J.xbar, g) + dxb;
    const f3 vb = ld(J.vbar, g) + dvb + fi * A.kair;
    J.ax_out[g] = make_float4(xb.x, xb.y, xb.z, 0.f);
    J.av_out[g] = make_float4(vb.x, vb.y, vb.z, 0.f);
}

__global__ void k_mesh_pack4(const float* __restrict__ in, float4* __restrict__ out, u32 voff, u32 n) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[voff + i] = make_float4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0.f);
}
__global__ void k_mesh_unpack4(const float4* __restrict__ in, float* __restrict__ out, u32 voff, u32 n) {
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { float4 q = in[voff + i]; out[3 * i] = q.x; out[3 * i + 1] = q.y; out[3 * i + 2] = q.z; }
}

}  // namespace ys

#include "ys_adj64.cuh"

struct ys_adjoint {
    ys_scene* s = nullptr;
    int mesh = 0;
    u32 T = 0, K = 0, nseg = 0, nV = 0, voff = 0, S = 0, N = 0;
    // initial scene state and checkpoints (whole-scene arrays)
    DBuf<float4> x0, v0;
    std::vector<DBuf<float4>> ck_x, ck_xp, ck_v;
    std::vector<uint64_t> ck_frame;
    std::vector<u32> ck_cursor;
    // one segment of replayed steps
    std::vector<DBuf<float4>> st_x, st_v;
    std::vector<DBuf<u32>> st_vstart, st_vcount;
    std::vector<DBuf<VContact>> st_pool;
    DBuf<float4> ax, av, ax2, av2, xbar, vbar, fbar;
    bool forward_done = false;
    // 64-bit mode (ys_adjoint_set_precision): the cloth's state in binary64
    // (local vertex index), the parameters, checkpoints, one segment of
    // recorded steps (states and sorted contacts), the reverse-pass buffers
    int bits = 32;
    DBuf<D4> d_x0, d_v0;
    DBuf<double> d_k, d_L;
    std::vector<DBuf<D4>> dck_x, dck_xp, dck_v, dst_x, dst_v;
    std::vector<DBuf<DContact>> dst_c;
    std::vector<DBuf<u32>> dst_f, dst_n;
    DBuf<D4> dX[3], dV[2];
    DBuf<DContact> dsc_c;  // contacts of steps that are not recorded
    DBuf<DContact> dls;    // contact search output per (vertex, search thread)
    DBuf<u32> dlf, dlk, dln;
    DBuf<u32> dsc_f, dsc_n;
    DBuf<D4> dax, dav, dax2, dav2, dxbar, dvbar, dfbar;
    DBuf<double> dgk, dgL;
    DBuf<unsigned long long> dbox;
    DBuf<u32> dstatus;
    cudaGraphExec_t g_fwd = nullptr, g_bwd = nullptr;  // the two passes, captured on first use
    const D4* g_fwd_xT = nullptr;                      // buffer holding x_T after the forward graph
    const D4* g_bwd_av = nullptr;                      // buffer holding dL/dv0 after the backward graph
    A64 g_args;                                        // the scene-derived arguments the graphs hold
};

namespace {

void restore_state(ys_scene* s, const float4* x, const float4* xp, const float4* v, uint64_t frame, u32 cursor) {
    const size_t bytes = sizeof(float4) * s->nV;
    cudaMemcpyAsync(s->X[s->cur].p, x, bytes, cudaMemcpyDeviceToDevice, s->stream);
    cudaMemcpyAsync(s->X[s->prev].p, xp, bytes, cudaMemcpyDeviceToDevice, s->stream);
    cudaMemcpyAsync(s->V[s->cv].p, v, bytes, cudaMemcpyDeviceToDevice, s->stream);
    // vertices that no substep rewrites keep one value in every buffer
    const int third = 3 - s->cur - s->prev;
    cudaMemcpyAsync(s->X[third].p, x, bytes, cudaMemcpyDeviceToDevice, s->stream);
    cudaMemcpyAsync(s->V[1 - s->cv].p, v, bytes, cudaMemcpyDeviceToDevice, s->stream);
    s->frame = frame;
    s->cursor = cursor;
    s->snapshot_pending = false;
}

// ---- 64-bit mode
void d64_drop_graphs(ys_adjoint* a);

void d64_free(ys_adjoint* a) {
    d64_drop_graphs(a);
    for (auto* v : {&a->dck_x, &a->dck_xp, &a->dck_v, &a->dst_x, &a->dst_v}) {
        for (auto& b : *v) b.free();
        v->clear();
    }
    for (auto& b : a->dst_c) b.free();
    for (auto& b : a->dst_f) b.free();
    for (auto& b : a->dst_n) b.free();
    a->dst_c.clear(); a->dst_f.clear(); a->dst_n.clear();
    for (auto* b : {&a->d_x0, &a->d_v0, &a->dX[0], &a->dX[1], &a->dX[2], &a->dV[0], &a->dV[1], &a->dax, &a->dav,
                    &a->dax2, &a->dav2, &a->dxbar, &a->dvbar, &a->dfbar})
        b->free();
    a->d_k.free(); a->d_L.free(); a->dgk.free(); a->dgL.free();
    a->dsc_c.free(); a->dsc_f.free(); a->dsc_n.free(); a->dbox.free(); a->dstatus.free();
    a->dls.free(); a->dlf.free(); a->dlk.free(); a->dln.free();
}

cudaError_t d64_alloc(ys_adjoint* a) {
    const size_t n = a->nV, c = (size_t)a->nV * D64_CAP;
    cudaError_t e;
    for (auto* b : {&a->d_x0, &a->d_v0, &a->dX[0], &a->dX[1], &a->dX[2], &a->dV[0], &a->dV[1], &a->dax, &a->dav,
                    &a->dax2, &a->dav2, &a->dxbar, &a->dvbar, &a->dfbar})
        if ((e = b->alloc(n))) return e;
    if ((e = a->d_k.alloc(a->S)) || (e = a->d_L.alloc(a->S)) || (e = a->dgk.alloc(a->S)) || (e = a->dgL.alloc(a->S)))
        return e;
    const size_t nl = n * D64_LANES, cl = nl * D64_LCAP;
    if ((e = a->dls.alloc(cl)) || (e = a->dlf.alloc(cl)) || (e = a->dlk.alloc(cl)) || (e = a->dln.alloc(nl))) return e;
    if ((e = a->dsc_c.alloc(c)) || (e = a->dsc_f.alloc(c)) || (e = a->dsc_n.alloc(n)) || (e = a->dbox.alloc(6)) ||
        (e = a->dstatus.alloc(1)))
        return e;
    a->dck_x.resize(a->nseg); a->dck_xp.resize(a->nseg); a->dck_v.resize(a->nseg);
    for (u32 i = 0; i < a->nseg; ++i)
        if ((e = a->dck_x[i].alloc(n)) || (e = a->dck_xp[i].alloc(n)) || (e = a->dck_v[i].alloc(n))) return e;
    a->dst_x.resize(a->K); a->dst_v.resize(a->K); a->dst_c.resize(a->K); a->dst_f.resize(a->K); a->dst_n.resize(a->K);
    for (u32 i = 0; i < a->K; ++i)
        if ((e = a->dst_x[i].alloc(n)) || (e = a->dst_v[i].alloc(n)) || (e = a->dst_c[i].alloc(c)) ||
            (e = a->dst_f[i].alloc(c)) || (e = a->dst_n[i].alloc(n)))
            return e;
    return cudaSuccess;
}

// The per-spring parameters the float path would use, widened: the mesh's
// per-spring arrays once set, else FastGridClothBehaviorParams' per-family
// stiffness and rest length.
ys_status d64_params_from_scene(ys_adjoint* a) {
    ys_scene* s = a->s;
    const HostMesh& H = s->meshes[a->mesh];
    const MeshDev& M = s->hmeshes[a->mesh];
    cudaStream_t st = s->stream;
    if (H.grid_springs_on) {
        k_d64_widen<<<ceil_div(a->S, 256), 256, 0, st>>>(s->gk.p + M.gspr, a->d_k.p, a->S);
        k_d64_widen<<<ceil_div(a->S, 256), 256, 0, st>>>(s->gL.p + M.gspr, a->d_L.p, a->S);
        YS_CK(cudaGetLastError());
        return YS_OK;
    }
    const size_t n = a->N;
    const size_t cnt[6] = {n * (n - 1), (n - 1) * n, (n - 1) * (n - 1), (n - 1) * (n - 1), n * (n - 2), (n - 2) * n};
    const float kf[6] = {M.kstretch, M.kstretch, M.kshear, M.kshear, M.kbend, M.kbend};
    std::vector<double> k, L;
    k.reserve(a->S); L.reserve(a->S);
    for (int f = 0; f < 6; ++f) {
        k.insert(k.end(), cnt[f], (double)kf[f]);
        L.insert(L.end(), cnt[f], (double)M.rest[f]);
    }
    YS_CK(cudaMemcpyAsync(a->d_k.p, k.data(), 8 * (size_t)a->S, cudaMemcpyHostToDevice, st));
    YS_CK(cudaMemcpyAsync(a->d_L.p, L.data(), 8 * (size_t)a->S, cudaMemcpyHostToDevice, st));
    YS_CK(cudaStreamSynchronize(st));  // k, L live on the host stack
    return YS_OK;
}

// Trees of the obstacles the cloth queries (built on first use).
ys_status d64_trees(ys_adjoint* a) {
    ys_scene* s = a->s;
    bool any = false;
    for (size_t m = 0; m < s->meshes.size(); ++m) {
        HostMesh& H = s->meshes[m];
        if ((int)m == a->mesh || H.built || !H.needs_tree || H.d.num_facets == 0) continue;
        ys_status r = build_tree(s, H);
        if (r) return r;
        any = true;
    }
    return any ? build_levels(s) : YS_OK;
}

A64 d64_args(ys_adjoint* a) {
    ys_scene* s = a->s;
    const MeshDev& M = s->hmeshes[a->mesh];
    A64 A;
    memset(&A, 0, sizeof(A));
    A.sx = s->X[s->cur].p;
    A.F = s->F4.p;
    A.nodes = s->nodes.p;
    A.meshes = s->dmeshes.p;
    A.targets = s->targets.p;
    A.ext = s->use_ext ? s->ext.p : nullptr;
    A.mass = s->mass.p;
    A.mask = s->mask.p;
    A.tgt_begin = M.tgt_begin;
    A.tgt_end = M.tgt_end;
    A.cloth = (u32)a->mesh;
    A.voff = a->voff;
    A.nV = a->nV;
    A.N = a->N;
    A.gx = s->P.gravity[0]; A.gy = s->P.gravity[1]; A.gz = s->P.gravity[2];
    A.kair = s->P.kair; A.kd = s->P.kd; A.subh = s->P.subh;
    A.thickness = M.thickness;
    A.margin = s->P.margin;
    A.radius = s->P.radius;
    A.k = a->d_k.p;
    A.L = a->d_L.p;
    A.box = a->dbox.p;
    A.status = a->dstatus.p;
    A.ls = a->dls.p;
    A.lf = a->dlf.p;
    A.lk = a->dlk.p;
    A.ln = a->dln.p;
    return A;
}

void d64_step(ys_adjoint* a, A64 A, cudaStream_t st) {
    cudaMemsetAsync(a->dbox.p, 0, 6 * sizeof(unsigned long long), st);
    const u32 gb = std::min<u32>(ceil_div(a->nV, 256), 148 * 4);
    k_d64_box<<<gb, 256, 0, st>>>(A);
    k_d64_cand<<<ceil_div(a->nV * D64_LANES, D64_BLOCK), D64_BLOCK, 0, st>>>(A);
    k_d64_step<<<ceil_div(a->nV, D64_BLOCK), D64_BLOCK, 0, st>>>(A);
}

ys_status d64_status(ys_adjoint* a) {
    u32 f = 0;
    YS_CK(cudaMemcpyAsync(&f, a->dstatus.p, 4, cudaMemcpyDeviceToHost, a->s->stream));
    YS_CK(cudaStreamSynchronize(a->s->stream));
    if (f & YS_FLAG_CONTACT_OVF) return fail(YS_ERR_CAPACITY, "FP64 rollout: more than 16 contacts at a vertex");
    if (f & YS_FLAG_STACK_OVF) return fail(YS_ERR_CAPACITY, "FP64 rollout: tree descent stack exceeded");
    return YS_OK;
}

// Enqueue the forward rollout in binary64 from (d_x0, d_v0), checkpoints
// every K steps; *xT receives the buffer that will hold x_T.
ys_status d64_enqueue_forward(ys_adjoint* a, const D4** xT) {
    cudaStream_t st = a->s->stream;
    const size_t bytes = sizeof(D4) * a->nV;
    D4 *x = a->dX[0].p, *xp = a->dX[1].p, *xn = a->dX[2].p, *v = a->dV[0].p, *vn = a->dV[1].p;
    YS_CK(cudaMemcpyAsync(x, a->d_x0.p, bytes, cudaMemcpyDeviceToDevice, st));
    YS_CK(cudaMemcpyAsync(xp, a->d_x0.p, bytes, cudaMemcpyDeviceToDevice, st));
    YS_CK(cudaMemcpyAsync(v, a->d_v0.p, bytes, cudaMemcpyDeviceToDevice, st));
    YS_CK(cudaMemsetAsync(a->dstatus.p, 0, 4, st));
    A64 A = d64_args(a);
    A.cs = a->dsc_c.p; A.cf = a->dsc_f.p; A.cn = a->dsc_n.p;
    for (u32 t = 0; t < a->T; ++t) {
        if (t % a->K == 0) {
            const u32 i = t / a->K;
            YS_CK(cudaMemcpyAsync(a->dck_x[i].p, x, bytes, cudaMemcpyDeviceToDevice, st));
            YS_CK(cudaMemcpyAsync(a->dck_xp[i].p, xp, bytes, cudaMemcpyDeviceToDevice, st));
            YS_CK(cudaMemcpyAsync(a->dck_v[i].p, v, bytes, cudaMemcpyDeviceToDevice, st));
        }
        A.x = x; A.xp = xp; A.v = v; A.xn = xn; A.vn = vn;
        d64_step(a, A, st);
        D4* old_xp = xp;
        xp = x; x = xn; xn = old_xp;
        std::swap(v, vn);
    }
    YS_CK(cudaGetLastError());
    *xT = x;
    return YS_OK;
}

// Enqueue the reverse pass in binary64; the seed dL/dx_T is in dax.  Each
// segment is replayed from its checkpoint with its states and contacts
// recorded, then reversed step by step.  The adjoints ping-pong between
// dax / dax2 and dav / dav2; the buffer holding dL/dv0 at the end (fixed by
// T) goes to g_bwd_av, the spring gradients to dgk, dgL.
ys_status d64_enqueue_backward(ys_adjoint* a) {
    cudaStream_t st = a->s->stream;
    const size_t bytes = sizeof(D4) * a->nV;
    D4 *ax = a->dax.p, *ax2 = a->dax2.p, *av = a->dav.p, *av2 = a->dav2.p;
    YS_CK(cudaMemsetAsync(av, 0, bytes, st));
    YS_CK(cudaMemsetAsync(a->dgk.p, 0, 8 * (size_t)a->S, st));
    YS_CK(cudaMemsetAsync(a->dgL.p, 0, 8 * (size_t)a->S, st));
    YS_CK(cudaMemsetAsync(a->dstatus.p, 0, 4, st));
    A64 A = d64_args(a);
    for (int seg = (int)a->nseg - 1; seg >= 0; --seg) {
        const u32 t0 = (u32)seg * a->K, t1 = std::min(a->T, t0 + a->K);
        D4 *xp = a->dX[1].p, *xn = a->dX[2].p, *vn = a->dV[1].p;
        YS_CK(cudaMemcpyAsync(xp, a->dck_xp[seg].p, bytes, cudaMemcpyDeviceToDevice, st));
        YS_CK(cudaMemcpyAsync(a->dst_x[0].p, a->dck_x[seg].p, bytes, cudaMemcpyDeviceToDevice, st));
        YS_CK(cudaMemcpyAsync(a->dst_v[0].p, a->dck_v[seg].p, bytes, cudaMemcpyDeviceToDevice, st));
        for (u32 t = t0; t < t1; ++t) {
            const u32 k = t - t0;
            A.x = a->dst_x[k].p; A.xp = xp; A.v = a->dst_v[k].p;
            // the step's outputs go straight into the next step's record
            const bool last = k + 1 == t1 - t0;
            A.xn = last ? xn : a->dst_x[k + 1].p;
            A.vn = last ? vn : a->dst_v[k + 1].p;
            A.cs = a->dst_c[k].p; A.cf = a->dst_f[k].p; A.cn = a->dst_n[k].p;
            d64_step(a, A, st);
            xp = a->dst_x[k].p;
        }
        for (int t = (int)t1 - 1; t >= (int)t0; --t) {
            const u32 k = (u32)t - t0;
            A.x = a->dst_x[k].p; A.v = a->dst_v[k].p;
            A.cs = a->dst_c[k].p; A.cf = a->dst_f[k].p; A.cn = a->dst_n[k].p;
            J64 J;
            J.ax = ax; J.av = av; J.xbar = a->dxbar.p; J.vbar = a->dvbar.p; J.fbar = a->dfbar.p;
            J.ax_out = ax2; J.av_out = av2; J.gk = a->dgk.p; J.gL = a->dgL.p;
            k_d64_adj_vertex<<<ceil_div(a->nV, D64_BLOCK), D64_BLOCK, 0, st>>>(A, J);
            k_d64_adj_springs<<<ceil_div(a->nV, D64_BLOCK), D64_BLOCK, 0, st>>>(A, J);
            std::swap(ax, ax2);
            std::swap(av, av2);
        }
    }
    YS_CK(cudaGetLastError());
    a->g_bwd_av = av;
    return YS_OK;
}

// One executable graph per direction, captured on first use: the whole
// T-step sequence is fixed by (T, K) and the adjoint's own buffers, so later
// calls replay it without host launch overhead.
template <class Fn>
ys_status d64_graph(ys_adjoint* a, cudaGraphExec_t& exec, Fn&& enqueue) {
    cudaStream_t st = a->s->stream;
    // scene-side arguments (external forces, parameters, buffers) changed
    // since the capture: capture again
    const A64 now = d64_args(a);
    if ((a->g_fwd || a->g_bwd) && memcmp(&now, &a->g_args, sizeof(A64)) != 0) d64_drop_graphs(a);
    a->g_args = now;
    if (!exec) {
        cudaGraph_t g = nullptr;
        YS_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        ys_status er = enqueue();
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        if (er) { if (g) cudaGraphDestroy(g); return er; }
        if (ce != cudaSuccess) return fail(YS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) { exec = nullptr; return fail(YS_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce)); }
    }
    YS_CK(cudaGraphLaunch(exec, st));
    return YS_OK;
}

void d64_drop_graphs(ys_adjoint* a) {
    if (a->g_fwd || a->g_bwd) cudaStreamSynchronize(a->s->stream);
    if (a->g_fwd) cudaGraphExecDestroy(a->g_fwd);
    if (a->g_bwd) cudaGraphExecDestroy(a->g_bwd);
    a->g_fwd = a->g_bwd = nullptr;
}

// Forward rollout in binary64; x_T stays in the returned buffer.
ys_status d64_forward(ys_adjoint* a, const D4** xT) {
    ys_status r = d64_trees(a);
    if (r) return r;
    r = d64_graph(a, a->g_fwd, [&]() { return d64_enqueue_forward(a, &a->g_fwd_xT); });
    if (r) return r;
    r = d64_status(a);
    if (r) return r;
    *xT = a->g_fwd_xT;
    a->forward_done = true;
    return YS_OK;
}

// Reverse pass in binary64; the seed dL/dx_T is in dax on entry, dL/dv0
// in g_bwd_av on return.
ys_status d64_backward(ys_adjoint* a) {
    ys_status r = d64_graph(a, a->g_bwd, [&]() { return d64_enqueue_backward(a); });
    if (r) return r;
    return d64_status(a);
}

}  // namespace

extern "C" {

ys_status ys_scene_set_grid_springs(ys_scene* s, int mesh, const float* d_k, const float* d_L) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (mesh < 0 || (size_t)mesh >= s->meshes.size()) return fail(YS_ERR_BAD_ARG, "bad mesh index");
    HostMesh& H = s->meshes[mesh];
    if (H.d.behavior != YS_FAST_GRID_CLOTH) return fail(YS_ERR_BAD_ARG, "per-spring parameters need a FastGridCloth");
    const u32 n = H.d.grid_n;
    const size_t S = 2 * (size_t)n * (n - 1) + 2 * (size_t)(n - 1) * (n - 1) + 2 * (size_t)n * (n - 2);
    if (!s->gk.p) {
        size_t total = 0;
        for (auto& M : s->meshes)
            if (M.d.behavior == YS_FAST_GRID_CLOTH) {
                const size_t q = M.d.grid_n;
                total += 2 * q * (q - 1) + 2 * (q - 1) * (q - 1) + 2 * q * (q - 2);
            }
        YS_CK(s->gk.alloc(total));
        YS_CK(s->gL.alloc(total));
        size_t off = 0;
        for (size_t m = 0; m < s->meshes.size(); ++m)
            if (s->meshes[m].d.behavior == YS_FAST_GRID_CLOTH) {
                s->hmeshes[m].gspr = (u32)off;
                const size_t q = s->meshes[m].d.grid_n;
                off += 2 * q * (q - 1) + 2 * (q - 1) * (q - 1) + 2 * q * (q - 2);
            }
        // a mesh switches to its per-spring arrays once they are set
    }
    const u32 base = s->hmeshes[mesh].gspr;
    if (d_k) YS_CK(cudaMemcpyAsync(s->gk.p + base, d_k, 4 * S, cudaMemcpyDeviceToDevice, s->stream));
    if (d_L) YS_CK(cudaMemcpyAsync(s->gL.p + base, d_L, 4 * S, cudaMemcpyDeviceToDevice, s->stream));
    std::vector<MeshDev> md = s->hmeshes;
    for (size_t m = 0; m < md.size(); ++m)
        if ((int)m != mesh && md[m].gspr != NO_SPRINGS && !s->meshes[m].grid_springs_on) md[m].gspr = NO_SPRINGS;
    H.grid_springs_on = true;
    YS_CK(cudaMemcpyAsync(s->dmeshes.p, md.data(), sizeof(MeshDev) * md.size(), cudaMemcpyHostToDevice, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));
    drop_graphs(s);
    return YS_OK;
}

ys_status ys_adjoint_create(ys_adjoint** out, ys_scene* s, int mesh, uint32_t steps, uint32_t checkpoint_every) {
    ys_status r = check_scene(s);
    if (r) return r;
    if (!out || steps == 0 || checkpoint_every == 0) return fail(YS_ERR_BAD_ARG, "bad argument");
    if (mesh < 0 || (size_t)mesh >= s->meshes.size()) return fail(YS_ERR_BAD_ARG, "bad mesh index");
    HostMesh& H = s->meshes[mesh];
    if (H.d.behavior != YS_FAST_GRID_CLOTH) return fail(YS_ERR_BAD_ARG, "the adjoint covers FastGridCloth meshes");
    for (size_t m = 0; m < s->meshes.size(); ++m)
        if ((int)m != mesh && (s->meshes[m].flags & MF_CLOTH))
            return fail(YS_ERR_BAD_ARG, "the adjoint scene holds one cloth (obstacles are static)");
    if (s->P.self_mode != YS_SELF_OFF) return fail(YS_ERR_BAD_ARG, "the adjoint needs self-collision off");
    if (!s->shape_mesh.empty())
        return fail(YS_ERR_BAD_ARG, "the adjoint differentiates triangle obstacles, not analytic colliders");
    ys_adjoint* a = new ys_adjoint();
    a->s = s; a->mesh = mesh; a->T = steps; a->K = checkpoint_every;
    a->nseg = (steps + checkpoint_every - 1) / checkpoint_every;
    a->nV = H.d.num_vertices; a->voff = H.voff; a->N = H.d.grid_n;
    const u32 n = a->N;
    a->S = 2 * n * (n - 1) + 2 * (n - 1) * (n - 1) + 2 * n * (n - 2);
    auto fail_free = [&](cudaError_t e) { delete a; return fail(YS_ERR_CUDA, cudaGetErrorString(e)); };
    cudaError_t e;
    if ((e = a->x0.alloc(s->nV)) || (e = a->v0.alloc(s->nV))) return fail_free(e);
    a->ck_x.resize(a->nseg); a->ck_xp.resize(a->nseg); a->ck_v.resize(a->nseg);
    a->ck_frame.resize(a->nseg); a->ck_cursor.resize(a->nseg);
    for (u32 i = 0; i < a->nseg; ++i)
        if ((e = a->ck_x[i].alloc(s->nV)) || (e = a->ck_xp[i].alloc(s->nV)) || (e = a->ck_v[i].alloc(s->nV)))
            return fail_free(e);
    a->st_x.resize(a->K); a->st_v.resize(a->K); a->st_vstart.resize(a->K); a->st_vcount.resize(a->K);
    a->st_pool.resize(a->K);
    for (u32 i = 0; i < a->K; ++i)
        if ((e = a->st_x[i].alloc(s->nV)) || (e = a->st_v[i].alloc(s->nV)) || (e = a->st_vstart[i].alloc(s->nV)) ||
            (e = a->st_vcount[i].alloc(s->nV)) || (e = a->st_pool[i].alloc(s->cap)))
            return fail_free(e);
    if ((e = a->ax.alloc(s->nV)) || (e = a->av.alloc(s->nV)) || (e = a->ax2.alloc(s->nV)) || (e = a->av2.alloc(s->nV)) ||
        (e = a->xbar.alloc(s->nV)) || (e = a->vbar.alloc(s->nV)) || (e = a->fbar.alloc(s->nV)))
        return fail_free(e);
    // the rollout starts from the scene's current state
    YS_CK(cudaMemcpyAsync(a->x0.p, s->X[s->cur].p, sizeof(float4) * s->nV, cudaMemcpyDeviceToDevice, s->stream));
    YS_CK(cudaMemcpyAsync(a->v0.p, s->V[s->cv].p, sizeof(float4) * s->nV, cudaMemcpyDeviceToDevice, s->stream));
    YS_CK(cudaStreamSynchronize(s->stream));
    *out = a;
    return YS_OK;
}

ys_status ys_adjoint_destroy(ys_adjoint* a) {
    if (!a) return YS_OK;
    cudaStreamSynchronize(a->s->stream);
    for (auto* v : {&a->ck_x, &a->ck_xp, &a->ck_v, &a->st_x, &a->st_v}) for (auto& b : *v) b.free();
    for (auto& b : a->st_vstart) b.free();
    for (auto& b : a->st_vcount) b.free();
    for (auto& b : a->st_pool) b.free();
    a->x0.free(); a->v0.free(); a->ax.free(); a->av.free(); a->ax2.free(); a->av2.free();
    a->xbar.free(); a->vbar.free(); a->fbar.free();
    d64_free(a);
    delete a;
    return YS_OK;
}

uint32_t ys_adjoint_num_springs(ys_adjoint* a) { return a ? a->S : 0; }

// Set the rollout's parameters (device pointers, any may be NULL to keep):
// per-spring stiffness and rest length (canonical spring order), and the
// cloth's initial velocity (3 floats per vertex).
ys_status ys_adjoint_set_params(ys_adjoint* a, const float* d_k, const float* d_L, const float* d_v0) {
    if (!a) return fail(YS_ERR_BAD_ARG, "null adjoint");
    ys_scene* s = a->s;
    if (d_k || d_L) {
        ys_status r = ys_scene_set_grid_springs(s, a->mesh, d_k, d_L);
        if (r) return r;
    }
    if (d_v0) k_mesh_pack4<<<ceil_div(a->nV, 256), 256, 0, s->stream>>>(d_v0, a->v0.p, a->voff, a->nV);
    if (a->bits == 64) {  // the same values, widened
        if (d_k) k_d64_widen<<<ceil_div(a->S, 256), 256, 0, s->stream>>>(d_k, a->d_k.p, a->S);
        if (d_L) k_d64_widen<<<ceil_div(a->S, 256), 256, 0, s->stream>>>(d_L, a->d_L.p, a->S);
        if (d_v0) k_d64_from_f3<<<ceil_div(a->nV, 256), 256, 0, s->stream>>>(d_v0, a->d_v0.p, a->nV);
    }
    YS_CK(cudaGetLastError());
    a->forward_done = false;
    return YS_OK;
}

// Arithmetic of the rollout and its reverse pass: 32 (the fused substep's
// own binary32 arithmetic, the default) or 64 (binary64 throughout, the
// operations of the FP64 reference rollout; the scene's state is left as it
// is).  Switching to 64 widens the current parameters and initial state.
ys_status ys_adjoint_set_precision(ys_adjoint* a, int bits) {
    if (!a) return fail(YS_ERR_BAD_ARG, "null adjoint");
    if (bits != 32 && bits != 64) return fail(YS_ERR_BAD_ARG, "precision is 32 or 64 bits");
    if (bits == a->bits) return YS_OK;
    ys_scene* s = a->s;
    a->forward_done = false;
    if (bits == 32) {
        YS_CK(cudaStreamSynchronize(s->stream));
        d64_free(a);
        a->bits = 32;
        return YS_OK;
    }
    for (size_t m = 0; m < s->meshes.size(); ++m)
        if ((int)m != a->mesh && s->meshes[m].d.num_facets && !(s->meshes[m].flags & MF_STATIC))
            return fail(YS_ERR_BAD_ARG, "the FP64 rollout needs static obstacles");
    cudaError_t e = d64_alloc(a);
    if (e) {
        d64_free(a);
        return fail(YS_ERR_CUDA, cudaGetErrorString(e));
    }
    k_d64_from_f4<<<ceil_div(a->nV, 256), 256, 0, s->stream>>>(a->x0.p, a->d_x0.p, a->voff, a->nV);
    k_d64_from_f4<<<ceil_div(a->nV, 256), 256, 0, s->stream>>>(a->v0.p, a->d_v0.p, a->voff, a->nV);
    YS_CK(cudaGetLastError());
    ys_status r = d64_params_from_scene(a);
    if (r) {
        d64_free(a);
        return r;
    }
    a->bits = 64;
    return YS_OK;
}

// 64-bit mode: parameters in binary64 (device pointers, NULL keeps).
ys_status ys_adjoint_set_params_f64(ys_adjoint* a, const double* d_k, const double* d_L, const double* d_v0) {
    if (!a) return fail(YS_ERR_BAD_ARG, "null adjoint");
    if (a->bits != 64) return fail(YS_ERR_STATE, "set the adjoint's precision to 64 first");
    cudaStream_t st = a->s->stream;
    if (d_k) YS_CK(cudaMemcpyAsync(a->d_k.p, d_k, 8 * (size_t)a->S, cudaMemcpyDeviceToDevice, st));
    if (d_L) YS_CK(cudaMemcpyAsync(a->d_L.p, d_L, 8 * (size_t)a->S, cudaMemcpyDeviceToDevice, st));
    if (d_v0) k_d64_from_d3<<<ceil_div(a->nV, 256), 256, 0, st>>>(d_v0, a->d_v0.p, a->nV);
    YS_CK(cudaGetLastError());
    a->forward_done = false;
    return YS_OK;
}

// 64-bit mode: forward rollout; x_T (3 doubles per vertex) into d_xT.
ys_status ys_adjoint_forward_f64(ys_adjoint* a, double* d_xT) {
    if (!a) return fail(YS_ERR_BAD_ARG, "null adjoint");
    if (a->bits != 64) return fail(YS_ERR_STATE, "set the adjoint's precision to 64 first");
    const D4* x = nullptr;
    ys_status r = d64_forward(a, &x);
    if (r) return r;
    if (d_xT) k_d64_to_d3<<<ceil_div(a->nV, 256), 256, 0, a->s->stream>>>(x, d_xT, a->nV);
    YS_CK(cudaGetLastError());
    YS_CK(cudaStreamSynchronize(a->s->stream));
    return YS_OK;
}

// 64-bit mode: reverse pass with binary64 seed and gradients.
ys_status ys_adjoint_backward_f64(ys_adjoint* a, const double* d_dLdx, double* d_gk, double* d_gL, double* d_gv0) {
    if (!a || !d_dLdx || !d_gk || !d_gL || !d_gv0) return fail(YS_ERR_BAD_ARG, "null argument");
    if (a->bits != 64) return fail(YS_ERR_STATE, "set the adjoint's precision to 64 first");
    if (!a->forward_done) return fail(YS_ERR_STATE, "run ys_adjoint_forward first");
    cudaStream_t st = a->s->stream;
    k_d64_from_d3<<<ceil_div(a->nV, 256), 256, 0, st>>>(d_dLdx, a->dax.p, a->nV);
    YS_CK(cudaGetLastError());
    ys_status r = d64_backward(a);
    if (r) return r;
    YS_CK(cudaMemcpyAsync(d_gk, a->dgk.p, 8 * (size_t)a->S, cudaMemcpyDeviceToDevice, st));
    YS_CK(cudaMemcpyAsync(d_gL, a->dgL.p, 8 * (size_t)a->S, cudaMemcpyDeviceToDevice, st));
    k_d64_to_d3<<<ceil_div(a->nV, 256), 256, 0, st>>>(a->g_bwd_av, d_gv0, a->nV);
    YS_CK(cudaGetLastError());
    YS_CK(cudaStreamSynchronize(st));
    return YS_OK;
}

// Forward rollout of T substeps from the initial state; x_T of the cloth
// (3 floats per vertex) into d_xT.
ys_status ys_adjoint_forward(ys_adjoint* a, float* d_xT) {
    if (!a) return fail(YS_ERR_BAD_ARG, "null adjoint");
    ys_scene* s = a->s;
    if (a->bits == 64) {
        const D4* x = nullptr;
        ys_status r = d64_forward(a, &x);
        if (r) return r;
        if (d_xT) k_d64_to_f3<<<ceil_div(a->nV, 256), 256, 0, s->stream>>>(x, d_xT, a->nV);
        YS_CK(cudaGetLastError());
        return YS_OK;
    }
    restore_state(s, a->x0.p, a->x0.p, a->v0.p, 0, 0);
    const bool rec = s->record;
    s->record = false;
    ys_status r = YS_OK;
    for (u32 t = 0; t < a->T && !r; ++t) {
        if (t % a->K == 0) {
            const u32 i = t / a->K;
            const size_t bytes = sizeof(float4) * s->nV;
            const float4* xp = s->snapshot_pending ? s->X[s->cur].p : s->X[s->prev].p;
            YS_CK(cudaMemcpyAsync(a->ck_x[i].p, s->X[s->cur].p, bytes, cudaMemcpyDeviceToDevice, s->stream));
            YS_CK(cudaMemcpyAsync(a->ck_xp[i].p, xp, bytes, cudaMemcpyDeviceToDevice, s->stream));
            YS_CK(cudaMemcpyAsync(a->ck_v[i].p, s->V[s->cv].p, bytes, cudaMemcpyDeviceToDevice, s->stream));
            a->ck_frame[i] = s->frame;
            a->ck_cursor[i] = s->cursor;
        }
        r = fused_substep(s);
    }
    s->record = rec;
    if (r) return r;
    if (d_xT) k_mesh_unpack4<<<ceil_div(a->nV, 256), 256, 0, s->stream>>>(s->X[s->cur].p, d_xT, a->voff, a->nV);
    YS_CK(cudaGetLastError());
    a->forward_done = true;
    return YS_OK;
}

// Reverse pass: dL/dx_T of the cloth in, gradients w.r.t. per-spring
// stiffness, rest length and the initial velocity out (device pointers).
ys_status ys_adjoint_backward(ys_adjoint* a, const float* d_dLdx, float* d_gk, float* d_gL, float* d_gv0) {
    if (!a || !d_dLdx || !d_gk || !d_gL || !d_gv0) return fail(YS_ERR_BAD_ARG, "null argument");
    if (!a->forward_done) return fail(YS_ERR_STATE, "run ys_adjoint_forward first");
    ys_scene* s = a->s;
    cudaStream_t st = s->stream;
    if (a->bits == 64) {
        k_d64_from_f3<<<ceil_div(a->nV, 256), 256, 0, st>>>(d_dLdx, a->dax.p, a->nV);
        YS_CK(cudaGetLastError());
        ys_status r = d64_backward(a);
        if (r) return r;
        k_d64_narrow<<<ceil_div(a->S, 256), 256, 0, st>>>(a->dgk.p, d_gk, a->S);
        k_d64_narrow<<<ceil_div(a->S, 256), 256, 0, st>>>(a->dgL.p, d_gL, a->S);
        k_d64_to_f3<<<ceil_div(a->nV, 256), 256, 0, st>>>(a->g_bwd_av, d_gv0, a->nV);
        YS_CK(cudaGetLastError());
        YS_CK(cudaStreamSynchronize(st));
        return YS_OK;
    }
    const size_t bytes = sizeof(float4) * s->nV;
    YS_CK(cudaMemsetAsync(a->ax.p, 0, bytes, st));
    YS_CK(cudaMemsetAsync(a->av.p, 0, bytes, st));
    k_mesh_pack4<<<ceil_div(a->nV, 256), 256, 0, st>>>(d_dLdx, a->ax.p, a->voff, a->nV);
    YS_CK(cudaMemsetAsync(d_gk, 0, 4 * (size_t)a->S, st));
    YS_CK(cudaMemsetAsync(d_gL, 0, 4 * (size_t)a->S, st));
    ys_status r = YS_OK;
    const bool rec = s->record;
    VContact* keep_pool = s->pool.p;
    u32* keep_vs = s->vstart.p;
    u32* keep_vc = s->vcount.p;
    if ((r = ensure_record(s))) return r;
    keep_pool = s->pool.p; keep_vs = s->vstart.p; keep_vc = s->vcount.p;
    for (int seg = (int)a->nseg - 1; seg >= 0 && !r; --seg) {
        const u32 t0 = (u32)seg * a->K, t1 = std::min(a->T, t0 + a->K);
        restore_state(s, a->ck_x[seg].p, a->ck_xp[seg].p, a->ck_v[seg].p, a->ck_frame[seg], a->ck_cursor[seg]);
        s->record = true;
        for (u32 t = t0; t < t1 && !r; ++t) {
            const u32 k = t - t0;
            YS_CK(cudaMemcpyAsync(a->st_x[k].p, s->X[s->cur].p, bytes, cudaMemcpyDeviceToDevice, st));
            YS_CK(cudaMemcpyAsync(a->st_v[k].p, s->V[s->cv].p, bytes, cudaMemcpyDeviceToDevice, st));
            s->pool.p = a->st_pool[k].p;
            s->vstart.p = a->st_vstart[k].p;
            s->vcount.p = a->st_vcount[k].p;
            r = fused_substep(s);
        }
        s->pool.p = keep_pool; s->vstart.p = keep_vs; s->vcount.p = keep_vc;
        s->record = rec;
        if (r) break;
        for (int t = (int)t1 - 1; t >= (int)t0; --t) {
            const u32 k = (u32)t - t0;
            StepArgs A = make_args(s);
            AdjArgs J;
            J.x = a->st_x[k].p; J.v = a->st_v[k].p;
            J.vstart = a->st_vstart[k].p; J.vcount = a->st_vcount[k].p; J.pool = a->st_pool[k].p;
            J.ax = a->ax.p; J.av = a->av.p; J.xbar = a->xbar.p; J.vbar = a->vbar.p; J.fbar = a->fbar.p;
            J.ax_out = a->ax2.p; J.av_out = a->av2.p;
            J.gk = d_gk; J.gL = d_gL;
            J.voff = a->voff; J.nV = a->nV; J.N = a->N;
            // forces at step t read the step's own state
            A.x = J.x; A.v = J.v;
            k_adj_vertex<<<ceil_div(a->nV, 128), 128, 0, st>>>(A, J, (u32)a->mesh);
            k_adj_springs<<<ceil_div(a->nV, 128), 128, 0, st>>>(A, J, (u32)a->mesh);
            YS_CK(cudaGetLastError());
            std::swap(a->ax.p, a->ax2.p);
            std::swap(a->av.p, a->av2.p);
        }
    }
    if (r) return r;
    k_mesh_unpack4<<<ceil_div(a->nV, 256), 256, 0, st>>>(a->av.p, d_gv0, a->voff, a->nV);
    YS_CK(cudaGetLastError());
    YS_CK(cudaStreamSynchronize(st));
    return YS_OK;
}

}  // extern "C"
