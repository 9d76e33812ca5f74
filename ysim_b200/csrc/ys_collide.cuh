// ys_collide.cuh -- device functions of the collision + solver path, shared by
// the fused substep kernel and the staged (one kernel per reference stage)
// kernels.  Every function restates one reference routine, cited inline.
#pragma once
#include "ys_common.cuh"

namespace ys {

static constexpr int STACK_DEPTH = 64;          // queryAABB stack (bvh.metal:1333)
// Visit cap of one descent.  The reference's wedge guard allows 2^22
// (bvh.metal:1352); a healthy query here visits a few hundred nodes, and a
// descent that reaches 2^16 is reported (YS_FLAG_STACK_OVF) and stopped so a
// degenerate tree cannot keep a kernel busy for minutes.
static constexpr u32 VISIT_CAP = 1u << 16;

// intersectAABB (bvh.metal:1285-1290): inclusive box overlap.
__device__ __forceinline__ bool overlap(f3 qmn, f3 qmx, float4 n0, float4 n1) {
    if (qmx.x < n0.x || qmn.x > n1.x) return false;
    if (qmx.y < n0.y || qmn.y > n1.y) return false;
    if (qmx.z < n0.z || qmn.z > n1.z) return false;
    return true;
}

// Depth-first descent from slot 0 (queryAABB, bvh.metal:1322-1392), calling
// fn(face) for every leaf whose box overlaps [qmn, qmx].  Returns status bits.
// Both children of a node are loaded and tested together (two independent
// loads per step); the walk goes on into an overlapping internal child and
// pushes the other only when both overlap.  The reference pops every child
// and tests it after the pop: the same nodes pass the test and the same
// leaves are reported (once per path, as there), with one dependent load per
// level instead of one per child and no stack traffic for rejected children.
template <class Fn>
__device__ __forceinline__ u32 traverse(const Node* __restrict__ nodes, u32 numNodes, f3 qmn, f3 qmx, Fn&& fn) {
    if (numNodes == 0) return 0;
    const float4* r = reinterpret_cast<const float4*>(nodes);
    const float4 r0 = __ldg(r), r1 = __ldg(r + 1);
    if (!overlap(qmn, qmx, r0, r1)) return 0;
    int a = __float_as_int(r0.w), b = __float_as_int(r1.w);
    if (a < 0) { fn((u32)b); return 0; }  // a tree of one leaf
    int stack[2 * STACK_DEPTH];  // pending (a, b) child pairs: STACK_DEPTH subtrees, as the reference's stack
    int sp = 0;
    u32 visited = 0, st = 0;
    while (true) {
        if (++visited > VISIT_CAP) { st |= ST_STACK_OVF; break; }
        // children a and b of the current node
        bool ga = false, gb = false;
        int aa = -1, ab = -1, ba = -1, bb = -1;
        if (a >= 0 && (u32)a < numNodes && b >= 0 && (u32)b < numNodes) {
            const float4* pa = reinterpret_cast<const float4*>(nodes + a);
            const float4* pb = reinterpret_cast<const float4*>(nodes + b);
            const float4 a0 = __ldg(pa), a1 = __ldg(pa + 1), b0 = __ldg(pb), b1 = __ldg(pb + 1);
            if (overlap(qmn, qmx, a0, a1)) {
                aa = __float_as_int(a0.w); ab = __float_as_int(a1.w);
                if (aa < 0) fn((u32)ab); else ga = true;
            }
            if (overlap(qmn, qmx, b0, b1)) {
                ba = __float_as_int(b0.w); bb = __float_as_int(b1.w);
                if (ba < 0) fn((u32)bb); else gb = true;
            }
        }
        if (ga) {
            if (gb) {
                if (sp + 2 > 2 * STACK_DEPTH) { st |= ST_STACK_OVF; } else { stack[sp++] = ba; stack[sp++] = bb; }
            }
            a = aa; b = ab;
        } else if (gb) {
            a = ba; b = bb;
        } else {
            if (sp == 0) break;
            b = stack[--sp];
            a = stack[--sp];
        }
    }
    return st;
}

__device__ __forceinline__ bool overlap_xyz(f3 qmn, f3 qmx, float lx, float ly, float lz, float hx, float hy,
                                            float hz) {
    if (qmx.x < lx || qmn.x > hx) return false;
    if (qmx.y < ly || qmn.y > hy) return false;
    if (qmx.z < lz || qmn.z > hz) return false;
    return true;
}

// One step of a 4-wide descent: the node's four child boxes against the
// query; internal children are pushed, leaves reported through leaf(slot,
// face).  Returns status bits (stack full).
template <class Leaf>
__device__ __forceinline__ u32 wide_step(const Wide4* __restrict__ w4, int w, f3 qmn, f3 qmx, int* stack, int& sp,
                                         Leaf&& leaf) {
    const float4* p = reinterpret_cast<const float4*>(w4 + w);
    const float4 lx = __ldg(p), ly = __ldg(p + 1), lz = __ldg(p + 2);
    const float4 hx = __ldg(p + 3), hy = __ldg(p + 4), hz = __ldg(p + 5);
    const int4 ch = __ldg(reinterpret_cast<const int4*>(p + 6));
    const float LX[4] = {lx.x, lx.y, lx.z, lx.w}, LY[4] = {ly.x, ly.y, ly.z, ly.w}, LZ[4] = {lz.x, lz.y, lz.z, lz.w};
    const float HX[4] = {hx.x, hx.y, hx.z, hx.w}, HY[4] = {hy.x, hy.y, hy.z, hy.w}, HZ[4] = {hz.x, hz.y, hz.z, hz.w};
    const int C[4] = {ch.x, ch.y, ch.z, ch.w};
    u32 st = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int c = C[k];
        if (c == W4_EMPTY || !overlap_xyz(qmn, qmx, LX[k], LY[k], LZ[k], HX[k], HY[k], HZ[k])) continue;
        if (c < 0) {
            leaf(k, (u32)~c);
        } else if (sp < STACK_DEPTH) {
            stack[sp++] = c;
        } else {
            st |= ST_STACK_OVF;
        }
    }
    return st;
}

// The same step with the pushes going through push(child), which returns
// false when the stack is full.
template <class Push, class Leaf>
__device__ __forceinline__ u32 wide_step_p(const Wide4* __restrict__ w4, int w, f3 qmn, f3 qmx, Push&& push,
                                           Leaf&& leaf) {
    const float4* p = reinterpret_cast<const float4*>(w4 + w);
    const float4 lx = __ldg(p), ly = __ldg(p + 1), lz = __ldg(p + 2);
    const float4 hx = __ldg(p + 3), hy = __ldg(p + 4), hz = __ldg(p + 5);
    const int4 ch = __ldg(reinterpret_cast<const int4*>(p + 6));
    const float LX[4] = {lx.x, lx.y, lx.z, lx.w}, LY[4] = {ly.x, ly.y, ly.z, ly.w}, LZ[4] = {lz.x, lz.y, lz.z, lz.w};
    const float HX[4] = {hx.x, hx.y, hx.z, hx.w}, HY[4] = {hy.x, hy.y, hy.z, hy.w}, HZ[4] = {hz.x, hz.y, hz.z, hz.w};
    const int C[4] = {ch.x, ch.y, ch.z, ch.w};
    u32 st = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int c = C[k];
        if (c == W4_EMPTY || !overlap_xyz(qmn, qmx, LX[k], LY[k], LZ[k], HX[k], HY[k], HZ[k])) continue;
        if (c < 0) {
            leaf(k, (u32)~c);
        } else if (!push(c)) {
            st |= ST_STACK_OVF;
        }
    }
    return st;
}

// Descent of the 4-wide form of a tree (same leaves as traverse on the binary
// form): the root box first (binary root node), then wide nodes from 0.
template <class Fn>
__device__ __forceinline__ u32 traverse_wide(const Node* __restrict__ root, const Wide4* __restrict__ w4, u32 cap,
                                             f3 qmn, f3 qmx, Fn&& fn) {
    if (cap == 0) return 0;
    {
        const float4* p = reinterpret_cast<const float4*>(root);
        if (!overlap(qmn, qmx, __ldg(p), __ldg(p + 1))) return 0;
    }
    int stack[STACK_DEPTH];
    int sp = 0;
    stack[sp++] = 0;
    u32 visited = 0, st = 0;
    while (sp > 0) {
        if (++visited > VISIT_CAP) { st |= ST_STACK_OVF; break; }
        const int w = stack[--sp];
        if (w < 0 || (u32)w >= cap) continue;
        st |= wide_step(w4, w, qmn, qmx, stack, sp, [&](int, u32 f) { fn(f); });
    }
    return st;
}

__device__ __forceinline__ bool root_overlap(const Node* __restrict__ a, const Node* __restrict__ b) {
    const float4* pa = reinterpret_cast<const float4*>(a);
    const float4* pb = reinterpret_cast<const float4*>(b);
    float4 a0 = __ldg(pa), a1 = __ldg(pa + 1), b0 = __ldg(pb), b1 = __ldg(pb + 1);
    // AABB4::intersect (bvh.hpp:64-69)
    if (a1.x < b0.x || a0.x > b1.x) return false;
    if (a1.y < b0.y || a0.y > b1.y) return false;
    if (a1.z < b0.z || a0.z > b1.z) return false;
    return true;
}

// ------------------------------------------------------------- H1 self rows
// pointTriSq (spatial_hash.hpp:1659-1711).
__device__ __forceinline__ float point_tri_sq(const float p[3], const float a[3], const float b[3], const float c[3]) {
    float ab[3], ac[3], ap[3], q[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) { ab[i] = b[i] - a[i]; ac[i] = c[i] - a[i]; ap[i] = p[i] - a[i]; }
    const float d1 = ab[0] * ap[0] + ab[1] * ap[1] + ab[2] * ap[2];
    const float d2 = ac[0] * ap[0] + ac[1] * ap[1] + ac[2] * ap[2];
    if (d1 <= 0.f && d2 <= 0.f) {
#pragma unroll
        for (int i = 0; i < 3; ++i) q[i] = a[i];
    } else {
        float bp[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) bp[i] = p[i] - b[i];
        const float d3 = ab[0] * bp[0] + ab[1] * bp[1] + ab[2] * bp[2];
        const float d4 = ac[0] * bp[0] + ac[1] * bp[1] + ac[2] * bp[2];
        if (d3 >= 0.f && d4 <= d3) {
#pragma unroll
            for (int i = 0; i < 3; ++i) q[i] = b[i];
        } else {
            const float vc = d1 * d4 - d3 * d2;
            if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
                const float den = d1 - d3;
                const float vv = (den != 0.f) ? d1 / den : 0.f;
#pragma unroll
                for (int i = 0; i < 3; ++i) q[i] = a[i] + vv * ab[i];
            } else {
                float cp[3];
#pragma unroll
                for (int i = 0; i < 3; ++i) cp[i] = p[i] - c[i];
                const float d5 = ab[0] * cp[0] + ab[1] * cp[1] + ab[2] * cp[2];
                const float d6 = ac[0] * cp[0] + ac[1] * cp[1] + ac[2] * cp[2];
                if (d6 >= 0.f && d5 <= d6) {
#pragma unroll
                    for (int i = 0; i < 3; ++i) q[i] = c[i];
                } else {
                    const float vb = d5 * d2 - d1 * d6;
                    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
                        const float den = d2 - d6;
                        const float w = (den != 0.f) ? d2 / den : 0.f;
#pragma unroll
                        for (int i = 0; i < 3; ++i) q[i] = a[i] + w * ac[i];
                    } else {
                        const float va = d3 * d6 - d5 * d4;
                        if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
                            const float den = (d4 - d3) + (d5 - d6);
                            const float w = (den != 0.f) ? (d4 - d3) / den : 0.f;
#pragma unroll
                            for (int i = 0; i < 3; ++i) q[i] = b[i] + w * (c[i] - b[i]);
                        } else {
                            const float den = va + vb + vc;
                            const float vv = (den != 0.f) ? vb / den : 0.f;
                            const float w = (den != 0.f) ? vc / den : 0.f;
#pragma unroll
                            for (int i = 0; i < 3; ++i) q[i] = a[i] + ab[i] * vv + ac[i] * w;
                        }
                    }
                }
            }
        }
    }
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 3; ++i) { const float e = p[i] - q[i]; s += e * e; }
    return s;
}

// Query side of the CPU spatial hash (probeMeshVertices,
// spatial_hash.hpp:1756-1781): swept vertex box, xPrev replaced by x when it
// is non-finite or more than 1 m away, vertices spanning > 64 cells skipped.
struct H1Vertex { float pc[3], pp[3], lo[3], hi[3]; };
__device__ __forceinline__ bool h1_vertex(f3 x, f3 xp, float inv, H1Vertex& h) {
    const float xc[3] = {x.x, x.y, x.z}, xq[3] = {xp.x, xp.y, xp.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float pc = xc[a], pp = xq[a];
        if (!isfinite(pc)) return false;
        if (!isfinite(pp) || fabsf(pp - pc) > 1.f) pp = pc;
        h.pc[a] = pc; h.pp[a] = pp;
        h.lo[a] = (pp < pc) ? pp : pc;   // std::min(pc, pp)
        h.hi[a] = (pc < pp) ? pp : pc;   // std::max(pc, pp)
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        int l = (int)floorf(h.lo[a] * inv), u = (int)floorf(h.hi[a] * inv);
        if (u - l > 64) return false;
    }
    return true;
}
// The box part of h1_vertex for a vertex that already passed its 64-cell check.
__device__ __forceinline__ void h1_vertex_box(f3 x, f3 xp, H1Vertex& h) {
    const float xc[3] = {x.x, x.y, x.z}, xq[3] = {xp.x, xp.y, xp.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float pc = xc[a], pp = xq[a];
        if (!isfinite(pp) || fabsf(pp - pc) > 1.f) pp = pc;
        h.pc[a] = pc; h.pp[a] = pp;
        h.lo[a] = (pp < pc) ? pp : pc;
        h.hi[a] = (pc < pp) ? pp : pc;
    }
}
// Traversal box that contains every face box the exact test can accept: the
// vertex box grown by m plus a few ulps of slack, so the BVH never prunes a
// row the grid would have produced.
__device__ __forceinline__ void h1_query_box(const H1Vertex& h, float m, f3& qmn, f3& qmx) {
    float s = fmaxf(fmaxf(fabsf(h.lo[0]), fabsf(h.hi[0])), fmaxf(fmaxf(fabsf(h.lo[1]), fabsf(h.hi[1])),
                    fmaxf(fabsf(h.lo[2]), fabsf(h.hi[2]))));
    float pad = m * (1.0f + 1.0f / 65536.0f) + (s + 1.0f) * (1.0f / 65536.0f);
    qmn = mk(h.lo[0] - pad, h.lo[1] - pad, h.lo[2] - pad);
    qmx = mk(h.hi[0] + pad, h.hi[1] + pad, h.hi[2] + pad);
}
// Exact row test for face f of the vertex's own mesh (h1_face): the face does
// not contain the vertex, the face key box (tri AABB +- m, collectFaceBoxes
// spatial_hash.hpp:1625-1643) overlaps the swept vertex box, and the
// point-triangle distance^2 at x or xPrev is <= m^2
// (spatial_hash.hpp:1804-1846).  h1_face_at is the part after the own-face
// check, on the face's three vertex positions.
// span_check = false skips the face's 64-cell test, for callers whose cell
// size is this mesh's largest key-box extent computed from the same positions
// (the refit's H1 extent): every key box then spans at most two cells.
__device__ __forceinline__ bool h1_face_at(f3 P0, f3 P1, f3 P2, float m, float inv, const H1Vertex& h,
                                           bool span_check) {
    const float A[3] = {P0.x, P0.y, P0.z}, B[3] = {P1.x, P1.y, P1.z}, C[3] = {P2.x, P2.y, P2.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (!isfinite(A[a]) || !isfinite(B[a]) || !isfinite(C[a])) return false;
    }
    float bmn[3], bmx[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        // std::min(p0, std::min(p1, p2))
        float mn12 = (C[a] < B[a]) ? C[a] : B[a];
        float lo = (mn12 < A[a]) ? mn12 : A[a];
        float mx12 = (B[a] < C[a]) ? C[a] : B[a];
        float hi = (A[a] < mx12) ? mx12 : A[a];
        bmn[a] = lo - m;
        bmx[a] = hi + m;
    }
    if (span_check) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            int l = (int)floorf(bmn[a] * inv), u = (int)floorf(bmx[a] * inv);
            if (u - l > 64) return false;  // face never entered the grid
        }
    }
    if (h.hi[0] < bmn[0] || h.lo[0] > bmx[0] || h.hi[1] < bmn[1] || h.lo[1] > bmx[1] || h.hi[2] < bmn[2] ||
        h.lo[2] > bmx[2])
        return false;
    const float m2 = m * m;
    if (point_tri_sq(h.pc, A, B, C) > m2 && point_tri_sq(h.pp, A, B, C) > m2) return false;
    return true;
}
__device__ __forceinline__ bool h1_face(const float4* __restrict__ X, u32 voff, uint4 tri, u32 v, float m, float inv,
                                        const H1Vertex& h, bool span_check = true) {
    if (tri.x == v || tri.y == v || tri.z == v) return false;
    return h1_face_at(ld(X, voff + tri.x), ld(X, voff + tri.y), ld(X, voff + tri.z), m, inv, h, span_check);
}

// ------------------------------------------------------------- N1 narrow
// pointInTriangleBary (bruteforce.metal:9-28).  b and c are quotients of
// the numerators below by den; an IEEE quotient is >= 0 exactly when its
// numerator is a zero or has den's sign, so a point with b < 0 or c < 0 is
// rejected from the signs alone, before the two divisions (the same result
// as dividing first).
__device__ __forceinline__ bool point_in_tri(f3 p, f3 e0, f3 e1) {
    float d00 = dot(e0, e0), d01 = dot(e0, e1), d11 = dot(e1, e1), d20 = dot(p, e0), d21 = dot(p, e1);
    float den = d00 * d11 - d01 * d01;
    if (fabsf(den) < 1e-12f) return false;
    const float nb = d11 * d20 - d01 * d21, nc = d00 * d21 - d01 * d20;
    const bool dneg = den < 0.0f;
    if ((nb != 0.0f && (nb < 0.0f) != dneg) || (nc != 0.0f && (nc < 0.0f) != dneg)) return false;
    float b = nb / den;
    float c = nc / den;
    float a = 1.0f - b - c;
    return (a >= 0.0f && b >= 0.0f && c >= 0.0f);
}
// narrow_pt_tri (bruteforce.metal:41-178) for one candidate: swept segment
// xPrev -> x against the triangle plane; rsqrt written as 1/sqrt (IEEE).
__device__ __forceinline__ bool narrow_one(f3 qcur, f3 qprev, f3 t0, f3 t1, f3 t2, float band, f3& nout, float& dout) {
    f3 e0 = t1 - t0, e1 = t2 - t0;
    f3 n = cross(e0, e1);
    float nl2 = dot(n, n);
    if (nl2 < 1e-12f) return false;
    n = n * (1.0f / sqrtf(nl2));
    float dp = dot(n, qprev - t0), dc = dot(n, qcur - t0);
    float dref = (dp != 0.0f) ? dp : dc;
    if (dref < 0.0f) { n = -n; dp = -dp; dc = -dc; }
    bool crossed = dc < 0.0f, inm = dc < band;
    if (!crossed && !inm) return false;
    f3 cp;
    if (crossed && dp > 0.0f) {
        float t = dp / (dp - dc);
        cp = qprev + (qcur - qprev) * t;  // mix(qprev, qcur, t)
    } else {
        cp = qcur;
    }
    f3 pc = cp - t0;
    float l = dot(n, pc);
    f3 inplane = pc - n * l;
    if (!point_in_tri(inplane, e0, e1)) return false;
    nout = n;
    dout = dc;
    return true;
}

// ------------------------------------------------------------- F / I
// calc_spring (physics.metal:146-153).
__device__ __forceinline__ f3 spring(f3 p0, f3 v0, f3 p1, f3 v1, float rest, float ks, float kd) {
    f3 dx = p1 - p0, dv = v1 - v0;
    float len = sqrtf(dot(dx, dx));
    if (len < 1e-7f) return mk(0.f, 0.f, 0.f);
    f3 nd = dx / len;
    return nd * (ks * (len - rest) + kd * dot(dv, nd));
}

// sanitizeIntegrateOutput (physics.metal:52-74).
__device__ __forceinline__ bool sanitize(f3& pos, f3& vel, f3 fb) {
    bool touched = false;
    if (nonfinite3(pos)) { pos = nonfinite3(fb) ? mk(0.f, 0.f, 0.f) : fb; vel = mk(0.f, 0.f, 0.f); touched = true; }
    if (nonfinite3(vel)) { vel = mk(0.f, 0.f, 0.f); touched = true; }
    const float B = 1.0e4f;
    f3 bx = mk(fminf(fmaxf(pos.x, -B), B), fminf(fmaxf(pos.y, -B), B), fminf(fmaxf(pos.z, -B), B));
    if (bx.x != pos.x || bx.y != pos.y || bx.z != pos.z) { pos = bx; vel = mk(0.f, 0.f, 0.f); touched = true; }
    return touched;
}

// Contact response of integrate_cloth / integrate_cloth_grid
// (physics.metal:254-297): skip duplicate (target object, triangle), then for
// d < thickness remove the approaching normal velocity and push the position
// out to thickness.
template <class Get>
__device__ __forceinline__ void contact_response(f3& pos, f3& vel, int nc, float thickness, Get&& get) {
    for (int i = 0; i < nc; ++i) {
        VContact ci = get(i);
        bool dup = false;
        for (int j = 0; j < i; ++j) {
            VContact cj = get(j);
            if (cj.tobj == ci.tobj && cj.tri == ci.tri) { dup = true; break; }
        }
        if (dup) continue;
        f3 n = mk(ci.nx, ci.ny, ci.nz);
        float nl2 = dot(n, n);
        if (nl2 < 1e-12f) continue;
        n = n * (1.0f / sqrtf(nl2));
        float vn = dot(vel, n);
        if (ci.d < thickness) {
            if (vn < 0.0f) vel = vel - n * vn;
            pos = pos + n * (thickness - ci.d);
        }
    }
}

}  // namespace ys
