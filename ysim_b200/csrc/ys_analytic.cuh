// ys_analytic.cuh -- analytic colliders: a cloth vertex against one sphere /
// ellipsoid, box, capped cylinder or half-space, with the swept test done by
// motion inversion (narrow_pt_analytic, src/metal/bruteforce.metal:236-499),
// and the host-side broad box and rotation margins of a shape
// (BVH::analyticWorldHalf / analyticRotBand / objectBroadAABB,
// include/sim/bvh.hpp:2431-2516; BruteForce::analyticRotMargin,
// include/sim/bruteforce.hpp:201-240).
//
// Arithmetic: every float operation rounds once, in the order the reference
// writes it (-fmad=false, IEEE division and square root); normalize(v) is
// v * (1 / sqrt(dot(v, v))) and length(v) is sqrt(dot(v, v)), min / max of
// floats are fminf / fmaxf.
#pragma once
#include <algorithm>
#include <cmath>

#include "ys_common.cuh"

namespace ys {

// ColliderKind (include/sim/collision_pod.hpp; YSIM_COLLIDER_*,
// src/metal/common_types.metalh:80-84).
enum : u32 { COL_MESH = 0u, COL_SPHERE = 1u, COL_BOX = 2u, COL_CYLINDER = 3u, COL_PLANE = 4u };

// AnalyticShape (collision_pod.hpp:295-309), 96 bytes: centre + radius,
// half extents + cylinder half height, orientation (w, x, y, z) local to
// world, the previous centre and orientation, kind, owning mesh index,
// behaviour, flags (bit 0 collidable).
struct __align__(16) AShape {
    float4 cr, he, rq, pc, prq;
    u32 kind, obj, beh, flags;
};
static_assert(sizeof(AShape) == 96, "AShape must be 96 bytes");

// Device table entry of a scene's analytic collider: the shape, its broad
// box (lo.w = 1 when finite; a half-space has none) and the narrow band's
// rotation margin.
struct __align__(16) DShape {
    AShape s;
    float4 lo, hi;
    float rot_margin;
    u32 pad[3];
};
static_assert(sizeof(DShape) == 144, "DShape must be 144 bytes");

__host__ __device__ __forceinline__ f3 mul3(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ f3 xyz(float4 q) { return mk(q.x, q.y, q.z); }
__host__ __device__ __forceinline__ f3 yzw(float4 q) { return mk(q.y, q.z, q.w); }
__host__ __device__ __forceinline__ float len3(f3 a) { return sqrtf(dot(a, a)); }
__host__ __device__ __forceinline__ f3 unit3(f3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
__host__ __device__ __forceinline__ float len2(float a, float b) { return sqrtf(a * a + b * b); }
__host__ __device__ __forceinline__ float comp(f3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

// quatRotate (bruteforce.metal:196-201): v + 2 (q_v x (q_v x v + q_w v)).
__host__ __device__ __forceinline__ f3 quat_rotate(float qw, f3 qv, f3 v) {
    const f3 inner = cross(qv, v) + mk(qw * v.x, qw * v.y, qw * v.z);
    const f3 c = cross(qv, inner);
    return v + mk(2.0f * c.x, 2.0f * c.y, 2.0f * c.z);
}

// boxDominantAxis (bruteforce.metal:203-216): the axis of the largest
// |q_k| - h_k (first one on ties) and the sign of q there.
__host__ __device__ __forceinline__ void box_axis(f3 q, f3 h, int& axis, float& sgn) {
    const float gx = fabsf(q.x) - h.x, gy = fabsf(q.y) - h.y, gz = fabsf(q.z) - h.z;
    axis = 0;
    float best = gx;
    if (gy > best) { best = gy; axis = 1; }
    if (gz > best) axis = 2;
    sgn = comp(q, axis) >= 0.0f ? 1.0f : -1.0f;
}

// narrow_pt_analytic (bruteforce.metal:259-499) for one vertex: the segment
// from x_prev mapped through the previous pose to x mapped through the
// current pose, against the static canonical shape.  On a contact returns
// true with the world normal and the signed distance of x along it.
__host__ __device__ inline bool analytic_narrow(const AShape& sh, f3 pcur, f3 pprev, float radius, float thickness,
                                                float rot_margin, f3& n_out, float& d_out) {
    if (!(sh.flags & 1u) || sh.kind == COL_MESH) return false;
    const f3 a = quat_rotate(sh.prq.x, -yzw(sh.prq), pprev - xyz(sh.pc));
    const f3 b = quat_rotate(sh.rq.x, -yzw(sh.rq), pcur - xyz(sh.cr));
    const f3 seg = b - a;
    const float band = radius + thickness + rot_margin;
    f3 nl = mk(0.0f, 1.0f, 0.0f);
    float d = 1e30f;

    if (sh.kind == COL_PLANE) {
        d = b.y;  // half-space y <= 0, outward +y
    } else if (sh.kind == COL_SPHERE) {
        // unit sphere in u = q / e; band scaled by the smallest semi-axis
        const f3 e = mk(fmaxf(sh.he.x, 1e-8f), fmaxf(sh.he.y, 1e-8f), fmaxf(sh.he.z, 1e-8f));
        const float R = 1.0f + band / fminf(e.x, fminf(e.y, e.z));
        const f3 ua = a / e, ub = b / e;
        const float la = len3(ua);
        f3 u;
        if (la < 1.0f) {
            // started inside: leave along a's radius
            u = la > 1e-6f ? ua : (len3(ub) > 1e-6f ? ub : mk(0.0f, 1.0f, 0.0f));
        } else {
            // first root in [0, 1] of |ua + t (ub - ua)| = R
            const f3 D = ub - ua;
            const float qa = dot(D, D), qb = dot(ua, D), qc = dot(ua, ua) - R * R;
            float t = -1.0f;
            if (qa > 1e-20f) {
                const float disc = qb * qb - qa * qc;
                if (disc >= 0.0f) {
                    const float t0 = (-qb - sqrtf(disc)) / qa;
                    if (t0 >= 0.0f && t0 <= 1.0f) t = t0;
                }
            }
            if (t >= 0.0f) u = ua + mk(t * D.x, t * D.y, t * D.z);
            else if (len3(ub) > 1e-6f) u = ub;
            else return false;
        }
        const f3 uh = unit3(u);
        const f3 s = mul3(e, uh);
        nl = unit3(uh / e);
        d = dot(nl, b - s);
    } else if (sh.kind == COL_BOX) {
        const f3 h = mk(fmaxf(sh.he.x, 1e-8f), fmaxf(sh.he.y, 1e-8f), fmaxf(sh.he.z, 1e-8f));
        const f3 H = h + mk(band, band, band);
        int k = 0;
        float sg = 1.0f;
        if (fabsf(a.x) < h.x && fabsf(a.y) < h.y && fabsf(a.z) < h.z) {
            box_axis(a, h, k, sg);  // started inside: minimum-penetration face of a
        } else {
            // slab test of the segment against the inflated box
            float t_in = 0.0f, t_out = 1.0f, esg = 1.0f;
            int ek = -1;
            bool miss = false;
            for (int i = 0; i < 3 && !miss; ++i) {
                const float di = comp(seg, i), ai = comp(a, i), Hi = comp(H, i);
                if (fabsf(di) < 1e-12f) {
                    if (fabsf(ai) > Hi) miss = true;
                } else {
                    const float inv = 1.0f / di;
                    const float t1 = (-Hi - ai) * inv, t2 = (Hi - ai) * inv;
                    const float tn = fminf(t1, t2), tf = fmaxf(t1, t2);
                    if (tn > t_in) { t_in = tn; ek = i; esg = di > 0.0f ? -1.0f : 1.0f; }
                    t_out = fminf(t_out, tf);
                }
            }
            if (!miss && ek >= 0 && t_in <= t_out && t_in <= 1.0f) { k = ek; sg = esg; }
            else box_axis(b, h, k, sg);  // closest face of b
        }
        nl = mk(k == 0 ? sg : 0.0f, k == 1 ? sg : 0.0f, k == 2 ? sg : 0.0f);
        d = sg * comp(b, k) - comp(h, k);
    } else if (sh.kind == COL_CYLINDER) {
        // axis +y, radius r, half height hh; wall (0) or cap (1)
        const float r = fmaxf(sh.cr.w, 1e-8f), hh = fmaxf(sh.he.w, 1e-8f);
        const float R = r + band, HH = hh + band;
        int feat = 0;
        float cap = 1.0f, nx = 1.0f, nz = 0.0f;
        const bool a_in = len2(a.x, a.z) < r && fabsf(a.y) < hh;
        bool done = false;
        if (!a_in) {
            float t_in = 0.0f, t_out = 1.0f, ecap = 1.0f, ex = 1.0f, ez = 0.0f;
            int ef = -1;
            bool miss = false;
            const float qa = seg.x * seg.x + seg.z * seg.z, qb = a.x * seg.x + a.z * seg.z;
            const float qc = (a.x * a.x + a.z * a.z) - R * R;
            if (qa > 1e-20f) {
                const float disc = qb * qb - qa * qc;
                if (disc < 0.0f) {
                    miss = true;
                } else {
                    const float sq = sqrtf(disc);
                    const float t1 = (-qb - sq) / qa, t2 = (-qb + sq) / qa;
                    if (t1 > t_in) { t_in = t1; ef = 0; }
                    t_out = fminf(t_out, t2);
                }
            } else if (qc > 0.0f) {
                miss = true;  // parallel to the axis, outside R
            }
            if (!miss) {
                if (fabsf(seg.y) < 1e-12f) {
                    if (fabsf(a.y) > HH) miss = true;
                } else {
                    const float inv = 1.0f / seg.y;
                    const float t1 = (-HH - a.y) * inv, t2 = (HH - a.y) * inv;
                    const float tn = fminf(t1, t2), tf = fmaxf(t1, t2);
                    if (tn > t_in) { t_in = tn; ef = 1; ecap = seg.y > 0.0f ? -1.0f : 1.0f; }
                    t_out = fminf(t_out, tf);
                }
            }
            if (!miss && ef >= 0 && t_in <= t_out && t_in <= 1.0f) {
                if (ef == 0) {
                    const float hx = a.x + t_in * seg.x, hz = a.z + t_in * seg.z;
                    const float l = len2(hx, hz);
                    if (l > 1e-9f) { ex = hx / l; ez = hz / l; }
                }
                feat = ef; cap = ecap; nx = ex; nz = ez;
                done = true;
            }
        }
        if (!done) {
            // inside: a's nearest feature; otherwise b's
            const f3 q = a_in ? a : b;
            const float lxz = len2(q.x, q.z);
            feat = (r - lxz) <= (hh - fabsf(q.y)) ? 0 : 1;
            cap = q.y >= 0.0f ? 1.0f : -1.0f;
            if (lxz > 1e-9f) { nx = q.x / lxz; nz = q.z / lxz; }
            else { nx = 1.0f; nz = 0.0f; }
        }
        if (feat == 0) {
            nl = mk(nx, 0.0f, nz);
            d = dot(nl, b) - r;
        } else {
            nl = mk(0.0f, cap, 0.0f);
            d = cap * b.y - hh;
        }
    } else {
        return false;
    }
    if (!(d < band)) return false;
    n_out = unit3(quat_rotate(sh.rq.x, yzw(sh.rq), nl));
    d_out = d;
    return true;
}

// Host side: Quat operator* (Hamilton product) and rotateVector
// (q (0, v) q*), include/sim/material_quat.hpp:27-63, (w, x, y, z) order.
struct HQuat { float w, x, y, z; };
inline HQuat hq_mul(const HQuat& a, const HQuat& b) {
    HQuat r;
    r.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
    r.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
    r.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
    r.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
    return r;
}
inline f3 hq_rotate(const HQuat& q, f3 v) {
    const HQuat p = {0.0f, v.x, v.y, v.z};
    const HQuat c = {q.w, -q.x, -q.y, -q.z};
    const HQuat r = hq_mul(hq_mul(q, p), c);
    return mk(r.x, r.y, r.z);
}

// analyticWorldHalf (bvh.hpp:2431-2462): world half extents of the shape's
// box at orientation q (w, x, y, z in q.x..q.w).
inline f3 analytic_world_half(const AShape& s, float4 q) {
    f3 h = mk(0.0f, 0.0f, 0.0f);
    if (s.kind == COL_SPHERE) {
        const float r = std::max(std::max(s.he.x, s.he.y), s.he.z);
        return mk(r, r, r);
    } else if (s.kind == COL_BOX) {
        h = mk(s.he.x, s.he.y, s.he.z);
    } else if (s.kind == COL_CYLINDER) {
        h = mk(s.cr.w, s.he.w, s.cr.w);
    } else {
        return h;
    }
    const HQuat Q = {q.x, q.y, q.z, q.w};
    const f3 cx = hq_rotate(Q, mk(1.0f, 0.0f, 0.0f)), cy = hq_rotate(Q, mk(0.0f, 1.0f, 0.0f)),
             cz = hq_rotate(Q, mk(0.0f, 0.0f, 1.0f));
    return mk(std::fabs(cx.x) * h.x + std::fabs(cy.x) * h.y + std::fabs(cz.x) * h.z,
              std::fabs(cx.y) * h.x + std::fabs(cy.y) * h.y + std::fabs(cz.y) * h.z,
              std::fabs(cx.z) * h.x + std::fabs(cy.z) * h.y + std::fabs(cz.z) * h.z);
}

// Geodesic angle between the two orientations, 2 acos |q . q_prev|, in double.
inline double analytic_theta(const AShape& s) {
    double dq = (double)s.rq.x * (double)s.prq.x + (double)s.rq.y * (double)s.prq.y +
                (double)s.rq.z * (double)s.prq.z + (double)s.rq.w * (double)s.prq.w;
    dq = std::fabs(dq);
    if (dq > 1.0) dq = 1.0;
    return 2.0 * std::acos(dq);
}

// analyticRotBand (bvh.hpp:2465-2479): theta * (|half| + radius).
inline float analytic_rot_band(const AShape& s) {
    const double theta = analytic_theta(s);
    if (theta <= 0.0) return 0.0f;
    const double rmax = std::sqrt((double)s.he.x * s.he.x + (double)s.he.y * s.he.y + (double)s.he.z * s.he.z) +
                        (double)s.cr.w;
    return (float)(theta * rmax);
}

// analyticRotMargin (bruteforce.hpp:201-240): theta * (r_max + radius +
// thickness); 0 for a half-space.
inline float analytic_rot_margin(const AShape& s, float radius, float thickness) {
    const double theta = analytic_theta(s);
    if (!(theta > 1e-9)) return 0.0f;
    double rmax = 0.0;
    if (s.kind == COL_SPHERE) {
        rmax = std::max(std::max((double)s.he.x, (double)s.he.y), (double)s.he.z);
    } else if (s.kind == COL_BOX) {
        rmax = std::sqrt((double)s.he.x * s.he.x + (double)s.he.y * s.he.y + (double)s.he.z * s.he.z);
    } else if (s.kind == COL_CYLINDER) {
        rmax = std::sqrt((double)s.cr.w * s.cr.w + (double)s.he.w * s.he.w);
    } else if (s.kind == COL_PLANE) {
        return 0.0f;
    }
    return (float)(theta * (rmax + (double)radius + (double)thickness));
}

// objectBroadAABB for an analytic collider (bvh.hpp:2494-2516): the union of
// the boxes at the previous and the current pose, padded by the contact band
// (inflate = radius + margin) and the rotation band.  Returns false for a
// half-space (no finite box: every pair with it overlaps).
inline bool analytic_broad_box(const AShape& s, float inflate, f3& lo, f3& hi) {
    const f3 c = xyz(s.cr);
    if (s.kind == COL_PLANE) {
        lo = c;
        hi = c;
        return false;
    }
    const f3 p = xyz(s.pc);
    const f3 hc = analytic_world_half(s, s.rq), hp = analytic_world_half(s, s.prq);
    const float pad = inflate + analytic_rot_band(s);
    const f3 pv = mk(pad, pad, pad);
    lo = vmin(c - hc, p - hp) - pv;
    hi = vmax(c + hc, p + hp) + pv;
    return true;
}

}  // namespace ys
