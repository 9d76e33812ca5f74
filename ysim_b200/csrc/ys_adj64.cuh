// ys_adj64.cuh -- FP64 rollout of one FastGridCloth over static triangle
// obstacles, and its reverse pass (the adjoint's 64-bit mode).
//
// The single-precision adjoint differentiates the substep exactly as the
// fused kernel computes it, so its gradients carry FP32 round-off amplified
// by the rollout's conditioning (stiff springs over hundreds of steps).  This
// mode runs the same step in binary64, operation for operation as the FP64
// reference rollout states it, so that the gradient differs from FP64 finite
// differences only by the differencing error:
//
//   f_i = (ext_i or g m_i) + kair v_i + sum_s (k_s (l - L_s) + kd (dv . n)) n,
//         n = dx (1 / l), springs in the stencil order of
//         compute_cloth_grid_forces_fast (physics.metal:197-218), l < 1e-7 skipped
//   v'  = v + f ((subh / m) mask)
//   for each contact (n_c, d_c) in (object, triangle) order with d_c < thickness:
//         { if v'.n_c < 0: v' -= (v'.n_c) n_c;  x += (thickness - d_c) n_c }
//   x'  = x + v' (subh mask)
//
// Contacts: the cloth's swept box (x and x + v subh over its vertices) culls
// each obstacle by its root box; the point query box x +- margin selects
// every face whose exact AABB it overlaps (queryPoints, bvh.metal:1322-1412),
// and narrow_pt_tri (bruteforce.metal:41-178) runs in double on each.  The
// candidates come from the scene's float tree of the obstacle, queried with
// the double box rounded outward to float: a float box that contains the
// double one overlaps every leaf whose face AABB the double box overlaps, so
// the exact double test then sees the same faces as a search over all faces.
// The contacts of a vertex are kept sorted by face, so the order of the tree
// descent does not reach the result.
//
// Every operation is a single IEEE binary64 add, multiply, divide or square
// root (the library is built without contraction), in the order of the
// expressions above, so the rollout is the FP64 reference's bit for bit.
#pragma once

namespace ys {

struct dd3 { double x, y, z; };
__device__ __forceinline__ dd3 dm(double a, double b, double c) { return dd3{a, b, c}; }
__device__ __forceinline__ dd3 operator+(dd3 a, dd3 b) { return dm(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ dd3 operator-(dd3 a, dd3 b) { return dm(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ dd3 operator*(dd3 a, double s) { return dm(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ double ddot(dd3 a, dd3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ dd3 dcross(dd3 a, dd3 b) {
    return dm(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// One vertex's position / velocity / adjoint in binary64 (32-byte aligned:
// two 16-byte loads).
struct __align__(32) D4 { double x, y, z, w; };
__device__ __forceinline__ dd3 ldd(const D4* p, u32 i) { const D4 q = p[i]; return dm(q.x, q.y, q.z); }
__device__ __forceinline__ void std4(D4* p, u32 i, dd3 a) { p[i] = D4{a.x, a.y, a.z, 0.0}; }
__device__ __forceinline__ dd3 ldf(const float4* p, u32 i) {
    const float4 q = p[i];
    return dm((double)q.x, (double)q.y, (double)q.z);
}

// A contact of one step: normal and signed distance.
struct __align__(32) DContact { double nx, ny, nz, d; };

static constexpr u32 D64_CAP = 16;    // contacts kept per vertex and step
static constexpr int D64_SPLIT = 4;   // the contact search splits a vertex's descent at this depth
static constexpr u32 D64_LANES = 1u << D64_SPLIT;  // into this many threads, one per subtree
static constexpr u32 D64_LCAP = 8;    // contacts one of those threads may find
static constexpr int D64_STACK = 64;  // tree descent stack
static constexpr u32 D64_VISIT_CAP = 1u << 20;
// Block size of the per-vertex kernels (32 measured the same on the
// 128x128 rollout: the step kernel is bound by its divergent descents).
static constexpr u32 D64_BLOCK = 128;

// Order-preserving map of binary64 onto u64 (larger double, larger key), so
// that min / max are integer atomics; NaN is left out by the callers.
__device__ __forceinline__ unsigned long long dord(double d) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(d);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dunord(unsigned long long o) {
    const unsigned long long b = (o >> 63) ? (o & 0x7FFFFFFFFFFFFFFFull) : ~o;
    return __longlong_as_double((long long)b);
}

struct A64 {
    // the scene: obstacle positions (the current buffer; obstacles are
    // static), faces, trees, meshes, the cloth's target list
    const float4* sx;
    const uint4* F;
    const Node* nodes;
    const MeshDev* meshes;
    const u32* targets;
    const float4* ext;  // external forces or null (then g m)
    const float* mass;
    const float* mask;
    u32 tgt_begin, tgt_end, cloth, voff, nV, N;
    double gx, gy, gz, kair, kd, subh, thickness, margin, radius;
    const double* k;  // per-spring stiffness / rest length (canonical order)
    const double* L;
    // state of step t and the step's outputs (cloth vertices, local index)
    const D4* x;
    const D4* xp;
    const D4* v;
    D4* xn;
    D4* vn;
    DContact* cs;  // D64_CAP slots per vertex, sorted by (object, face)
    u32* cf;       // their face ids
    u32* cn;       // contacts per vertex
    // the contact search's output, per (vertex, subtree): D64_LCAP contacts
    // in search order, their face ids and target ordinals, the count
    DContact* ls;
    u32* lf;
    u32* lk;
    u32* ln;
    unsigned long long* box;  // cloth swept box: ~dord(min) x3 then dord(max) x3, all by atomicMax
    u32* status;
};

__device__ __forceinline__ double grid_k64(const A64& A, u32 sid) { return A.k[sid]; }

// narrow_pt_tri in double (the FP64 reference's restatement): the face's
// plane normal oriented by the previous position (the current one when the
// previous lies on the plane), a crossing or a distance below radius +
// margin, the barycentric test at the crossing point (or the current point).
__device__ __forceinline__ bool narrow64(dd3 qc, dd3 qp, dd3 t0, dd3 t1, dd3 t2, double radius, double margin,
                                         dd3& nout, double& dout) {
    const dd3 e0 = t1 - t0, e1 = t2 - t0;
    dd3 n = dcross(e0, e1);
    const double nl2 = ddot(n, n);
    if (nl2 < 1e-12) return false;
    n = n * (1.0 / sqrt(nl2));
    double dp = ddot(n, qp - t0), dc = ddot(n, qc - t0);
    const double dref = (dp != 0.0) ? dp : dc;
    if (dref < 0.0) {
        n = n * -1.0;
        dp = -dp;
        dc = -dc;
    }
    const bool crossed = dc < 0.0, inm = dc < radius + margin;
    if (!crossed && !inm) return false;
    const dd3 cp = (crossed && dp > 0.0) ? qp + (qc - qp) * (dp / (dp - dc)) : qc;
    const dd3 pc = cp - t0;
    const dd3 inplane = pc - n * ddot(n, pc);
    const double d00 = ddot(e0, e0), d01 = ddot(e0, e1), d11 = ddot(e1, e1), d20 = ddot(inplane, e0),
                 d21 = ddot(inplane, e1);
    const double den = d00 * d11 - d01 * d01;
    if (fabs(den) < 1e-12) return false;
    const double b = (d11 * d20 - d01 * d21) / den, c = (d00 * d21 - d01 * d20) / den, a = 1.0 - b - c;
    if (!(a >= 0.0 && b >= 0.0 && c >= 0.0)) return false;
    nout = n;
    dout = dc;
    return true;
}

// Force on cloth vertex i (local) from the state (x, v).
__device__ __forceinline__ dd3 force64(const A64& A, const D4* x, const D4* v, u32 i) {
    const u32 g = A.voff + i;
    const dd3 p = ldd(x, i), w = ldd(v, i);
    const double m = (double)A.mass[g];
    const dd3 f0 = A.ext ? ldf(A.ext, g) : dm(A.gx * m, A.gy * m, A.gz * m);
    dd3 f = f0 + w * A.kair;
    const int N = (int)A.N, row = (int)(i / A.N), col = (int)(i % A.N);
    grid_stencil(N, row, col, [&](int r, int c, int, u32 sid) {
        const u32 j = (u32)(r * N + c);
        const dd3 dx = ldd(x, j) - p, dv = ldd(v, j) - w;
        const double l = sqrt(ddot(dx, dx));
        if (l < 1e-7) return;
        const dd3 nd = dx * (1.0 / l);
        f = f + nd * (A.k[sid] * (l - A.L[sid]) + A.kd * ddot(dv, nd));
    });
    return f;
}

// Cloth swept box of step t: x and x + v subh over the cloth's vertices.
__global__ void __launch_bounds__(256) k_d64_box(A64 A) {
    unsigned long long r[6] = {0, 0, 0, 0, 0, 0};
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < A.nV; i += gridDim.x * blockDim.x) {
        const dd3 p = ldd(A.x, i), s = p + ldd(A.v, i) * A.subh;
        const double c[6] = {p.x, p.y, p.z, s.x, s.y, s.z};
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            if (c[q] != c[q]) continue;  // NaN: fmin / fmax skip it
            const int a = q % 3;
            const unsigned long long o = dord(c[q]);
            r[a] = max(r[a], ~o);
            r[3 + a] = max(r[3 + a], o);
        }
    }
    __shared__ unsigned long long sh[6][8];
    const u32 lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        unsigned long long v = r[q];
        for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
        if (lane == 0) sh[q][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        unsigned long long v = 0;
        for (u32 w = 0; w < (blockDim.x >> 5); ++w) v = max(v, sh[threadIdx.x][w]);
        if (v) atomicMax(A.box + threadIdx.x, v);
    }
}

// Contact search of one step, D64_LANES threads per vertex: thread j of a
// vertex descends the subtree reached from the root by the bits of j (high
// bit first) over D64_SPLIT levels; a leaf met above that depth belongs to
// the thread whose remaining bits are zero.  Together the threads visit
// every root-to-leaf path the one-thread descent visits, with D64_LANES
// times the threads in flight (a 128x128 cloth is otherwise 512 warps, and
// the descents' dependent loads are the step's time).
__global__ void __launch_bounds__(D64_BLOCK) k_d64_cand(A64 A) {
    const u32 tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= A.nV * D64_LANES) return;
    const u32 i = tid / D64_LANES, j = tid % D64_LANES;
    const dd3 p = ldd(A.x, i), pp = ldd(A.xp, i);
    DContact* ls = A.ls + (size_t)tid * D64_LCAP;
    u32* lf = A.lf + (size_t)tid * D64_LCAP;
    u32* lk = A.lk + (size_t)tid * D64_LCAP;
    u32 n = 0, st = 0;
    const dd3 blo = dm(dunord(~A.box[0]), dunord(~A.box[1]), dunord(~A.box[2]));
    const dd3 bhi = dm(dunord(A.box[3]), dunord(A.box[4]), dunord(A.box[5]));
    const dd3 qmn = p - dm(A.margin, A.margin, A.margin), qmx = p + dm(A.margin, A.margin, A.margin);
    const float4 flo = make_float4(__double2float_rd(qmn.x), __double2float_rd(qmn.y), __double2float_rd(qmn.z), 0.f);
    const float4 fhi = make_float4(__double2float_ru(qmx.x), __double2float_ru(qmx.y), __double2float_ru(qmx.z), 0.f);
    for (u32 k = A.tgt_begin; k < A.tgt_end; ++k) {
        const u32 t = A.targets[k];
        const MeshDev& T = A.meshes[t];
        if (t == A.cloth || T.nF == 0 || (T.flags & MF_ANALYTIC)) continue;
        const Node* nodes = A.nodes + T.node_off;
        const Node root = nodes[0];
        if (bhi.x < (double)root.mnx || blo.x > (double)root.mxx || bhi.y < (double)root.mny ||
            blo.y > (double)root.mxy || bhi.z < (double)root.mnz || blo.z > (double)root.mxz)
            continue;
        const u32 nn = 2 * T.nF - 1;
        // this thread's subtree
        int id = 0;
        bool mine = true;
        for (int L = 0; L < D64_SPLIT; ++L) {
            const Node q = nodes[id];
            if (fhi.x < q.mnx || flo.x > q.mxx || fhi.y < q.mny || flo.y > q.mxy || fhi.z < q.mnz || flo.z > q.mxz) {
                mine = false;
                break;
            }
            if (q.a < 0) {  // a leaf above the split depth
                mine = (j & ((1u << (D64_SPLIT - L)) - 1u)) == 0u;
                break;
            }
            id = ((j >> (D64_SPLIT - 1 - L)) & 1u) ? q.b : q.a;
            if (id < 0 || (u32)id >= nn) { mine = false; break; }
        }
        if (!mine) continue;
        int stack[D64_STACK];
        int sp = 1;
        stack[0] = id;
        u32 visited = 0;
        while (sp > 0) {
            if (++visited > D64_VISIT_CAP) { st |= YS_FLAG_STACK_OVF; break; }
            const int nid = stack[--sp];
            if (nid < 0 || (u32)nid >= nn) continue;
            const Node q = nodes[nid];
            if (fhi.x < q.mnx || flo.x > q.mxx || fhi.y < q.mny || flo.y > q.mxy || fhi.z < q.mnz || flo.z > q.mxz)
                continue;
            if (q.a >= 0) {
                if (sp + 2 > D64_STACK) { st |= YS_FLAG_STACK_OVF; continue; }
                stack[sp++] = q.a;
                stack[sp++] = q.b;
                continue;
            }
            const u32 f = (u32)q.b;
            if (f >= T.nF) continue;
            const uint4 tri = A.F[T.foff + f];
            const dd3 t0 = ldf(A.sx, T.voff + tri.x), t1 = ldf(A.sx, T.voff + tri.y), t2 = ldf(A.sx, T.voff + tri.z);
            const double mnx = fmin(t0.x, fmin(t1.x, t2.x)), mxx = fmax(t0.x, fmax(t1.x, t2.x));
            const double mny = fmin(t0.y, fmin(t1.y, t2.y)), mxy = fmax(t0.y, fmax(t1.y, t2.y));
            const double mnz = fmin(t0.z, fmin(t1.z, t2.z)), mxz = fmax(t0.z, fmax(t1.z, t2.z));
            if (qmx.x < mnx || qmn.x > mxx || qmx.y < mny || qmn.y > mxy || qmx.z < mnz || qmn.z > mxz) continue;
            dd3 cn;
            double cd;
            if (!narrow64(p, pp, t0, t1, t2, A.radius, A.margin, cn, cd)) continue;
            if (n >= D64_LCAP) { st |= YS_FLAG_CONTACT_OVF; continue; }
            ls[n] = DContact{cn.x, cn.y, cn.z, cd};
            lf[n] = f;
            lk[n] = k - A.tgt_begin;
            ++n;
        }
    }
    A.ln[tid] = n;
    if (st) atomicOr(A.status, st);
}

// One step of the FP64 rollout for each vertex: its contacts from the
// search threads merged into one list sorted by (object, face) (a face
// reported twice -- the reference tree layout over runs of equal codes -- is
// one candidate, as in a search over all faces; recorded in cs / cf / cn),
// then forces, integration and the contact response.
__global__ void __launch_bounds__(D64_BLOCK) k_d64_step(A64 A) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nV) return;
    const u32 g = A.voff + i;
    const dd3 p = ldd(A.x, i);
    DContact* cs = A.cs + (size_t)i * D64_CAP;
    u32* cf = A.cf + (size_t)i * D64_CAP;
    unsigned long long key[D64_CAP];
    u32 n = 0, st = 0;
    for (u32 j = 0; j < D64_LANES; ++j) {
        const u32 tid = i * D64_LANES + j;
        const u32 m = min(A.ln[tid], D64_LCAP);
        for (u32 c = 0; c < m; ++c) {
            const size_t o = (size_t)tid * D64_LCAP + c;
            const unsigned long long kc = ((unsigned long long)A.lk[o] << 32) | A.lf[o];
            bool seen = false;
            for (u32 e = 0; e < n && !seen; ++e) seen = key[e] == kc;
            if (seen) continue;
            if (n >= D64_CAP) { st |= YS_FLAG_CONTACT_OVF; continue; }
            u32 s2 = n++;
            while (s2 > 0 && key[s2 - 1] > kc) {
                key[s2] = key[s2 - 1];
                cs[s2] = cs[s2 - 1];
                cf[s2] = cf[s2 - 1];
                --s2;
            }
            key[s2] = kc;
            cs[s2] = A.ls[o];
            cf[s2] = A.lf[o];
        }
    }
    A.cn[i] = n;
    const dd3 f = force64(A, A.x, A.v, i);
    const double m = (double)A.mass[g], mk_ = (double)A.mask[g];
    dd3 vel = ldd(A.v, i) + f * (A.subh / m * mk_);
    dd3 pos = p;
    for (u32 c = 0; c < n; ++c) {
        const DContact C = cs[c];
        const dd3 nc = dm(C.nx, C.ny, C.nz);
        if (C.d < A.thickness) {
            const double vn = ddot(vel, nc);
            if (vn < 0.0) vel = vel - nc * vn;
            pos = pos + nc * (A.thickness - C.d);
        }
    }
    pos = pos + vel * (A.subh * mk_);
    std4(A.xn, i, pos);
    std4(A.vn, i, vel);
    if (!isfinite(pos.x) || !isfinite(pos.y) || !isfinite(pos.z) || !isfinite(vel.x) || !isfinite(vel.y) ||
        !isfinite(vel.z))
        st |= YS_FLAG_NONFINITE;
    if (st) atomicOr(A.status, st);
}

struct J64 {
    const D4* ax;  // dL/dx_{t+1}, dL/dv_{t+1}
    const D4* av;
    D4* xbar;
    D4* vbar;
    D4* fbar;
    D4* ax_out;
    D4* av_out;
    double* gk;  // per-spring accumulators
    double* gL;
};

// Reverse of the integration and the contact response of step t (the
// forward's active set replayed from the recorded contacts).
__global__ void __launch_bounds__(D64_BLOCK) k_d64_adj_vertex(A64 A, J64 J) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nV) return;
    const u32 g = A.voff + i;
    const DContact* cs = A.cs + (size_t)i * D64_CAP;
    const u32 n = A.cn[i] < D64_CAP ? A.cn[i] : D64_CAP;
    const dd3 f = force64(A, A.x, A.v, i);
    const double m = (double)A.mass[g], mk_ = (double)A.mask[g];
    const double s = A.subh / m * mk_;
    dd3 vel = ldd(A.v, i) + f * s;
    u32 proj = 0;
    for (u32 c = 0; c < n; ++c) {
        const DContact C = cs[c];
        if (C.d < A.thickness) {
            const dd3 nc = dm(C.nx, C.ny, C.nz);
            const double vn = ddot(vel, nc);
            if (vn < 0.0) {
                vel = vel - nc * vn;
                proj |= 1u << c;
            }
        }
    }
    const dd3 axi = ldd(J.ax, i);
    dd3 vb = ldd(J.av, i) + axi * (A.subh * mk_);
    for (int c = (int)n - 1; c >= 0; --c)
        if (proj >> c & 1u) {
            const DContact C = cs[c];
            const dd3 nc = dm(C.nx, C.ny, C.nz);
            vb = vb - nc * ddot(nc, vb);
        }
    dd3 xb = axi;
    for (u32 c = 0; c < n; ++c) {
        const DContact C = cs[c];
        if (C.d < A.thickness) {
            const dd3 nc = dm(C.nx, C.ny, C.nz);
            xb = xb - nc * ddot(nc, axi);
        }
    }
    std4(J.xbar, i, xb);
    std4(J.vbar, i, vb);
    std4(J.fbar, i, vb * s);
}

// Reverse of the spring and drag forces of step t: gathered per vertex, the
// spring parameters' gradients accumulated by the lower-index end.
__global__ void __launch_bounds__(D64_BLOCK) k_d64_adj_springs(A64 A, J64 J) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nV) return;
    const int N = (int)A.N, row = (int)(i / A.N), col = (int)(i % A.N);
    const dd3 p = ldd(A.x, i), w = ldd(A.v, i), fi = ldd(J.fbar, i);
    const double kd = A.kd;
    dd3 dxb = dm(0.0, 0.0, 0.0), dvb = dm(0.0, 0.0, 0.0);
    grid_stencil(N, row, col, [&](int r, int c, int, u32 sid) {
        const u32 j = (u32)(r * N + c);
        const dd3 dx = ldd(A.x, j) - p, dv = ldd(A.v, j) - w;
        const double l = sqrt(ddot(dx, dx));
        if (l < 1e-7) return;
        const double k = A.k[sid], rest = A.L[sid];
        const dd3 nd = dx * (1.0 / l);
        const double a = k * (l - rest) + kd * ddot(dv, nd);
        const dd3 gdir = fi - ldd(J.fbar, j);
        const double ng = ddot(nd, gdir);
        const dd3 dvp = dv - nd * ddot(nd, dv), gp = gdir - nd * ng;
        const dd3 ddx = nd * (k * ng) + dvp * (kd * ng / l) + gp * (a / l);
        const dd3 ddv = nd * (kd * ng);
        dxb = dxb - ddx;
        dvb = dvb - ddv;
        if (i < j) {  // one owner per spring: no race on the accumulators
            J.gk[sid] += (l - rest) * ng;
            J.gL[sid] += -k * ng;
        }
    });
    std4(J.ax_out, i, ldd(J.xbar, i) + dxb);
    std4(J.av_out, i, ldd(J.vbar, i) + (dvb + fi * A.kair));
}

__global__ void k_d64_from_f4(const float4* __restrict__ in, D4* __restrict__ out, u32 voff, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { const float4 q = in[voff + i]; out[i] = D4{(double)q.x, (double)q.y, (double)q.z, 0.0}; }
}
__global__ void k_d64_from_f3(const float* __restrict__ in, D4* __restrict__ out, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = D4{(double)in[3 * i], (double)in[3 * i + 1], (double)in[3 * i + 2], 0.0};
}
__global__ void k_d64_from_d3(const double* __restrict__ in, D4* __restrict__ out, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = D4{in[3 * i], in[3 * i + 1], in[3 * i + 2], 0.0};
}
__global__ void k_d64_to_f3(const D4* __restrict__ in, float* __restrict__ out, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { const D4 q = in[i]; out[3 * i] = (float)q.x; out[3 * i + 1] = (float)q.y; out[3 * i + 2] = (float)q.z; }
}
__global__ void k_d64_to_d3(const D4* __restrict__ in, double* __restrict__ out, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { const D4 q = in[i]; out[3 * i] = q.x; out[3 * i + 1] = q.y; out[3 * i + 2] = q.z; }
}
__global__ void k_d64_widen(const float* __restrict__ in, double* __restrict__ out, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (double)in[i];
}
__global__ void k_d64_narrow(const double* __restrict__ in, float* __restrict__ out, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)in[i];
}

}  // namespace ys
