// ys_oracle.cpp -- CPU restatement of ysim's per-substep cloth hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: the CUDA path in
// ysim_b200/ is checked against it on identical seeded inputs.  Nothing in the
// product links, imports or calls it; only tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline / --impl reference legs load it.
//
// Each function restates one step of the reference (yeduk3/ysim) and cites the
// file:line it follows.  Compiled with -O3 -ffp-contract=off so every float op
// is a single IEEE-754 binary32 operation in source order (no FMA), which is
// the arithmetic the CUDA kernels reproduce with -fmad=false.
//
// Pinning: the restatement is checked against the reference's own Metal
// kernels compiled for the host (oracle/_ref, built by oracle/build_ref.py
// when the reference sources are present) and against brute-force
// enumerations for the candidate sets (tests/test_oracle_*.py).
//
// Documented deviations from the Metal build:
//   * rsqrt(x) (fast, bruteforce.metal:118, physics.metal:276) is written as
//     1.0f / sqrtf(x) (IEEE) on both sides.
//   * integrate reads the per-vertex mass m[v] where physics.metal:250 reads
//     m[id] from the 3V mass array; identical for the per-mesh-uniform masses
//     every scene uses.
//   * contacts of one vertex are applied in canonical (target object,
//     triangle) order; the reference's GPU bucketing order is nondeterministic
//     (physics.metal:596-599).
#include <algorithm>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

typedef uint32_t u32;
typedef int32_t i32;

struct V3 { float x, y, z; };
inline V3 v3(float a, float b, float c) { V3 r = {a, b, c}; return r; }
inline V3 ld3(const float* p, u32 i) { return v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
inline void st3(float* p, u32 i, V3 a) { p[3 * i] = a.x; p[3 * i + 1] = a.y; p[3 * i + 2] = a.z; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
inline V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
inline V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
inline V3 operator/(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
// dot = ((a.x*b.x + a.y*b.y) + a.z*b.z), left to right.
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// tinym::min/max (tinym.hpp:424-447): a > b ? b : a  /  a < b ? b : a.
inline float tmin(float a, float b) { return a > b ? b : a; }
inline float tmax(float a, float b) { return a < b ? b : a; }
inline V3 vmin(V3 a, V3 b) { return v3(tmin(a.x, b.x), tmin(a.y, b.y), tmin(a.z, b.z)); }
inline V3 vmax(V3 a, V3 b) { return v3(tmax(a.x, b.x), tmax(a.y, b.y), tmax(a.z, b.z)); }

inline u32 fbits(float f) { u32 u; std::memcpy(&u, &f, 4); return u; }
inline bool nonfinite3(V3 p) {
    return ((fbits(p.x) & 0x7F800000u) == 0x7F800000u) ||
           ((fbits(p.y) & 0x7F800000u) == 0x7F800000u) ||
           ((fbits(p.z) & 0x7F800000u) == 0x7F800000u);
}
inline int clz32(u32 v) { return v ? __builtin_clz(v) : 32; }

// BVHNode, 32 B (bvh.hpp:148-177, bvh.metal:14-19): leaf childA = -1, childB = primitive.
struct Node { float mn[3]; i32 a; float mx[3]; i32 b; };
static_assert(sizeof(Node) == 32, "node");
// BroadCollision, 32 B (collision_pod.hpp:256-261).
struct Row { u32 point, tri, qobj, tobj, qbeh, tbeh, qshape, tshape; };
static_assert(sizeof(Row) == 32, "row");
// NarrowCollision, 48 B (collision_pod.hpp:274-280).
struct Contact { u32 point, tri, qobj, tobj; float n[3]; float d; u32 qbeh, tbeh, qshape, tshape; };
static_assert(sizeof(Contact) == 48, "contact");

inline V3 nmin(const Node& n) { return v3(n.mn[0], n.mn[1], n.mn[2]); }
inline V3 nmax(const Node& n) { return v3(n.mx[0], n.mx[1], n.mx[2]); }
inline void nset(Node& n, V3 lo, V3 hi) {
    n.mn[0] = lo.x; n.mn[1] = lo.y; n.mn[2] = lo.z;
    n.mx[0] = hi.x; n.mx[1] = hi.y; n.mx[2] = hi.z;
}

// ---------------------------------------------------------------- M1 Morton
// Scene box over ALL vertices of one mesh (bvh.hpp:1229-1231).
void scene_box(const float* x, u32 nV, float out[6]) {
    V3 lo = ld3(x, 0), hi = lo;
    for (u32 i = 1; i < nV; ++i) { V3 p = ld3(x, i); lo = vmin(p, lo); hi = vmax(p, hi); }
    out[0] = lo.x; out[1] = lo.y; out[2] = lo.z; out[3] = hi.x; out[4] = hi.y; out[5] = hi.z;
}
// expandBits / mortonCode / fillMortons_Tri (bvh.metal:26-63): Metal semantics
// (width clamped to >= 1e-8), IEEE division.
inline u32 expand_bits(u32 v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
inline float clamp01023(float v) { return std::fmin(std::fmax(v, 0.f), 1023.f); }
inline u32 morton_of(V3 c) {
    V3 p = c * 1024.f;
    return expand_bits((u32)clamp01023(p.x)) * 4 + expand_bits((u32)clamp01023(p.y)) * 2 +
           expand_bits((u32)clamp01023(p.z));
}
void fill_mortons(const float* x, const u32* F, u32 nM, const float box[6], u32* codes, u32* idx) {
    V3 bmin = v3(box[0], box[1], box[2]), bmax = v3(box[3], box[4], box[5]);
    V3 w = bmax - bmin;
    w = v3(std::fmax(w.x, 1e-8f), std::fmax(w.y, 1e-8f), std::fmax(w.z, 1e-8f));
    for (u32 i = 0; i < nM; ++i) {
        V3 c = (ld3(x, F[3 * i]) + ld3(x, F[3 * i + 1]) + ld3(x, F[3 * i + 2])) / 3.0f;
        c = (c - bmin) / w;
        codes[i] = morton_of(c);
        idx[i] = i;
    }
}

// ---------------------------------------------------------------- S1 radix
// Stable LSD radix sort, 8-bit digits, 4 passes over the full key, value
// carried (radixSortCPU, bvh.hpp:723-765).
void radix_sort(u32* key, u32* val, u32 n) {
    std::vector<u32> k2(n), v2(n);
    u32 *sk = key, *sv = val, *dk = k2.data(), *dv = v2.data();
    for (int shift = 0; shift < 32; shift += 8) {
        size_t cnt[256] = {0};
        for (u32 i = 0; i < n; ++i) cnt[(sk[i] >> shift) & 255u]++;
        size_t off[256], s = 0;
        for (int b = 0; b < 256; ++b) { off[b] = s; s += cnt[b]; }
        for (u32 i = 0; i < n; ++i) {
            u32 b = (sk[i] >> shift) & 255u;
            dk[off[b]] = sk[i]; dv[off[b]] = sv[i]; off[b]++;
        }
        std::swap(sk, dk); std::swap(sv, dv);
    }
    if (sk != key) { std::memcpy(key, sk, n * 4); std::memcpy(val, sv, n * 4); }
}

// ---------------------------------------------------------------- K1 Karras
// delta / determineRange / findSplit / buildTree_Tri (bvh.metal:197-258, 352-393).
struct Karras {
    const u32* c; const u32* ix; int n;
    int delta(int i, int j) const {
        if (j < 0 || j >= n) return -1;
        if (c[i] != c[j]) return clz32(c[i] ^ c[j]);
        return 32 + clz32(ix[i] ^ ix[j]);
    }
    void range(int i, int& first, int& last) const {
        int d = (delta(i, i + 1) - delta(i, i - 1) >= 0) ? 1 : -1;
        int dmin = delta(i, i - d);
        int lmax = 2;
        while (delta(i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        if (d < 0) { first = j; last = i; } else { first = i; last = j; }
    }
    u32 split(int i0, int i1) const {
        u32 c0 = c[i0], c1 = c[i1];
        if (c0 == c1) return (u32)((i0 + i1) >> 1);
        int prefix = clz32(c0 ^ c1);
        u32 s = (u32)i0, step = (u32)(i1 - i0);
        do {
            step = (step + 1) >> 1;
            u32 ns = s + step;
            if (ns < (u32)i1) {
                if (clz32(c0 ^ c[ns]) > prefix) s = ns;
            }
        } while (step > 1);
        return s;
    }
};
void karras_topology(const u32* codes, const u32* idx, u32 n, Node* tree, i32* parent) {
    Karras K{codes, idx, (int)n};
    for (u32 i = 0; i < n; ++i) { Node& L = tree[n - 1 + i]; L.a = -1; L.b = (i32)idx[i]; }
    // unclaimed nodes keep -1; a node claimed twice (runs of >= 3 equal codes)
    // keeps the last writer of this ascending loop, the largest claimant
    for (u32 i = 0; i + 1 < 2 * n; ++i) parent[i] = -1;
    for (int i = 0; i + 1 < (int)n; ++i) {
        int f, l; K.range(i, f, l);
        int s = (int)K.split(f, l);
        int ca = (s == f) ? s + (int)n - 1 : s;
        int cb = (s + 1 == l) ? s + (int)n : s + 1;
        tree[i].a = ca; tree[i].b = cb;
        parent[ca] = i; parent[cb] = i;
    }
}

// ---------------------------------------------------------------- R1/R2 refit
// buildLeaf_Tri (bvh.metal:260-283) / buildSweptLeaf_Tri (bvh.metal:323-351):
// leaf box = min/max of the 3 verts, or of {x, x + v*dt} when swept.
void leaves(const float* x, const float* v, float dt, int swept, const u32* F, u32 n, Node* tree) {
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) {
        Node& L = tree[n - 1 + i];
        u32 f = (u32)L.b;
        V3 lo, hi;
        for (int k = 0; k < 3; ++k) {
            u32 vid = F[3 * f + k];
            V3 p = ld3(x, vid);
            V3 a = p, b = p;
            if (swept) { V3 s = p + ld3(v, vid) * dt; a = vmin(p, s); b = vmax(p, s); }
            if (k == 0) { lo = a; hi = b; } else { lo = vmin(lo, a); hi = vmax(hi, b); }
        }
        nset(L, lo, hi);
    }
}
// ---------------------------------------------------------------- K2 Apetrei
// agglomerativeBuild_Tri + agglomerativeSwapRoot (bvh.metal:884-1199).  Leaf i
// of the sorted order sits at slot N-1+i with its triangle's box.  Each leaf
// climbs: at range [L, R] it joins the side whose neighbouring key differs
// less (code XOR, ties by index XOR; a range touching an end can only grow the
// other way), so its parent is slot R (it is R's left child) or slot L-1 (the
// right child).  The first arrival at a node stops; the second combines the
// two boxes and climbs on with the node's full range.  The root, wherever it
// lands, is then moved to slot 0 and every link to either slot patched.
// Leaves run in order: a node's second arrival always comes from a later
// leaf, so this is the concurrent build's result.  Returns the slot the root
// was built in.
int apetrei_topology(const float* x, const u32* F, const u32* codes, const u32* idx, u32 n, Node* tree, i32* parent) {
    for (u32 i = 0; i < n; ++i) { tree[n - 1 + i].a = -1; tree[n - 1 + i].b = (i32)idx[i]; }
    leaves(x, nullptr, 0.f, 0, F, n, tree);
    if (n <= 1) return 0;
    const int N = (int)n;
    std::vector<u32> arrivals(n - 1, 0);
    std::vector<int> lo(n - 1, 0), hi(n - 1, 0);
    int root = -1;
    for (int id = 0; id < N; ++id) {
        int node = N - 1 + id, L = id, R = id;
        for (int step = 0; step < 2 * N; ++step) {
            if (L == 0 && R == N - 1) { root = node; break; }
            bool right;
            if (L == 0) right = true;
            else if (R == N - 1) right = false;
            else {
                const u32 dr = codes[R] ^ codes[R + 1], dl = codes[L - 1] ^ codes[L];
                right = (dr != dl) ? dr < dl : (idx[R] ^ idx[R + 1]) < (idx[L - 1] ^ idx[L]);
            }
            const int p = right ? R : L - 1;
            if (right) { tree[p].a = node; lo[p] = L; }
            else { tree[p].b = node; hi[p] = R; }
            parent[node] = p;
            if (arrivals[p]++ == 0) break;
            const Node& A = tree[tree[p].a];
            const Node& B = tree[tree[p].b];
            nset(tree[p], vmin(nmin(A), nmin(B)), vmax(nmax(A), nmax(B)));
            node = p; L = lo[p]; R = hi[p];
        }
    }
    const int k = root;
    if (k > 0) {
        const Node Rn = tree[k], O = tree[0];
        const int p0 = parent[0];
        const int ra = Rn.a == 0 ? k : Rn.a, rb = Rn.b == 0 ? k : Rn.b;
        tree[0] = Rn; tree[0].a = ra; tree[0].b = rb;
        tree[k] = O;
        parent[O.a] = k; parent[O.b] = k;
        parent[ra] = 0; parent[rb] = 0;
        if (p0 != k) {
            if (tree[p0].a == 0) tree[p0].a = k; else tree[p0].b = k;
            parent[k] = p0;
        }
        parent[0] = -1;
    }
    return root;
}

// bottomUpCombine (bvh.hpp:1534-1553): parent = min/max of children, exact.
void bottom_up(Node* tree, u32 nNodes) {
    if (nNodes == 0) return;
    std::vector<std::pair<int, bool>> st;
    st.emplace_back(0, false);
    while (!st.empty()) {
        auto e = st.back(); st.pop_back();
        Node& nd = tree[e.first];
        if (nd.a < 0) continue;
        if (!e.second) { st.emplace_back(e.first, true); st.emplace_back(nd.a, false); st.emplace_back(nd.b, false); }
        else nset(nd, vmin(nmin(tree[nd.a]), nmin(tree[nd.b])), vmax(nmax(tree[nd.a]), nmax(tree[nd.b])));
    }
}

// ---------------------------------------------------------------- H2 GPU hash
// SpatialHashing<METAL>::detectCollisions (spatial_hash.hpp:880-960; kernels
// spatialhashing.metal:64-478), the Pabst face-face hash, restated per cell:
//   * bounding sphere per face: centroid ((v0+v1)+v2)*(1/3), radius =
//     |centroid - v0| (sh_buildBV :84-87 uses v0 only);
//   * grid: scene box over all vertices, cell = 2*maxR*1 + margin, res =
//     ceil(extent/cell) >= 1 per axis (computeGrid :343-400);
//   * home cell (floor, clamped) plus the octant's phantom cells whose wall
//     is within r (sh_assignCells :143-238); a face's type mask holds the
//     parity types (x&1 | y&1<<1 | z&1<<2) of every cell it entered;
//   * in each cell, home-home and home-phantom pairs (phantom-phantom pairs
//     are not candidates, :292-301), dropped when self pairs are off and
//     both faces share a mesh, when both meshes are Float, when the type
//     masks share a type below the cell's (the marking dedup), or when the
//     centroids are farther apart than rA + rB + margin; each survivor gives
//     6 rows: A's vertices against B's face and B's against A's (:440-477).
struct ShHit { u32 cell; u32 face; bool phantom; };
void sh_face_face(const float* x, const u32* stateOff, const u32* F, const u32* facetOff, const u32* beh,
                  const u32* shape, u32 nM, float margin, bool self, std::vector<Row>& rows, u32 stats[6]) {
    for (int k = 0; k < 6; ++k) stats[k] = 0;
    const u32 nV = stateOff[nM], nF = facetOff[nM];
    if (nF == 0 || nV == 0) return;
    std::vector<u32> obj(nF);
    for (u32 m = 0; m < nM; ++m)
        for (u32 f = facetOff[m]; f < facetOff[m + 1]; ++f) obj[f] = m;
    std::vector<V3> c(nF);
    std::vector<float> r(nF);
    float maxR = 0.f;
    for (u32 f = 0; f < nF; ++f) {
        const u32 vb = stateOff[obj[f]];
        const V3 a = ld3(x, vb + F[3 * f]), b = ld3(x, vb + F[3 * f + 1]), d = ld3(x, vb + F[3 * f + 2]);
        c[f] = (a + b + d) * (1.0f / 3.0f);
        const V3 e = c[f] - a;
        r[f] = std::sqrt(dot(e, e));
        maxR = tmax(maxR, r[f]);
    }
    V3 lo = ld3(x, 0), hi = lo;
    for (u32 v = 0; v < nV; ++v) { lo = vmin(lo, ld3(x, v)); hi = vmax(hi, ld3(x, v)); }
    float cs = 2.0f * maxR * 1.0f + margin;
    if (cs <= 0.f) cs = std::max(margin, 1e-6f);
    const float o[3] = {lo.x, lo.y, lo.z}, ext[3] = {hi.x - lo.x, hi.y - lo.y, hi.z - lo.z};
    int res[3];
    for (int k = 0; k < 3; ++k) {
        u32 q = (u32)std::ceil(ext[k] / cs);
        res[k] = (int)(q == 0 ? 1 : q);
    }
    std::vector<ShHit> hits;
    std::vector<u32> mask(nF, 0u);
    const float hcs = cs * 0.5f;
    for (u32 f = 0; f < nF; ++f) {
        const float cc[3] = {c[f].x, c[f].y, c[f].z};
        int g[3], sg[3];
        float dist[3];
        for (int k = 0; k < 3; ++k) {
            g[k] = (int)std::floor((cc[k] - o[k]) / cs);
            g[k] = std::min(std::max(g[k], 0), res[k] - 1);
            const float local = cc[k] - (o[k] + (float)g[k] * cs);
            sg[k] = local > hcs ? 1 : -1;
            dist[k] = sg[k] > 0 ? cs - local : local;
        }
        for (int i = 0; i <= 1; ++i) {
            if (i && dist[0] > r[f]) continue;
            for (int j = 0; j <= 1; ++j) {
                if (j && dist[1] > r[f]) continue;
                for (int k = 0; k <= 1; ++k) {
                    if (k && dist[2] > r[f]) continue;
                    const int p[3] = {g[0] + i * sg[0], g[1] + j * sg[1], g[2] + k * sg[2]};
                    if (p[0] < 0 || p[0] >= res[0] || p[1] < 0 || p[1] >= res[1] || p[2] < 0 || p[2] >= res[2])
                        continue;
                    mask[f] |= 1u << ((p[0] & 1) | ((p[1] & 1) << 1) | ((p[2] & 1) << 2));
                    const u32 id = ((u32)p[2] * (u32)res[1] + (u32)p[1]) * (u32)res[0] + (u32)p[0];
                    hits.push_back(ShHit{id, f, (i | j | k) != 0});
                }
            }
        }
    }
    std::stable_sort(hits.begin(), hits.end(), [](const ShHit& a, const ShHit& b) { return a.cell < b.cell; });
    stats[0] = (u32)hits.size();
    stats[3] = (u32)res[0]; stats[4] = (u32)res[1]; stats[5] = (u32)res[2];
    auto emit = [&](u32 A, u32 B) {
        const u32 oA = obj[A], oB = obj[B];
        for (int side = 0; side < 2; ++side) {
            const u32 P = side ? B : A, T = side ? A : B, oP = obj[P], oT = obj[T];
            for (int k = 0; k < 3; ++k)
                rows.push_back(Row{F[3 * P + k], T - facetOff[oT], oP, oT, beh[oP], beh[oT], shape[oP], shape[oT]});
        }
        (void)oA; (void)oB;
    };
    for (size_t b = 0; b < hits.size();) {
        size_t e = b;
        while (e < hits.size() && hits[e].cell == hits[b].cell) ++e;
        ++stats[1];
        const u32 id = hits[b].cell;
        const u32 gx = id % (u32)res[0], gy = (id / (u32)res[0]) % (u32)res[1], gz = id / ((u32)res[0] * (u32)res[1]);
        const u32 below = (1u << ((gx & 1u) | ((gy & 1u) << 1) | ((gz & 1u) << 2))) - 1u;
        std::vector<u32> home, ph;
        for (size_t q = b; q < e; ++q) (hits[q].phantom ? ph : home).push_back(hits[q].face);
        auto test = [&](u32 A, u32 B) {
            ++stats[2];
            if (!self && obj[A] == obj[B]) return;
            if (beh[obj[A]] == 4u && beh[obj[B]] == 4u) return;  // Float-Float
            if (mask[A] & mask[B] & below) return;
            const V3 d = c[A] - c[B];
            if (std::sqrt(dot(d, d)) > r[A] + r[B] + margin) return;
            emit(A, B);
        };
        for (size_t i = 0; i < home.size(); ++i)
            for (size_t j = i + 1; j < home.size(); ++j) test(home[i], home[j]);
        for (u32 h : home)
            for (u32 p : ph) test(h, p);
        b = e;
    }
}

// ---------------------------------------------------------------- Q1 query
// intersectAABB (bvh.metal:1285-1290), inclusive.
inline bool overlap(V3 qmn, V3 qmx, const Node& n) {
    if (qmx.x < n.mn[0] || qmn.x > n.mx[0]) return false;
    if (qmx.y < n.mn[1] || qmn.y > n.mx[1]) return false;
    if (qmx.z < n.mn[2] || qmn.z > n.mx[2]) return false;
    return true;
}
// queryPoints/queryAABB (bvh.metal:1322-1412): DFS from slot 0, push childA
// then childB; self queries skip the triangles that contain the point.
template <class Emit>
void query_point(const Node* tree, u32 nNodes, const u32* F, V3 p, float m, u32 pid, bool self, Emit emit) {
    if (nNodes == 0) return;
    V3 qmn = p - v3(m, m, m), qmx = p + v3(m, m, m);
    int st[64]; int sp = 0; st[sp++] = 0;
    while (sp > 0) {
        int id = st[--sp];
        const Node& n = tree[id];
        if (!overlap(qmn, qmx, n)) continue;
        if (n.a < 0) {
            u32 f = (u32)n.b;
            if (self && (F[3 * f] == pid || F[3 * f + 1] == pid || F[3 * f + 2] == pid)) continue;
            emit(f);
            continue;
        }
        if (sp + 2 > 64) continue;
        st[sp++] = n.a; st[sp++] = n.b;
    }
}

// ---------------------------------------------------------------- H1 CPU hash
// pointTriSq (spatial_hash.hpp:1659-1711), Ericson closest point, same op order.
float point_tri_sq(const float p[3], const float a[3], const float b[3], const float c[3]) {
    auto dt = [](const float* u, const float* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
    float ab[3], ac[3], ap[3], q[3];
    for (int i = 0; i < 3; ++i) { ab[i] = b[i] - a[i]; ac[i] = c[i] - a[i]; ap[i] = p[i] - a[i]; }
    const float d1 = dt(ab, ap), d2 = dt(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f) { for (int i = 0; i < 3; ++i) q[i] = a[i]; }
    else {
        float bp[3]; for (int i = 0; i < 3; ++i) bp[i] = p[i] - b[i];
        const float d3 = dt(ab, bp), d4 = dt(ac, bp);
        if (d3 >= 0.f && d4 <= d3) { for (int i = 0; i < 3; ++i) q[i] = b[i]; }
        else {
            const float vc = d1 * d4 - d3 * d2;
            if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
                const float den = d1 - d3;
                const float vv = (den != 0.f) ? d1 / den : 0.f;
                for (int i = 0; i < 3; ++i) q[i] = a[i] + vv * ab[i];
            } else {
                float cp[3]; for (int i = 0; i < 3; ++i) cp[i] = p[i] - c[i];
                const float d5 = dt(ab, cp), d6 = dt(ac, cp);
                if (d6 >= 0.f && d5 <= d6) { for (int i = 0; i < 3; ++i) q[i] = c[i]; }
                else {
                    const float vb = d5 * d2 - d1 * d6;
                    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
                        const float den = d2 - d6;
                        const float w = (den != 0.f) ? d2 / den : 0.f;
                        for (int i = 0; i < 3; ++i) q[i] = a[i] + w * ac[i];
                    } else {
                        const float va = d3 * d6 - d5 * d4;
                        if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
                            const float den = (d4 - d3) + (d5 - d6);
                            const float w = (den != 0.f) ? (d4 - d3) / den : 0.f;
                            for (int i = 0; i < 3; ++i) q[i] = b[i] + w * (c[i] - b[i]);
                        } else {
                            const float den = va + vb + vc;
                            const float vv = (den != 0.f) ? vb / den : 0.f;
                            const float w = (den != 0.f) ? vc / den : 0.f;
                            for (int i = 0; i < 3; ++i) q[i] = a[i] + ab[i] * vv + ac[i] * w;
                        }
                    }
                }
            }
        }
    }
    float s = 0.f;
    for (int i = 0; i < 3; ++i) { const float e = p[i] - q[i]; s += e * e; }
    return s;
}

// Face key boxes (collectFaceBoxes, spatial_hash.hpp:1613-1655): tri AABB
// inflated by m, non-finite faces dropped; returns the largest axis extent.
struct FaceRec { float bmin[3], bmax[3]; u32 face; };
float face_boxes(const float* x, const u32* F, u32 nF, float m, std::vector<FaceRec>& out) {
    out.clear();
    float maxExt = 0.f;
    for (u32 f = 0; f < nF; ++f) {
        FaceRec r; bool ok = true;
        for (int a = 0; a < 3; ++a) {
            float p0 = x[3 * F[3 * f] + a], p1 = x[3 * F[3 * f + 1] + a], p2 = x[3 * F[3 * f + 2] + a];
            if (!std::isfinite(p0) || !std::isfinite(p1) || !std::isfinite(p2)) { ok = false; break; }
            float lo = std::min(p0, std::min(p1, p2)), hi = std::max(p0, std::max(p1, p2));
            r.bmin[a] = lo - m; r.bmax[a] = hi + m;
        }
        if (!ok) continue;
        r.face = f;
        for (int a = 0; a < 3; ++a) maxExt = std::max(maxExt, r.bmax[a] - r.bmin[a]);
        out.push_back(r);
    }
    return maxExt;
}
inline uint64_t cell_key(int32_t x, int32_t y, int32_t z) {
    const uint64_t ux = (uint64_t)(u32)(x + 0x100000) & 0x1FFFFFull;
    const uint64_t uy = (uint64_t)(u32)(y + 0x100000) & 0x1FFFFFull;
    const uint64_t uz = (uint64_t)(u32)(z + 0x100000) & 0x1FFFFFull;
    return ux | (uy << 21) | (uz << 42);
}
// Self rows of one mesh (detectSelfCollisions + probeMeshVertices,
// spatial_hash.hpp:1740-1869 and 1946-1989): uniform grid with cell = largest
// inflated face extent; swept vertex box [min(x,xPrev), max(x,xPrev)] (xPrev
// replaced by x when non-finite or more than 1 m away); box precull; skip own
// faces; exact point-triangle distance^2 <= m^2 at x or xPrev.
// Rows come out vertex-major in the reference's cell/insert order.
void self_hash_rows(const float* x, const float* xp, u32 nV, const u32* F, u32 nF, float m,
                    std::vector<std::pair<u32, u32>>& rows) {
    std::vector<FaceRec> faces;
    float maxExt = face_boxes(x, F, nF, m, faces);
    if (faces.empty()) return;
    float cs = (maxExt > 1e-5f) ? maxExt : 1e-5f;
    float inv = 1.f / cs;
    std::unordered_map<uint64_t, std::vector<u32>> grid;
    for (u32 fi = 0; fi < (u32)faces.size(); ++fi) {
        const FaceRec& fr = faces[fi];
        int lo[3], hi[3]; bool sane = true;
        for (int a = 0; a < 3; ++a) {
            lo[a] = (int)std::floor(fr.bmin[a] * inv); hi[a] = (int)std::floor(fr.bmax[a] * inv);
            if (hi[a] - lo[a] > 64) { sane = false; break; }
        }
        if (!sane) continue;
        for (int z = lo[2]; z <= hi[2]; ++z)
            for (int y = lo[1]; y <= hi[1]; ++y)
                for (int xx = lo[0]; xx <= hi[0]; ++xx) grid[cell_key(xx, y, z)].push_back(fi);
    }
    const int nth =
#ifdef _OPENMP
        omp_get_max_threads();
#else
        1;
#endif
    std::vector<std::vector<std::pair<u32, u32>>> part(nth);
#pragma omp parallel
    {
        int tid =
#ifdef _OPENMP
            omp_get_thread_num();
#else
            0;
#endif
        std::vector<u32> seen;
        std::vector<std::pair<u32, u32>>& my = part[tid];
        // static chunking keeps vertex-major order after concatenation
#pragma omp for schedule(static)
        for (long long vl = 0; vl < (long long)nV; ++vl) {
            u32 v = (u32)vl;
            float vlo[3], vhi[3], pc3[3], pp3[3]; bool ok = true;
            for (int a = 0; a < 3; ++a) {
                float pc = x[3 * v + a], pp = xp[3 * v + a];
                if (!std::isfinite(pc)) { ok = false; break; }
                if (!std::isfinite(pp) || std::abs(pp - pc) > 1.f) pp = pc;
                pc3[a] = pc; pp3[a] = pp; vlo[a] = std::min(pc, pp); vhi[a] = std::max(pc, pp);
            }
            if (!ok) continue;
            int lo[3], hi[3]; bool sane = true;
            for (int a = 0; a < 3; ++a) {
                lo[a] = (int)std::floor(vlo[a] * inv); hi[a] = (int)std::floor(vhi[a] * inv);
                if (hi[a] - lo[a] > 64) { sane = false; break; }
            }
            if (!sane) continue;
            bool multi = (lo[0] != hi[0]) || (lo[1] != hi[1]) || (lo[2] != hi[2]);
            if (multi) seen.clear();
            for (int z = lo[2]; z <= hi[2]; ++z)
                for (int y = lo[1]; y <= hi[1]; ++y)
                    for (int xx = lo[0]; xx <= hi[0]; ++xx) {
                        auto it = grid.find(cell_key(xx, y, z));
                        if (it == grid.end()) continue;
                        for (u32 fi : it->second) {
                            if (multi) {
                                bool dup = false;
                                for (u32 s : seen) if (s == fi) { dup = true; break; }
                                if (dup) continue;
                                seen.push_back(fi);
                            }
                            const FaceRec& fr = faces[fi];
                            if (vhi[0] < fr.bmin[0] || vlo[0] > fr.bmax[0] || vhi[1] < fr.bmin[1] ||
                                vlo[1] > fr.bmax[1] || vhi[2] < fr.bmin[2] || vlo[2] > fr.bmax[2])
                                continue;
                            u32 f = fr.face;
                            if (F[3 * f] == v || F[3 * f + 1] == v || F[3 * f + 2] == v) continue;
                            float A[3], B[3], C[3];
                            for (int a = 0; a < 3; ++a) {
                                A[a] = x[3 * F[3 * f] + a]; B[a] = x[3 * F[3 * f + 1] + a]; C[a] = x[3 * F[3 * f + 2] + a];
                            }
                            const float m2 = m * m;
                            if (point_tri_sq(pc3, A, B, C) > m2 && point_tri_sq(pp3, A, B, C) > m2) continue;
                            my.emplace_back(v, f);
                        }
                    }
        }
    }
    for (auto& p : part) rows.insert(rows.end(), p.begin(), p.end());
}

// ---------------------------------------------------------------- N1 narrow
// pointInTriangleBary (bruteforce.metal:9-28).
inline bool point_in_tri(V3 p, V3 e0, V3 e1) {
    float d00 = dot(e0, e0), d01 = dot(e0, e1), d11 = dot(e1, e1), d20 = dot(p, e0), d21 = dot(p, e1);
    float den = d00 * d11 - d01 * d01;
    if (std::fabs(den) < 1e-12f) return false;
    float b = (d11 * d20 - d01 * d21) / den;
    float c = (d00 * d21 - d01 * d20) / den;
    float a = 1.0f - b - c;
    return (a >= 0.0f && b >= 0.0f && c >= 0.0f);
}
// narrow_pt_tri (bruteforce.metal:41-178) for one broad row; the self-row
// vertexAdjFacets skip is done by the caller.  Returns true and fills n, d on a
// contact.
inline bool narrow_one(V3 qcur, V3 qprev, V3 t0, V3 t1, V3 t2, float band, float n_out[3], float* d_out) {
    V3 e0 = t1 - t0, e1 = t2 - t0;
    V3 n = cross(e0, e1);
    float nl2 = dot(n, n);
    if (nl2 < 1e-12f) return false;
    n = n * (1.0f / std::sqrt(nl2));
    float dp = dot(n, qprev - t0), dc = dot(n, qcur - t0);
    float dref = (dp != 0.0f) ? dp : dc;
    if (dref < 0.0f) { n = -n; dp = -dp; dc = -dc; }
    bool crossed = dc < 0.0f, inm = dc < band;
    if (!crossed && !inm) return false;
    V3 cp;
    if (crossed && dp > 0.0f) { float t = dp / (dp - dc); cp = qprev + (qcur - qprev) * t; }
    else cp = qcur;
    V3 pc = cp - t0;
    float l = dot(n, pc);
    V3 inplane = pc - n * l;
    if (!point_in_tri(inplane, e0, e1)) return false;
    n_out[0] = n.x; n_out[1] = n.y; n_out[2] = n.z; *d_out = dc;
    return true;
}

// ---------------------------------------------------------------- analytic
// AnalyticShape (collision_pod.hpp:295-309): centerRadius, halfExtHeight,
// rotQuat (w,x,y,z), prevCenterPad, prevRotQuat, kind, objIndex,
// behaviorType, flags.  ColliderKind: 0 Mesh, 1 Sphere, 2 Box, 3 Cylinder,
// 4 Plane.
struct Shape {
    float cr[4], he[4], rq[4], pc[4], prq[4];
    u32 kind, obj, beh, flags;
};
static_assert(sizeof(Shape) == 96, "shape");
enum Collider : u32 { CMesh = 0, CSphere = 1, CBox = 2, CCyl = 3, CPlane = 4 };

inline float fmn(float a, float b) { return std::fmin(a, b); }
inline float fmx(float a, float b) { return std::fmax(a, b); }
inline float len(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 unit(V3 a) { return a * (1.0f / std::sqrt(dot(a, a))); }
inline V3 hadamard(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float axis_of(V3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
// quatRotate (bruteforce.metal:196-201): v + 2 * cross(qv, cross(qv, v) + qw * v).
inline V3 qrot(float qw, V3 qv, V3 v) { return v + 2.0f * cross(qv, cross(qv, v) + qw * v); }
// boxDominantAxis (bruteforce.metal:203-216).
inline void dominant_axis(V3 q, V3 h, int& k, float& sg) {
    V3 gap = v3(std::fabs(q.x) - h.x, std::fabs(q.y) - h.y, std::fabs(q.z) - h.z);
    k = 0;
    float best = gap.x;
    if (gap.y > best) { best = gap.y; k = 1; }
    if (gap.z > best) { best = gap.z; k = 2; }
    sg = axis_of(q, k) >= 0.0f ? 1.0f : -1.0f;
}

// narrow_pt_analytic (bruteforce.metal:259-499) for one vertex; band =
// radius + thickness + rotMargin.  Returns true with the world normal and
// signed distance when the vertex is in contact.
bool analytic_one(const Shape& sh, V3 pcur, V3 pprev, float radius, float thickness, float rot_margin,
                  float n_out[3], float* d_out) {
    if ((sh.flags & 1u) == 0u || sh.kind == CMesh) return false;
    V3 a = qrot(sh.prq[0], -v3(sh.prq[1], sh.prq[2], sh.prq[3]), pprev - v3(sh.pc[0], sh.pc[1], sh.pc[2]));
    V3 b = qrot(sh.rq[0], -v3(sh.rq[1], sh.rq[2], sh.rq[3]), pcur - v3(sh.cr[0], sh.cr[1], sh.cr[2]));
    V3 seg = b - a;
    const float band = radius + thickness + rot_margin;
    V3 nl = v3(0.0f, 1.0f, 0.0f);
    float d = 1e30f;
    switch (sh.kind) {
    case CPlane:
        d = b.y;
        break;
    case CSphere: {
        V3 e = v3(fmx(sh.he[0], 1e-8f), fmx(sh.he[1], 1e-8f), fmx(sh.he[2], 1e-8f));
        float R = 1.0f + band / fmn(e.x, fmn(e.y, e.z));
        V3 A = a / e, B = b / e;
        float lenA = len(A);
        V3 u;
        bool got = false;
        if (lenA < 1.0f) {
            u = (lenA > 1e-6f) ? A : ((len(B) > 1e-6f) ? B : v3(0.0f, 1.0f, 0.0f));
            got = true;
        } else {
            V3 D = B - A;
            float qa = dot(D, D), qb = dot(A, D), qc = dot(A, A) - R * R, t = -1.0f;
            if (qa > 1e-20f) {
                float disc = qb * qb - qa * qc;
                if (disc >= 0.0f) {
                    float t0 = (-qb - std::sqrt(disc)) / qa;
                    if (t0 >= 0.0f && t0 <= 1.0f) t = t0;
                }
            }
            if (t >= 0.0f) { u = A + t * D; got = true; }
            else if (len(B) > 1e-6f) { u = B; got = true; }
        }
        if (!got) return false;
        V3 uh = unit(u);
        V3 sp = hadamard(e, uh);
        nl = unit(uh / e);
        d = dot(nl, b - sp);
        break;
    }
    case CBox: {
        V3 h = v3(fmx(sh.he[0], 1e-8f), fmx(sh.he[1], 1e-8f), fmx(sh.he[2], 1e-8f));
        V3 H = v3(h.x + band, h.y + band, h.z + band);
        int k = 0;
        float sg = 1.0f;
        if (std::fabs(a.x) < h.x && std::fabs(a.y) < h.y && std::fabs(a.z) < h.z) {
            dominant_axis(a, h, k, sg);
        } else {
            float tE = 0.0f, tX = 1.0f, esg = 1.0f;
            int ek = -1;
            bool miss = false;
            for (int i = 0; i < 3 && !miss; ++i) {
                float di = axis_of(seg, i), ai = axis_of(a, i), Hi = axis_of(H, i);
                if (std::fabs(di) < 1e-12f) {
                    if (std::fabs(ai) > Hi) miss = true;
                    continue;
                }
                float inv = 1.0f / di;
                float t1 = (-Hi - ai) * inv, t2 = (Hi - ai) * inv;
                float tn = fmn(t1, t2), tf = fmx(t1, t2);
                if (tn > tE) { tE = tn; ek = i; esg = (di > 0.0f) ? -1.0f : 1.0f; }
                tX = fmn(tX, tf);
            }
            if (!miss && ek >= 0 && tE <= tX && tE <= 1.0f) { k = ek; sg = esg; }
            else dominant_axis(b, h, k, sg);
        }
        nl = v3(k == 0 ? sg : 0.0f, k == 1 ? sg : 0.0f, k == 2 ? sg : 0.0f);
        d = sg * axis_of(b, k) - axis_of(h, k);
        break;
    }
    case CCyl: {
        float r = fmx(sh.cr[3], 1e-8f), hh = fmx(sh.he[3], 1e-8f);
        float R = r + band, HH = hh + band;
        int feat = 0;
        float capSg = 1.0f, nx = 1.0f, nz = 0.0f;
        bool aIn = (std::sqrt(a.x * a.x + a.z * a.z) < r) && (std::fabs(a.y) < hh);
        bool resolved = false;
        if (!aIn) {
            float tE = 0.0f, tX = 1.0f, ecap = 1.0f, ex = 1.0f, ez = 0.0f;
            int ef = -1;
            bool miss = false;
            float qa = seg.x * seg.x + seg.z * seg.z;
            float qb = a.x * seg.x + a.z * seg.z;
            float qc = (a.x * a.x + a.z * a.z) - R * R;
            if (qa > 1e-20f) {
                float disc = qb * qb - qa * qc;
                if (disc < 0.0f) miss = true;
                else {
                    float sq = std::sqrt(disc);
                    float t1 = (-qb - sq) / qa, t2 = (-qb + sq) / qa;
                    if (t1 > tE) { tE = t1; ef = 0; }
                    tX = fmn(tX, t2);
                }
            } else if (qc > 0.0f) {
                miss = true;
            }
            if (!miss) {
                if (std::fabs(seg.y) < 1e-12f) {
                    if (std::fabs(a.y) > HH) miss = true;
                } else {
                    float inv = 1.0f / seg.y;
                    float t1 = (-HH - a.y) * inv, t2 = (HH - a.y) * inv;
                    float tn = fmn(t1, t2), tf = fmx(t1, t2);
                    if (tn > tE) { tE = tn; ef = 1; ecap = (seg.y > 0.0f) ? -1.0f : 1.0f; }
                    tX = fmn(tX, tf);
                }
            }
            if (!miss && ef >= 0 && tE <= tX && tE <= 1.0f) {
                if (ef == 0) {
                    float hx = a.x + tE * seg.x, hz = a.z + tE * seg.z;
                    float l = std::sqrt(hx * hx + hz * hz);
                    if (l > 1e-9f) { ex = hx / l; ez = hz / l; }
                }
                feat = ef; capSg = ecap; nx = ex; nz = ez; resolved = true;
            }
        }
        if (!resolved) {
            V3 q = aIn ? a : b;
            float lxz = std::sqrt(q.x * q.x + q.z * q.z);
            feat = ((r - lxz) <= (hh - std::fabs(q.y))) ? 0 : 1;
            capSg = (q.y >= 0.0f) ? 1.0f : -1.0f;
            if (lxz > 1e-9f) { nx = q.x / lxz; nz = q.z / lxz; } else { nx = 1.0f; nz = 0.0f; }
        }
        if (feat == 0) { nl = v3(nx, 0.0f, nz); d = dot(nl, b) - r; }
        else { nl = v3(0.0f, capSg, 0.0f); d = capSg * b.y - hh; }
        break;
    }
    default:
        return false;
    }
    if (!(d < band)) return false;
    V3 n = unit(qrot(sh.rq[0], v3(sh.rq[1], sh.rq[2], sh.rq[3]), nl));
    n_out[0] = n.x; n_out[1] = n.y; n_out[2] = n.z;
    *d_out = d;
    return true;
}

// Quat operator* and rotateVector (material_quat.hpp:27-63).
struct Q4 { float w, x, y, z; };
inline Q4 qmul(const Q4& a, const Q4& b) {
    return Q4{a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
              a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
inline V3 qapply(const Q4& q, V3 v) {
    Q4 r = qmul(qmul(q, Q4{0.0f, v.x, v.y, v.z}), Q4{q.w, -q.x, -q.y, -q.z});
    return v3(r.x, r.y, r.z);
}
// analyticWorldHalf (bvh.hpp:2431-2462).
V3 world_half(const Shape& s, const float* q) {
    V3 h = v3(0.0f, 0.0f, 0.0f);
    if (s.kind == CSphere) {
        float r = std::max(std::max(s.he[0], s.he[1]), s.he[2]);
        return v3(r, r, r);
    }
    if (s.kind == CBox) h = v3(s.he[0], s.he[1], s.he[2]);
    else if (s.kind == CCyl) h = v3(s.cr[3], s.he[3], s.cr[3]);
    else return h;
    Q4 Q{q[0], q[1], q[2], q[3]};
    V3 cx = qapply(Q, v3(1.0f, 0.0f, 0.0f)), cy = qapply(Q, v3(0.0f, 1.0f, 0.0f)), cz = qapply(Q, v3(0.0f, 0.0f, 1.0f));
    return v3(std::fabs(cx.x) * h.x + std::fabs(cy.x) * h.y + std::fabs(cz.x) * h.z,
              std::fabs(cx.y) * h.x + std::fabs(cy.y) * h.y + std::fabs(cz.y) * h.z,
              std::fabs(cx.z) * h.x + std::fabs(cy.z) * h.y + std::fabs(cz.z) * h.z);
}
inline double quat_angle(const Shape& s) {
    double dq = (double)s.rq[0] * s.prq[0] + (double)s.rq[1] * s.prq[1] + (double)s.rq[2] * s.prq[2] +
                (double)s.rq[3] * s.prq[3];
    dq = std::fabs(dq);
    if (dq > 1.0) dq = 1.0;
    return 2.0 * std::acos(dq);
}
// analyticRotBand (bvh.hpp:2465-2479).
float rot_band(const Shape& s) {
    double th = quat_angle(s);
    if (th <= 0.0) return 0.0f;
    double rmax = std::sqrt((double)s.he[0] * s.he[0] + (double)s.he[1] * s.he[1] + (double)s.he[2] * s.he[2]) +
                  (double)s.cr[3];
    return (float)(th * rmax);
}
// analyticRotMargin (bruteforce.hpp:201-240).
float rot_margin(const Shape& s, float radius, float thickness) {
    double th = quat_angle(s);
    if (!(th > 1e-9)) return 0.0f;
    double rmax = 0.0;
    switch (s.kind) {
    case CSphere: rmax = std::max({(double)s.he[0], (double)s.he[1], (double)s.he[2]}); break;
    case CBox: rmax = std::sqrt((double)s.he[0] * s.he[0] + (double)s.he[1] * s.he[1] + (double)s.he[2] * s.he[2]); break;
    case CCyl: rmax = std::sqrt((double)s.cr[3] * s.cr[3] + (double)s.he[3] * s.he[3]); break;
    case CPlane: return 0.0f;
    default: break;
    }
    return (float)(th * (rmax + (double)radius + (double)thickness));
}
// objectBroadAABB for an analytic collider (bvh.hpp:2494-2516); false = a
// half-space, which overlaps everything.
bool broad_box(const Shape& s, float inflate, Node& out) {
    V3 c = v3(s.cr[0], s.cr[1], s.cr[2]);
    if (s.kind == CPlane) { nset(out, c, c); return false; }
    V3 p = v3(s.pc[0], s.pc[1], s.pc[2]);
    V3 hc = world_half(s, s.rq), hp = world_half(s, s.prq);
    float pad = inflate + rot_band(s);
    V3 pv = v3(pad, pad, pad);
    nset(out, vmin(c - hc, p - hp) - pv, vmax(c + hc, p + hp) + pv);
    return true;
}

// ---------------------------------------------------------------- F / I
// calc_spring (physics.metal:146-153).
inline V3 spring(V3 p0, V3 v0, V3 p1, V3 v1, float rest, float ks, float kd) {
    V3 dx = p1 - p0, dv = v1 - v0;
    float len = std::sqrt(dot(dx, dx));
    if (len < 1e-7f) return v3(0.f, 0.f, 0.f);
    V3 nd = dx / len;
    return nd * (ks * (len - rest) + kd * dot(dv, nd));
}
// sanitizeIntegrateOutput (physics.metal:52-74).
inline bool sanitize(V3& pos, V3& vel, V3 fb) {
    bool touched = false;
    if (nonfinite3(pos)) { pos = nonfinite3(fb) ? v3(0.f, 0.f, 0.f) : fb; vel = v3(0.f, 0.f, 0.f); touched = true; }
    if (nonfinite3(vel)) { vel = v3(0.f, 0.f, 0.f); touched = true; }
    const float B = 1.0e4f;
    V3 bx = v3(std::fmin(std::fmax(pos.x, -B), B), std::fmin(std::fmax(pos.y, -B), B), std::fmin(std::fmax(pos.z, -B), B));
    if (bx.x != pos.x || bx.y != pos.y || bx.z != pos.z) { pos = bx; vel = v3(0.f, 0.f, 0.f); touched = true; }
    return touched;
}

// ---------------------------------------------------------------- adjacency
// MeshAdjacencyInitializer::initialize (mesh_state.hpp:236-411).
struct Adjacency {
    std::vector<u32> vaf_off, vaf;          // vertexAdjFacets CSR
    std::vector<u32> edges;                 // unique (v0 < v1), sorted
    std::vector<float> rest_edge;
    std::vector<u32> vae_off, vae;          // vertexAdjEdges CSR
    std::vector<u32> opp_off, opp;          // vertexOppVertices CSR
    std::vector<float> rest_opp;
};
struct EInfo { i32 v0, v1, f0, f1, o0, o1; };
void build_adjacency(const float* x, u32 nV, const u32* F, u32 nF, Adjacency& A) {
    A.vaf_off.assign(nV + 1, 0);
    for (u32 f = 0; f < nF; ++f) for (int k = 0; k < 3; ++k) A.vaf_off[F[3 * f + k] + 1]++;
    for (u32 v = 0; v < nV; ++v) A.vaf_off[v + 1] += A.vaf_off[v];
    A.vaf.assign(A.vaf_off[nV], 0);
    {
        std::vector<u32> o(nV, 0);
        for (u32 f = 0; f < nF; ++f) for (int k = 0; k < 3; ++k) { u32 v = F[3 * f + k]; A.vaf[A.vaf_off[v] + o[v]++] = f; }
    }
    std::vector<EInfo> tmp; tmp.reserve(3 * (size_t)nF);
    auto fill = [&](u32 a, u32 b, u32 o, u32 f) {
        if (a > b) std::swap(a, b);
        tmp.push_back(EInfo{(i32)a, (i32)b, (i32)f, -1, (i32)o, -1});
    };
    for (u32 f = 0; f < nF; ++f) {
        u32 a = F[3 * f], b = F[3 * f + 1], c = F[3 * f + 2];
        fill(a, b, c, f); fill(b, c, a, f); fill(c, a, b, f);
    }
    // std::sort in the reference is not stable; only (v0, v1) decides the
    // unique-edge order, and the o0/o1 assignment is symmetric in use.
    std::stable_sort(tmp.begin(), tmp.end(), [](const EInfo& p, const EInfo& q) {
        return p.v0 < q.v0 || (p.v0 == q.v0 && p.v1 < q.v1);
    });
    auto elen = [&](u32 a, u32 b) { V3 l = ld3(x, b) - ld3(x, a); return std::sqrt(l.x * l.x + l.y * l.y + l.z * l.z); };
    A.vae_off.assign(nV + 1, 0); A.opp_off.assign(nV + 1, 0);
    std::vector<EInfo> ei;
    A.edges.clear(); A.rest_edge.clear();
    for (size_t i = 0; i < tmp.size(); ++i) {
        if (ei.empty() || tmp[i].v0 != ei.back().v0 || tmp[i].v1 != ei.back().v1) {
            ei.push_back(tmp[i]);
            A.edges.push_back((u32)tmp[i].v0); A.edges.push_back((u32)tmp[i].v1);
            A.rest_edge.push_back(elen((u32)tmp[i].v0, (u32)tmp[i].v1));
            A.vae_off[tmp[i].v0 + 1]++; A.vae_off[tmp[i].v1 + 1]++;
        } else {
            ei.back().o1 = tmp[i].o0; ei.back().f1 = tmp[i].f0;
            A.opp_off[ei.back().o0 + 1]++; A.opp_off[ei.back().o1 + 1]++;
        }
    }
    for (u32 v = 0; v < nV; ++v) { A.opp_off[v + 1] += A.opp_off[v]; A.vae_off[v + 1] += A.vae_off[v]; }
    A.opp.assign(A.opp_off[nV], 0); A.rest_opp.assign(A.opp_off[nV], 0.f); A.vae.assign(A.vae_off[nV], 0);
    std::vector<u32> oo(nV, 0), ao(nV, 0);
    for (size_t e = 0; e < ei.size(); ++e) {
        if (ei[e].o1 != -1) {
            u32 o0 = (u32)ei[e].o0, o1 = (u32)ei[e].o1;
            u32 b0 = A.opp_off[o0] + oo[o0], b1 = A.opp_off[o1] + oo[o1];
            A.opp[b0] = o1; A.opp[b1] = o0;
            A.rest_opp[b0] = elen(o0, o1); A.rest_opp[b1] = elen(o0, o1);
            oo[o0]++; oo[o1]++;
        }
        u32 v0 = (u32)ei[e].v0, v1 = (u32)ei[e].v1;
        A.vae[A.vae_off[v0] + ao[v0]++] = (u32)e;
        A.vae[A.vae_off[v1] + ao[v1]++] = (u32)e;
    }
}

// ---------------------------------------------------------------- scene
enum Behavior : u32 { TriangularCloth = 0, FastGridCloth = 1, Elastic = 2, Rigid = 3, Float = 4, Kinematic = 7 };
enum SelfMode : u32 { SELF_OFF = 0, SELF_HASH = 1, SELF_BVH = 2 };

struct Mesh {
    u32 behavior, is_static, collidable, self_collide;
    u32 nV, nF, voff, foff;
    std::vector<u32> F;
    std::vector<float> mass, mask;
    float kstretch, kshear, kbend, thickness;
    u32 grid_n; float rest[6];
    Adjacency adj;
    // tree
    bool built = false;
    std::vector<Node> tree; std::vector<i32> parent;
    std::vector<u32> codes, idx;
    // colliderKind and the collider's pose (centre, local half extents,
    // orientation w, x, y, z)
    u32 collider = CMesh;
    float pose[10] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f};
    // GeneralMesh::applyGravity / applyWind (the per-object environment gates)
    bool gravity_on = true, wind_on = false;
    bool cloth() const { return behavior == TriangularCloth || behavior == FastGridCloth; }
};

struct SimParams {
    float subh, kair, kd, gx, gy, gz, margin, radius;
    u32 substeps, rebuild_frames, self_mode, cols_per_point;
};


struct Scene {
    SimParams P;
    std::vector<Mesh> meshes;
    std::vector<float> x, xp, v, f, ext;   // packed, 3 floats per vertex
    std::vector<u32> voff;                  // statesOffsets (vertices), size nmesh+1
    std::vector<u32> vaf_off, vaf;          // packed vertexAdjFacets (global offsets, local faces)
    u32 nV = 0;
    uint64_t frame = 0; u32 cursor = 0;
    u32 anomaly = 0, status = 0;
    u32 nbroad = 0, nnarrow = 0;
    std::vector<Row> rows;
    std::vector<Contact> contacts;
    std::vector<u32> csr_off;
    std::vector<Contact> csr;
    bool packed = false;
    // analytic colliders: compact shape table (Scene::meshAnalytic) and its
    // owners, the marker sets (PackedCollisionData::analyticPairs*)
    std::vector<u32> shape_mesh;
    std::vector<Shape> shapes;
    bool primed = false;
    std::vector<std::pair<u32, u32>> mk_fresh, mk_held, mk_pairs;
    int builder = 0;  // 0 Karras (buildTree_Tri + bottomUpBoxes), 1 Apetrei (agglomerativeBuild_Tri)
    float wind[3] = {0.f, 0.f, 0.f};  // Scene::environment.wind
};

// Scene::refreshAnalyticShapes (scene.hpp:659-745).
void refresh_shapes(Scene& S) {
    for (size_t k = 0; k < S.shape_mesh.size(); ++k) {
        const Mesh& M = S.meshes[S.shape_mesh[k]];
        const float *c = M.pose, *h = M.pose + 3, *q = M.pose + 6;
        Shape& dst = S.shapes[k];
        Shape a;
        std::memset(&a, 0, sizeof(a));
        for (int i = 0; i < 4; ++i) a.rq[i] = q[i];
        if (S.primed) {
            a.pc[0] = dst.cr[0]; a.pc[1] = dst.cr[1]; a.pc[2] = dst.cr[2];
            for (int i = 0; i < 4; ++i) a.prq[i] = dst.rq[i];
        } else {
            a.pc[0] = c[0]; a.pc[1] = c[1]; a.pc[2] = c[2];
            for (int i = 0; i < 4; ++i) a.prq[i] = q[i];
        }
        a.kind = M.collider; a.obj = S.shape_mesh[k]; a.beh = M.behavior; a.flags = M.collidable ? 1u : 0u;
        a.cr[0] = c[0]; a.cr[1] = c[1]; a.cr[2] = c[2];
        switch (M.collider) {
        case CSphere: a.cr[3] = h[0]; a.he[0] = h[0]; a.he[1] = h[1]; a.he[2] = h[2]; a.he[3] = h[1]; break;
        case CBox: a.he[0] = h[0]; a.he[1] = h[1]; a.he[2] = h[2]; break;
        case CCyl: a.cr[3] = std::max(h[0], h[2]); a.he[0] = h[0]; a.he[1] = h[1]; a.he[2] = h[2]; a.he[3] = h[1]; break;
        default: break;
        }
        dst = a;
    }
    S.primed = true;
}

enum Status : u32 { ST_NONFINITE = 1u, ST_STACK_OVF = 2u, ST_PAIR_OVF = 4u, ST_ITER_CAP = 8u };

// BVH<..,LINEAR,TRIANGLE>::build (bvh.hpp:1194-1301): box, Morton, sort,
// Karras, leaves from x, bottom-up.
void build_tree(Scene& S, Mesh& M) {
    u32 n = M.nF;
    if (n == 0) return;
    const float* x = S.x.data() + 3 * (size_t)M.voff;
    float box[6]; scene_box(x, M.nV, box);
    M.codes.resize(n); M.idx.resize(n);
    fill_mortons(x, M.F.data(), n, box, M.codes.data(), M.idx.data());
    radix_sort(M.codes.data(), M.idx.data(), n);
    M.tree.assign(2 * (size_t)n - 1, Node{});
    M.parent.assign(2 * (size_t)n - 1, -1);
    if (S.builder == 1) {
        apetrei_topology(x, M.F.data(), M.codes.data(), M.idx.data(), n, M.tree.data(), M.parent.data());
    } else {
        karras_topology(M.codes.data(), M.idx.data(), n, M.tree.data(), M.parent.data());
        leaves(x, nullptr, 0.f, 0, M.F.data(), n, M.tree.data());
        bottom_up(M.tree.data(), 2 * n - 1);
    }
    M.built = true;
}

void refit_tree(Scene& S, Mesh& M) {
    if (!M.built) return;
    const float* x = S.x.data() + 3 * (size_t)M.voff;
    const float* v = S.v.data() + 3 * (size_t)M.voff;
    leaves(x, v, S.P.subh, 1, M.F.data(), M.nF, M.tree.data());
    bottom_up(M.tree.data(), 2 * M.nF - 1);
}

inline bool root_overlap(const Mesh& a, const Mesh& b) {
    const Node& p = a.tree[0]; const Node& q = b.tree[0];
    if (p.mx[0] < q.mn[0] || p.mn[0] > q.mx[0]) return false;
    if (p.mx[1] < q.mn[1] || p.mn[1] > q.mx[1]) return false;
    if (p.mx[2] < q.mn[2] || p.mn[2] > q.mx[2]) return false;
    return true;
}

void push_row(Scene& S, u32 cap, u32 p, u32 t, u32 q, u32 tt) {
    S.nbroad++;
    if (S.rows.size() >= cap) { S.status |= ST_PAIR_OVF; return; }
    const Mesh& Q = S.meshes[q]; const Mesh& T = S.meshes[tt];
    S.rows.push_back(Row{p, t, q, tt, Q.behavior, T.behavior, 0u, 0u});
}

// BVH query of mesh q's vertices against mesh t's tree, appended in
// vertex-major DFS order.
void bvh_rows(Scene& S, u32 q, u32 t, u32 cap) {
    Mesh& Q = S.meshes[q]; Mesh& T = S.meshes[t];
    const float* xq = S.x.data() + 3 * (size_t)Q.voff;
    int nth =
#ifdef _OPENMP
        omp_get_max_threads();
#else
        1;
#endif
    std::vector<std::vector<std::pair<u32, u32>>> part(nth);
    const bool self = (q == t);
#pragma omp parallel
    {
        int tid =
#ifdef _OPENMP
            omp_get_thread_num();
#else
            0;
#endif
#pragma omp for schedule(static)
        for (long long pl = 0; pl < (long long)Q.nV; ++pl) {
            u32 p = (u32)pl;
            query_point(T.tree.data(), 2 * T.nF - 1, T.F.data(), ld3(xq, p), S.P.margin, p, self,
                        [&](u32 f) { part[tid].emplace_back(p, f); });
        }
    }
    for (auto& pt : part) for (auto& r : pt) push_row(S, cap, r.first, r.second, q, t);
}

// BroadPhase::detectCollisions (bvh.hpp:2853-2949) with the hybrid CPU-hash
// self pass in front (simulator.hpp:3678-3701) when self_mode == SELF_HASH.
void detect(Scene& S) {
    S.rows.clear(); S.nbroad = 0;
    // beginAnalyticPairs (scene.hpp:511-515)
    S.mk_held = S.mk_fresh;
    S.mk_fresh.clear();
    const float inflate = S.P.radius + S.P.margin;
    const u32 cap = S.P.cols_per_point * S.nV;
    const u32 nm = (u32)S.meshes.size();
    if (S.P.self_mode == SELF_HASH) {
        for (u32 q = 0; q < nm; ++q) {
            Mesh& Q = S.meshes[q];
            if (!Q.collidable || !Q.cloth() || !Q.self_collide || Q.nF == 0) continue;
            std::vector<std::pair<u32, u32>> r;
            self_hash_rows(S.x.data() + 3 * (size_t)Q.voff, S.xp.data() + 3 * (size_t)Q.voff, Q.nV,
                           Q.F.data(), Q.nF, S.P.margin, r);
            for (auto& e : r) push_row(S, cap, e.first, e.second, q, q);
        }
    }
    for (u32 q = 0; q < nm; ++q) {
        Mesh& Q = S.meshes[q];
        if (Q.behavior == Float || Q.behavior == Kinematic) continue;
        if (!Q.collidable) continue;
        for (u32 t = 0; t < nm; ++t) {
            Mesh& T = S.meshes[t];
            if (q == t) {
                if (Q.collider != CMesh) continue;  // no live tree
                if (S.P.self_mode != SELF_BVH || !Q.built) continue;
                bvh_rows(S, q, q, cap);
                continue;
            }
            if (!T.collidable) continue;
            if (T.collider != CMesh || Q.collider != CMesh) {
                // one marker per overlapping (cloth query, analytic target)
                // (bvh.hpp:2903-2937); the cloth's box is its tree root
                if (T.collider == CMesh || !Q.cloth() || !Q.built) continue;
                u32 slot = 0;
                while (S.shape_mesh[slot] != t) ++slot;
                Node tb;
                const Node& qb = Q.tree[0];
                bool hit = true;
                if (broad_box(S.shapes[slot], inflate, tb))
                    hit = !(tb.mx[0] < qb.mn[0] || tb.mn[0] > qb.mx[0] || tb.mx[1] < qb.mn[1] ||
                            tb.mn[1] > qb.mx[1] || tb.mx[2] < qb.mn[2] || tb.mn[2] > qb.mx[2]);
                if (hit) S.mk_fresh.push_back({q, t});
                continue;
            }
            if (!T.built || !Q.built) continue;
            if (!root_overlap(Q, T)) continue;
            bvh_rows(S, q, t, cap);
        }
    }
    // endAnalyticPairs (scene.hpp:519-531): this detect's markers, then the
    // previous detect's that are not among them
    S.mk_pairs = S.mk_fresh;
    for (auto& h : S.mk_held)
        if (std::find(S.mk_pairs.begin(), S.mk_pairs.end(), h) == S.mk_pairs.end()) S.mk_pairs.push_back(h);
}

// narrowAndSortByVertices (bruteforce.hpp:311-383): narrow every row, keep
// contacts in row order, then bucket them per global vertex.
void narrow(Scene& S) {
    const u32 cap = S.P.cols_per_point * S.nV;
    const float band = S.P.radius + S.P.margin;
    const size_t nr = S.rows.size();
    std::vector<Contact> out(nr);
    std::vector<unsigned char> hit(nr, 0);
#pragma omp parallel for schedule(dynamic, 4096)
    for (long long i = 0; i < (long long)nr; ++i) {
        const Row& r = S.rows[i];
        const Mesh& T = S.meshes[r.tobj];
        u32 f0 = T.F[3 * r.tri], f1 = T.F[3 * r.tri + 1], f2 = T.F[3 * r.tri + 2];
        if (r.qobj == r.tobj) {
            u32 g = r.point + S.voff[r.tobj];
            bool adj = false;
            for (u32 k = S.vaf_off[g]; k < S.vaf_off[g + 1]; ++k) if (S.vaf[k] == r.tri) { adj = true; break; }
            if (adj) continue;
        }
        u32 qo = S.voff[r.qobj], to = S.voff[r.tobj];
        Contact c;
        if (!narrow_one(ld3(S.x.data(), r.point + qo), ld3(S.xp.data(), r.point + qo), ld3(S.x.data(), f0 + to),
                        ld3(S.x.data(), f1 + to), ld3(S.x.data(), f2 + to), band, c.n, &c.d))
            continue;
        c.point = r.point; c.tri = r.tri; c.qobj = r.qobj; c.tobj = r.tobj;
        c.qbeh = r.qbeh; c.tbeh = r.tbeh; c.qshape = r.qshape; c.tshape = r.tshape;
        out[i] = c; hit[i] = 1;
    }
    S.contacts.clear(); S.nnarrow = 0;
    for (size_t i = 0; i < nr; ++i) {
        if (!hit[i]) continue;
        S.nnarrow++;
        if (S.contacts.size() >= cap) { S.status |= ST_PAIR_OVF; continue; }
        S.contacts.push_back(out[i]);
    }
    // narrowAnalytic (bruteforce.hpp:245-309): every vertex of the cloth of
    // each live marker against the collider's shape, appended
    for (auto& pr : S.mk_pairs) {
        u32 slot = 0;
        while (S.shape_mesh[slot] != pr.second) ++slot;
        const Shape& sh = S.shapes[slot];
        if (!(sh.flags & 1u)) continue;
        const Mesh& Q = S.meshes[pr.first];
        const float rm = rot_margin(sh, S.P.radius, S.P.margin);
        for (u32 id = 0; id < Q.nV; ++id) {
            Contact c;
            const u32 g = Q.voff + id;
            if (!analytic_one(sh, ld3(S.x.data(), g), ld3(S.xp.data(), g), S.P.radius, S.P.margin, rm, c.n, &c.d))
                continue;
            c.point = id; c.tri = 0; c.qobj = pr.first; c.tobj = pr.second;
            c.qbeh = Q.behavior; c.tbeh = sh.beh; c.qshape = CMesh; c.tshape = sh.kind;
            S.nnarrow++;
            if (S.contacts.size() >= cap) { S.status |= ST_PAIR_OVF; continue; }
            S.contacts.push_back(c);
        }
    }
    // CPU CSR (bruteforce.hpp:358-383), then canonical order per vertex.
    S.csr_off.assign(S.nV + 1, 0);
    for (auto& c : S.contacts) S.csr_off[S.voff[c.qobj] + c.point + 1]++;
    for (u32 i = 0; i < S.nV; ++i) S.csr_off[i + 1] += S.csr_off[i];
    S.csr.resize(S.contacts.size());
    std::vector<u32> o(S.nV, 0);
    for (auto& c : S.contacts) { u32 g = S.voff[c.qobj] + c.point; S.csr[S.csr_off[g] + o[g]++] = c; }
#pragma omp parallel for schedule(dynamic, 4096)
    for (long long g = 0; g < (long long)S.nV; ++g) {
        u32 b = S.csr_off[g], e = S.csr_off[g + 1];
        if (e - b > 1)
            std::stable_sort(S.csr.begin() + b, S.csr.begin() + e, [](const Contact& p, const Contact& q) {
                return p.tobj < q.tobj || (p.tobj == q.tobj && p.tri < q.tri);
            });
    }
}

// compute_cloth_grid_forces_fast (physics.metal:171-224).
V3 grid_force(const Scene& S, const Mesh& M, u32 id) {
    const float* x = S.x.data() + 3 * (size_t)M.voff;
    const float* v = S.v.data() + 3 * (size_t)M.voff;
    const float* e = S.ext.data() + 3 * (size_t)M.voff;
    u32 N = M.grid_n, row = id / N, col = id % N;
    V3 pos = ld3(x, id), vel = ld3(v, id);
    V3 force = ld3(e, id) + vel * S.P.kair;
    float kd = S.P.kd;
    auto g = [&](u32 r, u32 c, float rest, float k) {
        u32 j = r * N + c; force = force + spring(pos, vel, ld3(x, j), ld3(v, j), rest, k, kd);
    };
    const float sX = M.rest[0], sY = M.rest[1], shA = M.rest[2], shB = M.rest[3], bX = M.rest[4], bY = M.rest[5];
    if (col > 0) g(row, col - 1, sX, M.kstretch);
    if (col < N - 1) g(row, col + 1, sX, M.kstretch);
    if (row > 0) g(row - 1, col, sY, M.kstretch);
    if (row < N - 1) g(row + 1, col, sY, M.kstretch);
    if (col > 0 && row > 0) g(row - 1, col - 1, shA, M.kshear);
    if (col < N - 1 && row > 0) g(row - 1, col + 1, shB, M.kshear);
    if (col > 0 && row < N - 1) g(row + 1, col - 1, shB, M.kshear);
    if (col < N - 1 && row < N - 1) g(row + 1, col + 1, shA, M.kshear);
    if (col > 1) g(row, col - 2, bX, M.kbend);
    if (col < N - 2) g(row, col + 2, bX, M.kbend);
    if (row > 1) g(row - 2, col, bY, M.kbend);
    if (row < N - 2) g(row + 2, col, bY, M.kbend);
    return force;
}
// compute_tri_spring_forces (physics.metal:319-378): stretch over adjacent
// edges, bend over opposite vertices, no shear.
V3 tri_force(const Scene& S, const Mesh& M, u32 id) {
    const float* x = S.x.data() + 3 * (size_t)M.voff;
    const float* v = S.v.data() + 3 * (size_t)M.voff;
    const float* e = S.ext.data() + 3 * (size_t)M.voff;
    V3 pos = ld3(x, id), vel = ld3(v, id);
    V3 force = ld3(e, id) + vel * S.P.kair;
    const Adjacency& A = M.adj;
    for (u32 i = A.vae_off[id]; i < A.vae_off[id + 1]; ++i) {
        u32 eid = A.vae[i], e0 = A.edges[2 * eid], e1 = A.edges[2 * eid + 1];
        u32 o = (e0 == id) ? e1 : e0;
        force = force + spring(pos, vel, ld3(x, o), ld3(v, o), A.rest_edge[eid], M.kstretch, S.P.kd);
    }
    for (u32 i = A.opp_off[id]; i < A.opp_off[id + 1]; ++i) {
        u32 o = A.opp[i];
        force = force + spring(pos, vel, ld3(x, o), ld3(v, o), A.rest_opp[i], M.kbend, S.P.kd);
    }
    return force;
}

// integrate_cloth / integrate_cloth_grid (physics.metal:226-312, 380-466).
u32 integrate_vertex(Scene& S, const Mesh& M, u32 id, V3 force, std::vector<float>& xn, std::vector<float>& vn) {
    u32 g = M.voff + id;
    float mask = M.mask[id];
    V3 vel = ld3(S.v.data(), g), pos = ld3(S.x.data(), g);
    V3 dv = ((force * S.P.subh) / M.mass[id]) * mask;
    vel = vel + dv;
    u32 b = S.csr_off[g], e = S.csr_off[g + 1];
    for (u32 i = b; i < e; ++i) {
        bool dup = false;
        for (u32 j = b; j < i; ++j)
            if (S.csr[j].tobj == S.csr[i].tobj && S.csr[j].tri == S.csr[i].tri) { dup = true; break; }
        if (dup) continue;
        V3 n = v3(S.csr[i].n[0], S.csr[i].n[1], S.csr[i].n[2]);
        float nl2 = dot(n, n);
        if (nl2 < 1e-12f) continue;
        n = n * (1.0f / std::sqrt(nl2));
        float vnn = dot(vel, n);
        float d = S.csr[i].d, th = M.thickness;
        if (d < th) {
            if (vnn < 0.0f) vel = vel - n * vnn;
            pos = pos + n * (th - d);
        }
    }
    pos = pos + (vel * S.P.subh) * mask;
    u32 bad = sanitize(pos, vel, ld3(S.x.data(), g)) ? 1u : 0u;
    st3(xn.data(), g, pos); st3(vn.data(), g, vel);
    return bad;
}

// SymplecticSystem<METAL>::update (symplectic_system.hpp:341-409): forces for
// every cloth mesh from the old state, then integrate.
void system_update(Scene& S) {
    std::vector<float> xn = S.x, vn = S.v;
    u32 bad = 0;
    for (auto& M : S.meshes) {
        if (!M.cloth()) continue;
#pragma omp parallel for schedule(static) reduction(| : bad)
        for (long long il = 0; il < (long long)M.nV; ++il) {
            u32 id = (u32)il;
            V3 f = (M.behavior == FastGridCloth) ? grid_force(S, M, id) : tri_force(S, M, id);
            st3(S.f.data(), M.voff + id, f);
            bad |= integrate_vertex(S, M, id, f, xn, vn);
        }
    }
    S.x.swap(xn); S.v.swap(vn);
    if (bad) { S.anomaly = 1; S.status |= ST_NONFINITE; }
}

// applyEnvironmentForces (simulator.hpp:3123-3166): zero for Float, Rigid and
// Kinematic meshes; otherwise g * m when the mesh's gravity gate is on (else
// zero), plus the wind vector (a force per particle, no mass) when its wind
// gate is on and it is cloth.
void env_forces(Scene& S) {
    for (auto& M : S.meshes) {
        const bool moved = !(M.behavior == Float || M.behavior == Rigid || M.behavior == Kinematic);
        const bool wind = M.wind_on && M.cloth();
        for (u32 i = 0; i < M.nV; ++i) {
            u32 g = M.voff + i;
            V3 e = v3(0.f, 0.f, 0.f);
            if (moved) {
                if (M.gravity_on) e = v3(S.P.gx * M.mass[i], S.P.gy * M.mass[i], S.P.gz * M.mass[i]);
                if (wind) e = v3(e.x + S.wind[0], e.y + S.wind[1], e.z + S.wind[2]);
            }
            st3(S.ext.data(), g, e);
        }
    }
}

// One substep of Simulator::update (simulator.hpp:3512-3815), frame preamble
// (periodic rebuild, environment forces) at cursor 0.
void substep(Scene& S) {
    if (S.cursor == 0) {
        refresh_shapes(S);
        if (S.P.rebuild_frames && S.frame % S.P.rebuild_frames == 0)
            for (auto& M : S.meshes) {
                if (M.built && M.behavior == Float) continue;
                build_tree(S, M);
            }
        env_forces(S);
    }
    for (auto& M : S.meshes) if (!M.is_static) refit_tree(S, M);
    detect(S);
    narrow(S);
    for (auto& M : S.meshes) {
        if (M.behavior == Float || M.behavior == Kinematic) continue;
        std::memcpy(S.xp.data() + 3 * (size_t)M.voff, S.x.data() + 3 * (size_t)M.voff, 12 * (size_t)M.nV);
    }
    system_update(S);
    if (++S.cursor >= S.P.substeps) { S.cursor = 0; S.frame++; }
}

} // namespace

// =====================================================================
// C ABI for ctypes (tests / bench baseline only).
extern "C" {

void yso_set_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n > 0 ? n : 1);
#else
    (void)n;
#endif
}
int yso_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void yso_scene_box(const float* x, u32 nV, float* out6) { scene_box(x, nV, out6); }
void yso_fill_mortons(const float* x, const u32* F, u32 nM, const float* box6, u32* codes, u32* idx) {
    fill_mortons(x, F, nM, box6, codes, idx);
}
void yso_radix_sort(u32* codes, u32* idx, u32 n) { radix_sort(codes, idx, n); }
void yso_karras(const u32* codes, const u32* idx, u32 n, void* tree, int32_t* parent) {
    karras_topology(codes, idx, n, (Node*)tree, parent);
}
void yso_leaves(const float* x, const float* v, float dt, int swept, const u32* F, u32 n, void* tree) {
    leaves(x, v, dt, swept, F, n, (Node*)tree);
}
void yso_bottom_up(void* tree, u32 nNodes) { bottom_up((Node*)tree, nNodes); }

// Full build of one mesh's tree; tree has 2n-1 nodes.
void yso_build_tree(const float* x, u32 nV, const u32* F, u32 nF, void* tree, int32_t* parent, u32* codes, u32* idx) {
    if (nF == 0) return;
    float box[6]; scene_box(x, nV, box);
    fill_mortons(x, F, nF, box, codes, idx);
    radix_sort(codes, idx, nF);
    karras_topology(codes, idx, nF, (Node*)tree, parent);
    leaves(x, nullptr, 0.f, 0, F, nF, (Node*)tree);
    bottom_up((Node*)tree, 2 * nF - 1);
}

// The same with the Apetrei build; returns the slot the root was built in.
int yso_build_tree_apetrei(const float* x, u32 nV, const u32* F, u32 nF, void* tree, int32_t* parent, u32* codes,
                           u32* idx) {
    if (nF == 0) return -1;
    float box[6]; scene_box(x, nV, box);
    fill_mortons(x, F, nF, box, codes, idx);
    radix_sort(codes, idx, nF);
    return apetrei_topology(x, F, codes, idx, nF, (Node*)tree, parent);
}
// Tree builder of a scene's meshes: 0 Karras, 1 Apetrei.
void yso_scene_set_builder(void* h, int builder) { ((Scene*)h)->builder = builder; }

// Point query: writes (point, tri) pairs in vertex-major DFS order; returns the
// number of candidates (pairs beyond cap are counted, not written).
uint64_t yso_query_points(const void* tree, u32 nNodes, const u32* F, const float* qx, u32 nQ, float margin, int self,
                          u32* out_pairs, uint64_t cap) {
    uint64_t cnt = 0;
    for (u32 p = 0; p < nQ; ++p)
        query_point((const Node*)tree, nNodes, F, ld3(qx, p), margin, p, self != 0, [&](u32 f) {
            if (cnt < cap) { out_pairs[2 * cnt] = p; out_pairs[2 * cnt + 1] = f; }
            cnt++;
        });
    return cnt;
}
uint64_t yso_self_hash(const float* x, const float* xp, u32 nV, const u32* F, u32 nF, float m, u32* out_pairs, uint64_t cap) {
    std::vector<std::pair<u32, u32>> r;
    self_hash_rows(x, xp, nV, F, nF, m, r);
    for (uint64_t i = 0; i < r.size() && i < cap; ++i) { out_pairs[2 * i] = r[i].first; out_pairs[2 * i + 1] = r[i].second; }
    return r.size();
}
// Brute-force enumerations used to pin the tree / grid restatements.
uint64_t yso_brute_q1(const float* tx, const u32* F, u32 nF, const float* qx, u32 nQ, float m, int self, u32* out, uint64_t cap) {
    uint64_t cnt = 0;
    for (u32 p = 0; p < nQ; ++p) {
        V3 q = ld3(qx, p); V3 qmn = q - v3(m, m, m), qmx = q + v3(m, m, m);
        for (u32 f = 0; f < nF; ++f) {
            Node L; V3 a = ld3(tx, F[3 * f]), b = ld3(tx, F[3 * f + 1]), c = ld3(tx, F[3 * f + 2]);
            nset(L, vmin(vmin(a, b), c), vmax(vmax(a, b), c));
            if (!overlap(qmn, qmx, L)) continue;
            if (self && (F[3 * f] == p || F[3 * f + 1] == p || F[3 * f + 2] == p)) continue;
            if (cnt < cap) { out[2 * cnt] = p; out[2 * cnt + 1] = f; }
            cnt++;
        }
    }
    return cnt;
}
uint64_t yso_brute_h1(const float* x, const float* xp, u32 nV, const u32* F, u32 nF, float m, u32* out, uint64_t cap) {
    std::vector<FaceRec> faces; face_boxes(x, F, nF, m, faces);
    uint64_t cnt = 0;
    for (u32 v = 0; v < nV; ++v) {
        float vlo[3], vhi[3], pc3[3], pp3[3]; bool ok = true;
        for (int a = 0; a < 3; ++a) {
            float pc = x[3 * v + a], pp = xp[3 * v + a];
            if (!std::isfinite(pc)) { ok = false; break; }
            if (!std::isfinite(pp) || std::abs(pp - pc) > 1.f) pp = pc;
            pc3[a] = pc; pp3[a] = pp; vlo[a] = std::min(pc, pp); vhi[a] = std::max(pc, pp);
        }
        if (!ok) continue;
        for (auto& fr : faces) {
            if (vhi[0] < fr.bmin[0] || vlo[0] > fr.bmax[0] || vhi[1] < fr.bmin[1] || vlo[1] > fr.bmax[1] ||
                vhi[2] < fr.bmin[2] || vlo[2] > fr.bmax[2]) continue;
            u32 f = fr.face;
            if (F[3 * f] == v || F[3 * f + 1] == v || F[3 * f + 2] == v) continue;
            float A[3], B[3], C[3];
            for (int a = 0; a < 3; ++a) { A[a] = x[3 * F[3 * f] + a]; B[a] = x[3 * F[3 * f + 1] + a]; C[a] = x[3 * F[3 * f + 2] + a]; }
            if (point_tri_sq(pc3, A, B, C) > m * m && point_tri_sq(pp3, A, B, C) > m * m) continue;
            if (cnt < cap) { out[2 * cnt] = v; out[2 * cnt + 1] = f; }
            cnt++;
        }
    }
    return cnt;
}
float yso_point_tri_sq(const float* p, const float* a, const float* b, const float* c) { return point_tri_sq(p, a, b, c); }
// H2 rows (Row, 32 B each); returns the row count, stats6 = entries, cells,
// candidate pairs, grid resolution.
uint64_t yso_sh_face_face(const float* x, const u32* stateOff, const u32* F, const u32* facetOff, const u32* beh,
                          const u32* shape, u32 nM, float margin, int self, void* out, uint64_t cap, u32* stats6) {
    std::vector<Row> rows;
    sh_face_face(x, stateOff, F, facetOff, beh, shape, nM, margin, self != 0, rows, stats6);
    std::memcpy(out, rows.data(), sizeof(Row) * std::min<uint64_t>(cap, rows.size()));
    return rows.size();
}
// One narrow-phase evaluation (returns 1 on contact).
int yso_narrow_one(const float* qcur, const float* qprev, const float* t0, const float* t1, const float* t2, float band,
                   float* n_out, float* d_out) {
    return narrow_one(ld3(qcur, 0), ld3(qprev, 0), ld3(t0, 0), ld3(t1, 0), ld3(t2, 0), band, n_out, d_out) ? 1 : 0;
}

// Adjacency handle.
void* yso_adj_new(const float* x, u32 nV, const u32* F, u32 nF) {
    Adjacency* A = new Adjacency(); build_adjacency(x, nV, F, nF, *A); return A;
}
uint64_t yso_adj_size(void* h, int which) {
    Adjacency* A = (Adjacency*)h;
    switch (which) {
        case 0: return A->vaf_off.size(); case 1: return A->vaf.size(); case 2: return A->edges.size();
        case 3: return A->rest_edge.size(); case 4: return A->vae_off.size(); case 5: return A->vae.size();
        case 6: return A->opp_off.size(); case 7: return A->opp.size(); case 8: return A->rest_opp.size();
    }
    return 0;
}
void yso_adj_get(void* h, int which, void* out) {
    Adjacency* A = (Adjacency*)h;
    const void* src = nullptr; size_t n = yso_adj_size(h, which);
    switch (which) {
        case 0: src = A->vaf_off.data(); break; case 1: src = A->vaf.data(); break; case 2: src = A->edges.data(); break;
        case 3: src = A->rest_edge.data(); break; case 4: src = A->vae_off.data(); break; case 5: src = A->vae.data(); break;
        case 6: src = A->opp_off.data(); break; case 7: src = A->opp.data(); break; case 8: src = A->rest_opp.data(); break;
    }
    if (src && n) std::memcpy(out, src, 4 * n);
}
void yso_adj_free(void* h) { delete (Adjacency*)h; }

// ---- scene
// fp: subh, kair, kd, gx, gy, gz, margin, radius ; ip: substeps, rebuild_frames, self_mode, cols_per_point
void* yso_scene_new(const float* fp, const u32* ip) {
    Scene* S = new Scene();
    S->P = SimParams{fp[0], fp[1], fp[2], fp[3], fp[4], fp[5], fp[6], fp[7], ip[0], ip[1], ip[2], ip[3]};
    return S;
}
void yso_scene_free(void* h) { delete (Scene*)h; }
// flags: bit0 static, bit1 collidable, bit2 self_collide.  kp: stretch, shear,
// bend, thickness.  rest6: FastGridCloth directional rest lengths.
int yso_scene_add_mesh(void* h, u32 behavior, u32 flags, u32 nV, const float* x, const float* v, const float* mass,
                       const float* mask, u32 nF, const u32* F, const float* kp, u32 grid_n, const float* rest6) {
    Scene* S = (Scene*)h;
    Mesh M;
    M.behavior = behavior; M.is_static = flags & 1u; M.collidable = (flags >> 1) & 1u; M.self_collide = (flags >> 2) & 1u;
    M.nV = nV; M.nF = nF; M.voff = S->nV; M.foff = 0;
    M.F.assign(F, F + 3 * (size_t)nF);
    M.mass.assign(mass, mass + nV); M.mask.assign(mask, mask + nV);
    M.kstretch = kp[0]; M.kshear = kp[1]; M.kbend = kp[2]; M.thickness = kp[3];
    M.grid_n = grid_n; for (int i = 0; i < 6; ++i) M.rest[i] = rest6 ? rest6[i] : 0.f;
    build_adjacency(x, nV, F, nF, M.adj);
    S->x.insert(S->x.end(), x, x + 3 * (size_t)nV);
    S->v.insert(S->v.end(), v, v + 3 * (size_t)nV);
    S->nV += nV;
    S->meshes.push_back(std::move(M));
    return (int)S->meshes.size() - 1;
}
void yso_scene_pack(void* h) {
    Scene* S = (Scene*)h;
    S->xp = S->x;
    S->f.assign(S->x.size(), 0.f); S->ext.assign(S->x.size(), 0.f);
    S->voff.clear();
    S->vaf_off.assign(S->nV + 1, 0); S->vaf.clear();
    for (auto& M : S->meshes) {
        S->voff.push_back(M.voff);
        for (u32 i = 0; i < M.nV; ++i) S->vaf_off[M.voff + i + 1] = M.adj.vaf_off[i + 1] - M.adj.vaf_off[i];
        S->vaf.insert(S->vaf.end(), M.adj.vaf.begin(), M.adj.vaf.end());
    }
    S->voff.push_back(S->nV);
    for (u32 i = 0; i < S->nV; ++i) S->vaf_off[i + 1] += S->vaf_off[i];
    // Scene::packAnalyticShapes (scene.hpp:762-781): seeded, not primed
    S->shape_mesh.clear();
    for (u32 m = 0; m < S->meshes.size(); ++m)
        if (S->meshes[m].collider != CMesh) S->shape_mesh.push_back(m);
    S->shapes.assign(S->shape_mesh.size(), Shape{});
    S->primed = false;
    refresh_shapes(*S);
    S->primed = false;
    S->mk_fresh.clear(); S->mk_held.clear(); S->mk_pairs.clear();
    S->packed = true;
}
// Analytic collider of a mesh: kind (0 = triangles), centre, half extents,
// orientation (w, x, y, z); the kind is fixed once packed.  Returns 0 on success.
int yso_scene_set_collider(void* h, int mesh, u32 kind, const float* c, const float* hx, const float* q) {
    Scene* S = (Scene*)h;
    if (mesh < 0 || (size_t)mesh >= S->meshes.size() || kind > CPlane) return -1;
    Mesh& M = S->meshes[mesh];
    if (S->packed && kind != M.collider) return -1;
    M.collider = kind;
    for (int i = 0; i < 3; ++i) { M.pose[i] = c[i]; M.pose[3 + i] = hx ? hx[i] : 0.f; }
    for (int i = 0; i < 4; ++i) M.pose[6 + i] = q[i];
    return 0;
}
// Environment of the scene (wind) and the gravity / wind gates of a mesh;
// they act from the next frame start.  Returns 0 on success.
void yso_scene_set_wind(void* h, const float* wind) {
    Scene* S = (Scene*)h;
    for (int k = 0; k < 3; ++k) S->wind[k] = wind[k];
}
int yso_scene_set_mesh_env(void* h, int mesh, int gravity_on, int wind_on) {
    Scene* S = (Scene*)h;
    if (mesh < 0 || (size_t)mesh >= S->meshes.size()) return -1;
    S->meshes[mesh].gravity_on = gravity_on != 0;
    S->meshes[mesh].wind_on = wind_on != 0;
    return 0;
}
uint64_t yso_scene_shapes(void* h, void* out) {
    Scene* S = (Scene*)h;
    if (out) std::memcpy(out, S->shapes.data(), sizeof(Shape) * S->shapes.size());
    return S->shapes.size();
}
// One analytic narrow evaluation (returns 1 on contact).
int yso_analytic_one(const void* shape, const float* pcur, const float* pprev, float radius, float thickness,
                     float rot, float* n_out, float* d_out) {
    return analytic_one(*(const Shape*)shape, ld3(pcur, 0), ld3(pprev, 0), radius, thickness, rot, n_out, d_out) ? 1
                                                                                                                   : 0;
}
float yso_rot_margin(const void* shape, float radius, float thickness) {
    return rot_margin(*(const Shape*)shape, radius, thickness);
}
// Broad box (6 floats lo, hi); returns 1 when finite.
int yso_broad_box(const void* shape, float inflate, float* out6) {
    Node n;
    int f = broad_box(*(const Shape*)shape, inflate, n) ? 1 : 0;
    for (int i = 0; i < 3; ++i) { out6[i] = n.mn[i]; out6[3 + i] = n.mx[i]; }
    return f;
}
// narrowAnalytic over explicit pairs (2 u32 each: cloth mesh, collider mesh),
// contacts (48 B) in pair-then-vertex order; returns the contact count
// (contacts beyond cap are counted, not written).
uint64_t yso_narrow_analytic(const float* x, const float* xp, const u32* state_off, const u32* beh, u32 nmesh,
                             const void* shapes, u32 nshapes, const u32* pairs, u32 npairs, float radius,
                             float thickness, void* out, uint64_t cap) {
    const Shape* sh = (const Shape*)shapes;
    Contact* o = (Contact*)out;
    uint64_t n = 0;
    for (u32 p = 0; p < npairs; ++p) {
        u32 cloth = pairs[2 * p], obj = pairs[2 * p + 1];
        if (cloth >= nmesh) continue;
        int slot = -1;
        for (u32 k = 0; k < nshapes; ++k) if (sh[k].obj == obj) { slot = (int)k; break; }
        if (slot < 0 || !(sh[slot].flags & 1u)) continue;
        const float rm = rot_margin(sh[slot], radius, thickness);
        for (u32 id = 0; id < state_off[cloth + 1] - state_off[cloth]; ++id) {
            const u32 g = state_off[cloth] + id;
            Contact c;
            if (!analytic_one(sh[slot], ld3(x, g), ld3(xp, g), radius, thickness, rm, c.n, &c.d)) continue;
            c.point = id; c.tri = 0; c.qobj = cloth; c.tobj = obj;
            c.qbeh = beh[cloth]; c.tbeh = sh[slot].beh; c.qshape = CMesh; c.tshape = sh[slot].kind;
            if (n < cap) o[n] = c;
            ++n;
        }
    }
    return n;
}
void yso_scene_step(void* h, u32 nsub) {
    Scene* S = (Scene*)h;
    for (u32 i = 0; i < nsub; ++i) substep(*S);
}
// Individual stages of one substep, for stage-by-stage parity tests.
void yso_scene_stage(void* h, int which) {
    Scene& S = *(Scene*)h;
    switch (which) {
        case 0:  // frame preamble
            if (S.cursor == 0) {
                refresh_shapes(S);
                if (S.P.rebuild_frames && S.frame % S.P.rebuild_frames == 0)
                    for (auto& M : S.meshes) { if (M.built && M.behavior == Float) continue; build_tree(S, M); }
                env_forces(S);
            }
            break;
        case 1: for (auto& M : S.meshes) if (!M.is_static) refit_tree(S, M); break;
        case 2: detect(S); break;
        case 3: narrow(S); break;
        case 4:
            for (auto& M : S.meshes) {
                if (M.behavior == Float || M.behavior == Kinematic) continue;
                std::memcpy(S.xp.data() + 3 * (size_t)M.voff, S.x.data() + 3 * (size_t)M.voff, 12 * (size_t)M.nV);
            }
            break;
        case 5: system_update(S); if (++S.cursor >= S.P.substeps) { S.cursor = 0; S.frame++; } break;
    }
}
// which: 0 x, 1 v, 2 xPrev, 3 f, 4 ext
void yso_scene_get(void* h, int which, float* out) {
    Scene* S = (Scene*)h;
    const std::vector<float>* src = which == 0 ? &S->x : which == 1 ? &S->v : which == 2 ? &S->xp : which == 3 ? &S->f : &S->ext;
    std::memcpy(out, src->data(), 4 * src->size());
}
void yso_scene_set(void* h, int which, const float* in) {
    Scene* S = (Scene*)h;
    std::vector<float>* dst = which == 0 ? &S->x : which == 1 ? &S->v : &S->xp;
    std::memcpy(dst->data(), in, 4 * dst->size());
}
// out: frame, cursor, nbroad, nnarrow (stored contacts), anomaly, status, ncontacts_total
void yso_scene_stats(void* h, uint64_t* out) {
    Scene* S = (Scene*)h;
    out[0] = S->frame; out[1] = S->cursor; out[2] = S->nbroad; out[3] = S->contacts.size();
    out[4] = S->anomaly; out[5] = S->status; out[6] = S->nnarrow;
}
uint64_t yso_scene_nrows(void* h) { return ((Scene*)h)->rows.size(); }
void yso_scene_rows(void* h, void* out) { Scene* S = (Scene*)h; std::memcpy(out, S->rows.data(), 32 * S->rows.size()); }
uint64_t yso_scene_ncontacts(void* h) { return ((Scene*)h)->csr.size(); }
void yso_scene_contacts(void* h, u32* off_out, void* out) {
    Scene* S = (Scene*)h;
    std::memcpy(off_out, S->csr_off.data(), 4 * S->csr_off.size());
    std::memcpy(out, S->csr.data(), 48 * S->csr.size());
}
uint64_t yso_scene_tree_nodes(void* h, int mesh) { Scene* S = (Scene*)h; return S->meshes[mesh].tree.size(); }
void yso_scene_tree(void* h, int mesh, void* nodes, int32_t* parent, u32* codes, u32* idx) {
    Scene* S = (Scene*)h; Mesh& M = S->meshes[mesh];
    if (nodes) std::memcpy(nodes, M.tree.data(), 32 * M.tree.size());
    if (parent) std::memcpy(parent, M.parent.data(), 4 * M.parent.size());
    if (codes) std::memcpy(codes, M.codes.data(), 4 * M.codes.size());
    if (idx) std::memcpy(idx, M.idx.data(), 4 * M.idx.size());
}

}  // extern "C"
