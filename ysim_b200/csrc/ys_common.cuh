// ys_common.cuh -- shared device types and arithmetic for the ysim B200 path.
//
// All translation units are compiled with -fmad=false and IEEE division /
// square root, so each float expression below rounds once per operation in
// source order, the same arithmetic as the reference's CPU build
// (-ffp-contract=off).  That is what makes Morton codes, AABBs and candidate
// sets bit-exact and keeps positions bit-identical to the CPU restatement.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ys {

typedef uint32_t u32;
typedef int32_t i32;
typedef uint64_t u64;

// Device-side status word bits (latched with atomicOr, read at host sync points).
enum : u32 {
    ST_NONFINITE = 1u,    // integrate sanitised a non-finite / out-of-box vertex
    ST_STACK_OVF = 2u,    // traversal stack full
    ST_PAIR_OVF = 4u,     // broad rows or narrow contacts beyond capacity
    ST_ITER_CAP = 8u,     // a bounded loop hit its iteration cap
    ST_CONTACT_OVF = 16u, // more contacts on one vertex than the per-vertex buffer
};

// BVHNode (bvh.hpp:148-177): {min.xyz, childA, max.xyz, childB}, 32 B.
// Leaf: childA = -1, childB = primitive.  Stored as two float4 so a node is
// one aligned 32-byte sector.
struct __align__(16) Node {
    float mnx, mny, mnz; i32 a;
    float mxx, mxy, mxz; i32 b;
};
static_assert(sizeof(Node) == 32, "Node must be 32 bytes");

// 4-wide node of the scene trees in the cube layout: the boxes of up to four
// children side by side (one 128-byte line holds everything a descent step
// tests), the child words, the child count and the link to the parent's slot.
// child >= 0: a wide node; child < 0: a leaf, ~child = face; W4_EMPTY: unused
// slot (its box is inverted so it never overlaps).
struct __align__(128) Wide4 {
    float lox[4], loy[4], loz[4];
    float hix[4], hiy[4], hiz[4];
    i32 child[4];
    u32 nchild;
    i32 parent;  // wide parent, -1 at the root
    u32 slot;    // this node's slot in the parent
    u32 pad;
};
static_assert(sizeof(Wide4) == 128, "Wide4 must be 128 bytes");
static constexpr i32 W4_EMPTY = 0x7FFFFFFF;

// BroadCollision (collision_pod.hpp:256-261), 32 B.
struct Row { u32 point, tri, qobj, tobj, qbeh, tbeh, qshape, tshape; };
static_assert(sizeof(Row) == 32, "Row must be 32 bytes");

// NarrowCollision (collision_pod.hpp:274-280), 48 B.
struct __align__(16) Contact {
    u32 point, tri, qobj, tobj;
    float nx, ny, nz, d;
    u32 qbeh, tbeh, qshape, tshape;
};
static_assert(sizeof(Contact) == 48, "Contact must be 48 bytes");

// Compact per-vertex contact used inside the fused kernel and the CSR.
struct VContact { u32 tobj, tri; float nx, ny, nz, d; };

struct f3 { float x, y, z; };
__host__ __device__ __forceinline__ f3 mk(float a, float b, float c) { f3 r; r.x = a; r.y = b; r.z = c; return r; }
__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ f3 operator-(f3 a) { return mk(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ f3 operator/(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
__host__ __device__ __forceinline__ f3 operator/(f3 a, f3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
// ((a.x*b.x + a.y*b.y) + a.z*b.z)
__host__ __device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// tinym::min / max (tinym.hpp:424-447).
__host__ __device__ __forceinline__ float tmin(float a, float b) { return a > b ? b : a; }
__host__ __device__ __forceinline__ float tmax(float a, float b) { return a < b ? b : a; }
__host__ __device__ __forceinline__ f3 vmin(f3 a, f3 b) { return mk(tmin(a.x, b.x), tmin(a.y, b.y), tmin(a.z, b.z)); }
__host__ __device__ __forceinline__ f3 vmax(f3 a, f3 b) { return mk(tmax(a.x, b.x), tmax(a.y, b.y), tmax(a.z, b.z)); }

__device__ __forceinline__ f3 ld(const float4* p, u32 i) { float4 q = p[i]; return mk(q.x, q.y, q.z); }
__device__ __forceinline__ f3 ldp(const float* p, u32 i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

__device__ __forceinline__ bool nonfinite3(f3 p) {
    return ((__float_as_uint(p.x) & 0x7F800000u) == 0x7F800000u) ||
           ((__float_as_uint(p.y) & 0x7F800000u) == 0x7F800000u) ||
           ((__float_as_uint(p.z) & 0x7F800000u) == 0x7F800000u);
}

__device__ __forceinline__ int clz32(u32 v) { return __clz(v); }  // __clz(0) == 32

// Packed-xyz (reference VectorBase layout, 3 floats per vertex) and padded
// float4 accessors, so stage kernels take either layout.
struct Pos3 {
    const float* p;
    __device__ __forceinline__ f3 operator[](u32 i) const { return ldp(p, i); }
};
struct Pos4 {
    const float4* p;
    __device__ __forceinline__ f3 operator[](u32 i) const { return ld(p, i); }
};

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace ys
