// metal_shim.h -- just enough of the Metal Shading Language surface, in plain
// C++17, to compile the reference's compute kernels (src/metal/bvh.metal,
// bruteforce.metal, physics.metal) for the host.  TEST INFRASTRUCTURE ONLY:
// it exists so the CPU oracle can be checked against the reference's own
// kernel code (oracle/_ref), never shipped with the product.
//
// Mapping:
//   * address-space qualifiers (device, constant, thread, threadgroup) and
//     the `kernel` qualifier vanish; [[buffer(n)]]-style attributes are
//     ignored by the compiler (-Wno-attributes);
//   * vector types are plain structs; floatN is 4*N bytes here (packed), the
//     reference only places packed_* types and float4 in buffers, which keep
//     their Metal sizes;
//   * min/max/clamp on floats follow fmin/fmax; rsqrt(x) is 1/sqrt(x) (IEEE),
//     the same documented replacement the oracle and the CUDA path use;
//   * atomics are std::atomic with the requested order; fences map to
//     std::atomic_thread_fence, threadgroup barriers to no-ops (only kernels
//     without threadgroup cooperation are ever executed by the harness);
//   * swizzles .xyz / .xz become calls via macros.
#pragma once
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>

#define kernel
#define device
#define constant const
#define thread
#define threadgroup
#define xyz xyz_sw()
#define xz xz_sw()
#define yzw yzw_sw()

namespace metal {

typedef unsigned int uint;
typedef unsigned short ushort;
typedef unsigned char uchar;

template <class T> struct V2;
template <class T> struct V3;
template <class T> struct V4;

template <class T>
struct V2 {
    T x, y;
    V2() = default;
    constexpr V2(T a, T b) : x(a), y(b) {}
    explicit constexpr V2(T s) : x(s), y(s) {}
    template <class U> explicit constexpr V2(const V2<U>& o) : x((T)o.x), y((T)o.y) {}
    T& operator[](int i) { return (&x)[i]; }
    const T& operator[](int i) const { return (&x)[i]; }
};

template <class T>
struct V3 {
    T x, y, z;
    V3() = default;
    constexpr V3(T a, T b, T c) : x(a), y(b), z(c) {}
    explicit constexpr V3(T s) : x(s), y(s), z(s) {}
    template <class U> explicit constexpr V3(const V3<U>& o) : x((T)o.x), y((T)o.y), z((T)o.z) {}
    T& operator[](int i) { return (&x)[i]; }
    const T& operator[](int i) const { return (&x)[i]; }
    V2<T> xz_sw() const { return V2<T>(x, z); }
};

template <class T>
struct V4 {
    T x, y, z, w;
    V4() = default;
    constexpr V4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    constexpr V4(V3<T> v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
    explicit constexpr V4(T s) : x(s), y(s), z(s), w(s) {}
    T& operator[](int i) { return (&x)[i]; }
    const T& operator[](int i) const { return (&x)[i]; }
    V3<T> xyz_sw() const { return V3<T>(x, y, z); }
    V3<T> yzw_sw() const { return V3<T>(y, z, w); }
    V2<T> xz_sw() const { return V2<T>(x, z); }
};

typedef V2<float> float2;
typedef V3<float> float3;
typedef V4<float> float4;
typedef V2<uint> uint2;
typedef V3<uint> uint3;
typedef V4<uint> uint4;
typedef V2<int> int2;
typedef V3<int> int3;
typedef V4<int> int4;
typedef V3<bool> bool3;
typedef float3 packed_float3;
typedef uint3 packed_uint3;
typedef uint2 packed_uint2;
typedef float2 packed_float2;
typedef int3 packed_int3;

// ---- element-wise operators
#define YS_V2(OP) template <class T> V2<T> operator OP(V2<T> a, V2<T> b) { return V2<T>(a.x OP b.x, a.y OP b.y); } \
    template <class T> V2<T> operator OP(V2<T> a, T s) { return V2<T>(a.x OP s, a.y OP s); } \
    template <class T> V2<T> operator OP(T s, V2<T> a) { return V2<T>(s OP a.x, s OP a.y); }
#define YS_V3(OP) template <class T> V3<T> operator OP(V3<T> a, V3<T> b) { return V3<T>(a.x OP b.x, a.y OP b.y, a.z OP b.z); } \
    template <class T> V3<T> operator OP(V3<T> a, T s) { return V3<T>(a.x OP s, a.y OP s, a.z OP s); } \
    template <class T> V3<T> operator OP(T s, V3<T> a) { return V3<T>(s OP a.x, s OP a.y, s OP a.z); }
#define YS_V4(OP) template <class T> V4<T> operator OP(V4<T> a, V4<T> b) { return V4<T>(a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w); } \
    template <class T> V4<T> operator OP(V4<T> a, T s) { return V4<T>(a.x OP s, a.y OP s, a.z OP s, a.w OP s); } \
    template <class T> V4<T> operator OP(T s, V4<T> a) { return V4<T>(s OP a.x, s OP a.y, s OP a.z, s OP a.w); }
YS_V2(+) YS_V2(-) YS_V2(*) YS_V2(/) YS_V2(^) YS_V2(&) YS_V2(|)
YS_V3(+) YS_V3(-) YS_V3(*) YS_V3(/) YS_V3(^) YS_V3(&) YS_V3(|)
YS_V4(+) YS_V4(-) YS_V4(*) YS_V4(/) YS_V4(^) YS_V4(&) YS_V4(|)
#undef YS_V2
#undef YS_V3
#undef YS_V4
template <class T> V2<T> operator-(V2<T> a) { return V2<T>(-a.x, -a.y); }
template <class T> V3<T> operator-(V3<T> a) { return V3<T>(-a.x, -a.y, -a.z); }
template <class T> V4<T> operator-(V4<T> a) { return V4<T>(-a.x, -a.y, -a.z, -a.w); }
template <class T, class R> V2<T>& operator+=(V2<T>& a, R b) { a = a + b; return a; }
template <class T, class R> V3<T>& operator+=(V3<T>& a, R b) { a = a + b; return a; }
template <class T, class R> V4<T>& operator+=(V4<T>& a, R b) { a = a + b; return a; }
template <class T, class R> V2<T>& operator-=(V2<T>& a, R b) { a = a - b; return a; }
template <class T, class R> V3<T>& operator-=(V3<T>& a, R b) { a = a - b; return a; }
template <class T, class R> V4<T>& operator-=(V4<T>& a, R b) { a = a - b; return a; }
template <class T, class R> V2<T>& operator*=(V2<T>& a, R b) { a = a * b; return a; }
template <class T, class R> V3<T>& operator*=(V3<T>& a, R b) { a = a * b; return a; }
template <class T, class R> V4<T>& operator*=(V4<T>& a, R b) { a = a * b; return a; }
template <class T, class R> V3<T>& operator/=(V3<T>& a, R b) { a = a / b; return a; }
template <class T> V3<bool> operator!=(V3<T> a, V3<T> b) { return V3<bool>(a.x != b.x, a.y != b.y, a.z != b.z); }
template <class T> V3<bool> operator==(V3<T> a, V3<T> b) { return V3<bool>(a.x == b.x, a.y == b.y, a.z == b.z); }
template <class T> V3<bool> operator<(V3<T> a, V3<T> b) { return V3<bool>(a.x < b.x, a.y < b.y, a.z < b.z); }
template <class T> V3<bool> operator>(V3<T> a, V3<T> b) { return V3<bool>(a.x > b.x, a.y > b.y, a.z > b.z); }
inline bool any(V3<bool> b) { return b.x || b.y || b.z; }
inline bool all(V3<bool> b) { return b.x && b.y && b.z; }
inline bool any(bool b) { return b; }

// ---- math
inline float min(float a, float b) { return std::fmin(a, b); }
inline float max(float a, float b) { return std::fmax(a, b); }
inline uint min(uint a, uint b) { return a < b ? a : b; }
inline uint max(uint a, uint b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline float2 min(float2 a, float2 b) { return float2(min(a.x, b.x), min(a.y, b.y)); }
inline float2 max(float2 a, float2 b) { return float2(max(a.x, b.x), max(a.y, b.y)); }
inline float3 min(float3 a, float3 b) { return float3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline float3 max(float3 a, float3 b) { return float3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline float3 min3(float3 a, float3 b, float3 c) { return min(min(a, b), c); }
inline float3 max3(float3 a, float3 b, float3 c) { return max(max(a, b), c); }
inline float min3(float a, float b, float c) { return min(min(a, b), c); }
inline float max3(float a, float b, float c) { return max(max(a, b), c); }
inline float clamp(float x, float a, float b) { return min(max(x, a), b); }
inline int3 min(int3 a, int3 b) { return int3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline int3 max(int3 a, int3 b) { return int3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline int3 clamp(int3 x, int3 a, int3 b) { return min(max(x, a), b); }
inline int clamp(int x, int a, int b) { return min(max(x, a), b); }
inline uint clamp(uint x, uint a, uint b) { return min(max(x, a), b); }
inline float3 clamp(float3 x, float3 a, float3 b) { return min(max(x, a), b); }
inline float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float3 cross(float3 a, float3 b) {
    return float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(float2 a) { return std::sqrt(dot(a, a)); }
inline float length(float3 a) { return std::sqrt(dot(a, a)); }
inline float distance(float3 a, float3 b) { return length(a - b); }
inline float3 normalize(float3 a) { return a * (1.0f / std::sqrt(dot(a, a))); }
inline float rsqrt(float x) { return 1.0f / std::sqrt(x); }
inline float3 mix(float3 a, float3 b, float t) { return a + (b - a) * t; }
inline float mix(float a, float b, float t) { return a + (b - a) * t; }
inline float fabs(float x) { return std::fabs(x); }
inline float abs(float x) { return std::fabs(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline float3 abs(float3 a) { return float3(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)); }
inline float3 fabs(float3 a) { return abs(a); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float floor(float x) { return std::floor(x); }
inline float3 floor(float3 a) { return float3(std::floor(a.x), std::floor(a.y), std::floor(a.z)); }
inline float log(float x) { return std::log(x); }
inline float sign(float x) { return (x > 0.f) ? 1.f : ((x < 0.f) ? -1.f : 0.f); }
inline uint clz(uint v) { return v ? (uint)__builtin_clz(v) : 32u; }
inline int clz(int v) { return v ? __builtin_clz((uint)v) : 32; }
inline uint popcount(uint v) { return (uint)__builtin_popcount(v); }
template <class T> inline T select(T a, T b, bool c) { return c ? b : a; }
template <class To, class From> inline To as_type(const From& f) {
    static_assert(sizeof(To) == sizeof(From), "as_type size");
    To t; std::memcpy(&t, &f, sizeof(To)); return t;
}

// ---- atomics
enum memory_order { memory_order_relaxed = 0, memory_order_seq_cst = 5, memory_order_acquire = 2,
                    memory_order_release = 3, memory_order_acq_rel = 4 };
enum class mem_flags { mem_none = 0, mem_device = 1, mem_threadgroup = 2, mem_texture = 4 };
enum thread_scope { thread_scope_thread, thread_scope_simdgroup, thread_scope_threadgroup, thread_scope_device };
inline std::memory_order to_std(memory_order o) {
    switch (o) {
        case memory_order_relaxed: return std::memory_order_relaxed;
        case memory_order_acquire: return std::memory_order_acquire;
        case memory_order_release: return std::memory_order_release;
        case memory_order_acq_rel: return std::memory_order_acq_rel;
        default: return std::memory_order_seq_cst;
    }
}
template <class T> struct Atomic { std::atomic<T> v; };
typedef Atomic<uint> atomic_uint;
typedef Atomic<int> atomic_int;
typedef Atomic<float> atomic_float;
static_assert(sizeof(atomic_uint) == 4, "atomic_uint size");
template <class T> inline T atomic_fetch_add_explicit(Atomic<T>* a, T v, memory_order o) { return a->v.fetch_add(v, to_std(o)); }
template <class T> inline T atomic_fetch_sub_explicit(Atomic<T>* a, T v, memory_order o) { return a->v.fetch_sub(v, to_std(o)); }
inline float atomic_fetch_add_explicit(atomic_float* a, float v, memory_order) {
    float old = a->v.load();
    while (!a->v.compare_exchange_weak(old, old + v)) {}
    return old;
}
inline float atomic_fetch_sub_explicit(atomic_float* a, float v, memory_order) {
    float old = a->v.load();
    while (!a->v.compare_exchange_weak(old, old - v)) {}
    return old;
}
template <class T> inline T atomic_load_explicit(Atomic<T>* a, memory_order o) { return a->v.load(to_std(o)); }
template <class T> inline void atomic_store_explicit(Atomic<T>* a, T v, memory_order o) { a->v.store(v, to_std(o)); }
template <class T> inline T atomic_exchange_explicit(Atomic<T>* a, T v, memory_order o) { return a->v.exchange(v, to_std(o)); }
template <class T> inline T atomic_fetch_max_explicit(Atomic<T>* a, T v, memory_order) {
    T old = a->v.load();
    while (old < v && !a->v.compare_exchange_weak(old, v)) {}
    return old;
}
template <class T> inline T atomic_fetch_min_explicit(Atomic<T>* a, T v, memory_order) {
    T old = a->v.load();
    while (old > v && !a->v.compare_exchange_weak(old, v)) {}
    return old;
}
template <class T> inline bool atomic_compare_exchange_weak_explicit(Atomic<T>* a, T* exp, T des, memory_order, memory_order) {
    return a->v.compare_exchange_weak(*exp, des);
}
inline void atomic_thread_fence(mem_flags, memory_order o, thread_scope = thread_scope_device) { std::atomic_thread_fence(to_std(o)); }
inline void threadgroup_barrier(mem_flags) {}
inline void simdgroup_barrier(mem_flags) {}

}  // namespace metal
