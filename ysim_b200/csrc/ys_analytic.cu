// ys_analytic.cu -- standalone analytic narrow phase (BruteForce::narrowAnalytic,
// include/sim/bruteforce.hpp:245-309, with narrow_pt_analytic,
// src/metal/bruteforce.metal:236-499).
//
// The reference dispatches one kernel per (cloth, collider) pair.  Here up to
// PAIRS_PER_LAUNCH pairs go into one launch: their shapes, rotation margins
// and vertex ranges travel in the kernel's parameter block (no device
// allocation), and thread i finds its pair among the launch's ranges.
#include <cstring>
#include <string>

#include "ys_analytic.cuh"
#include "ysim_b200.h"

namespace ys {
ys_status fail(ys_status code, const std::string& msg);
}

namespace ys {
namespace {

struct __align__(16) AJob {
    AShape sh;
    u32 oid, voff, nV, first;  // cloth mesh, its first packed vertex, count, first thread
    u32 qbeh;
    float rot_margin;
    u32 pad[2];
};
static_assert(sizeof(AJob) == 128, "AJob must be 128 bytes");

static constexpr int PAIRS_PER_LAUNCH = 24;  // 24 x 128 B + header < 4 KB of parameters

struct AJobs {
    AJob j[PAIRS_PER_LAUNCH];
    u32 n, total;
    float radius, thickness;
};

__global__ void __launch_bounds__(128) k_narrow_analytic(const __grid_constant__ AJobs J, const float* __restrict__ x,
                                                         const float* __restrict__ xp, Contact* __restrict__ out,
                                                         unsigned long long cap, unsigned long long* count) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= J.total) return;
    u32 k = 0;
    while (k + 1 < J.n && J.j[k + 1].first <= i) ++k;
    const AJob& b = J.j[k];
    const u32 id = i - b.first, g = b.voff + id;
    f3 n;
    float d;
    if (!analytic_narrow(b.sh, ldp(x, g), ldp(xp, g), J.radius, J.thickness, b.rot_margin, n, d)) return;
    const unsigned long long o = atomicAdd(count, 1ull);
    if (o >= cap) return;
    Contact c;
    c.point = id; c.tri = 0u; c.qobj = b.oid; c.tobj = b.sh.obj;
    c.nx = n.x; c.ny = n.y; c.nz = n.z; c.d = d;
    c.qbeh = b.qbeh; c.tbeh = b.sh.beh; c.qshape = COL_MESH; c.tshape = b.sh.kind;
    out[o] = c;
}

}  // namespace
}  // namespace ys

using namespace ys;

extern "C" ys_status ys_narrow_analytic(const float* d_x, const float* d_xprev, const uint32_t* state_off,
                                        const uint32_t* behaviors, uint32_t num_meshes,
                                        const ys_analytic_shape* shapes, uint32_t num_shapes, const uint32_t* pairs,
                                        uint32_t num_pairs, float radius, float thickness, void* d_out,
                                        uint64_t cap, unsigned long long* d_count, void* stream) {
    if (!d_x || !d_xprev || !state_off || !behaviors || !d_count || (num_shapes && !shapes) ||
        (num_pairs && !pairs) || (cap && !d_out))
        return fail(YS_ERR_BAD_ARG, "ys_narrow_analytic: null argument");
    static_assert(sizeof(ys_analytic_shape) == sizeof(AShape), "ys_analytic_shape layout");
    cudaStream_t st = (cudaStream_t)stream;
    AJobs J;
    memset(&J, 0, sizeof(J));
    J.radius = radius;
    J.thickness = thickness;
    auto launch = [&]() -> ys_status {
        if (J.n == 0) return YS_OK;
        k_narrow_analytic<<<ceil_div(J.total, 128), 128, 0, st>>>(J, d_x, d_xprev, (Contact*)d_out, cap, d_count);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return fail(YS_ERR_CUDA, std::string("ys_narrow_analytic: ") + cudaGetErrorString(e));
        J.n = 0;
        J.total = 0;
        return YS_OK;
    };
    for (uint32_t p = 0; p < num_pairs; ++p) {
        const uint32_t cloth = pairs[2 * p], obj = pairs[2 * p + 1];
        if (cloth >= num_meshes) continue;
        // compact slot of the collider (the reference's linear objIndex scan)
        int slot = -1;
        for (uint32_t k = 0; k < num_shapes; ++k)
            if (shapes[k].obj_index == obj) { slot = (int)k; break; }
        if (slot < 0) continue;
        AShape sh;
        memcpy(&sh, &shapes[slot], sizeof(sh));
        if (!(sh.flags & 1u)) continue;
        const uint32_t nV = state_off[cloth + 1] - state_off[cloth];
        if (nV == 0) continue;
        if ((uint64_t)J.total + nV > 0x7FFFFFFFull) {  // keep thread indices in range
            ys_status r = launch();
            if (r) return r;
        }
        AJob& b = J.j[J.n++];
        b.sh = sh;
        b.oid = cloth;
        b.voff = state_off[cloth];
        b.nV = nV;
        b.first = J.total;
        b.qbeh = behaviors[cloth];
        b.rot_margin = analytic_rot_margin(sh, radius, thickness);
        J.total += nV;
        if (J.n == PAIRS_PER_LAUNCH) {
            ys_status r = launch();
            if (r) return r;
        }
    }
    return launch();
}
