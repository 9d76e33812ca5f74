// ref_sceneio.cpp -- host harness over the reference's own scene-file,
// run-config, primitive-geometry and frame-profiler headers
// (include/scene_format.hpp, sim_config.hpp, primitive_geometry.hpp,
// FrameProfiler.hpp; they are plain C++
// with the bundled nlohmann/json and no Metal).  TEST INFRASTRUCTURE ONLY:
// compiled by oracle/build_ref.py from the reference checkout in place into
// oracle/_ref/libysref.so, so that the loader in ysim_b200/scene_format.py
// and ysim_b200/primitives.py can be checked against the reference itself.
// FrameProfiler.hpp's CSV export is driven with given frames.  Also exposes
// libstdc++'s std::mt19937 + std::uniform_real_distribution<float>
// (the grid initializer's jiggle source) so the restated generator can be
// checked against the standard library it follows.
#include <cstdint>
#include <cstring>
#include <random>
#include <string>

#include "FrameProfiler.hpp"
#include "primitive_geometry.hpp"
#include "scene_format.hpp"
#include "sim_config.hpp"

namespace {
int put(const std::string& s, char* out, size_t cap) {
    if (!out || cap == 0) return -1;
    size_t n = s.size() < cap - 1 ? s.size() : cap - 1;
    std::memcpy(out, s.data(), n);
    out[n] = 0;
    return (int)s.size();
}
}  // namespace

extern "C" {

// scene_format::parseString then toString: returns 0 and the re-encoded JSON,
// or 1 and the load error.  *warnings receives the number of load warnings.
int yref_scene_roundtrip(const char* text, char* out, size_t cap, int* warnings) {
    auto r = scene_format::parseString(text);
    if (!r.ok) {
        put(r.error.message, out, cap);
        return 1;
    }
    if (warnings) *warnings = (int)r.value.warnings.messages.size();
    put(scene_format::toString(r.value), out, cap);
    return 0;
}

// The same through sim_config (scene + engine + profile blocks).
int yref_runconfig_roundtrip(const char* text, char* out, size_t cap) {
    auto r = sim_config::parseString(text);
    if (!r.ok) {
        put(r.error.message, out, cap);
        return 1;
    }
    put(sim_config::toString(r.value), out, cap);
    return 0;
}

// primitive::sphere / cube / cylinder (kind 0 / 1 / 2) at the origin:
// vertex and facet counts, positions and facets into the buffers (when
// large enough).
int yref_primitive(int kind, float size, int tess, float* pos, uint32_t* facets, size_t cap_v, size_t cap_f,
                   uint32_t* nv, uint32_t* nf) {
    primitive::Geometry g = kind == 0 ? primitive::sphere(size, tess)
                                      : (kind == 1 ? primitive::cube(size, tess) : primitive::cylinder(size, tess));
    *nv = (uint32_t)(g.positions.size() / 3);
    *nf = (uint32_t)(g.facets.size() / 3);
    if (pos && g.positions.size() <= 3 * cap_v) std::memcpy(pos, g.positions.data(), 4 * g.positions.size());
    if (facets && g.facets.size() <= 3 * cap_f) std::memcpy(facets, g.facets.data(), 4 * g.facets.size());
    return 0;
}

// n draws of std::uniform_real_distribution<float>(lo, hi) over
// std::mt19937(seed), as the grid initializer's jiggle makes them.
void yref_uniform_float(uint32_t seed, float lo, float hi, uint32_t n, float* out) {
    std::mt19937 rng(seed);
    std::uniform_real_distribution<float> d(lo, hi);
    for (uint32_t i = 0; i < n; ++i) out[i] = d(rng);
}

// FrameProfilerHistory::push + exportCsv for given frames (fps from frame_ms
// as FrameProfiler::endFrame computes it); sec_ms is nframes x nsec.
int yref_profiler_csv(const char* path, int nframes, const uint64_t* seq, const double* wall, const double* frame_ms,
                      const uint64_t* broad, const uint64_t* narrow, int nsec, const char* const* names,
                      const double* sec_ms, int max_frames) {
    profiler::FrameProfilerHistory h((std::size_t)max_frames);
    for (int k = 0; k < nsec; ++k) h.ensureSection(names[k]);
    for (int i = 0; i < nframes; ++i) {
        profiler::FrameSnapshot s;
        s.sequence = seq[i];
        s.wall_time_seconds = wall[i];
        s.frame_ms = frame_ms[i];
        s.fps = frame_ms[i] > 0.0 ? 1000.0 / frame_ms[i] : 0.0;
        s.broad_collisions = broad[i];
        s.narrow_collisions = narrow[i];
        s.section_ms.assign(sec_ms + (size_t)i * nsec, sec_ms + (size_t)(i + 1) * nsec);
        h.push(s);
    }
    return h.exportCsv(path) ? 0 : 1;
}

// sim_config::defaultProfilePath / sidecarScenePath / pathStem.
int yref_profile_paths(const char* root, const char* scene_path, int frames, char* out, size_t cap) {
    std::string s = sim_config::defaultProfilePath(root, sim_config::pathStem(scene_path), frames);
    s += "\n" + sim_config::sidecarScenePath(s);
    return put(s, out, cap);
}

}  // extern "C"
