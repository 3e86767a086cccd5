// extern "C" entry points: the reference's zo_* ABI (src/exports.zig, src/native_api.zig),
// bound by ctypes from Python (python/zxtalori/api.py:29-50). 0 is success, -1 failure with
// the message in the engine's 2,048-byte error buffer, prefixed as the reference does.
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>

#include "engine.h"
#include "hopf.h"
#include "zxtalori.h"

using zo::Engine;

namespace {
char g_create_error[1024] = {0};

template <class F>
int guarded(void* h, const char* prefix, F&& f) {
  Engine* e = static_cast<Engine*>(h);
  try {
    zo::AllocScope scope(e->stream());  // the call's device buffers are ordered on its stream
    f(*e);
    return 0;
  } catch (const std::exception& x) {
    std::snprintf(e->err, sizeof e->err, "%s: %s", prefix, x.what());
    return -1;
  }
}

int fail(void* h, const char* message) {
  Engine* e = static_cast<Engine*>(h);
  std::snprintf(e->err, sizeof e->err, "%s", message);
  return -1;
}

}  // namespace

extern "C" {

const char* zo_version(void) { return "0.3.0"; }

void* zo_create(const char* wgpu_dir) {
  (void)wgpu_dir;
  try {
    return new Engine();
  } catch (const std::exception& x) {
    std::snprintf(g_create_error, sizeof g_create_error, "GPU init: %s", x.what());
    return nullptr;
  }
}

const char* zo_create_error(void) { return g_create_error; }

void zo_destroy(void* h) { delete static_cast<Engine*>(h); }

int zo_generate(void* h, uint32_t group, uint32_t freq, uint32_t target, uint32_t seed, uint32_t kind) {
  if (group >= 11) return fail(h, "Unknown group");
  if (kind > 2) return fail(h, "Unknown grid kind");
  return guarded(h, "Generation failed", [&](Engine& e) { e.generate_grid((int)group, freq, target, seed, kind); });
}

int zo_generate_exact(void* h, uint32_t group, uint32_t target, uint32_t flags) {
  if (group >= 11) return fail(h, "Unknown group");
  // flags: bit 0 adds the identity; bits 8-15 are the grid kind, as in zo_generate.
  if (((flags >> 8) & 0xffu) > 2) return fail(h, "Unknown grid kind");
  return guarded(h, "Exact-count generation", [&](Engine& e) {
    e.generate_exact((int)group, target, (flags & 1u) != 0, (flags >> 8) & 0xffu);
  });
}

int zo_random(void* h, uint32_t group, uint32_t count, uint32_t seed) {
  if (group >= 11) return fail(h, "Unknown group");
  return guarded(h, "Haar initialization", [&](Engine& e) { e.generate_random((int)group, count, seed); });
}

int zo_set(void* h, uint32_t group, const float* q, uint32_t n) {
  if (group >= 11) return fail(h, "Unknown group");
  return guarded(h, "Import failed", [&](Engine& e) {
    if (n > 0 && !q) throw zo::Failure("InvalidCount");
    e.set((int)group, q, n);
  });
}

uint32_t zo_count(void* h) { return static_cast<Engine*>(h)->count(); }
uint32_t zo_order(void* h) { return static_cast<Engine*>(h)->order(); }
const float* zo_quaternions(void* h) { return static_cast<Engine*>(h)->quaternions(); }
const float* zo_operations(void* h) { return zo::host_ops32(static_cast<Engine*>(h)->group()); }

int zo_measure(void* h) { return guarded(h, "Measure failed", [](Engine& e) { e.measure(); }); }
int zo_measure_full(void* h) { return guarded(h, "Measure failed", [](Engine& e) { e.measure_full(); }); }
int zo_spacing(void* h) { return guarded(h, "Spacing failed", [](Engine& e) { e.spacing(); }); }
int zo_relax(void* h, uint32_t steps) { return guarded(h, "Relaxation failed", [&](Engine& e) { e.relax(steps); }); }

int zo_relax_neighbourhood(void* h, float delta) {
  return guarded(h, "Relaxation neighbourhood", [&](Engine& e) { e.set_neighbourhood((double)delta); });
}

const float* zo_point_values(void* h, uint32_t kind) { return static_cast<Engine*>(h)->point_values(kind); }

int zo_identity(void* h, uint32_t flags) {
  return guarded(h, "Identity constraint", [&](Engine& e) { e.identity((flags & 1u) != 0, (flags & 2u) != 0); });
}

int zo_cover(void* h) { return guarded(h, "Covering radius", [](Engine& e) { e.cover(); }); }
int zo_cover_optimize(void* h, uint32_t steps, uint32_t mode, uint32_t finish, float floor_deg) {
  return guarded(h, "Covering optimization",
                 [&](Engine& e) { e.optimize_covering(steps, mode, finish != 0, (double)floor_deg); });
}
int zo_cover_kicks(void* h, uint32_t patience, float progress, float size, float trust) {
  return guarded(h, "Covering kicks", [&](Engine& e) { e.set_kicks(patience, progress, size, trust); });
}
int zo_mesh(void* h) { return guarded(h, "DT display", [](Engine& e) { e.build_mesh(); }); }
const float* zo_mesh_vertices(void* h) {
  const auto& v = static_cast<Engine*>(h)->mesh_vertices();
  return v.empty() ? nullptr : v.data();
}
const uint32_t* zo_mesh_tets(void* h) {
  const auto& t = static_cast<Engine*>(h)->mesh_tets();
  return t.empty() ? nullptr : t.data();
}
uint32_t zo_mesh_vertex_count(void* h) { return (uint32_t)(static_cast<Engine*>(h)->mesh_vertices().size() / 4); }
uint32_t zo_mesh_tet_count(void* h) { return (uint32_t)(static_cast<Engine*>(h)->mesh_tets().size() / 4); }

const char* zo_stats(void* h) { return static_cast<Engine*>(h)->stats(); }
const char* zo_error(void* h) { return static_cast<Engine*>(h)->err; }
void zo_cancel(void* h) { static_cast<Engine*>(h)->cancel(); }

void zo_pair_budget(void* h, float scale) { static_cast<Engine*>(h)->set_pair_budget((double)scale); }
bool zo_profile(void* h, bool enabled) {
  (void)h;
  (void)enabled;
  return false;
}
size_t zo_profile_report(void* h, uint8_t* output, size_t capacity) {
  (void)h;
  if (output && capacity) output[0] = 0;
  return 0;
}

int zo_precision(void* h, uint32_t mode) {
  return guarded(h, "Precision", [&](Engine& e) { e.set_precision((int)mode); });
}
uint32_t zo_get_precision(void* h) { return (uint32_t) static_cast<Engine*>(h)->precision(); }
const int32_t* zo_point_neighbours(void* h) {
  Engine* e = static_cast<Engine*>(h);
  try {
    return e->point_neighbours();
  } catch (const std::exception& x) {
    std::snprintf(e->err, sizeof e->err, "Neighbours: %s", x.what());
    return nullptr;
  }
}

int zo_near_tiles(void* h, uint32_t sources_per_warp, float sites_per_cell) {
  return guarded(h, "Tiles", [&](Engine& e) {
    if (sources_per_warp == 0) e.force_tiles(std::nullopt);
    else e.force_tiles(zo::NearTiles{(int)sources_per_warp, (double)sites_per_cell});
  });
}

int zo_near_walk(void* h, float fraction) {
  return guarded(h, "Tiles", [&](Engine& e) { e.force_walk((double)fraction); });
}

int zo_tiles_lookup(uint32_t kind, uint32_t group, uint32_t n, double* out) {
  if (group >= 11 || kind > 1 || !out) return -1;
  const zo::NearTiles t = zo::lookup_tiles((int)kind, (int)group, (int)n);
  out[0] = t.group_size;
  out[1] = t.sites_per_cell;
  out[2] = t.walk;
  return 0;
}

uint64_t zo_device_bytes(void* h) { return h ? (uint64_t) static_cast<Engine*>(h)->device_bytes() : 0; }

int zo_spacing_exact(void* h, uint32_t* out) {
  return guarded(h, "Spacing", [&](Engine& e) { e.spacing_exact(out, out + 1); });
}

int zo_debug_shell_capacity(void* h, uint32_t sites) {
  return guarded(h, "Rows", [&](Engine& e) { e.debug_shell_capacity(sites); });
}

int zo_debug_cover_mode(void* h, uint32_t mode) {
  return guarded(h, "Covering radius", [&](Engine& e) { e.debug_cover_mode(mode); });
}

int zo_debug_pair_counts(void* h, double* out) {
  return guarded(h, "Rows", [&](Engine& e) { e.debug_pair_counts(out); });
}

int zo_debug_rows(void* h, uint32_t what, double* out) {
  return guarded(h, "Rows", [&](Engine& e) { e.debug_rows(what, out); });
}

int zo_bench(void* h, uint32_t steps, uint32_t warmup, double flush_bytes, double* out, uint32_t out_len) {
  return guarded(h, "Bench", [&](Engine& e) { e.bench(steps, warmup, flush_bytes, out, out_len); });
}

int zo_bench_spacing(void* h, uint32_t passes, uint32_t warmup, double flush_bytes, double* out, uint32_t out_len) {
  return guarded(h, "Bench", [&](Engine& e) { e.bench_spacing(passes, warmup, flush_bytes, out, out_len); });
}

int zo_relax_async(void* h, uint32_t steps) {
  return guarded(h, "Relaxation failed", [&](Engine& e) { e.relax_async(steps); });
}

int zo_relax_finish(void* h) { return guarded(h, "Relaxation failed", [](Engine& e) { e.relax_finish(); }); }

int zo_idle(void* h) {
  int idle = 0;
  if (guarded(h, "Relaxation failed", [&](Engine& e) { idle = e.idle() ? 1 : 0; }) != 0) return -1;
  return idle;
}

int zo_graphs(void* h, uint32_t enabled) {
  return guarded(h, "Graphs", [&](Engine& e) { e.set_graphs(enabled != 0); });
}

int64_t zo_hopf_points(uint32_t group, uint32_t freq, float* out, uint64_t capacity) {
  if (group >= 11) return -1;
  try {
    const uint64_t n = zo::hopf::count((int)group, freq);
    if (!out) return (int64_t)n;
    if (capacity < n) return -2;
    const std::vector<float> rows = zo::hopf::points((int)group, freq);
    std::memcpy(out, rows.data(), rows.size() * sizeof(float));
    return (int64_t)n;
  } catch (const std::exception&) {
    return -1;
  }
}

int zo_zone_planes(uint32_t group, uint8_t* order, float* reach) {
  if (group >= 11 || !order || !reach) return -1;
  const zo::HostTables& t = zo::host_tables();
  const int off = t.plane_offset[group], planes = 2 * t.group_order[group] - 1;
  for (int r = 0; r < planes; ++r) {
    order[r] = t.plane_order[off + r];
    reach[r] = t.plane_reach[off + r];
  }
  return planes;
}

double zo_fp32_peak(void* h) {
  double value = -1.0;
  if (guarded(h, "Probe", [&](Engine& e) { value = e.fp32_peak(); }) != 0) return -1.0;
  return value;
}

double zo_fp32x2_peak(void* h) {
  double value = -1.0;
  if (guarded(h, "Probe", [&](Engine& e) { value = e.fp32_peak(true); }) != 0) return -1.0;
  return value;
}

}  // extern "C"
