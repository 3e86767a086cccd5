// The covering radius of a sample (src/engine.zig:377-399 checkCovering/measureCovering, the
// stats keys of src/engine.zig:959-975): each source's star in the spherical Delaunay
// triangulation of its orbit, built on the GPU (k_cover.cuh), and the largest empty cap over
// all stars. Rounds: every source collects the orbit points within a reach expected to hold
// kCoverTarget of them; a source whose star is not proven within its reach runs again with
// the reach it reported, from the chart grid while the grid holds that reach, else from
// every image.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "engine.h"

namespace zo {
namespace {

constexpr double kPiH = 3.14159265358979323846;
constexpr double kCoverTarget = 48;         // expected orbit points within the first reach
constexpr double kCoverDensePairs = 4e9;    // n * n * |K| up to which every image is scanned
constexpr double kCoverGridRadius = 0.9;    // widest chart-grid reach (S3 angle)
constexpr int kCoverRounds = 8;

// The S3 angle of a cap holding `fraction` of the sphere: (phi - sin phi cos phi) / pi.
double cap_angle(double fraction) {
  double lo = 0, hi = kPiH;
  for (int k = 0; k < 80; ++k) {
    const double m = 0.5 * (lo + hi);
    if ((m - std::sin(m) * std::cos(m)) / kPiH < fraction) lo = m;
    else hi = m;
  }
  return 0.5 * (lo + hi);
}
double chord2_of(double angle) {
  const double c = 2.0 * std::sin(0.5 * std::min(angle, kPiH));
  return c * c;
}
double angle_of(double chord2) { return 2.0 * std::asin(std::min(1.0, 0.5 * std::sqrt(std::max(0.0, chord2)))); }

}  // namespace

double simplex_degrees(double count) {
  static const double c[] = {1.889832101454757, 0.573930763512449, 0.581069217539205, 0.859789414116394,
                             1.490131881944242, 2.791922498626376, 5.481645765756282, 11.12163594341394};
  const double t = std::cbrt(1.0 / count);
  double v = 0;
  for (int i = 7; i >= 0; --i) v = c[i] + t * t * v;
  return t * v * 360.0 / kPiH;
}

// A 64-bit hash of the group and the float32 orientations: four FNV-1a-style chains over
// 8-byte words (independent, so the multiplies overlap), each finished with a xor-shift
// multiply mix and combined. About 1 ms for a million orientations.
uint64_t Engine::sample_key() const {
  constexpr uint64_t kPrime = 1099511628211ull, kMix = 0x9e3779b97f4a7c15ull;
  uint64_t h[4] = {1469598103934665603ull ^ (uint64_t)group_, 0x243f6a8885a308d3ull, 0x13198a2e03707344ull,
                   0xa4093822299f31d0ull};
  const size_t floats = host_.size();
  const uint32_t* p = reinterpret_cast<const uint32_t*>(host_.data());
  size_t k = 0;
  for (; k + 8 <= floats; k += 8)
    for (int c = 0; c < 4; ++c) h[c] = (h[c] ^ ((uint64_t)p[k + 2 * c] | (uint64_t)p[k + 2 * c + 1] << 32)) * kPrime;
  for (; k < floats; ++k) h[0] = (h[0] ^ p[k]) * kPrime;
  uint64_t out = floats;
  for (int c = 0; c < 4; ++c) {
    uint64_t x = h[c] ^ (h[c] >> 31);
    x *= kMix;
    out = (out ^ (x ^ (x >> 29))) * kPrime;
  }
  return out;
}

void Engine::cover() {
  if (n_ < 4) throw Failure("TooFewOrientations");
  ZO_CUDA(cudaSetDevice(device_));
  cancelled_.store(false);
  const uint64_t key = sample_key();
  cover_cached_ = cover_ && cover_key_ == key && cover_iteration_ == iteration_ && point_covering_iteration_ &&
                  *point_covering_iteration_ == iteration_;
  if (cover_cached_) return;
  measure_covering();
  cover_key_ = key;
}

void Engine::measure_covering() {
  const int n = (int)n_;
  if (n >= (1 << 24)) throw Failure("TooManyOrientationsForCovering");
  const int order = (int)this->order();
  const double count_ext = 2.0 * order * n;
  const double phi = cap_angle(std::min(0.5, kCoverTarget / count_ext));
  const double reach2 = chord2_of(phi);
  cover_alpha_.ensure((size_t)n * sizeof(double));
  cover_centre_.ensure((size_t)n * sizeof(double4));
  cover_faces_.ensure((size_t)n * 4);
  cover_facets_.ensure((size_t)n * 4);
  cover_status_.ensure((size_t)n * 4);
  cover_need_.ensure((size_t)n * sizeof(double));
  cover_list_.ensure((size_t)n * 4);
  cover_probes_.ensure(sizeof(unsigned long long));
  ZO_CUDA(cudaMemsetAsync(cover_probes_.as<void>(), 0, sizeof(unsigned long long), stream_));

  CoverArgs A{};
  A.q = q32();
  A.n = n;
  A.gid = group_;
  A.alpha = cover_alpha_.as<double>();
  A.centre = cover_centre_.as<double4>();
  A.faces = cover_faces_.as<uint32_t>();
  A.facets = cover_facets_.as<uint32_t>();
  A.status = cover_status_.as<uint32_t>();
  A.need2 = cover_need_.as<double>();
  A.probes = cover_probes_.as<unsigned long long>();

  // The chart grid, complete to a reach well past the first one (most second runs stay in it).
  CoverResult r;
  // Forced to the chart grid (a development mode), the grid's reach stays below the widths
  // that the near field sums over every image for small samples.
  const bool dense_first = cover_mode_ == 1 ||
                           (cover_mode_ == 0 && ((double)n * n * order <= kCoverDensePairs || phi >= 0.3));
  double grid_reach2 = 0;
  if (!dense_first) {
    const double radius = std::min(cover_mode_ == 2 ? 0.45 : kCoverGridRadius, 3.0 * phi);
    const double d_r = mean_radius((double)n * order);
    if (!cover_near_) cover_near_ = std::make_unique<NearField>(group_, radius / d_r);
    else cover_near_->reconfigure(group_, radius / d_r);
    if (cover_near_->structure(stream_, q32(), q64(), n, d_r, sms_)) {
      grid_reach2 = chord2_of(cover_near_->radius());
      A.scode = cover_near_->sorted_codes();
      A.simg = cover_near_->sorted_images();
      A.cell_off = cover_near_->cell_offsets();
      A.grid = cover_near_->grid_device();
      A.grid_reach2 = grid_reach2;
      r.shell_points = (uint32_t)cover_near_->site_count(stream_);
      if (cover_near_->overflowed(stream_)) throw Failure("NearShellTooLarge");
    }
  }
  const NearGrid* grid = A.grid;

  // Round 0: every source at the first reach, in the narrow star.
  A.reach2 = reach2;
  A.reach2_of = nullptr;
  A.list = nullptr;
  A.count = n;
  ZO_CUDA(launch_cover(A, sms_, stream_, 0));
  r.rounds = 1;
  std::vector<uint32_t> status(n);
  std::vector<double> need(n);
  std::vector<double> used(n, reach2);  // the reach each source's star was built in
  std::vector<uint8_t> width(n, 0);     // the star width it was built in (0 narrow .. 2 wide)
  std::vector<uint32_t> listed, part[6];  // reruns: (grid, every image) x width
  for (int round = 1;; ++round) {
    ZO_CUDA(cudaMemcpyAsync(status.data(), A.status, (size_t)n * 4, cudaMemcpyDeviceToHost, stream_));
    ZO_CUDA(cudaMemcpyAsync(need.data(), A.need2, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    ZO_CUDA(cudaStreamSynchronize(stream_));
    if (cancelled_.load()) throw Failure("Cancelled");
    for (auto& p : part) p.clear();
    for (int i = 0; i < n; ++i) {
      if (status[i] != kCoverShort && status[i] != kCoverSparse) continue;
      if (round == 1) ++(status[i] == kCoverShort ? r.first_short : r.first_sparse);
      // A star short of a reach past the grid's is tried once at the grid's full reach first
      // (the kernel clamps to it): a star left open by points missing beyond a short reach
      // can show a cap much wider than its true one.
      const bool fits = grid && (need[i] <= grid_reach2 || used[i] < grid_reach2);
      used[i] = fits ? std::min(need[i], grid_reach2) : need[i];
      width[i] = (uint8_t)std::min(2, width[i] + 1);
      part[(fits ? 0 : 3) + width[i]].push_back((uint32_t)i);
    }
    size_t total = 0;
    for (const auto& p : part) total += p.size();
    if (total == 0 || round == kCoverRounds) break;
    r.rerun_grid += (uint32_t)(part[1].size() + part[2].size());
    r.rerun_dense += (uint32_t)(part[4].size() + part[5].size());
    // need2 holds each listed source's next reach: the kernel reads it before it writes.
    A.reach2_of = A.need2;
    listed.clear();
    for (const auto& p : part) listed.insert(listed.end(), p.begin(), p.end());
    ZO_CUDA(cudaMemcpyAsync(cover_list_.as<uint32_t>(), listed.data(), listed.size() * 4, cudaMemcpyHostToDevice,
                            stream_));
    size_t first = 0;
    for (int k = 0; k < 6; ++k) {
      if (!part[k].empty()) {
        A.grid = k < 3 ? grid : nullptr;
        A.list = cover_list_.as<uint32_t>() + first;
        A.count = (int)part[k].size();
        ZO_CUDA(launch_cover(A, sms_, stream_, k % 3));
      }
      first += part[k].size();
    }
    ++r.rounds;
  }

  // Results to the host: each source's largest cap and faces, the largest over all.
  std::vector<double> alpha(n);
  std::vector<uint32_t> faces(n), facets(n);
  ZO_CUDA(cudaMemcpyAsync(alpha.data(), A.alpha, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaMemcpyAsync(faces.data(), A.faces, (size_t)n * 4, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaMemcpyAsync(facets.data(), A.facets, (size_t)n * 4, cudaMemcpyDeviceToHost, stream_));
  unsigned long long probes = 0;
  ZO_CUDA(cudaMemcpyAsync(&probes, A.probes, sizeof probes, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaStreamSynchronize(stream_));
  point_covering_.resize(n_);
  point_faces_.resize(n_);
  int top = 0;
  double widest = 0;
  for (int i = 0; i < n; ++i) {
    if (status[i] != kCoverOk) ++r.unresolved;
    else widest = std::max(widest, used[i]);
    if (alpha[i] > alpha[top]) top = i;
    point_covering_.data()[i] = (float)(2.0 * alpha[i] * 180.0 / kPiH);
    point_faces_.data()[i] = (float)faces[i];
    r.facets += facets[i];
  }
  double4 centre;
  ZO_CUDA(cudaMemcpyAsync(&centre, A.centre + top, sizeof centre, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaStreamSynchronize(stream_));
  r.radius_deg = 2.0 * alpha[top] * 180.0 / kPiH;
  r.witness[0] = centre.x;
  r.witness[1] = centre.y;
  r.witness[2] = centre.z;
  r.witness[3] = centre.w;
  // A proven star's caps lie within its reach of its source: 2 a <= reach (S3), so every
  // empty cap is at most the widest such reach, in SO(3) degrees (twice the S3 angle of a).
  r.domain_bound_deg = std::max(r.radius_deg, angle_of(widest) * 180.0 / kPiH);
  r.probes = probes;
  cover_ = r;
  cover_iteration_ = iteration_;
  point_covering_iteration_ = iteration_;
  cover_reach_ = std::move(used);
  cover_width_ = std::move(width);
  cover_facet_counts_ = std::move(facets);
  cover_grid_reach2_ = grid ? grid_reach2 : 0.0;
}

void Engine::swap_covering() {
  CoverSaved& o = cover_saved_;
  std::swap(cover_, o.result);
  std::swap(cover_iteration_, o.iteration);
  std::swap(cover_key_, o.key);
  std::swap(point_covering_iteration_, o.point_iteration);
  point_covering_.swap(o.point_covering);
  point_faces_.swap(o.point_faces);
  cover_alpha_.swap(o.alpha);
  cover_centre_.swap(o.centre);
  cover_faces_.swap(o.faces);
  cover_facets_.swap(o.facets);
  cover_status_.swap(o.status);
  std::swap(cover_near_, o.near);
  std::swap(cover_reach_, o.reach);
  std::swap(cover_width_, o.width);
  std::swap(cover_facet_counts_, o.facet_counts);
  std::swap(cover_grid_reach2_, o.grid_reach2);
}

void Engine::set_covering_aside() {
  const bool current = cover_ && cover_key_ == sample_key() && cover_iteration_ == iteration_ &&
                       point_covering_iteration_ && *point_covering_iteration_ == iteration_;
  swap_covering();
  cover_saved_.valid = current;
  cover_.reset();  // what came back is older: the next cover() measures afresh
  cover_cached_ = false;
}

bool Engine::restore_covering() {
  if (!cover_saved_.valid || cover_saved_.iteration != iteration_ || cover_saved_.key != sample_key()) return false;
  swap_covering();
  cover_saved_.valid = false;
  return true;
}

// Every source's star again, in the reach and the star width that proved it (so that the
// same points are collected and the same facets found), written out as tetrahedra of point
// keys ((source << 8) | image; the source first) with each facet's unit normal (its cap's
// centre). The covering is brought up to date first.
void Engine::export_stars(std::vector<uint4>& tets, std::vector<double4>& normals) {
  cover();
  const int n = (int)n_;
  if (cover_reach_.size() != (size_t)n || cover_facet_counts_.size() != (size_t)n || cover_width_.size() != (size_t)n)
    throw Failure("CoveringNotMeasured");
  std::vector<uint32_t> offset(n + 1, 0);
  uint64_t total = 0;
  for (int i = 0; i < n; ++i) {
    offset[i] = (uint32_t)total;
    total += cover_facet_counts_[i];
    if (total > (1ull << 31)) throw Failure("MeshTooLarge");
  }
  offset[n] = (uint32_t)total;
  const uint64_t slots = std::max<uint64_t>(total, 1);
  cover_mesh_.ensure(slots * sizeof(uint4));
  cover_mesh_normal_.ensure(slots * sizeof(double4));
  cover_mesh_offset_.ensure((size_t)(n + 1) * 4);
  cover_need_.ensure((size_t)n * sizeof(double));
  ZO_CUDA(cudaMemcpyAsync(cover_mesh_offset_.as<uint32_t>(), offset.data(), (size_t)(n + 1) * 4,
                          cudaMemcpyHostToDevice, stream_));
  ZO_CUDA(cudaMemcpyAsync(cover_need_.as<double>(), cover_reach_.data(), (size_t)n * sizeof(double),
                          cudaMemcpyHostToDevice, stream_));
  ZO_CUDA(cudaMemsetAsync(cover_mesh_.as<void>(), 0xff, slots * sizeof(uint4), stream_));
  CoverArgs A{};
  A.q = q32();
  A.n = n;
  A.gid = group_;
  A.alpha = cover_alpha_.as<double>();
  A.centre = cover_centre_.as<double4>();
  A.faces = cover_faces_.as<uint32_t>();
  A.facets = cover_facets_.as<uint32_t>();
  A.status = cover_status_.as<uint32_t>();
  A.need2 = cover_need_.as<double>();
  A.reach2_of = cover_need_.as<double>();
  A.mesh = cover_mesh_.as<uint4>();
  A.mesh_offset = cover_mesh_offset_.as<uint32_t>();
  A.mesh_normal = cover_mesh_normal_.as<double4>();
  // Each source from the chart grid when its reach is within the grid's (the grid of the
  // covering pass, built for these positions), else from every image; in the star width
  // that proved it.
  std::vector<uint32_t> part[6];  // (grid, every image) x width
  for (int i = 0; i < n; ++i) {
    const bool in_grid = cover_grid_reach2_ > 0 && cover_reach_[i] <= cover_grid_reach2_;
    part[(in_grid ? 0 : 3) + cover_width_[i]].push_back((uint32_t)i);
  }
  std::vector<uint32_t> all;
  for (const auto& p : part) all.insert(all.end(), p.begin(), p.end());
  cover_list_.ensure((size_t)n * 4);
  ZO_CUDA(cudaMemcpyAsync(cover_list_.as<uint32_t>(), all.data(), all.size() * 4, cudaMemcpyHostToDevice, stream_));
  size_t first = 0;
  for (int k = 0; k < 6; ++k) {
    if (!part[k].empty()) {
      if (k < 3) {
        A.scode = cover_near_->sorted_codes();
        A.simg = cover_near_->sorted_images();
        A.cell_off = cover_near_->cell_offsets();
        A.grid = cover_near_->grid_device();
        A.grid_reach2 = cover_grid_reach2_;
      } else {
        A.grid = nullptr;
      }
      A.list = cover_list_.as<uint32_t>() + first;
      A.count = (int)part[k].size();
      ZO_CUDA(launch_cover(A, sms_, stream_, k % 3));
    }
    first += part[k].size();
  }
  tets.resize(total);
  normals.resize(total);
  if (total) {
    ZO_CUDA(cudaMemcpyAsync(tets.data(), A.mesh, total * sizeof(uint4), cudaMemcpyDeviceToHost, stream_));
    ZO_CUDA(cudaMemcpyAsync(normals.data(), A.mesh_normal, total * sizeof(double4), cudaMemcpyDeviceToHost, stream_));
  }
  ZO_CUDA(cudaStreamSynchronize(stream_));
}

// The orbit point of `key` ((source << 8) | 2 operator + sign), unit, FP64, from the float32
// sample and the float32 operator table (the kernels' definition).
void Engine::orbit_point(uint32_t key, double out[4]) const {
  const uint32_t j = key >> 8, im = key & 0xffu;
  const float* p = &host_[(size_t)j * 4];
  double a[4] = {p[0], p[1], p[2], p[3]};
  if (im >> 1) {
    const float* g = host_ops32(group_) + 4 * (im >> 1);
    const double b[4] = {g[0], g[1], g[2], g[3]};
    const double w = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
    const double x = a[0] * b[1] + b[0] * a[1] + a[2] * b[3] - a[3] * b[2];
    const double y = a[0] * b[2] + b[0] * a[2] + a[3] * b[1] - a[1] * b[3];
    const double z = a[0] * b[3] + b[0] * a[3] + a[1] * b[2] - a[2] * b[1];
    a[0] = w, a[1] = x, a[2] = y, a[3] = z;
  }
  const double norm = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3]);
  const double sign = (im & 1u) ? -1.0 : 1.0;
  for (int c = 0; c < 4; ++c) out[c] = sign * a[c] / norm;
}

// The triangulation display (src/exports.zig:88-103, Engine.buildMesh): the stars of every
// source as one mesh. The host numbers the points (the sources first, as their own vertices
// 0 .. n-1, then every other orbit point a star touches) and keeps each tetrahedron once.
// Vertices are stereographic (x, y, z) / (1 + w) of the unit orbit point, fourth component 0.
void Engine::build_mesh() {
  std::vector<uint4> tets;
  std::vector<double4> normals;
  export_stars(tets, normals);
  const int n = (int)n_;
  // Points: the sources first, then the other keys in order of first use.
  std::unordered_map<uint32_t, uint32_t> index;
  std::vector<uint32_t> keys;
  keys.reserve((size_t)n * 2);
  for (int i = 0; i < n; ++i) {
    index.emplace((uint32_t)i << 8, (uint32_t)i);
    keys.push_back((uint32_t)i << 8);
  }
  auto vertex = [&](uint32_t key) {
    auto it = index.find(key);
    if (it != index.end()) return it->second;
    const uint32_t v = (uint32_t)keys.size();
    index.emplace(key, v);
    keys.push_back(key);
    return v;
  };
  // Each tetrahedron once: its sorted vertex numbers as two 64-bit words.
  struct PairHash {
    size_t operator()(const std::pair<uint64_t, uint64_t>& k) const {
      return (size_t)(k.first * 0x9E3779B97F4A7C15ull ^ (k.second + 0x632BE59BD9B4E019ull) * 0xC2B2AE3D27D4EB4Full);
    }
  };
  std::unordered_set<std::pair<uint64_t, uint64_t>, PairHash> seen;
  mesh_tets_.clear();
  for (const uint4& t : tets) {
    if (t.x == 0xffffffffu || t.y == 0xffffffffu) continue;  // a star the export did not reproduce
    uint32_t v[4] = {vertex(t.x), vertex(t.y), vertex(t.z), vertex(t.w)};
    std::sort(v, v + 4);
    if (!seen.insert({((uint64_t)v[0] << 32) | v[1], ((uint64_t)v[2] << 32) | v[3]}).second) continue;
    mesh_tets_.insert(mesh_tets_.end(), v, v + 4);
  }
  mesh_vertices_.assign(keys.size() * 4, 0.f);
  for (size_t k = 0; k < keys.size(); ++k) {
    double p[4];
    orbit_point(keys[k], p);
    const double s = 1.0 / (1.0 + p[0]);
    for (int c = 0; c < 3; ++c) mesh_vertices_[k * 4 + c] = (float)(p[c + 1] * s);
  }
}

}  // namespace zo
