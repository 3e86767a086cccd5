// Exact-count generation (src/engine.zig:199-231 generateExact): the largest inverse-Hopf grid
// that fits the target, then points inserted at the centres of the largest empty Delaunay
// caps until the sample has exactly the target count. The caps come from the GPU's Delaunay
// stars (export_stars, k_cover.cuh); the selection follows the steps of src/insert.zig:150-241
// (largest cap first; a centre is taken only if its cap holds no point of the sample's orbit
// and no centre taken before, up to symmetry) and the distinctness pass of src/dedup.zig.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "hopf.h"

namespace zo {
namespace {

void qmul4(const double a[4], const double b[4], double out[4]) {
  out[0] = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  out[1] = a[0] * b[1] + b[0] * a[1] + a[2] * b[3] - a[3] * b[2];
  out[2] = a[0] * b[2] + b[0] * a[2] + a[3] * b[1] - a[1] * b[3];
  out[3] = a[0] * b[3] + b[0] * a[3] + a[1] * b[2] - a[2] * b[1];
}
double dot4h(const double a[4], const double b[4]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3]; }

// Unit quaternions hashed by their (x, y, z) in cubes of side `cell`.
class PointGrid {
 public:
  explicit PointGrid(double cell) : cell_(cell) {}
  void add(const double q[4]) {
    const size_t at = points_.size() / 4;
    points_.insert(points_.end(), q, q + 4);
    cells_[key(cell_of(q[1]), cell_of(q[2]), cell_of(q[3]))].push_back((uint32_t)at);
  }
  // Adds q and -q.
  void add_both(const double q[4]) {
    const double m[4] = {-q[0], -q[1], -q[2], -q[3]};
    add(q);
    add(m);
  }
  // Whether a stored point p has q . p > threshold (p within the chord of that threshold).
  bool near(const double q[4], double threshold) const {
    const double chord = std::sqrt(std::max(0.0, 2.0 - 2.0 * threshold)) * (1 + 1e-9) + 1e-12;
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = cell_of(q[a + 1] - chord);
      hi[a] = cell_of(q[a + 1] + chord);
    }
    for (int x = lo[0]; x <= hi[0]; ++x)
      for (int y = lo[1]; y <= hi[1]; ++y)
        for (int z = lo[2]; z <= hi[2]; ++z) {
          auto it = cells_.find(key(x, y, z));
          if (it == cells_.end()) continue;
          for (uint32_t p : it->second)
            if (dot4h(q, &points_[(size_t)p * 4]) > threshold) return true;
        }
    return false;
  }
  // Whether a stored point lies within Euclidean distance `tol` of q.
  bool within(const double q[4], double tol) const {
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = cell_of(q[a + 1] - tol);
      hi[a] = cell_of(q[a + 1] + tol);
    }
    for (int x = lo[0]; x <= hi[0]; ++x)
      for (int y = lo[1]; y <= hi[1]; ++y)
        for (int z = lo[2]; z <= hi[2]; ++z) {
          auto it = cells_.find(key(x, y, z));
          if (it == cells_.end()) continue;
          for (uint32_t p : it->second) {
            const double* s = &points_[(size_t)p * 4];
            double d = 0;
            for (int c = 0; c < 4; ++c) d += (q[c] - s[c]) * (q[c] - s[c]);
            if (d < tol * tol) return true;
          }
        }
    return false;
  }

 private:
  int cell_of(double v) const { return (int)std::floor(v / cell_); }
  static uint64_t key(int x, int y, int z) {
    return ((uint64_t)(uint32_t)(x + (1 << 20)) << 42) | ((uint64_t)(uint32_t)(y + (1 << 20)) << 21) |
           (uint64_t)(uint32_t)(z + (1 << 20));
  }
  double cell_;
  std::vector<double> points_;
  std::unordered_map<uint64_t, std::vector<uint32_t>> cells_;
};

struct Cap {
  double c[4];
  double radius;
};

}  // namespace

// Up to `wanted` new orientations at the centres of the sample's largest empty caps
// (src/insert.zig:150-241). Every Delaunay facet that touches an orientation comes from the
// GPU stars with its normal (its cap's centre); a cap is an image of one whose centre is in
// the zone, so each centre is taken to its zone image (the image nearest the identity).
// Largest caps first, a centre is taken when it is not already taken and its cap, less
// 3e-7 in cosine, holds no orbit point of the sample and no image of a centre taken before.
std::vector<float> Engine::insertion_centres(uint32_t wanted) {
  std::vector<uint4> tets;
  std::vector<double4> normals;
  export_stars(tets, normals);
  const int order = (int)this->order();
  std::vector<double> ops((size_t)order * 4);
  for (int k = 0; k < order; ++k) {
    const float* g = host_ops32(group_) + 4 * k;
    const double norm = std::sqrt((double)g[0] * g[0] + (double)g[1] * g[1] + (double)g[2] * g[2] + (double)g[3] * g[3]);
    for (int c = 0; c < 4; ++c) ops[(size_t)k * 4 + c] = g[c] / norm;
  }
  std::vector<Cap> caps;
  caps.reserve(tets.size());
  double widest = 0;
  for (size_t t = 0; t < tets.size(); ++t) {
    if (tets[t].x == 0xffffffffu) continue;
    double x[4];
    orbit_point(tets[t].x, x);
    const double n[4] = {normals[t].x, normals[t].y, normals[t].z, normals[t].w};
    const double h = dot4h(n, x);
    if (!(h > 0.0 && h < 1.0)) continue;
    Cap cap;
    cap.radius = std::acos(h);
    double best = -2;
    for (int k = 0; k < order; ++k) {
      double img[4];
      qmul4(n, &ops[(size_t)k * 4], img);
      const double s = img[0] < 0 ? -1.0 : 1.0;
      if (s * img[0] > best) {
        best = s * img[0];
        for (int c = 0; c < 4; ++c) cap.c[c] = s * img[c];
      }
    }
    widest = std::max(widest, cap.radius);
    caps.push_back(cap);
  }
  if (caps.empty()) throw Failure("NoDelaunayCentres");
  std::stable_sort(caps.begin(), caps.end(), [](const Cap& a, const Cap& b) { return a.radius > b.radius; });
  // The sample's orientations (both signs) and the centres taken, hashed.
  PointGrid occupied(std::max(1e-3, 2.0 * std::sin(0.5 * widest)));
  for (uint32_t j = 0; j < n_; ++j) {
    double q[4];
    orbit_point(j << 8, q);
    occupied.add_both(q);
  }
  std::vector<float> out;
  for (const Cap& cap : caps) {
    if (cancelled_.load()) throw Failure("Cancelled");
    if (occupied.near(cap.c, 1 - 1e-12)) continue;  // a centre already taken (co-spherical facets)
    const double height = std::cos(cap.radius);
    bool blocked = false;
    for (int k = 0; k < order && !blocked; ++k) {
      const double inv[4] = {ops[(size_t)k * 4], -ops[(size_t)k * 4 + 1], -ops[(size_t)k * 4 + 2],
                             -ops[(size_t)k * 4 + 3]};
      double query[4];
      qmul4(cap.c, inv, query);
      blocked = occupied.near(query, height + 3e-7);
    }
    if (blocked) continue;
    occupied.add_both(cap.c);
    for (int c = 0; c < 4; ++c) out.push_back((float)cap.c[c]);
    if (out.size() / 4 == wanted) break;
  }
  if (out.empty()) throw Failure("NoEmptyDelaunayCentres");
  return out;
}

// The leading `unique` rows are distinct already; of the rest, keep each row no image of which
// lies within 2e-6 of a row kept before it (src/dedup.zig). Returns the rows kept.
uint32_t Engine::distinct_rows(std::vector<float>& values, uint32_t unique) const {
  const int order = (int)this->order();
  const float* ops = host_ops32(group_);
  const double tol = 2e-6;
  PointGrid kept(4 * tol);
  const uint32_t rows = (uint32_t)(values.size() / 4);
  uint32_t count = 0;
  for (uint32_t i = 0; i < rows; ++i) {
    const double q[4] = {values[i * 4], values[i * 4 + 1], values[i * 4 + 2], values[i * 4 + 3]};
    bool duplicate = false;
    for (int k = 0; k < order && i >= unique && !duplicate; ++k) {
      const double g[4] = {ops[k * 4], ops[k * 4 + 1], ops[k * 4 + 2], ops[k * 4 + 3]};
      double p[4];
      qmul4(q, g, p);
      const double norm = std::sqrt(dot4h(p, p));
      for (int c = 0; c < 4; ++c) p[c] /= norm;
      const double m[4] = {-p[0], -p[1], -p[2], -p[3]};
      duplicate = kept.within(p, tol) || kept.within(m, tol);
    }
    if (duplicate) continue;
    for (int c = 0; c < 4; ++c) values[count * 4 + c] = (float)q[c];
    kept.add(q);
    ++count;
  }
  values.resize((size_t)count * 4);
  return count;
}

void Engine::generate_exact(int gid, uint32_t target, bool add_identity, uint32_t kind) {
  if (target < 32 || target > 1000000) throw Failure("ExactCountRange32To1000000");
  if (kind == 2) throw Failure(gid < 8 ? "TransportNeedsTOrOOrI" : "TransportNotAvailable");
  const uint32_t budget = target - (add_identity ? 1 : 0);
  const std::optional<uint32_t> h = hopf::largest_frequency(gid, budget);
  if (!h) throw Failure("BaseGridExceedsTarget");
  generate_grid(gid, *h, target, 0, kind);
  const uint32_t base_count = n_;
  if (add_identity) identity(true, fix_identity_);
  const std::string generator = generator_, grid_kind = grid_kind_;
  for (int round = 0; round < 8 && n_ != target; ++round) {
    if (n_ > target) throw Failure("BaseGridExceedsTarget");
    std::vector<float> values(host_);
    const std::vector<float> additions = insertion_centres(target - n_);
    values.insert(values.end(), additions.begin(), additions.end());
    const uint32_t keep = distinct_rows(values, n_);
    if (keep <= n_) throw Failure("NoDistinctDelaunayCentres");
    const bool fixed = fix_identity_;
    set(gid, values.data(), keep);
    if (fixed) identity(false, true);
  }
  if (n_ != target) throw Failure("InsufficientDelaunayCentres");
  generator_ = generator;
  grid_kind_ = grid_kind;
  h_ = *h;
  base_count_ = base_count;
  inserted_count_ = target - base_count;
}

}  // namespace zo
