// Inverse-Hopf product grids (src/hopf.zig), FP64 on the host.
//
// pi(q) = q^-1 z maps SO(3) onto the sphere with fibres {R_z(t) q}, and pi(q g) = g^-1 pi(q),
// so a K-invariant sphere mesh times n fibre angles is a grid on SO(3)/K. Three root grids
// are built directly (octahedral and icosahedral meshes mapped to the sphere by an
// area-preserving Knothe-Rosenblatt map, and equal-area latitude rings for D6); every other
// group inherits one through a rotation R with R H R^-1 inside the root. Each K-orbit of
// mesh nodes contributes R_z(t_j) s(v) c R for the orbit's sector node v, its section s(v),
// the cosets c and n / stabiliser fibre angles t_j, alternate layers half a step apart.
//
// The row order, the base polyhedra's vertex and face tables, the embeddings and the
// tie-breaking rules follow the reference exactly: they define which rows the grid has and
// in which order, which its fixtures (SO3K_Grids product grids) pin.
#include "hopf.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <thread>
#include <unordered_map>
#include <unordered_set>

#include "engine.h"

namespace zo::hopf {
namespace {

using Quat = std::array<double, 4>;
using Vec = std::array<double, 3>;
using Mat = std::array<Vec, 3>;
constexpr double kPi = 3.14159265358979323846;

enum Group { C2, C3, C4, C6, D2, D3, D4, D6, T, O, I };
constexpr int kOrder[11] = {2, 3, 4, 6, 4, 6, 8, 12, 12, 24, 60};

Quat qmul(const Quat& a, const Quat& b) {
  return {a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
          a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2],
          a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1],
          a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0]};
}
double qdot(const Quat& a, const Quat& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3]; }
Quat qnormalize(const Quat& q) {
  const double s = 1 / std::sqrt(qdot(q, q));
  return {q[0] * s, q[1] * s, q[2] * s, q[3] * s};
}
double vdot(const Vec& a, const Vec& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
Vec vunit(const Vec& v) {
  const double s = 1 / std::sqrt(vdot(v, v));
  return {v[0] * s, v[1] * s, v[2] * s};
}
Vec mul(const Mat& m, const Vec& v) { return {vdot(m[0], v), vdot(m[1], v), vdot(m[2], v)}; }
Vec mul_transposed(const Mat& m, const Vec& v) {
  return {m[0][0] * v[0] + m[1][0] * v[1] + m[2][0] * v[2], m[0][1] * v[0] + m[1][1] * v[1] + m[2][1] * v[2],
          m[0][2] * v[0] + m[1][2] * v[1] + m[2][2] * v[2]};
}
Mat rotation_matrix(const Quat& q) {
  const double w = q[0], x = q[1], y = q[2], z = q[3];
  return Mat{Vec{1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)},
             Vec{2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)},
             Vec{2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)}};
}
// Rotation by 2 pi / turns about `axis`.
Quat turn(const Vec& axis, double turns) {
  const Vec a = vunit(axis);
  const double s = std::sin(kPi / turns);
  return {std::cos(kPi / turns), a[0] * s, a[1] * s, a[2] * s};
}

int root_group(int gid) {
  switch (gid) {
    case C2: case C3: case D2: case D3: case T: case I: return I;
    case C4: case D4: case O: return O;
    default: return D6;
  }
}

// R with R H R^-1 inside the root (so3k.product.embedding; src/hopf.zig:37-43).
Quat embedding(int gid) {
  switch (gid) {
    case C2: case D2: case T: return {0.9619383577839175, 0, 0.2732665289126717, 0};
    case C3: case D3: return {0.9459753748917731, 0.17451645846277514, 0.2687317799958305, -0.04957646865452023};
    default: return {1, 0, 0, 0};
  }
}

// Group elements in FP64: closure of the generators, normalised with w >= 0 and stably
// sorted by decreasing scalar part (src/hopf.zig:153-216).
std::vector<Quat> elements(int gid) {
  const Vec z{0, 0, 1}, x{1, 0, 0}, d{1, 1, 1};
  std::vector<Quat> gens;
  switch (gid) {
    case C2: gens = {turn(z, 2)}; break;
    case C3: gens = {turn(z, 3)}; break;
    case C4: gens = {turn(z, 4)}; break;
    case C6: gens = {turn(z, 6)}; break;
    case D2: gens = {turn(z, 2), turn(x, 2)}; break;
    case D3: gens = {turn(z, 3), turn(x, 2)}; break;
    case D4: gens = {turn(z, 4), turn(x, 2)}; break;
    case D6: gens = {turn(z, 6), turn(x, 2)}; break;
    case T: gens = {turn(z, 2), turn(x, 2), turn(d, 3)}; break;
    case O: gens = {turn(z, 4), turn(d, 3)}; break;
    default: gens = {turn(z, 5), turn(Vec{2, 0, 1}, 5)}; break;
  }
  std::vector<Quat> e{Quat{1, 0, 0, 0}};
  for (size_t i = 0; i < e.size(); ++i) {
    for (const Quat& g : gens) {
      const Quat p = qmul(e[i], g);
      bool known = false;
      for (const Quat& k : e)
        if (std::fabs(qdot(k, p)) > 1 - 1e-9) {
          known = true;
          break;
        }
      if (!known) e.push_back(p);
    }
  }
  if ((int)e.size() != kOrder[gid]) throw Failure("GroupClosure");
  for (Quat& q : e) {
    q = qnormalize(q);
    if (q[0] < 0) q = {-q[0], -q[1], -q[2], -q[3]};
  }
  std::stable_sort(e.begin(), e.end(), [](const Quat& a, const Quat& b) { return a[0] > b[0]; });
  return e;
}

// Rotations per full fibre, n (src/hopf.zig:48-55).
uint32_t fibre_count(int root, uint32_t f) {
  if (root == O) return f < 6 ? 4 * f : 4 * f - 12 * ((2 * f + 9) / 18);
  if (root == I) return 5 * f;
  return 6 * ((4 * f + 5) / 6);
}
// Nodes on ring j of the D6 grid (j = f is the equator).
uint32_t ring_size(uint32_t f, uint32_t j) {
  const uint32_t mult = j == f ? 12 : 6;
  const double x = 4.0 * f * std::sin(kPi * j / (2.0 * f));
  return std::max<uint32_t>(mult, mult * (uint32_t)std::floor(x / mult + 0.5));
}
uint32_t node_count(int root, uint32_t f) {
  if (root == O) return 4 * f * f + 2;
  if (root == I) return 10 * f * f + 2;
  uint32_t total = 2 + ring_size(f, f);
  for (uint32_t j = 1; j < f; ++j) total += 2 * ring_size(f, j);
  return total;
}

// Base polyhedra in the reference's vertex and face order (its unique-sorted vertices and
// Qhull simplices), so nodes and orbits come in the same order (src/hopf.zig:218-224).
constexpr uint8_t kOctaFaces[8][3] = {{5, 4, 3}, {5, 4, 0}, {2, 4, 3}, {2, 4, 0},
                                      {1, 5, 0}, {1, 5, 3}, {1, 2, 0}, {1, 2, 3}};
constexpr uint8_t kIcoFaces[20][3] = {{5, 3, 0},  {1, 3, 0},  {4, 5, 0},  {9, 5, 3},  {7, 1, 3},
                                      {7, 9, 11}, {7, 9, 3},  {10, 4, 5}, {10, 9, 5}, {10, 8, 11},
                                      {10, 9, 11}, {10, 8, 4}, {6, 7, 1},  {6, 7, 11}, {6, 8, 11},
                                      {2, 8, 4},  {2, 1, 0},  {2, 4, 0},  {2, 6, 1},  {2, 6, 8}};
// Icosahedron vertices off the poles: ring (z = +-1/sqrt 5, or 0 for the two pole slots)
// and azimuth in degrees.
constexpr double kIcoRing[12][2] = {{-1, 180}, {1, -144}, {1, 144}, {-1, -108}, {-1, 108}, {0, 0},
                                    {0, 0},    {1, -72},  {1, 72},  {-1, -36},  {-1, 36},  {1, 0}};

std::vector<Vec> polyhedron(bool ico) {
  if (!ico) return {Vec{1, 0, 0}, Vec{0, 1, 0}, Vec{0, 0, 1}, Vec{-1, 0, 0}, Vec{0, -1, 0}, Vec{0, 0, -1}};
  std::vector<Vec> v(12);
  const double r = 2 / std::sqrt(5.0);
  for (int k = 0; k < 12; ++k) {
    const double a = kIcoRing[k][1] * kPi / 180;
    v[k] = {r * std::cos(a), r * std::sin(a), kIcoRing[k][0] / std::sqrt(5.0)};
  }
  v[5] = {0, 0, -1};
  v[6] = {0, 0, 1};
  return v;
}

// One chamber of O_h or I_h: a spherical triangle with the pole z as a vertex, azimuths
// [lo, hi] and one far edge on the plane edge . x = 0, lying on one flat face of the
// polyhedron (normal). map() takes a point on the polyhedron's surface, moves it into the
// chamber, applies the area-preserving map there and moves it back (src/hopf.zig:232-354).
class Chamber {
 public:
  Chamber(bool ico, const std::vector<Vec>& v) {
    const Vec p = ico ? Vec{std::sin(0.2) * std::cos(0.1 * kPi), std::sin(0.2) * std::sin(0.1 * kPi), std::cos(0.2)}
                      : vunit(Vec{1, 2, 3});
    lo_ = ico ? 0 : kPi / 4;
    hi_ = ico ? kPi / 5 : kPi / 2;
    normal_ = ico ? vunit(Vec{v[6][0] + v[11][0] + v[8][0], v[6][1] + v[11][1] + v[8][1], v[6][2] + v[11][2] + v[8][2]})
                  : vunit(Vec{1, 1, 1});
    const std::vector<Quat> e = elements(ico ? I : O);
    const size_t ne = e.size();
    ops_.resize(2 * ne);
    for (size_t k = 0; k < ne; ++k) {
      Mat m = rotation_matrix(e[k]);
      // Exact symmetries: snap the near-integers that composition leaves (1 - 4e-16),
      // which would otherwise open slivers between the sector planes.
      for (Vec& row : m)
        for (double& x : row)
          if (std::fabs(x - std::round(x)) < 1e-10) x = std::round(x);
      Mat neg = m;
      for (Vec& row : neg)
        for (double& x : row) x = -x;
      ops_[k] = m;
      ops_[k + ne] = neg;
    }
    rotated_.resize(ops_.size());
    const double mid = 0.5 * (lo_ + hi_);
    double best = -1;
    for (size_t k = 0; k < ops_.size(); ++k) {
      const Vec mp = mul_transposed(ops_[k], p);
      rotated_[k] = mp;
      Vec h{p[0] - mp[0], p[1] - mp[1], p[2] - mp[2]};
      if (std::sqrt(vdot(h, h)) <= 1e-9) continue;
      h = vunit(h);
      if (std::fabs(h[2]) < 1e-12) continue;  // planes through the pole bound the azimuth
      const double psi = std::atan2(h[2], h[0] * std::cos(mid) + h[1] * std::sin(mid));
      if (psi > best) {
        best = psi;
        edge_ = h;
      }
    }
    source_lo_ = source(lo_);
    source_span_ = source(hi_) - source_lo_;
    target_lo_ = target(lo_);
    target_span_ = target(hi_) - target_lo_;
  }

  Vec map(const Vec& v) const {
    size_t best = 0;
    double score = vdot(v, rotated_[0]);
    for (size_t g = 1; g < ops_.size(); ++g) {
      const double s = vdot(v, rotated_[g]);
      if (s > score) {
        score = s;
        best = g;
      }
    }
    const Vec w = mul(ops_[best], v);
    const double phi = std::clamp(std::atan2(w[1], w[0]), lo_, hi_);
    const double theta = std::atan2(std::sqrt(w[0] * w[0] + w[1] * w[1]), w[2]);
    const double a = normal_[0] * std::cos(phi) + normal_[1] * std::sin(phi);
    const double t = std::tan(theta);
    const double tm = std::tan(theta_high(phi));
    // Radial fraction of the flat face's sector, kept as the fraction of the target's solid
    // angle at the mapped azimuth.
    const double ratio = (t / (normal_[2] + a * t)) / (tm / (normal_[2] + a * tm));
    const double new_phi = target_inverse(std::clamp((source(phi) - source_lo_) / source_span_, 0.0, 1.0));
    const double new_theta =
        2 * std::asin(std::sqrt(std::clamp(ratio * ratio, 0.0, 1.0)) * std::sin(0.5 * theta_high(new_phi)));
    const Vec out{std::sin(new_theta) * std::cos(new_phi), std::sin(new_theta) * std::sin(new_phi), std::cos(new_theta)};
    return vunit(mul_transposed(ops_[best], out));
  }

 private:
  // Polar extent of the chamber at azimuth phi.
  double theta_high(double phi) const {
    return kPi - std::atan2(edge_[2], edge_[0] * std::cos(phi) + edge_[1] * std::sin(phi));
  }
  // Flat-face area per unit azimuth is proportional to 1 / (P cos + Q sin)^2, whose
  // integral is this (up to a constant).
  double source(double phi) const {
    const double p = edge_[2] * normal_[0] - normal_[2] * edge_[0];
    const double q = edge_[2] * normal_[1] - normal_[2] * edge_[1];
    return (p * std::sin(phi) - q * std::cos(phi)) / (p * std::cos(phi) + q * std::sin(phi));
  }
  // Solid angle 1 - cos(theta_high) per unit azimuth, integrated.
  double target(double phi) const {
    return phi - std::asin(std::clamp(-edge_[0] * std::sin(phi) + edge_[1] * std::cos(phi), -1.0, 1.0));
  }
  // Azimuth at which the target's cumulative fraction is `fraction`: Newton steps kept
  // inside a shrinking bracket.
  double target_inverse(double fraction) const {
    double lo = lo_, hi = hi_;
    double x = lo + fraction * (hi - lo);
    for (int it = 0; it < 64; ++it) {
      const double residual = (target(x) - target_lo_) / target_span_ - fraction;
      if (residual < 0) lo = x;
      else hi = x;
      const double slope = (1 - std::cos(theta_high(x))) / target_span_;
      const double step = x - residual / slope;
      const double next = (step > lo && step < hi) ? step : 0.5 * (lo + hi);
      if (std::fabs(next - x) < 1e-15) return next;
      x = next;
    }
    return x;
  }

  std::vector<Mat> ops_;
  std::vector<Vec> rotated_;
  double lo_, hi_;
  Vec normal_, edge_{0, 0, 1};
  double source_lo_ = 0, source_span_ = 1, target_lo_ = 0, target_span_ = 1;
};

struct Base {
  std::vector<Vec> nodes;
  // Lattice row from the nearest polyhedron vertex (or ring index from the nearest pole):
  // odd layers take the staggered fibre angles.
  std::vector<uint32_t> layers;
};

// The area-mapped frequency-f nodes of every face, each shared node once, in first
// occurrence order over faces and barycentric rows (src/hopf.zig:368-417).
Base polyhedral_base(int root, uint32_t f) {
  const bool ico = root == I;
  const std::vector<Vec> v = polyhedron(ico);
  const Chamber chamber(ico, v);
  const size_t nfaces = ico ? 20 : 8;
  const uint32_t total = node_count(root, f);
  Base base;
  base.nodes.reserve(total);
  base.layers.reserve(total);
  std::vector<Vec> flat;
  flat.reserve(total);
  // A node is identified by its nonzero barycentric weights on polyhedron vertices.
  std::unordered_set<uint64_t> seen;
  seen.reserve(2 * (size_t)total);
  const double scale = 1 / (double)f;
  for (size_t fi = 0; fi < nfaces; ++fi) {
    const uint8_t* face = ico ? kIcoFaces[fi] : kOctaFaces[fi];
    for (uint32_t i = 0; i <= f; ++i) {
      for (uint32_t j = 0; j <= f - i; ++j) {
        const uint32_t weights[3] = {i, j, f - i - j};
        std::array<std::pair<uint32_t, uint32_t>, 3> pairs;
        int np = 0;
        for (int m = 0; m < 3; ++m)
          if (weights[m]) pairs[np++] = {face[m], weights[m]};
        std::sort(pairs.begin(), pairs.begin() + np);
        uint64_t key = 0;  // (vertex 4 bits, weight 10 bits) x up to 3, in vertex order
        for (int m = 0; m < 3; ++m) {
          const uint64_t part = m < np ? ((uint64_t)pairs[m].first << 10 | pairs[m].second) : 0x3fffu;
          key = key << 14 | part;
        }
        if (!seen.insert(key).second) continue;
        if (flat.size() == total) throw Failure("BaseMeshCount");
        Vec x{0, 0, 0};
        for (int m = 0; m < 3; ++m) {
          const double b = (double)weights[m] * scale;
          for (int e = 0; e < 3; ++e) x[e] += b * v[face[m]][e];
        }
        flat.push_back(vunit(x));
        base.layers.push_back(f - std::max(weights[0], std::max(weights[1], weights[2])));
      }
    }
  }
  if (flat.size() != total) throw Failure("BaseMeshCount");
  // The area-preserving map, node by node, on the host's threads.
  base.nodes.resize(total);
  const unsigned threads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const size_t per = (total + threads - 1) / threads;
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < threads; ++t) {
    const size_t a = t * per, b = std::min<size_t>(total, a + per);
    if (a >= b) break;
    pool.emplace_back([&, a, b] {
      for (size_t k = a; k < b; ++k) base.nodes[k] = chamber.map(flat[k]);
    });
  }
  for (std::thread& th : pool) th.join();
  return base;
}

// D6-invariant equal-area rings: both poles, 2f - 2 rings and the equator, each ring at
// the middle height of a band of area 4 pi / |V| per node; alternate rings staggered by
// half a step, the equator not (it holds every two-fold axis) (src/hopf.zig:419-456).
Base ring_base(uint32_t f) {
  const uint32_t total = node_count(D6, f);
  Base base;
  base.nodes.reserve(total);
  base.layers.reserve(total);
  base.nodes.push_back({0, 0, 1});
  base.nodes.push_back({0, 0, -1});
  base.layers = {0, 0};
  const double size = total;
  double top = 1 - 2 / size;
  for (uint32_t j = 1; j < f; ++j) {
    const uint32_t m = ring_size(f, j);
    const double width = 2 * (double)m / size;
    const double z = top - 0.5 * width;
    const double radius = std::sqrt(1 - z * z);
    for (const double height : {z, -z}) {
      for (uint32_t i = 0; i < m; ++i) {
        const double phi = 2 * kPi * ((double)i + 0.5 * (double)(j % 2)) / (double)m;
        base.nodes.push_back({radius * std::cos(phi), radius * std::sin(phi), height});
        base.layers.push_back(j);
      }
    }
    top -= width;
  }
  const uint32_t equator = ring_size(f, f);
  for (uint32_t i = 0; i < equator; ++i) {
    const double phi = 2 * kPi * (double)i / (double)equator;
    base.nodes.push_back({std::cos(phi), std::sin(phi), 0});
    base.layers.push_back(f);
  }
  if (base.nodes.size() != total) throw Failure("BaseMeshCount");
  return base;
}

// Nodes are found again by their coordinates rounded to 1e-7.
struct Cell {
  int32_t k[3];
  bool operator==(const Cell& o) const { return k[0] == o.k[0] && k[1] == o.k[1] && k[2] == o.k[2]; }
};
struct CellHash {
  size_t operator()(const Cell& c) const {
    uint64_t h = (uint32_t)c.k[0];
    h = h * 0x9e3779b97f4a7c15ull ^ (uint32_t)c.k[1];
    h = h * 0x9e3779b97f4a7c15ull ^ (uint32_t)c.k[2];
    return (size_t)(h ^ (h >> 29));
  }
};
Cell cell_of(const Vec& v, int dx = 0, int dy = 0, int dz = 0) {
  return Cell{{(int32_t)std::round(v[0] * 1e7) + dx, (int32_t)std::round(v[1] * 1e7) + dy,
               (int32_t)std::round(v[2] * 1e7) + dz}};
}

// A rotation taking the unit vector v to z; a fixed half turn about x at v = -z.
Quat section(const Vec& v) {
  const Quat q{1 + v[2], v[1], -v[0], 0};
  if (std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) < 1e-12) return {0, 1, 0, 0};
  return qnormalize(q);
}

// The sector at z that holds each orbit's chosen node: the cell of the vertex z among the
// root polyhedron's vertices (for D6, the northern hemisphere), azimuths 0 .. 2 pi / m.
struct Sector {
  std::vector<Vec> poles;
  double wedge;
  explicit Sector(int root) {
    if (root == O) {
      poles = polyhedron(false);
      wedge = 2 * kPi / 4;
    } else if (root == I) {
      poles = polyhedron(true);
      wedge = 2 * kPi / 5;
    } else {
      poles = {Vec{0, 0, 1}, Vec{0, 0, -1}};
      wedge = 2 * kPi / 6;
    }
  }
  bool contains(const Vec& w) const {
    for (const Vec& p : poles)
      if (vdot(w, p) > w[2] + 1e-11) return false;
    if (std::sqrt(w[0] * w[0] + w[1] * w[1]) < 1e-11) return true;
    const double az = std::atan2(w[1], w[0]);
    return az >= -1e-11 && az <= wedge + 1e-11;
  }
};
// On the sector's edges the orbit keeps the node with the largest x, then y (to 1e-11).
bool preferred(const Vec& a, const Vec& b) {
  const double ax = std::round(a[0] * 1e11), bx = std::round(b[0] * 1e11);
  if (ax != bx) return ax > bx;
  return std::round(a[1] * 1e11) > std::round(b[1] * 1e11);
}

}  // namespace

int root_of(int gid) { return root_group(gid); }

uint64_t raw_count(int gid, uint32_t f) {
  const int root = root_group(gid);
  return (uint64_t)fibre_count(root, f) * node_count(root, f) / (uint64_t)kOrder[gid];
}

uint32_t count(int gid, uint32_t f) {
  if (f < 1 || f > kMaxFrequency) throw Failure("InvalidGridResolution");
  const uint64_t n = raw_count(gid, f);
  if (n > kMaxCount) throw Failure("GridTooLarge");
  return (uint32_t)n;
}

uint32_t nearest_frequency(int gid, uint32_t target) {
  uint32_t best = 1;
  double score = INFINITY;
  for (uint32_t f = 1; f <= kMaxFrequency; ++f) {
    const uint64_t n = raw_count(gid, f);
    if (n > kMaxCount) continue;
    const double s = std::fabs(std::log((double)n / (double)std::max<uint32_t>(target, 1)));
    if (s < score) {
      score = s;
      best = f;
    }
  }
  return best;
}

std::optional<uint32_t> largest_frequency(int gid, uint32_t budget) {
  std::optional<uint32_t> best;
  uint64_t most = 0;
  for (uint32_t f = 1; f <= kMaxFrequency; ++f) {
    const uint64_t n = raw_count(gid, f);
    if (n <= budget && n > most) {
      most = n;
      best = f;
    }
  }
  return best;
}

const char* generator_name(int gid) {
  switch (root_group(gid)) {
    case I: return "Inverse Hopf product grid (icosahedral root)";
    case O: return "Inverse Hopf product grid (octahedral root)";
    default: return "Inverse Hopf product grid (hexagonal root)";
  }
}

std::vector<float> points(int gid, uint32_t f) {
  const uint32_t total = count(gid, f);
  const int root = root_group(gid);
  const Base base = root == D6 ? ring_base(f) : polyhedral_base(root, f);
  const std::vector<Vec>& nodes = base.nodes;
  const std::vector<Quat> parent = elements(root);
  std::vector<Mat> mats;
  for (const Quat& q : parent) mats.push_back(rotation_matrix(q));
  const std::vector<Quat> own = elements(gid);

  // Cosets c H' of H' = R H R^-1 in the root, each represented by its first element in the
  // root's order; one point q c R per H-orbit.
  const Quat r = embedding(gid);
  const Quat r_inverse{r[0], -r[1], -r[2], -r[3]};
  std::vector<Quat> cosets;
  std::vector<bool> covered(parent.size(), false);
  for (size_t i = 0; i < parent.size(); ++i) {
    if (covered[i]) continue;
    cosets.push_back(parent[i]);
    for (const Quat& h : own) {
      const Quat member = qmul(parent[i], qmul(qmul(r, h), r_inverse));
      for (size_t k = 0; k < parent.size(); ++k)
        if (std::fabs(qdot(parent[k], member)) > 1 - 1e-9) covered[k] = true;
    }
  }
  if (cosets.size() * own.size() != parent.size()) throw Failure("GroupNotInRoot");
  std::vector<Quat> tails;
  for (const Quat& c : cosets) tails.push_back(qmul(c, r));

  std::unordered_map<Cell, uint32_t, CellHash> index;
  index.reserve(2 * nodes.size());
  for (uint32_t i = 0; i < nodes.size(); ++i) index[cell_of(nodes[i])] = i;
  auto find = [&](const Vec& image) -> uint32_t {
    auto it = index.find(cell_of(image));
    if (it != index.end()) return it->second;
    for (int o = 0; o < 27; ++o) {  // a rounding boundary between the image and its node
      it = index.find(cell_of(image, o % 3 - 1, o / 3 % 3 - 1, o / 9 - 1));
      if (it != index.end()) return it->second;
    }
    throw Failure("BaseMeshNotInvariant");
  };

  const uint32_t n = fibre_count(root, f);
  // Fibre rotations R_z(t) of both phases; odd layers are half a step on.
  std::vector<Quat> spins(2 * (size_t)n);
  for (uint32_t phase = 0; phase < 2; ++phase)
    for (uint32_t j = 0; j < n; ++j) {
      const double t = (2 * kPi * (double)j + kPi * (double)phase) / (double)n;
      spins[phase * n + j] = {std::cos(0.5 * t), 0, 0, std::sin(0.5 * t)};
    }
  const Sector sector(root);
  std::vector<bool> seen(nodes.size(), false);
  std::vector<float> out((size_t)total * 4);
  size_t at = 0;
  std::vector<Quat> heads(tails.size());
  for (uint32_t i = 0; i < nodes.size(); ++i) {
    if (seen[i]) continue;
    // Mark the orbit; the stabiliser order is the number of images landing on node i.
    uint32_t stabiliser = 0;
    std::optional<Vec> chosen;
    for (const Mat& m : mats) {
      const Vec image = mul_transposed(m, nodes[i]);
      const uint32_t j = find(image);
      const Vec d{nodes[j][0] - image[0], nodes[j][1] - image[1], nodes[j][2] - image[2]};
      if (vdot(d, d) > 1e-18) throw Failure("BaseMeshNotInvariant");
      seen[j] = true;
      if (j == i) ++stabiliser;
      if (sector.contains(image) && (!chosen || preferred(image, *chosen))) chosen = image;
    }
    if (n % stabiliser != 0) throw Failure("FibreNotDivisible");
    if (!chosen) throw Failure("OrbitOutsideSector");
    const Quat s = section(*chosen);
    for (size_t k = 0; k < tails.size(); ++k) heads[k] = qmul(s, tails[k]);
    const Quat* row = &spins[(size_t)(base.layers[i] % 2) * n];
    const uint32_t len = n / stabiliser;
    if (at + (size_t)len * heads.size() > total) throw Failure("ProductCount");
    for (uint32_t j = 0; j < len; ++j)
      for (const Quat& h : heads) {
        const Quat q = qmul(row[j], h);
        for (int c = 0; c < 4; ++c) out[at * 4 + c] = (float)q[c];
        ++at;
      }
  }
  if (at != total) throw Failure("ProductCount");
  return out;
}

}  // namespace zo::hopf
