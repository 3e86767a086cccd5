// Host copies of the group tables and the zone bisector planes.
#include <algorithm>
#include <array>
#include <cmath>
#include <numeric>
#include <vector>

#include "kernels.h"

namespace zo {

namespace {
#include "groups_table.inc"

// Zone bisector half-spaces between the identity and +-g_k (src/covering.zig:382-396):
// normal (1 - s g0, -s g1, -s g2, -s g3) normalised in FP64, for every operator and sign
// s = +1, -1 except (identity, +1); in that order.
template <class Out>
void planes_of(const double (*ops)[4], int order, Out out) {
  int row = 0;
  for (int k = 0; k < order; ++k) {
    for (int t = 0; t < 2; ++t) {
      const double s = t == 0 ? 1.0 : -1.0;
      if (k == 0 && t == 0) continue;
      double v[4] = {1.0 - s * ops[k][0], -s * ops[k][1], -s * ops[k][2], -s * ops[k][3]};
      const double len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
      for (int c = 0; c < 4; ++c) v[c] /= len;
      out(row++, v);
    }
  }
}

// Reach of each plane over the zone {x unit: h_k . x >= 0 for all k}. When the planes span
// R^4 the zone is the spherical hull of its vertices (the unit points where three planes
// meet and every half-space holds), and for any zone point x = sum l_i v_i / |sum l_i v_i|
// (l_i >= 0) and a plane whose dot products with all vertices are >= 0,
// h . x >= sum l_i (h . v_i) / sum l_i >= min_i h . v_i, by the triangle inequality. So
// min over the vertices bounds the plane's dot product below over the whole zone; the 1e-5
// taken off covers float32 planes and sources that the fold leaves within rounding of the
// zone.
void plane_reach(const double (*h)[4], int planes, float* reach) {
  std::vector<std::array<double, 4>> vertices;
  for (int a = 0; a < planes; ++a)
    for (int b = a + 1; b < planes; ++b)
      for (int c = b + 1; c < planes; ++c) {
        // The line orthogonal to three normals: cofactors of the 3x4 matrix.
        const double* r[3] = {h[a], h[b], h[c]};
        auto minor = [&](int skip) {
          int col[3], n = 0;
          for (int i = 0; i < 4; ++i)
            if (i != skip) col[n++] = i;
          return r[0][col[0]] * (r[1][col[1]] * r[2][col[2]] - r[1][col[2]] * r[2][col[1]]) -
                 r[0][col[1]] * (r[1][col[0]] * r[2][col[2]] - r[1][col[2]] * r[2][col[0]]) +
                 r[0][col[2]] * (r[1][col[0]] * r[2][col[1]] - r[1][col[1]] * r[2][col[0]]);
        };
        std::array<double, 4> v = {minor(0), -minor(1), minor(2), -minor(3)};
        const double len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
        if (len < 1e-9) continue;
        for (double sign : {1.0, -1.0}) {
          std::array<double, 4> u;
          for (int i = 0; i < 4; ++i) u[i] = sign * v[i] / len;
          bool inside = true;
          for (int k = 0; k < planes && inside; ++k)
            inside = h[k][0] * u[0] + h[k][1] * u[1] + h[k][2] * u[2] + h[k][3] * u[3] >= -1e-9;
          if (inside) vertices.push_back(u);
        }
      }
  for (int k = 0; k < planes; ++k) {
    double least = vertices.empty() ? -1.0 : 2.0;
    for (const auto& u : vertices)
      least = std::min(least, h[k][0] * u[0] + h[k][1] * u[1] + h[k][2] * u[2] + h[k][3] * u[3]);
    reach[k] = least <= 1e-9 ? -1.0f : (float)(least - 1e-5);
  }
}

HostTables build() {
  HostTables t{};
  int plane = 0;
  for (int g = 0; g < 11; ++g) {
    t.group_offset[g] = kGroupOffset[g];
    t.group_order[g] = kGroupOrder[g];
    t.plane_offset[g] = plane;
    const int off = kGroupOffset[g], order = kGroupOrder[g];
    double f32ops[64][4];
    for (int k = 0; k < order; ++k)
      for (int c = 0; c < 4; ++c) {
        t.ops64[off + k][c] = kOps64[off + k][c];
        t.ops32[off + k][c] = kOps32[off + k][c];
        f32ops[k][c] = (double)kOps32[off + k][c];
      }
    planes_of(&kOps64[off], order, [&](int r, const double* v) {
      for (int c = 0; c < 4; ++c) t.planes64[plane + r][c] = v[c];
    });
    planes_of(f32ops, order, [&](int r, const double* v) {
      for (int c = 0; c < 4; ++c) t.planes32[plane + r][c] = (float)v[c];
    });
    const int planes = 2 * order - 1;
    float reach[kMaxPlaneRows];
    plane_reach(&t.planes64[plane], planes, reach);
    std::vector<int> sorted(planes);
    std::iota(sorted.begin(), sorted.end(), 0);
    std::stable_sort(sorted.begin(), sorted.end(), [&](int x, int y) { return reach[x] < reach[y]; });
    for (int r = 0; r < planes; ++r) {
      t.plane_order[plane + r] = (uint8_t)sorted[r];
      t.plane_reach[plane + r] = reach[sorted[r]];
    }
    plane += planes;
  }
  return t;
}
}  // namespace

const HostTables& host_tables() {
  static const HostTables tables = build();
  return tables;
}
int host_group_offset(int gid) { return kGroupOffset[gid]; }
int host_group_order(int gid) { return kGroupOrder[gid]; }
const char* host_group_name(int gid) { return kGroupName[gid]; }
const float* host_ops32(int gid) { return kOps32[kGroupOffset[gid]]; }

}  // namespace zo
