// Host copies of the group tables and the zone bisector planes.
#include <cmath>

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
    plane += 2 * order - 1;
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
