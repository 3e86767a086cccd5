// Types and limits shared by the host engine and the CUDA kernels.
#pragma once
#include <stdint.h>

namespace zo {

constexpr int kMaxOperatorRows = 141;   // sum of |K| over the eleven groups
constexpr int kMaxGroupOrder = 60;      // |K| of the largest group (I)
constexpr int kMaxPlaneRows = 271;      // sum of 2|K|-1 zone bisector planes
constexpr uint32_t kIdentityBit = 0x80000000u;  // site code: the source's identity image
// Largest chart grid side. The reference clamps it at 128 (src/near.zig:135); at ten million
// sources that holds about six sites per cell, so the cap here is 256, which keeps the target
// sites per cell up to about 33 million shell sites.
constexpr int kMaxCellDim = 256;
// Sources are ordered along a Hilbert curve over a 64^3 grid of the chart box (the
// reference sorts them into a 32^3 Morton grid, src/near.zig:23).
constexpr int kOrderBits = 6;
constexpr int kOrderDim = 1 << kOrderBits;
// Default tile shape of the FP32 near-field gather (the tile table can pick others per group
// and size): target shell sites per chart cell (the reference uses 8, src/near.zig:135) and
// sources per warp (each source's sites split over 32 / kNearGroup lanes; small groups keep
// the union of the sources' neighbourhoods close to each one's).
constexpr double kSitesPerCell = 2.0;
constexpr int kNearGroup = 4;
// The spacing pass's first walk covers this fraction of its cutoff (the 4 mean radii) unless
// the tile table names another: 2.5 of the 4 radii, about a quarter of the cutoff ball's
// volume, so nearly every source's nearest lies within it; the few whose nearest may not
// are searched again over the whole cutoff in FP64.
constexpr double kSpacingWalk = 2.5 / 4.0;

// Precision of one sample's arithmetic.
//  kFP32: FP32 pair arithmetic (approximate SFU reciprocals, own atan), FP64 row sums,
//         BB inner products, move, renormalisation and fold; float32 state.
//  kFP64: FP64 everywhere (IEEE division/sqrt/atan), FP64 master state.
enum Precision : int { kFP32 = 0, kFP64 = 1 };

// Per-source rows, structure of arrays (the reference's 48-byte Row, src/pairs.zig:11-15).
struct Rows {
  double4* force;     // xyz: left-tangent force, w: curvature
  double* energy;     // Quey energy (own orbit excluded)
  double* nearest;    // smallest squared chord to another orbit point
  int* nearest_at;    // where it is: image index k*n+j (all pairs) or sorted site (near)
};

// Device-resident chart grid of one near pass, derived on the device from the shell.
struct NearGrid {
  float lower[3];
  float cells_per_unit;     // sdim / width
  float order_per_unit;     // kOrderDim / width
  float width;
  int sdim;
  int sites;                // shell sites written (clamped to capacity)
  unsigned int box_bits[6]; // ordered-bits min xyz, max xyz of site positions (next pass)
  unsigned int overflow;    // a pass produced more sites than capacity
  unsigned int pad;
};

// Device-resident BB step state (shaders/relax.wgsl:18-23), FP64 sums.
struct RelaxDev {
  int iteration;
  unsigned int flags;               // 1 non-finite force, 2 duplicate orientation
  unsigned long long step_bits;     // largest move (double bits, non-negative)
  double sums[5];                   // s.y, y.y, s.s, f.f, energy
  unsigned long long prefix[2];     // radix select: digit prefixes of the two middle ranks
  unsigned long long rank[2];       // remaining ranks within the prefix
  double median;
  double alpha;
  unsigned int ticket;              // last-block-done counter
  unsigned int pad;
};

// Result of a row summary reduction (quick measures, src/pairs.zig:130-140).
struct RowSummary {
  double energy;     // sum of row energies
  double force2;     // sum of |force|^2
  double nearest;    // min nearest chord^2
  int nearest_row;   // its source
  float least_degrees;  // the smallest per-source nearest angle, degrees, rounded as the point values are
  unsigned int ticket;
};

}  // namespace zo
