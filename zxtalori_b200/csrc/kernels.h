// Host-callable launchers of the CUDA kernels (kernels.cu). Plain pointers only.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "qvm_shared.h"

namespace zo {

struct HostTables {
  double ops64[kMaxOperatorRows][4];
  float ops32[kMaxOperatorRows][4];
  double planes64[kMaxPlaneRows][4];
  float planes32[kMaxPlaneRows][4];
  // Each group's planes sorted by their reach, the least dot product of the plane's normal
  // with any point of the zone (from the zone's vertices), less 1e-5; -1 for groups whose
  // zone has no vertices (cyclic groups) and for planes that touch the zone. plane_order holds
  // the group-local plane index of each sorted row, plane_reach its reach.
  uint8_t plane_order[kMaxPlaneRows];
  float plane_reach[kMaxPlaneRows];
  int group_offset[11];
  int group_order[11];
  int plane_offset[11];
};
const HostTables& host_tables();
int host_group_offset(int gid);
int host_group_order(int gid);

// Copies the group tables into the current device's constant memory.
cudaError_t upload_tables(const HostTables& t);
// upload_tables once per device (device current; the first caller uploads, under a lock),
// for engines and the allocation-free entry point alike.
constexpr int kMaxTableDevices = 64;
cudaError_t ensure_device_tables(int device);

cudaError_t launch_haar(float4* q, int n, uint32_t seed, cudaStream_t s);
cudaError_t launch_fold(float4* q32, double4* q64, int n, int gid, int prec, bool from_q32, cudaStream_t s);
cudaError_t launch_scan(const uint32_t* in, uint32_t* out, int max_count, const int* count_dev, uint32_t* block_sums,
                        cudaStream_t s);

// All-pairs work split: 128 sources per block, `chunks` ranges of image tiles per source block.
struct PairsPlan {
  int jtiles = 0, total_tiles = 0, tiles_per_chunk = 0, chunks = 1;
};
PairsPlan plan_pairs(int n, int order, double budget_scale, int sms);

// Force-pass rows over all pairs; `partial` holds chunks*n rows when chunks > 1.
cudaError_t launch_pairs(int prec, bool track, const float4* q32, const double4* q64, int n, int gid, const PairsPlan& pl,
                         Rows partial, Rows out, cudaStream_t s);
// Full measure rows: `extra` 5 doubles per source (riesz1, riesz2, riesz3, green, log).
cudaError_t launch_full(int prec, const float4* q32, const double4* q64, int n, int gid, const PairsPlan& pl,
                        Rows partial, double* pextra, int* pdegen, Rows out, double* extra, int* degen, cudaStream_t s);

// Cutoff of a near-field pass (pairs.wgsl:352-361): squared chord and chord of r, the
// window's start taper r and inverse width 1/((1 - taper) r).
struct NearCut {
  double cut2, chord, cut_z, cut_w;
  // Squared chord at angle 1.25 r, where the window is exactly zero: the packed gather
  // evaluates an out-of-cutoff site with its chord clamped to this (finite terms, zero
  // contribution) when the other site of its pair is within the cutoff.
  double cut_hi;
  // Squared chord of the ball the FP32 gather walks: the cutoff's, except in the spacing
  // pass, whose first walk takes a smaller ball (sources it cannot settle are searched
  // again over the whole cutoff).
  double walk2;
};

// The arguments of one FP32 gather: one sample's sources, sorted sites and chart grid.
struct NearArgs {
  const float4* q;
  int n;
  const uint32_t* src_perm;
  const float4* sq;
  const uint32_t* scode;
  const uint32_t* cell_off;
  const float* site_x;
  const NearGrid* gp;
  NearCut cut;
  int slices;
  Rows out;
  int stride;
  int direct;  // one slice: rows written in place by source (else partial rows by slice)
  uint32_t* exact_list;   // spacing pass: the sources left to the exact search
  uint32_t* exact_count;
  // A diagnostic force pass only (else null): adds the candidate sites evaluated and the
  // pairs inside the cutoff that exert a force.
  unsigned long long* pair_counts;
};

// One sample's FP32 gather as a task of a shared launch: its arguments, tile shape (sources
// per warp), pair form (chord form for cutoffs up to 0.4 rad), warps and slices.
struct NearTask {
  NearArgs a;
  int group_size, short_atan, warps, slices;
};

// One near-field pass; every pointer is device memory sized by the host (Near workspace).
struct NearLaunch {
  int prec, gid, n, capacity, sdim_max, slices;
  int slices32;  // slices of the FP32 gather (group_size sources per warp); <= slices
  int group_size;  // FP32 gather tile shape: sources per warp (2, 4 or 8)
  double sites_per_cell;  // target shell sites per chart cell (sets the grid's side)
  bool track;
  bool short_atan;  // cutoff r <= 0.4 rad: the short-range arctangent applies
  bool nearest_only;  // FP32 gather: nearest chord and site only (forces, curvature, energy left 0)
  double s_margin, cut2, chord, cut_z, cut_w;
  // Spacing pass (nearest_only): squared chord of the first walk's ball (at most cut2), and
  // the sources it leaves to the exact FP64 search: their list (n entries) and two counters
  // (listed sources, sources with an exact tie).
  double walk_cut2;
  uint32_t* exact_list;
  uint32_t* exact_count;
  unsigned long long* pair_counts;  // diagnostic force pass: candidates and in-cutoff pairs (else null)
  const float4* q32;
  const double4* q64;
  uint32_t *counts, *offsets, *scan_tmp;
  uint4* shell_mask;  // per source: which images are sites (bit 2 operator + sign)
  uint32_t* rim_list;  // FP32 shell: rim sources, their normalised positions, their count
  float4* rim_q;
  uint32_t* rim_count;
  float4* site_q32;
  double4* site_q64;
  uint4* site_meta;  // per unsorted site: code, image number, chart x (bits), 0
  uint32_t *site_cell, *site_rank;
  float4* site_pos;
  uint32_t *cell_count, *cell_off, *perm;
  float4* sq32;
  double4* sq64;
  uint32_t *scode, *simg;
  float* sx;  // chart x of each sorted site (sites are sorted by x within each cell)
  uint32_t *src_key, *src_rank, *mcount, *moff, *src_perm;
  NearGrid* grid;
  int* cells;
  Rows partial;  // slices * n rows
  Rows out;
};
cudaError_t launch_near(const NearLaunch& L, cudaStream_t s);
// The same pass in parts, for many samples sharing one gather launch: the structure (shell,
// chart grid, site sort, source order), the FP32 gather as a task (near_task), and the
// slices' reduction into the rows.
cudaError_t launch_near_structure(const NearLaunch& L, cudaStream_t s, int* launches);
NearTask near_task(const NearLaunch& L);
cudaError_t launch_near_reduce(const NearLaunch& L, cudaStream_t s);
// The FP32 gathers of many samples of one tile variant (near_variant; device arrays: `count`
// tasks, prefix[k] the first warp task of sample k, `total` warp tasks) in one persistent
// launch; `counter` is a device word.
int near_variant(const NearTask& t);
constexpr int kNearVariants = 6;
cudaError_t launch_near32_batch(const NearTask* tasks, const uint32_t* prefix, int count, uint32_t total,
                                uint32_t* counter, int variant, int sms, cudaStream_t s);
// The near field for wide cutoffs, summed over every image (all-pairs tiles, near-field
// cutoff and window); `partial` holds chunks*n rows when chunks > 1.
cudaError_t launch_dense_near(int prec, bool track, bool short_atan, const float4* q32, const double4* q64, int n,
                              int gid, const PairsPlan& pl, double cut2, double chord, double cut_z, double cut_w,
                              Rows partial, Rows out, cudaStream_t s);
cudaError_t launch_shell_count(int prec, const float4* q32, const double4* q64, int n, int gid, double s_margin,
                               uint32_t* counts, uint32_t* offsets, uint32_t* scan_tmp, uint4* masks,
                               uint32_t* rim_list, float4* rim_q, uint32_t* rim_count, cudaStream_t s);

// Covering pass (k_cover.cuh): each listed source's star in the spherical Delaunay
// triangulation of the orbit, gift-wrapped in FP64 over the orbit points within a reach.
enum CoverStatus : uint32_t {
  kCoverOk = 0,        // the star is exact (every cap within the reach)
  kCoverShort = 1,     // some cap reaches past the reach: run again with need2
  kCoverCrowded = 2,   // more points than a star holds even after shrinking the reach
  kCoverStarFull = 3,  // more facets than a star holds
  kCoverSparse = 4,    // too few points to close a star: run again with need2 (wider)
};
struct CoverArgs {
  const float4* q;  // the float32 sample
  int n, gid;
  // Grid collection: the near-field structure's sorted sites and chart grid, complete to
  // the squared chord grid_reach2; grid == null: every image (dense).
  const uint32_t* scode;
  const uint32_t* simg;
  const uint32_t* cell_off;
  const NearGrid* grid;
  double grid_reach2;
  double reach2;            // squared chord of the reach, or per source:
  const double* reach2_of;  // (null: reach2 for all)
  const uint32_t* list;     // the sources to build (null: 0 .. n-1)
  int count;                // listed sources
  double* alpha;            // per source: largest cap of its star (S3 angle, rad)
  double4* centre;          // that cap's centre
  uint32_t* faces;          // distinct neighbours its star touches
  uint32_t* facets;         // facets of its star
  uint32_t* status;         // CoverStatus
  double* need2;            // squared chord of the reach a second run needs (else 0)
  unsigned long long* probes;  // pivots evaluated (added to; may be null)
  // Export of the stars (null: none): source i writes its facets as (x, y_a, y_b, y_c) point
  // keys ((source << 8) | image) into mesh[mesh_offset[i] .. mesh_offset[i + 1]).
  uint4* mesh;
  const uint32_t* mesh_offset;
  double4* mesh_normal;  // with mesh (may be null): each facet's unit normal, its cap's centre
};
// width: the star's capacity. 0 narrow (64 neighbours, 128 facets: the first pass), 1
// middle (128, 256: the first rerun), 2 wide (256, 256). A narrower star keeps more warps
// resident; a source it cannot hold comes back short at its reach for the next width.
cudaError_t launch_cover(const CoverArgs& A, int sms, cudaStream_t s, int width);

// Relaxation step pieces.
cudaError_t launch_relax_stats(Rows rows, const double4* prev_f, const double4* prev_d, int n, int fixed,
                               double* partials, RelaxDev* st, cudaStream_t s);
cudaError_t launch_median(int prec, Rows rows, int n, RelaxDev* st, unsigned int* hist, double alpha0, double radius,
                          int sms, cudaStream_t s);
cudaError_t launch_move_fold(float4* q32, double4* q64, int n, int gid, int prec, Rows rows, double4* prev_f,
                             double4* prev_d, RelaxDev* st, int fixed, double radius, double step_scale, cudaStream_t s);
cudaError_t launch_row_summary(Rows rows, int n, double* partials, double* near_partials, int* near_rows,
                               RowSummary* out, cudaStream_t s, bool nearest_only = false);
cudaError_t launch_nearest_degrees(const double* nearest, int n, float* out, cudaStream_t s);
cudaError_t launch_refine_nearest(const float4* q32, int n, int gid, Rows rows, bool near_sites, const uint32_t* scode,
                                  const uint32_t* simg, int* neighbour, cudaStream_t s);
cudaError_t launch_neighbour_index(Rows rows, int n, bool near_sites, const uint32_t* scode, int* neighbour,
                                   cudaStream_t s);

// Measured FP32 FMA throughput of the current device (TFLOP/s, 2 flops per FMA).
cudaError_t measure_fp32_peak(int sms, double* tflops, double* packed_tflops);

// Blocks used by the row-summary and stats reductions for n rows.
inline int reduce_blocks(int n) { return (n + 255) / 256; }

// Measurement hook: while set (on the launching thread), launchers count their kernel
// launches and bracket the pass's dominant kernel (the all-pairs or near-field row kernel)
// with the next pair of events from `events`.
struct LaunchProbe {
  long long launches = 0;
  cudaEvent_t* events = nullptr;
  int capacity = 0;  // events available (pairs * 2)
  int used = 0;
};
extern thread_local LaunchProbe* t_probe;
inline void probe_count(int k = 1) {
  if (t_probe) t_probe->launches += k;
}
inline void probe_mark(cudaStream_t s) {
  if (t_probe && t_probe->events && t_probe->used < t_probe->capacity) cudaEventRecord(t_probe->events[t_probe->used++], s);
}

}  // namespace zo
