// The engine behind the zo_* C ABI: one orientation sample resident on one GPU, with the
// reference's relaxation, measure and spacing policies (src/engine.zig:17-1021,
// src/pairs.zig:217-413, src/near.zig:31-196).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <limits>
#include <memory>
#include <optional>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.h"

namespace zo {

const char* host_group_name(int gid);
const float* host_ops32(int gid);

// An error carrying the reference's error name (src/exports.zig prefixes it).
struct Failure : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void check_cuda(cudaError_t e, const char* what);
#define ZO_CUDA(expr) ::zo::check_cuda((expr), #expr)

// Memory that outlives engines. Device buffers come from a per-device stream-ordered pool
// (cudaMallocFromPoolAsync / cudaFreeAsync) that keeps freed blocks for the next engine:
// creating and dropping samples costs no cudaMalloc/cudaFree, whose device-wide
// synchronisation also stalls every other engine. Each block is allocated and freed on the
// stream of the engine call that asked for it (AllocScope, set around every ABI call), so
// it is reused only after the work queued on that stream before the free.
cudaStream_t alloc_stream();
void* device_pool_alloc(size_t bytes, cudaStream_t s);
class AllocScope {
 public:
  explicit AllocScope(cudaStream_t s);
  ~AllocScope();
  AllocScope(const AllocScope&) = delete;
  AllocScope& operator=(const AllocScope&) = delete;

 private:
  cudaStream_t prev_;
};
// Pinned host blocks, cached across engines by size (up to a bound; beyond it they are freed).
void* pinned_alloc(size_t bytes);
void pinned_free(void* p);

// Host array in pinned memory (from the cache above) that only grows: device-to-host copies
// into it run at full PCIe/C2C speed instead of through the driver's pageable staging.
template <class T>
class PinnedArray {
 public:
  PinnedArray() = default;
  PinnedArray(const PinnedArray&) = delete;
  PinnedArray& operator=(const PinnedArray&) = delete;
  ~PinnedArray() { pinned_free(p_); }
  void resize(size_t n) {
    if (n > cap_) {
      pinned_free(p_);
      p_ = nullptr;
      cap_ = 0;
      p_ = static_cast<T*>(pinned_alloc(n * sizeof(T)));
      cap_ = n;
    }
    n_ = n;
  }
  T* data() { return p_; }
  const T* data() const { return p_; }
  size_t size() const { return n_; }
  void swap(PinnedArray& o) noexcept {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    std::swap(cap_, o.cap_);
  }

 private:
  T* p_ = nullptr;
  size_t n_ = 0, cap_ = 0;
};

// Device allocation that only grows; contents are not preserved across growth. Outside an
// AllocScope it falls back to cudaMalloc/cudaFree.
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() { release(); }
  void* ensure(size_t bytes);
  void release();
  template <class T>
  T* as() const { return static_cast<T*>(ptr_); }
  size_t bytes() const { return bytes_; }
  void swap(DeviceBuffer& o) noexcept {
    std::swap(ptr_, o.ptr_);
    std::swap(bytes_, o.bytes_);
    std::swap(stream_, o.stream_);
  }

 private:
  void* ptr_ = nullptr;
  size_t bytes_ = 0;
  cudaStream_t stream_ = nullptr;  // the stream it was allocated on; null: cudaMalloc
};

struct Measures {
  double count_extended = 0;
  double riesz_1 = NAN, riesz_2 = NAN, riesz_3 = NAN, green_ratio = NAN, log_ratio = NAN;
  double quey_energy = NAN, separation_deg = NAN, force_rms = NAN;
};

// A covering pass's result (the reference's covering.Result, src/covering.zig).
struct CoverResult {
  double radius_deg = NAN;         // largest empty cap of the orbit, SO(3) degrees
  double witness[4] = {1, 0, 0, 0};  // its centre (a unit quaternion of the orbit's image space)
  double domain_bound_deg = NAN;   // every empty cap is at most this: the widest reach a star was proven in
  uint32_t unresolved = 0;         // sources whose star could not be proven exact
  uint64_t facets = 0;             // star facets over all sources
  uint64_t probes = 0;             // pivots evaluated
  uint32_t rounds = 0;             // collection rounds (sources with a short reach run again)
  uint32_t shell_points = 0;       // shell sites of the chart grid the stars were collected from (0: every image)
  // After the first pass: sources short of reach, sources without a closed star; sources
  // built again from the chart grid and from every image (over all later rounds).
  uint32_t first_short = 0, first_sparse = 0, rerun_grid = 0, rerun_dense = 0;
};

// Plateau kicks of the covering optimiser (src/engine.zig:407-413 setKicks).
struct KickSettings {
  uint32_t patience = 150;
  double progress = 5e-4, size = 0.04, trust = 0.03;
};
// A covering-optimiser run: the best and current samples (host rows), their radii, the trust
// angle of a move (S3 radians) and the counts the stats report.
struct CoverOptimizer {
  bool active = false;
  uint64_t key = 0;  // the sample the last batch ended on
  std::vector<float> best, current;
  double best_radius = NAN, current_radius = NAN, gain_ref = NAN, trust = 0, separation = 0;
  uint32_t steps = 0, kicks = 0, jobs = 0, improved = 0, skipped = 0, full_steps = 0, since_gain = 0;
  std::mt19937_64 rng;
};

struct StepResult {
  double max_step_deg = 0, force_rms = 0, energy = 0;
};

// Rows of n sources in one set of device buffers.
struct RowBuffers {
  DeviceBuffer force, energy, nearest, nearest_at;
  Rows ensure(size_t n);
  size_t bytes() const { return force.bytes() + energy.bytes() + nearest.bytes() + nearest_at.bytes(); }
  Rows rows() const { return Rows{force.as<double4>(), energy.as<double>(), nearest.as<double>(), nearest_at.as<int>()}; }
};

// Tile shape of the FP32 near-field gather: sources per warp (2, 4 or 8; for the spacing
// pass also 1, one source per thread walking its own ball) and target shell sites per chart
// cell.
struct NearTiles {
  int group_size = kNearGroup;
  double sites_per_cell = kSitesPerCell;
  double walk = kSpacingWalk;  // spacing passes: the first walk's fraction of the cutoff
};
// The smallest first-walk fraction accepted (below it most sources would need the exact
// search).
constexpr double kMinSpacingWalk = 0.3;
// Which near-field pass a tile choice is for.
enum TileKind : int { kTilesRelax = 0, kTilesSpacing = 1 };
// The tile table's choice for a group and sample size: the entry of (kind, group,
// floor(log2 n)), else the group's entry of the nearest size bucket, else the defaults. The
// table is read once per process from $ZXTALORI_TILES, or near_tiles.txt in the package
// directory beside the library's _lib folder; lines "kind group bucket sources_per_warp
// sites_per_cell [walk]" (kind relax|spacing, group by name; walk, for spacing lines, the
// first walk's fraction of the cutoff), '#' comments.
NearTiles lookup_tiles(int kind, int gid, int n);

// Near-field workspace (src/near.zig:31-196): sized by one shell pass, then reused.
class NearField {
 public:
  NearField(int gid, double delta) : gid_(gid), delta_(delta) {}
  int gid() const { return gid_; }
  double delta() const { return delta_; }
  double radius() const { return radius_; }
  // Records a pass writing rows of q into `out`.
  void pass(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n, double mean_radius, bool track,
            Rows out, int sms, bool nearest_only = false);
  // The pass in parts, for a batch whose samples share one gather launch. pass_structure
  // records the shell, chart grid, site sort and source order and returns the FP32 gather
  // as a task (true); a pass with no such gather (FP64, dense, or a workspace still to be
  // sized) is recorded whole instead (false). pass_reduce then sums the task's slices.
  bool pass_structure(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n, double mean_radius,
                      Rows out, int sms, NearTask* task);
  void pass_reduce(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n, Rows out);
  // Whether the last pass produced more sites than the workspace holds (after a sync);
  // the next pass sizes it again.
  bool overflowed(cudaStream_t s);
  // The shell, chart grid and site order of the float32 positions q32 without a gather (the
  // covering pass walks them itself); false when the cutoff takes the dense path (no grid).
  // Sizes the workspace first when it is not ready for n FP32 sources.
  bool structure(cudaStream_t s, const float4* q32, const double4* q64, int n, double mean_radius, int sms);
  const uint32_t* cell_offsets() const { return cell_off_.as<uint32_t>(); }
  const NearGrid* grid_device() const { return grid_.as<NearGrid>(); }
  const uint32_t* sorted_codes() const { return scode_.as<uint32_t>(); }
  const uint32_t* sorted_images() const { return simg_.as<uint32_t>(); }
  int capacity() const { return capacity_; }
  int slices() const { return slices_; }
  // Spacing pass: of the last nearest-only pass, how many sources the first walk left to the
  // exact FP64 search and how many of those had an exact tie (waits for the stream).
  void exact_report(cudaStream_t s, uint32_t* listed, uint32_t* ties);
  // Shell sites of the last pass (waits for the stream).
  int site_count(cudaStream_t s);
  // Device bytes the workspace holds.
  size_t bytes() const;
  // Changes whenever the workspace is sized again (buffers move): captured graphs go stale.
  uint64_t generation() const { return generation_; }
  bool ready() const { return ready_; }
  // Summed over every image instead of the shell and chart grid (wide cutoffs).
  bool dense() const { return dense_; }
  // Device word set when a pass produced more sites than the workspace holds (null when dense).
  const unsigned int* overflow_flag() const {
    return dense_ || !ready_ ? nullptr : &grid_.as<NearGrid>()->overflow;
  }
  // The next pass sizes the workspace again (after an observed overflow, or for a new
  // sample); allocations large enough are reused.
  void invalidate() { ready_ = false; }
  // Diagnostic: while on, each FP32 grid gather of a force pass adds its candidate sites and
  // in-cutoff pairs to two device counters (pair_counts()).
  void count_pairs(bool on) { counting_ = on; }
  unsigned long long* pair_counts() {
    pair_counts_.ensure(2 * sizeof(unsigned long long));
    return pair_counts_.as<unsigned long long>();
  }
  // Development: the next sizing of the workspace holds only `sites` shell sites (once), so
  // a pass overflows and the resize-and-redo path runs without a GPU fault.
  void override_capacity(uint32_t sites) {
    next_capacity_ = sites;
    ready_ = false;
  }
  // The tile shape to use instead of the table's (none: the table), from the next sizing on.
  void force_tiles(std::optional<NearTiles> tiles) {
    const bool same = tiles.has_value() == forced_.has_value() &&
                      (!tiles || (tiles->group_size == forced_->group_size &&
                                  tiles->sites_per_cell == forced_->sites_per_cell));
    if (same) return;
    forced_ = tiles;
    ready_ = false;
  }
  // The spacing pass's first-walk fraction to use instead of the tile choice's (0: none); it
  // changes no workspace, only the next launches.
  void force_walk(double fraction) { walk_override_ = fraction; }
  const NearTiles& tiles() const { return tiles_; }
  void reconfigure(int gid, double delta) {
    gid_ = gid;
    delta_ = delta;
    ready_ = false;
  }

 private:
  uint64_t generation_ = 0;
  bool dense_ = false;
  PairsPlan plan_;
  void setup(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n, double mean_radius, int sms,
             int kind);
  NearLaunch make_launch(int prec, const float4* q32, const double4* q64, int n, bool track, Rows out,
                         bool nearest_only);
  int gid_;
  double delta_;
  double taper_ = 0.5;
  NearTiles tiles_;
  std::optional<NearTiles> forced_;
  double walk_override_ = 0;
  bool counting_ = false;
  DeviceBuffer pair_counts_;
  bool ready_ = false;
  int n_ = 0, prec_ = -1, capacity_ = 0, sdim_max_ = 1, slices_ = 1, slices32_ = 1;
  uint32_t next_capacity_ = 0;
  double radius_ = 0, s_margin_ = 0, chord_ = 0;
  DeviceBuffer counts_, offsets_, scan_tmp_, shell_mask_, rim_list_, rim_q_, rim_count_;
  DeviceBuffer site_q_, site_meta_, site_cell_, site_rank_, site_pos_;
  DeviceBuffer cell_count_, cell_off_, perm_, sq_, scode_, simg_, sx_, src_key_, src_rank_, mcount_, moff_, src_perm_;
  DeviceBuffer grid_, cells_;
  DeviceBuffer exact_list_, exact_count_;
  RowBuffers partial_;
};

// BB relaxation state (src/pairs.zig:220-413): rows of the current positions, the previous
// force and move per source, and the device-resident step state.
class RelaxState {
 public:
  void reset();
  void set_near(int gid, std::optional<double> delta);
  bool near() const { return near_ != nullptr; }
  std::optional<double> near_delta() const {
    return near_ ? std::optional<double>(near_->delta()) : std::nullopt;
  }
  Rows rows() const { return rows_.rows(); }
  bool current = false;
  // Passes of this state only find each source's nearest site (the spacing pass): the FP32
  // near-field gather then skips the pair terms, whose rows stay 0.
  bool nearest_only = false;
  // The row summary of the last summarize().
  const RowSummary& last_summary() const { return last_summary_; }

  void prepare(cudaStream_t s, int n, int prec);
  void record_forces(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n, int gid, bool track,
                     double budget_scale, int sms);
  void step(cudaStream_t s, int prec, float4* q32, double4* q64, int n, int gid, int fixed, double budget_scale, int sms);
  // The same step in two parts around a shared gather launch: step_structure records what
  // comes before the near-field gather and returns it as a task (true), or records the whole
  // force pass (false); step_finish sums the task's slices (had_task) and makes the BB update.
  bool step_structure(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n, int gid,
                      double budget_scale, int sms, NearTask* task);
  void step_finish(cudaStream_t s, int prec, float4* q32, double4* q64, int n, int gid, int fixed, int sms,
                   bool had_task);
  StepResult finish(cudaStream_t s);
  // Quick measures of `rows()` (after a force pass), nearest degrees and neighbours to host.
  Measures summarize(cudaStream_t s, int n, int order, float* degrees, int* neighbours, int prec, const float4* q32,
                     int gid);
  // The same, split: enqueue the kernels and the copies of the summary, degrees and
  // neighbours into host memory; then, after the stream is synchronised, the measures.
  void summarize_async(cudaStream_t s, int n, int order, RowSummary* summary, float* degrees, int* neighbours,
                       int prec, const float4* q32, int gid);
  Measures measures_of(const RowSummary& sum, int n, int order) const;
  const RelaxDev* state_device() const { return state_.as<RelaxDev>(); }
  // Each source's nearest neighbour's source index from the last summarize (device).
  const int* neighbours_device() const { return neighbours_.as<int>(); }
  StepResult result_of(const RelaxDev& st) const { return step_result(st); }
  bool near_overflowed(cudaStream_t s) { return near_ && near_->overflowed(s); }
  NearField* near_field() { return near_.get(); }
  // Device bytes the state (and its near-field workspace) holds.
  size_t bytes() const;
  // Identifies the buffers and settings a captured step reads; any change makes it stale.
  uint64_t generation() const { return generation_ * 1000003ull + (near_ ? near_->generation() * 7 + 1 : 0); }
  // Whether a step would run without sizing anything (so it can be captured in a graph).
  bool sized(int n, int prec) const { return n_ == n && prec_ == prec && (!near_ || near_->ready()); }

 private:
  RowSummary last_summary_{};
  uint64_t generation_ = 0;
  StepResult step_result(const RelaxDev& st) const;
  void step_update(cudaStream_t s, int prec, float4* q32, double4* q64, int n, int gid, int fixed, int sms);
  int n_ = 0, prec_ = -1, order_ = 0;
  RowBuffers rows_, partial_;
  DeviceBuffer prev_f_, prev_d_, state_, stats_partials_, hist_, summary_, summary_partials_, near_partials_,
      near_rows_, degrees_, neighbours_;
  std::unique_ptr<NearField> near_;
};

class Engine {
 public:
  Engine();
  ~Engine();
  // Reference entry points (src/engine.zig). Each throws Failure on error.
  void set(int gid, const float* values, size_t count);
  void generate_random(int gid, uint32_t count, uint32_t seed);
  void generate_grid(int gid, uint32_t freq, uint32_t target, uint32_t seed, uint32_t kind);
  // Exact-count generation (src/engine.zig:199-231): the largest inverse-Hopf grid within
  // the target, then points at the centres of the largest empty Delaunay caps until the
  // sample holds exactly `target` orientations (insert.cpp).
  void generate_exact(int gid, uint32_t target, bool add_identity, uint32_t kind);
  void measure();
  // measure() with every ratio over all pairs at any count (above the ratio limit too).
  void measure_full();
  void spacing();
  // The covering radius on request (src/engine.zig:377-399): measured again only when the
  // sample (group and float32 orientations) or the iteration has changed since the last one.
  void cover();
  // Covering optimisation (optimize.cpp; src/engine.zig:407-534): `steps` steps that lower
  // the covering radius, continuing the run while the sample is the one the last batch ended
  // on; `finish` restores the best sample and measures it. mode bit 0: face (a wider band of
  // caps moves) else tet; floor_deg: separation floor (SO(3) degrees, 0: none).
  void set_kicks(uint32_t patience, double progress, double size, double trust);
  void optimize_covering(uint32_t steps, uint32_t mode, bool finish, double floor_deg);
  // The triangulation display (src/engine.zig buildMesh): every source's star as one mesh of
  // stereographic vertices (4 floats each, the sources first) and tetrahedra (4 indices).
  void build_mesh();
  const std::vector<float>& mesh_vertices() const { return mesh_vertices_; }
  const std::vector<uint32_t>& mesh_tets() const { return mesh_tets_; }
  void relax(uint32_t steps);
  void set_neighbourhood(double delta);
  void identity(bool add, bool fixed);
  const char* stats();
  const float* point_values(uint32_t kind) const;
  // The neighbour indices of the last pass that made point values; after a spacing pass they
  // are copied to the host here, on the first request.
  const int* point_neighbours();
  // Device memory this engine holds now (every buffer it sized, from the pool).
  size_t device_bytes() const;
  // Of the last spacing pass: sources settled by the exact FP64 search instead of the FP32
  // gather, and sources whose nearest distance two different sources share exactly.
  void spacing_exact(uint32_t* listed, uint32_t* ties);
  void cancel() { cancelled_.store(true); }
  // Extensions.
  void set_precision(int prec);
  int precision() const { return prec_; }
  void set_pair_budget(double scale) {
    budget_scale_ = scale;
    ++config_gen_;
  }
  // Relaxation split in two: enqueue `steps` BB steps on the engine's stream and return
  // (FP32 mode replays a CUDA graph of one step), then finish with the closing force pass
  // and readback of relax(). Several engines relax concurrently this way.
  void relax_async(uint32_t steps);
  void relax_finish();
  // relax_finish in two halves for batches: enqueue the closing force pass and the copies
  // of its results into pinned host memory, then collect them after one wait.
  void finish_async();
  void finish_collect();
  // Whether the engine's stream has no work pending.
  bool idle();
  // A batch's part of this engine (zo_batch_relax): batch_begin as relax_async starts a run;
  // each step is batch_structure (on the engine's stream; true when it leaves its near-field
  // gather to the batch's shared launch, as `task`), then batch_finish after that launch.
  // batch_ready: FP32 with graphs on and everything sized, so a step can be captured.
  void batch_begin();
  bool batch_structure(NearTask* task);
  void batch_finish(bool had_task);
  // Counts one step that the batch recorded or replayed (host bookkeeping, once per step).
  void batch_stepped();
  bool batch_ready() const;
  uint64_t batch_key() const { return graph_key(); }
  int device() const { return device_; }
  int sms() const { return sms_; }
  void set_graphs(bool enabled) {
    use_graphs_ = enabled;
    drop_graph();
  }
  bool graphs_enabled() const { return use_graphs_; }
  // Tuning: the tile shape of this engine's near-field gathers (relaxation and spacing)
  // instead of the table's; nullopt returns to the table.
  void force_tiles(std::optional<NearTiles> tiles);
  // Development: the next near-field pass (of the relaxation and of the spacing pass) sizes
  // its workspace for only `sites` shell sites, once; 0 cancels.
  void debug_shell_capacity(uint32_t sites) { shell_override_ = sites; }
  // Development: where the covering pass collects neighbours (0 by size, 1 every image, 2
  // the chart grid); the result does not depend on it.
  void debug_cover_mode(uint32_t mode) {
    if (mode > 2) throw Failure("UnknownCoverMode");
    cover_mode_ = (int)mode;
    cover_.reset();
  }
  // The spacing pass's first-walk fraction of the cutoff, instead of the tile table's (0:
  // the table's); the result does not depend on it, only the time.
  void force_walk(double fraction);
  // Development: one pass's raw rows to host. what 0: force pass of the relaxation
  // (8 doubles per source), 1: full measure rows (12 doubles per source).
  void debug_rows(uint32_t what, double* out);
  // One force pass of the relaxation counting its pairs: out[0] candidate sites evaluated,
  // out[1] pairs inside the cutoff that exert a force; -1 for both when the pass has no FP32
  // grid gather (all pairs, a dense cutoff, FP64 mode).
  void debug_pair_counts(double* out);
  // Measurement: `steps` relaxation steps after `warmup`, each bracketed by CUDA events on
  // the engine's stream with an L2 flush (a memset of flush_bytes) before it, outside the
  // events. out[0] total step ms, out[1] dominant-kernel ms, out[2] its launches, out[3]
  // kernel launches per step, out[4 ..] each step's ms (as room allows).
  void bench(uint32_t steps, uint32_t warmup, double flush_bytes, double* out, uint32_t out_len);
  // Measurement of the spacing pass: `passes` passes after `warmup`, each bracketed by CUDA
  // events (an L2 flush before it, outside the events). out[0] ms per pass (gather, exact
  // search, refinement, degrees and neighbours into host memory), out[1] ms per launch of
  // the gather kernel, out[2] its launches, out[3] shell sites, out[4] points settled by
  // the exact search, out[5] kernel launches per pass.
  void bench_spacing(uint32_t passes, uint32_t warmup, double flush_bytes, double* out, uint32_t out_len);
  // Measured FP32 FMA throughput of this engine's device, TFLOP/s, with scalar FMAs or
  // with packed (f32x2) FMAs.
  double fp32_peak(bool packed = false) {
    ZO_CUDA(cudaSetDevice(device_));
    double t = 0, t2 = 0;
    ZO_CUDA(measure_fp32_peak(sms_, &t, packed ? &t2 : nullptr));
    return packed ? t2 : t;
  }

  int group() const { return group_; }
  cudaStream_t stream() const { return stream_; }
  uint32_t count() const { return n_; }
  uint32_t order() const { return (uint32_t)host_group_order(group_); }
  const float* quaternions() const { return host_.data(); }
  uint32_t ratio_limit() const;
  char err[2048] = {0};

 private:
  // Pinned host copies of a closing pass's results (asynchronous finish); the nearest
  // degrees and neighbours go straight to the pinned point arrays.
  struct Staging {
    RowSummary* summary = nullptr;
    RelaxDev* state = nullptr;
    unsigned int* overflow = nullptr;
    float* positions = nullptr;
    size_t capacity = 0;
    void ensure(size_t n);
    void release();
    ~Staging() { release(); }
  };
  Staging stage_;
  bool finishing_ = false, finish_recorded_ = false, finish_has_overflow_ = false;
  void step_once();
  void capture_step_graph();
  void drop_graph();
  uint64_t graph_key() const;
  cudaGraphExec_t step_graph_ = nullptr;
  uint64_t graph_key_ = 0;
  uint64_t config_gen_ = 0;
  bool use_graphs_ = true;
  bool relaxing_ = false, recorded_ = false;
  void adopt(uint32_t n);
  void reset_run();
  void sync_neighbourhood();
  // The development shell capacity (once) and the forced tile shape, onto the state's near field.
  void apply_overrides(RelaxState& state);
  uint32_t shell_override_ = 0;
  std::optional<NearTiles> forced_tiles_;
  double forced_walk_ = 0;
  void fetch();
  Measures full_measure(bool fp64 = false);
  Measures relax_state_measure();
  int fixed_arg() const { return fixed_index_ ? (int)*fixed_index_ : -1; }
  std::optional<uint32_t> identity_index() const;
  // identity_index() of the current host copy (a scan of every orientation), kept until
  // the host copy changes.
  mutable std::optional<std::optional<uint32_t>> identity_cache_;
  // Positions: the FP64 master copy, moved by every BB step in both modes, and its float32
  // rounding, which FP32 mode's pair kernels read and the host copy mirrors. Keeping the
  // master in FP64 stops the float32 rounding of each step from accumulating along the
  // trajectory (it dominated the relaxed sample's drift from the FP64 method).
  float4* q32() { return q32_.as<float4>(); }
  double4* q64() { return q64_.as<double4>(); }

  int device_ = 0, sms_ = 148;
  std::string adapter_;  // the device's name, for stats
  // The engine's stream, declared before every device buffer so that it is destroyed after
  // them (their frees are ordered on it); its destructor waits for the stream.
  struct OwnedStream {
    cudaStream_t s = nullptr;
    ~OwnedStream();
  };
  OwnedStream owned_stream_;
  cudaStream_t stream_ = nullptr;
  int group_ = 9;
  int prec_ = kFP32;
  uint32_t n_ = 0;
  DeviceBuffer q32_, q64_;
  std::vector<float> host_;
  uint32_t iteration_ = 0;
  uint32_t seed_ = 0;
  std::string generator_ = "none";
  // Construction of a generated grid ("hopf"), its frequency and its row count before any
  // identity was added; empty, 0 and the count for imported or random samples.
  std::string grid_kind_;
  uint32_t h_ = 0, base_count_ = 0;
  std::optional<Measures> measures_;
  uint32_t measure_iteration_ = 0;
  bool full_measures_ = false;
  RelaxState relax_state_, spacing_state_;
  double neighbourhood_ = 0, measure_neighbourhood_ = 0;
  PinnedArray<float> point_separation_;
  PinnedArray<int> point_neighbours_;
  bool neighbours_on_device_ = false;  // the last spacing pass's indices are still on the device
  std::optional<uint32_t> point_separation_iteration_;
  double step_deg_ = 0, force_rms_ = 0;
  std::atomic<bool> cancelled_{false};
  bool fix_identity_ = false;
  std::optional<uint32_t> fixed_index_;
  double budget_scale_ = 1.0;
  // Covering.
  std::optional<CoverResult> cover_;
  int cover_mode_ = 0;
  uint32_t cover_iteration_ = 0;
  uint64_t cover_key_ = 0;
  bool cover_cached_ = false;
  uint64_t sample_key() const;
  void measure_covering();
  PinnedArray<float> point_covering_, point_faces_;
  std::optional<uint32_t> point_covering_iteration_;
  DeviceBuffer cover_alpha_, cover_centre_, cover_faces_, cover_facets_, cover_status_, cover_need_, cover_list_,
      cover_probes_;
  std::unique_ptr<NearField> cover_near_;
  // Of the last covering pass: the reach each source's star was proven in, the star width
  // that proved it (0 narrow, 1 middle, 2 wide), its facet count, and the reach its chart
  // grid holds (0: no grid).
  std::vector<double> cover_reach_;
  std::vector<uint8_t> cover_width_;
  std::vector<uint32_t> cover_facet_counts_;
  double cover_grid_reach2_ = 0;
  DeviceBuffer cover_mesh_, cover_mesh_offset_, cover_mesh_normal_;
  // A covering set aside (the optimiser's current sample while a candidate step is
  // measured): everything a covering pass leaves for later calls, swapped in and out whole.
  struct CoverSaved {
    bool valid = false;
    std::optional<CoverResult> result;
    uint32_t iteration = 0;
    uint64_t key = 0;
    std::optional<uint32_t> point_iteration;
    PinnedArray<float> point_covering, point_faces;
    DeviceBuffer alpha, centre, faces, facets, status;
    std::unique_ptr<NearField> near;
    std::vector<double> reach;
    std::vector<uint8_t> width;
    std::vector<uint32_t> facet_counts;
    double grid_reach2 = 0;
  } cover_saved_;
  void swap_covering();       // exchanges the covering state with cover_saved_
  void set_covering_aside();  // the current covering to cover_saved_; none current after it
  bool restore_covering();    // back from cover_saved_ when it is of the current sample
  void export_stars(std::vector<uint4>& tets, std::vector<double4>& normals);
  std::vector<float> insertion_centres(uint32_t wanted);
  uint32_t distinct_rows(std::vector<float>& values, uint32_t unique) const;
  uint32_t inserted_count_ = 0;
  CoverOptimizer opt_;
  KickSettings kicks_;
  void move_to(const std::vector<float>& values);
  double least_separation();
  void orbit_point(uint32_t key, double out[4]) const;
  std::vector<float> mesh_vertices_;
  std::vector<uint32_t> mesh_tets_;
  // Full-measure scratch.
  RowBuffers full_rows_, full_partial_;
  DeviceBuffer full_extra_, full_pextra_, full_degen_, full_pdegen_;
  std::string text_;
};

double mean_radius(double count);
// Simplex bound on the covering radius of `count` points on S3 (images and antipodes
// included), SO(3) degrees (src/covering_reference.zig:4-15).
double simplex_degrees(double count);

}  // namespace zo
