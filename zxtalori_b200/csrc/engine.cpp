// Engine: sample state and the reference's policies over the CUDA kernels.
#include "engine.h"
#include "hopf.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>

#include <map>
#include <mutex>
#include <tuple>

namespace zo {

namespace {
constexpr double kPiH = 3.14159265358979323846;
constexpr uint32_t kMaxCount = 10000000;          // hopf.max_count (src/hopf.zig:23)
constexpr double kFullMeasurePairs = 5e10;        // src/engine.zig:1123
constexpr uint32_t kSpacingAllPairs = 20000;      // src/engine.zig:1126
constexpr double kSpacingDelta = 4;               // src/engine.zig:1127
// Near field over every image ("dense") or over the chart grid. FP64 mode: dense from a
// 0.5 rad cutoff on. FP32 mode (the gather walks exact chart balls): dense from 0.9 rad on,
// or from 0.5 rad for samples of at most 1e8 image pairs, where the grid's fixed cost and
// few warps lose to testing every image (measured on B200 over C2..I, r = 0.57..0.98).
constexpr double kDenseRadius = 0.5;
constexpr double kDenseRadius32 = 0.9;
constexpr double kDenseSmallPairs = 1e8;
constexpr const char* kVersion = "0.3.0";

void ensure_tables(int device) {
  if (device < 0 || device >= kMaxTableDevices) throw Failure("InvalidDevice");
  ZO_CUDA(ensure_device_tables(device));
}

double separation_of(double chord2) {
  return 4.0 * std::asin(std::min(1.0, std::sqrt(std::max(chord2, 0.0)) / 2.0)) * 180.0 / kPiH;
}
}  // namespace

// One upload flag per device, shared by engines and the allocation-free entry point.
namespace {
std::mutex g_tables_mutex;
bool g_tables_uploaded[kMaxTableDevices] = {false};
}  // namespace

cudaError_t ensure_device_tables(int device) {
  if (device < 0 || device >= kMaxTableDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_tables_mutex);
  if (g_tables_uploaded[device]) return cudaSuccess;
  const cudaError_t e = upload_tables(host_tables());
  if (e == cudaSuccess) g_tables_uploaded[device] = true;
  return e;
}

void check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  char msg[512];
  std::snprintf(msg, sizeof msg, "CudaError %s (%s)", cudaGetErrorString(e), what);
  throw Failure(msg);
}

double mean_radius(double count) {
  // d_r: half the m with pi (m - sin m) = pi^2 / count, 60 bisections (src/pairs.zig:205-215).
  const double target = kPiH * kPiH / count;
  double lo = 0, hi = kPiH;
  for (int k = 0; k < 60; ++k) {
    const double middle = 0.5 * (lo + hi);
    if (kPiH * (middle - std::sin(middle)) < target) lo = middle;
    else hi = middle;
  }
  return 0.25 * (lo + hi);
}

// ------------------------------------------------------------------ buffers
void* DeviceBuffer::ensure(size_t bytes) {
  if (bytes <= bytes_ && ptr_) return ptr_;
  release();
  const size_t want = std::max<size_t>(bytes, 256);
  const cudaStream_t s = alloc_stream();
  if (s) {
    ptr_ = device_pool_alloc(want, s);
    stream_ = s;
  } else {
    ZO_CUDA(cudaMalloc(&ptr_, want));
  }
  bytes_ = want;
  return ptr_;
}
void DeviceBuffer::release() {
  if (ptr_) {
    if (stream_) cudaFreeAsync(ptr_, stream_);
    else cudaFree(ptr_);
  }
  ptr_ = nullptr;
  bytes_ = 0;
  stream_ = nullptr;
}

Rows RowBuffers::ensure(size_t n) {
  force.ensure(n * sizeof(double4));
  energy.ensure(n * sizeof(double));
  nearest.ensure(n * sizeof(double));
  nearest_at.ensure(n * sizeof(int));
  return rows();
}

// ------------------------------------------------------------------ near field
// ------------------------------------------------------------------ tile table
namespace {
struct TileTable {
  std::map<std::tuple<int, int, int>, NearTiles> entries;  // (kind, group, log2 bucket)
};

std::string tile_table_path() {
  if (const char* env = std::getenv("ZXTALORI_TILES")) return env;
  Dl_info info;
  if (dladdr(reinterpret_cast<void*>(&lookup_tiles), &info) && info.dli_fname) {
    std::string lib = info.dli_fname;
    const size_t slash = lib.rfind('/');
    const std::string dir = slash == std::string::npos ? std::string(".") : lib.substr(0, slash);
    return dir + "/../near_tiles.txt";
  }
  return "near_tiles.txt";
}

const TileTable& tile_table() {
  static std::once_flag once;
  static TileTable table;
  std::call_once(once, [] {
    FILE* f = std::fopen(tile_table_path().c_str(), "r");
    if (!f) return;
    char line[256];
    while (std::fgets(line, sizeof line, f)) {
      char kind[32], group[8];
      int bucket = 0, g = 0;
      double spc = 0, walk = kSpacingWalk;
      const int fields = line[0] == '#' ? 0 : std::sscanf(line, "%31s %7s %d %d %lf %lf", kind, group, &bucket, &g, &spc, &walk);
      if (fields < 5) continue;
      const int k = std::strcmp(kind, "spacing") == 0 ? kTilesSpacing : std::strcmp(kind, "relax") == 0 ? kTilesRelax : -1;
      int gid = -1;
      for (int c = 0; c < 11; ++c)
        if (std::strcmp(group, host_group_name(c)) == 0) gid = c;
      if (k < 0 || gid < 0 || (g != 1 && g != 2 && g != 4 && g != 8) || !(spc >= 0.5 && spc <= 16)) continue;
      if (g == 1 && k != kTilesSpacing) continue;  // one source per thread: spacing passes only
      if (fields == 6 && !(walk >= kMinSpacingWalk && walk <= 1.0)) continue;
      table.entries[{k, gid, bucket}] = NearTiles{g, spc, k == kTilesSpacing ? walk : kSpacingWalk};
    }
    std::fclose(f);
  });
  return table;
}
}  // namespace

NearTiles lookup_tiles(int kind, int gid, int n) {
  const TileTable& t = tile_table();
  const int bucket = n > 0 ? 31 - __builtin_clz((unsigned)n) : 0;
  const NearTiles* best = nullptr;
  int distance = 1 << 30;
  for (auto it = t.entries.lower_bound({kind, gid, -1000}); it != t.entries.end(); ++it) {
    const auto& [k, g, b] = it->first;
    if (k != kind || g != gid) break;
    const int d = std::abs(b - bucket);
    if (d < distance) {  // the nearest bucket; the lower one on a tie
      distance = d;
      best = &it->second;
    }
  }
  return best ? *best : NearTiles{};
}

void NearField::setup(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n, double mean_r, int sms,
                      int kind) {
  ready_ = false;
  ++generation_;
  n_ = n;
  prec_ = prec;
  tiles_ = forced_ ? *forced_ : lookup_tiles(kind, gid_, n);
  // One source per thread is a spacing-pass search only; relaxation passes keep the default.
  if (tiles_.group_size == 1 && kind != kTilesSpacing) tiles_.group_size = kNearGroup;
  radius_ = std::min(1.5, delta_ * mean_r);
  s_margin_ = std::sin(radius_ + 1e-4);
  chord_ = 2.0 * std::sin(radius_ / 2.0);
  // Wide cutoffs: every image is tested (the shell holds most images anyway, and images
  // near the chart's far pole spread the chart box until the grid degenerates).
  const double image_pairs = (double)n * n * host_group_order(gid_);
  dense_ = prec == kFP64 ? radius_ >= kDenseRadius
                         : radius_ >= kDenseRadius32 || (radius_ >= kDenseRadius && image_pairs <= kDenseSmallPairs);
  if (dense_) {
    plan_ = plan_pairs(n, host_group_order(gid_), 1.0, sms);
    if (plan_.chunks > 1) partial_.ensure((size_t)plan_.chunks * n);
    ready_ = true;
    return;
  }
  counts_.ensure((size_t)(n + 1) * 4);
  offsets_.ensure((size_t)(n + 1) * 4);
  shell_mask_.ensure((size_t)n * sizeof(uint4));
  rim_list_.ensure((size_t)n * sizeof(uint32_t));
  rim_q_.ensure((size_t)n * sizeof(float4));
  rim_count_.ensure(sizeof(uint32_t));
  scan_tmp_.ensure(4096 * 4);
  ZO_CUDA(launch_shell_count(prec, q32, q64, n, gid_, s_margin_, counts_.as<uint32_t>(), offsets_.as<uint32_t>(),
                             scan_tmp_.as<uint32_t>(), shell_mask_.as<uint4>(), rim_list_.as<uint32_t>(),
                             rim_q_.as<float4>(), rim_count_.as<uint32_t>(), s));
  uint32_t total = 0;
  ZO_CUDA(cudaMemcpyAsync(&total, offsets_.as<uint32_t>() + n, 4, cudaMemcpyDeviceToHost, s));
  ZO_CUDA(cudaStreamSynchronize(s));
  // Room for the shell to change as the sources move (src/near.zig:115-123).
  const uint64_t order = (uint64_t)host_group_order(gid_);
  uint64_t cap = (uint64_t)total + total / 4 + 1024;
  cap = std::min<uint64_t>(cap, 2 * order * (uint64_t)n);
  cap = std::max<uint64_t>(cap, (uint64_t)total);
  if (next_capacity_ > 0) cap = next_capacity_;  // development override, once
  next_capacity_ = 0;
  if (cap > (1ull << 31) - 1) throw Failure("NearShellTooLarge");
  capacity_ = (int)cap;
  sdim_max_ = (int)std::lround(std::cbrt((double)capacity_ / tiles_.sites_per_cell));
  sdim_max_ = std::max(1, std::min(sdim_max_, kMaxCellDim));
  const size_t cells = (size_t)sdim_max_ * sdim_max_ * sdim_max_ + 1;
  const size_t qsize = prec == kFP64 ? sizeof(double4) : sizeof(float4);
  site_q_.ensure(capacity_ * qsize);
  site_meta_.ensure(capacity_ * sizeof(uint4));
  site_cell_.ensure(capacity_ * 4ull);
  site_rank_.ensure(capacity_ * 4ull);
  site_pos_.ensure(capacity_ * sizeof(float4));
  cell_count_.ensure(cells * 4);
  cell_off_.ensure(cells * 4);
  perm_.ensure(capacity_ * 4ull);
  sq_.ensure(capacity_ * qsize);
  scode_.ensure(capacity_ * 4ull);
  sx_.ensure(capacity_ * 4ull);
  simg_.ensure(capacity_ * 4ull);
  const size_t mcells = (size_t)kOrderDim * kOrderDim * kOrderDim + 1;
  src_key_.ensure((size_t)n * 4);
  src_rank_.ensure((size_t)n * 4);
  mcount_.ensure(mcells * 4);
  moff_.ensure(mcells * 4);
  src_perm_.ensure((size_t)n * 4);
  grid_.ensure(sizeof(NearGrid));
  cells_.ensure(sizeof(int));
  exact_list_.ensure((size_t)n * 4);
  exact_count_.ensure(2 * sizeof(uint32_t));
  ZO_CUDA(cudaMemsetAsync(exact_count_.as<void>(), 0, 2 * sizeof(uint32_t), s));
  NearGrid g{};
  for (int a = 0; a < 3; ++a) {
    g.box_bits[a] = 0xffffffffu;
    g.box_bits[3 + a] = 0u;
  }
  ZO_CUDA(cudaMemcpyAsync(grid_.as<NearGrid>(), &g, sizeof g, cudaMemcpyHostToDevice, s));
  // Warp tasks (32 sources x one slice of their cell rows): several waves of resident warps.
  const int warps = (n + 31) / 32;
  slices_ = std::max(1, std::min(64, (sms * 48 + warps - 1) / warps));
  const int warps32 = (n + tiles_.group_size - 1) / tiles_.group_size;
  slices32_ = std::max(1, std::min(slices_, (sms * 48 + warps32 - 1) / warps32));
  partial_.ensure((size_t)slices_ * n);
  ZO_CUDA(cudaStreamSynchronize(s));
  ready_ = true;
}

NearLaunch NearField::make_launch(int prec, const float4* q32, const double4* q64, int n, bool track, Rows out,
                                  bool nearest_only) {
  NearLaunch L{};
  L.prec = prec;
  L.gid = gid_;
  L.n = n;
  L.capacity = capacity_;
  L.sdim_max = sdim_max_;
  L.slices = slices_;
  L.slices32 = slices32_;
  L.group_size = tiles_.group_size;
  L.sites_per_cell = tiles_.sites_per_cell;
  L.track = track;
  L.short_atan = radius_ <= 0.4;
  L.nearest_only = nearest_only && track;
  const double walk = 2.0 * std::sin(0.5 * (walk_override_ > 0 ? walk_override_ : tiles_.walk) * radius_);
  L.walk_cut2 = walk * walk;
  L.exact_list = exact_list_.as<uint32_t>();
  L.exact_count = exact_count_.as<uint32_t>();
  L.pair_counts = counting_ ? pair_counts_.as<unsigned long long>() : nullptr;
  L.s_margin = s_margin_;
  L.cut2 = chord_ * chord_;
  L.chord = chord_;
  L.cut_z = taper_ * radius_;
  L.cut_w = 1.0 / std::max(1e-9, (1.0 - taper_) * radius_);
  L.q32 = q32;
  L.q64 = q64;
  L.counts = counts_.as<uint32_t>();
  L.offsets = offsets_.as<uint32_t>();
  L.scan_tmp = scan_tmp_.as<uint32_t>();
  L.shell_mask = shell_mask_.as<uint4>();
  L.rim_list = rim_list_.as<uint32_t>();
  L.rim_q = rim_q_.as<float4>();
  L.rim_count = rim_count_.as<uint32_t>();
  L.site_q32 = prec == kFP64 ? nullptr : site_q_.as<float4>();
  L.site_q64 = prec == kFP64 ? site_q_.as<double4>() : nullptr;
  L.site_meta = site_meta_.as<uint4>();
  L.site_cell = site_cell_.as<uint32_t>();
  L.site_rank = site_rank_.as<uint32_t>();
  L.site_pos = site_pos_.as<float4>();
  L.cell_count = cell_count_.as<uint32_t>();
  L.cell_off = cell_off_.as<uint32_t>();
  L.perm = perm_.as<uint32_t>();
  L.sq32 = prec == kFP64 ? nullptr : sq_.as<float4>();
  L.sq64 = prec == kFP64 ? sq_.as<double4>() : nullptr;
  L.scode = scode_.as<uint32_t>();
  L.sx = sx_.as<float>();
  L.simg = simg_.as<uint32_t>();
  L.src_key = src_key_.as<uint32_t>();
  L.src_rank = src_rank_.as<uint32_t>();
  L.mcount = mcount_.as<uint32_t>();
  L.moff = moff_.as<uint32_t>();
  L.src_perm = src_perm_.as<uint32_t>();
  L.grid = grid_.as<NearGrid>();
  L.cells = cells_.as<int>();
  L.partial = partial_.rows();
  L.out = out;
  return L;
}

void NearField::pass(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n, double mean_r, bool track,
                     Rows out, int sms, bool nearest_only) {
  if (!ready_ || n != n_ || prec != prec_)
    setup(s, prec, q32, q64, n, mean_r, sms, nearest_only ? kTilesSpacing : kTilesRelax);
  if (dense_) {
    ZO_CUDA(launch_dense_near(prec, track, radius_ <= 0.4, q32, q64, n, gid_, plan_, chord_ * chord_, chord_,
                              taper_ * radius_, 1.0 / std::max(1e-9, (1.0 - taper_) * radius_),
                              plan_.chunks > 1 ? partial_.rows() : Rows{}, out, s));
    return;
  }
  ZO_CUDA(launch_near(make_launch(prec, q32, q64, n, track, out, nearest_only), s));
}

bool NearField::structure(cudaStream_t s, const float4* q32, const double4* q64, int n, double mean_r, int sms) {
  if (!ready_ || n != n_ || prec_ != kFP32) setup(s, kFP32, q32, q64, n, mean_r, sms, kTilesRelax);
  if (dense_) return false;
  int launches = 0;
  ZO_CUDA(launch_near_structure(make_launch(kFP32, q32, q64, n, false, Rows{}, false), s, &launches));
  probe_count(launches);
  return true;
}

bool NearField::pass_structure(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n,
                               double mean_r, Rows out, int sms, NearTask* task) {
  if (prec != kFP32 || !ready_ || n != n_ || prec != prec_ || dense_) {
    pass(s, prec, q32, q64, n, mean_r, false, out, sms);  // the whole pass, on this stream
    return false;
  }
  const NearLaunch L = make_launch(prec, q32, q64, n, false, out, false);
  int launches = 0;
  ZO_CUDA(launch_near_structure(L, s, &launches));
  probe_count(launches);
  *task = near_task(L);
  return true;
}

void NearField::pass_reduce(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n, Rows out) {
  ZO_CUDA(launch_near_reduce(make_launch(prec, q32, q64, n, false, out, false), s));
}

void NearField::exact_report(cudaStream_t s, uint32_t* listed, uint32_t* ties) {
  uint32_t c[2] = {0, 0};
  if (ready_ && !dense_) {
    ZO_CUDA(cudaMemcpyAsync(c, exact_count_.as<uint32_t>(), sizeof c, cudaMemcpyDeviceToHost, s));
    ZO_CUDA(cudaStreamSynchronize(s));
  }
  *listed = c[0];
  *ties = c[1];
}

size_t NearField::bytes() const {
  const DeviceBuffer* all[] = {&counts_,    &offsets_,  &scan_tmp_, &shell_mask_, &rim_list_,  &rim_q_,
                               &rim_count_, &site_q_,   &site_meta_, &site_cell_, &site_rank_,
                               &site_pos_,  &cell_count_, &cell_off_, &perm_,     &sq_,        &scode_,
                               &simg_,      &sx_,       &src_key_,  &src_rank_,  &mcount_,    &moff_,
                               &src_perm_,  &grid_,     &cells_,    &exact_list_, &exact_count_};
  size_t total = partial_.bytes();
  for (const DeviceBuffer* b : all) total += b->bytes();
  return total;
}

int NearField::site_count(cudaStream_t s) {
  if (!ready_ || dense_) return 0;
  int sites = 0;
  ZO_CUDA(cudaMemcpyAsync(&sites, &grid_.as<NearGrid>()->sites, sizeof sites, cudaMemcpyDeviceToHost, s));
  ZO_CUDA(cudaStreamSynchronize(s));
  return sites;
}

bool NearField::overflowed(cudaStream_t s) {
  if (!ready_ || dense_) return false;
  unsigned int flag = 0;
  ZO_CUDA(cudaMemcpyAsync(&flag, &grid_.as<NearGrid>()->overflow, 4, cudaMemcpyDeviceToHost, s));
  ZO_CUDA(cudaStreamSynchronize(s));
  if (!flag) return false;
  ready_ = false;
  return true;
}

// ------------------------------------------------------------------ relaxation state
void RelaxState::reset() {
  ++generation_;
  n_ = 0;
  prec_ = -1;
  current = false;
  // The near-field settings stay; the workspace is sized again on the next pass, reusing
  // its allocations where they are large enough (a new sample of similar size frees and
  // allocates nothing).
  if (near_) near_->invalidate();
}

size_t RelaxState::bytes() const {
  const DeviceBuffer* all[] = {&prev_f_,           &prev_d_,        &state_,       &stats_partials_,
                               &hist_,             &summary_,       &summary_partials_, &near_partials_,
                               &near_rows_,        &degrees_,       &neighbours_};
  size_t total = rows_.bytes() + partial_.bytes() + (near_ ? near_->bytes() : 0);
  for (const DeviceBuffer* b : all) total += b->bytes();
  return total;
}

void RelaxState::set_near(int gid, std::optional<double> delta) {
  if (near_) {
    if (delta && near_->gid() == gid && near_->delta() == *delta) return;
    current = false;
    ++generation_;
    if (delta) {
      near_->reconfigure(gid, *delta);  // keeps the allocations
      return;
    }
    near_.reset();
  }
  if (delta) {
    near_ = std::make_unique<NearField>(gid, *delta);
    current = false;
    ++generation_;
  }
}

void RelaxState::prepare(cudaStream_t s, int n, int prec) {
  if (n_ == n && prec_ == prec) return;
  ++generation_;
  n_ = n;
  prec_ = prec;
  current = false;
  rows_.ensure(n);
  prev_f_.ensure((size_t)n * sizeof(double4));
  prev_d_.ensure((size_t)n * sizeof(double4));
  ZO_CUDA(cudaMemsetAsync(prev_f_.as<void>(), 0, (size_t)n * sizeof(double4), s));
  ZO_CUDA(cudaMemsetAsync(prev_d_.as<void>(), 0, (size_t)n * sizeof(double4), s));
  state_.ensure(sizeof(RelaxDev));
  ZO_CUDA(cudaMemsetAsync(state_.as<void>(), 0, sizeof(RelaxDev), s));
  const int blocks = reduce_blocks(n);
  stats_partials_.ensure((size_t)blocks * 5 * sizeof(double));
  hist_.ensure(512 * 4);
  ZO_CUDA(cudaMemsetAsync(hist_.as<void>(), 0, 512 * 4, s));
  summary_.ensure(sizeof(RowSummary));
  ZO_CUDA(cudaMemsetAsync(summary_.as<void>(), 0, sizeof(RowSummary), s));
  summary_partials_.ensure((size_t)blocks * 2 * sizeof(double));
  near_partials_.ensure((size_t)blocks * sizeof(double));
  near_rows_.ensure((size_t)blocks * sizeof(int));
  degrees_.ensure((size_t)n * sizeof(float));
  neighbours_.ensure((size_t)n * sizeof(int));
}

void RelaxState::record_forces(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n, int gid,
                               bool track, double budget_scale, int sms) {
  const int order = host_group_order(gid);
  if (near_) {
    near_->pass(s, prec, q32, q64, n, mean_radius((double)n * order), track, rows_.rows(), sms, nearest_only);
    return;
  }
  const PairsPlan pl = plan_pairs(n, order, budget_scale, sms);
  Rows partial{};
  if (pl.chunks > 1) partial = partial_.ensure((size_t)pl.chunks * n);
  ZO_CUDA(launch_pairs(prec, track, q32, q64, n, gid, pl, partial, rows_.rows(), s));
}

void RelaxState::step(cudaStream_t s, int prec, float4* q32, double4* q64, int n, int gid, int fixed,
                      double budget_scale, int sms) {
  prepare(s, n, prec);
  if (!current) record_forces(s, prec, q32, q64, n, gid, false, budget_scale, sms);
  step_update(s, prec, q32, q64, n, gid, fixed, sms);
}

bool RelaxState::step_structure(cudaStream_t s, int prec, const float4* q32, const double4* q64, int n, int gid,
                                double budget_scale, int sms, NearTask* task) {
  prepare(s, n, prec);
  if (current) return false;  // the forces of these positions are recorded already
  if (!near_) {
    record_forces(s, prec, q32, q64, n, gid, false, budget_scale, sms);
    return false;
  }
  return near_->pass_structure(s, prec, q32, q64, n, mean_radius((double)n * host_group_order(gid)), rows_.rows(),
                               sms, task);
}

void RelaxState::step_finish(cudaStream_t s, int prec, float4* q32, double4* q64, int n, int gid, int fixed, int sms,
                             bool had_task) {
  if (had_task) near_->pass_reduce(s, prec, q32, q64, n, rows_.rows());
  step_update(s, prec, q32, q64, n, gid, fixed, sms);
}

void RelaxState::step_update(cudaStream_t s, int prec, float4* q32, double4* q64, int n, int gid, int fixed, int sms) {
  current = false;
  order_ = host_group_order(gid);
  const double radius = mean_radius((double)n * order_);
  const double alpha0 = (0.8 / 3.4) * radius * radius * radius;
  RelaxDev* st = state_.as<RelaxDev>();
  ZO_CUDA(launch_relax_stats(rows_.rows(), prev_f_.as<double4>(), prev_d_.as<double4>(), n, fixed,
                             stats_partials_.as<double>(), st, s));
  ZO_CUDA(launch_median(prec, rows_.rows(), n, st, hist_.as<unsigned int>(), alpha0, radius, sms, s));
  ZO_CUDA(launch_move_fold(q32, q64, n, gid, prec, rows_.rows(), prev_f_.as<double4>(), prev_d_.as<double4>(), st,
                           fixed, radius, 1.0, s));
}

StepResult RelaxState::step_result(const RelaxDev& st) const {
  if (st.flags & 1u) throw Failure("NonFiniteForce");
  if (st.flags & 2u) throw Failure("DuplicateOrientations");
  const double n = n_;
  double step_max;
  std::memcpy(&step_max, &st.step_bits, 8);
  StepResult r;
  r.max_step_deg = step_max * 360.0 / kPiH;
  r.force_rms = std::sqrt(st.sums[3] / n);
  r.energy = st.sums[4] / (n * order_ * std::max(n - 1, 1.0));
  return r;
}

StepResult RelaxState::finish(cudaStream_t s) {
  RelaxDev st;
  ZO_CUDA(cudaMemcpyAsync(&st, state_.as<RelaxDev>(), sizeof st, cudaMemcpyDeviceToHost, s));
  ZO_CUDA(cudaStreamSynchronize(s));
  return step_result(st);
}

void RelaxState::summarize_async(cudaStream_t s, int n, int order, RowSummary* summary, float* degrees,
                                 int* neighbours, int prec, const float4* q32, int gid) {
  const Rows r = rows_.rows();
  const bool near_sites = near_ != nullptr && !near_->dense();
  const uint32_t* scode = near_sites ? near_->sorted_codes() : nullptr;
  const uint32_t* simg = near_sites ? near_->sorted_images() : nullptr;
  if (prec == kFP32) ZO_CUDA(launch_refine_nearest(q32, n, gid, r, near_sites, scode, simg, neighbours_.as<int>(), s));
  else ZO_CUDA(launch_neighbour_index(r, n, near_sites, scode, neighbours_.as<int>(), s));
  ZO_CUDA(launch_row_summary(r, n, summary_partials_.as<double>(), near_partials_.as<double>(), near_rows_.as<int>(),
                             summary_.as<RowSummary>(), s, nearest_only));
  ZO_CUDA(launch_nearest_degrees(r.nearest, n, degrees_.as<float>(), s));
  ZO_CUDA(cudaMemcpyAsync(summary, summary_.as<RowSummary>(), sizeof(RowSummary), cudaMemcpyDeviceToHost, s));
  if (degrees) ZO_CUDA(cudaMemcpyAsync(degrees, degrees_.as<float>(), (size_t)n * 4, cudaMemcpyDeviceToHost, s));
  if (neighbours) ZO_CUDA(cudaMemcpyAsync(neighbours, neighbours_.as<int>(), (size_t)n * 4, cudaMemcpyDeviceToHost, s));
  order_ = order;
}

Measures RelaxState::summarize(cudaStream_t s, int n, int order, float* degrees, int* neighbours, int prec,
                               const float4* q32, int gid) {
  summarize_async(s, n, order, &last_summary_, degrees, neighbours, prec, q32, gid);
  ZO_CUDA(cudaStreamSynchronize(s));
  return measures_of(last_summary_, n, order);
}

Measures RelaxState::measures_of(const RowSummary& sum, int n, int order) const {
  if (!(sum.nearest > 0)) throw Failure("DuplicateOrientations");
  Measures m;
  m.count_extended = 2.0 * order * n;
  m.quey_energy = sum.energy / ((double)n * order * std::max<double>(n - 1, 1));
  m.separation_deg = separation_of(sum.nearest);
  m.force_rms = std::sqrt(sum.force2 / n);
  return m;
}

// ------------------------------------------------------------------ engine
namespace {
// The device's name, queried once per process (cudaGetDeviceProperties takes milliseconds).
std::string device_name(int device) {
  static std::mutex mutex;
  static std::vector<std::string> names;
  std::lock_guard<std::mutex> lock(mutex);
  if ((int)names.size() <= device) names.resize(device + 1);
  if (names[device].empty()) {
    cudaDeviceProp prop;
    ZO_CUDA(cudaGetDeviceProperties(&prop, device));
    names[device] = prop.name;
  }
  return names[device];
}
}  // namespace

Engine::Engine() {
  const char* dev = std::getenv("ZXTALORI_DEVICE");
  int count = 0;
  ZO_CUDA(cudaGetDeviceCount(&count));
  if (count <= 0) throw Failure("NoCudaDevice");
  if (dev && *dev) device_ = std::atoi(dev);
  else ZO_CUDA(cudaGetDevice(&device_));
  if (device_ < 0 || device_ >= count) throw Failure("InvalidDevice");
  ZO_CUDA(cudaSetDevice(device_));
  int major = 0;
  ZO_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device_));
  if (major < 10) throw Failure("NeedsSm100");
  ZO_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_));
  adapter_ = device_name(device_);
  ensure_tables(device_);
  ZO_CUDA(cudaStreamCreateWithFlags(&owned_stream_.s, cudaStreamNonBlocking));
  stream_ = owned_stream_.s;
}

Engine::~Engine() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  drop_graph();
  // The buffers are freed on stream_ as the members go; owned_stream_ then waits for those
  // frees and destroys the stream.
}

Engine::OwnedStream::~OwnedStream() {
  if (s) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
}

// ------------------------------------------------------------------ graph-captured steps
uint64_t Engine::graph_key() const {
  uint64_t k = relax_state_.generation();
  k = k * 1000033ull + config_gen_;
  k = k * 1000037ull + (uint64_t)(fixed_arg() + 1);
  k = k * 1000039ull + n_;
  return k;
}

void Engine::drop_graph() {
  if (step_graph_) cudaGraphExecDestroy(step_graph_);
  step_graph_ = nullptr;
}

// Captures one BB step (force pass, statistics, median, move and fold) of the current
// sample. Every kernel reads its parameters from the sample's buffers, so the graph replays
// step after step until the buffers or settings change (graph_key).
void Engine::capture_step_graph() {
  drop_graph();
  cudaGraph_t graph = nullptr;
  ZO_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  try {
    relax_state_.current = false;
    relax_state_.step(stream_, prec_, q32(), q64(), (int)n_, group_, fixed_arg(), budget_scale_, sms_);
  } catch (...) {
    cudaStreamEndCapture(stream_, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  ZO_CUDA(cudaStreamEndCapture(stream_, &graph));
  const cudaError_t e = cudaGraphInstantiate(&step_graph_, graph, 0);
  cudaGraphDestroy(graph);
  ZO_CUDA(e);
  graph_key_ = graph_key();
}

// One BB step: the captured graph when it is current, else direct launches (which also
// size the workspace) followed by a capture for the next steps. FP64 mode, the plain
// method, always launches kernel by kernel.
void Engine::step_once() {
  if (fix_identity_ && !fixed_index_) throw Failure("IdentityMissingEnableAddIdentity");
  const bool graphable = use_graphs_ && prec_ == kFP32;
  if (graphable && step_graph_ && !relax_state_.current && graph_key_ == graph_key() &&
      relax_state_.sized((int)n_, prec_)) {
    ZO_CUDA(cudaGraphLaunch(step_graph_, stream_));
  } else {
    relax_state_.step(stream_, prec_, q32(), q64(), (int)n_, group_, fixed_arg(), budget_scale_, sms_);
    if (graphable && relax_state_.sized((int)n_, prec_) && (!step_graph_ || graph_key_ != graph_key()))
      capture_step_graph();
  }
  ++iteration_;
}

void Engine::relax_async(uint32_t steps) {
  if (n_ < 2) throw Failure("TooFewOrientations");
  ZO_CUDA(cudaSetDevice(device_));
  if (!relaxing_) {
    cancelled_.store(false);
    sync_neighbourhood();
    relaxing_ = true;
  }
  for (uint32_t k = 0; k < steps; ++k) {
    step_once();
    recorded_ = true;
  }
}

void Engine::batch_begin() {
  if (n_ < 2) throw Failure("TooFewOrientations");
  ZO_CUDA(cudaSetDevice(device_));
  if (!relaxing_) {
    cancelled_.store(false);
    sync_neighbourhood();
    relaxing_ = true;
  }
}

bool Engine::batch_structure(NearTask* task) {
  if (fix_identity_ && !fixed_index_) throw Failure("IdentityMissingEnableAddIdentity");
  return relax_state_.step_structure(stream_, prec_, q32(), q64(), (int)n_, group_, budget_scale_, sms_, task);
}

void Engine::batch_finish(bool had_task) {
  relax_state_.step_finish(stream_, prec_, q32(), q64(), (int)n_, group_, fixed_arg(), sms_, had_task);
}

void Engine::batch_stepped() {
  ++iteration_;
  recorded_ = true;
}

bool Engine::batch_ready() const {
  return use_graphs_ && prec_ == kFP32 && !relax_state_.current && relax_state_.sized((int)n_, prec_);
}

void Engine::relax_finish() {
  finish_async();
  finish_collect();
}

// One pinned block holds every staging array (one cached allocation per engine).
void Engine::Staging::ensure(size_t n) {
  if (n <= capacity && summary) return;
  release();
  const size_t cap = std::max<size_t>(n, 1);
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t o_state = up(sizeof(RowSummary)), o_overflow = o_state + up(sizeof(RelaxDev)),
               o_positions = o_overflow + 256, total = o_positions + up(cap * 4 * sizeof(float));
  char* base = static_cast<char*>(pinned_alloc(total));
  summary = reinterpret_cast<RowSummary*>(base);
  state = reinterpret_cast<RelaxDev*>(base + o_state);
  overflow = reinterpret_cast<unsigned int*>(base + o_overflow);
  positions = reinterpret_cast<float*>(base + o_positions);
  capacity = cap;
}

void Engine::Staging::release() {
  pinned_free(summary);
  summary = nullptr;
  state = nullptr;
  overflow = nullptr;
  positions = nullptr;
  capacity = 0;
}

// The closing force pass of a relaxation (RelaxState.complete, src/pairs.zig:377-399),
// enqueued with the copies of the last step's state, the summary, nearest degrees and
// neighbours, the overflow flag and the positions into pinned host memory.
void Engine::finish_async() {
  ZO_CUDA(cudaSetDevice(device_));
  if (!relaxing_) sync_neighbourhood();
  relaxing_ = false;
  measures_.reset();
  finish_recorded_ = recorded_;
  recorded_ = false;
  const int n = (int)n_;
  stage_.ensure(n_);
  relax_state_.prepare(stream_, n, prec_);
  if (finish_recorded_)
    ZO_CUDA(cudaMemcpyAsync(stage_.state, relax_state_.state_device(), sizeof(RelaxDev), cudaMemcpyDeviceToHost,
                            stream_));
  relax_state_.current = false;
  relax_state_.record_forces(stream_, prec_, q32(), q64(), n, group_, true, budget_scale_, sms_);
  const NearField* nf = relax_state_.near_field();
  const unsigned int* flag = nf ? nf->overflow_flag() : nullptr;
  finish_has_overflow_ = flag != nullptr;
  if (flag) ZO_CUDA(cudaMemcpyAsync(stage_.overflow, flag, 4, cudaMemcpyDeviceToHost, stream_));
  point_separation_.resize(n_);
  point_neighbours_.resize(n_);
  neighbours_on_device_ = false;
  relax_state_.summarize_async(stream_, n, (int)order(), stage_.summary, point_separation_.data(),
                               point_neighbours_.data(), prec_, q32(), group_);
  ZO_CUDA(cudaMemcpyAsync(stage_.positions, q32(), (size_t)n * 16, cudaMemcpyDeviceToHost, stream_));
  finishing_ = true;
}

void Engine::finish_collect() {
  if (!finishing_) throw Failure("NoFinishPending");
  finishing_ = false;
  ZO_CUDA(cudaStreamSynchronize(stream_));
  std::optional<StepResult> last;
  if (finish_recorded_) last = relax_state_.result_of(*stage_.state);
  Measures m;
  if (finish_has_overflow_ && *stage_.overflow) {
    // The shell outgrew its workspace: size it again and redo the pass synchronously.
    relax_state_.near_field()->invalidate();
    m = relax_state_measure();
    fetch();
  } else {
    m = relax_state_.measures_of(*stage_.summary, (int)n_, (int)order());
    point_separation_iteration_ = iteration_;  // the degrees and neighbours were copied in place
    host_.assign(stage_.positions, stage_.positions + 4 * (size_t)n_);
    identity_cache_.reset();
    relax_state_.current = true;
  }
  if (last) {
    step_deg_ = last->max_step_deg;
    force_rms_ = last->force_rms;
  }
  measures_ = m;
  full_measures_ = false;
  measure_iteration_ = iteration_;
}

bool Engine::idle() {
  const cudaError_t e = cudaStreamQuery(stream_);
  if (e == cudaErrorNotReady) return false;
  ZO_CUDA(e);
  return true;
}

uint32_t Engine::ratio_limit() const {
  return (uint32_t)std::floor(std::sqrt(kFullMeasurePairs / (double)order()));
}

std::optional<uint32_t> Engine::identity_index() const {
  if (identity_cache_) return *identity_cache_;
  std::optional<uint32_t> found;
  for (uint32_t i = 0; i < n_; ++i) {
    const float* a = &host_[(size_t)i * 4];
    if (std::fabs(a[1]) + std::fabs(a[2]) + std::fabs(a[3]) < 1e-6f) {
      found = i;
      break;
    }
  }
  identity_cache_ = found;
  return found;
}

void Engine::fetch() {
  host_.resize((size_t)n_ * 4);
  identity_cache_.reset();
  ZO_CUDA(cudaMemcpyAsync(host_.data(), q32_.as<float4>(), (size_t)n_ * 16, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::reset_run() {
  inserted_count_ = 0;
  point_separation_iteration_.reset();
  point_covering_iteration_.reset();
  cover_.reset();
  cover_cached_ = false;
  cover_saved_.valid = false;
  relax_state_.reset();
  iteration_ = 0;
  step_deg_ = 0;
  force_rms_ = 0;
  measures_.reset();
  full_measures_ = false;
  cancelled_.store(false);
  err[0] = 0;
}

void Engine::adopt(uint32_t n) {
  n_ = n;
  fixed_index_.reset();
  if (fix_identity_) fixed_index_ = identity_index();
  reset_run();
}

void Engine::set(int gid, const float* values, size_t count) {
  if (count == 0 || count > kMaxCount) throw Failure("InvalidCount");
  for (size_t i = 0; i < count; ++i) {
    double norm = 0;
    for (int c = 0; c < 4; ++c) {
      const float x = values[i * 4 + c];
      if (!std::isfinite(x)) throw Failure("NonFiniteQuaternion");
      norm += (double)x * x;
    }
    if (norm < 1e-20) throw Failure("ZeroQuaternion");
  }
  ZO_CUDA(cudaSetDevice(device_));
  const uint32_t n = (uint32_t)count;
  q32_.ensure((size_t)n * 16);
  ZO_CUDA(cudaMemcpyAsync(q32_.as<float4>(), values, (size_t)n * 16, cudaMemcpyHostToDevice, stream_));
  q64_.ensure((size_t)n * 32);
  ZO_CUDA(launch_fold(q32_.as<float4>(), q64(), (int)n, gid, prec_, true, stream_));
  group_ = gid;
  n_ = n;
  fetch();
  adopt(n);
  generator_ = "Imported quaternions";
  grid_kind_.clear();
  h_ = 0;
  base_count_ = n;
}

void Engine::generate_random(int gid, uint32_t count, uint32_t seed) {
  if (count < 1 || count > kMaxCount) throw Failure("InvalidCount");
  ZO_CUDA(cudaSetDevice(device_));
  q32_.ensure((size_t)count * 16);
  q64_.ensure((size_t)count * 32);
  ZO_CUDA(launch_haar(q32_.as<float4>(), (int)count, seed, stream_));
  group_ = gid;
  ZO_CUDA(launch_fold(q32_.as<float4>(), q64(), (int)count, gid, prec_, true, stream_));
  n_ = count;
  fetch();
  adopt(count);
  generator_ = "Haar random";
  grid_kind_.clear();
  h_ = 0;
  base_count_ = count;
  seed_ = seed;
}

// src/engine.zig:244-281: freq = 0 takes the frequency whose count is nearest the target;
// counts are never cut. The rows are orbit images: the zone fold picks each one's
// representative. FCC transports (kind 2) are not part of this engine.
void Engine::generate_grid(int gid, uint32_t freq, uint32_t target, uint32_t seed, uint32_t kind) {
  if (target > hopf::kMaxCount) throw Failure("GridTooLarge");
  if (kind == 2) throw Failure(gid < 8 ? "TransportNeedsTOrOOrI" : "TransportNotAvailable");
  const uint32_t f = freq == 0 ? hopf::nearest_frequency(gid, target == 0 ? 2048 : target) : freq;
  const std::vector<float> rows = hopf::points(gid, f);
  const uint32_t n = (uint32_t)(rows.size() / 4);
  ZO_CUDA(cudaSetDevice(device_));
  q32_.ensure((size_t)n * 16);
  ZO_CUDA(cudaMemcpyAsync(q32_.as<float4>(), rows.data(), (size_t)n * 16, cudaMemcpyHostToDevice, stream_));
  q64_.ensure((size_t)n * 32);
  ZO_CUDA(launch_fold(q32_.as<float4>(), q64(), (int)n, gid, prec_, true, stream_));
  group_ = gid;
  n_ = n;
  fetch();
  adopt(n);
  generator_ = hopf::generator_name(gid);
  grid_kind_ = "hopf";
  h_ = f;
  base_count_ = n;
  seed_ = seed;
}

void Engine::set_precision(int prec) {
  if (prec != kFP32 && prec != kFP64) throw Failure("UnknownPrecision");
  if (prec == prec_) return;
  ZO_CUDA(cudaSetDevice(device_));
  if (prec == kFP64 && n_ > 0) {
    std::vector<double> wide(host_.begin(), host_.end());
    q64_.ensure((size_t)n_ * 32);
    ZO_CUDA(cudaMemcpyAsync(q64_.as<double4>(), wide.data(), (size_t)n_ * 32, cudaMemcpyHostToDevice, stream_));
    ZO_CUDA(cudaStreamSynchronize(stream_));
  }
  prec_ = prec;
  relax_state_.reset();
  spacing_state_.reset();
}

void Engine::set_neighbourhood(double delta) {
  if (!(delta == 0 || (delta >= 2 && delta <= 1000))) throw Failure("NeighbourhoodOutside2To1000");
  neighbourhood_ = delta;
}

void Engine::sync_neighbourhood() {
  relax_state_.set_near(group_, neighbourhood_ > 0 ? std::optional<double>(neighbourhood_) : std::nullopt);
  measure_neighbourhood_ = neighbourhood_;
  apply_overrides(relax_state_);
}

void Engine::force_tiles(std::optional<NearTiles> tiles) {
  if (tiles && tiles->group_size != 1 && tiles->group_size != 2 && tiles->group_size != 4 && tiles->group_size != 8)
    throw Failure("InvalidTiles");
  if (tiles && !(tiles->sites_per_cell >= 0.5 && tiles->sites_per_cell <= 16)) throw Failure("InvalidTiles");
  forced_tiles_ = tiles;
  for (RelaxState* st : {&relax_state_, &spacing_state_})
    if (NearField* nf = st->near_field()) nf->force_tiles(tiles);
}

void Engine::force_walk(double fraction) {
  if (fraction != 0 && !(fraction >= kMinSpacingWalk && fraction <= 1.0)) throw Failure("InvalidWalk");
  forced_walk_ = fraction;
  if (NearField* nf = spacing_state_.near_field()) nf->force_walk(fraction);
}

void Engine::apply_overrides(RelaxState& state) {
  NearField* nf = state.near_field();
  if (nf) nf->force_tiles(forced_tiles_);
  if (nf && &state == &spacing_state_) nf->force_walk(forced_walk_);
  if (!shell_override_ || !nf) return;
  nf->override_capacity(shell_override_);
  shell_override_ = 0;
}

Measures Engine::relax_state_measure() {
  relax_state_.prepare(stream_, (int)n_, prec_);
  for (int attempt = 0; attempt < 4; ++attempt) {
    relax_state_.current = false;
    relax_state_.record_forces(stream_, prec_, q32(), q64(), (int)n_, group_, true, budget_scale_, sms_);
    ZO_CUDA(cudaStreamSynchronize(stream_));
    if (relax_state_.near_overflowed(stream_)) continue;
    point_separation_.resize(n_);
    point_neighbours_.resize(n_);
    neighbours_on_device_ = false;
    point_separation_iteration_ = iteration_;
    Measures m = relax_state_.summarize(stream_, (int)n_, (int)order(), point_separation_.data(),
                                        point_neighbours_.data(), prec_, q32(), group_);
    relax_state_.current = true;
    return m;
  }
  throw Failure("NearShellTooLarge");
}

Measures Engine::full_measure(bool fp64) {
  const int prec = fp64 ? kFP64 : prec_;
  const int n = (int)n_, order = (int)this->order();
  const PairsPlan pl = plan_pairs(n, order, budget_scale_, sms_);
  const Rows out = full_rows_.ensure(n);
  Rows partial{};
  double* pextra = nullptr;
  int* pdegen = nullptr;
  if (pl.chunks > 1) {
    partial = full_partial_.ensure((size_t)pl.chunks * n);
    pextra = (double*)full_pextra_.ensure((size_t)pl.chunks * n * 5 * sizeof(double));
    pdegen = (int*)full_pdegen_.ensure((size_t)pl.chunks * n * sizeof(int));
  }
  double* extra = (double*)full_extra_.ensure((size_t)n * 5 * sizeof(double));
  int* degen = (int*)full_degen_.ensure((size_t)n * sizeof(int));
  ZO_CUDA(launch_full(prec, q32(), q64(), n, group_, pl, partial, pextra, pdegen, out, extra, degen, stream_));
  if (prec == kFP32) {
    DeviceBuffer scratch;
    ZO_CUDA(launch_refine_nearest(q32(), n, group_, out, false, nullptr, nullptr, (int*)scratch.ensure((size_t)n * 4),
                                  stream_));
    ZO_CUDA(cudaStreamSynchronize(stream_));
  }
  std::vector<double> hx((size_t)n * 5), he(n), hn(n);
  std::vector<double4> hf(n);
  std::vector<int> hd(n);
  ZO_CUDA(cudaMemcpyAsync(hx.data(), extra, hx.size() * 8, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaMemcpyAsync(he.data(), out.energy, he.size() * 8, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaMemcpyAsync(hn.data(), out.nearest, hn.size() * 8, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaMemcpyAsync(hf.data(), out.force, hf.size() * sizeof(double4), cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaMemcpyAsync(hd.data(), degen, hd.size() * 4, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaStreamSynchronize(stream_));
  // Host FP64 sums and normalisations (src/pairs.zig:142-173); the self pair's antipode
  // adds (1/2, 1/4, 1/8) to the Riesz rows, -3/(8 pi^2) to Green and 1/4 - ln 2 to log.
  double sum[5] = {0, 0, 0, 0, 0}, energy = 0, force2 = 0, nearv = 4;
  bool degenerate = false;
  for (int i = 0; i < n; ++i) {
    sum[0] += hx[(size_t)i * 5 + 0] + 0.5;
    sum[1] += hx[(size_t)i * 5 + 1] + 0.25;
    sum[2] += hx[(size_t)i * 5 + 2] + 0.125;
    sum[3] += hx[(size_t)i * 5 + 4] + (0.25 - std::log(2.0));
    sum[4] += hx[(size_t)i * 5 + 3] - 3.0 / (8.0 * kPiH * kPiH);
    degenerate |= hd[i] != 0;
    energy += he[i];
    force2 += hf[i].x * hf[i].x + hf[i].y * hf[i].y + hf[i].z * hf[i].z;
    nearv = std::min(nearv, hn[i]);
  }
  if (degenerate) sum[3] = 1e30 * n;
  if (nearv <= 0) throw Failure("DuplicateOrientations");
  const double ext = 2.0 * order, total = n * ext;
  for (double& v : sum) v *= ext;
  const double c_green = std::pow(3.0, 5.0 / 3.0) /
                         (5.0 * std::pow(2.0 * kPiH * kPiH, 1.0 / 3.0) * std::pow(4.0 * kPiH, 2.0 / 3.0));
  const double delta_log = (sum[3] + 0.25 * total + std::log(total) * total / 3.0) / total;
  Measures m;
  m.count_extended = total;
  m.riesz_1 = sum[0] / (total * total * (8.0 / (3.0 * kPiH)));
  m.riesz_2 = sum[1] / (total * total);
  m.riesz_3 = sum[2] / ((2.0 / (3.0 * kPiH)) * total * total * std::log(total));
  m.green_ratio = sum[4] / (-c_green * std::pow(total, 4.0 / 3.0));
  m.log_ratio = delta_log / (-5.0 / 12.0);
  m.quey_energy = energy / ((double)n * order * std::max(n - 1.0, 1.0));
  m.separation_deg = separation_of(nearv);
  m.force_rms = std::sqrt(force2 / n);
  return m;
}

void Engine::measure() {
  if (n_ == 0) throw Failure("NoOrientations");
  ZO_CUDA(cudaSetDevice(device_));
  if (n_ > ratio_limit()) {
    sync_neighbourhood();
    measures_ = relax_state_measure();
    full_measures_ = false;
  } else {
    measures_ = full_measure();
    full_measures_ = true;
    measure_neighbourhood_ = 0;
    sync_neighbourhood();
    relax_state_measure();
    measure_neighbourhood_ = 0;
  }
  measure_iteration_ = iteration_;
}

// Every energy ratio over all pairs whatever the count (above the ratio limit too): the
// explicit extension of measure() for large samples. Above the ratio limit the sums are
// taken in FP64 in both modes: the ratios are small remainders of sums of more than 1e10
// terms (Green's cancels to about N^(-2/3) of its terms' magnitudes), where the FP32 pair
// terms' rounding, about one ulp and biased, shows at the 1e-3 level (I, N = 30,000: Green
// 0.4 % from the FP64 sum).
// The separation is then the spacing pass's (exact, from the float32 sample and the float32
// operator table in FP32-refined mode, as measure() reports it).
void Engine::measure_full() {
  if (n_ == 0) throw Failure("NoOrientations");
  ZO_CUDA(cudaSetDevice(device_));
  const bool above = n_ > ratio_limit();
  measures_ = full_measure(above);
  full_measures_ = true;
  measure_neighbourhood_ = 0;
  measure_iteration_ = iteration_;
  if (above && prec_ == kFP32 && n_ >= 2) spacing();
}

void Engine::spacing() {
  if (n_ < 2) throw Failure("TooFewOrientations");
  ZO_CUDA(cudaSetDevice(device_));
  spacing_state_.set_near(group_, n_ > kSpacingAllPairs ? std::optional<double>(kSpacingDelta) : std::nullopt);
  spacing_state_.nearest_only = true;
  apply_overrides(spacing_state_);
  spacing_state_.prepare(stream_, (int)n_, prec_);
  point_separation_.resize(n_);
  point_separation_iteration_ = iteration_;
  neighbours_on_device_ = false;
  for (int attempt = 0;; ++attempt) {
    if (attempt == 4) throw Failure("NearShellTooLarge");
    spacing_state_.record_forces(stream_, prec_, q32(), q64(), (int)n_, group_, true, budget_scale_, sms_);
    ZO_CUDA(cudaStreamSynchronize(stream_));
    if (!spacing_state_.near_overflowed(stream_)) break;
  }
  try {
    // The per-point degrees come to the host with the pass (the reference's spacing makes
    // them); the neighbour indices stay on the device until point_neighbours() asks.
    spacing_state_.summarize(stream_, (int)n_, (int)order(), point_separation_.data(), nullptr, prec_, q32(),
                             group_);
    neighbours_on_device_ = true;
  } catch (const Failure& x) {
    // A duplicate shows as a zero separation below.
    if (std::strcmp(x.what(), "DuplicateOrientations") != 0) throw;
  }
  const float least = spacing_state_.last_summary().least_degrees;  // the smallest point value
  if (!(least > 0)) throw Failure("DuplicateOrientations");
  if (measures_ && measure_iteration_ == iteration_) {
    measures_->separation_deg = least;
    return;
  }
  Measures m;
  m.count_extended = 2.0 * order() * n_;
  m.separation_deg = least;
  measures_ = m;
  measure_iteration_ = iteration_;
  full_measures_ = false;
}

void Engine::relax(uint32_t steps) {
  if (n_ < 2) throw Failure("TooFewOrientations");
  ZO_CUDA(cudaSetDevice(device_));
  cancelled_.store(false);
  sync_neighbourhood();
  const double n = n_, order = this->order();
  // Wait every ~2e10 pair evaluations so a cancel is seen (src/engine.zig:899-907).
  const double neighbours =
      neighbourhood_ > 0 ? std::min(n * order, 0.94 * std::pow(neighbourhood_, 3) + 64) : n * order;
  const uint64_t sync_every = (uint64_t)std::max(1.0, std::floor(2e10 / (n * neighbours)));
  const uint32_t run = std::min<uint32_t>(steps, 1000);
  bool recorded = false;
  relaxing_ = false;
  recorded_ = false;
  for (uint32_t index = 0; index < run; ++index) {
    if (cancelled_.load()) break;
    step_once();
    recorded = true;
    if ((index + 1) % sync_every == 0 && index + 1 < run) {
      const StepResult r = relax_state_.finish(stream_);
      step_deg_ = r.max_step_deg;
      force_rms_ = r.force_rms;
      recorded = false;
    }
  }
  measures_.reset();
  // One wait ends the batch: the last step, positions, energy and separation, whose forces
  // start the next step (RelaxState.complete, src/pairs.zig:377-399).
  relaxing_ = true;
  recorded_ = recorded;
  finish_async();
  finish_collect();
}

void Engine::identity(bool add, bool fixed) {
  if (n_ == 0) throw Failure("NoOrientations");
  std::optional<uint32_t> index = identity_index();
  if (add && !index) {
    std::vector<float> values(host_);
    values.insert(values.end(), {1.f, 0.f, 0.f, 0.f});
    const std::string generator = generator_, grid_kind = grid_kind_;
    const uint32_t h = h_, base_count = base_count_;
    set(group_, values.data(), values.size() / 4);
    generator_ = generator;
    grid_kind_ = grid_kind;
    h_ = h;
    base_count_ = base_count;
    index = n_ - 1;
  }
  if (fixed && !index) throw Failure("IdentityMissingEnableAddIdentity");
  if (fix_identity_ != fixed) relax_state_.reset();
  fix_identity_ = fixed;
  fixed_index_ = fixed ? index : std::nullopt;
  if (fixed) {
    const uint32_t i = *index;
    const float one[4] = {1.f, 0.f, 0.f, 0.f};
    std::memcpy(&host_[(size_t)i * 4], one, 16);
    identity_cache_.reset();
    ZO_CUDA(cudaMemcpyAsync(q32() + i, one, 16, cudaMemcpyHostToDevice, stream_));
    const double one64[4] = {1, 0, 0, 0};
    ZO_CUDA(cudaMemcpyAsync(q64() + i, one64, 32, cudaMemcpyHostToDevice, stream_));
    ZO_CUDA(cudaStreamSynchronize(stream_));
    relax_state_.current = false;
  }
}

void Engine::debug_pair_counts(double* out) {
  if (n_ == 0) throw Failure("NoOrientations");
  ZO_CUDA(cudaSetDevice(device_));
  const int n = (int)n_;
  sync_neighbourhood();
  relax_state_.prepare(stream_, n, prec_);
  out[0] = out[1] = -1;
  // Size the workspace with an ordinary pass first, then count one pass.
  relax_state_.current = false;
  relax_state_.record_forces(stream_, prec_, q32(), q64(), n, group_, false, budget_scale_, sms_);
  NearField* nf = relax_state_.near_field();
  if (prec_ == kFP64 || !nf || nf->dense()) return;
  unsigned long long* counts = nf->pair_counts();
  ZO_CUDA(cudaMemsetAsync(counts, 0, 2 * sizeof(unsigned long long), stream_));
  nf->count_pairs(true);
  try {
    relax_state_.current = false;
    relax_state_.record_forces(stream_, prec_, q32(), q64(), n, group_, false, budget_scale_, sms_);
  } catch (...) {
    nf->count_pairs(false);
    throw;
  }
  nf->count_pairs(false);
  unsigned long long host[2];
  ZO_CUDA(cudaMemcpyAsync(host, counts, sizeof host, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaStreamSynchronize(stream_));
  relax_state_.current = false;
  out[0] = (double)host[0];
  out[1] = (double)host[1];
}

void Engine::debug_rows(uint32_t what, double* out) {
  if (n_ == 0) throw Failure("NoOrientations");
  if (what > 1) throw Failure("UnknownRows");
  ZO_CUDA(cudaSetDevice(device_));
  const int n = (int)n_;
  Rows r;
  std::vector<double> extra;
  std::vector<int> degen;
  if (what == 0) {
    sync_neighbourhood();
    relax_state_.prepare(stream_, n, prec_);
    relax_state_.current = false;
    relax_state_.record_forces(stream_, prec_, q32(), q64(), n, group_, true, budget_scale_, sms_);
    r = relax_state_.rows();
  } else {
    const PairsPlan pl = plan_pairs(n, (int)order(), budget_scale_, sms_);
    r = full_rows_.ensure(n);
    Rows partial{};
    double* pextra = nullptr;
    int* pdegen = nullptr;
    if (pl.chunks > 1) {
      partial = full_partial_.ensure((size_t)pl.chunks * n);
      pextra = (double*)full_pextra_.ensure((size_t)pl.chunks * n * 5 * sizeof(double));
      pdegen = (int*)full_pdegen_.ensure((size_t)pl.chunks * n * sizeof(int));
    }
    double* dx = (double*)full_extra_.ensure((size_t)n * 5 * sizeof(double));
    int* dd = (int*)full_degen_.ensure((size_t)n * sizeof(int));
    ZO_CUDA(launch_full(prec_, q32(), q64(), n, group_, pl, partial, pextra, pdegen, r, dx, dd, stream_));
    extra.resize((size_t)n * 5);
    degen.resize(n);
    ZO_CUDA(cudaMemcpyAsync(extra.data(), dx, extra.size() * 8, cudaMemcpyDeviceToHost, stream_));
    ZO_CUDA(cudaMemcpyAsync(degen.data(), dd, degen.size() * 4, cudaMemcpyDeviceToHost, stream_));
  }
  std::vector<double4> f(n);
  std::vector<double> e(n), nb(n);
  std::vector<int> at(n);
  ZO_CUDA(cudaMemcpyAsync(f.data(), r.force, (size_t)n * sizeof(double4), cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaMemcpyAsync(e.data(), r.energy, (size_t)n * 8, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaMemcpyAsync(nb.data(), r.nearest, (size_t)n * 8, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaMemcpyAsync(at.data(), r.nearest_at, (size_t)n * 4, cudaMemcpyDeviceToHost, stream_));
  ZO_CUDA(cudaStreamSynchronize(stream_));
  const int width = what == 0 ? 8 : 12;
  for (int i = 0; i < n; ++i) {
    double* o = out + (size_t)i * width;
    o[0] = f[i].x;
    o[1] = f[i].y;
    o[2] = f[i].z;
    o[3] = f[i].w;
    o[4] = e[i];
    o[5] = nb[i];
    if (what == 0) {
      o[6] = at[i];
      o[7] = 0;
    } else {
      for (int c = 0; c < 5; ++c) o[6 + c] = extra[(size_t)i * 5 + c];
      o[11] = degen[i];
    }
  }
}

void Engine::bench(uint32_t steps, uint32_t warmup, double flush_bytes, double* out, uint32_t out_len) {
  if (n_ < 2) throw Failure("TooFewOrientations");
  if (steps == 0 || out_len < 4) throw Failure("InvalidBench");
  ZO_CUDA(cudaSetDevice(device_));
  sync_neighbourhood();
  relax_state_.prepare(stream_, (int)n_, prec_);
  relax_state_.current = false;
  for (uint32_t w = 0; w < std::max<uint32_t>(warmup, 1); ++w) step_once();
  ZO_CUDA(cudaStreamSynchronize(stream_));
  DeviceBuffer flush;
  const size_t fbytes = flush_bytes > 0 ? (size_t)flush_bytes : 0;
  if (fbytes) flush.ensure(fbytes);
  std::vector<cudaEvent_t> ev(4 * (size_t)steps);
  for (auto& e : ev) ZO_CUDA(cudaEventCreate(&e));
  // The timed steps take the product path: graph replays in FP32 mode, kernel by kernel in
  // FP64 mode.
  for (uint32_t k = 0; k < steps; ++k) {
    if (fbytes) ZO_CUDA(cudaMemsetAsync(flush.as<void>(), (int)(k & 0xff), fbytes, stream_));
    ZO_CUDA(cudaEventRecord(ev[2 * k], stream_));
    step_once();
    ZO_CUDA(cudaEventRecord(ev[2 * k + 1], stream_));
  }
  ZO_CUDA(cudaStreamSynchronize(stream_));
  // The dominant kernel's own time and the launch count come from the same number of
  // direct steps, each kernel bracketed by events.
  LaunchProbe probe;
  probe.events = ev.data() + 2 * (size_t)steps;
  probe.capacity = 2 * (int)steps;
  t_probe = &probe;
  try {
    for (uint32_t k = 0; k < steps; ++k) {
      if (fbytes) ZO_CUDA(cudaMemsetAsync(flush.as<void>(), (int)(k & 0xff), fbytes, stream_));
      relax_state_.step(stream_, prec_, q32(), q64(), (int)n_, group_, fixed_arg(), budget_scale_, sms_);
    }
  } catch (...) {
    t_probe = nullptr;
    throw;
  }
  t_probe = nullptr;
  ZO_CUDA(cudaStreamSynchronize(stream_));
  double total = 0, kernel = 0;
  for (uint32_t k = 0; k < steps; ++k) {
    float ms = 0;
    ZO_CUDA(cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]));
    total += ms;
    if (4 + k < out_len) out[4 + k] = ms;
  }
  for (int k = 0; k + 1 < probe.used; k += 2) {
    float ms = 0;
    ZO_CUDA(cudaEventElapsedTime(&ms, probe.events[k], probe.events[k + 1]));
    kernel += ms;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  out[0] = total;
  out[1] = kernel;
  out[2] = probe.used / 2;
  out[3] = (double)probe.launches / steps;
  iteration_ += steps;  // the direct steps (step_once counts its own)
  relax_state_.current = false;
  measures_.reset();
  fetch();
}

size_t Engine::device_bytes() const {
  return q32_.bytes() + q64_.bytes() + relax_state_.bytes() + spacing_state_.bytes() + full_rows_.bytes() +
         full_partial_.bytes() + full_extra_.bytes() + full_pextra_.bytes() + full_degen_.bytes() +
         full_pdegen_.bytes() + cover_alpha_.bytes() + cover_centre_.bytes() + cover_faces_.bytes() +
         cover_facets_.bytes() + cover_status_.bytes() + cover_need_.bytes() + cover_list_.bytes() +
         cover_probes_.bytes() + cover_mesh_.bytes() + cover_mesh_offset_.bytes() + cover_mesh_normal_.bytes() +
         (cover_near_ ? cover_near_->bytes() : 0) + cover_saved_.alpha.bytes() + cover_saved_.centre.bytes() +
         cover_saved_.faces.bytes() + cover_saved_.facets.bytes() + cover_saved_.status.bytes() +
         (cover_saved_.near ? cover_saved_.near->bytes() : 0);
}

void Engine::spacing_exact(uint32_t* listed, uint32_t* ties) {
  *listed = 0;
  *ties = 0;
  NearField* nf = spacing_state_.near_field();
  if (!nf || prec_ != kFP32) return;
  ZO_CUDA(cudaSetDevice(device_));
  nf->exact_report(stream_, listed, ties);
}

void Engine::bench_spacing(uint32_t passes, uint32_t warmup, double flush_bytes, double* out, uint32_t out_len) {
  if (passes == 0 || out_len < 6) throw Failure("InvalidBench");
  for (uint32_t w = 0; w < std::max<uint32_t>(warmup, 1); ++w) spacing();  // sizes the workspace
  ZO_CUDA(cudaSetDevice(device_));
  DeviceBuffer flush;
  const size_t fbytes = flush_bytes > 0 ? (size_t)flush_bytes : 0;
  if (fbytes) flush.ensure(fbytes);
  std::vector<cudaEvent_t> ev(4 * (size_t)passes);
  for (auto& e : ev) ZO_CUDA(cudaEventCreate(&e));
  LaunchProbe probe;
  probe.events = ev.data() + 2 * (size_t)passes;
  probe.capacity = 2 * (int)passes;
  t_probe = &probe;
  RowSummary summary{};
  try {
    for (uint32_t k = 0; k < passes; ++k) {
      if (fbytes) ZO_CUDA(cudaMemsetAsync(flush.as<void>(), (int)(k & 0xff), fbytes, stream_));
      ZO_CUDA(cudaEventRecord(ev[2 * k], stream_));
      spacing_state_.record_forces(stream_, prec_, q32(), q64(), (int)n_, group_, true, budget_scale_, sms_);
      spacing_state_.summarize_async(stream_, (int)n_, (int)order(), &summary, point_separation_.data(), nullptr,
                                     prec_, q32(), group_);
      ZO_CUDA(cudaEventRecord(ev[2 * k + 1], stream_));
    }
  } catch (...) {
    t_probe = nullptr;
    throw;
  }
  t_probe = nullptr;
  ZO_CUDA(cudaStreamSynchronize(stream_));
  double total = 0, kernel = 0;
  for (uint32_t k = 0; k < passes; ++k) {
    float ms = 0;
    ZO_CUDA(cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]));
    total += ms;
  }
  for (int k = 0; k + 1 < probe.used; k += 2) {
    float ms = 0;
    ZO_CUDA(cudaEventElapsedTime(&ms, probe.events[k], probe.events[k + 1]));
    kernel += ms;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  NearField* nf = spacing_state_.near_field();
  uint32_t listed = 0, ties = 0;
  if (nf) nf->exact_report(stream_, &listed, &ties);
  out[0] = total / passes;
  out[1] = probe.used ? kernel / (probe.used / 2) : 0;
  out[2] = probe.used / 2;
  out[3] = nf ? nf->site_count(stream_) : 0;
  out[4] = listed;
  out[5] = (double)probe.launches / passes;
}

const float* Engine::point_values(uint32_t kind) const {
  if (kind == 1 || kind == 2) {
    const PinnedArray<float>& v = kind == 1 ? point_covering_ : point_faces_;
    if (!point_covering_iteration_ || v.size() != n_) return nullptr;
    return v.data();
  }
  if (kind != 0 || !point_separation_iteration_ || point_separation_.size() != n_) return nullptr;
  return point_separation_.data();
}
const int* Engine::point_neighbours() {
  if (!point_separation_iteration_) return nullptr;
  if (neighbours_on_device_) {
    point_neighbours_.resize(n_);
    ZO_CUDA(cudaSetDevice(device_));
    ZO_CUDA(cudaMemcpyAsync(point_neighbours_.data(), spacing_state_.neighbours_device(), (size_t)n_ * sizeof(int),
                            cudaMemcpyDeviceToHost, stream_));
    ZO_CUDA(cudaStreamSynchronize(stream_));
    neighbours_on_device_ = false;
  }
  if (point_neighbours_.size() != n_) return nullptr;
  return point_neighbours_.data();
}

// ------------------------------------------------------------------ stats JSON
namespace {
struct Json {
  std::string s = "{";
  bool first = true;
  void key(const char* k) {
    if (!first) s += ",";
    first = false;
    s += "\"";
    s += k;
    s += "\":";
  }
  void num(const char* k, double v) {
    key(k);
    if (!std::isfinite(v)) {
      s += "null";
      return;
    }
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", v);
    s += b;
  }
  void opt(const char* k, std::optional<double> v) {
    if (v) num(k, *v);
    else null(k);
  }
  void integer(const char* k, long long v) {
    key(k);
    s += std::to_string(v);
  }
  void str(const char* k, const std::string& v) {
    key(k);
    s += "\"";
    for (char c : v) {
      if (c == '"' || c == '\\') s += '\\';
      s += c;
    }
    s += "\"";
  }
  void boolean(const char* k, bool v) {
    key(k);
    s += v ? "true" : "false";
  }
  void null(const char* k) {
    key(k);
    s += "null";
  }
};
std::optional<double> finite(double v) { return std::isfinite(v) ? std::optional<double>(v) : std::nullopt; }
}  // namespace

const char* Engine::stats() {
  const std::optional<Measures>& m = measures_;
  const bool current = m && measure_iteration_ == iteration_;
  Json j;
  j.str("version", kVersion);
  j.str("group", host_group_name(group_));
  j.integer("order", order());
  j.integer("count", n_);
  j.integer("count_extended", 2ll * order() * n_);
  j.str("generator", generator_);
  if (grid_kind_.empty()) j.null("grid");
  else j.str("grid", grid_kind_);
  j.integer("h", h_);
  j.integer("seed", seed_);
  j.integer("iteration", iteration_);
  j.boolean("fixed_identity", fix_identity_);
  if (auto idx = identity_index()) j.integer("identity_index", *idx);
  else j.null("identity_index");
  j.integer("base_count", base_count_);
  j.integer("inserted_count", inserted_count_);
  j.str("triangulation_backend", "cuda");
  const double count_ext = 2.0 * order() * n_;
  const std::optional<double> bound = n_ > 0 ? std::optional<double>(simplex_degrees(count_ext)) : std::nullopt;
  const bool covering_current = cover_ && cover_iteration_ == iteration_;
  j.opt("simplex_bound_deg", bound);
  j.opt("covering_excess", cover_ && bound ? finite(cover_->radius_deg / *bound - 1.0) : std::nullopt);
  j.opt("mesh_ratio", covering_current && current && m->separation_deg > 0
                          ? finite(cover_->radius_deg / m->separation_deg)
                          : std::nullopt);
  j.opt("covering_radius_deg", cover_ ? finite(cover_->radius_deg) : std::nullopt);
  j.boolean("covering_current", covering_current);
  j.boolean("covering_cached", cover_cached_);
  if (cover_) {
    j.integer("covering_unresolved_caps", cover_->unresolved);
    j.integer("covering_iteration", cover_iteration_);
    j.key("covering_witness");
    char b[160];
    std::snprintf(b, sizeof b, "[%.9g,%.9g,%.9g,%.9g]", cover_->witness[0], cover_->witness[1], cover_->witness[2],
                  cover_->witness[3]);
    j.s += b;
    j.opt("covering_domain_bound_deg", finite(cover_->domain_bound_deg));
    j.integer("covering_shell_points", cover_->shell_points);
    j.null("covering_fence_points");
    j.integer("covering_tetrahedra", (long long)(cover_->facets / 4));
    j.integer("covering_certificate_probes", (long long)cover_->probes);
    j.null("covering_exact_predicates");
    j.integer("covering_rounds", cover_->rounds);
    j.integer("covering_first_pass_short", cover_->first_short);
    j.integer("covering_first_pass_sparse", cover_->first_sparse);
    j.integer("covering_rerun_grid", cover_->rerun_grid);
    j.integer("covering_rerun_dense", cover_->rerun_dense);
  } else {
    for (const char* k : {"covering_unresolved_caps", "covering_iteration", "covering_witness",
                          "covering_domain_bound_deg", "covering_shell_points", "covering_fence_points",
                          "covering_tetrahedra", "covering_certificate_probes", "covering_exact_predicates",
                          "covering_rounds", "covering_first_pass_short", "covering_first_pass_sparse",
                          "covering_rerun_grid", "covering_rerun_dense"})
      j.null(k);
  }
  j.boolean("measured", m.has_value());
  j.boolean("measures_current", current);
  if (m) j.integer("measures_iteration", measure_iteration_);
  else j.null("measures_iteration");
  j.boolean("energy_ratios_current", full_measures_ && current);
  if (neighbourhood_ > 0) j.num("relax_neighbourhood", neighbourhood_);
  else j.null("relax_neighbourhood");
  if (point_separation_iteration_) j.integer("point_separation_iteration", *point_separation_iteration_);
  else j.null("point_separation_iteration");
  if (point_covering_iteration_) j.integer("point_covering_iteration", *point_covering_iteration_);
  else j.null("point_covering_iteration");
  if (m && measure_neighbourhood_ > 0) j.num("energy_neighbourhood", measure_neighbourhood_);
  else j.null("energy_neighbourhood");
  j.integer("ratio_limit", ratio_limit());
  const char* precision = !m                          ? "Not measured"
                          : !current                  ? "Energy and separation from an earlier iteration"
                          : !std::isfinite(m->quey_energy) ? "Separation current; energy not measured"
                          : full_measures_            ? "All measures current"
                          : n_ > ratio_limit()        ? "Energy and separation current; this sample exceeds the ratio limit"
                                                      : "Energy and separation current; refresh energy ratios";
  j.str("precision", precision);
  j.opt("energy", m ? finite(m->quey_energy) : std::nullopt);
  j.opt("quey_energy", m ? finite(m->quey_energy) : std::nullopt);
  j.opt("riesz_1", m ? finite(m->riesz_1) : std::nullopt);
  j.opt("riesz_2", m ? finite(m->riesz_2) : std::nullopt);
  j.opt("riesz_3", m ? finite(m->riesz_3) : std::nullopt);
  j.opt("green_ratio", m ? finite(m->green_ratio) : std::nullopt);
  j.opt("log_ratio", m ? finite(m->log_ratio) : std::nullopt);
  j.opt("separation_deg", m ? finite(m->separation_deg) : std::nullopt);
  j.num("step_deg", step_deg_);
  j.opt("force_rms", m ? finite(m->force_rms) : finite(force_rms_));
  j.integer("covering_optimizer_steps", opt_.steps);
  j.integer("covering_optimizer_kicks", opt_.kicks);
  j.opt("covering_optimizer_best_deg", opt_.active ? finite(opt_.best_radius) : std::nullopt);
  j.integer("covering_optimizer_jobs", opt_.jobs);
  j.integer("covering_optimizer_improved", opt_.improved);
  j.integer("covering_optimizer_skipped", opt_.skipped);
  j.integer("covering_optimizer_full_steps", opt_.full_steps);
  j.integer("covering_optimizer_mismatches", 0);
  j.key("covering_kick_settings");
  {
    char b[192];
    std::snprintf(b, sizeof b, "{\"patience\":%u,\"progress\":%.9g,\"size\":%.9g,\"trust\":%.9g}", kicks_.patience,
                  kicks_.progress, kicks_.size, kicks_.trust);
    j.s += b;
  }
  j.str("arithmetic", prec_ == kFP64 ? "fp64" : "fp32-refined");
  j.str("adapter", adapter_);
  j.s += "}";
  text_ = j.s;
  return text_.c_str();
}

}  // namespace zo
