/* zxtalori B200 engine: the C ABI.
 *
 * Drop-in replacement for the reference engine's shared library (libzxtalori.so) as bound
 * by python/zxtalori/api.py:18-55 through ctypes: every symbol that file binds is exported
 * with the same signature, return convention and error-message prefixes. Each declaration
 * cites the reference entry point it replaces (path:line in the reference project).
 *
 * Conventions (src/exports.zig, src/engine.zig:75,110-113):
 *   - int results: 0 success, -1 failure; zo_error(h) then holds "<prefix>: <ErrorName>".
 *   - Host arrays returned (quaternions, operations, point values) are owned by the engine
 *     and valid until the next call that changes the sample; copy them.
 *   - One engine per handle, called from one thread; zo_cancel may come from another.
 *   - Quaternions are float32 [n][4], scalar first, symmetry acting on the right (q*g).
 *   - Groups: 0 C2, 1 C3, 2 C4, 3 C6, 4 D2, 5 D3, 6 D4, 7 D6, 8 T, 9 O, 10 I.
 */
#ifndef ZXTALORI_H
#define ZXTALORI_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* src/exports.zig:4 */
const char* zo_version(void);

/* src/native_api.zig:129. The wgpu directory argument is accepted and ignored; the engine
 * runs on CUDA device ZXTALORI_DEVICE (default: the current device). NULL on failure. */
void* zo_create(const char* wgpu_dir);
/* src/native_api.zig:140 */
const char* zo_create_error(void);
/* src/native_api.zig:143 */
void zo_destroy(void* h);

/* src/exports.zig:9. Inverse Hopf product grids (kind 0/1); transports (kind 2). */
int zo_generate(void* h, uint32_t group, uint32_t freq, uint32_t target, uint32_t seed, uint32_t kind);
/* src/exports.zig:16-22 (Engine.generateExact): exactly `target` (32 .. 1,000,000)
 * orientations: the inverse-Hopf grid with the largest count within the target, then points
 * at the centres of the largest empty Delaunay caps. flags bit 0 adds the identity; bits
 * 8-15 the grid kind (2, transport: -1, "TransportNotAvailable"). */
int zo_generate_exact(void* h, uint32_t group, uint32_t target, uint32_t flags);
/* src/exports.zig:83. Seeded Haar-uniform sample folded into the zone (shaders/haar.wgsl). */
int zo_random(void* h, uint32_t group, uint32_t count, uint32_t seed);
/* src/exports.zig:23. Import n quaternions (folded into the zone). */
int zo_set(void* h, uint32_t group, const float* q, uint32_t n);

/* src/exports.zig:29-40 */
uint32_t zo_count(void* h);
uint32_t zo_order(void* h);
const float* zo_quaternions(void* h);
const float* zo_operations(void* h);

/* src/exports.zig:41. Full measures below the ratio limit, else Quey energy + separation. */
int zo_measure(void* h);
/* Extension (no reference counterpart; src/engine.zig:308-351 gates the ratios off above the
 * ratio limit): zo_measure with Riesz 1/2/3, Green and log ratios over all pairs at any
 * count, for samples above the ratio limit that want them (N^2 |K| pair evaluations). */
int zo_measure_full(void* h);
/* src/exports.zig:60. Nearest orbit neighbour of every point (near field above 20,000). */
int zo_spacing(void* h);
/* src/exports.zig:49. Up to 1,000 Barzilai-Borwein steps of QVM repulsion. */
int zo_relax(void* h, uint32_t steps);
/* src/exports.zig:55. Forces within delta mean orientation radii; 0 for all pairs. */
int zo_relax_neighbourhood(void* h, float delta);
/* src/exports.zig:66. kind 0: nearest-neighbour SO(3) degrees; NULL before a pass. Kinds 1
 * and 2 (covering) are always NULL here. */
const float* zo_point_values(void* h, uint32_t kind);
/* src/exports.zig:69. bit 0 add the identity, bit 1 hold it fixed. */
int zo_identity(void* h, uint32_t flags);

/* src/exports.zig:45-48 (Engine.checkCovering, src/engine.zig:377-399): the covering
 * radius, the largest empty cap of the sample's full orbit {+-q_j g_k} on S3, in SO(3)
 * degrees, into stats (covering_radius_deg, covering_excess, mesh_ratio, covering_witness,
 * covering_*), and point values kind 1 (each orientation's largest Delaunay cap, degrees)
 * and kind 2 (its Voronoi cell's faces). Measured again only when the group, the float32
 * orientations or the iteration changed since the last call (stats covering_cached).
 * Fewer than 4 orientations: -1 ("Covering radius: TooFewOrientations"). */
int zo_cover(void* h);
/* src/exports.zig:104-120 (Engine.optimizeCovering, setKicks): covering optimisation.
 * zo_cover_optimize runs `steps` steps that lower the covering radius (mode bit 0: "face", a
 * wider band of caps moves, else "tet"; other bits of the reference's mode word are accepted
 * and ignored); a run continues while the sample is the one the last call ended on; `finish`
 * restores the best sample seen and measures it; floor_deg (SO(3) degrees, 0: none) keeps
 * the closest pair from being brought below it. zo_cover_kicks sets the plateau kicks
 * (patience 1..1e6 steps, progress in [0,1), size in [0,1], trust in (0,1]). */
int zo_cover_optimize(void* h, uint32_t steps, uint32_t mode, uint32_t finish, float floor_deg);
int zo_cover_kicks(void* h, uint32_t patience, float progress, float size, float trust);
/* src/exports.zig:88-103 (the triangulation display): zo_mesh brings the covering up to date
 * (zo_cover) and assembles every orientation's Delaunay star into one mesh; the vertices are
 * 4 floats each, stereographic (x, y, z) / (1 + w) of the orbit points and 0, the
 * orientations first (vertex i is orientation i), then every other orbit point a star
 * touches; the tetrahedra are 4 vertex indices each, every hull facet that touches an
 * orientation once. Engine-owned, valid until the next zo_mesh (NULL / 0 before one). */
int zo_mesh(void* h);
const float* zo_mesh_vertices(void* h);
const uint32_t* zo_mesh_tets(void* h);
uint32_t zo_mesh_vertex_count(void* h);
uint32_t zo_mesh_tet_count(void* h);

/* src/exports.zig:73-81 */
const char* zo_stats(void* h);
const char* zo_error(void* h);
void zo_cancel(void* h);

/* src/native_api.zig:161. Scales the all-pairs work split (smaller: more chunks). */
void zo_pair_budget(void* h, float scale);
/* src/native_api.zig:151-156. Per-dispatch profiling is not offered: false / 0. */
bool zo_profile(void* h, bool enabled);
size_t zo_profile_report(void* h, uint8_t* output, size_t capacity);

/* Extension, no reference counterpart: arithmetic of this engine's pair path.
 * 0 FP32 pair arithmetic with FP64 sums, BB products and renormalisation (default);
 * 1 FP64 throughout (the plain method). Resets the BB history. */
int zo_precision(void* h, uint32_t mode);
uint32_t zo_get_precision(void* h);
/* Extension: the nearest orbit neighbour's source index of every point (same pass as
 * zo_point_values kind 0), or NULL before such a pass (or on a CUDA error, with the message
 * in zo_error). After zo_spacing the indices are copied to the host on this call. */
const int32_t* zo_point_neighbours(void* h);
/* Tuning extension, no reference counterpart: the tile shape of this engine's FP32
 * near-field gathers (relaxation and spacing), instead of the tile table's choice:
 * sources per warp 2, 4 or 8 and target shell sites per chart cell (0.5..16); applies from
 * the next pass (the workspace is sized again). 1 (one source per thread, no shared tiles)
 * applies to spacing passes only; relaxation passes then keep 4. sources_per_warp 0
 * returns to the table.
 * The reference's tiling knobs are constants (src/pairs.zig:100-128, src/near.zig:22-29). */
int zo_near_tiles(void* h, uint32_t sources_per_warp, float sites_per_cell);
/* Tuning extension: the fraction of the spacing pass's cutoff (4 mean radii) that its first
 * FP32 walk covers, instead of the tile table's choice (0 returns to the table); 0.3..1.
 * Sources whose nearest neighbour the first walk cannot prove are searched again over the
 * whole cutoff in FP64, so the spacing results do not depend on it, only the pass's time. */
int zo_near_walk(void* h, float fraction);
/* The tile table's choice for a pass kind (0 relaxation, 1 spacing), group and sample size:
 * out[0] sources per warp, out[1] sites per chart cell, out[2] the spacing pass's first-walk
 * fraction (out must hold 3). The table (near_tiles.txt beside the library's folder, or
 * $ZXTALORI_TILES) is read once per process. Needs no GPU; -1 on a bad argument. */
int zo_tiles_lookup(uint32_t kind, uint32_t group, uint32_t n, double* out);
/* Extension, no reference counterpart: the device memory the engine holds now, in bytes
 * (positions, rows, BB history, near-field workspace, measure scratch; all of it from the
 * library's per-device pool). A request server admits samples by it. */
uint64_t zo_device_bytes(void* h);
/* Extension, no reference counterpart: of the last zo_spacing pass (FP32 mode, near field
 * above 20,000 points), out[0] = points whose nearest neighbour the exact FP64 search
 * settled (the FP32 gather could not prove its own choice), out[1] = points whose nearest
 * distance two different points share exactly (exact ties, broken by the lower index).
 * Zeros for all-pairs or FP64-mode passes. Waits for the engine's stream. */
int zo_spacing_exact(void* h, uint32_t* out);
/* Development hook, in the spirit of the reference's dev symbols (src/native_api.zig:150-175):
 * one pass's raw per-source rows into `out` (the caller's n * width doubles).
 * what 0: the relaxation's force pass (all pairs, or the near field when a neighbourhood is
 *   set): force x y z, curvature, Quey energy, nearest squared chord, neighbour position
 *   (image index k*n+j for all pairs, sorted site for the near field), 0 (width 8).
 * what 1: full measure rows: force x y z, curvature, Quey energy, nearest squared chord,
 *   Riesz 1, 2, 3, Green, log sums (the self pair's antipode not yet added), degenerate
 *   flag (width 12). */
int zo_debug_rows(void* h, uint32_t what, double* out);
/* Diagnostic extension: one relaxation force pass that counts its pairs (the rows are the
 * ordinary pass's). out[0]: candidate sites the FP32 near-field gather evaluated (each
 * source against every site of its warp's cell-row runs), out[1]: pairs inside the cutoff
 * that exert a force (the own source's images excluded); both -1 when the pass has no FP32
 * grid gather (all pairs, a dense cutoff, FP64 mode). The reference's metric counts
 * N min(N|K|, 0.94 delta^3 + 64) pairs per pass (src/engine.zig:905-907). */
int zo_debug_pair_counts(void* h, double* out);
/* Development hook (no reference counterpart): the next near-field pass, of the relaxation
 * or of the spacing pass, sizes its shell workspace for only `sites` sites, once (0
 * cancels). A pass that then produces more sites than that overflows, and the engine's
 * resize-and-redo path runs as after a real overflow (src/pairs.zig:391-394, near.zig:191-195). */
int zo_debug_shell_capacity(void* h, uint32_t sites);
/* Development hook (no reference counterpart): where zo_cover collects each orientation's
 * neighbours: 0 by the sample's size (every image for small samples, else the chart grid),
 * 1 every image, 2 the chart grid (when the grid's reach is narrow enough to build one).
 * The result does not depend on it. */
int zo_debug_cover_mode(void* h, uint32_t mode);
/* Measurement hook (no reference counterpart): `steps` relaxation steps of the current
 * sample after `warmup`, each timed with CUDA events on the engine's stream and preceded,
 * outside its events, by a memset of flush_bytes (an L2 flush when larger than L2).
 * out[0] total step ms, out[1] ms of the force pass's row kernel, out[2] its launches,
 * out[3] kernel launches per step, out[4 ..] per-step ms while out_len allows. */
int zo_bench(void* h, uint32_t steps, uint32_t warmup, double flush_bytes, double* out, uint32_t out_len);
/* Measurement hook (no reference counterpart): `passes` spacing passes after `warmup`
 * (src/engine.zig:334-347 is one pass), timed like zo_bench. out[0] ms per pass, out[1] ms
 * per launch of the nearest-only gather kernel, out[2] its launches, out[3] shell sites,
 * out[4] points settled by the exact FP64 search, out[5] kernel launches per pass. */
int zo_bench_spacing(void* h, uint32_t passes, uint32_t warmup, double flush_bytes, double* out, uint32_t out_len);
/* Extensions (no reference counterpart): relaxation in two halves, so many engines relax
 * concurrently. zo_relax_async enqueues `steps` BB steps on the engine's stream and returns
 * at once (in FP32 mode each step replays a CUDA graph captured from the first one);
 * zo_relax_finish waits, runs the closing force pass and reads back positions and measures
 * exactly as zo_relax does at its end. zo_idle: 1 when no work is pending, 0 while busy,
 * -1 on error. zo_graphs(h, 0) turns graph replay off (direct kernel launches). */
int zo_relax_async(void* h, uint32_t steps);
int zo_relax_finish(void* h);
int zo_idle(void* h);
int zo_graphs(void* h, uint32_t enabled);
/* Extension: relax `count` engines by `steps` each, then finish each; status[k] is 0 or -1
 * (message in zo_error(handles[k])); returns the failures. FP32 engines with graphs on (per
 * device) step together: each step is one CUDA graph over all of them, and the near-field
 * gathers of all of them run in one persistent launch. Each result is the same as the
 * engine's own zo_relax would give. Other engines step one launch at a time alongside. */
int zo_batch_relax(void* const* handles, uint32_t count, uint32_t steps, int32_t* status);
/* Measurement hook (no reference counterpart): FP32 FMA throughput of the engine's device
 * in TFLOP/s (2 flops per FMA), the denominator of the pair kernels' roofline; -1 on error. */
double zo_fp32_peak(void* h);
/* The same probe with packed f32x2 FMAs (two FMAs per instruction); -1 on error. */
double zo_fp32x2_peak(void* h);
/* Rows of the inverse-Hopf product grid of frequency `freq` before the zone fold, on the
 * host (src/hopf.zig:528-607 points(); zo_generate folds them on the GPU): 4 floats per
 * row, scalar first, in the reference's row order. With out == NULL returns the row count
 * (src/hopf.zig:78 count()); else writes the rows when capacity (in rows) suffices. Returns
 * the row count, -1 for an unknown group, a frequency outside 1..512 or a grid above ten
 * million rows, -2 when capacity is too small. Needs no GPU. */
int64_t zo_hopf_points(uint32_t group, uint32_t freq, float* out, uint64_t capacity);
/* Diagnostic extension: the group's 2|K|-1 zone bisector planes in the order the shell's rim
 * test takes them (order[r], group-local plane index as in the reference's plane list,
 * src/covering.zig:382-396) with each one's reach (reach[r]: a lower bound, less 1e-5, on the
 * plane's dot product with any point of the zone, from the zone's vertices; -1 for planes
 * that touch the zone and for groups whose zone has no vertices). The rim test of a source
 * stops at the first plane whose reach exceeds the shell margin. Each array holds 119 at
 * most. Returns the plane count, -1 for an unknown group. Needs no GPU. */
int zo_zone_planes(uint32_t group, uint8_t* order, float* reach);

/* No counterpart in the reference. The all-pairs force pass (FP32 pair arithmetic, FP64
 * sums) for callers that cannot allocate device memory: a framework that owns every
 * allocation through its own pool, a caller with a fixed pre-reserved budget, or a thread
 * that must not risk an allocation's synchronisation. It needs no engine handle and
 * allocates nothing; its scratch (the per-chunk partial rows) is a fixed array compiled
 * into the library, 3 MiB per GPU that loads the library, held until the process exits.
 *   q_device:    n float32 quaternions [n][4] on the current device (16-byte aligned),
 *                zone representatives as zo_quaternions returns them;
 *   rows_device: n * 6 doubles on the device (32-byte aligned), written as: [0, 4n) per
 *                source force x, y, z and curvature; [4n, 5n) Quey energy; [5n, 6n)
 *                smallest squared chord to another orbit point;
 *   stream:      the cudaStream_t to run on (NULL: the default stream).
 * Returns 0, or -1 bad argument, -2 n outside 1..65,536 (the scratch's limit), -3 CUDA
 * error (also when an error from the caller's earlier work is still pending on the thread:
 * the call then launches nothing and leaves that error pending); the message goes to
 * `error` (error_len bytes) when given. The first call on a
 * device sets it up (scratch address, group tables); make it before any stream capture.
 * Calls share the scratch: calls that overlap on the GPU race and must be serialised. */
int zo_pair_rows_noalloc(uint32_t group, const float* q_device, uint32_t n, double* rows_device, void* stream,
                         char* error, size_t error_len);

/* Extension (no reference counterpart): the continuous-batching relax + measure service on
 * one GPU, run to completion. Each request is a Haar sample (group, count, seed) relaxed for
 * `steps` BB steps (neighbourhood 0: all pairs) and then measured; `arrival` is its arrival
 * time in seconds from the call. Requests are admitted in arrival order while their device
 * memory fits the budget, every resident sample steps on its own stream in chunks so that
 * the samples' kernels overlap, and the closing pass and measure() run on worker threads.
 * settings (n_settings of them, the rest default): [0] memory budget in bytes (0: 80 % of
 * the free device memory), [1] most resident samples (64), [2] seconds of device work per
 * chunk (0.02), [3] measure (1), [4] precision (0 FP32-refined, 1 FP64), [5] worker
 * threads (4), [6] pair evaluations per second for chunk sizing (2.5e11). results: n entries
 * in completion order (status 0, or -1 with the request's error). Returns 0, or -1 with the
 * message in `error` when the service itself failed. */
typedef struct {
  uint32_t id, group, count, steps, seed;
  float neighbourhood;
  double arrival;
} zo_serve_request;
typedef struct {
  uint32_t id, iteration, count, order;
  double arrival, admitted, finished, neighbourhood, energy, separation_deg;
  int32_t status;
  char error[108];
} zo_serve_result;
int zo_serve(const zo_serve_request* requests, uint32_t n, const double* settings, uint32_t n_settings,
             zo_serve_result* results, char* error, size_t error_len);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* ZXTALORI_H */
