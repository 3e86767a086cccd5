// The engine's CUDA kernels, compiled as one translation unit so that every kernel reads
// the same constant-memory group tables. Parts:
//   k_pairs.cuh  sampler, fold, scan, all-pairs force rows
//   k_full.cuh   full pair measures (Riesz, Green, log)
//   k_near.cuh   near-field shell, chart-grid sorts and gather
//   k_relax.cuh  BB step, median, move+fold, row summaries
//   k_cover.cuh  covering radius: per-source Delaunay stars
#include <cuda_runtime.h>

#include "qvm_shared.h"

#include "k_pairs.cuh"
#include "k_full.cuh"
#include "k_near.cuh"
#include "k_relax.cuh"
#include "k_cover.cuh"

namespace zo {

thread_local LaunchProbe* t_probe = nullptr;

cudaError_t launch_relax_stats(Rows rows, const double4* prev_f, const double4* prev_d, int n, int fixed,
                               double* partials, RelaxDev* st, cudaStream_t s) {
  k_relax_stats<<<reduce_blocks(n), kRelaxBlock, 0, s>>>(rows, prev_f, prev_d, n, fixed, partials, st);
  probe_count();
  return cudaGetLastError();
}

cudaError_t launch_median(int prec, Rows rows, int n, RelaxDev* st, unsigned int* hist, double alpha0, double radius,
                          int sms, cudaStream_t s) {
  const int blocks = max(1, min((n + 255) / 256, 2 * sms));
  if (prec == kFP64) {
    for (int r = 0; r < 8; ++r) k_median_round<true><<<blocks, 256, 0, s>>>(rows, n, r, st, hist, alpha0, radius);
    probe_count(8);
  } else {
    for (int r = 0; r < 4; ++r) k_median_round<false><<<blocks, 256, 0, s>>>(rows, n, r, st, hist, alpha0, radius);
    probe_count(4);
  }
  return cudaGetLastError();
}

cudaError_t launch_move_fold(float4* q32, double4* q64, int n, int gid, int prec, Rows rows, double4* prev_f,
                             double4* prev_d, RelaxDev* st, int fixed, double radius, double step_scale, cudaStream_t s) {
  k_move_fold<<<(n + 127) / 128, 128, 0, s>>>(q32, q64, n, gid, prec, rows, prev_f, prev_d, st, fixed, radius,
                                              step_scale);
  probe_count();
  return cudaGetLastError();
}

cudaError_t launch_row_summary(Rows rows, int n, double* partials, double* near_partials, int* near_rows,
                               RowSummary* out, cudaStream_t s, bool nearest_only) {
  k_row_summary<<<reduce_blocks(n), kRelaxBlock, 0, s>>>(rows, n, partials, near_partials, near_rows, out,
                                                          nearest_only ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_nearest_degrees(const double* nearest, int n, float* out, cudaStream_t s) {
  k_nearest_degrees<<<(n + 255) / 256, 256, 0, s>>>(nearest, n, out);
  return cudaGetLastError();
}

cudaError_t launch_refine_nearest(const float4* q32, int n, int gid, Rows rows, bool near_sites, const uint32_t* scode,
                                  const uint32_t* simg, int* neighbour, cudaStream_t s) {
  k_refine_nearest<<<(n + 255) / 256, 256, 0, s>>>(q32, n, gid, rows, near_sites ? 1 : 0, scode, simg, neighbour);
  return cudaGetLastError();
}

template <int NB, int NF>
static cudaError_t launch_cover_star(const CoverArgs& A, int count, int sms, cudaStream_t s) {
  const size_t smem = kCoverWarps * sizeof(CoverStar<NB, NF>);
  cudaError_t e = cudaFuncSetAttribute(k_cover_star<NB, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  // Warps loop over the sources: as many blocks as stay resident.
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cover_star<NB, NF>, kCoverWarps * 32, smem);
  if (e != cudaSuccess) return e;
  const int blocks = std::max(1, std::min((count + kCoverWarps - 1) / kCoverWarps, std::max(1, per_sm) * sms));
  k_cover_star<NB, NF><<<blocks, kCoverWarps * 32, smem, s>>>(A);
  probe_count();
  return cudaGetLastError();
}

cudaError_t launch_cover(const CoverArgs& A, int sms, cudaStream_t s, int width) {
  const int count = A.list ? A.count : A.n;
  if (count <= 0) return cudaSuccess;
  if (A.n >= (1 << 24)) return cudaErrorInvalidValue;  // point keys hold the source in 24 bits
  switch (width) {
    case 0: return launch_cover_star<kCoverMaxNarrow, kCoverFacetsNarrow>(A, count, sms, s);
    case 1: return launch_cover_star<kCoverMaxMiddle, kCoverFacetsMiddle>(A, count, sms, s);
    default: return launch_cover_star<kCoverMax, kCoverFacets>(A, count, sms, s);
  }
}

// FP32 FMA throughput probe: 8 independent FMA chains per thread (latency hidden by ILP and
// occupancy), the result stored so nothing is eliminated. 16 flops per thread per iteration.
// PACKED: the chains are float2 pairs advanced by one f32x2 FMA each (32 flops per thread
// per iteration), to see whether packed FMAs raise the FP32 rate or only save issue slots.
template <bool PACKED>
__global__ void __launch_bounds__(256) k_fma_probe(float* out, int iterations, float seed) {
  float2 a[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) a[c] = make_float2(seed + (float)(threadIdx.x + c), seed - (float)c);
  const float m = 0.999999f, b = 1e-7f;
  for (int it = 0; it < iterations; ++it) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (PACKED) a[c] = fma2(a[c], splat(m), splat(b));
      else a[c].x = fmaf(a[c].x, m, b);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < 8; ++c) s += a[c].x + (PACKED ? a[c].y : 0.f);
  if (s == 12345.678f) out[blockIdx.x] = s;
}

template <bool PACKED>
static cudaError_t time_fma_probe(int sms, float* out, double* tflops) {
  const int blocks = sms * 8, iterations = 1 << 16;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  k_fma_probe<PACKED><<<blocks, 256>>>(out, 1024, 1.0f);
  cudaEventRecord(a);
  for (int r = 0; r < 4; ++r) k_fma_probe<PACKED><<<blocks, 256>>>(out, iterations, 1.0f + r);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *tflops = 4.0 * blocks * 256.0 * iterations * (PACKED ? 32.0 : 16.0) / (ms * 1e-3) / 1e12;
  return cudaGetLastError();
}

cudaError_t measure_fp32_peak(int sms, double* tflops, double* packed_tflops) {
  float* out = nullptr;
  cudaError_t e = cudaMalloc(&out, sizeof(float) * sms * 64);
  if (e) return e;
  e = time_fma_probe<false>(sms, out, tflops);
  if (!e && packed_tflops) e = time_fma_probe<true>(sms, out, packed_tflops);
  cudaFree(out);
  return e;
}

cudaError_t launch_neighbour_index(Rows rows, int n, bool near_sites, const uint32_t* scode, int* neighbour,
                                   cudaStream_t s) {
  k_neighbour_index<<<(n + 255) / 256, 256, 0, s>>>(rows, n, near_sites ? 1 : 0, scode, neighbour);
  return cudaGetLastError();
}

}  // namespace zo
