// zo_pair_rows_noalloc: the all-pairs force pass for callers that cannot allocate device
// memory.
//
// Who needs it: code that is handed device buffers but may not call cudaMalloc itself -
// a host framework that owns every allocation through its own pool, a caller that has
// pre-reserved its memory and must not grow it, or a latency-critical thread that cannot
// risk the synchronisation an allocation can cause. The engine's zo_* entry points size
// their buffers with cudaMalloc; this one uses only the caller's input and output and a
// fixed scratch array compiled into the library.
//
// The scratch is the force pass's partial rows (one per chunk of image tiles and source),
// summed afterwards in chunk order. It lives in g_pair_scratch below: 65,536 partial rows,
// 3 MiB, held by every GPU that loads the library until the process exits. Sizes that would
// need more are refused (n above 65,536), and the work is split into fewer chunks when the
// scratch cannot hold the usual split, so results match the engine's force pass to rounding.
//
// Every call shares the array: calls that overlap on the GPU (concurrent streams, or
// another thread's call) race on it and must be serialised by the caller. Each call writes
// every partial row it later reads, so no contents carry over between calls.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "kernels.h"
#include "zxtalori.h"

namespace {

constexpr int kScratchRows = 1 << 16;
constexpr size_t kScratchBytes = (size_t)kScratchRows * (sizeof(double4) + 2 * sizeof(double));

static __device__ __align__(256) unsigned char g_pair_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
bool g_ready[kMaxDevices] = {false};
unsigned char* g_scratch[kMaxDevices] = {nullptr};
int g_sms[kMaxDevices] = {0};

void put_error(char* error, size_t error_len, const char* message) {
  if (error && error_len) std::snprintf(error, error_len, "%s", message);
}

// Once per device, with that device current: the scratch array's device address (the
// array's name is only a host-side stand-in), the SM count, and the group tables in
// constant memory (through the engine's own once-per-device upload). No allocation.
int setup(int device, char* error, size_t error_len) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_ready[device]) return 0;
  void* ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_pair_scratch);
  if (e != cudaSuccess) {
    char msg[256];
    std::snprintf(msg, sizeof msg, "scratch address: %s", cudaGetErrorString(e));
    put_error(error, error_len, msg);
    return -3;
  }
  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = zo::ensure_device_tables(device);
  if (e != cudaSuccess) {
    char msg[256];
    std::snprintf(msg, sizeof msg, "device set-up: %s", cudaGetErrorString(e));
    put_error(error, error_len, msg);
    return -3;
  }
  g_scratch[device] = static_cast<unsigned char*>(ptr);
  g_sms[device] = sms;
  g_ready[device] = true;
  return 0;
}

}  // namespace

extern "C" int zo_pair_rows_noalloc(uint32_t group, const float* q_device, uint32_t n, double* rows_device,
                                    void* stream, char* error, size_t error_len) {
  if (group >= 11) {
    put_error(error, error_len, "unknown group (0-10)");
    return -1;
  }
  if (n == 0 || n > (uint32_t)kScratchRows) {
    put_error(error, error_len, "n must be 1..65536: the fixed scratch holds 65,536 partial rows");
    return -2;
  }
  if (!q_device || !rows_device || ((uintptr_t)q_device % 16) || ((uintptr_t)rows_device % 32)) {
    put_error(error, error_len, "q_device must be 16-byte and rows_device 32-byte aligned device pointers");
    return -1;
  }
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess || device < 0 || device >= kMaxDevices || device >= zo::kMaxTableDevices) {
    put_error(error, error_len, "no current CUDA device");
    return -3;
  }
  // An error left pending by the caller's earlier work would otherwise be reported (and
  // cleared) as this call's launch failure: refuse, and leave it pending for its owner.
  e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    char msg[256];
    std::snprintf(msg, sizeof msg, "a CUDA error is pending from earlier work on this thread: %s",
                  cudaGetErrorString(e));
    put_error(error, error_len, msg);
    return -3;
  }
  const int rc = setup(device, error, error_len);
  if (rc) return rc;
  // The engine's split of the image tiles, with no more chunks than the scratch holds.
  zo::PairsPlan pl = zo::plan_pairs((int)n, zo::host_group_order((int)group), 1.0, g_sms[device]);
  const int max_chunks = kScratchRows / (int)n;
  if (pl.chunks > max_chunks) {
    pl.tiles_per_chunk = (pl.total_tiles + max_chunks - 1) / max_chunks;
    pl.chunks = (pl.total_tiles + pl.tiles_per_chunk - 1) / pl.tiles_per_chunk;
  }
  unsigned char* base = g_scratch[device];
  const size_t rows_cap = (size_t)kScratchRows;
  zo::Rows partial{reinterpret_cast<double4*>(base), reinterpret_cast<double*>(base + rows_cap * sizeof(double4)),
                   reinterpret_cast<double*>(base + rows_cap * (sizeof(double4) + sizeof(double))), nullptr};
  zo::Rows out{reinterpret_cast<double4*>(rows_device), rows_device + 4 * (size_t)n, rows_device + 5 * (size_t)n,
               nullptr};
  e = zo::launch_pairs(zo::kFP32, false, reinterpret_cast<const float4*>(q_device), nullptr, (int)n, (int)group, pl,
                       partial, out, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    char msg[256];
    std::snprintf(msg, sizeof msg, "launch: %s", cudaGetErrorString(e));
    put_error(error, error_len, msg);
    return -3;
  }
  put_error(error, error_len, "");
  return 0;
}
