// Memory that outlives engines: the per-device stream-ordered pool behind DeviceBuffer and
// a cache of pinned host blocks. Samples come and go (a server creates one per request,
// the Python API one per Grid); with plain cudaMalloc/cudaFree and cudaMallocHost/
// cudaFreeHost each of them paid milliseconds of allocation and a device-wide
// synchronisation that also stalled every other engine's stream.
#include <cstdint>
#include <map>
#include <mutex>

#include "engine.h"

namespace zo {
namespace {

thread_local cudaStream_t t_stream = nullptr;

constexpr int kMaxDevices = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[kMaxDevices] = {};

// The device's pool: device memory, kept when freed (release threshold: unlimited), reused
// by any stream once the free has completed on its own stream, never by making one
// stream wait for another.
cudaMemPool_t device_pool(int device) {
  if (device < 0 || device >= kMaxDevices) throw Failure("InvalidDevice");
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  if (!g_pools[device]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    ZO_CUDA(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = UINT64_MAX;
    ZO_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    int no = 0;
    ZO_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no));
    g_pools[device] = pool;
  }
  return g_pools[device];
}

constexpr size_t kPinnedKeep = size_t(512) << 20;  // cached pinned bytes at most
std::mutex g_pinned_mutex;
std::multimap<size_t, void*> g_pinned_free;  // cached blocks by size
std::map<void*, size_t> g_pinned_size;       // every live or cached block's size
size_t g_pinned_cached = 0;

}  // namespace

cudaStream_t alloc_stream() { return t_stream; }

AllocScope::AllocScope(cudaStream_t s) : prev_(t_stream) { t_stream = s; }
AllocScope::~AllocScope() { t_stream = prev_; }

void* device_pool_alloc(size_t bytes, cudaStream_t s) {
  int device = 0;
  ZO_CUDA(cudaStreamGetDevice(s, &device));
  cudaMemPool_t pool = device_pool(device);
  cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
  ZO_CUDA(cudaStreamIsCapturing(s, &capture));
  if (capture != cudaStreamCaptureStatusNone) throw Failure("AllocationDuringCapture");
  void* p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, s);
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    // Give the pool's idle blocks back to the device and try once more.
    ZO_CUDA(cudaDeviceSynchronize());
    ZO_CUDA(cudaMemPoolTrimTo(pool, 0));
    e = cudaMallocFromPoolAsync(&p, bytes, pool, s);
  }
  ZO_CUDA(e);
  return p;
}

void* pinned_alloc(size_t bytes) {
  const size_t want = (std::max<size_t>(bytes, 1) + 4095) & ~size_t(4095);
  {
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    // A cached block of at least the size asked and at most twice it.
    auto it = g_pinned_free.lower_bound(want);
    if (it != g_pinned_free.end() && it->first <= 2 * want) {
      void* p = it->second;
      g_pinned_cached -= it->first;
      g_pinned_free.erase(it);
      return p;
    }
  }
  void* p = nullptr;
  ZO_CUDA(cudaMallocHost(&p, want));
  std::lock_guard<std::mutex> lock(g_pinned_mutex);
  g_pinned_size[p] = want;
  return p;
}

void pinned_free(void* p) {
  if (!p) return;
  size_t size = 0;
  {
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    auto it = g_pinned_size.find(p);
    if (it == g_pinned_size.end()) return;
    size = it->second;
    if (g_pinned_cached + size <= kPinnedKeep) {
      g_pinned_free.emplace(size, p);
      g_pinned_cached += size;
      return;
    }
    g_pinned_size.erase(it);
  }
  cudaFreeHost(p);
}

}  // namespace zo
