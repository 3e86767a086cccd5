// Many samples relaxed together (zo_batch_relax): each BB step of every sample runs as one
// CUDA graph, and the near-field gathers of all the samples - about nine tenths of a step's
// device time - run in one persistent launch (per tile variant present, usually one or two)
// that takes warp tasks from a shared counter (launch_near32_batch), instead of one gather
// launch per sample.
//
// One step of a batch:
//   - every sample, on its own stream: the shell, chart grid, site sort and source order of
//     its near-field pass (or its whole force pass when it has no FP32 near-field gather:
//     all pairs, a dense cutoff);
//   - the batch's stream, after all of them: the gathers of every sample, largest first, in
//     one persistent launch per tile variant;
//   - every sample, on its own stream again: the slices' sums and the BB update (statistics,
//     exact median, move and fold).
// The first step runs these launches directly (they size the samples' workspaces); from the
// second on the step is captured once as a graph over all the streams and replayed, until
// a sample's workspace or settings change. A sample's gather tasks run the same warp
// function as its own gather launch, so every sample's result is the same alone and in the
// batch, bit for bit.
#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>
#include <vector>

#include "engine.h"
#include "zxtalori.h"

namespace zo {
namespace {

class BatchRun {
 public:
  BatchRun(std::vector<Engine*> engines) : engines_(std::move(engines)) {
    device_ = engines_.front()->device();
    ZO_CUDA(cudaSetDevice(device_));
    ZO_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    AllocScope scope(stream_);  // the batch's buffers come from the pool, ordered on its stream
    ZO_CUDA(cudaEventCreateWithFlags(&start_, cudaEventDisableTiming));
    ZO_CUDA(cudaEventCreateWithFlags(&gathered_, cudaEventDisableTiming));
    const size_t k = engines_.size();
    structured_.resize(k);
    done_.resize(k);
    for (size_t i = 0; i < k; ++i) {
      ZO_CUDA(cudaEventCreateWithFlags(&structured_[i], cudaEventDisableTiming));
      ZO_CUDA(cudaEventCreateWithFlags(&done_[i], cudaEventDisableTiming));
    }
    had_.assign(k, false);
    tasks_.ensure(k * sizeof(NearTask));
    prefix_.ensure(k * sizeof(uint32_t));
    counter_.ensure(sizeof(uint32_t));
    host_tasks_.resize(k);
    host_prefix_.resize(k);
  }
  BatchRun(const BatchRun&) = delete;
  BatchRun& operator=(const BatchRun&) = delete;
  ~BatchRun() {
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (graph_) cudaGraphExecDestroy(graph_);
    for (cudaEvent_t e : structured_) cudaEventDestroy(e);
    for (cudaEvent_t e : done_) cudaEventDestroy(e);
    if (start_) cudaEventDestroy(start_);
    if (gathered_) cudaEventDestroy(gathered_);
    tasks_.release();
    prefix_.release();
    counter_.release();
    if (stream_) cudaStreamDestroy(stream_);
  }

  // One BB step of every sample.
  void step() {
    ZO_CUDA(cudaSetDevice(device_));
    const bool ready = std::all_of(engines_.begin(), engines_.end(), [](Engine* e) { return e->batch_ready(); });
    if (!ready || !graph_ || key_ != key()) {
      // Recording rewrites the staged tasks, which an earlier step's copies may still read.
      ZO_CUDA(cudaStreamSynchronize(stream_));
      if (!ready) {
        drop_graph();
        record();  // direct launches; they size the workspaces
      } else {
        capture();
      }
    }
    if (ready) ZO_CUDA(cudaGraphLaunch(graph_, stream_));
    for (Engine* e : engines_) e->batch_stepped();
  }

  // Waits for the batch's own stream (every engine stream has joined it).
  void sync() { ZO_CUDA(cudaStreamSynchronize(stream_)); }

 private:
  uint64_t key() const {
    uint64_t k = engines_.size();
    for (Engine* e : engines_) k = k * 1000003ull + e->batch_key();
    return k;
  }

  void drop_graph() {
    if (graph_) cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }

  void capture() {
    drop_graph();
    cudaGraph_t graph = nullptr;
    ZO_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    try {
      record();
    } catch (...) {
      cudaStreamEndCapture(stream_, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    ZO_CUDA(cudaStreamEndCapture(stream_, &graph));
    const cudaError_t e = cudaGraphInstantiate(&graph_, graph, 0);
    cudaGraphDestroy(graph);
    ZO_CUDA(e);
    key_ = key();
  }

  // The launches of one step, on the batch's stream and the engines' streams.
  void record() {
    const size_t k = engines_.size();
    ZO_CUDA(cudaEventRecord(start_, stream_));
    std::vector<NearTask> tasks(k);
    for (size_t i = 0; i < k; ++i) {
      Engine* e = engines_[i];
      AllocScope scope(e->stream());
      ZO_CUDA(cudaStreamWaitEvent(e->stream(), start_, 0));
      had_[i] = e->batch_structure(&tasks[i]);
      ZO_CUDA(cudaEventRecord(structured_[i], e->stream()));
      ZO_CUDA(cudaStreamWaitEvent(stream_, structured_[i], 0));
    }
    // The gathers: one persistent launch per tile variant present (a batch has one or a
    // few), each over its samples largest first (the last warp tasks to start are the
    // small ones). Tasks and first-task offsets are staged variant by variant.
    std::vector<size_t> order;
    for (size_t i = 0; i < k; ++i)
      if (had_[i]) order.push_back(i);
    auto work = [&](size_t i) { return (uint64_t)tasks[i].warps * (uint64_t)tasks[i].slices; };
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
      const int va = near_variant(tasks[a]), vb = near_variant(tasks[b]);
      return va != vb ? va < vb : work(a) > work(b);
    });
    struct Segment {
      int variant;
      size_t first, count;
      uint32_t total;
    };
    std::vector<Segment> segments;
    for (size_t j = 0; j < order.size(); ++j) {
      const int v = near_variant(tasks[order[j]]);
      if (segments.empty() || segments.back().variant != v) segments.push_back(Segment{v, j, 0, 0});
      Segment& g = segments.back();
      host_tasks_.data()[j] = tasks[order[j]];
      host_prefix_.data()[j] = g.total;
      g.total += (uint32_t)work(order[j]);
      ++g.count;
    }
    if (!order.empty()) {
      ZO_CUDA(cudaMemcpyAsync(tasks_.as<NearTask>(), host_tasks_.data(), order.size() * sizeof(NearTask),
                              cudaMemcpyHostToDevice, stream_));
      ZO_CUDA(cudaMemcpyAsync(prefix_.as<uint32_t>(), host_prefix_.data(), order.size() * sizeof(uint32_t),
                              cudaMemcpyHostToDevice, stream_));
      for (const Segment& g : segments)
        ZO_CUDA(launch_near32_batch(tasks_.as<NearTask>() + g.first, prefix_.as<uint32_t>() + g.first, (int)g.count,
                                    g.total, counter_.as<uint32_t>(), g.variant, engines_.front()->sms(), stream_));
    }
    ZO_CUDA(cudaEventRecord(gathered_, stream_));
    for (size_t i = 0; i < k; ++i) {
      Engine* e = engines_[i];
      AllocScope scope(e->stream());
      ZO_CUDA(cudaStreamWaitEvent(e->stream(), gathered_, 0));
      e->batch_finish(had_[i]);
      ZO_CUDA(cudaEventRecord(done_[i], e->stream()));
      ZO_CUDA(cudaStreamWaitEvent(stream_, done_[i], 0));
    }
  }

  std::vector<Engine*> engines_;
  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t start_ = nullptr, gathered_ = nullptr;
  std::vector<cudaEvent_t> structured_, done_;
  std::vector<bool> had_;
  // Device copies of the tasks (read by the shared gather) and their host staging, pinned
  // so a captured copy reads them at replay; fixed while the graph is.
  DeviceBuffer tasks_, prefix_, counter_;
  PinnedArray<NearTask> host_tasks_;
  PinnedArray<uint32_t> host_prefix_;
  cudaGraphExec_t graph_ = nullptr;
  uint64_t key_ = 0;
};

// Runs f on an engine as an ABI call would (its allocations ordered on its stream); 0 or -1
// with the message in its error buffer.
template <class F>
int engine_call(Engine* e, F&& f) {
  try {
    AllocScope scope(e->stream());
    f(*e);
    return 0;
  } catch (const std::exception& x) {
    std::snprintf(e->err, sizeof e->err, "Relaxation failed: %s", x.what());
    return -1;
  }
}

}  // namespace
}  // namespace zo

extern "C" int zo_batch_relax(void* const* handles, uint32_t count, uint32_t steps, int32_t* status) {
  using zo::Engine;
  std::vector<Engine*> engines(count);
  for (uint32_t k = 0; k < count; ++k) {
    engines[k] = static_cast<Engine*>(handles[k]);
    status[k] = 0;
  }
  // FP32 engines with graphs on share batches, one per device; the others (the plain FP64
  // method, graphs off) step one launch at a time on their own streams.
  std::map<int, std::vector<uint32_t>> by_device;
  std::vector<uint32_t> alone;
  for (uint32_t k = 0; k < count; ++k) {
    status[k] = zo::engine_call(engines[k], [](Engine& e) { e.batch_begin(); });
    if (status[k] != 0) continue;
    if (engines[k]->precision() == zo::kFP32 && engines[k]->graphs_enabled()) by_device[engines[k]->device()].push_back(k);
    else alone.push_back(k);
  }
  std::vector<std::unique_ptr<zo::BatchRun>> runs;
  std::vector<std::vector<uint32_t>> members;
  for (auto& [device, ks] : by_device) {
    std::vector<Engine*> es;
    for (uint32_t k : ks) es.push_back(engines[k]);
    try {
      runs.push_back(std::make_unique<zo::BatchRun>(es));
      members.push_back(ks);
    } catch (const std::exception& x) {
      for (uint32_t k : ks) {
        std::snprintf(engines[k]->err, sizeof engines[k]->err, "Relaxation failed: %s", x.what());
        status[k] = -1;
      }
    }
  }
  for (uint32_t s = 0; s < steps; ++s) {
    for (size_t r = 0; r < runs.size(); ++r) {
      if (!runs[r]) continue;
      try {
        runs[r]->step();
      } catch (const std::exception& x) {
        for (uint32_t k : members[r]) {
          std::snprintf(engines[k]->err, sizeof engines[k]->err, "Relaxation failed: %s", x.what());
          status[k] = -1;
        }
        runs[r].reset();
      }
    }
    for (uint32_t k : alone)
      if (status[k] == 0) status[k] = zo::engine_call(engines[k], [](Engine& e) { e.relax_async(1); });
  }
  for (auto& run : runs)
    if (run) run->sync();
  runs.clear();
  // Every closing pass is enqueued before any is waited for.
  for (uint32_t k = 0; k < count; ++k)
    if (status[k] == 0) status[k] = zo::engine_call(engines[k], [](Engine& e) { e.finish_async(); });
  int failures = 0;
  for (uint32_t k = 0; k < count; ++k) {
    if (status[k] == 0) status[k] = zo::engine_call(engines[k], [](Engine& e) { e.finish_collect(); });
    failures += status[k] != 0;
  }
  return failures;
}
