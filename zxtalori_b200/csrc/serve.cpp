// Continuous-batching relax + measure service on one GPU, in the library (zo_serve): requests
// arrive over time; the loop admits waiting requests in arrival order while their device
// memory fits the budget, keeps each admitted sample resident in its own engine (own CUDA
// stream, FP32 steps replayed from a captured graph) and advances every active sample by a
// chunk of steps whenever its stream is idle, so the kernels of all active samples overlap on
// the device. A request whose steps are done goes to a worker thread for its blocking part
// (closing force pass, measure(), engine freed) while the loop keeps feeding the others; its
// memory then goes to the next admission. Admission counts a resident sample at the bytes its
// engine reports once its workspace is sized (an estimate before that, and only one sample at
// a time is admitted on an estimate). A request's results do not depend on what else runs:
// every sample's kernels read only its own buffers and sum in a fixed order.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <future>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "zxtalori.h"

namespace zo {
namespace {

const uint32_t kOrders[11] = {2, 3, 4, 6, 4, 6, 8, 12, 12, 24, 60};

// Orbit points a source feels (the reference's count, src/engine.zig:905-907).
double neighbours(double count, double order, double delta) {
  return delta > 0 ? std::min(count * order, 0.94 * delta * delta * delta + 64) : count * order;
}

// Device memory a request holds while resident, generously: positions, rows and BB history
// about 450 B per source; a near field adds shell sites (about 80 B each, a few per source),
// partial rows of up to 64 slices and the chart grids.
double estimate_bytes(double count, uint32_t group, double delta, int sms) {
  const double order = kOrders[group];
  double total = 450 * count + (64 << 20);
  if (delta > 0) {
    const double slices = std::min(64.0, std::max(1.0, std::ceil(sms * 48.0 / std::max(1.0, count / 32))));
    total += count * 80 * std::min(2 * order, 10.0) + slices * count * 52 + (40 << 20);
  } else {
    total += 32.0 * 52 * count;
  }
  return total;
}

// The number after "key": in the engine's stats JSON (NaN when absent or null).
double json_number(const char* json, const char* key) {
  const std::string k = std::string("\"") + key + "\":";
  const char* at = std::strstr(json, k.c_str());
  if (!at) return NAN;
  at += k.size();
  if (std::strncmp(at, "null", 4) == 0) return NAN;
  return std::strtod(at, nullptr);
}

struct Active {
  zo_serve_request request;
  std::unique_ptr<Engine> engine;
  uint32_t remaining = 0;
  double admitted = 0, bytes = 0, per_step_s = 0;
  bool sized = false;
};

// The blocking part of a request, on a worker thread (the loop no longer touches its engine):
// the closing force pass, measure(), the numbers of the result; the engine is freed here.
zo_serve_result finish(Active a, bool measure, double t0_seconds) {
  zo_serve_result r{};
  r.id = a.request.id;
  r.arrival = a.request.arrival;
  r.admitted = a.admitted;
  r.neighbourhood = a.request.neighbourhood;
  r.count = a.request.count;
  r.order = kOrders[a.request.group];
  // This thread works on the engine's device from here on, the engine's release included.
  const cudaError_t device = cudaSetDevice(a.engine->device());
  try {
    ZO_CUDA(device);
    AllocScope scope(a.engine->stream());
    a.engine->relax_finish();
    if (measure) a.engine->measure();
    const char* json = a.engine->stats();
    r.iteration = (uint32_t)json_number(json, "iteration");
    r.energy = json_number(json, "quey_energy");
    r.separation_deg = json_number(json, "separation_deg");
    r.status = 0;
  } catch (const std::exception& x) {
    r.status = -1;
    std::snprintf(r.error, sizeof r.error, "%s", x.what());
  }
  {
    AllocScope scope(a.engine->stream());
    a.engine.reset();
  }
  r.finished = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count() -
               t0_seconds;
  return r;
}

struct Settings {
  double budget = 0;          // bytes; 0: 80 % of the device's free memory
  uint32_t max_active = 64;
  double chunk_seconds = 0.02;
  bool measure = true;
  int precision = kFP32;
  uint32_t workers = 4;
  double pair_rate = 2.5e11;  // pair evaluations per second, for chunk sizing only
};

void serve(const zo_serve_request* requests, uint32_t n, const Settings& set, zo_serve_result* out) {
  using clock = std::chrono::steady_clock;
  std::vector<zo_serve_request> pending(requests, requests + n);
  std::stable_sort(pending.begin(), pending.end(), [](const zo_serve_request& a, const zo_serve_request& b) {
    return a.arrival < b.arrival || (a.arrival == b.arrival && a.id < b.id);
  });
  for (const zo_serve_request& r : pending)
    if (r.group >= 11 || r.count < 2) throw Failure("InvalidRequest");
  // The engines' device ($ZXTALORI_DEVICE, else the current one), for the budget and sizes.
  int device = 0, sms = 148;
  const char* chosen = std::getenv("ZXTALORI_DEVICE");
  if (chosen && *chosen) device = std::atoi(chosen);
  else ZO_CUDA(cudaGetDevice(&device));
  ZO_CUDA(cudaSetDevice(device));
  double budget = set.budget;
  if (!(budget > 0)) {
    size_t free_bytes = 0, total_bytes = 0;
    ZO_CUDA(cudaMemGetInfo(&free_bytes, &total_bytes));
    budget = 0.8 * (double)free_bytes;
  }
  ZO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const double t0 = std::chrono::duration<double>(clock::now().time_since_epoch()).count();
  auto now = [&] { return std::chrono::duration<double>(clock::now().time_since_epoch()).count() - t0; };
  size_t next = 0, done = 0;
  std::vector<Active> stepping;
  std::deque<Active> waiting;  // done stepping, waiting for a worker
  struct Running {
    std::future<zo_serve_result> result;
    double bytes;
  };
  std::vector<Running> running;
  double held = 0;
  while (done < n) {
    bool progressed = false;
    const double t = now();
    // Admission (one sample at a time on an estimate: the next waits until the first chunk
    // has sized its workspace and its engine has reported its bytes).
    const size_t resident = stepping.size() + waiting.size() + running.size();
    if (next < n && pending[next].arrival <= t && resident < set.max_active &&
        std::all_of(stepping.begin(), stepping.end(), [](const Active& a) { return a.sized; })) {
      const zo_serve_request& r = pending[next];
      const double estimate = estimate_bytes(r.count, r.group, r.neighbourhood, sms);
      if (held + estimate <= budget || resident == 0) {
        Active a;
        a.request = r;
        a.engine = std::make_unique<Engine>();
        AllocScope scope(a.engine->stream());
        a.engine->set_precision(set.precision);
        a.engine->generate_random((int)r.group, r.count, r.seed);
        a.engine->set_neighbourhood(r.neighbourhood);
        a.remaining = r.steps;
        a.admitted = t;
        a.bytes = estimate;
        a.per_step_s = r.count * neighbours(r.count, kOrders[r.group], r.neighbourhood) / set.pair_rate;
        held += a.bytes;
        stepping.push_back(std::move(a));
        ++next;
        progressed = true;
      }
    }
    // Feed every idle sample a chunk of steps; a sample with none left goes to the workers.
    for (size_t k = 0; k < stepping.size();) {
      Active& a = stepping[k];
      AllocScope scope(a.engine->stream());
      if (!a.engine->idle()) {
        ++k;
        continue;
      }
      if (a.remaining > 0) {
        const uint32_t chunk = std::max<uint32_t>(
            1, std::min<uint32_t>(a.remaining, (uint32_t)(set.chunk_seconds / std::max(a.per_step_s, 1e-9))));
        a.engine->relax_async(chunk);
        a.remaining -= chunk;
        if (!a.sized) {  // the first chunk sized the workspace: count the engine's own bytes
          const double real = (double)a.engine->device_bytes();
          held += real - a.bytes;
          a.bytes = real;
          a.sized = true;
        }
        ++k;
      } else {
        waiting.push_back(std::move(a));
        stepping.erase(stepping.begin() + (ptrdiff_t)k);
      }
      progressed = true;
    }
    while (!waiting.empty() && running.size() < std::max<uint32_t>(1, set.workers)) {
      const double bytes = waiting.front().bytes;
      running.push_back({std::async(std::launch::async, finish, std::move(waiting.front()), set.measure, t0), bytes});
      waiting.pop_front();
      progressed = true;
    }
    for (size_t k = 0; k < running.size();) {
      if (running[k].result.wait_for(std::chrono::seconds(0)) != std::future_status::ready) {
        ++k;
        continue;
      }
      out[done++] = running[k].result.get();
      held -= running[k].bytes;
      running.erase(running.begin() + (ptrdiff_t)k);
      progressed = true;
    }
    if (!progressed) {
      // Nothing to do: wait for the next arrival when idle, else briefly for a stream.
      const double wait = (stepping.empty() && running.empty() && waiting.empty() && next < n)
                              ? std::min(0.05, std::max(0.0, pending[next].arrival - now()))
                              : 2e-4;
      std::this_thread::sleep_for(std::chrono::duration<double>(wait));
    }
  }
}

}  // namespace
}  // namespace zo

extern "C" int zo_serve(const zo_serve_request* requests, uint32_t n, const double* settings, uint32_t n_settings,
                        zo_serve_result* results, char* error, size_t error_len) {
  try {
    zo::Settings set;
    const double* v = settings;
    if (n_settings > 0 && v[0] > 0) set.budget = v[0];
    if (n_settings > 1 && v[1] >= 1) set.max_active = (uint32_t)v[1];
    if (n_settings > 2 && v[2] > 0) set.chunk_seconds = v[2];
    if (n_settings > 3) set.measure = v[3] != 0;
    if (n_settings > 4) set.precision = v[4] != 0 ? zo::kFP64 : zo::kFP32;
    if (n_settings > 5 && v[5] >= 1) set.workers = (uint32_t)v[5];
    if (n_settings > 6 && v[6] > 0) set.pair_rate = v[6];
    if (n > 0 && (!requests || !results)) throw zo::Failure("InvalidArguments");
    zo::serve(requests, n, set, results);
    return 0;
  } catch (const std::exception& x) {
    if (error && error_len) std::snprintf(error, error_len, "Serve failed: %s", x.what());
    return -1;
  }
}
