// Covering optimisation (src/engine.zig:407-534, optimizeCovering and setKicks; the Python
// surface is api.py optimize_covering): steps that lower the covering radius and keep the
// best sample seen. This engine's step is its own: every orientation that touches one of the
// largest empty caps (within a band of the largest) moves toward the centre of its largest
// cap by the trust angle; the whole sample is measured again (the GPU stars of cover.cpp) and
// the step is kept only if the covering radius went down, else undone with the trust angle
// halved. After `patience` steps without a relative gain of `progress` the best sample is
// restored and every orientation kicked by a random rotation (RMS angle `size` times the best
// radius), the trust angle restarting at `trust` times it. A separation floor rejects steps
// that bring the closest pair below it (pairs already nearer are never brought nearer).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "engine.h"

namespace zo {
namespace {
constexpr double kPiO = 3.14159265358979323846;
}  // namespace

void Engine::set_kicks(uint32_t patience, double progress, double size, double trust) {
  if (patience < 1 || patience > 1000000) throw Failure("InvalidKickPatience");
  if (!(progress >= 0 && progress < 1)) throw Failure("InvalidKickProgress");
  if (!(size >= 0 && size <= 1)) throw Failure("InvalidKickSize");
  if (!(trust > 0 && trust <= 1)) throw Failure("InvalidKickTrust");
  kicks_ = KickSettings{patience, progress, size, trust};
}

// New positions for the same sample (an optimiser step): folded into the zone on the GPU,
// mirrored on the host; the relaxation history and the measures are dropped, the iteration
// and the generator kept.
void Engine::move_to(const std::vector<float>& values) {
  ZO_CUDA(cudaMemcpyAsync(q32_.as<float4>(), values.data(), (size_t)n_ * 16, cudaMemcpyHostToDevice, stream_));
  ZO_CUDA(launch_fold(q32_.as<float4>(), q64(), (int)n_, group_, prec_, true, stream_));
  fetch();
  if (fixed_index_) {
    const uint32_t i = *fixed_index_;
    const float one[4] = {1.f, 0.f, 0.f, 0.f};
    const double one64[4] = {1, 0, 0, 0};
    std::memcpy(&host_[(size_t)i * 4], one, 16);
    ZO_CUDA(cudaMemcpyAsync(q32() + i, one, 16, cudaMemcpyHostToDevice, stream_));
    ZO_CUDA(cudaMemcpyAsync(q64() + i, one64, 32, cudaMemcpyHostToDevice, stream_));
  }
  relax_state_.reset();
  spacing_state_.reset();
  measures_.reset();
  full_measures_ = false;
  point_separation_iteration_.reset();
}

// The smallest SO(3) angle between two orbit points of the current sample (a spacing pass).
double Engine::least_separation() {
  spacing();
  const double sep = measures_ ? measures_->separation_deg : NAN;
  measures_.reset();
  return sep;
}

void Engine::optimize_covering(uint32_t steps, uint32_t mode, bool finish, double floor_deg) {
  if (n_ < 4) throw Failure("TooFewOrientations");
  if ((mode & 3u) > 1 || (mode & ~0xff001fu) != 0) throw Failure("InvalidCoveringMode");
  if (!(floor_deg >= 0 && floor_deg < 180)) throw Failure("InvalidSeparationFloor");
  if (fix_identity_ && !fixed_index_) throw Failure("IdentityMissingEnableAddIdentity");
  ZO_CUDA(cudaSetDevice(device_));
  cancelled_.store(false);
  const bool face = (mode & 1u) != 0;
  const double band = face ? 0.02 : 0.005;  // caps within this fraction of the largest move
  CoverOptimizer& o = opt_;
  if (!o.active || o.key != sample_key()) {
    // A new run, or the sample moved since the last batch.
    cover();
    o = CoverOptimizer{};
    o.active = true;
    o.best = o.current = host_;
    o.best_radius = o.current_radius = o.gain_ref = cover_->radius_deg;
    o.trust = 0.05 * cover_->radius_deg * kPiO / 360.0;
    o.separation = floor_deg > 0 ? least_separation() : 0.0;
    o.rng.seed(0x5eed5eedull ^ n_);
  }
  const int n = (int)n_;
  std::vector<double4> centre(n);
  for (uint32_t s = 0; s < steps; ++s) {
    if (cancelled_.load()) break;
    // The current sample is loaded and measured: its orientations on the largest caps.
    cover();  // cached when the sample is the one last measured
    ZO_CUDA(cudaMemcpyAsync(centre.data(), cover_centre_.as<double4>(), (size_t)n * sizeof(double4),
                            cudaMemcpyDeviceToHost, stream_));
    ZO_CUDA(cudaStreamSynchronize(stream_));
    const double top = o.current_radius;
    std::vector<float> candidate(o.current);
    uint32_t jobs = 0;
    for (int i = 0; i < n; ++i) {
      if (fixed_index_ && (uint32_t)i == *fixed_index_) continue;
      if (point_covering_.data()[i] < top * (1.0 - band)) continue;
      double x[4];
      orbit_point((uint32_t)i << 8, x);
      const double c[4] = {centre[i].x, centre[i].y, centre[i].z, centre[i].w};
      const double xc = x[0] * c[0] + x[1] * c[1] + x[2] * c[2] + x[3] * c[3];
      double u[4], un = 0;
      for (int k = 0; k < 4; ++k) {
        u[k] = c[k] - xc * x[k];
        un += u[k] * u[k];
      }
      if (!(un > 1e-30)) continue;
      un = std::sqrt(un);
      const double ct = std::cos(o.trust), st = std::sin(o.trust);
      for (int k = 0; k < 4; ++k) candidate[(size_t)i * 4 + k] = (float)(ct * x[k] + st * u[k] / un);
      ++jobs;
    }
    o.jobs = jobs;
    ++o.steps;
    ++o.full_steps;
    bool accepted = false;
    if (jobs > 0) {
      set_covering_aside();  // the current sample's covering, back unchanged if the step is undone
      move_to(candidate);
      cover();
      const double radius = cover_->radius_deg;
      bool floor_ok = true;
      double sep = o.separation;
      if (floor_deg > 0) {
        sep = least_separation();
        floor_ok = sep >= floor_deg || sep >= o.separation;
      }
      if (radius < top * (1.0 - 1e-12) && floor_ok) {
        accepted = true;
        o.current = host_;
        o.current_radius = radius;
        o.separation = sep;
        ++o.improved;
        o.trust = std::min(o.trust * 1.25, 0.25 * radius * kPiO / 360.0);
        if (radius < o.best_radius) {
          o.best = host_;
          o.best_radius = radius;
        }
      }
    }
    if (!accepted) {
      ++o.skipped;
      o.trust *= 0.5;
      if (jobs > 0) {
        move_to(o.current);
        restore_covering();
      }
    }
    // Plateau: restore the best sample and kick every orientation.
    if (o.current_radius < o.gain_ref * (1.0 - kicks_.progress)) {
      o.gain_ref = o.current_radius;
      o.since_gain = 0;
    } else if (++o.since_gain >= kicks_.patience) {
      std::normal_distribution<double> gauss(0.0, 1.0);
      // A rotation by angle a (SO(3)) about a random axis is the unit quaternion
      // (cos a/2, sin a/2 axis); its components are drawn so the angle's RMS is
      // size x best radius.
      const double rms = kicks_.size * o.best_radius * kPiO / 180.0;
      std::vector<float> kicked(o.best);
      for (int i = 0; i < n; ++i) {
        if (fixed_index_ && (uint32_t)i == *fixed_index_) continue;
        double axis[3] = {gauss(o.rng), gauss(o.rng), gauss(o.rng)};
        const double a = rms / std::sqrt(3.0) * std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
        const double norm = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
        if (!(norm > 0)) continue;
        const double r[4] = {std::cos(0.5 * a), std::sin(0.5 * a) * axis[0] / norm, std::sin(0.5 * a) * axis[1] / norm,
                             std::sin(0.5 * a) * axis[2] / norm};
        const float* p = &o.best[(size_t)i * 4];
        const double q[4] = {p[0], p[1], p[2], p[3]};
        const double w = r[0] * q[0] - r[1] * q[1] - r[2] * q[2] - r[3] * q[3];
        const double x = r[0] * q[1] + q[0] * r[1] + r[2] * q[3] - r[3] * q[2];
        const double y = r[0] * q[2] + q[0] * r[2] + r[3] * q[1] - r[1] * q[3];
        const double z = r[0] * q[3] + q[0] * r[3] + r[1] * q[2] - r[2] * q[1];
        kicked[(size_t)i * 4 + 0] = (float)w;
        kicked[(size_t)i * 4 + 1] = (float)x;
        kicked[(size_t)i * 4 + 2] = (float)y;
        kicked[(size_t)i * 4 + 3] = (float)z;
      }
      move_to(kicked);
      cover();
      o.current = host_;
      o.current_radius = o.gain_ref = cover_->radius_deg;
      o.separation = floor_deg > 0 ? least_separation() : 0.0;
      o.trust = kicks_.trust * o.best_radius * kPiO / 360.0;
      o.since_gain = 0;
      ++o.kicks;
    }
  }
  if (finish) {
    // The best sample, measured in full.
    if (o.current != o.best) move_to(o.best);
    o.current = o.best;
    o.current_radius = o.best_radius;
    cover();
  }
  measures_.reset();
  o.key = sample_key();
}

}  // namespace zo
