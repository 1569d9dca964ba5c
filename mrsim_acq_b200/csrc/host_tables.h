// host_tables.h — host-side tables of the 2D EPI path, bit-exact with the reference crate.
// These are small O(ny) / O(nx*ny) integer and f64 computations that decide WHICH samples exist
// and WHEN they are read; they run on the host in the product (as the reference's plan code
// does) and feed the device kernels.  Each function cites the reference item it restates.
#pragma once

#include <stdint.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/mrsim_acq.h"

namespace mrsim {

constexpr double kTau = 6.283185307179586;

// SplitMix64 + Box-Muller (`Rng`, kspace.rs:59-77).  Counter-based: draw k of a stream seeded s
// is mix(s + (k+1) * gamma), which the device noise kernel uses directly.
struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  static uint64_t mix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  uint64_t next_u64() {
    s += 0x9E3779B97F4A7C15ull;
    return mix(s);
  }
  double unit() { return ((double)(next_u64() >> 11) + 0.5) / (double)(1ull << 53); }
  double gauss() {
    double u1 = unit(), u2 = unit();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(kTau * u2);
  }
};

struct LineTimingTab {
  std::vector<double> t_ms, trf_ms, tread_ms;
  std::vector<int8_t> polarity;
};

mrsim_acquisition acquisition_default();
size_t pf_skipped_lines(size_t ny, const mrsim_acquisition& a);                  // kspace.rs:110
LineTimingTab line_timing(const mrsim_acquisition& a, size_t nx, size_t ny);     // kspace.rs:310
std::vector<uint8_t> sampling_mask(size_t nx, size_t ny, const mrsim_acquisition& a);  // :546
std::vector<int64_t> epi_order(const mrsim_acquisition& a, size_t nx, size_t ny);      // :353
void validate_acquisition_timing(const mrsim_acquisition& a, size_t nx, size_t ny);    // :411
double coil_sensitivity(size_t coil, size_t n, double x, double y, size_t nx, size_t ny);  // :226
double window_at(const mrsim_acquisition& a, double kx, double ky);              // kspace.rs:140
uint64_t echo_salt(uint64_t e);                                                  // kspace.rs:2130

// `PrepPhase::shot` (phase.rs:108-128): q_eff, dx, rot of one shot.
struct ShotParams {
  double q[3] = {0, 0, 0}, dx[3] = {0, 0, 0}, rot[3] = {0, 0, 0};
};
ShotParams prep_shot(const mrsim_phase_model& p, double magnitude, const double dir[3], size_t volume,
                     size_t slice_group, uint64_t seed);

constexpr uint64_t kSeedSaltGrappaCal = 0x47525043414Cull;  // kspace.rs:1652
constexpr double kGrappaLambda = 1e-3;                      // kspace.rs:1522

}  // namespace mrsim
