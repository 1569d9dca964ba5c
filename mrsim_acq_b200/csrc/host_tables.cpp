// host_tables.cpp — see host_tables.h.
#include "host_tables.h"

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "mrsim_internal.h"

namespace mrsim {

mrsim_acquisition acquisition_default() {  // `impl Default for Acquisition` kspace.rs:239-267
  mrsim_acquisition a;
  std::memset(&a, 0, sizeof a);
  a.t_line = 1.0;
  a.t_echo = 90.0;
  a.t_inhom = 50.0;
  a.signal_scale = 100.0;
  a.do_distortions = 1;
  a.do_relaxation = 1;
  a.partial_fourier = 1.0;
  a.pf_mode = MRSIM_PF_FIBERFOX;
  a.eddy_tau = 70.0;
  a.spike_amplitude = 1.0;
  a.window_kind = MRSIM_WINDOW_NONE;
  a.n_coils = 1;
  a.accel = 1;
  a.acs_lines = 24;
  a.echo = MRSIM_ECHO_SPIN;
  return a;
}

size_t pf_skipped_lines(size_t ny, const mrsim_acquisition& a) {
  if (a.partial_fourier < 1.0 && a.pf_mode == MRSIM_PF_SCANNER) {
    size_t keep = (size_t)std::round((double)ny * a.partial_fourier);
    return ny - std::min(keep, ny);
  }
  return 0;
}

namespace {
// `SingleShotEpi` readout.rs:23-69: snake trajectory starting at the maximum ky line unless
// reversed, odd lines read backwards.
struct Epi {
  size_t kx_max, ky_max;
  double t_line, t_echo;
  bool reverse;
  double dt() const { return t_line / (double)kx_max; }
  double half_read() const { return (double)(kx_max * ky_max) * dt() / 2.0; }
  void index(size_t tick, size_t& kx, size_t& ky) const {
    size_t x = tick % kx_max, y = tick / kx_max;
    if (!reverse) {
      y = ky_max - 1 - y;
      if (y % 2 == 1) x = kx_max - x - 1;
    } else if (y % 2 == 1) {
      x = kx_max - x - 1;
    }
    kx = x;
    ky = y;
  }
  double from_echo(size_t tick) const { return dt() * ((double)tick + 0.5) - half_read(); }
  double from_prep(size_t tick) const { return (double)tick * dt() + dt() / 2.0; }
  double from_rf(size_t tick) const { return t_echo + from_echo(tick); }
};
}  // namespace

LineTimingTab line_timing(const mrsim_acquisition& a, size_t nx, size_t ny) {
  Epi epi{nx, ny, a.t_line, a.t_echo, a.reverse_phase != 0};
  LineTimingTab lt;
  lt.t_ms.assign(ny, 0.0);
  lt.trf_ms.assign(ny, 0.0);
  lt.tread_ms.assign(ny, 0.0);
  lt.polarity.resize(ny);
  const size_t xs = nx / 2;
  for (size_t tick = 0; tick < nx * ny; ++tick) {
    size_t kx, ky;
    epi.index(tick, kx, ky);
    if (kx == xs) {
      lt.t_ms[ky] = epi.from_echo(tick);
      lt.trf_ms[ky] = epi.from_rf(tick);
      lt.tread_ms[ky] = epi.from_prep(tick);
    }
  }
  for (size_t k = 0; k < ny; ++k) lt.polarity[k] = (k % 2 == 1) ? -1 : 1;
  double offset = (double)pf_skipped_lines(ny, a) * a.t_line;
  if (offset > 0.0)
    for (double& v : lt.tread_ms) v -= offset;
  return lt;
}

std::vector<uint8_t> sampling_mask(size_t nx, size_t ny, const mrsim_acquisition& a) {
  const size_t ys = ny / 2;
  const size_t accel = (size_t)std::max<int64_t>(a.accel, 1);
  std::vector<uint8_t> m(nx * ny, 0);
  const size_t keep_n = (size_t)std::round((double)ny * a.partial_fourier);
  for (size_t kyi = 0; kyi < ny; ++kyi) {
    bool skip = false;
    if (a.partial_fourier < 1.0 && a.pf_mode == MRSIM_PF_SCANNER) {
      skip = a.reverse_phase ? (kyi < ny - keep_n) : (kyi >= keep_n);
    } else if (a.partial_fourier < 1.0 && a.pf_mode == MRSIM_PF_CONTIGUOUS) {
      skip = a.reverse_phase ? (kyi >= keep_n) : (kyi < ny - keep_n);
    } else if (a.partial_fourier < 1.0) {
      if (a.reverse_phase)
        skip = (double)kyi > std::ceil((double)ny * a.partial_fourier);
      else
        skip = (double)kyi < std::floor((double)ny * (1.0 - a.partial_fourier)) && (kyi > 0 || ny % 2 == 1);
    }
    if (skip) continue;
    if (!(accel <= 1 || kyi % accel == ys % accel)) continue;
    for (size_t kxi = 0; kxi < nx; ++kxi) m[kxi + nx * kyi] = 1;
  }
  return m;
}

std::vector<int64_t> epi_order(const mrsim_acquisition& a, size_t nx, size_t ny) {
  Epi epi{nx, ny, a.t_line, a.t_echo, a.reverse_phase != 0};
  std::vector<int64_t> order(ny);
  for (size_t line = 0; line < ny; ++line) {
    size_t kx, ky;
    epi.index(line * nx, kx, ky);
    order[line] = (int64_t)ky;
  }
  return order;
}

void validate_acquisition_timing(const mrsim_acquisition& a, size_t nx, size_t ny) {
  LineTimingTab lt = line_timing(a, nx, ny);
  auto mask = sampling_mask(nx, ny, a);
  double worst = INFINITY;
  for (size_t ky = 0; ky < ny; ++ky)
    if (mask[ky * nx] && lt.trf_ms[ky] < worst) worst = lt.trf_ms[ky];
  if (worst <= 0.0) {
    char buf[512];
    std::snprintf(buf, sizeof buf,
                  "trf = %.3f ms <= 0 on an acquired line: the readout starts before the excitation. Raise "
                  "t_echo above %.3f ms or shorten t_line. Partial Fourier helps only in Scanner mode (it "
                  "skips the first lines); the Fiberfox and Contiguous modes drop lines this trajectory reads "
                  "last.",
                  worst, a.t_echo - worst);
    fail(buf);
  }
}

double coil_sensitivity(size_t coil, size_t n, double x, double y, size_t nx, size_t ny) {
  if (n <= 1) return 1.0;
  const double cx = (double)nx / 2.0, cy = (double)ny / 2.0;
  const double r = 0.6 * (double)std::max(nx, ny);
  const double ang = kTau * (double)coil / (double)n;
  const double px = cx + r * std::cos(ang), py = cy + r * std::sin(ang);
  const double dx = x - px, dy = y - py;
  const double sigma = 0.9 * (double)std::max(nx, ny);
  return std::exp(-(dx * dx + dy * dy) / (2.0 * sigma * sigma)) + 0.15;
}

double window_at(const mrsim_acquisition& a, double kx, double ky) {
  const double r = 2.0 * std::sqrt(kx * kx + ky * ky);
  const double pi = kTau / 2.0;
  switch (a.window_kind) {
    case MRSIM_WINDOW_HANN:
      return r >= 1.0 ? 0.0 : 0.5 * (1.0 + std::cos(pi * r));
    case MRSIM_WINDOW_TUKEY: {
      const double al = std::min(std::max(a.window_a, 0.0), 1.0);
      if (r <= 1.0 - al) return 1.0;
      if (r >= 1.0) return 0.0;
      return 0.5 * (1.0 + std::cos(pi * (r - (1.0 - al)) / std::max(al, 1e-12)));
    }
    case MRSIM_WINDOW_FERMI:
      return 1.0 / (1.0 + std::exp((r - a.window_a) / std::max(a.window_b, 1e-12)));
    default:
      return 1.0;
  }
}

uint64_t echo_salt(uint64_t e) { return e * 0xD1B54A32D192ED03ull; }

ShotParams prep_shot(const mrsim_phase_model& p, double magnitude, const double dir[3], size_t volume,
                     size_t slice_group, uint64_t seed) {
  ShotParams s;
  const double n = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  if (magnitude <= 0.0 || n < 1e-12) return s;
  const double sc = p.c_q * std::sqrt(magnitude) / n;
  for (int i = 0; i < 3; ++i) s.q[i] = dir[i] * sc;
  Rng rng(seed ^ ((uint64_t)volume * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)slice_group * 0xBF58476D1CE4E5B9ull));
  for (int i = 0; i < 3; ++i) s.dx[i] = rng.gauss() * p.sigma_dx;
  for (int i = 0; i < 3; ++i) s.rot[i] = rng.gauss() * p.sigma_rot;
  return s;
}

}  // namespace mrsim
