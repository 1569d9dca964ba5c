// mrsim_oracle.cpp — TEST INFRASTRUCTURE ONLY.  A CPU FP64 restatement of the reference crate's
// 2D EPI k-space path and of its stack-of-spirals pieces (the 2D NUFFT pair, the exact and
// time-segmented spiral forwards) — Rust `mrsim-acq`, which cannot be compiled in this image: no
// Rust toolchain.  It is the parity checker for the CUDA library and the timed CPU baseline.  Only
// `tests/`, `__graft_entry__.smoke()` and `bench.py`'s CPU-baseline / reference arm may load it;
// the product library never links or calls it.
//
// Pinning: `oracle_golden_*` regenerates the reference's golden record
// (tests/golden_baseline.rs:28-126) and the tests compare it bit for bit with the reference's
// committed fixtures (tests/fixtures/p4_baseline/default/*.bin, copied to tests/golden/).
//
// Build rule: -O2 -ffp-contract=off -fno-fast-math, glibc libm — Rust never fuses multiply-adds
// and calls the platform libm for sin/cos/exp/ln, so every expression below keeps the reference's
// operation order.  Each function cites the reference file:line it restates.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <stdexcept>
#include <atomic>
#include <mutex>
#include <thread>
#include <functional>
#include <map>
#include <tuple>

#include "../include/mrsim_acq.h"

namespace {

constexpr double TAU = 6.283185307179586;  // std::f64::consts::TAU
constexpr double PI = 3.141592653589793;

// ---- complex helper: `C` kspace.rs:29-55 ----
struct Cx {
  double re, im;
};
inline Cx cadd(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
inline Cx cmul(Cx a, Cx o) { return {a.re * o.re - a.im * o.im, a.re * o.im + a.im * o.re}; }
inline Cx cscale(Cx a, double s) { return {a.re * s, a.im * s}; }
inline double cabs_(Cx a) { return std::sqrt(a.re * a.re + a.im * a.im); }
inline Cx ccis(double th) { return {std::cos(th), std::sin(th)}; }
const Cx CZERO = {0.0, 0.0};

// ---- `Rng` kspace.rs:59-77 (SplitMix64 + Box-Muller) ----
struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next_u64() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double unit() { return ((double)(next_u64() >> 11) + 0.5) / (double)(1ull << 53); }
  double gauss() {
    double u1 = unit();
    double u2 = unit();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(TAU * u2);
  }
};

struct Fail : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// Dynamic-schedule parallel loop over [0, n) on `threads` std::threads (the reference's rayon
// `par` feature parallelises the same loops; results do not depend on the thread count).
void parallel_for(size_t n, int threads, const std::function<void(size_t)>& body) {
  if (threads <= 1 || n <= 1) {
    for (size_t i = 0; i < n; ++i) body(i);
    return;
  }
  std::atomic<size_t> next{0};
  std::mutex mu;
  std::string err;
  auto worker = [&] {
    for (;;) {
      size_t i = next.fetch_add(1);
      if (i >= n) return;
      try {
        body(i);
      } catch (std::exception& e) {
        std::lock_guard<std::mutex> lk(mu);
        err = e.what();
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < threads && (size_t)t < n; ++t) pool.emplace_back(worker);
  for (auto& t : pool) t.join();
  if (!err.empty()) throw Fail(err);
}

// ---- `SingleShotEpi` readout.rs:23-69 ----
struct Epi {
  size_t kx_max, ky_max;
  double t_line, t_echo;
  bool reverse_phase;
  double dt() const { return t_line / (double)kx_max; }
  double half_read_time() const { return (double)(kx_max * ky_max) * dt() / 2.0; }
  void kspace_index(size_t tick, size_t& kx, size_t& ky) const {
    size_t x = tick % kx_max;
    size_t y = tick / kx_max;
    if (!reverse_phase) {
      y = ky_max - 1 - y;
      if (y % 2 == 1) x = kx_max - x - 1;
    } else if (y % 2 == 1) {
      x = kx_max - x - 1;
    }
    kx = x;
    ky = y;
  }
  double time_from_max_echo(size_t tick) const { return dt() * ((double)tick + 0.5) - half_read_time(); }
  double time_from_prep_gradient(size_t tick) const { return (double)tick * dt() + dt() / 2.0; }
  double time_from_rf(size_t tick) const { return t_echo + time_from_max_echo(tick); }
};

// ---- `pf_skipped_lines` kspace.rs:110-116 ----
size_t pf_skipped_lines(size_t ny, const mrsim_acquisition& a) {
  if (a.partial_fourier < 1.0 && a.pf_mode == MRSIM_PF_SCANNER) {
    size_t keep = (size_t)std::round((double)ny * a.partial_fourier);
    return ny - std::min(keep, ny);
  }
  return 0;
}

// ---- `LineTiming` kspace.rs:271-325 ----
struct LineTiming {
  std::vector<double> t_ms, trf_ms, tread_ms;
  std::vector<int8_t> polarity;
};

LineTiming line_timing_for(const mrsim_acquisition& a, size_t nx, size_t ny) {
  Epi epi{nx, ny, a.t_line, a.t_echo, a.reverse_phase != 0};
  LineTiming lt;
  lt.t_ms.assign(ny, 0.0);
  lt.trf_ms.assign(ny, 0.0);
  lt.tread_ms.assign(ny, 0.0);
  size_t xs = nx / 2;
  for (size_t tick = 0; tick < nx * ny; ++tick) {
    size_t kx, ky;
    epi.kspace_index(tick, kx, ky);
    if (kx == xs) {
      lt.t_ms[ky] = epi.time_from_max_echo(tick);
      lt.trf_ms[ky] = epi.time_from_rf(tick);
      lt.tread_ms[ky] = epi.time_from_prep_gradient(tick);
    }
  }
  lt.polarity.resize(ny);
  for (size_t k = 0; k < ny; ++k) lt.polarity[k] = (k % 2 == 1) ? -1 : 1;
  double offset = (double)pf_skipped_lines(ny, a) * a.t_line;
  if (offset > 0.0)
    for (auto& v : lt.tread_ms) v -= offset;
  return lt;
}

// ---- `sampling_mask` kspace.rs:546-588 ----
std::vector<uint8_t> sampling_mask(size_t nx, size_t ny, const mrsim_acquisition& a) {
  size_t ys = ny / 2;
  size_t accel = std::max<int64_t>(a.accel, 1);
  std::vector<uint8_t> m(nx * ny, 0);
  size_t keep_n = (size_t)std::round((double)ny * a.partial_fourier);
  for (size_t kyi = 0; kyi < ny; ++kyi) {
    if (a.partial_fourier < 1.0 && a.pf_mode == MRSIM_PF_SCANNER) {
      bool skip = a.reverse_phase ? (kyi < ny - keep_n) : (kyi >= keep_n);
      if (skip) continue;
    } else if (a.partial_fourier < 1.0 && a.pf_mode == MRSIM_PF_CONTIGUOUS) {
      bool skip = a.reverse_phase ? (kyi >= keep_n) : (kyi < ny - keep_n);
      if (skip) continue;
    } else if (a.partial_fourier < 1.0) {
      bool skip;
      if (a.reverse_phase)
        skip = (double)kyi > std::ceil((double)ny * a.partial_fourier);
      else
        skip = (double)kyi < std::floor((double)ny * (1.0 - a.partial_fourier)) && (kyi > 0 || ny % 2 == 1);
      if (skip) continue;
    }
    bool acquired = accel <= 1 || kyi % accel == ys % accel;
    if (!acquired) continue;
    for (size_t kxi = 0; kxi < nx; ++kxi) m[kxi + nx * kyi] = 1;
  }
  return m;
}

std::vector<uint8_t> acquired_lines(size_t ny, const mrsim_acquisition& a) { return sampling_mask(1, ny, a); }

// ---- `validate_acquisition_timing` kspace.rs:411-431 ----
void validate_acquisition_timing(const mrsim_acquisition& a, size_t nx, size_t ny) {
  LineTiming lt = line_timing_for(a, nx, ny);
  auto mask = sampling_mask(nx, ny, a);
  double worst = INFINITY;
  for (size_t ky = 0; ky < ny; ++ky)
    if (mask[ky * nx] && lt.trf_ms[ky] < worst) worst = lt.trf_ms[ky];
  if (worst <= 0.0) {
    char buf[512];
    snprintf(buf, sizeof buf,
             "trf = %.3f ms <= 0 on an acquired line: the readout starts before the excitation. Raise "
             "t_echo above %.3f ms or shorten t_line. Partial Fourier helps only in Scanner mode (it skips "
             "the first lines); the Fiberfox and Contiguous modes drop lines this trajectory reads last.",
             worst, a.t_echo - worst);
    throw Fail(buf);
  }
}

// ---- `coil_sensitivity` kspace.rs:226-237 ----
double coil_sensitivity(size_t coil, size_t n_coils, double x, double y, size_t nx, size_t ny) {
  if (n_coils <= 1) return 1.0;
  double cx = (double)nx / 2.0, cy = (double)ny / 2.0;
  double r = 0.6 * (double)std::max(nx, ny);
  double ang = TAU * (double)coil / (double)n_coils;
  double px = cx + r * std::cos(ang), py = cy + r * std::sin(ang);
  double dx = x - px, dy = y - py;
  double d2 = dx * dx + dy * dy;
  double sigma = 0.9 * (double)std::max(nx, ny);
  return std::exp(-d2 / (2.0 * sigma * sigma)) + 0.15;
}

// ---- `KspaceWindow::at` kspace.rs:140-161 ----
double window_at(const mrsim_acquisition& a, double kx, double ky) {
  double r = 2.0 * std::sqrt(kx * kx + ky * ky);
  switch (a.window_kind) {
    case MRSIM_WINDOW_NONE:
      return 1.0;
    case MRSIM_WINDOW_HANN:
      return r >= 1.0 ? 0.0 : 0.5 * (1.0 + std::cos(PI * r));
    case MRSIM_WINDOW_TUKEY: {
      double al = std::min(std::max(a.window_a, 0.0), 1.0);
      if (r <= 1.0 - al) return 1.0;
      if (r >= 1.0) return 0.0;
      return 0.5 * (1.0 + std::cos(PI * (r - (1.0 - al)) / std::max(al, 1e-12)));
    }
    case MRSIM_WINDOW_FERMI:
      return 1.0 / (1.0 + std::exp((r - a.window_a) / std::max(a.window_b, 1e-12)));
  }
  return 1.0;
}

bool eddy_enabled(const mrsim_acquisition& a, const mrsim_slice_input& inp) {
  return a.eddy_strength != 0.0 && inp.has_eddy_drive;
}

// T2 accessors (`T2Slice` kspace.rs:380-386)
inline double t2_value(const mrsim_t2& t, size_t i) { return t.is_map ? (double)t.map[i] : (double)t.value; }

// ---- the reference's two builds ------------------------------------------------------------
// 0: the default build (rotor y-stage, twiddle x-stage, direct inverse); 1: the `kspace` cargo
// feature (NUFFT y-stage kspace.rs:769-833, FFT x-stage kspace.rs:1079-1123, `inverse_2d_fft`
// kspace.rs:1385-1424).  rustfft's transforms are restated by fft1d (the same linear maps).
int g_kspace_build = 0;

void fft1d(std::vector<Cx>& a, int sign);

// `Nufft1` nufft.rs:25-112, FP64: sources at positions (cells, period n), any number of weight
// vectors, outputs at integer frequencies k_lo .. k_lo + n_out.
struct Nufft1O {
  size_t nf, w, n_out;
  double beta;
  int64_t k_lo;
  std::vector<double> corr, kern;
  Nufft1O(size_t n, int64_t k_lo_, size_t n_out_, double tol) : nf(2 * n), n_out(n_out_), k_lo(k_lo_) {
    if (!(n_out > 0 && k_lo >= -(int64_t)n / 2 && k_lo + (int64_t)n_out - 1 <= (int64_t)n / 2))
      throw Fail("output band must sit inside the coarse Nyquist band");
    w = (size_t)std::min(16.0, std::max(2.0, std::ceil(-std::log10(tol)) + 1.0));
    beta = 2.30 * (double)w;
    const double half = (double)w / 2.0;
    for (size_t j = 0; j < n_out; ++j) {  // `deapodization` nufft.rs:48-63
      const double k = (double)(k_lo + (int64_t)j);
      double s = psi(0.0);
      for (double m = 1.0; m < half; m += 1.0) s += 2.0 * psi(m / half) * std::cos(TAU * k * m / (double)nf);
      corr.push_back(1.0 / s);
    }
    kern.assign(w, 0.0);
  }
  double psi(double z) const { return std::fabs(z) < 1.0 ? std::exp(beta * (std::sqrt(1.0 - z * z) - 1.0)) : 0.0; }
  static double rem_euclid(double x, double m) {
    const double r = std::fmod(x, m);
    return r < 0.0 ? r + std::fabs(m) : r;
  }
  // `Nufft1::run` nufft.rs:70-108
  void run(const std::vector<double>& pos, const std::vector<std::vector<double>>& wre,
           const std::vector<std::vector<double>>& wim, std::vector<std::vector<Cx>>& out) {
    const size_t nw = wre.size();
    const double half = (double)w / 2.0;
    std::vector<std::vector<Cx>> grid(nw, std::vector<Cx>(nf, CZERO));
    for (size_t j = 0; j < pos.size(); ++j) {
      const double p = rem_euclid(2.0 * pos[j], (double)nf);
      const int64_t m0 = (int64_t)std::floor(p - half) + 1;
      for (size_t i = 0; i < w; ++i) kern[i] = psi(((double)m0 + (double)i - p) / half);
      for (size_t q = 0; q < nw; ++q) {
        const double wr = wre[q][j], wi = wim[q][j];
        for (size_t i = 0; i < w; ++i) {
          int64_t m = (m0 + (int64_t)i) % (int64_t)nf;
          if (m < 0) m += (int64_t)nf;
          grid[q][(size_t)m].re += wr * kern[i];
          grid[q][(size_t)m].im += wi * kern[i];
        }
      }
    }
    out.assign(nw, std::vector<Cx>(n_out));
    for (size_t q = 0; q < nw; ++q) {
      fft1d(grid[q], +1);
      for (size_t j = 0; j < n_out; ++j) {
        int64_t bin = (k_lo + (int64_t)j) % (int64_t)nf;
        if (bin < 0) bin += (int64_t)nf;
        const Cx v = grid[q][(size_t)bin];
        out[q][j] = {v.re * corr[j], v.im * corr[j]};
      }
    }
  }
};

// ---- `XStage` (default build, twiddle tables) kspace.rs:1052-1140 ----
struct XStage {
  size_t snx, nx, xs_ = 0;
  bool fft = false;
  std::vector<Cx> tw[2];
  std::vector<Cx> ramp[2], centre;  // the `kspace` build (kspace.rs:1079-1096)
  XStage(size_t snx_, size_t nx_, size_t xs, size_t sxs, double xoff, double ghost) : snx(snx_), nx(nx_) {
    double c = (double)sxs + xoff;
    double gh[2] = {ghost, -ghost};
    if (g_kspace_build) {
      fft = true;
      xs_ = xs;
      for (int p = 0; p < 2; ++p)
        for (size_t x = 0; x < snx; ++x) {
          const double ph = TAU * gh[p] * ((double)x - c) / (double)snx;
          ramp[p].push_back({std::cos(ph), std::sin(ph)});
        }
      for (size_t kxi = 0; kxi < nx; ++kxi) {
        const double ph = -TAU * ((double)kxi - (double)xs) * c / (double)snx;
        centre.push_back({std::cos(ph), std::sin(ph)});
      }
      return;
    }
    for (int p = 0; p < 2; ++p) {
      tw[p].reserve(snx * nx);
      for (size_t kxi = 0; kxi < nx; ++kxi) {
        double kx_norm = ((double)kxi - (double)xs + gh[p]) / (double)snx;
        for (size_t x = 0; x < snx; ++x) {
          double ph = TAU * kx_norm * ((double)x - c);
          tw[p].push_back({std::cos(ph), std::sin(ph)});
        }
      }
    }
  }
  void run(const double* g_re, const double* g_im, double ghost_shift, Cx* out) const {
    int pol = ghost_shift < 0.0 ? 1 : 0;
    if (fft) {  // `XStage::run` kspace.rs:1102-1115: ramp, inverse FFT of length snx, centre phase
      std::vector<Cx> buf(snx);
      for (size_t x = 0; x < snx; ++x) {
        const double rr = ramp[pol][x].re, ri = ramp[pol][x].im;
        buf[x] = {g_re[x] * rr - g_im[x] * ri, g_re[x] * ri + g_im[x] * rr};
      }
      fft1d(buf, +1);
      for (size_t kxi = 0; kxi < nx; ++kxi) {
        int64_t bin = ((int64_t)kxi - (int64_t)xs_) % (int64_t)snx;
        if (bin < 0) bin += (int64_t)snx;
        const double cr = centre[kxi].re, ci = centre[kxi].im;
        const Cx v = buf[(size_t)bin];
        out[kxi] = {v.re * cr - v.im * ci, v.re * ci + v.im * cr};
      }
      return;
    }
    const std::vector<Cx>& t = tw[pol];
    for (size_t kxi = 0; kxi < nx; ++kxi) {
      const Cx* row = &t[snx * kxi];
      double ar = 0.0, ai = 0.0;
      for (size_t x = 0; x < snx; ++x) {
        double tr = row[x].re, ti = row[x].im;
        ar += g_re[x] * tr - g_im[x] * ti;
        ai += g_re[x] * ti + g_im[x] * tr;
      }
      out[kxi] = {ar, ai};
    }
  }
};

// ---- `build_coil_kspace_timed` kspace.rs:607-1042 (default build: rotor y-stage) ----
std::vector<Cx> build_coil_kspace_timed(const mrsim_slice_input& inp, const mrsim_acquisition& acq, size_t coil,
                                        size_t ncoils, const LineTiming& timing, const double* log_amp) {
  size_t snx = inp.sim[0], sny = inp.sim[1], nx = inp.acq_matrix[0], ny = inp.acq_matrix[1];
  if (!(snx % nx == 0 && sny % ny == 0)) throw Fail("sim grid must be an integer multiple of the acquired matrix");
  if (!(timing.t_ms.size() == ny && timing.trf_ms.size() == ny && timing.tread_ms.size() == ny &&
        timing.polarity.size() == ny))
    throw Fail("line-timing table must have one entry per phase-encode line");
  size_t z = inp.z, nz = inp.nz;
  size_t ncomp = inp.ncomp;
  const double* t_ms = timing.t_ms.data();
  const double* trf_ms = timing.trf_ms.data();
  const double* tread_ms = timing.tread_ms.data();
  double gradient[3] = {0.0, 0.0, 0.0};
  if (inp.has_eddy_drive)
    for (int i = 0; i < 3; ++i) gradient[i] = inp.eddy_drive[i];
  bool do_eddy = eddy_enabled(acq, inp);
  bool do_eddy_phase = acq.eddy_phase != 0.0 && inp.has_eddy_drive;
  size_t xs = nx / 2, ys = ny / 2, zs = nz / 2;
  size_t ox = snx / nx, oy = sny / ny;
  size_t sxs = ox * xs, sys = oy * ys;
  double xoff = ((double)ox - 1.0) / 2.0, yoff = ((double)oy - 1.0) / 2.0;
  size_t nvox = snx * sny;
  auto mask = sampling_mask(nx, ny, acq);

  const size_t REANCHOR = 32;
  double zc = (double)z - (double)zs;
  double zc_c = (double)z - ((double)nz - 1.0) / 2.0;
  std::vector<double> amp(nvox), phi0(nvox), rate(nvox);
  for (size_t y = 0; y < sny; ++y) {
    for (size_t x = 0; x < snx; ++x) {
      size_t i = x + snx * y;
      double xa = ((double)x - xoff) / (double)ox, ya = ((double)y - yoff) / (double)oy;
      amp[i] = acq.signal_scale * coil_sensitivity(coil, ncoils, xa, ya, nx, ny);
      double xc = ((double)x - (double)sxs - xoff) / (double)ox;
      double yc = ((double)y - (double)sys - yoff) / (double)oy;
      double p0 = inp.phase0 ? inp.phase0[i] : 0.0;
      if (do_eddy_phase) p0 += acq.eddy_phase * (gradient[0] * xc + gradient[1] * yc + gradient[2] * zc_c);
      if (acq.echo == MRSIM_ECHO_GRADIENT && acq.do_distortions)
        p0 += TAU * (double)inp.fmap[i] * (acq.t_echo / 1000.0);
      phi0[i] = p0;
      rate[i] = acq.do_distortions ? (double)inp.fmap[i] : 0.0;
    }
  }
  auto xc_of = [&](size_t x) { return ((double)x - (double)sxs - xoff) / (double)ox; };
  auto yc_of = [&](size_t y) { return ((double)y - (double)sys - yoff) / (double)oy; };
  auto ky_norm_of = [&](size_t kyi) { return ((double)kyi - (double)ys) / (double)sny; };

  std::vector<double> st_re(nvox, 0.0), st_im(nvox, 0.0);
  auto set_state = [&](size_t kyi) {
    double t = t_ms[kyi] / 1000.0;
    double kyn = ky_norm_of(kyi);
    for (size_t y = 0; y < sny; ++y) {
      double yy = (double)y - (double)sys - yoff;
      for (size_t x = 0; x < snx; ++x) {
        size_t i = x + snx * y;
        double ph = phi0[i] + TAU * (rate[i] * t + kyn * yy);
        st_re[i] = amp[i] * std::cos(ph);
        st_im[i] = amp[i] * std::sin(ph);
      }
    }
  };
  struct Rotor {
    size_t k0, k1;
    double dt, dkyn;
    std::vector<double> re, im;
  };
  std::vector<Rotor> rotors;

  bool uniform = true;
  for (size_t c = 0; c < ncomp; ++c) uniform = uniform && !inp.t2[c].is_map;
  if (inp.t_inhom)
    for (size_t c = 0; c < ncomp; ++c) uniform = uniform && !inp.t_inhom[c].is_map;
  uniform = uniform && log_amp == nullptr;

  std::vector<double> rel(ncomp, 1.0);
  std::vector<double> ex_re(snx, 1.0), ex_im(snx, 0.0), ey_re(sny, 1.0), ey_im(sny, 0.0);
  std::vector<double> g_re(snx, 0.0), g_im(snx, 0.0);
  XStage xstage(snx, nx, xs, sxs, xoff, acq.ghost_offset);

  // the `kspace` build's NUFFT y-stage (kspace.rs:769-833): with t affine in the line index per
  // parity, every column's y-sum is one type-1 NUFFT of sources displaced by the fieldmap
  std::vector<std::vector<Cx>> nufft_rows;  // [c][x + snx kyi]
  bool have_rows = false;
  if (g_kspace_build && !do_eddy && ny >= 3 && uniform) {
    const double tau = (t_ms[2] - t_ms[0]) / 2.0;
    const double t0 = t_ms[0];
    const double delta = t_ms[1] - (tau + t0);
    double tmax = 0.0;
    for (size_t k = 0; k < ny; ++k) tmax = std::fmax(tmax, std::fabs(t_ms[k]));
    tmax = std::fmax(tmax, 1e-300);
    bool affine = true;
    for (size_t k = 0; k < ny; ++k) {
      const double pred = tau * (double)k + t0 + (k % 2 == 1 ? delta : 0.0);
      affine = affine && std::fabs(t_ms[k] - pred) <= 1e-9 * tmax && timing.polarity[k] == (k % 2 == 1 ? -1 : 1);
    }
    if (affine) {
      const double tau_s = tau / 1000.0, delta_s = delta / 1000.0;
      const double t_centre = (tau * (double)ys + t0) / 1000.0;
      Nufft1O nufft(sny, -(int64_t)ys, ny, 1e-13);
      std::vector<double> pos(sny, 0.0);
      std::vector<std::vector<double>> wre(2 * ncomp, std::vector<double>(sny, 0.0)),
          wim(2 * ncomp, std::vector<double>(sny, 0.0));
      std::vector<std::vector<Cx>> out;
      nufft_rows.assign(ncomp, std::vector<Cx>(snx * ny, CZERO));
      for (size_t x = 0; x < snx; ++x) {
        for (size_t y = 0; y < sny; ++y) {
          const size_t i = x + snx * y;
          pos[y] = ((double)y - (double)sys - yoff) + (double)sny * tau_s * rate[i];
          const double ph = phi0[i] + TAU * rate[i] * t_centre;
          const double c0 = std::cos(ph), s0 = std::sin(ph);
          const double phd = TAU * rate[i] * delta_s;
          const double cd = std::cos(phd), sd = std::sin(phd);
          const double c1 = c0 * cd - s0 * sd, s1 = c0 * sd + s0 * cd;
          for (size_t c = 0; c < ncomp; ++c) {
            const double a = amp[i] * (double)inp.compartments[c][i];
            wre[2 * c][y] = a * c0;
            wim[2 * c][y] = a * s0;
            wre[2 * c + 1][y] = a * c1;
            wim[2 * c + 1][y] = a * s1;
          }
        }
        nufft.run(pos, wre, wim, out);
        for (size_t c = 0; c < ncomp; ++c)
          for (size_t kyi = 0; kyi < ny; ++kyi) nufft_rows[c][x + snx * kyi] = out[2 * c + (kyi % 2)][kyi];
      }
      have_rows = true;
    }
  }

  std::vector<Cx> kspace(nx * ny, CZERO);
  bool have_prev = false;
  size_t prev = 0;
  size_t since_anchor = 0;
  for (size_t kyi = 0; kyi < ny; ++kyi) {
    if (!mask[nx * kyi]) continue;
    double t = t_ms[kyi] / 1000.0;
    double trf = trf_ms[kyi];
    if (have_rows) {
      // the NUFFT rows replace the rotor state (kspace.rs:848)
    } else if (have_prev && since_anchor < REANCHOR) {
      size_t p = prev;
      size_t k0 = kyi - p, k1 = p % 2;
      double dt = t - t_ms[p] / 1000.0;
      double dkyn = ky_norm_of(kyi) - ky_norm_of(p);
      size_t idx = rotors.size();
      for (size_t r = 0; r < rotors.size(); ++r)
        if (rotors[r].k0 == k0 && rotors[r].k1 == k1) {
          idx = r;
          break;
        }
      if (idx == rotors.size()) {
        Rotor R{k0, k1, dt, dkyn, std::vector<double>(nvox), std::vector<double>(nvox)};
        for (size_t y = 0; y < sny; ++y) {
          double yy = (double)y - (double)sys - yoff;
          for (size_t x = 0; x < snx; ++x) {
            size_t i = x + snx * y;
            double ph = TAU * (rate[i] * dt + dkyn * yy);
            R.re[i] = std::cos(ph);
            R.im[i] = std::sin(ph);
          }
        }
        rotors.push_back(std::move(R));
      }
      const Rotor& r = rotors[idx];
      if (std::fabs(r.dt - dt) <= 1e-12 * std::max(std::fabs(dt), 1e-300) && r.dkyn == dkyn) {
        for (size_t i = 0; i < nvox; ++i) {
          double a = st_re[i], b = st_im[i];
          st_re[i] = a * r.re[i] - b * r.im[i];
          st_im[i] = a * r.im[i] + b * r.re[i];
        }
        since_anchor += 1;
      } else {
        set_state(kyi);
        since_anchor = 0;
      }
    } else {
      set_state(kyi);
      since_anchor = 0;
    }
    prev = kyi;
    have_prev = true;

    if (uniform) {
      for (size_t c = 0; c < ncomp; ++c) {
        if (acq.do_relaxation) {
          double t2c = (double)inp.t2[c].value;
          double tic = inp.t_inhom ? (double)inp.t_inhom[c].value : acq.t_inhom;
          if (acq.echo == MRSIM_ECHO_SPIN)
            rel[c] = std::exp(-trf / t2c - std::fabs(t) * 1000.0 / tic);
          else
            rel[c] = std::exp(-trf / t2c - trf / tic);
        } else {
          rel[c] = 1.0;
        }
      }
    }
    double ez_re = 1.0, ez_im = 0.0;
    if (do_eddy) {
      double eddy_decay = std::exp(-tread_ms[kyi] / acq.eddy_tau) * t;
      for (size_t x = 0; x < snx; ++x) {
        double xc = xc_of(x);
        double ph = TAU * (acq.eddy_strength * gradient[0] * xc + acq.eddy_quad * gradient[0] * xc * xc) * eddy_decay;
        ex_re[x] = std::cos(ph);
        ex_im[x] = std::sin(ph);
      }
      for (size_t y = 0; y < sny; ++y) {
        double yc = yc_of(y);
        double ph = TAU * (acq.eddy_strength * gradient[1] * yc + acq.eddy_quad * gradient[1] * yc * yc) * eddy_decay;
        ey_re[y] = std::cos(ph);
        ey_im[y] = std::sin(ph);
      }
      double ph = TAU * (acq.eddy_strength * gradient[2] * zc + acq.eddy_quad * gradient[2] * zc * zc) * eddy_decay;
      ez_re = std::cos(ph);
      ez_im = std::sin(ph);
    }
    std::fill(g_re.begin(), g_re.end(), 0.0);
    std::fill(g_im.begin(), g_im.end(), 0.0);
    if (have_rows) {  // kspace.rs:929-937
      for (size_t c = 0; c < ncomp; ++c)
        for (size_t x = 0; x < snx; ++x) {
          g_re[x] += rel[c] * nufft_rows[c][x + snx * kyi].re;
          g_im[x] += rel[c] * nufft_rows[c][x + snx * kyi].im;
        }
    }
    for (size_t y = 0; y < sny && !have_rows; ++y) {
      size_t row = snx * y;
      double eyr = ey_re[y], eyi = ey_im[y];
      for (size_t x = 0; x < snx; ++x) {
        size_t i = row + x;
        double w = 0.0;
        for (size_t c = 0; c < ncomp; ++c) {
          double r;
          if (uniform) {
            r = rel[c];
          } else if (acq.do_relaxation) {
            double t2c = t2_value(inp.t2[c], i);
            double tic = inp.t_inhom ? t2_value(inp.t_inhom[c], i) : acq.t_inhom;
            bool spin = acq.echo == MRSIM_ECHO_SPIN;
            if (!log_amp)
              r = spin ? std::exp(-trf / t2c - std::fabs(t) * 1000.0 / tic) : std::exp(-trf / t2c - trf / tic);
            else
              r = spin ? std::exp(log_amp[i] - trf / t2c - std::fabs(t) * 1000.0 / tic)
                       : std::exp(log_amp[i] - trf / t2c - trf / tic);
          } else {
            r = 1.0;
          }
          w += r * (double)inp.compartments[c][i];
        }
        double sr = st_re[i], si = st_im[i];
        double mr, mi;
        if (do_eddy) {
          mr = sr * eyr - si * eyi;
          mi = sr * eyi + si * eyr;
        } else {
          mr = sr;
          mi = si;
        }
        g_re[x] += w * mr;
        g_im[x] += w * mi;
      }
    }
    if (do_eddy) {
      for (size_t x = 0; x < snx; ++x) {
        double a = g_re[x], b = g_im[x];
        double fr = ex_re[x] * ez_re - ex_im[x] * ez_im, fi = ex_re[x] * ez_im + ex_im[x] * ez_re;
        g_re[x] = a * fr - b * fi;
        g_im[x] = a * fi + b * fr;
      }
    }
    double ghost_shift = timing.polarity[kyi] < 0 ? -acq.ghost_offset : acq.ghost_offset;
    xstage.run(g_re.data(), g_im.data(), ghost_shift, &kspace[nx * kyi]);
  }
  double n_inv = 1.0 / (double)nvox;
  for (auto& k : kspace) {
    k.re *= n_inv;
    k.im *= n_inv;
  }
  // spikes kspace.rs:997-1019
  if (acq.n_spikes > 0) {
    Cx peak = CZERO;
    double peak_mag = 0.0;
    for (auto& k : kspace) {
      double m = cabs_(k);
      if (m > peak_mag) {
        peak_mag = m;
        peak = k;
      }
    }
    Cx spike = cscale(peak, acq.spike_amplitude);
    std::vector<size_t> acquired;
    for (size_t i = 0; i < nx * ny; ++i)
      if (mask[i]) acquired.push_back(i);
    if (!acquired.empty()) {
      Rng rng(inp.slice_seed ^ 0xA5A5123456789ABCull);
      for (int64_t s = 0; s < acq.n_spikes; ++s) {
        size_t pick = acquired[(size_t)(rng.next_u64() % (uint64_t)acquired.size())];
        kspace[pick] = spike;
      }
    }
  }
  // noise kspace.rs:1021-1039
  if (acq.noise_variance > 0.0) {
    Rng rng((inp.slice_seed ^ ((uint64_t)coil * 0x9E3779B9ull)) | 1ull);
    double sigma = std::sqrt(acq.noise_variance / (double)(nx * ny));
    for (size_t i = 0; i < nx * ny; ++i) {
      if (mask[i]) {
        kspace[i].re += rng.gauss() * sigma;
        kspace[i].im += rng.gauss() * sigma;
      }
    }
  }
  return kspace;
}

std::vector<Cx> build_coil_kspace(const mrsim_slice_input& inp, const mrsim_acquisition& acq, size_t coil,
                                  size_t ncoils) {
  return build_coil_kspace_timed(inp, acq, coil, ncoils,
                                 line_timing_for(acq, inp.acq_matrix[0], inp.acq_matrix[1]), nullptr);
}

std::vector<std::vector<Cx>> build_coil_kspaces(const mrsim_slice_input& inp, const mrsim_acquisition& acq) {
  size_t nc = std::max<int64_t>(acq.n_coils, 1);
  std::vector<std::vector<Cx>> out;
  for (size_t c = 0; c < nc; ++c) out.push_back(build_coil_kspace(inp, acq, c, nc));
  return out;
}

// ---- literal per-line sum, `reference_coil_kspace` kspace.rs:2225-2406 (test oracle) ----
std::vector<Cx> reference_coil_kspace(const mrsim_slice_input& inp, const mrsim_acquisition& acq, size_t coil,
                                      size_t ncoils) {
  size_t snx = inp.sim[0], sny = inp.sim[1], nx = inp.acq_matrix[0], ny = inp.acq_matrix[1];
  if (!(snx % nx == 0 && sny % ny == 0)) throw Fail("sim grid must be an integer multiple of the acquired matrix");
  size_t z = inp.z;
  Epi epi{nx, ny, acq.t_line, acq.t_echo, acq.reverse_phase != 0};
  std::vector<double> t_ms(ny, 0.0), trf_ms(ny, 0.0), tread_ms(ny, 0.0);
  for (size_t tick = 0; tick < nx * ny; ++tick) {
    size_t kx, ky;
    epi.kspace_index(tick, kx, ky);
    if (kx == nx / 2) {
      t_ms[ky] = epi.time_from_max_echo(tick);
      trf_ms[ky] = epi.time_from_rf(tick);
      tread_ms[ky] = epi.time_from_prep_gradient(tick);
    }
  }
  double skip = (double)pf_skipped_lines(ny, acq) * acq.t_line;
  for (auto& v : tread_ms) v -= skip;
  double gradient[3] = {0, 0, 0};
  if (inp.has_eddy_drive)
    for (int i = 0; i < 3; ++i) gradient[i] = inp.eddy_drive[i];
  bool do_eddy = eddy_enabled(acq, inp);
  bool do_eddy_phase = acq.eddy_phase != 0.0 && inp.has_eddy_drive;
  size_t xs = nx / 2, ys = ny / 2, zs = inp.nz / 2;
  size_t ox = snx / nx, oy = sny / ny;
  size_t sxs = ox * xs, sys = oy * ys;
  double xoff = ((double)ox - 1.0) / 2.0, yoff = ((double)oy - 1.0) / 2.0;
  auto mask = sampling_mask(nx, ny, acq);
  std::vector<Cx> kspace(nx * ny, CZERO);
  double n_inv = 1.0 / (double)(snx * sny);
  std::vector<Cx> modimg(snx * sny);
  std::vector<Cx> g(snx);
  for (size_t kyi = 0; kyi < ny; ++kyi) {
    if (!mask[nx * kyi]) continue;
    double t = t_ms[kyi] / 1000.0;
    double trf = trf_ms[kyi];
    double ky_norm = ((double)kyi - (double)ys) / (double)sny;
    double ghost_shift = (kyi % 2 == 1) ? -acq.ghost_offset : acq.ghost_offset;
    double eddy_decay = do_eddy ? std::exp(-tread_ms[kyi] / acq.eddy_tau) * t : 0.0;
    for (size_t y = 0; y < sny; ++y) {
      for (size_t x = 0; x < snx; ++x) {
        size_t i = x + snx * y;
        double f_real = 0.0;
        for (size_t c = 0; c < (size_t)inp.ncomp; ++c) {
          double v = (double)inp.compartments[c][i];
          if (acq.do_relaxation) {
            double t2c = t2_value(inp.t2[c], i);
            double tic = inp.t_inhom ? t2_value(inp.t_inhom[c], i) : acq.t_inhom;
            double inhom_ms = acq.echo == MRSIM_ECHO_SPIN ? std::fabs(t) * 1000.0 : trf;
            v *= std::exp(-trf / t2c - inhom_ms / tic);
          }
          f_real += v;
        }
        double xa = ((double)x - xoff) / (double)ox, ya = ((double)y - yoff) / (double)oy;
        f_real *= acq.signal_scale * coil_sensitivity(coil, ncoils, xa, ya, nx, ny);
        double t_b0 = acq.echo == MRSIM_ECHO_SPIN ? t : t + acq.t_echo / 1000.0;
        double phi = acq.do_distortions ? (double)inp.fmap[i] * t_b0 : 0.0;
        double phi0 = inp.phase0 ? inp.phase0[i] : 0.0;
        if (do_eddy || do_eddy_phase) {
          double xc = ((double)x - (double)sxs - xoff) / (double)ox;
          double yc = ((double)y - (double)sys - yoff) / (double)oy;
          double zc = (double)z - (double)zs;
          if (do_eddy) {
            double lin = gradient[0] * xc + gradient[1] * yc + gradient[2] * zc;
            double quad = gradient[0] * xc * xc + gradient[1] * yc * yc + gradient[2] * zc * zc;
            phi += (acq.eddy_strength * lin + acq.eddy_quad * quad) * eddy_decay;
          }
          if (do_eddy_phase) {
            double zc_c = (double)z - ((double)inp.nz - 1.0) / 2.0;
            phi0 += acq.eddy_phase * (gradient[0] * xc + gradient[1] * yc + gradient[2] * zc_c);
          }
        }
        modimg[i] = cscale(ccis(TAU * phi + phi0), f_real);
      }
    }
    for (size_t x = 0; x < snx; ++x) {
      Cx acc = CZERO;
      for (size_t y = 0; y < sny; ++y) {
        Cx ph = ccis(TAU * ky_norm * ((double)y - (double)sys - yoff));
        acc = cadd(acc, cmul(modimg[x + snx * y], ph));
      }
      g[x] = acc;
    }
    for (size_t kxi = 0; kxi < nx; ++kxi) {
      double kx_norm = ((double)kxi - (double)xs + ghost_shift) / (double)snx;
      Cx acc = CZERO;
      for (size_t x = 0; x < snx; ++x)
        acc = cadd(acc, cmul(g[x], ccis(TAU * kx_norm * ((double)x - (double)sxs - xoff))));
      kspace[kxi + nx * kyi] = cscale(acc, n_inv);
    }
  }
  return kspace;
}

// ---- `inverse_2d_fft` kspace.rs:1385-1424 (the `kspace` build): pre-modulation, forward FFTs
// along x then y (rustfft's e^{-i}, here fft1d), post-modulation with the constant phase ----
std::vector<Cx> inverse_2d_fft(const std::vector<Cx>& k, size_t nx, size_t ny, size_t xs, size_t ys) {
  const double nxf = (double)nx, nyf = (double)ny, xsf = (double)xs, ysf = (double)ys;
  std::vector<Cx> buf(nx * ny);
  for (size_t i = 0; i < nx * ny; ++i) {
    const double kx = (double)(i % nx), ky = (double)(i / nx);
    const double ph = TAU * (kx * xsf / nxf + ky * ysf / nyf);
    const double c = std::cos(ph), sn = std::sin(ph);
    buf[i] = {k[i].re * c - k[i].im * sn, k[i].re * sn + k[i].im * c};
  }
  std::vector<Cx> line(nx);
  for (size_t ky = 0; ky < ny; ++ky) {
    for (size_t x = 0; x < nx; ++x) line[x] = buf[ky * nx + x];
    fft1d(line, -1);
    for (size_t x = 0; x < nx; ++x) buf[ky * nx + x] = line[x];
  }
  std::vector<Cx> col(ny);
  for (size_t kx = 0; kx < nx; ++kx) {
    for (size_t y = 0; y < ny; ++y) col[y] = buf[y * nx + kx];
    fft1d(col, -1);
    for (size_t y = 0; y < ny; ++y) buf[y * nx + kx] = col[y];
  }
  const double const_ph = -TAU * (xsf * xsf / nxf + ysf * ysf / nyf);
  std::vector<Cx> out(nx * ny);
  for (size_t i = 0; i < nx * ny; ++i) {
    const double x = (double)(i % nx), y = (double)(i / nx);
    const double ph = TAU * (x * xsf / nxf + y * ysf / nyf) + const_ph;
    const double c = std::cos(ph), sn = std::sin(ph);
    out[i] = {buf[i].re * c - buf[i].im * sn, buf[i].re * sn + buf[i].im * c};
  }
  return out;
}

// ---- `inverse_2d` kspace.rs:1428-1453 ----
std::vector<Cx> inverse_2d(const std::vector<Cx>& k, size_t nx, size_t ny, size_t xs, size_t ys) {
  std::vector<Cx> h(nx * ny, CZERO), out(nx * ny, CZERO);
  for (size_t kxi = 0; kxi < nx; ++kxi)
    for (size_t y = 0; y < ny; ++y) {
      Cx acc = CZERO;
      for (size_t kyi = 0; kyi < ny; ++kyi) {
        double ky_norm = ((double)kyi - (double)ys) / (double)ny;
        acc = cadd(acc, cmul(k[kxi + nx * kyi], ccis(-TAU * ky_norm * ((double)y - (double)ys))));
      }
      h[kxi + nx * y] = acc;
    }
  for (size_t y = 0; y < ny; ++y)
    for (size_t x = 0; x < nx; ++x) {
      Cx acc = CZERO;
      for (size_t kxi = 0; kxi < nx; ++kxi) {
        double kx_norm = ((double)kxi - (double)xs) / (double)nx;
        acc = cadd(acc, cmul(h[kxi + nx * y], ccis(-TAU * kx_norm * ((double)x - (double)xs))));
      }
      out[x + nx * y] = acc;
    }
  return out;
}

// ---- `solve_hermitian` kspace.rs:1457-1491 ----
std::vector<Cx> solve_hermitian(std::vector<std::vector<Cx>> h, std::vector<Cx> b) {
  size_t n = b.size();
  auto recip = [](Cx d) -> Cx {
    double m2 = d.re * d.re + d.im * d.im;
    if (m2 < 1e-18) return CZERO;
    return {d.re / m2, -d.im / m2};
  };
  for (size_t col = 0; col < n; ++col) {
    size_t piv = col;
    double best = cabs_(h[col][col]);
    for (size_t r = col + 1; r < n; ++r) {
      double m = cabs_(h[r][col]);
      if (m > best) {
        best = m;
        piv = r;
      }
    }
    std::swap(h[col], h[piv]);
    std::swap(b[col], b[piv]);
    Cx dinv = recip(h[col][col]);
    for (size_t r = col + 1; r < n; ++r) {
      Cx f = cmul(h[r][col], dinv);
      for (size_t c = col; c < n; ++c) {
        Cx s = cmul(f, h[col][c]);
        h[r][c] = cadd(h[r][c], cscale(s, -1.0));
      }
      Cx sb = cmul(f, b[col]);
      b[r] = cadd(b[r], cscale(sb, -1.0));
    }
  }
  std::vector<Cx> x(n, CZERO);
  for (size_t col = n; col-- > 0;) {
    Cx s = b[col];
    for (size_t c = col + 1; c < n; ++c) s = cadd(s, cscale(cmul(h[col][c], x[c]), -1.0));
    x[col] = cmul(s, recip(h[col][col]));
  }
  return x;
}

// ---- `GrappaKernel` kspace.rs:1508-1633 ----
const int64_t GRAPPA_DKX[3] = {-1, 0, 1};
const double GRAPPA_LAMBDA = 1e-3;

void grappa_feature(const std::vector<std::vector<Cx>>& coil, size_t nx, size_t s0, size_t s1, size_t kx,
                    std::vector<Cx>& f) {
  size_t nc = coil.size();
  f.assign(6 * nc, CZERO);
  size_t sl[2] = {s0, s1};
  for (size_t li = 0; li < 2; ++li)
    for (size_t ki = 0; ki < 3; ++ki) {
      int64_t v = ((int64_t)kx + GRAPPA_DKX[ki]) % (int64_t)nx;
      if (v < 0) v += (int64_t)nx;
      for (size_t ci = 0; ci < nc; ++ci) f[(li * 3 + ki) * nc + ci] = coil[ci][(size_t)v + nx * sl[li]];
    }
}

struct GrappaKernel {
  size_t accel = 1;
  std::vector<std::vector<std::vector<Cx>>> weights;  // [d-1][out coil][feature]
};

GrappaKernel grappa_fit(const std::vector<std::vector<Cx>>& coil, size_t nx, size_t ny, size_t accel, size_t acs_lines,
                        const std::vector<uint8_t>& lines) {
  if (lines.size() != ny) throw Fail("one acquired-line flag per PE line");
  size_t nc = coil.size();
  size_t ys = ny / 2;
  size_t nfeat = 6 * nc;
  int64_t acs_half = (int64_t)(acs_lines / 2);
  size_t acs_lo = (size_t)std::max<int64_t>((int64_t)ys - acs_half, 0);
  size_t acs_hi = std::min<size_t>((size_t)((int64_t)ys + acs_half), ny - 1);
  GrappaKernel K;
  K.accel = accel;
  std::vector<Cx> f;
  for (size_t d = 1; d < accel; ++d) {
    std::vector<std::vector<Cx>> aha(nfeat, std::vector<Cx>(nfeat, CZERO));
    std::vector<std::vector<Cx>> ahb(nc, std::vector<Cx>(nfeat, CZERO));
    for (size_t b = acs_lo; b < acs_hi; ++b) {
      size_t s0 = b, s1 = b + accel, tgt = b + d;
      if (s1 > acs_hi || tgt > acs_hi || !(lines[s0] && lines[s1] && lines[tgt])) continue;
      for (size_t kx = 0; kx < nx; ++kx) {
        grappa_feature(coil, nx, s0, s1, kx, f);
        for (size_t i = 0; i < nfeat; ++i) {
          Cx fic = {f[i].re, -f[i].im};
          for (size_t j = 0; j < nfeat; ++j) aha[i][j] = cadd(aha[i][j], cmul(fic, f[j]));
          for (size_t co = 0; co < nc; ++co) ahb[co][i] = cadd(ahb[co][i], cmul(fic, coil[co][kx + nx * tgt]));
        }
      }
    }
    double sum = -0.0;
    for (size_t i = 0; i < nfeat; ++i) sum = sum + aha[i][i].re;
    double mean_diag = sum / (double)nfeat;
    if (mean_diag <= 0.0) {
      K.weights.push_back(std::vector<std::vector<Cx>>(nc, std::vector<Cx>(nfeat, CZERO)));
      continue;
    }
    double s = 1.0 / mean_diag;
    for (size_t i = 0; i < nfeat; ++i) {
      for (auto& x : aha[i]) x = cscale(x, s);
      aha[i][i].re += GRAPPA_LAMBDA;
    }
    for (auto& bb : ahb)
      for (auto& x : bb) x = cscale(x, s);
    std::vector<std::vector<Cx>> w;
    for (size_t co = 0; co < nc; ++co) w.push_back(solve_hermitian(aha, ahb[co]));
    K.weights.push_back(std::move(w));
  }
  return K;
}

void grappa_apply(const GrappaKernel& K, std::vector<std::vector<Cx>>& coil, size_t nx, size_t ny,
                  const std::vector<uint8_t>& acquired) {
  if (acquired.size() != ny) throw Fail("one acquired-line flag per PE line");
  size_t ys = ny / 2;
  size_t accel = K.accel, nc = coil.size();
  std::vector<Cx> f;
  for (size_t di = 0; di < K.weights.size(); ++di) {
    size_t d = di + 1;
    const auto& weights = K.weights[di];
    if (weights.size() != nc) throw Fail("the GRAPPA kernel was fitted for another coil count");
    for (size_t ky = 0; ky < ny; ++ky) {
      int64_t r = ((int64_t)ky - (int64_t)ys) % (int64_t)accel;
      if (r < 0) r += (int64_t)accel;
      if (r != (int64_t)d || ky < d || ky + accel - d >= ny) continue;
      size_t s0 = ky - d, s1 = ky - d + accel;
      if (!(acquired[s0] && acquired[s1])) continue;
      for (size_t kx = 0; kx < nx; ++kx) {
        grappa_feature(coil, nx, s0, s1, kx, f);
        for (size_t co = 0; co < nc; ++co) {
          Cx v = CZERO;
          for (size_t i = 0; i < f.size(); ++i) v = cadd(v, cmul(weights[co][i], f[i]));
          coil[co][kx + nx * ky] = v;
        }
      }
    }
  }
}

const uint64_t SEED_SALT_GRAPPA_CAL = 0x47525043414Cull;

// `grappa_reference_kernel` kspace.rs:1253-1262
GrappaKernel grappa_reference_kernel(const mrsim_slice_input& inp, const mrsim_acquisition& acq) {
  mrsim_slice_input ref = inp;
  ref.has_eddy_drive = 0;
  ref.has_prep_drive = 0;
  mrsim_acquisition acq_ref = acq;
  acq_ref.accel = 1;
  acq_ref.n_spikes = 0;
  auto coils = build_coil_kspaces(ref, acq_ref);
  return grappa_fit(coils, inp.acq_matrix[0], inp.acq_matrix[1], (size_t)acq.accel, (size_t)acq.acs_lines,
                    acquired_lines(inp.acq_matrix[1], acq_ref));
}

// ---- `reconstruct_coils_full` kspace.rs:1301-1378 ----
struct SliceRecon {
  std::vector<std::vector<Cx>> acquired, reconstructed, coil_images;
  std::vector<std::vector<double>> sensitivities;
  std::vector<Cx> combined;
  std::vector<uint8_t> mask;
};

SliceRecon reconstruct_coils_full(std::vector<std::vector<Cx>> coil_kspace, const mrsim_acquisition& acq, size_t nx,
                                  size_t ny, bool cap_acq, bool cap_rec, bool cap_img, const GrappaKernel* kernel) {
  size_t xs = nx / 2, ys = ny / 2;
  size_t ncoils = std::max<int64_t>(acq.n_coils, 1);
  size_t accel = std::max<int64_t>(acq.accel, 1);
  if (coil_kspace.size() != ncoils) throw Fail("one k-space per coil");
  SliceRecon R;
  if (cap_acq) R.acquired = coil_kspace;
  if (accel > 1) {
    if (!kernel) throw Fail("an accelerated slice needs its GRAPPA kernel (fitted on a reference scan)");
    if (kernel->accel != accel) throw Fail("the GRAPPA kernel was fitted for another acceleration");
    grappa_apply(*kernel, coil_kspace, nx, ny, acquired_lines(ny, acq));
  }
  if (acq.window_kind != MRSIM_WINDOW_NONE) {
    for (auto& ks : coil_kspace)
      for (size_t kyi = 0; kyi < ny; ++kyi)
        for (size_t kxi = 0; kxi < nx; ++kxi) {
          double kx = ((double)kxi - (double)xs) / (double)nx;
          double ky = ((double)kyi - (double)ys) / (double)ny;
          double w = window_at(acq, kx, ky);
          Cx& k = ks[kxi + nx * kyi];
          k.re *= w;
          k.im *= w;
        }
  }
  if (cap_rec) R.reconstructed = coil_kspace;
  R.sensitivities.resize(ncoils);
  for (size_t coil = 0; coil < ncoils; ++coil) {
    R.sensitivities[coil].resize(nx * ny);
    for (size_t i = 0; i < nx * ny; ++i)
      R.sensitivities[coil][i] = coil_sensitivity(coil, ncoils, (double)(i % nx), (double)(i / nx), nx, ny);
  }
  std::vector<Cx> wsum(nx * ny, CZERO);
  std::vector<double> ssum(nx * ny, 0.0);
  for (size_t coil = 0; coil < ncoils; ++coil) {
    auto img = g_kspace_build ? inverse_2d_fft(coil_kspace[coil], nx, ny, xs, ys)
                              : inverse_2d(coil_kspace[coil], nx, ny, xs, ys);
    for (size_t i = 0; i < nx * ny; ++i) {
      double s = R.sensitivities[coil][i];
      wsum[i] = cadd(wsum[i], cscale(img[i], s));
      ssum[i] += s * s;
    }
    if (cap_img) R.coil_images.push_back(std::move(img));
  }
  R.combined.resize(nx * ny);
  for (size_t i = 0; i < nx * ny; ++i) {
    double s = std::max(ssum[i], 1e-12);
    R.combined[i] = {wsum[i].re / s, wsum[i].im / s};
  }
  R.mask = sampling_mask(nx, ny, acq);
  return R;
}

// `simulate_slice_with` kspace.rs:1271-1284
SliceRecon simulate_slice_with(const mrsim_slice_input& inp, const mrsim_acquisition& acq, bool ca, bool cr, bool ci,
                               const GrappaKernel* kernel) {
  GrappaKernel own;
  if (!kernel && acq.accel > 1) {
    mrsim_slice_input salted = inp;
    salted.slice_seed = inp.slice_seed ^ SEED_SALT_GRAPPA_CAL;
    own = grappa_reference_kernel(salted, acq);
    kernel = &own;
  }
  return reconstruct_coils_full(build_coil_kspaces(inp, acq), acq, inp.acq_matrix[0], inp.acq_matrix[1], ca, cr, ci,
                                kernel);
}

// ---- object phase: `PhaseModel` phase.rs:48-205, `phase_slice` kspace.rs:1156-1180 ----
struct Shot {
  double q[3] = {0, 0, 0}, dx[3] = {0, 0, 0}, rot[3] = {0, 0, 0};
};

double shot_at(const Shot& s, const double r[3]) {
  double c[3] = {s.rot[1] * r[2] - s.rot[2] * r[1], s.rot[2] * r[0] - s.rot[0] * r[2],
                 s.rot[0] * r[1] - s.rot[1] * r[0]};
  double sum = -0.0;
  for (int i = 0; i < 3; ++i) sum = sum + s.q[i] * (s.dx[i] + c[i]);
  return sum;
}

Shot prep_shot(const mrsim_phase_model& p, double magnitude, const double dir[3], size_t volume, size_t slice_group,
               uint64_t seed) {
  Shot s;
  double n = std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  if (magnitude <= 0.0 || n < 1e-12) return s;
  double sc = p.c_q * std::sqrt(magnitude) / n;
  for (int i = 0; i < 3; ++i) s.q[i] = dir[i] * sc;
  Rng rng(seed ^ ((uint64_t)volume * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)slice_group * 0xBF58476D1CE4E5B9ull));
  for (int i = 0; i < 3; ++i) s.dx[i] = rng.gauss() * p.sigma_dx;
  for (int i = 0; i < 3; ++i) s.rot[i] = rng.gauss() * p.sigma_rot;
  return s;
}

double model_at(const mrsim_phase_model& m, const double r[3], const Shot& s) {
  const double* c = m.background;
  double x = r[0], y = r[1], z = r[2];
  double bg = c[0] + c[1] * x + c[2] * y + c[3] * z + c[4] * x * x + c[5] * y * y + c[6] * z * z + c[7] * x * y +
              c[8] * x * z + c[9] * y * z;
  return m.global + bg + shot_at(s, r);
}

std::vector<double> phase_slice(const mrsim_phase_model& m, const Shot& s, size_t snx, size_t sny, size_t o, size_t z,
                                size_t nz) {
  double sxs = (double)snx / 2.0, sys = (double)sny / 2.0;
  double off = ((double)o - 1.0) / 2.0;
  double zc = (double)z - (double)nz / 2.0;
  std::vector<double> v(snx * sny);
  for (size_t y = 0; y < sny; ++y)
    for (size_t x = 0; x < snx; ++x) {
      double r[3] = {((double)x - sxs - off) / (double)o, ((double)y - sys - off) / (double)o, zc};
      v[x + snx * y] = model_at(m, r, s);
    }
  return v;
}

// ---- series: `acquire_volumes_complex` kspace.rs:1851-2125 ----
uint64_t grappa_cal_slice_seed(size_t z, uint64_t seed) {
  return ((uint64_t)z * 0x9E37ull) ^ seed ^ SEED_SALT_GRAPPA_CAL;
}

void validate_t2_volumes(const char* what, const mrsim_t2* vols, size_t ncomp, size_t nvox) {
  (void)nvox;
  for (size_t c = 0; c < ncomp; ++c) {
    if (!vols[c].is_map) continue;
    for (size_t i = 0; i < nvox; ++i) {
      float v = vols[c].map[i];
      if (std::isnan(v) || v <= 0.0f) {
        char buf[256];
        snprintf(buf, sizeof buf, "%s map for compartment %zu: T2 map value %g at index %zu is not strictly positive",
                 what, c, (double)v, i);
        throw Fail(buf);
      }
    }
  }
}

struct SeriesOut {
  std::vector<float> re, im;
  // capture
  std::vector<float> acquired, reconstructed, coil_images, combined, sensitivities;
  std::vector<uint8_t> mask;
};

SeriesOut acquire_volumes_complex(const mrsim_acquisition_input& in, const mrsim_acquisition& acq,
                                  const mrsim_acquisition_options* opts, uint64_t excitation_seed,
                                  uint64_t receiver_seed, int threads) {
  mrsim_acquisition_options dflt;
  memset(&dflt, 0, sizeof dflt);
  if (!opts) opts = &dflt;
  size_t snx = in.sim_dims[0], sny = in.sim_dims[1], nz = in.sim_dims[2];
  size_t nx = in.acq_dims[0], ny = in.acq_dims[1], nzo = in.acq_dims[2];
  size_t nv = in.n_volumes;
  if (nz != nzo) throw Fail("slice count must match; z is never oversampled");
  if (!(snx % nx == 0 && sny % ny == 0)) throw Fail("sim grid must be an integer multiple of the acquired matrix");
  size_t o = snx / nx;
  if (o != sny / ny) throw Fail("oversampling must match on both axes");
  size_t nvox_sim = snx * sny * nz, nvox_acq = nx * ny * nz;
  size_t ncomp = in.ncomp;
  validate_t2_volumes("T2", in.t2, ncomp, nvox_sim);
  if (in.t_inhom) validate_t2_volumes("T2'", in.t_inhom, ncomp, nvox_sim);
  if (!opts->t_echo_per_volume) {
    validate_acquisition_timing(acq, nx, ny);
  } else {
    for (size_t g = 0; g < nv; ++g) {
      mrsim_acquisition a = acq;
      a.t_echo = opts->t_echo_per_volume[g];
      try {
        validate_acquisition_timing(a, nx, ny);
      } catch (Fail& e) {
        throw Fail("volume " + std::to_string(g) + ": " + e.what());
      }
    }
  }
  size_t nz_full = opts->nz_full > 0 ? (size_t)opts->nz_full : nz;
  if (opts->slice_z)
    for (size_t zl = 0; zl < nz; ++zl)
      if ((size_t)opts->slice_z[zl] >= nz_full)
        throw Fail("slice_z entries must be below nz_full " + std::to_string(nz_full));
  auto global_z = [&](size_t zl) { return opts->slice_z ? (size_t)opts->slice_z[zl] : zl; };
  std::vector<size_t> captured;
  for (int64_t i = 0; i < opts->n_kspace_slices; ++i) {
    if ((size_t)opts->kspace_slices[i] >= nz)
      throw Fail("kspace_slices index " + std::to_string(opts->kspace_slices[i]) + " out of range for " +
                 std::to_string(nz) + " slices");
    captured.push_back((size_t)opts->kspace_slices[i]);
  }
  auto slice_t2 = [&](const mrsim_t2* vols, size_t zl) {
    std::vector<mrsim_t2> s(ncomp);
    for (size_t c = 0; c < ncomp; ++c) {
      s[c] = vols[c];
      if (vols[c].is_map) s[c].map = vols[c].map + zl * snx * sny;
    }
    return s;
  };
  // GRAPPA kernels: one per distinct TE per slice, kspace.rs:1906-1968
  std::vector<double> tes;
  if (opts->t_echo_per_volume)
    tes.assign(opts->t_echo_per_volume, opts->t_echo_per_volume + nv);
  else
    tes.push_back(acq.t_echo);
  std::sort(tes.begin(), tes.end());
  tes.erase(std::unique(tes.begin(), tes.end(),
                        [](double a, double b) {
                          uint64_t x, y;
                          memcpy(&x, &a, 8);
                          memcpy(&y, &b, 8);
                          return x == y;
                        }),
            tes.end());
  std::vector<std::pair<double, std::vector<GrappaKernel>>> kernels;
  if (std::max<int64_t>(acq.accel, 1) > 1 && nv > 0) {
    std::vector<std::vector<float>> owned;
    std::vector<const float*> cal(ncomp);
    uint64_t cal_seed;
    if (opts->has_grappa_calibration) {
      for (size_t c = 0; c < ncomp; ++c) cal[c] = opts->grappa_calibration_images[c];
      cal_seed = opts->grappa_calibration_seed;
    } else {
      owned.resize(ncomp);
      for (size_t c = 0; c < ncomp; ++c) {
        owned[c].resize(nvox_sim);
        for (size_t v = 0; v < nvox_sim; ++v) owned[c][v] = in.images[c][v * nv + 0];
        cal[c] = owned[c].data();
      }
      cal_seed = receiver_seed;
    }
    Shot no_shot;
    for (double te : tes) {
      mrsim_acquisition acq_cal = acq;
      acq_cal.t_echo = te;
      std::vector<GrappaKernel> ks(nz);
      parallel_for(nz, threads, [&](size_t zl) {
        size_t z = global_z(zl);
        std::vector<const float*> refs(ncomp);
        for (size_t c = 0; c < ncomp; ++c) refs[c] = cal[c] + snx * sny * zl;
        auto t2s = slice_t2(in.t2, zl);
        std::vector<mrsim_t2> tis;
        if (in.t_inhom) tis = slice_t2(in.t_inhom, zl);
        auto phi = phase_slice(*in.phase, no_shot, snx, sny, o, z, nz_full);
        mrsim_slice_input si;
        memset(&si, 0, sizeof si);
        si.compartments = refs.data();
        si.ncomp = ncomp;
        si.t2 = t2s.data();
        si.t_inhom = in.t_inhom ? tis.data() : nullptr;
        si.fmap = in.fmap + snx * sny * zl;
        si.phase0 = phi.data();
        si.sim[0] = snx;
        si.sim[1] = sny;
        si.acq_matrix[0] = nx;
        si.acq_matrix[1] = ny;
        si.z = z;
        si.nz = nz_full;
        si.slice_seed = grappa_cal_slice_seed(z, cal_seed);
        ks[zl] = grappa_reference_kernel(si, acq_cal);
      });
      kernels.emplace_back(te, std::move(ks));
    }
  }
  auto kernel_at = [&](double te, size_t zl) -> const GrappaKernel* {
    for (auto& kv : kernels) {
      uint64_t a, b;
      memcpy(&a, &kv.first, 8);
      memcpy(&b, &te, 8);
      if (a == b) return zl < kv.second.size() ? &kv.second[zl] : nullptr;
    }
    return nullptr;
  };

  SeriesOut out;
  out.re.assign(nvox_acq * nv, 0.0f);
  out.im.assign(nvox_acq * nv, 0.0f);
  size_t ncoils = std::max<int64_t>(acq.n_coils, 1);
  size_t nsl = captured.size();
  size_t per = nx * ny;
  if (nsl) {
    if (opts->capture_acquired) out.acquired.assign(nv * nsl * ncoils * per * 2, 0.0f);
    if (opts->capture_reconstructed) out.reconstructed.assign(nv * nsl * ncoils * per * 2, 0.0f);
    if (opts->capture_coil_images) out.coil_images.assign(nv * nsl * ncoils * per * 2, 0.0f);
    out.combined.assign(nv * nsl * per * 2, 0.0f);
  }
  std::mutex mu;
  parallel_for(nv, threads, [&](size_t g) {
    {
      mrsim_acquisition acq_g = acq;
      if (opts->t_echo_per_volume) acq_g.t_echo = opts->t_echo_per_volume[g];
      std::vector<std::vector<float>> cslices(ncomp, std::vector<float>(snx * sny));
      std::vector<float> fslice(snx * sny);
      for (size_t zl = 0; zl < nz; ++zl) {
        size_t z = global_z(zl);
        for (size_t y = 0; y < sny; ++y)
          for (size_t x = 0; x < snx; ++x) {
            size_t vox = x + snx * (y + sny * zl);
            for (size_t c = 0; c < ncomp; ++c) cslices[c][x + snx * y] = in.images[c][vox * nv + g];
            fslice[x + snx * y] = in.fmap[vox];
          }
        std::vector<const float*> refs(ncomp);
        for (size_t c = 0; c < ncomp; ++c) refs[c] = cslices[c].data();
        auto t2s = slice_t2(in.t2, zl);
        std::vector<mrsim_t2> tis;
        if (in.t_inhom) tis = slice_t2(in.t_inhom, zl);
        Shot shot;
        bool has_prep = in.prep_drive_set && in.prep_drive_set[g];
        if (in.phase->has_prep && has_prep)
          shot = prep_shot(*in.phase, in.prep_drive[4 * g], &in.prep_drive[4 * g + 1], g, z, excitation_seed);
        auto phi = phase_slice(*in.phase, shot, snx, sny, o, z, nz_full);
        uint64_t slice_seed = (((uint64_t)g * 0x1000001ull) + (uint64_t)z) * 0x9E37ull ^ receiver_seed;
        size_t cap_pos = nsl;
        for (size_t i = 0; i < nsl; ++i)
          if (captured[i] == zl) {
            cap_pos = i;
            break;
          }
        bool want = cap_pos < nsl;
        mrsim_slice_input si;
        memset(&si, 0, sizeof si);
        si.compartments = refs.data();
        si.ncomp = ncomp;
        si.t2 = t2s.data();
        si.t_inhom = in.t_inhom ? tis.data() : nullptr;
        si.fmap = fslice.data();
        si.phase0 = phi.data();
        si.sim[0] = snx;
        si.sim[1] = sny;
        si.acq_matrix[0] = nx;
        si.acq_matrix[1] = ny;
        si.z = z;
        si.nz = nz_full;
        bool has_eddy = in.eddy_drive_set && in.eddy_drive_set[g];
        si.has_eddy_drive = has_eddy;
        if (has_eddy)
          for (int i = 0; i < 3; ++i) si.eddy_drive[i] = in.eddy_drive[3 * g + i];
        si.has_prep_drive = has_prep;
        if (has_prep) {
          si.prep_magnitude = in.prep_drive[4 * g];
          for (int i = 0; i < 3; ++i) si.prep_direction[i] = in.prep_drive[4 * g + 1 + i];
        }
        si.slice_seed = slice_seed;
        const GrappaKernel* K = kernel_at(acq_g.t_echo, zl);
        SliceRecon r = simulate_slice_with(si, acq_g, want && opts->capture_acquired,
                                           want && opts->capture_reconstructed, want && opts->capture_coil_images,
                                           K);
        for (size_t y = 0; y < ny; ++y)
          for (size_t x = 0; x < nx; ++x) {
            Cx c = r.combined[x + nx * y];
            float re = (float)c.re, im = (float)c.im;
            size_t vox = x + nx * (y + ny * zl);
            if (in.noise_sigma) {
              double sd = (double)in.noise_sigma[vox];
              if (sd > 0.0) {
                size_t vox_g = x + nx * (y + ny * z);
                Rng rng((receiver_seed ^ ((uint64_t)g * 0x9E3779B97F4A7C15ull) ^
                         ((uint64_t)vox_g * 0xBF58476D1CE4E5B9ull)) |
                        1ull);
                re += (float)(rng.gauss() * sd);
                im += (float)(rng.gauss() * sd);
              }
            }
            out.re[vox * nv + g] = re;
            out.im[vox * nv + g] = im;
          }
        if (want) {
          size_t base = (g * nsl + cap_pos);
          auto put = [&](std::vector<float>& dst, const std::vector<std::vector<Cx>>& src) {
            for (size_t c = 0; c < ncoils; ++c)
              for (size_t i = 0; i < per; ++i) {
                dst[((base * ncoils + c) * per + i) * 2] = (float)src[c][i].re;
                dst[((base * ncoils + c) * per + i) * 2 + 1] = (float)src[c][i].im;
              }
          };
          if (opts->capture_acquired) put(out.acquired, r.acquired);
          if (opts->capture_reconstructed) put(out.reconstructed, r.reconstructed);
          if (opts->capture_coil_images) put(out.coil_images, r.coil_images);
          for (size_t i = 0; i < per; ++i) {
            out.combined[(base * per + i) * 2] = (float)r.combined[i].re;
            out.combined[(base * per + i) * 2 + 1] = (float)r.combined[i].im;
          }
          if (g == 0) {
            std::lock_guard<std::mutex> lk(mu);
            {
              out.mask = r.mask;
              out.sensitivities.resize(ncoils * per);
              for (size_t c = 0; c < ncoils; ++c)
                for (size_t i = 0; i < per; ++i) out.sensitivities[c * per + i] = (float)r.sensitivities[c][i];
            }
          }
        }
      }
    }
  });
  return out;
}

// ---- the series operator pair (no reference counterpart for the adjoint) ----
// Forward: for every (volume g, slice z, echo e, coil q) the noiseless, spike-free
// `build_coil_kspace_timed` (kspace.rs:607-1042) of the series' slice input (kspace.rs:1985-2030
// for the slice input, `echo_times` as in `simulate_acquisition_echoes` kspace.rs:2152).
// Adjoint: the FP64 transpose of that forward with respect to complex compartment images, plus
// dL/dfmap and dL/dR2_c for L = sum |k|^2 (the k-space passed in is the residual).  It uses the
// same factoring as the forward: x-stage twiddles, and per-voxel states advanced line to line by
// memoised rotors re-anchored to the closed form every 32 lines (kspace.rs:848-884).
struct SeriesSlice {
  std::vector<std::vector<float>> comps;
  std::vector<const float*> refs;
  std::vector<float> fmap;
  std::vector<double> phi;
  std::vector<mrsim_t2> t2s, tis;
  mrsim_slice_input si;
};

SeriesSlice series_slice(const mrsim_acquisition_input& in, size_t g, size_t zl, size_t nz_full, const int64_t* slice_z,
                         uint64_t seed) {
  size_t snx = in.sim_dims[0], sny = in.sim_dims[1], nz = in.sim_dims[2];
  size_t nv = in.n_volumes, ncomp = in.ncomp, o = snx / in.acq_dims[0];
  size_t z = slice_z ? (size_t)slice_z[zl] : zl;
  SeriesSlice S;
  S.comps.assign(ncomp, std::vector<float>(snx * sny));
  S.fmap.resize(snx * sny);
  for (size_t p = 0; p < snx * sny; ++p) {
    size_t vox = p + snx * sny * zl;
    for (size_t c = 0; c < ncomp; ++c) S.comps[c][p] = in.images[c][vox * nv + g];
    S.fmap[p] = in.fmap[vox];
  }
  for (auto& c : S.comps) S.refs.push_back(c.data());
  S.t2s.resize(ncomp);
  for (size_t c = 0; c < ncomp; ++c) {
    S.t2s[c] = in.t2[c];
    if (in.t2[c].is_map) S.t2s[c].map = in.t2[c].map + zl * snx * sny;
  }
  if (in.t_inhom) {
    S.tis.resize(ncomp);
    for (size_t c = 0; c < ncomp; ++c) {
      S.tis[c] = in.t_inhom[c];
      if (in.t_inhom[c].is_map) S.tis[c].map = in.t_inhom[c].map + zl * snx * sny;
    }
  }
  Shot shot;
  bool has_prep = in.prep_drive_set && in.prep_drive_set[g];
  if (in.phase && in.phase->has_prep && has_prep)
    shot = prep_shot(*in.phase, in.prep_drive[4 * g], &in.prep_drive[4 * g + 1], g, z, seed);
  mrsim_phase_model zero;
  memset(&zero, 0, sizeof zero);
  S.phi = phase_slice(in.phase ? *in.phase : zero, shot, snx, sny, o, z, nz_full);
  (void)nz;
  memset(&S.si, 0, sizeof S.si);
  S.si.compartments = S.refs.data();
  S.si.ncomp = ncomp;
  S.si.t2 = S.t2s.data();
  S.si.t_inhom = in.t_inhom ? S.tis.data() : nullptr;
  S.si.fmap = S.fmap.data();
  S.si.phase0 = S.phi.data();
  S.si.sim[0] = snx;
  S.si.sim[1] = sny;
  S.si.acq_matrix[0] = in.acq_dims[0];
  S.si.acq_matrix[1] = in.acq_dims[1];
  S.si.z = z;
  S.si.nz = nz_full;
  bool has_eddy = in.eddy_drive_set && in.eddy_drive_set[g];
  S.si.has_eddy_drive = has_eddy;
  if (has_eddy)
    for (int i = 0; i < 3; ++i) S.si.eddy_drive[i] = in.eddy_drive[3 * g + i];
  return S;
}

void series_forward(const mrsim_acquisition_input& in, const mrsim_acquisition& acq0, const double* tes, size_t ne,
                    const int64_t* slice_z, size_t nz_full, int threads, double* out) {
  size_t nx = in.acq_dims[0], ny = in.acq_dims[1], nz = in.sim_dims[2], nv = in.n_volumes;
  size_t nc = std::max<int64_t>(acq0.n_coils, 1);
  if (nz_full == 0) nz_full = nz;
  parallel_for(nv * nz, threads, [&](size_t u) {
    size_t g = u / nz, zl = u % nz;
    SeriesSlice S = series_slice(in, g, zl, nz_full, slice_z, in.seed);
    for (size_t e = 0; e < ne; ++e) {
      mrsim_acquisition a = acq0;
      a.t_echo = tes ? tes[e] : acq0.t_echo;
      a.noise_variance = 0.0;
      a.n_spikes = 0;
      LineTiming lt = line_timing_for(a, nx, ny);
      for (size_t q = 0; q < nc; ++q) {
        auto k = build_coil_kspace_timed(S.si, a, q, nc, lt, nullptr);
        double* dst = out + 2 * (((u * nc + q) * ne + e) * ny * nx);
        for (size_t i = 0; i < nx * ny; ++i) {
          dst[2 * i] = k[i].re;
          dst[2 * i + 1] = k[i].im;
        }
      }
    }
  });
}

// Adjoint of one (unit, echo, coil): accumulates into cg [c][p] (complex), U, V [c][p] (complex).
void unit_adjoint(const mrsim_slice_input& inp, const mrsim_acquisition& acq, size_t coil, size_t ncoils,
                  const LineTiming& timing, const double* r, std::vector<Cx>& cg, std::vector<Cx>& U,
                  std::vector<Cx>& V) {
  size_t snx = inp.sim[0], sny = inp.sim[1], nx = inp.acq_matrix[0], ny = inp.acq_matrix[1];
  size_t ncomp = inp.ncomp, nvox = snx * sny;
  size_t z = inp.z, nz = inp.nz;
  double gradient[3] = {0, 0, 0};
  if (inp.has_eddy_drive)
    for (int i = 0; i < 3; ++i) gradient[i] = inp.eddy_drive[i];
  bool do_eddy = eddy_enabled(acq, inp);
  bool do_eddy_phase = acq.eddy_phase != 0.0 && inp.has_eddy_drive;
  size_t xs = nx / 2, ys = ny / 2, zs = nz / 2;
  size_t ox = snx / nx, oy = sny / ny, sxs = ox * xs, sys = oy * ys;
  double xoff = ((double)ox - 1.0) / 2.0, yoff = ((double)oy - 1.0) / 2.0;
  auto mask = sampling_mask(nx, ny, acq);
  double zc = (double)z - (double)zs, zc_c = (double)z - ((double)nz - 1.0) / 2.0;
  std::vector<double> amp(nvox), phi0(nvox), rate(nvox);
  for (size_t y = 0; y < sny; ++y)
    for (size_t x = 0; x < snx; ++x) {
      size_t i = x + snx * y;
      amp[i] = acq.signal_scale *
               coil_sensitivity(coil, ncoils, ((double)x - xoff) / (double)ox, ((double)y - yoff) / (double)oy, nx, ny);
      double xc = ((double)x - (double)sxs - xoff) / (double)ox, yc = ((double)y - (double)sys - yoff) / (double)oy;
      double p0 = inp.phase0 ? inp.phase0[i] : 0.0;
      if (do_eddy_phase) p0 += acq.eddy_phase * (gradient[0] * xc + gradient[1] * yc + gradient[2] * zc_c);
      if (acq.echo == MRSIM_ECHO_GRADIENT && acq.do_distortions) p0 += TAU * (double)inp.fmap[i] * (acq.t_echo / 1000.0);
      phi0[i] = p0;
      rate[i] = acq.do_distortions ? (double)inp.fmap[i] : 0.0;
    }
  XStage xst(snx, nx, xs, sxs, xoff, acq.ghost_offset);
  double n_inv = 1.0 / (double)nvox;
  std::vector<Cx> h(snx);
  std::vector<Cx> st(nvox);
  auto set_state = [&](size_t kyi) {
    double t = timing.t_ms[kyi] / 1000.0;
    double kyn = ((double)kyi - (double)ys) / (double)sny;
    for (size_t y = 0; y < sny; ++y) {
      double yy = (double)y - (double)sys - yoff;
      for (size_t x = 0; x < snx; ++x) {
        size_t i = x + snx * y;
        double ph = phi0[i] + TAU * (rate[i] * t + kyn * yy);
        st[i] = {amp[i] * std::cos(ph), amp[i] * std::sin(ph)};
      }
    }
  };
  struct ARotor {
    size_t k0, k1;
    double dt, dkyn;
    std::vector<Cx> rot;
  };
  std::vector<ARotor> rotors;
  bool have_prev = false;
  size_t prev = 0, since_anchor = 0;
  bool rel_uniform = true;
  for (size_t c = 0; c < ncomp; ++c) rel_uniform = rel_uniform && !inp.t2[c].is_map;
  if (inp.t_inhom)
    for (size_t c = 0; c < ncomp; ++c) rel_uniform = rel_uniform && !inp.t_inhom[c].is_map;
  for (size_t kyi = 0; kyi < ny; ++kyi) {
    if (!mask[nx * kyi]) continue;
    double t = timing.t_ms[kyi] / 1000.0, trf = timing.trf_ms[kyi];
    double tph = acq.echo == MRSIM_ECHO_SPIN ? t : t + acq.t_echo / 1000.0;
    double kyn = ((double)kyi - (double)ys) / (double)sny;
    double ghost_shift = timing.polarity[kyi] < 0 ? -acq.ghost_offset : acq.ghost_offset;
    const std::vector<Cx>& tw = xst.tw[ghost_shift < 0.0 ? 1 : 0];
    double eddy_decay = do_eddy ? std::exp(-timing.tread_ms[kyi] / acq.eddy_tau) * t : 0.0;
    // x-adjoint: h[x] = (1/N) conj(E(x)) sum_kx conj(tw[kx][x]) r[kx]
    for (size_t x = 0; x < snx; ++x) {
      double ar = 0.0, ai = 0.0;
      for (size_t kx = 0; kx < nx; ++kx) {
        Cx w = tw[snx * kx + x];
        double rr = r[2 * (kx + nx * kyi)], ri = r[2 * (kx + nx * kyi) + 1];
        ar += w.re * rr + w.im * ri;
        ai += w.re * ri - w.im * rr;
      }
      Cx v = {ar * n_inv, ai * n_inv};
      if (do_eddy) {
        double xc = ((double)x - (double)sxs - xoff) / (double)ox;
        double ph = TAU * ((acq.eddy_strength * gradient[0] * xc + acq.eddy_quad * gradient[0] * xc * xc) +
                           (acq.eddy_strength * gradient[2] * zc + acq.eddy_quad * gradient[2] * zc * zc)) *
                    eddy_decay;
        v = cmul(v, Cx{std::cos(ph), -std::sin(ph)});
      }
      h[x] = v;
    }
    // advance the per-voxel state amp*e^{i(phi0 + 2pi(rate t + kyn yy))} to this line: closed form
    // on the first line and every REANCHOR lines, else a memoised rotor (kspace.rs:848-884)
    if (have_prev && since_anchor < 32) {
      size_t p = prev, k0 = kyi - p, k1 = p % 2;
      double dt = t - timing.t_ms[p] / 1000.0;
      double dkyn = kyn - (((double)p - (double)ys) / (double)sny);
      size_t idx = rotors.size();
      for (size_t rr = 0; rr < rotors.size(); ++rr)
        if (rotors[rr].k0 == k0 && rotors[rr].k1 == k1) {
          idx = rr;
          break;
        }
      if (idx == rotors.size()) {
        ARotor R{k0, k1, dt, dkyn, std::vector<Cx>(nvox)};
        for (size_t y = 0; y < sny; ++y) {
          double yy = (double)y - (double)sys - yoff;
          for (size_t x = 0; x < snx; ++x) {
            size_t i = x + snx * y;
            double ph = TAU * (rate[i] * dt + dkyn * yy);
            R.rot[i] = {std::cos(ph), std::sin(ph)};
          }
        }
        rotors.push_back(std::move(R));
      }
      const ARotor& R = rotors[idx];
      if (std::fabs(R.dt - dt) <= 1e-12 * std::max(std::fabs(dt), 1e-300) && R.dkyn == dkyn) {
        for (size_t i = 0; i < nvox; ++i) st[i] = cmul(st[i], R.rot[i]);
        since_anchor += 1;
      } else {
        set_state(kyi);
        since_anchor = 0;
      }
    } else {
      set_state(kyi);
      since_anchor = 0;
    }
    prev = kyi;
    have_prev = true;
    bool uniform = rel_uniform;
    std::vector<double> rl(ncomp, 1.0);
    if (uniform && acq.do_relaxation)
      for (size_t c = 0; c < ncomp; ++c) {
        double tic = inp.t_inhom ? (double)inp.t_inhom[c].value : acq.t_inhom;
        double inh = acq.echo == MRSIM_ECHO_SPIN ? std::fabs(t) * 1000.0 : trf;
        rl[c] = std::exp(-trf / (double)inp.t2[c].value - inh / tic);
      }
    for (size_t y = 0; y < sny; ++y) {
      Cx eyc = {1.0, 0.0};
      if (do_eddy) {
        double yc = ((double)y - (double)sys - yoff) / (double)oy;
        double eyph = TAU * (acq.eddy_strength * gradient[1] * yc + acq.eddy_quad * gradient[1] * yc * yc) * eddy_decay;
        eyc = {std::cos(eyph), std::sin(eyph)};
      }
      for (size_t x = 0; x < snx; ++x) {
        size_t i = x + snx * y;
        Cx sv = do_eddy ? cmul(st[i], eyc) : st[i];
        // Z = conj(state) h
        Cx Z = cmul(Cx{sv.re, -sv.im}, h[x]);
        for (size_t c = 0; c < ncomp; ++c) {
          double r_ = rl[c];
          if (!uniform && acq.do_relaxation) {
            double t2c = t2_value(inp.t2[c], i);
            double tic = inp.t_inhom ? t2_value(inp.t_inhom[c], i) : acq.t_inhom;
            double inh = acq.echo == MRSIM_ECHO_SPIN ? std::fabs(t) * 1000.0 : trf;
            r_ = std::exp(-trf / t2c - inh / tic);
          }
          size_t k = c * nvox + i;
          cg[k] = cadd(cg[k], cscale(Z, r_));
          U[k] = cadd(U[k], cscale(Z, r_ * tph));
          V[k] = cadd(V[k], cscale(Z, r_ * trf));
        }
      }
    }
  }
}

void series_adjoint(const mrsim_acquisition_input& in, const mrsim_acquisition& acq0, const double* tes, size_t ne,
                    const int64_t* slice_z, size_t nz_full, int threads, const double* kspace, double* comp_grad,
                    double* fmap_grad, double* r2_grad) {
  size_t snx = in.sim_dims[0], sny = in.sim_dims[1], nx = in.acq_dims[0], ny = in.acq_dims[1], nz = in.sim_dims[2];
  size_t nv = in.n_volumes, ncomp = in.ncomp, nvox = snx * sny;
  size_t nc = std::max<int64_t>(acq0.n_coils, 1);
  if (nz_full == 0) nz_full = nz;
  parallel_for(nv * nz, threads, [&](size_t u) {
    size_t g = u / nz, zl = u % nz;
    SeriesSlice S = series_slice(in, g, zl, nz_full, slice_z, in.seed);
    std::vector<Cx> cg(ncomp * nvox, CZERO), U(ncomp * nvox, CZERO), V(ncomp * nvox, CZERO);
    for (size_t e = 0; e < ne; ++e) {
      mrsim_acquisition a = acq0;
      a.t_echo = tes ? tes[e] : acq0.t_echo;
      LineTiming lt = line_timing_for(a, nx, ny);
      for (size_t q = 0; q < nc; ++q)
        unit_adjoint(S.si, a, q, nc, lt, kspace + 2 * (((u * nc + q) * ne + e) * ny * nx), cg, U, V);
    }
    for (size_t c = 0; c < ncomp; ++c)
      for (size_t p = 0; p < nvox; ++p) {
        size_t k = c * nvox + p;
        comp_grad[2 * (u * ncomp * nvox + k)] = cg[k].re;
        comp_grad[2 * (u * ncomp * nvox + k) + 1] = cg[k].im;
        if (r2_grad) r2_grad[u * ncomp * nvox + k] = -2.0 * (double)S.comps[c][p] * V[k].re;
      }
    if (fmap_grad)
      for (size_t p = 0; p < nvox; ++p) {
        double fg = 0.0;
        for (size_t c = 0; c < ncomp; ++c) fg += (double)S.comps[c][p] * U[c * nvox + p].im;
        fmap_grad[u * nvox + p] = acq0.do_distortions ? 2.0 * TAU * fg : 0.0;
      }
  });
}

// ---- golden record: tests/golden_baseline.rs:28-126 ----
struct GoldenCase {
  std::string name;
  std::vector<uint32_t> bits;
};

mrsim_acquisition acq_default() {
  mrsim_acquisition a;
  memset(&a, 0, sizeof a);
  a.t_line = 1.0;
  a.t_echo = 90.0;
  a.t_inhom = 50.0;
  a.signal_scale = 100.0;
  a.reverse_phase = 0;
  a.do_distortions = 1;
  a.do_relaxation = 1;
  a.noise_variance = 0.0;
  a.partial_fourier = 1.0;
  a.pf_mode = MRSIM_PF_FIBERFOX;
  a.ghost_offset = 0.0;
  a.eddy_strength = 0.0;
  a.eddy_quad = 0.0;
  a.eddy_phase = 0.0;
  a.eddy_tau = 70.0;
  a.n_spikes = 0;
  a.spike_amplitude = 1.0;
  a.window_kind = MRSIM_WINDOW_NONE;
  a.n_coils = 1;
  a.accel = 1;
  a.acs_lines = 24;
  a.seed = 0;
  a.echo = MRSIM_ECHO_SPIN;
  return a;
}

uint32_t f32bits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}

std::vector<GoldenCase> golden_outputs() {
  std::vector<GoldenCase> out;
  Rng rng(0xC0FFEE);
  const size_t geo[3][3] = {{17, 70, 2}, {16, 40, 1}, {8, 9, 3}};
  for (auto& gm : geo) {
    size_t nx = gm[0], ny = gm[1], o = gm[2];
    size_t snx = nx * o, sny = ny * o, n = snx * sny;
    std::vector<std::vector<float>> comps(3, std::vector<float>(n));
    for (size_t c = 0; c < 3; ++c)
      for (size_t i = 0; i < n; ++i) {
        double x = (double)(i % snx) / (double)snx, y = (double)(i / snx) / (double)sny;
        double a = x - 0.5, b = y - 0.45;
        double blob = std::exp(-((a * a + b * b) / (0.03 * (double)(c + 1))));
        comps[c][i] = (float)(blob + 0.05 * rng.unit());
      }
    std::vector<float> fmap(n);
    for (size_t i = 0; i < n; ++i) {
      double x = (double)(i % snx) / (double)snx, y = (double)(i / snx) / (double)sny;
      fmap[i] = (float)(300.0 * (std::sin(3.0 * x) * std::cos(2.0 * y + 1.0)) + 20.0 * rng.unit());
    }
    std::vector<double> phase0(n);
    for (size_t i = 0; i < n; ++i) phase0[i] = TAU * rng.unit();
    std::vector<float> t2map(n), timap(n);
    for (size_t i = 0; i < n; ++i) {
      t2map[i] = (float)(60.0 + 80.0 * ((double)(i % snx) / (double)snx));
      timap[i] = (float)(30.0 + 40.0 * ((double)(i / snx) / (double)sny));
    }
    mrsim_acquisition full = acq_default();
    full.do_distortions = 1;
    full.do_relaxation = 1;
    full.signal_scale = 100.0;
    mrsim_t2 uniform[3] = {{nullptr, 70.0f, 0}, {nullptr, 100.0f, 0}, {nullptr, 2000.0f, 0}};
    mrsim_t2 mapped[3] = {{t2map.data(), 0.0f, 1}, {nullptr, 100.0f, 0}, {t2map.data(), 0.0f, 1}};
    mrsim_t2 ti_mapped[3] = {{timap.data(), 0.0f, 1}, {nullptr, 45.0f, 0}, {timap.data(), 0.0f, 1}};
    struct Case {
      const char* name;
      mrsim_acquisition a;
      bool has_eddy;
      double eddy[3];
      bool maps;
    };
    std::vector<Case> cases;
    auto mk = [&](const char* name) {
      Case c;
      c.name = name;
      c.a = full;
      c.has_eddy = false;
      c.eddy[0] = c.eddy[1] = c.eddy[2] = 0;
      c.maps = false;
      return c;
    };
    {
      Case c = mk("clean");
      c.a.do_distortions = 0;
      c.a.do_relaxation = 0;
      cases.push_back(c);
    }
    cases.push_back(mk("distortion+relaxation"));
    {
      Case c = mk("reverse");
      c.a.reverse_phase = 1;
      cases.push_back(c);
    }
    {
      Case c = mk("ghost");
      c.a.ghost_offset = 0.015;
      cases.push_back(c);
    }
    {
      Case c = mk("eddy-poly");
      c.a.eddy_strength = 3.0;
      c.a.eddy_quad = 0.4;
      c.a.eddy_tau = 70.0;
      c.has_eddy = true;
      c.eddy[0] = 0.3;
      c.eddy[1] = -0.8;
      c.eddy[2] = 0.5;
      cases.push_back(c);
    }
    {
      Case c = mk("eddy-phase");
      c.a.eddy_phase = 0.2;
      c.has_eddy = true;
      c.eddy[0] = 0.6;
      c.eddy[1] = 0.6;
      c.eddy[2] = 0.5;
      cases.push_back(c);
    }
    {
      Case c = mk("pf-fiberfox");
      c.a.partial_fourier = 0.75;
      cases.push_back(c);
    }
    {
      Case c = mk("pf-contiguous-reverse");
      c.a.partial_fourier = 0.75;
      c.a.pf_mode = MRSIM_PF_CONTIGUOUS;
      c.a.reverse_phase = 1;
      cases.push_back(c);
    }
    {
      Case c = mk("grappa-coils");
      c.a.accel = 2;
      c.a.acs_lines = 6;
      c.a.n_coils = 4;
      cases.push_back(c);
    }
    {
      Case c = mk("grappa3");
      c.a.accel = 3;
      c.a.acs_lines = 8;
      c.a.n_coils = 4;
      cases.push_back(c);
    }
    {
      Case c = mk("everything");
      c.a.ghost_offset = 0.02;
      c.a.eddy_strength = 2.0;
      c.a.eddy_quad = 0.3;
      c.a.eddy_phase = 0.1;
      c.a.partial_fourier = 0.8;
      c.a.accel = 2;
      c.a.acs_lines = 8;
      c.a.n_coils = 3;
      c.has_eddy = true;
      c.eddy[0] = 0.5;
      c.eddy[1] = 0.5;
      c.eddy[2] = 0.7;
      cases.push_back(c);
    }
    {
      Case c = mk("maps");
      c.maps = true;
      cases.push_back(c);
    }
    {
      Case c = mk("maps-coils-noise");
      c.a.n_coils = 3;
      c.a.noise_variance = 4.0;
      c.maps = true;
      cases.push_back(c);
    }
    std::vector<const float*> refs = {comps[0].data(), comps[1].data(), comps[2].data()};
    for (auto& cs : cases) {
      mrsim_slice_input si;
      memset(&si, 0, sizeof si);
      si.compartments = refs.data();
      si.ncomp = 3;
      si.t2 = cs.maps ? mapped : uniform;
      si.t_inhom = cs.maps ? ti_mapped : nullptr;
      si.fmap = fmap.data();
      si.phase0 = phase0.data();
      si.sim[0] = snx;
      si.sim[1] = sny;
      si.acq_matrix[0] = nx;
      si.acq_matrix[1] = ny;
      si.z = 3;
      si.nz = 9;
      si.has_eddy_drive = cs.has_eddy;
      for (int i = 0; i < 3; ++i) si.eddy_drive[i] = cs.eddy[i];
      si.slice_seed = 7;
      SliceRecon r = simulate_slice_with(si, cs.a, false, false, false, nullptr);
      GoldenCase g;
      g.name = "slice-" + std::to_string(nx) + "x" + std::to_string(ny) + "o" + std::to_string(o) + "-" + cs.name;
      for (auto& c : r.combined) {
        g.bits.push_back(f32bits((float)c.re));
        g.bits.push_back(f32bits((float)c.im));
      }
      out.push_back(std::move(g));
    }
  }
  // the two series cases
  {
    size_t nx = 16, ny = 16, nz = 3, o = 2, nv = 4;
    size_t snx = nx * o, sny = ny * o, nsim = snx * sny * nz;
    Rng r2(0xBA5E);
    std::vector<std::vector<float>> images(2);
    for (size_t c = 0; c < 2; ++c) {
      std::vector<float> byv(nsim * nv);
      for (size_t i = 0; i < nsim * nv; ++i) {
        size_t v = i / nsim, vox = i % nsim;
        double x = (double)(vox % snx) / (double)snx, y = (double)((vox / snx) % sny) / (double)sny;
        double a = x - 0.5, b = y - 0.5;
        double blob = std::exp(-((a * a + b * b) / 0.05));
        byv[i] = (float)((1.0 + 0.1 * (double)c + 0.01 * (double)v) * blob + 0.02 * r2.unit());
      }
      images[c].resize(nsim * nv);
      for (size_t g = 0; g < nv; ++g)
        for (size_t vox = 0; vox < nsim; ++vox) images[c][vox * nv + g] = byv[g * nsim + vox];
    }
    std::vector<float> fmap(nsim), t2map(nsim);
    for (size_t i = 0; i < nsim; ++i) {
      fmap[i] = (float)(40.0 * ((double)(i % snx) / (double)snx - 0.5));
      t2map[i] = (float)(50.0 + (double)(i % 7) * 10.0);
    }
    mrsim_acquisition a = acq_default();
    a.n_coils = 3;
    a.accel = 2;
    a.acs_lines = 6;
    a.noise_variance = 2.0;
    a.signal_scale = 100.0;
    a.t_echo = 30.0;
    a.t_line = 0.5;
    mrsim_phase_model pm;
    memset(&pm, 0, sizeof pm);
    pm.background[1] = 0.13;
    pm.background[2] = 0.10;
    pm.background[3] = 0.02;
    pm.has_prep = 1;
    pm.c_q = 0.0425;
    pm.sigma_dx = 1.0;
    pm.sigma_rot = 2.0e-3;
    mrsim_t2 tu[2] = {{nullptr, 80.0f, 0}, {nullptr, 160.0f, 0}};
    mrsim_t2 tm[2] = {{t2map.data(), 0.0f, 1}, {nullptr, 160.0f, 0}};
    const char* names[2] = {"series-uniform", "series-mapped"};
    std::vector<const float*> imgs = {images[0].data(), images[1].data()};
    for (int k = 0; k < 2; ++k) {
      mrsim_acquisition_input in;
      memset(&in, 0, sizeof in);
      in.sim_dims[0] = snx;
      in.sim_dims[1] = sny;
      in.sim_dims[2] = nz;
      in.acq_dims[0] = nx;
      in.acq_dims[1] = ny;
      in.acq_dims[2] = nz;
      in.n_volumes = nv;
      in.ncomp = 2;
      in.images = imgs.data();
      in.t2 = k == 0 ? tu : tm;
      in.fmap = fmap.data();
      in.phase = &pm;
      in.seed = 42;
      SeriesOut so = acquire_volumes_complex(in, a, nullptr, 42, 42, 1);
      GoldenCase g;
      g.name = names[k];
      size_t nn = so.re.size();
      std::vector<uint32_t> mag(nn), ph(nn);
      for (size_t i = 0; i < nn; ++i) {
        float re = so.re[i], im = so.im[i];
        mag[i] = f32bits(std::sqrt(re * re + im * im));
        ph[i] = f32bits(std::atan2(im, re));
      }
      g.bits = mag;
      g.bits.insert(g.bits.end(), ph.begin(), ph.end());
      out.push_back(std::move(g));
    }
  }
  return out;
}



// ---- FFT (the reference calls rustfft): radix-2 for powers of two, else the direct DFT; the
// same unnormalized transform e^{sign i2pi jk/n}, within rounding ----
void fft1d(std::vector<Cx>& a, int sign) {
  const size_t n = a.size();
  if (n <= 1) return;
  if ((n & (n - 1)) != 0) {
    std::vector<Cx> out(n);
    for (size_t k = 0; k < n; ++k) {
      Cx acc{0.0, 0.0};
      for (size_t j = 0; j < n; ++j) acc = cadd(acc, cmul(a[j], ccis((double)sign * TAU * (double)((j * k) % n) / (double)n)));
      out[k] = acc;
    }
    a = out;
    return;
  }
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    for (size_t i = 0; i < n; i += len)
      for (size_t k = 0; k < len / 2; ++k) {
        Cx w = ccis((double)sign * TAU * (double)k / (double)len);
        Cx u = a[i + k], v = cmul(a[i + k + len / 2], w);
        a[i + k] = cadd(u, v);
        a[i + k + len / 2] = {u.re - v.re, u.im - v.im};
      }
  }
}

void fft2d(std::vector<Cx>& g, size_t n0, size_t n1, int sign) {
  std::vector<Cx> line(n0);
  for (size_t l = 0; l < n1; ++l) {
    for (size_t i = 0; i < n0; ++i) line[i] = g[i + n0 * l];
    fft1d(line, sign);
    for (size_t i = 0; i < n0; ++i) g[i + n0 * l] = line[i];
  }
  line.resize(n1);
  for (size_t l = 0; l < n0; ++l) {
    for (size_t i = 0; i < n1; ++i) line[i] = g[l + n0 * i];
    fft1d(line, sign);
    for (size_t i = 0; i < n1; ++i) g[l + n0 * i] = line[i];
  }
}

// ============================ stack-of-spirals path =========================================
// `Nufft2` nufft.rs:125-299, FP64.  The fine-grid transform is a separable direct DFT (the
// reference calls rustfft; a DFT is the same linear map, within rounding).
struct Nufft2O {
  size_t n[2], nf[2], w;
  double beta;
  int64_t m_lo[2];
  size_t m_out[2];
  std::vector<double> corr[2];
  Nufft2O(const int64_t* n_, const int64_t* m_lo_, const int64_t* m_out_, double tol) {
    for (int a = 0; a < 2; ++a) {
      if (!(m_out_[a] > 0 && m_lo_[a] >= -(n_[a] / 2) && m_lo_[a] + m_out_[a] - 1 <= n_[a] / 2))
        throw Fail("mode band must sit inside the coarse Nyquist band");
      n[a] = (size_t)n_[a];
      nf[a] = 2 * n[a];
      m_lo[a] = m_lo_[a];
      m_out[a] = (size_t)m_out_[a];
    }
    w = (size_t)std::min(16.0, std::max(2.0, std::ceil(-std::log10(tol)) + 1.0));
    beta = 2.30 * (double)w;
    for (int a = 0; a < 2; ++a) {  // `deapodization` nufft.rs:113-123
      double half = (double)w / 2.0;
      for (size_t j = 0; j < m_out[a]; ++j) {
        double k = (double)(m_lo[a] + (int64_t)j);
        double s = psi(0.0);
        for (double m = 1.0; m < half; m += 1.0) s += 2.0 * psi(m / half) * std::cos(TAU * k * m / (double)nf[a]);
        corr[a].push_back(1.0 / s);
      }
    }
  }
  double psi(double z) const { return std::fabs(z) < 1.0 ? std::exp(beta * (std::sqrt(1.0 - z * z) - 1.0)) : 0.0; }
  int64_t kernel(int a, double u, double* k) const {  // nufft.rs:196-205
    double half = (double)w / 2.0;
    double p = std::fmod(2.0 * u, (double)nf[a]);
    if (p < 0.0) p += (double)nf[a];
    if (p >= (double)nf[a]) p -= (double)nf[a];
    int64_t m0 = (int64_t)std::floor(p - half) + 1;
    for (size_t i = 0; i < w; ++i) k[i] = psi(((double)m0 + (double)i - p) / half);
    return m0;
  }
  static size_t wrap(int64_t m, size_t n) {
    int64_t r = m % (int64_t)n;
    return (size_t)(r < 0 ? r + (int64_t)n : r);
  }
  void dft2(std::vector<Cx>& g, int sign) const { fft2d(g, nf[0], nf[1], sign); }  // nufft.rs:209-229
  std::vector<Cx> type1(const double* u, size_t npts, const Cx* wts, int sign) const {  // nufft.rs:236-262
    std::vector<Cx> g(nf[0] * nf[1], Cx{0.0, 0.0});
    std::vector<double> k0(w), k1(w);
    for (size_t j = 0; j < npts; ++j) {
      int64_t a0 = kernel(0, u[2 * j], k0.data()), a1 = kernel(1, u[2 * j + 1], k1.data());
      for (size_t i1 = 0; i1 < w; ++i1) {
        size_t c1 = wrap(a1 + (int64_t)i1, nf[1]);
        for (size_t i0 = 0; i0 < w; ++i0) {
          size_t c0 = wrap(a0 + (int64_t)i0, nf[0]);
          double v = k0[i0] * k1[i1];
          g[c0 + nf[0] * c1].re += wts[j].re * v;
          g[c0 + nf[0] * c1].im += wts[j].im * v;
        }
      }
    }
    dft2(g, sign);
    std::vector<Cx> out;
    for (size_t j1 = 0; j1 < m_out[1]; ++j1)
      for (size_t j0 = 0; j0 < m_out[0]; ++j0) {
        size_t b0 = wrap(m_lo[0] + (int64_t)j0, nf[0]), b1 = wrap(m_lo[1] + (int64_t)j1, nf[1]);
        out.push_back(cscale(g[b0 + nf[0] * b1], corr[0][j0] * corr[1][j1]));
      }
    return out;
  }
  std::vector<Cx> type2(const Cx* c, const double* u, size_t npts, int sign) const {  // nufft.rs:265-292
    std::vector<Cx> g(nf[0] * nf[1], Cx{0.0, 0.0});
    for (size_t j1 = 0; j1 < m_out[1]; ++j1)
      for (size_t j0 = 0; j0 < m_out[0]; ++j0) {
        size_t b0 = wrap(m_lo[0] + (int64_t)j0, nf[0]), b1 = wrap(m_lo[1] + (int64_t)j1, nf[1]);
        g[b0 + nf[0] * b1] = cscale(c[j0 + m_out[0] * j1], corr[0][j0] * corr[1][j1]);
      }
    dft2(g, sign);
    std::vector<Cx> out(npts);
    std::vector<double> k0(w), k1(w);
    for (size_t j = 0; j < npts; ++j) {
      int64_t a0 = kernel(0, u[2 * j], k0.data()), a1 = kernel(1, u[2 * j + 1], k1.data());
      double re = 0.0, im = 0.0;
      for (size_t i1 = 0; i1 < w; ++i1) {
        size_t c1 = wrap(a1 + (int64_t)i1, nf[1]);
        for (size_t i0 = 0; i0 < w; ++i0) {
          size_t c0 = wrap(a0 + (int64_t)i0, nf[0]);
          double v = k0[i0] * k1[i1];
          re += g[c0 + nf[0] * c1].re * v;
          im += g[c0 + nf[0] * c1].im * v;
        }
      }
      out[j] = {re, im};
    }
    return out;
  }
};

// The literal sums the reference pins `Nufft2` against (nufft.rs:370-445).
std::vector<Cx> nufft2_direct(int type, const int64_t* n, const int64_t* m_lo, const int64_t* m_out, const double* u,
                              size_t npts, const Cx* in, int sign) {
  size_t nm = (size_t)(m_out[0] * m_out[1]);
  std::vector<Cx> out(type == 1 ? nm : npts, Cx{0.0, 0.0});
  for (size_t j = 0; j < npts; ++j)
    for (int64_t j1 = 0; j1 < m_out[1]; ++j1)
      for (int64_t j0 = 0; j0 < m_out[0]; ++j0) {
        double m0 = (double)(m_lo[0] + j0), m1 = (double)(m_lo[1] + j1);
        Cx e = ccis((double)sign * TAU * (u[2 * j] * m0 / (double)n[0] + u[2 * j + 1] * m1 / (double)n[1]));
        size_t mi = (size_t)(j0 + m_out[0] * j1);
        if (type == 1)
          out[mi] = cadd(out[mi], cmul(in[j], e));
        else
          out[j] = cadd(out[j], cmul(in[mi], e));
      }
  return out;
}

// `statics`, `decay_rate`, `spiral_kspace_exact` spiral.rs:33-137.
double spiral_decay_rate(const mrsim_slice_input& inp, const mrsim_acquisition& acq, size_t c, size_t i) {
  double t2 = t2_value(inp.t2[c], i);
  double tp = inp.t_inhom ? t2_value(inp.t_inhom[c], i) : acq.t_inhom;
  return 1.0 / t2 + 1.0 / tp;
}

std::vector<Cx> spiral_kspace_exact(const mrsim_slice_input& inp, const mrsim_acquisition& acq, size_t coil,
                                    size_t ncoils, const double* k, const double* tau, size_t npts,
                                    const double* log_amp) {
  size_t snx = inp.sim[0], sny = inp.sim[1], nx = inp.acq_matrix[0], ny = inp.acq_matrix[1];
  if (!(snx % nx == 0 && sny % ny == 0)) throw Fail("sim grid must be an integer multiple of the acquired matrix");
  if (acq.echo != MRSIM_ECHO_SPIN) throw Fail("the spiral train is a spin-echo train");
  size_t ox = snx / nx, oy = sny / ny, sxs = ox * (nx / 2), sys = oy * (ny / 2);
  double xoff = ((double)ox - 1.0) / 2.0, yoff = ((double)oy - 1.0) / 2.0;
  size_t n = snx * sny;
  std::vector<double> amp(n), phi0(n), xc(n), yc(n), rate(n);
  for (size_t y = 0; y < sny; ++y)
    for (size_t x = 0; x < snx; ++x) {
      size_t i = x + snx * y;
      double xa = ((double)x - xoff) / (double)ox, ya = ((double)y - yoff) / (double)oy;
      amp[i] = acq.signal_scale * coil_sensitivity(coil, ncoils, xa, ya, nx, ny);
      xc[i] = ((double)x - (double)sxs - xoff) / (double)ox;
      yc[i] = ((double)y - (double)sys - yoff) / (double)oy;
      phi0[i] = inp.phase0 ? inp.phase0[i] : 0.0;
      rate[i] = acq.do_distortions ? (double)inp.fmap[i] : 0.0;
    }
  std::vector<Cx> out(npts);
  for (size_t j = 0; j < npts; ++j) {
    Cx acc{0.0, 0.0};
    for (size_t i = 0; i < n; ++i) {
      double w = 0.0;
      for (size_t c = 0; c < (size_t)inp.ncomp; ++c) {
        double m = (double)inp.compartments[c][i];
        if (m != 0.0) {
          double dec = acq.do_relaxation
                           ? std::exp((log_amp ? log_amp[i] : 0.0) - tau[j] * spiral_decay_rate(inp, acq, c, i))
                           : 1.0;
          w += m * dec;
        }
      }
      if (w == 0.0) continue;
      double ph = phi0[i] + TAU * (rate[i] * tau[j] / 1000.0 + k[2 * j] * xc[i] / (double)nx +
                                   k[2 * j + 1] * yc[i] / (double)ny);
      double a = amp[i] * w;
      acc = cadd(acc, Cx{a * std::cos(ph), a * std::sin(ph)});
    }
    out[j] = cscale(acc, 1.0 / (double)n);
  }
  return out;
}

// `SegmentedForward::apply` with `segment_inputs` (spiral.rs:83-103, 174-201), the L type-2
// transforms taken as exact sums, for a given plan (tau_l, b).
std::vector<Cx> spiral_segmented(const mrsim_slice_input& inp, const mrsim_acquisition& acq, size_t coil,
                                 size_t ncoils, const double* k, const int64_t* tau_idx, size_t npts,
                                 const double* tau_l, size_t L, const double* b, const double* log_amp,
                                 bool decay_inside) {
  size_t snx = inp.sim[0], sny = inp.sim[1], nx = inp.acq_matrix[0], ny = inp.acq_matrix[1];
  size_t ox = snx / nx, oy = sny / ny, sxs = ox * (nx / 2), sys = oy * (ny / 2);
  double xoff = ((double)ox - 1.0) / 2.0, yoff = ((double)oy - 1.0) / 2.0;
  size_t n = snx * sny;
  std::vector<Cx> x(n);
  std::vector<double> rd(n), rw(n);
  for (size_t yy = 0; yy < sny; ++yy)
    for (size_t xx = 0; xx < snx; ++xx) {
      size_t i = xx + snx * yy;
      double xa = ((double)xx - xoff) / (double)ox, ya = ((double)yy - yoff) / (double)oy;
      double a = acq.signal_scale * coil_sensitivity(coil, ncoils, xa, ya, nx, ny) * (double)inp.compartments[0][i];
      double d = 0.0;
      if (decay_inside && acq.do_relaxation) {
        a *= log_amp ? std::exp(log_amp[i]) : 1.0;
        d = spiral_decay_rate(inp, acq, 0, i);
      }
      x[i] = cscale(ccis(inp.phase0 ? inp.phase0[i] : 0.0), a);
      rd[i] = -d;
      rw[i] = TAU * (acq.do_distortions ? (double)inp.fmap[i] : 0.0) / 1000.0;
    }
  int64_t nn[2] = {(int64_t)snx, (int64_t)sny}, lo[2] = {-(int64_t)sxs, -(int64_t)sys}, mo[2] = {(int64_t)snx, (int64_t)sny};
  std::vector<Cx> out(npts, Cx{0.0, 0.0}), seg(n);
  for (size_t l = 0; l < L; ++l) {
    for (size_t i = 0; i < n; ++i) seg[i] = cmul(x[i], cscale(ccis(rw[i] * tau_l[l]), std::exp(rd[i] * tau_l[l])));
    std::vector<Cx> ks = nufft2_direct(2, nn, lo, mo, k, npts, seg.data(), 1);
    for (size_t j = 0; j < npts; ++j) {
      Cx bl{b[2 * ((size_t)tau_idx[j] * L + l)], b[2 * ((size_t)tau_idx[j] * L + l) + 1]};
      out[j] = cadd(out[j], cmul(bl, ks[j]));
    }
  }
  for (size_t j = 0; j < npts; ++j) {
    Cx st = cscale(ccis(-TAU * (k[2 * j] * xoff / (double)snx + k[2 * j + 1] * yoff / (double)sny)), 1.0 / (double)n);
    out[j] = cmul(out[j], st);
  }
  return out;
}


// `SpiralRecon` grid_recon.rs:54-325, FP64 with the NUFFT pair as the reference applies it.
struct SpiralReconO {
  size_t n;
  std::vector<double> k, w, win;
  Nufft2O nufft;
  std::vector<bool> keep;
  bool band;
  double lambda_hi = 0.0, kappa;
  size_t iterations;
  int64_t power_its = 0;
  static Nufft2O make(size_t n) {
    int64_t nn[2] = {(int64_t)n, (int64_t)n}, lo[2] = {-(int64_t)(n / 2), -(int64_t)(n / 2)}, mo[2] = {(int64_t)n, (int64_t)n};
    return Nufft2O(nn, lo, mo, 1e-12);
  }
  static double norm(const std::vector<Cx>& v) {
    double s = 0.0;
    for (const Cx& c : v) s += c.re * c.re + c.im * c.im;
    return std::sqrt(s);
  }
  SpiralReconO(const double* k_, size_t npts, size_t n_, const mrsim_acquisition& wa, size_t its, double kap, bool band_)
      : n(n_), k(k_, k_ + 2 * npts), nufft(make(n_)), band(band_), kappa(kap), iterations(its) {
    w.assign(npts, 1.0);
    for (int it = 0; it < 10; ++it) {  // `pipe_menon` grid_recon.rs:54-66
      std::vector<Cx> wts(npts);
      for (size_t j = 0; j < npts; ++j) wts[j] = {w[j], 0.0};
      std::vector<Cx> img = nufft.type1(k.data(), npts, wts.data(), -1);
      std::vector<Cx> back = nufft.type2(img.data(), k.data(), npts, 1);
      for (size_t j = 0; j < npts; ++j) w[j] /= std::hypot(back[j].re, back[j].im);
    }
    auto dirichlet = [&](double kk) {
      Cx acc{0.0, 0.0};
      for (size_t x = 0; x < n; ++x) acc = cadd(acc, ccis(TAU * kk * ((double)x - (double)(n / 2)) / (double)n));
      return cscale(acc, 1.0 / (double)n);
    };
    Cx centre{0.0, 0.0};
    for (size_t j = 0; j < npts; ++j) centre = cadd(centre, cscale(cmul(dirichlet(k[2 * j]), dirichlet(k[2 * j + 1])), w[j]));
    double s = 1.0 / centre.re;
    for (double& x : w) x *= s;
    double radius = 0.0;
    for (size_t j = 0; j < npts; ++j) {
      win.push_back(window_at(wa, k[2 * j] / (double)n, k[2 * j + 1] / (double)n));
      radius = std::max(radius, std::hypot(k[2 * j], k[2 * j + 1]));
    }
    size_t hu = (n + 1) / 2;
    auto sg = [&](size_t i) { return i < hu ? (double)i : (double)i - (double)n; };
    for (size_t i = 0; i < n * n; ++i) keep.push_back(std::hypot(sg(i % n), sg(i / n)) <= radius);
    uint64_t st = 0x9E3779B97F4A7C15ull;
    auto rnd = [&]() {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      return (double)(st >> 11) / (double)(1ull << 53) - 0.5;
    };
    std::vector<Cx> v(n * n);
    for (Cx& c : v) {
      c.re = rnd();
      c.im = rnd();
    }
    double lam = 0.0;
    for (int it = 0; it < 1000; ++it) {
      double nv = norm(v);
      std::vector<Cx> u = normal(v);
      double nu = norm(u);
      double next = nu / nv;
      for (size_t i = 0; i < v.size(); ++i) v[i] = cscale(u[i], 1.0 / nu);
      bool done = std::fabs(next - lam) <= 1e-10 * next;
      lam = next;
      ++power_its;
      if (done) break;
    }
    lambda_hi = 1.1 * lam;
  }
  std::vector<Cx> forward(const std::vector<Cx>& x) const {
    double sc = 1.0 / (double)(n * n);
    std::vector<Cx> o = nufft.type2(x.data(), k.data(), k.size() / 2, 1);
    for (Cx& c : o) c = {c.re * sc, c.im * sc};
    return o;
  }
  std::vector<Cx> adjoint(const std::vector<Cx>& r) const {
    double sc = 1.0 / (double)(n * n);
    std::vector<Cx> wts(r.size());
    for (size_t j = 0; j < r.size(); ++j) wts[j] = {r[j].re * w[j] * sc, r[j].im * w[j] * sc};
    return nufft.type1(k.data(), r.size(), wts.data(), -1);
  }
  void project(std::vector<Cx>& x) const {
    if (!band) return;
    fft2d(x, n, n, -1);
    for (size_t i = 0; i < x.size(); ++i)
      if (!keep[i]) x[i] = {0.0, 0.0};
    fft2d(x, n, n, 1);
    double s = 1.0 / (double)(n * n);
    for (Cx& c : x) c = {c.re * s, c.im * s};
  }
  std::vector<Cx> normal(const std::vector<Cx>& x) const {
    std::vector<Cx> xq = x;
    project(xq);
    std::vector<Cx> y = adjoint(forward(xq));
    project(y);
    return y;
  }
  std::vector<Cx> gridding(const std::vector<Cx>& d) const {
    std::vector<Cx> o = adjoint(d);
    for (Cx& c : o) c = cscale(c, (double)(n * n));
    return o;
  }
  std::vector<Cx> image(const std::vector<Cx>& d) const {
    std::vector<Cx> dw(d.size());
    for (size_t j = 0; j < d.size(); ++j) dw[j] = cscale(d[j], win[j]);
    double hi = lambda_hi, lo = lambda_hi / kappa;
    double theta = (hi + lo) / 2.0, delta = (hi - lo) / 2.0;
    double sigma1 = theta / delta;
    double rho = 1.0 / sigma1;
    std::vector<Cx> x(n * n, Cx{0.0, 0.0});
    std::vector<Cx> r = adjoint(dw);
    project(r);
    double r0 = norm(r);
    std::vector<Cx> dir(r.size());
    for (size_t i = 0; i < r.size(); ++i) dir[i] = cscale(r[i], 1.0 / theta);
    for (size_t it = 0; it < iterations; ++it) {
      for (size_t i = 0; i < x.size(); ++i) x[i] = cadd(x[i], dir[i]);
      std::vector<Cx> nd = normal(dir);
      for (size_t i = 0; i < r.size(); ++i) r[i] = {r[i].re - nd[i].re, r[i].im - nd[i].im};
      double rho1 = 1.0 / (2.0 * sigma1 - rho);
      for (size_t i = 0; i < dir.size(); ++i) dir[i] = cadd(cscale(dir[i], rho1 * rho), cscale(r[i], 2.0 * rho1 / delta));
      rho = rho1;
    }
    double rn = norm(r);
    if (!(rn <= (1.0 + 1e-6) * r0 + 1e-300)) throw Fail("spiral reconstruction: the residual grew");
    return x;
  }
  std::vector<Cx> rings(const Cx* coil, size_t ncoils, size_t ring, const double* zsens) const {
    size_t npts = k.size() / 2, rows = ncoils / ring;
    std::vector<Cx> wsum(n * n, Cx{0.0, 0.0});
    std::vector<double> ssum(n * n, 0.0);
    for (size_t a = 0; a < ring; ++a) {
      std::vector<Cx> img;
      if (rows == 1 && zsens[a] == 1.0) {
        img = image(std::vector<Cx>(coil + a * npts, coil + (a + 1) * npts));
      } else {
        std::vector<Cx> d(npts, Cx{0.0, 0.0});
        for (size_t r = 0; r < rows; ++r) {
          size_t q = r * ring + a;
          for (size_t j = 0; j < npts; ++j) d[j] = cadd(d[j], cscale(coil[q * npts + j], zsens[q]));
        }
        img = image(d);
      }
      double z2 = 0.0;
      for (size_t r = 0; r < rows; ++r) z2 += zsens[r * ring + a] * zsens[r * ring + a];
      for (size_t y = 0; y < n; ++y)
        for (size_t x = 0; x < n; ++x) {
          double s = coil_sensitivity(a, ring, (double)x, (double)y, n, n);
          size_t i = x + n * y;
          wsum[i] = cadd(wsum[i], cscale(img[i], s));
          ssum[i] += s * s * z2;
        }
    }
    std::vector<Cx> out(n * n);
    for (size_t i = 0; i < n * n; ++i) {
      double s = std::max(ssum[i], 1e-12);
      out[i] = {wsum[i].re / s, wsum[i].im / s};
    }
    return out;
  }
};


// ============================ the 3D GRASE echo train =====================================
// readout.rs:167-322 (kz order, GRASE block and lines), epg.rs:47-125 (CPMG amplitudes),
// kspace3d.rs:42-547 (modes, z-DFT, compartments, line weights, partitions, reconstruction).
std::vector<size_t> kz_order_o(size_t nz, int order) {
  std::vector<size_t> out;
  if (order == MRSIM_KZ_LINEAR) {
    for (size_t p = 0; p < nz; ++p) out.push_back(p);
    return out;
  }
  size_t c = nz / 2;
  out.push_back(c);
  size_t d = 1;
  while (out.size() < nz) {
    if (c + d < nz) out.push_back(c + d);
    if (d <= c && out.size() < nz) out.push_back(c - d);
    ++d;
  }
  return out;
}

struct GLine {
  size_t shot, echo;
  double t_ms, trf_ms;
  int8_t pol;
};
struct GTable {
  size_t ny, nz, e_c, n_shots;
  std::vector<GLine> lines;
  std::vector<double> t_ms;
  std::vector<int8_t> pol;
  const GLine& line(size_t p, size_t ky) const { return lines[p * ny + ky]; }
};

GTable grase_lines_o(const mrsim_echo_train& tr, const mrsim_grase_readout& ro, size_t ny, size_t nz) {
  size_t kys = (size_t)ro.ky_segments, kzs = (size_t)tr.kz_segments;
  if (kys == 0 || ny % kys != 0) throw Fail("phase-encode lines do not divide into ky segments");
  size_t epi = ny / kys;
  GTable T;
  T.ny = ny;
  T.nz = nz;
  T.t_ms.resize(ny);
  T.pol.resize(ny);
  for (size_t ky = 0; ky < ny; ++ky) {
    size_t j = ky / kys;
    size_t a = ro.reverse_phase ? j : epi - 1 - j;
    T.t_ms[ky] = ((double)a - ((double)epi - 1.0) / 2.0) * ro.t_line_ms;
    T.pol[ky] = a % 2 == 1 ? -1 : 1;
  }
  if (kzs == 0 || nz % kzs != 0) throw Fail("partitions do not divide into kz segments");
  if ((size_t)tr.etl != nz / kzs) throw Fail("echo train length mismatch");
  std::vector<size_t> order = kz_order_o(nz, tr.kz_order);
  T.lines.assign(ny * nz, GLine{0, 0, 0.0, 0.0, 0});
  for (size_t sy = 0; sy < kys; ++sy)
    for (size_t sz = 0; sz < kzs; ++sz) {
      size_t shot = sy * kzs + sz;
      for (size_t e = 1; e <= (size_t)tr.etl; ++e) {
        size_t pp = order[sz + kzs * (e - 1)];
        for (size_t j = 0; j < epi; ++j) {
          size_t ky = sy + kys * j;
          double t = T.t_ms[ky];
          T.lines[pp * ny + ky] = GLine{shot, e, t, (double)e * tr.esp_ms + t, T.pol[ky]};
        }
      }
    }
  size_t n = 0;
  while (order[n] != nz / 2) ++n;
  T.e_c = n / kzs + 1;
  T.n_shots = kys * kzs;
  return T;
}

// `epg_cpmg` epg.rs:101-125 (Weigel's extended phase graphs; ln of the echo amplitudes)
std::vector<double> epg_cpmg_o(size_t n_echoes, double esp, double b_deg, double t1, double t2) {
  size_t n = 2 * n_echoes + 2;
  std::vector<Cx> fp(n, Cx{0, 0}), fm(n, Cx{0, 0}), z(n, Cx{0, 0});
  z[0] = {1.0, 0.0};
  auto rot = [&](double alpha, double phi) {
    double ch = std::cos(alpha / 2.0), sh = std::sin(alpha / 2.0);
    double c2 = ch * ch, s2 = sh * sh, sa = std::sin(alpha), ca = std::cos(alpha);
    Cx e2p = ccis(2.0 * phi), e2m = ccis(-2.0 * phi), e1p = ccis(phi), e1m = ccis(-phi);
    Cx I{0.0, 1.0}, mI{0.0, -1.0};
    for (size_t k = 0; k < n; ++k) {
      Cx a = fp[k], b = fm[k], c = z[k];
      fp[k] = cadd(cadd(cscale(a, c2), cscale(cmul(e2p, b), s2)), cscale(cmul(cmul(mI, e1p), c), sa));
      fm[k] = cadd(cadd(cscale(cmul(e2m, a), s2), cscale(b, c2)), cscale(cmul(cmul(I, e1m), c), sa));
      z[k] = cadd(cadd(cscale(cmul(cmul(mI, e1m), a), sa / 2.0), cscale(cmul(cmul(I, e1p), b), sa / 2.0)), cscale(c, ca));
    }
  };
  auto relax = [&](double e1, double e2) {
    for (size_t k = 0; k < n; ++k) {
      fp[k] = cscale(fp[k], e2);
      fm[k] = cscale(fm[k], e2);
      z[k] = cscale(z[k], e1);
    }
    z[0] = cadd(z[0], Cx{1.0 - e1, 0.0});
  };
  auto shift = [&]() {
    for (size_t k = n - 1; k >= 1; --k) fp[k] = fp[k - 1];
    for (size_t k = 0; k + 1 < n; ++k) fm[k] = fm[k + 1];
    fm[n - 1] = {0.0, 0.0};
    fp[0] = {fm[0].re, -fm[0].im};
  };
  auto decay = [](double dt, double t) { return std::isinf(t) ? 1.0 : std::exp(-dt / t); };
  rot(PI / 2.0, 0.0);
  double norm = std::hypot(fp[0].re, fp[0].im);
  double e1 = decay(esp / 2.0, t1), e2 = decay(esp / 2.0, t2);
  std::vector<double> out(n_echoes);
  for (size_t e = 0; e < n_echoes; ++e) {
    relax(e1, e2);
    shift();
    rot(b_deg * PI / 180.0, PI / 2.0);
    shift();
    relax(e1, e2);
    double a = std::hypot(fp[0].re, fp[0].im) / norm;
    out[e] = a == 0.0 ? -INFINITY : std::log(a);
  }
  return out;
}

struct Mode3 {
  bool voxel = false;
  std::vector<double> ln_a;
  double t2 = 0, t2p = 0;
  std::vector<std::vector<double>> maps;
};

std::vector<Mode3> resolve_modes_o(const mrsim_t2* t2, const mrsim_t2* t1, const mrsim_t2* ti, size_t ncomp,
                                   const mrsim_acquisition& acq, const mrsim_echo_train& tr, size_t nvox) {
  if (acq.do_relaxation && tr.refocusing_deg != 180.0 && !t1) throw Fail("refocusing below 180 degrees needs T1");
  size_t etl = (size_t)tr.etl;
  std::vector<Mode3> modes(ncomp);
  for (size_t c = 0; c < ncomp; ++c) {
    mrsim_t2 t1c = t1 ? t1[c] : mrsim_t2{nullptr, INFINITY, 0};
    mrsim_t2 tic = ti ? ti[c] : mrsim_t2{nullptr, (float)acq.t_inhom, 0};
    if (!t2[c].is_map && !t1c.is_map && !tic.is_map) {
      modes[c].ln_a = epg_cpmg_o(etl, tr.esp_ms, tr.refocusing_deg, (double)t1c.value, (double)t2[c].value);
      modes[c].t2 = t2[c].value;
      modes[c].t2p = tic.value;
    } else if (!acq.do_relaxation) {
      modes[c].ln_a.assign(etl, 0.0);
      modes[c].t2 = INFINITY;
      modes[c].t2p = INFINITY;
    } else {
      modes[c].voxel = true;
      modes[c].maps.assign(etl, std::vector<double>(nvox));
      for (size_t i = 0; i < nvox; ++i) {
        float a = t1c.is_map ? t1c.map[i] : t1c.value, b = t2[c].is_map ? t2[c].map[i] : t2[c].value;
        std::vector<double> la = epg_cpmg_o(etl, tr.esp_ms, tr.refocusing_deg, (double)a, (double)b);
        for (size_t e = 0; e < etl; ++e) modes[c].maps[e][i] = la[e];
      }
    }
  }
  return modes;
}

double line_weight_o(double ln_a, double t, double t2, double t2p) {
  double d2 = std::isinf(t2) ? 0.0 : t / t2;
  double dp = std::isinf(t2p) ? 0.0 : std::fabs(t) / t2p;
  return std::exp(ln_a - d2 - dp);
}

// The first shot set holding `shot` (`sets.iter().position(|s| s.shots.contains(&shot))`,
// kspace3d.rs:216), or -1.
int set_of(const mrsim_shot_set* sets, size_t n_sets, int64_t shot) {
  for (size_t i = 0; i < n_sets; ++i)
    for (int64_t j = 0; j < sets[i].n_shots; ++j)
      if (sets[i].shots[j] == shot) return (int)i;
  return -1;
}
// The shot-image checks (kspace3d.rs:369-377): every set's shots inside the train.
void check_sets(const mrsim_shot_set* sets, size_t n_sets, int64_t n_shots) {
  for (size_t i = 0; i < n_sets; ++i)
    for (int64_t j = 0; j < sets[i].n_shots; ++j)
      if (sets[i].shots[j] < 0 || sets[i].shots[j] >= n_shots)
        throw std::runtime_error("a shot index beyond the train's " + std::to_string(n_shots));
}
const mrsim_shot_set* sets_of(const mrsim_acquisition_3d_input& in, size_t g) {
  return in.shot_sets && in.n_shot_sets ? in.shot_sets[g] : nullptr;
}
size_t n_sets_of(const mrsim_acquisition_3d_input& in, size_t g) {
  return in.shot_sets && in.n_shot_sets ? (size_t)in.n_shot_sets[g] : 0;
}
void check_all_sets(const mrsim_acquisition_3d_input& in, int64_t n_shots) {
  for (int64_t g = 0; g < in.n_volumes; ++g) check_sets(sets_of(in, (size_t)g), n_sets_of(in, (size_t)g), n_shots);
}

struct Plan3 {
  size_t snx, sny, nz, nx, ny, o, ncomp;
  mrsim_acquisition acq;
  GTable table;
  LineTiming within;
  std::vector<Mode3> modes;
  const mrsim_t2* t2;
  const mrsim_t2* ti;
  const float* fmap;
  mrsim_phase_model phase;
  std::vector<Cx> zk;
  std::vector<uint8_t> mask;

  // `Plan::compartments` kspace3d.rs:125-204: img(c, vox) of one volume, coil q
  std::vector<std::vector<Cx>> compartments(const std::function<float(size_t, size_t)>& img, size_t q,
                                            size_t ncoils) const {
    size_t nplane = snx * sny;
    mrsim_acquisition norel = acq, rel = acq;
    norel.do_relaxation = 0;
    norel.noise_variance = 0.0;
    norel.n_spikes = 0;
    rel.do_relaxation = 1;
    rel.noise_variance = 0.0;
    rel.n_spikes = 0;
    Shot zero;
    std::vector<std::vector<double>> phis(nz);
    for (size_t z = 0; z < nz; ++z) phis[z] = phase_slice(phase, zero, snx, sny, o, z, nz);
    std::vector<std::vector<Cx>> out(ncomp, std::vector<Cx>(nz * ny * nx, Cx{0, 0}));
    for (size_t c = 0; c < ncomp; ++c) {
      auto plane = [&](size_t z) {
        std::vector<float> v(nplane);
        for (size_t i = 0; i < nplane; ++i) v[i] = img(c, z * nplane + i);
        return v;
      };
      auto one = [&](size_t z, const std::vector<float>& pl, const mrsim_acquisition& a, const double* la) {
        const float* comps[1] = {pl.data()};
        mrsim_t2 t2s[1] = {t2[c].is_map ? mrsim_t2{t2[c].map + z * nplane, 0.f, 1} : t2[c]};
        mrsim_t2 tis[1];
        if (ti) tis[0] = ti[c].is_map ? mrsim_t2{ti[c].map + z * nplane, 0.f, 1} : ti[c];
        mrsim_slice_input inp;
        std::memset(&inp, 0, sizeof inp);
        inp.compartments = comps;
        inp.ncomp = 1;
        inp.t2 = t2s;
        inp.t_inhom = ti ? tis : nullptr;
        inp.fmap = fmap + z * nplane;
        inp.phase0 = phis[z].data();
        inp.sim[0] = (int64_t)snx;
        inp.sim[1] = (int64_t)sny;
        inp.acq_matrix[0] = (int64_t)nx;
        inp.acq_matrix[1] = (int64_t)ny;
        inp.z = (int64_t)z;
        inp.nz = (int64_t)nz;
        return build_coil_kspace_timed(inp, a, q, ncoils, within, la);
      };
      const Mode3& m = modes[c];
      if (!m.voxel) {
        std::vector<std::vector<Cx>> k2(nz);
        for (size_t z = 0; z < nz; ++z) k2[z] = one(z, plane(z), norel, nullptr);
        for (size_t p = 0; p < nz; ++p)
          for (size_t ky = 0; ky < ny; ++ky) {
            const GLine& L = table.line(p, ky);
            double w = acq.do_relaxation ? line_weight_o(m.ln_a[L.echo - 1], L.t_ms, m.t2, m.t2p) : 1.0;
            for (size_t kx = 0; kx < nx; ++kx) {
              Cx acc{0, 0};
              for (size_t z = 0; z < nz; ++z) acc = cadd(acc, cmul(k2[z][ky * nx + kx], zk[p * nz + z]));
              out[c][(p * ny + ky) * nx + kx] = cscale(acc, w);
            }
          }
      } else {
        std::vector<std::vector<float>> planes(nz);
        for (size_t z = 0; z < nz; ++z) planes[z] = plane(z);
        size_t emax = 0;
        for (auto& L : table.lines) emax = std::max(emax, L.echo);
        for (size_t e = 1; e <= emax; ++e) {
          std::vector<size_t> ps;
          for (size_t p = 0; p < nz; ++p)
            if (table.line(p, 0).echo == e) ps.push_back(p);
          if (ps.empty()) continue;
          std::vector<std::vector<Cx>> k2(nz);
          for (size_t z = 0; z < nz; ++z) k2[z] = one(z, planes[z], rel, m.maps[e - 1].data() + z * nplane);
          for (size_t p : ps)
            for (size_t ky = 0; ky < ny; ++ky)
              for (size_t kx = 0; kx < nx; ++kx) {
                Cx acc{0, 0};
                for (size_t z = 0; z < nz; ++z) acc = cadd(acc, cmul(k2[z][ky * nx + kx], zk[p * nz + z]));
                out[c][(p * ny + ky) * nx + kx] = acc;
              }
        }
      }
    }
    return out;
  }

  // `Plan::kspace` kspace3d.rs:206-232: each line from the images its shot saw (the first set
  // holding the shot, else the volume's own)
  std::vector<Cx> kspace(const float* const* images, size_t n_volumes, size_t g, size_t q, size_t ncoils,
                         const double* lw, const mrsim_shot_set* sets = nullptr, size_t n_sets = 0) const {
    auto base = compartments([&](size_t c, size_t v) { return images[c][v * n_volumes + g]; }, q, ncoils);
    std::vector<std::vector<std::vector<Cx>>> moved(n_sets);
    for (size_t i = 0; i < n_sets; ++i)
      moved[i] = compartments([&](size_t c, size_t v) { return sets[i].images[c][v]; }, q, ncoils);
    std::vector<Cx> k(nz * ny * nx, Cx{0, 0});
    for (size_t p = 0; p < nz; ++p)
      for (size_t ky = 0; ky < ny; ++ky) {
        const GLine& L = table.line(p, ky);
        const std::vector<std::vector<Cx>>* src = &base;
        const int si = set_of(sets, n_sets, (int64_t)L.shot);
        if (si >= 0) src = &moved[(size_t)si];
        for (size_t c = 0; c < ncomp; ++c) {
          double w = lw ? lw[(g * table.n_shots + L.shot) * ncomp + c] : 1.0;
          for (size_t kx = 0; kx < nx; ++kx) {
            size_t i = (p * ny + ky) * nx + kx;
            k[i] = cadd(k[i], cscale((*src)[c][i], w));
          }
        }
        if (!mask[ky * nx])
          for (size_t kx = 0; kx < nx; ++kx) k[(p * ny + ky) * nx + kx] = Cx{0, 0};
      }
    return k;
  }
};

Plan3 plan3(const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq, const mrsim_echo_train& tr,
            const mrsim_grase_readout& ro) {
  Plan3 P;
  P.snx = in.sim_dims[0];
  P.sny = in.sim_dims[1];
  P.nz = in.sim_dims[2];
  P.nx = in.acq_dims[0];
  P.ny = in.acq_dims[1];
  if ((size_t)in.acq_dims[2] != P.nz) throw Fail("partition count must match; z is never oversampled");
  P.o = P.snx / P.nx;
  P.ncomp = in.ncomp;
  P.acq = acq;
  P.table = grase_lines_o(tr, ro, P.ny, P.nz);
  P.within.t_ms = P.table.t_ms;
  P.within.trf_ms = P.table.t_ms;
  P.within.tread_ms = P.table.t_ms;
  P.within.polarity = P.table.pol;
  P.modes = resolve_modes_o(in.t2, in.t1, in.t_inhom, P.ncomp, acq, tr, P.snx * P.sny * P.nz);
  P.t2 = in.t2;
  P.ti = in.t_inhom;
  P.fmap = in.fmap;
  if (in.phase) P.phase = *in.phase;
  else std::memset(&P.phase, 0, sizeof P.phase);
  double zs = (double)(P.nz / 2);
  P.zk.resize(P.nz * P.nz);
  for (size_t p = 0; p < P.nz; ++p)
    for (size_t z = 0; z < P.nz; ++z) {
      double th = TAU * ((double)p - zs) * ((double)z - zs) / (double)P.nz;
      P.zk[p * P.nz + z] = Cx{std::cos(th), std::sin(th)};
    }
  P.mask = sampling_mask(P.nx, P.ny, acq);
  check_all_sets(in, (int64_t)P.table.n_shots);
  return P;
}

// `partitions_to_slices` kspace3d.rs:235-281
std::vector<std::vector<Cx>> partitions_to_slices_o(std::vector<Cx>& k, const std::vector<uint8_t>& mask,
                                                    const std::vector<Cx>& zk, size_t nx, size_t ny, size_t nz,
                                                    size_t g, size_t q, uint64_t seed, const mrsim_acquisition& acq,
                                                    double sigma) {
  const uint64_t salt3d = 0x334452454144ull;
  for (size_t p = 0; p < nz; ++p) {
    Cx* part = k.data() + p * ny * nx;
    uint64_t pseed = (((uint64_t)g * 0x1000001ull) + (uint64_t)p) * 0x9E37ull ^ seed ^ salt3d;
    if (acq.n_spikes > 0) {
      Cx peak{0, 0};
      double pm = 0.0;
      for (size_t i = 0; i < nx * ny; ++i)
        if (cabs_(part[i]) > pm) {
          pm = cabs_(part[i]);
          peak = part[i];
        }
      std::vector<size_t> acquired;
      for (size_t i = 0; i < nx * ny; ++i)
        if (mask[i]) acquired.push_back(i);
      Rng rng(pseed ^ 0xA5A5123456789ABCull ^ ((uint64_t)q * 0xC2B2AE3D27D4EB4Full));
      for (int64_t s2 = 0; s2 < acq.n_spikes; ++s2) {
        size_t pick = acquired[(size_t)(rng.next_u64() % (uint64_t)acquired.size())];
        part[pick] = cscale(peak, acq.spike_amplitude);
      }
    }
    if (acq.noise_variance > 0.0) {
      Rng rng((pseed ^ ((uint64_t)q * 0x9E3779B9ull)) | 1ull);
      for (size_t i = 0; i < nx * ny; ++i)
        if (mask[i]) {
          part[i].re += rng.gauss() * sigma;
          part[i].im += rng.gauss() * sigma;
        }
    }
  }
  std::vector<std::vector<Cx>> slices(nz, std::vector<Cx>(ny * nx, Cx{0, 0}));
  for (size_t z = 0; z < nz; ++z) {
    for (size_t p = 0; p < nz; ++p) {
      Cx kc = zk[p * nz + z];
      Cx conj{kc.re, -kc.im};
      for (size_t i = 0; i < ny * nx; ++i) slices[z][i] = cadd(slices[z][i], cmul(k[p * ny * nx + i], conj));
    }
    for (Cx& c : slices[z]) c = cscale(c, 1.0 / (double)nz);
  }
  return slices;
}

// `simulate_acquisition_3d_complex_cal` kspace3d.rs:483-547 (GRASE, no shot images)
std::vector<std::vector<Cx>> acquire_3d_o(const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                                          const mrsim_echo_train& tr, const mrsim_grase_readout& ro, uint64_t seed,
                                          int threads) {
  Plan3 pl = plan3(in, acq, tr, ro);
  size_t nz = pl.nz, nx = pl.nx, ny = pl.ny, nv = in.n_volumes;
  size_t ncoils = std::max<int64_t>(acq.n_coils, 1);
  double sigma = std::sqrt(acq.noise_variance / (double)(nx * ny));
  std::vector<GrappaKernel> kernels;
  if (acq.accel > 1 && nv > 0) {
    mrsim_acquisition acq_cal = acq;
    acq_cal.accel = 1;
    acq_cal.n_spikes = 0;
    const float* const* cal_images = in.images;
    size_t cal_nv = nv;
    uint64_t cal_seed = seed;
    if (in.has_grappa_calibration) {
      cal_images = in.grappa_calibration_images;
      cal_nv = 1;
      cal_seed = in.grappa_calibration_seed;
    }
    Plan3 cal = plan3(in, acq_cal, tr, ro);
    std::vector<std::vector<std::vector<Cx>>> parts(ncoils);
    parallel_for(ncoils, threads, [&](size_t q) {
      std::vector<Cx> k = cal.kspace(cal_images, cal_nv, 0, q, ncoils, nullptr);
      parts[q] = partitions_to_slices_o(k, cal.mask, cal.zk, nx, ny, nz, 0, q, cal_seed ^ SEED_SALT_GRAPPA_CAL, acq_cal,
                                        sigma);
    });
    std::vector<uint8_t> lines = sampling_mask(1, ny, acq_cal);
    for (size_t z = 0; z < nz; ++z) {
      std::vector<std::vector<Cx>> coils(ncoils);
      for (size_t q = 0; q < ncoils; ++q) coils[q] = parts[q][z];
      kernels.push_back(grappa_fit(coils, nx, ny, acq.accel, acq.acs_lines, lines));
    }
  }
  std::vector<std::vector<Cx>> vols(nv);
  parallel_for(nv, threads, [&](size_t g) {
    std::vector<std::vector<std::vector<Cx>>> parts(ncoils);
    for (size_t q = 0; q < ncoils; ++q) {
      std::vector<Cx> k = pl.kspace(in.images, nv, g, q, ncoils, in.line_weights, sets_of(in, g), n_sets_of(in, g));
      parts[q] = partitions_to_slices_o(k, pl.mask, pl.zk, nx, ny, nz, g, q, seed, acq, sigma);
    }
    std::vector<Cx> out(nx * ny * nz);
    for (size_t z = 0; z < nz; ++z) {
      std::vector<std::vector<Cx>> coils(ncoils);
      for (size_t q = 0; q < ncoils; ++q) coils[q] = parts[q][z];
      SliceRecon R = reconstruct_coils_full(coils, acq, nx, ny, false, false, false, kernels.empty() ? nullptr : &kernels[z]);
      for (size_t i = 0; i < nx * ny; ++i) out[i + nx * ny * z] = R.combined[i];
    }
    vols[g] = out;
  });
  return vols;
}


// ============================ the stack of spirals ========================================
// readout.rs:107-160 (KzSampling), 564-700 (trajectory, spiral_lines, spiral_kz_order),
// kspace3d.rs:858-1569 (plan, samples, KzGrappa, POCS, spiral noise, spiral_volumes).  The
// in-plane forward is the exact spiral sum (`spiral_kspace_exact`), which the reference's
// time-segmented forward approximates to its certified 1e-7.
struct SpiralTabO {
  size_t nz, band_start, kz_segments, e_c, n_shots, ns, nsamp, interleaves;
  double readout_ms;
  std::vector<double> k, tau;
  std::vector<uint8_t> acquired;
  std::vector<size_t> echo, kz_segment;
};

SpiralTabO spiral_table_o(const mrsim_echo_train& tr, const mrsim_spiral_readout& ro, size_t n, size_t nz) {
  SpiralTabO T;
  size_t il = (size_t)ro.interleaves;
  double k_max = (double)n / 2.0, n_turns = ro.radial_oversampling * (double)n / (2.0 * (double)il), t = ro.readout_ms;
  double den = 1.0 / std::pow(k_max * ro.dwell_ms, 2) - 4.0 * PI * PI * n_turns * n_turns / (t * t);
  double tau_c = 1.0 / (t * den);
  size_t ns = (size_t)std::floor(t / ro.dwell_ms * (1.0 + 1e-12));
  for (size_t j = 0; j < ns; ++j) T.tau.push_back(((double)j + 0.5) * ro.dwell_ms);
  for (size_t s = 0; s < il; ++s)
    for (size_t j = 0; j < ns; ++j) {
      double tau = T.tau[j];
      double u = tau < tau_c ? tau / std::sqrt(tau_c * t) : std::sqrt(tau / t);
      double th = TAU * (n_turns * u + (double)s / (double)il);
      T.k.push_back(k_max * u * std::cos(th));
      T.k.push_back(k_max * u * std::sin(th));
    }
  T.ns = ns;
  T.nsamp = ns * il;
  T.interleaves = il;
  T.readout_ms = t;
  T.nz = nz;
  size_t kept = std::min(nz, (size_t)std::round((double)nz * ro.kz.partial_fourier));
  T.band_start = nz - kept;
  int64_t c = (int64_t)(nz / 2), a = ro.kz.accel;
  T.acquired.resize(nz);
  for (size_t p = 0; p < nz; ++p) T.acquired[p] = p >= T.band_start && (((int64_t)p - c) % a + a) % a == 0;
  std::vector<size_t> order;
  for (size_t p : kz_order_o(nz, tr.kz_order))
    if (T.acquired[p]) order.push_back(p);
  size_t kzs = (size_t)tr.kz_segments;
  if (kzs == 0 || order.size() % kzs != 0) throw Fail("partitions read do not divide into kz segments");
  if ((size_t)tr.etl != order.size() / kzs) throw Fail("echo train length mismatch");
  T.echo.assign(nz, 0);
  T.kz_segment.assign(nz, 0);
  for (size_t i = 0; i < order.size(); ++i) {
    T.echo[order[i]] = i / kzs + 1;
    T.kz_segment[order[i]] = i % kzs;
  }
  T.kz_segments = kzs;
  T.e_c = T.echo[nz / 2];
  T.n_shots = il * kzs;
  return T;
}

double coil_row_sensitivity_o(size_t row, size_t rows, double z, size_t nz) {
  if (rows <= 1) return 1.0;
  double centre = (double)nz * ((double)row + 0.5) / (double)rows - 0.5;
  double sigma = 0.6 * (double)nz / (double)rows;
  return std::exp(-std::pow(z - centre, 2) / (2.0 * sigma * sigma)) + 0.15;
}

struct SpiralPlanO {
  size_t snx, sny, nz, n, o, ncomp, rows, ring;
  mrsim_acquisition acq;
  SpiralTabO table;
  std::vector<Mode3> modes;
  const mrsim_t2* t2;
  const mrsim_t2* ti;
  const float* fmap;
  mrsim_phase_model phase;
  std::vector<Cx> zk;

  // `SpiralPlan::compartments` (kspace3d.rs:942-1012) with the exact in-plane sum, element a of
  // the rings: out[r][c][p * nsamp + j]
  std::vector<std::vector<std::vector<Cx>>> compartments(const std::function<float(size_t, size_t)>& img, size_t a)
      const {
    size_t nplane = snx * sny, nsamp = table.nsamp;
    Shot zero;
    std::vector<std::vector<Cx>> zkq(rows, zk);
    if (rows > 1)
      for (size_t r = 0; r < rows; ++r)
        for (size_t i = 0; i < nz * nz; ++i) zkq[r][i] = cscale(zk[i], coil_row_sensitivity_o(r, rows, (double)(i % nz), nz));
    std::vector<double> taus(nsamp);
    for (size_t j = 0; j < nsamp; ++j) taus[j] = table.tau[j % table.ns];
    std::vector<std::vector<std::vector<Cx>>> out(rows, std::vector<std::vector<Cx>>(ncomp, std::vector<Cx>(nz * nsamp, Cx{0, 0})));
    for (size_t c = 0; c < ncomp; ++c) {
      std::vector<std::vector<float>> planes(nz, std::vector<float>(nplane));
      for (size_t z = 0; z < nz; ++z)
        for (size_t i = 0; i < nplane; ++i) planes[z][i] = img(c, z * nplane + i);
      auto one = [&](size_t z, const double* la, bool voxel) {
        std::vector<double> phi = phase_slice(phase, zero, snx, sny, o, z, nz);
        const float* comps[1] = {planes[z].data()};
        mrsim_t2 t2s[1] = {t2[c].is_map ? mrsim_t2{t2[c].map + z * nplane, 0.f, 1} : t2[c]};
        mrsim_t2 tis[1];
        if (ti) tis[0] = ti[c].is_map ? mrsim_t2{ti[c].map + z * nplane, 0.f, 1} : ti[c];
        mrsim_slice_input inp;
        std::memset(&inp, 0, sizeof inp);
        inp.compartments = comps;
        inp.ncomp = 1;
        inp.t2 = t2s;
        inp.t_inhom = ti ? tis : nullptr;
        inp.fmap = fmap + z * nplane;
        inp.phase0 = phi.data();
        inp.sim[0] = (int64_t)snx;
        inp.sim[1] = (int64_t)sny;
        inp.acq_matrix[0] = inp.acq_matrix[1] = (int64_t)n;
        inp.z = (int64_t)z;
        inp.nz = (int64_t)nz;
        mrsim_acquisition a2 = acq;
        a2.do_relaxation = voxel ? 1 : 0;
        return spiral_kspace_exact(inp, a2, a, ring, table.k.data(), taus.data(), nsamp, la);
      };
      auto zsum = [&](const std::vector<Cx>& zkr, const std::vector<std::vector<Cx>>& k2, size_t p, size_t j) {
        Cx acc{0, 0};
        for (size_t z = 0; z < nz; ++z) acc = cadd(acc, cmul(k2[z][j], zkr[p * nz + z]));
        return acc;
      };
      const Mode3& m = modes[c];
      if (!m.voxel) {
        std::vector<std::vector<Cx>> k2(nz);
        for (size_t z = 0; z < nz; ++z) k2[z] = one(z, nullptr, false);
        for (size_t p = 0; p < nz; ++p) {
          if (!table.acquired[p]) continue;
          size_t e = table.echo[p];
          for (size_t j = 0; j < nsamp; ++j) {
            double w = acq.do_relaxation ? line_weight_o(m.ln_a[e - 1], table.tau[j % table.ns], m.t2, m.t2p) : 1.0;
            for (size_t r = 0; r < rows; ++r) out[r][c][p * nsamp + j] = cscale(zsum(zkq[r], k2, p, j), w);
          }
        }
      } else {
        size_t emax = 0;
        for (size_t e : table.echo) emax = std::max(emax, e);
        for (size_t e = 1; e <= emax; ++e) {
          std::vector<size_t> ps;
          for (size_t p = 0; p < nz; ++p)
            if (table.acquired[p] && table.echo[p] == e) ps.push_back(p);
          if (ps.empty()) continue;
          std::vector<std::vector<Cx>> k2(nz);
          for (size_t z = 0; z < nz; ++z) k2[z] = one(z, m.maps[e - 1].data() + z * nplane, true);
          for (size_t p : ps)
            for (size_t j = 0; j < nsamp; ++j)
              for (size_t r = 0; r < rows; ++r) out[r][c][p * nsamp + j] = zsum(zkq[r], k2, p, j);
        }
      }
    }
    return out;
  }

  // `samples_all` (kspace3d.rs:1014-1060): out[q] with q = r ring + a
  // `samples_rings` kspace3d.rs:1028-1051: each sample from the images its shot saw
  std::vector<std::vector<Cx>> samples_all(const float* const* images, size_t nv, size_t g, const double* lw,
                                           const mrsim_shot_set* sets = nullptr, size_t n_sets = 0) const {
    size_t nsamp = table.nsamp;
    std::vector<std::vector<Cx>> out(ring * rows);
    for (size_t a = 0; a < ring; ++a) {
      auto base = compartments([&](size_t c, size_t v) { return images[c][v * nv + g]; }, a);
      std::vector<decltype(base)> moved;
      for (size_t si = 0; si < n_sets; ++si)
        moved.push_back(compartments([&](size_t c, size_t v) { return sets[si].images[c][v]; }, a));
      for (size_t r = 0; r < rows; ++r) {
        std::vector<Cx> k(nz * nsamp, Cx{0, 0});
        for (size_t p = 0; p < nz; ++p) {
          if (!table.acquired[p]) continue;
          for (size_t j = 0; j < nsamp; ++j) {
            size_t shot = (j / table.ns) * table.kz_segments + table.kz_segment[p];
            size_t i = p * nsamp + j;
            const int si = set_of(sets, n_sets, (int64_t)shot);
            const auto& src = si >= 0 ? moved[(size_t)si] : base;
            for (size_t c = 0; c < ncomp; ++c) {
              double w = lw ? lw[(g * table.n_shots + shot) * ncomp + c] : 1.0;
              k[i] = cadd(k[i], cscale(src[r][c][i], w));
            }
          }
        }
        out[r * ring + a] = k;
      }
    }
    return out;
  }
};

void spiral_noise_o(std::vector<Cx>& k, const std::vector<uint8_t>& acquired, size_t nsamp, size_t g, size_t q,
                    uint64_t seed, double sigma) {
  const uint64_t salt3d = 0x334452454144ull;
  for (size_t p = 0; p < acquired.size(); ++p) {
    if (!acquired[p]) continue;
    uint64_t pseed = (((uint64_t)g * 0x1000001ull) + (uint64_t)p) * 0x9E37ull ^ seed ^ salt3d;
    Rng rng((pseed ^ ((uint64_t)q * 0x9E3779B9ull)) | 1ull);
    for (size_t j = 0; j < nsamp; ++j) {
      k[p * nsamp + j].re += rng.gauss() * sigma;
      k[p * nsamp + j].im += rng.gauss() * sigma;
    }
  }
}

// `KzGrappa` (kspace3d.rs:1261-1389)
struct KzGrappaO {
  size_t accel, nc;
  std::map<std::pair<size_t, unsigned>, std::vector<Cx>> weights;
  static std::vector<int64_t> offsets(size_t accel, size_t d) {
    int64_t r = (int64_t)accel, dd = (int64_t)d;
    return {-dd - r, -dd, r - dd, 2 * r - dd};
  }
  static std::vector<std::tuple<size_t, size_t, unsigned>> targets(const SpiralTabO& T, size_t accel) {
    std::vector<std::tuple<size_t, size_t, unsigned>> out;
    int64_t c = (int64_t)(T.nz / 2);
    for (size_t p = T.band_start; p < T.nz; ++p) {
      if (T.acquired[p]) continue;
      size_t d = (size_t)((((int64_t)p - c) % (int64_t)accel + (int64_t)accel) % (int64_t)accel);
      unsigned pat = 0;
      auto offs = offsets(accel, d);
      for (size_t s = 0; s < 4; ++s) {
        int64_t src = (int64_t)p + offs[s];
        if (src >= 0 && (size_t)src < T.nz && T.acquired[(size_t)src]) pat |= 1u << s;
      }
      out.emplace_back(p, d, pat);
    }
    return out;
  }
  static KzGrappaO fit(const SpiralTabO& T, size_t accel, const std::vector<std::vector<Cx>>& cal, size_t nsamp) {
    KzGrappaO K;
    K.accel = accel;
    K.nc = cal.size();
    size_t nz = T.nz, nc = cal.size(), lo = T.band_start;
    for (auto& [p, d, pat] : targets(T, accel)) {
      if (pat == 0) throw Fail("partition of the partial-Fourier band has no acquired partition within reach");
      if (K.weights.count({d, pat})) continue;
      std::vector<int64_t> offs;
      auto all = offsets(accel, d);
      for (size_t s = 0; s < 4; ++s)
        if (pat & (1u << s)) offs.push_back(all[s]);
      size_t nfeat = offs.size() * nc;
      std::vector<std::vector<Cx>> aha(nfeat, std::vector<Cx>(nfeat, Cx{0, 0})), ahb(nc, std::vector<Cx>(nfeat, Cx{0, 0}));
      std::vector<Cx> f(nfeat);
      size_t rows = 0;
      for (size_t t = lo; t < nz; ++t) {
        std::vector<size_t> srcs;
        for (int64_t o2 : offs) {
          int64_t pp = (int64_t)t + o2;
          if (pp >= (int64_t)lo && pp < (int64_t)nz) srcs.push_back((size_t)pp);
        }
        if (srcs.size() != offs.size()) continue;
        for (size_t j = 0; j < nsamp; ++j) {
          for (size_t s = 0; s < srcs.size(); ++s)
            for (size_t q = 0; q < nc; ++q) f[s * nc + q] = cal[q][srcs[s] * nsamp + j];
          for (size_t i = 0; i < nfeat; ++i) {
            Cx fic{f[i].re, -f[i].im};
            for (size_t jj = 0; jj < nfeat; ++jj) aha[i][jj] = cadd(aha[i][jj], cmul(fic, f[jj]));
            for (size_t q = 0; q < nc; ++q) ahb[q][i] = cadd(ahb[q][i], cmul(fic, cal[q][t * nsamp + j]));
          }
          ++rows;
        }
      }
      if (rows == 0) throw Fail("the calibration band holds no partition with the kernel's sources");
      double trace = 0.0;
      for (size_t i = 0; i < nfeat; ++i) trace += aha[i][i].re;
      if (!(trace > 0.0)) throw Fail("the kz calibration acquisition is empty");
      double sc = (double)nfeat / trace;
      for (auto& row : aha)
        for (Cx& a : row) a = cscale(a, sc);
      for (auto& b : ahb)
        for (Cx& v : b) v = cscale(v, sc);
      for (size_t i = 0; i < nfeat; ++i) aha[i][i].re += 1e-8;
      std::vector<Cx> w;
      for (auto& b : ahb)
        for (const Cx& x : solve_hermitian(aha, b)) w.push_back(x);
      K.weights[{d, pat}] = w;
    }
    return K;
  }
  void fill(const SpiralTabO& T, std::vector<std::vector<Cx>>& k, size_t nsamp) const {
    for (auto& [p, d, pat] : targets(T, accel)) {
      auto it = weights.find({d, pat});
      if (it == weights.end()) continue;
      const std::vector<Cx>& w = it->second;
      std::vector<size_t> srcs;
      auto all = offsets(accel, d);
      for (size_t s = 0; s < 4; ++s)
        if (pat & (1u << s)) srcs.push_back((size_t)((int64_t)p + all[s]));
      size_t nfeat = srcs.size() * nc;
      for (size_t j = 0; j < nsamp; ++j)
        for (size_t qt = 0; qt < nc; ++qt) {
          Cx v{0, 0};
          for (size_t s = 0; s < srcs.size(); ++s)
            for (size_t qs = 0; qs < nc; ++qs) v = cadd(v, cmul(w[qt * nfeat + s * nc + qs], k[qs][srcs[s] * nsamp + j]));
          k[qt][p * nsamp + j] = v;
        }
    }
  }
};

// `pocs_along_z` (kspace3d.rs:1201-1259)
std::vector<std::vector<Cx>> pocs_along_z_o(const std::vector<std::vector<Cx>>& h, size_t lo, const std::vector<Cx>& zk,
                                            size_t nz) {
  size_t nplane = h[0].size(), c = nz / 2;
  size_t m = std::min(c - lo, nz - 1 - c);
  auto hann = [&](size_t p) {
    double d = std::fabs((double)p - (double)c);
    return d > (double)m ? 0.0 : 0.5 * (1.0 + std::cos(PI * d / ((double)m + 1.0)));
  };
  auto inv = [&](const std::vector<Cx>& k, size_t z) {
    Cx acc{0, 0};
    for (size_t p = 0; p < nz; ++p) acc = cadd(acc, cmul(k[p], Cx{zk[p * nz + z].re, -zk[p * nz + z].im}));
    return cscale(acc, 1.0 / (double)nz);
  };
  auto fwd = [&](const std::vector<Cx>& x, size_t p) {
    Cx acc{0, 0};
    for (size_t z = 0; z < nz; ++z) acc = cadd(acc, cmul(x[z], zk[p * nz + z]));
    return acc;
  };
  std::vector<std::vector<Cx>> out(nz, std::vector<Cx>(nplane));
  std::vector<Cx> k(nz), x(nz), low(nz), unit(nz);
  for (size_t i = 0; i < nplane; ++i) {
    for (size_t p = 0; p < nz; ++p) {
      k[p] = p >= lo ? h[p][i] : Cx{0, 0};
      low[p] = cscale(k[p], hann(p));
    }
    for (size_t z = 0; z < nz; ++z) {
      Cx v = inv(low, z);
      double a = cabs_(v);
      unit[z] = a > 0.0 ? cscale(v, 1.0 / a) : Cx{1.0, 0.0};
    }
    for (int it = 0; it < 10; ++it) {
      for (size_t z = 0; z < nz; ++z) x[z] = cscale(unit[z], cabs_(inv(k, z)));
      for (size_t p = 0; p < lo; ++p) k[p] = fwd(x, p);
    }
    for (size_t z = 0; z < nz; ++z) out[z][i] = inv(k, z);
  }
  return out;
}

// `spiral_volumes` (kspace3d.rs:1472-1569)
std::vector<std::vector<Cx>> spiral_volumes_o(const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                                              const mrsim_echo_train& tr, const mrsim_spiral_readout& ro,
                                              const mrsim_kz_options* opts, uint64_t seed, int threads) {
  SpiralPlanO pl;
  pl.snx = in.sim_dims[0];
  pl.sny = in.sim_dims[1];
  pl.nz = in.sim_dims[2];
  pl.n = in.acq_dims[0];
  pl.o = pl.snx / pl.n;
  pl.ncomp = in.ncomp;
  size_t ncoils = std::max<int64_t>(acq.n_coils, 1);
  pl.rows = opts ? (size_t)opts->coil_rows : 1;
  pl.ring = ncoils / pl.rows;
  pl.acq = acq;
  pl.table = spiral_table_o(tr, ro, pl.n, pl.nz);
  check_all_sets(in, (int64_t)pl.table.n_shots);
  pl.modes = resolve_modes_o(in.t2, in.t1, in.t_inhom, pl.ncomp, acq, tr, pl.snx * pl.sny * pl.nz);
  pl.t2 = in.t2;
  pl.ti = in.t_inhom;
  pl.fmap = in.fmap;
  if (in.phase) pl.phase = *in.phase;
  else std::memset(&pl.phase, 0, sizeof pl.phase);
  double zs = (double)(pl.nz / 2);
  pl.zk.resize(pl.nz * pl.nz);
  for (size_t p = 0; p < pl.nz; ++p)
    for (size_t z = 0; z < pl.nz; ++z) pl.zk[p * pl.nz + z] = ccis(TAU * ((double)p - zs) * ((double)z - zs) / (double)pl.nz);
  size_t nz = pl.nz, n = pl.n, nsamp = pl.table.nsamp, nv = in.n_volumes;
  double sigma = std::sqrt(acq.noise_variance / (double)(n * n));
  KzGrappaO kzk;
  bool accel = ro.kz.accel > 1;
  if (accel) {
    mrsim_spiral_readout cro = ro;
    cro.kz.accel = 1;
    mrsim_echo_train ctr = tr;
    size_t n_cal = pl.nz - pl.table.band_start;  // the band without the acceleration
    ctr.etl = (int64_t)(n_cal / (size_t)tr.kz_segments);
    SpiralPlanO cal = pl;
    cal.table = spiral_table_o(ctr, cro, pl.n, pl.nz);
    cal.modes = resolve_modes_o(in.t2, in.t1, in.t_inhom, pl.ncomp, acq, ctr, pl.snx * pl.sny * pl.nz);
    auto samples = cal.samples_all(opts->calibration_images, 1, 0, nullptr);
    if (sigma > 0.0)
      for (size_t q = 0; q < samples.size(); ++q)
        spiral_noise_o(samples[q], cal.table.acquired, nsamp, 0, q, opts->calibration_seed ^ 0x4B5A43414C00ull, sigma);
    kzk = KzGrappaO::fit(pl.table, (size_t)ro.kz.accel, samples, nsamp);
  }
  std::vector<std::vector<double>> zsens(ncoils, std::vector<double>(nz));
  for (size_t q = 0; q < ncoils; ++q)
    for (size_t z = 0; z < nz; ++z) zsens[q][z] = coil_row_sensitivity_o(q / pl.ring, pl.rows, (double)z, nz);
  bool pocs = ro.kz.partial_fourier < 1.0 && pl.table.band_start > 0 && opts && opts->pocs;
  mrsim_acquisition wa = acq;
  SpiralReconO rec(pl.table.k.data(), nsamp, n, wa, 80, 100.0, true);
  std::vector<std::vector<Cx>> vols(nv);
  parallel_for(nv, threads, [&](size_t g) {
    auto coil_k = pl.samples_all(in.images, nv, g, in.line_weights, sets_of(in, g), n_sets_of(in, g));
    if (acq.noise_variance > 0.0)
      for (size_t q = 0; q < coil_k.size(); ++q) spiral_noise_o(coil_k[q], pl.table.acquired, nsamp, g, q, seed, sigma);
    if (accel) kzk.fill(pl.table, coil_k, nsamp);
    std::vector<Cx> out(n * n * nz);
    if (pocs) {
      size_t lo = pl.table.band_start;
      std::vector<Cx> wsum(n * n * nz, Cx{0, 0});
      std::vector<double> ssum(n * n * nz, 0.0);
      for (size_t q = 0; q < coil_k.size(); ++q) {
        std::vector<std::vector<Cx>> h(nz);
        for (size_t p = 0; p < nz; ++p)
          h[p] = p >= lo ? rec.image(std::vector<Cx>(coil_k[q].begin() + p * nsamp, coil_k[q].begin() + (p + 1) * nsamp))
                         : std::vector<Cx>(n * n, Cx{0, 0});
        auto img = pocs_along_z_o(h, lo, pl.zk, nz);
        for (size_t z = 0; z < nz; ++z)
          for (size_t i = 0; i < n * n; ++i) {
            double s = coil_sensitivity(q % pl.ring, pl.ring, (double)(i % n), (double)(i / n), n, n) * zsens[q][z];
            wsum[i + n * n * z] = cadd(wsum[i + n * n * z], cscale(img[z][i], s));
            ssum[i + n * n * z] += s * s;
          }
      }
      for (size_t i = 0; i < out.size(); ++i) {
        double s = std::max(ssum[i], 1e-12);
        out[i] = {wsum[i].re / s, wsum[i].im / s};
      }
    } else {
      std::vector<std::vector<std::vector<Cx>>> parts(coil_k.size(), std::vector<std::vector<Cx>>(nz, std::vector<Cx>(nsamp, Cx{0, 0})));
      for (size_t q = 0; q < coil_k.size(); ++q)
        for (size_t z = 0; z < nz; ++z) {
          for (size_t p = 0; p < nz; ++p) {
            Cx kc = pl.zk[p * nz + z];
            Cx conj{kc.re, -kc.im};
            for (size_t j = 0; j < nsamp; ++j) parts[q][z][j] = cadd(parts[q][z][j], cmul(coil_k[q][p * nsamp + j], conj));
          }
          for (Cx& v : parts[q][z]) v = cscale(v, 1.0 / (double)nz);
        }
      for (size_t z = 0; z < nz; ++z) {
        std::vector<Cx> coils;
        std::vector<double> zz;
        for (size_t q = 0; q < coil_k.size(); ++q) {
          coils.insert(coils.end(), parts[q][z].begin(), parts[q][z].end());
          zz.push_back(zsens[q][z]);
        }
        auto img = rec.rings(coils.data(), coil_k.size(), pl.ring, zz.data());
        for (size_t i = 0; i < n * n; ++i) out[i + n * n * z] = img[i];
      }
    }
    vols[g] = out;
  });
  return vols;
}


// ============================ the 3D gradient-echo train ==================================
// readout.rs:356-450 (`ExcitationTrain`, `ge3d_lines`), kspace3d.rs:590-856 (`GePlan`,
// `simulate_acquisition_3d_ge_complex`).
struct GeSetO {
  std::vector<int64_t> shots;
  std::vector<std::vector<float>> images;
};
struct GeVolO {
  std::vector<std::vector<float>> images;  // empty = unused
  std::vector<double> weights;
  std::vector<GeSetO> sets;                // `shot_images`
};

// `GeVolume` with its shot images (kspace3d.rs:592-603; checks kspace3d.rs:801-807); the
// reference scan takes none (`shot_images: None`, kspace3d.rs:775).
GeVolO ge_copy(const mrsim_ge_volume& v, size_t ncomp, size_t nvox, size_t n_exc_lines, size_t g = 0,
               int64_t n_shots = 0, bool with_sets = false) {
  GeVolO o;
  o.images.resize(ncomp);
  for (size_t c = 0; c < ncomp; ++c)
    if (v.images[c]) o.images[c].assign(v.images[c], v.images[c] + nvox);
  o.weights.assign(v.weights, v.weights + n_exc_lines);
  if (with_sets && v.shot_sets)
    for (int64_t i = 0; i < v.n_shot_sets; ++i) {
      const mrsim_shot_set& ss = v.shot_sets[i];
      GeSetO so;
      so.shots.assign(ss.shots, ss.shots + ss.n_shots);
      so.images.resize(ncomp);
      for (size_t c = 0; c < ncomp; ++c) {
        const bool has = ss.images && ss.images[c];
        if (has != (v.images[c] != nullptr))
          throw std::runtime_error("volume " + std::to_string(g) + ": shot images are not the volume's compartments");
        if (has) so.images[c].assign(ss.images[c], ss.images[c] + nvox);
      }
      for (int64_t x : so.shots)
        if (x < 0 || x >= n_shots) throw std::runtime_error("a shot index beyond the train's " + std::to_string(n_shots));
      o.sets.push_back(std::move(so));
    }
  return o;
}

struct GePlanO {
  size_t snx, sny, nz, nx, ny, o, ncomp, kys;
  std::vector<int64_t> line_shot;  // [p][ky]: `ge3d_lines` shot sy * kz_segments + sz (readout.rs:440-450)
  int64_t n_shots = 0;
  mrsim_acquisition acq;
  std::vector<double> t_ms;
  std::vector<int8_t> pol;
  std::vector<std::pair<bool, std::pair<double, double>>> cls;  // (class?, (T2, T2'))
  const mrsim_t2* t2;
  const mrsim_t2* ti;
  const float* fmap;
  mrsim_phase_model phase;
  std::vector<Cx> zk;
  std::vector<uint8_t> mask;

  std::vector<std::vector<Cx>> compartments(const GeVolO& vol, size_t q, size_t ncoils, double te) const {
    size_t nplane = snx * sny;
    mrsim_acquisition base = acq;
    base.echo = MRSIM_ECHO_GRADIENT;
    base.t_echo = te;
    base.noise_variance = 0.0;
    base.n_spikes = 0;
    mrsim_acquisition norel = base, rel = base;
    norel.do_relaxation = 0;
    rel.do_relaxation = 1;
    LineTiming within;
    within.t_ms = t_ms;
    for (double t : t_ms) within.trf_ms.push_back(te + t);
    within.tread_ms = t_ms;
    within.polarity = pol;
    Shot zero;
    std::vector<std::vector<Cx>> out(ncomp);
    for (size_t c = 0; c < ncomp; ++c) {
      if (vol.images[c].empty()) continue;
      bool voxel = !cls[c].first && acq.do_relaxation;
      const mrsim_acquisition& ac = voxel ? rel : norel;
      std::vector<std::vector<Cx>> k2(nz);
      for (size_t z = 0; z < nz; ++z) {
        std::vector<double> phi = phase_slice(phase, zero, snx, sny, o, z, nz);
        const float* comps[1] = {vol.images[c].data() + z * nplane};
        mrsim_t2 t2s[1] = {t2[c].is_map ? mrsim_t2{t2[c].map + z * nplane, 0.f, 1} : t2[c]};
        mrsim_t2 tis[1];
        if (ti) tis[0] = ti[c].is_map ? mrsim_t2{ti[c].map + z * nplane, 0.f, 1} : ti[c];
        mrsim_slice_input inp;
        std::memset(&inp, 0, sizeof inp);
        inp.compartments = comps;
        inp.ncomp = 1;
        inp.t2 = t2s;
        inp.t_inhom = ti ? tis : nullptr;
        inp.fmap = fmap + z * nplane;
        inp.phase0 = phi.data();
        inp.sim[0] = (int64_t)snx;
        inp.sim[1] = (int64_t)sny;
        inp.acq_matrix[0] = (int64_t)nx;
        inp.acq_matrix[1] = (int64_t)ny;
        inp.z = (int64_t)z;
        inp.nz = (int64_t)nz;
        k2[z] = build_coil_kspace_timed(inp, ac, q, ncoils, within, nullptr);
      }
      std::vector<Cx> kc(nz * ny * nx);
      for (size_t p = 0; p < nz; ++p)
        for (size_t ky = 0; ky < ny; ++ky) {
          double w = 1.0;
          if (cls[c].first && acq.do_relaxation) {
            double trf = te + t_ms[ky], t2v = cls[c].second.first, tpv = cls[c].second.second;
            double d2 = std::isinf(t2v) ? 0.0 : trf / t2v, dp = std::isinf(tpv) ? 0.0 : trf / tpv;
            w = std::exp(-d2 - dp);
          }
          for (size_t kx = 0; kx < nx; ++kx) {
            Cx acc{0, 0};
            for (size_t z = 0; z < nz; ++z) acc = cadd(acc, cmul(k2[z][ky * nx + kx], zk[p * nz + z]));
            kc[(p * ny + ky) * nx + kx] = cscale(acc, w);
          }
        }
      out[c] = kc;
    }
    return out;
  }

  // `GePlan::kspace` kspace3d.rs:697-728: each line from the images its shot saw
  std::vector<Cx> kspace(const GeVolO& vol, size_t q, size_t ncoils, double te) const {
    auto base = compartments(vol, q, ncoils, te);
    std::vector<std::vector<std::vector<Cx>>> moved;
    for (const GeSetO& st : vol.sets) {
      GeVolO sv;
      sv.images = st.images;
      moved.push_back(compartments(sv, q, ncoils, te));
    }
    std::vector<Cx> k(nz * ny * nx, Cx{0, 0});
    for (size_t p = 0; p < nz; ++p)
      for (size_t ky = 0; ky < ny; ++ky) {
        if (!mask[ky * nx]) continue;
        size_t sy = ky % kys;
        const std::vector<std::vector<Cx>>* src = &base;
        const int64_t shot = line_shot[p * ny + ky];
        for (size_t i = 0; i < vol.sets.size(); ++i)
          if (std::find(vol.sets[i].shots.begin(), vol.sets[i].shots.end(), shot) != vol.sets[i].shots.end()) {
            src = &moved[i];
            break;
          }
        for (size_t c = 0; c < ncomp; ++c) {
          if (vol.images[c].empty()) continue;
          double w = vol.weights[(p * kys + sy) * ncomp + c];
          for (size_t kx = 0; kx < nx; ++kx) {
            size_t i = (p * ny + ky) * nx + kx;
            k[i] = cadd(k[i], cscale((*src)[c][i], w));
          }
        }
      }
    return k;
  }
};

std::vector<std::vector<std::vector<Cx>>> ge_volumes_o(const mrsim_acquisition_ge_input& in, const mrsim_acquisition& acq,
                                                       const mrsim_excitation_train& tr, const mrsim_ge3d_readout& ro,
                                                       uint64_t seed, int threads) {
  GePlanO pl;
  pl.snx = in.sim_dims[0];
  pl.sny = in.sim_dims[1];
  pl.nz = in.sim_dims[2];
  pl.nx = in.acq_dims[0];
  pl.ny = in.acq_dims[1];
  pl.o = pl.snx / pl.nx;
  pl.ncomp = in.ncomp;
  pl.kys = (size_t)ro.ky_segments;
  pl.acq = acq;
  {
    const size_t kzs = (size_t)tr.kz_segments;
    std::vector<size_t> order = kz_order_o(pl.nz, tr.kz_order), pos(pl.nz, 0);
    for (size_t i = 0; i < order.size(); ++i) pos[order[i]] = i;
    pl.line_shot.resize(pl.nz * pl.ny);
    for (size_t p = 0; p < pl.nz; ++p)
      for (size_t ky = 0; ky < pl.ny; ++ky)
        pl.line_shot[p * pl.ny + ky] = (int64_t)((ky % pl.kys) * kzs + pos[p] % kzs);
    pl.n_shots = (int64_t)(pl.kys * kzs);
  }
  size_t epi = pl.ny / pl.kys;
  for (size_t ky = 0; ky < pl.ny; ++ky) {  // `grase_block`
    size_t j = ky / pl.kys, a = ro.reverse_phase ? j : epi - 1 - j;
    pl.t_ms.push_back(((double)a - ((double)epi - 1.0) / 2.0) * ro.t_line_ms);
    pl.pol.push_back(a % 2 == 1 ? -1 : 1);
  }
  for (size_t c = 0; c < pl.ncomp; ++c) {
    mrsim_t2 tic = in.t_inhom ? in.t_inhom[c] : mrsim_t2{nullptr, (float)acq.t_inhom, 0};
    bool u = !in.t2[c].is_map && !tic.is_map;
    pl.cls.push_back({u, {(double)in.t2[c].value, (double)tic.value}});
  }
  pl.t2 = in.t2;
  pl.ti = in.t_inhom;
  pl.fmap = in.fmap;
  if (in.phase) pl.phase = *in.phase;
  else std::memset(&pl.phase, 0, sizeof pl.phase);
  double zs = (double)(pl.nz / 2);
  pl.zk.resize(pl.nz * pl.nz);
  for (size_t p = 0; p < pl.nz; ++p)
    for (size_t z = 0; z < pl.nz; ++z) pl.zk[p * pl.nz + z] = ccis(TAU * ((double)p - zs) * ((double)z - zs) / (double)pl.nz);
  pl.mask = sampling_mask(pl.nx, pl.ny, acq);
  size_t nz = pl.nz, nx = pl.nx, ny = pl.ny, nv = in.n_volumes, nvox = pl.snx * pl.sny * nz;
  size_t ncoils = std::max<int64_t>(acq.n_coils, 1), n_echoes = tr.n_echoes;
  size_t n_exc_lines = nz * pl.kys * pl.ncomp;
  double sigma = std::sqrt(acq.noise_variance / (double)(nx * ny));
  std::vector<GeVolO> vols(nv);
  for (size_t g = 0; g < nv; ++g) {
    mrsim_ge_volume v;
    std::memset(&v, 0, sizeof v);
    if (in.volume((int64_t)g, in.user, &v) != 0) throw Fail("the volume callback failed");
    vols[g] = ge_copy(v, pl.ncomp, nvox, n_exc_lines, g, pl.n_shots, true);
  }
  std::vector<std::vector<GrappaKernel>> kernels(n_echoes);
  if (acq.accel > 1 && nv > 0) {
    GeVolO cal;
    if (in.reference) {
      cal = ge_copy(*in.reference, pl.ncomp, nvox, n_exc_lines);
    } else {
      mrsim_ge_volume v;
      std::memset(&v, 0, sizeof v);
      if (in.volume(0, in.user, &v) != 0) throw Fail("the volume callback failed");
      cal = ge_copy(v, pl.ncomp, nvox, n_exc_lines);
    }
    mrsim_acquisition acq_cal = acq;
    acq_cal.accel = 1;
    acq_cal.n_spikes = 0;
    GePlanO cpl = pl;
    cpl.acq = acq_cal;
    cpl.mask = sampling_mask(nx, ny, acq_cal);
    std::vector<uint8_t> lines = sampling_mask(1, ny, acq_cal);
    for (size_t e = 0; e < n_echoes; ++e) {
      uint64_t se = seed ^ ((uint64_t)e * 0xD1B54A32D192ED03ull);
      std::vector<std::vector<std::vector<Cx>>> parts(ncoils);
      parallel_for(ncoils, threads, [&](size_t q) {
        std::vector<Cx> k = cpl.kspace(cal, q, ncoils, tr.echo_times_ms[e]);
        parts[q] = partitions_to_slices_o(k, cpl.mask, cpl.zk, nx, ny, nz, 0, q, se ^ SEED_SALT_GRAPPA_CAL, acq_cal, sigma);
      });
      for (size_t z = 0; z < nz; ++z) {
        std::vector<std::vector<Cx>> coils(ncoils);
        for (size_t q = 0; q < ncoils; ++q) coils[q] = parts[q][z];
        kernels[e].push_back(grappa_fit(coils, nx, ny, acq.accel, acq.acs_lines, lines));
      }
    }
  }
  std::vector<std::vector<std::vector<Cx>>> out(nv, std::vector<std::vector<Cx>>(n_echoes));
  parallel_for(nv, threads, [&](size_t g) {
    for (size_t e = 0; e < n_echoes; ++e) {
      uint64_t se = seed ^ ((uint64_t)e * 0xD1B54A32D192ED03ull);
      std::vector<std::vector<std::vector<Cx>>> parts(ncoils);
      for (size_t q = 0; q < ncoils; ++q) {
        std::vector<Cx> k = pl.kspace(vols[g], q, ncoils, tr.echo_times_ms[e]);
        parts[q] = partitions_to_slices_o(k, pl.mask, pl.zk, nx, ny, nz, g, q, se, acq, sigma);
      }
      std::vector<Cx> v(nx * ny * nz);
      for (size_t z = 0; z < nz; ++z) {
        std::vector<std::vector<Cx>> coils(ncoils);
        for (size_t q = 0; q < ncoils; ++q) coils[q] = parts[q][z];
        SliceRecon R = reconstruct_coils_full(coils, acq, nx, ny, false, false, false,
                                              kernels[e].empty() ? nullptr : &kernels[e][z]);
        for (size_t i = 0; i < nx * ny; ++i) v[i + nx * ny * z] = R.combined[i];
      }
      out[g][e] = v;
    }
  });
  return out;
}

thread_local std::string g_err;
std::vector<GoldenCase>* g_golden = nullptr;

template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

void put_cx(const std::vector<Cx>& v, double* out) {
  for (size_t i = 0; i < v.size(); ++i) {
    out[2 * i] = v[i].re;
    out[2 * i + 1] = v[i].im;
  }
}

LineTiming timing_from(const mrsim_acquisition& acq, size_t nx, size_t ny, const double* t, const double* trf,
                       const double* tread, const int8_t* pol) {
  if (!t) return line_timing_for(acq, nx, ny);
  LineTiming lt;
  lt.t_ms.assign(t, t + ny);
  lt.trf_ms.assign(trf, trf + ny);
  lt.tread_ms.assign(tread, tread + ny);
  lt.polarity.assign(pol, pol + ny);
  return lt;
}

}  // namespace

// ============================ C ABI for the test harness ===================================
extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

int oracle_acquisition_default(mrsim_acquisition* a) {
  *a = acq_default();
  return 0;
}

int oracle_sampling_mask(int64_t nx, int64_t ny, const mrsim_acquisition* acq, uint8_t* mask) {
  auto m = sampling_mask(nx, ny, *acq);
  memcpy(mask, m.data(), m.size());
  return 0;
}

int64_t oracle_pf_skipped_lines(int64_t ny, const mrsim_acquisition* acq) { return pf_skipped_lines(ny, *acq); }

int oracle_line_timing(const mrsim_acquisition* acq, int64_t nx, int64_t ny, double* t, double* trf, double* tread,
                       int8_t* pol) {
  auto lt = line_timing_for(*acq, nx, ny);
  memcpy(t, lt.t_ms.data(), ny * 8);
  memcpy(trf, lt.trf_ms.data(), ny * 8);
  memcpy(tread, lt.tread_ms.data(), ny * 8);
  memcpy(pol, lt.polarity.data(), ny);
  return 0;
}

int oracle_epi_order(const mrsim_acquisition* acq, int64_t nx, int64_t ny, int64_t* order) {
  Epi epi{(size_t)nx, (size_t)ny, acq->t_line, acq->t_echo, acq->reverse_phase != 0};
  for (int64_t line = 0; line < ny; ++line) {
    size_t kx, ky;
    epi.kspace_index(line * nx, kx, ky);
    order[line] = ky;
  }
  return 0;
}

int oracle_validate_acquisition_timing(const mrsim_acquisition* acq, int64_t nx, int64_t ny) {
  return guard([&] { validate_acquisition_timing(*acq, nx, ny); });
}

double oracle_coil_sensitivity(int64_t coil, int64_t n_coils, double x, double y, int64_t nx, int64_t ny) {
  return coil_sensitivity(coil, n_coils, x, y, nx, ny);
}

double oracle_window_at(const mrsim_acquisition* acq, double kx, double ky) { return window_at(*acq, kx, ky); }

// build_coil_kspace_timed for one coil (spikes and noise included).
int oracle_build_coil_kspace(const mrsim_slice_input* inp, const mrsim_acquisition* acq, int64_t coil, int64_t ncoils,
                             const double* t, const double* trf, const double* tread, const int8_t* pol,
                             const double* log_amp, double* out) {
  return guard([&] {
    auto lt = timing_from(*acq, inp->acq_matrix[0], inp->acq_matrix[1], t, trf, tread, pol);
    put_cx(build_coil_kspace_timed(*inp, *acq, coil, ncoils, lt, log_amp), out);
  });
}

// the literal sum (no spikes/noise)
int oracle_reference_coil_kspace(const mrsim_slice_input* inp, const mrsim_acquisition* acq, int64_t coil,
                                 int64_t ncoils, double* out) {
  return guard([&] { put_cx(reference_coil_kspace(*inp, *acq, coil, ncoils), out); });
}

int oracle_inverse_2d(const double* k, int64_t nx, int64_t ny, double* out) {
  std::vector<Cx> v(nx * ny);
  for (int64_t i = 0; i < nx * ny; ++i) v[i] = {k[2 * i], k[2 * i + 1]};
  put_cx(inverse_2d(v, nx, ny, nx / 2, ny / 2), out);
  return 0;
}

// simulate_slice_full: combined (f64 pairs), optional captures (n_coils*nx*ny pairs each).
int oracle_simulate_slice_full(const mrsim_slice_input* inp, const mrsim_acquisition* acq, double* combined,
                               double* acquired, double* reconstructed, double* coil_images, double* sens) {
  return guard([&] {
    SliceRecon r = simulate_slice_with(*inp, *acq, acquired != nullptr, reconstructed != nullptr,
                                       coil_images != nullptr, nullptr);
    put_cx(r.combined, combined);
    size_t per = r.combined.size();
    for (size_t c = 0; c < r.acquired.size(); ++c) put_cx(r.acquired[c], acquired + 2 * per * c);
    for (size_t c = 0; c < r.reconstructed.size(); ++c) put_cx(r.reconstructed[c], reconstructed + 2 * per * c);
    for (size_t c = 0; c < r.coil_images.size(); ++c) put_cx(r.coil_images[c], coil_images + 2 * per * c);
    if (sens)
      for (size_t c = 0; c < r.sensitivities.size(); ++c)
        memcpy(sens + per * c, r.sensitivities[c].data(), per * 8);
  });
}

int oracle_simulate_slice(const mrsim_slice_input* inp, const mrsim_acquisition* acq, float* out) {
  return guard([&] {
    SliceRecon r = simulate_slice_with(*inp, *acq, false, false, false, nullptr);
    for (size_t i = 0; i < r.combined.size(); ++i) {
      out[2 * i] = (float)r.combined[i].re;
      out[2 * i + 1] = (float)r.combined[i].im;
    }
  });
}

// GRAPPA fit on given coil k-spaces; weights out: (accel-1)*nc*6nc complex pairs.
int oracle_grappa_fit(const double* coils, int64_t nc, int64_t nx, int64_t ny, int64_t accel, int64_t acs_lines,
                      const uint8_t* lines, double* weights) {
  return guard([&] {
    std::vector<std::vector<Cx>> cv(nc, std::vector<Cx>(nx * ny));
    for (int64_t c = 0; c < nc; ++c)
      for (int64_t i = 0; i < nx * ny; ++i) cv[c][i] = {coils[2 * (c * nx * ny + i)], coils[2 * (c * nx * ny + i) + 1]};
    std::vector<uint8_t> l(lines, lines + ny);
    GrappaKernel K = grappa_fit(cv, nx, ny, accel, acs_lines, l);
    size_t p = 0;
    for (auto& d : K.weights)
      for (auto& co : d)
        for (auto& w : co) {
          weights[p++] = w.re;
          weights[p++] = w.im;
        }
  });
}

int oracle_acquire_volumes_complex(const mrsim_acquisition_input* in, const mrsim_acquisition* acq,
                                   const mrsim_acquisition_options* opts, uint64_t excitation_seed,
                                   uint64_t receiver_seed, int threads, mrsim_acquisition_output* out) {
  return guard([&] {
    SeriesOut so = acquire_volumes_complex(*in, *acq, opts, excitation_seed, receiver_seed, threads);
    memcpy(out->re, so.re.data(), so.re.size() * 4);
    memcpy(out->im, so.im.data(), so.im.size() * 4);
    if (out->acquired && !so.acquired.empty()) memcpy(out->acquired, so.acquired.data(), so.acquired.size() * 4);
    if (out->reconstructed && !so.reconstructed.empty())
      memcpy(out->reconstructed, so.reconstructed.data(), so.reconstructed.size() * 4);
    if (out->coil_images && !so.coil_images.empty())
      memcpy(out->coil_images, so.coil_images.data(), so.coil_images.size() * 4);
    if (out->combined && !so.combined.empty()) memcpy(out->combined, so.combined.data(), so.combined.size() * 4);
    if (out->mask && !so.mask.empty()) memcpy(out->mask, so.mask.data(), so.mask.size());
    if (out->sensitivities && !so.sensitivities.empty())
      memcpy(out->sensitivities, so.sensitivities.data(), so.sensitivities.size() * 4);
  });
}

// `echo_salt` kspace.rs:2130
uint64_t oracle_echo_salt(uint64_t e) { return e * 0xD1B54A32D192ED03ull; }

// `phase_slice` with an optional prep shot
int oracle_phase_slice(const mrsim_phase_model* m, int32_t has_shot, double magnitude, const double* dir,
                       int64_t volume, uint64_t seed, int64_t snx, int64_t sny, int64_t o, int64_t z, int64_t nz,
                       double* out) {
  Shot s;
  if (has_shot && m->has_prep) s = prep_shot(*m, magnitude, dir, volume, z, seed);
  auto v = phase_slice(*m, s, snx, sny, o, z, nz);
  memcpy(out, v.data(), v.size() * 8);
  return 0;
}

uint64_t oracle_rng_next(uint64_t seed, int64_t n, uint64_t* out) {
  Rng r(seed);
  for (int64_t i = 0; i < n; ++i) out[i] = r.next_u64();
  return r.s;
}

// The series operator pair: kspace [g][z][coil][echo][ny][nx] complex128; grads [g][z][c][p].
int oracle_series_forward(const mrsim_acquisition_input* in, const mrsim_acquisition* acq, const double* tes,
                          int64_t ne, const int64_t* slice_z, int64_t nz_full, int threads, double* out) {
  return guard([&] { series_forward(*in, *acq, tes, ne > 0 ? ne : 1, slice_z, nz_full, threads, out); });
}

int oracle_series_adjoint(const mrsim_acquisition_input* in, const mrsim_acquisition* acq, const double* tes,
                          int64_t ne, const int64_t* slice_z, int64_t nz_full, int threads, const double* kspace,
                          double* comp_grad, double* fmap_grad, double* r2_grad) {
  return guard([&] {
    series_adjoint(*in, *acq, tes, ne > 0 ? ne : 1, slice_z, nz_full, threads, kspace, comp_grad, fmap_grad, r2_grad);
  });
}

int oracle_golden_count(void) {
  if (!g_golden) g_golden = new std::vector<GoldenCase>(golden_outputs());
  return (int)g_golden->size();
}

const char* oracle_golden_name(int i) {
  oracle_golden_count();
  return (*g_golden)[i].name.c_str();
}

int64_t oracle_golden_output(int i, uint32_t* out, int64_t cap) {
  oracle_golden_count();
  auto& b = (*g_golden)[i].bits;
  if (out && cap >= (int64_t)b.size()) memcpy(out, b.data(), b.size() * 4);
  return (int64_t)b.size();
}

// The reference's `kspace` build (1) or its default build (0) for every later oracle call.
void oracle_set_kspace_build(int on) {
  if ((on ? 1 : 0) != g_kspace_build) {  // the cached golden outputs belong to the other build
    delete g_golden;
    g_golden = nullptr;
  }
  g_kspace_build = on ? 1 : 0;
}
int oracle_kspace_build(void) { return g_kspace_build; }


int oracle_nufft2(int32_t type, const int64_t* n, const int64_t* m_lo, const int64_t* m_out, double tol,
                  const double* u, int64_t npts, const double* in, int32_t sign, double* out) {
  return guard([&] {
    Nufft2O f(n, m_lo, m_out, tol);
    std::vector<Cx> r = type == 1 ? f.type1(u, (size_t)npts, reinterpret_cast<const Cx*>(in), sign)
                                  : f.type2(reinterpret_cast<const Cx*>(in), u, (size_t)npts, sign);
    put_cx(r, out);
  });
}

int oracle_nufft2_direct(int32_t type, const int64_t* n, const int64_t* m_lo, const int64_t* m_out, const double* u,
                         int64_t npts, const double* in, int32_t sign, double* out) {
  return guard([&] { put_cx(nufft2_direct(type, n, m_lo, m_out, u, (size_t)npts, reinterpret_cast<const Cx*>(in), sign), out); });
}

int oracle_spiral_kspace_exact(const mrsim_slice_input* inp, const mrsim_acquisition* acq, int64_t coil, int64_t ncoils,
                               const double* k, const double* tau, int64_t npts, const double* log_amp, double* out) {
  return guard([&] {
    put_cx(spiral_kspace_exact(*inp, *acq, (size_t)coil, (size_t)ncoils, k, tau, (size_t)npts, log_amp), out);
  });
}

int oracle_spiral_segmented(const mrsim_slice_input* inp, const mrsim_acquisition* acq, int64_t coil, int64_t ncoils,
                            const double* k, const int64_t* tau_idx, int64_t npts, const double* tau_l, int64_t L,
                            const double* b, const double* log_amp, int32_t decay_inside, double* out) {
  return guard([&] {
    put_cx(spiral_segmented(*inp, *acq, (size_t)coil, (size_t)ncoils, k, tau_idx, (size_t)npts, tau_l, (size_t)L, b,
                            log_amp, decay_inside != 0),
           out);
  });
}

// mode 0: reconstruct_rings of batch partitions; 1: image of each of batch sample sets; 2: gridding
int oracle_spiral_recon(const double* k, int64_t npts, int64_t n, int32_t window_kind, double window_a, double window_b,
                        int64_t iterations, double kappa, int32_t band, int32_t mode, const double* data, int64_t batch,
                        int64_t ncoils, int64_t ring, const double* zsens, double* out, double* lambda_hi,
                        int64_t* power_its, double* weights) {
  return guard([&] {
    mrsim_acquisition wa = acq_default();
    wa.window_kind = window_kind;
    wa.window_a = window_a;
    wa.window_b = window_b;
    SpiralReconO r(k, (size_t)npts, (size_t)n, wa, (size_t)iterations, kappa, band != 0);
    if (lambda_hi) *lambda_hi = r.lambda_hi;
    if (power_its) *power_its = r.power_its;
    if (weights) std::memcpy(weights, r.w.data(), r.w.size() * 8);
    const Cx* d = reinterpret_cast<const Cx*>(data);
    size_t nn = (size_t)(n * n);
    for (int64_t b = 0; b < batch; ++b) {
      std::vector<Cx> o;
      if (mode == 0)
        o = r.rings(d + (size_t)b * ncoils * npts, (size_t)ncoils, (size_t)ring, zsens + (size_t)b * ncoils);
      else if (mode == 1)
        o = r.image(std::vector<Cx>(d + (size_t)b * npts, d + (size_t)(b + 1) * npts));
      else
        o = r.gridding(std::vector<Cx>(d + (size_t)b * npts, d + (size_t)(b + 1) * npts));
      put_cx(o, out + 2 * nn * (size_t)b);
    }
  });
}

int oracle_kz_order(int64_t nz, int32_t order, int64_t* out) {
  return guard([&] {
    auto v = kz_order_o((size_t)nz, order);
    for (size_t i = 0; i < v.size(); ++i) out[i] = (int64_t)v[i];
  });
}

int oracle_epg_cpmg(int64_t n, double esp, double b, double t1, double t2, double* out) {
  return guard([&] {
    auto v = epg_cpmg_o((size_t)n, esp, b, t1, t2);
    std::memcpy(out, v.data(), v.size() * 8);
  });
}

int oracle_grase_lines(const mrsim_echo_train* tr, const mrsim_grase_readout* ro, int64_t ny, int64_t nz, int64_t* shot,
                       int64_t* echo, double* t_ms, double* trf_ms, int8_t* pol, int64_t* e_c, int64_t* n_shots) {
  return guard([&] {
    GTable T = grase_lines_o(*tr, *ro, (size_t)ny, (size_t)nz);
    for (size_t i = 0; i < T.lines.size(); ++i) {
      shot[i] = (int64_t)T.lines[i].shot;
      echo[i] = (int64_t)T.lines[i].echo;
      t_ms[i] = T.lines[i].t_ms;
      trf_ms[i] = T.lines[i].trf_ms;
      pol[i] = T.lines[i].pol;
    }
    *e_c = (int64_t)T.e_c;
    *n_shots = (int64_t)T.n_shots;
  });
}

int oracle_kspace_3d_observed(const mrsim_acquisition_3d_input* in, const mrsim_acquisition* acq,
                              const mrsim_echo_train* tr, const mrsim_grase_readout* ro, int64_t g, double* out) {
  return guard([&] {
    Plan3 pl = plan3(*in, *acq, *tr, *ro);
    size_t ncoils = std::max<int64_t>(acq->n_coils, 1), per = pl.nz * pl.ny * pl.nx;
    for (size_t q = 0; q < ncoils; ++q) {
      std::vector<Cx> k = pl.kspace(in->images, in->n_volumes, (size_t)g, q, ncoils, in->line_weights,
                                    sets_of(*in, (size_t)g), n_sets_of(*in, (size_t)g));
      put_cx(k, out + 2 * per * q);
    }
  });
}

// `simulate_acquisition_3d` (kspace3d.rs:549-589): complex volumes [g][vox] (FP64) and the f32
// magnitude / phase at vox * nv + g
int oracle_simulate_acquisition_3d(const mrsim_acquisition_3d_input* in, const mrsim_acquisition* acq,
                                   const mrsim_echo_train* tr, const mrsim_grase_readout* ro, uint64_t seed,
                                   int32_t threads, double* vols_out, float* mag, float* ph) {
  return guard([&] {
    auto vols = acquire_3d_o(*in, *acq, *tr, *ro, seed, threads);
    size_t nv = in->n_volumes;
    for (size_t g = 0; g < vols.size(); ++g) {
      if (vols_out) put_cx(vols[g], vols_out + 2 * vols[g].size() * g);
      for (size_t vox = 0; vox < vols[g].size(); ++vox) {
        float re = (float)vols[g][vox].re, im = (float)vols[g][vox].im;
        if (mag) mag[vox * nv + g] = std::sqrt(re * re + im * im);
        if (ph) ph[vox * nv + g] = std::atan2(im, re);
      }
    }
  });
}

int oracle_spiral_lines(const mrsim_echo_train* tr, const mrsim_spiral_readout* ro, int64_t n, int64_t nz,
                        uint8_t* acquired, int64_t* echo, int64_t* kz_segment, int64_t* band_start, int64_t* e_c,
                        int64_t* n_shots, double* k, double* tau) {
  return guard([&] {
    SpiralTabO T = spiral_table_o(*tr, *ro, (size_t)n, (size_t)nz);
    for (size_t p = 0; p < T.nz; ++p) {
      acquired[p] = T.acquired[p];
      echo[p] = (int64_t)T.echo[p];
      kz_segment[p] = (int64_t)T.kz_segment[p];
    }
    *band_start = (int64_t)T.band_start;
    *e_c = (int64_t)T.e_c;
    *n_shots = (int64_t)T.n_shots;
    if (k) std::memcpy(k, T.k.data(), T.k.size() * 8);
    if (tau) std::memcpy(tau, T.tau.data(), T.tau.size() * 8);
  });
}

int oracle_spiral_samples_3d(const mrsim_acquisition_3d_input* in, const mrsim_acquisition* acq,
                             const mrsim_echo_train* tr, const mrsim_spiral_readout* ro, const mrsim_kz_options* opts,
                             int64_t g, double* out) {
  return guard([&] {
    SpiralPlanO pl;
    pl.snx = in->sim_dims[0];
    pl.sny = in->sim_dims[1];
    pl.nz = in->sim_dims[2];
    pl.n = in->acq_dims[0];
    pl.o = pl.snx / pl.n;
    pl.ncomp = in->ncomp;
    size_t ncoils = std::max<int64_t>(acq->n_coils, 1);
    pl.rows = opts ? (size_t)opts->coil_rows : 1;
    pl.ring = ncoils / pl.rows;
    pl.acq = *acq;
    pl.table = spiral_table_o(*tr, *ro, pl.n, pl.nz);
    check_all_sets(*in, (int64_t)pl.table.n_shots);
    pl.modes = resolve_modes_o(in->t2, in->t1, in->t_inhom, pl.ncomp, *acq, *tr, pl.snx * pl.sny * pl.nz);
    pl.t2 = in->t2;
    pl.ti = in->t_inhom;
    pl.fmap = in->fmap;
    if (in->phase) pl.phase = *in->phase;
    else std::memset(&pl.phase, 0, sizeof pl.phase);
    double zs = (double)(pl.nz / 2);
    pl.zk.resize(pl.nz * pl.nz);
    for (size_t p = 0; p < pl.nz; ++p)
      for (size_t z = 0; z < pl.nz; ++z)
        pl.zk[p * pl.nz + z] = ccis(TAU * ((double)p - zs) * ((double)z - zs) / (double)pl.nz);
    auto s = pl.samples_all(in->images, in->n_volumes, (size_t)g, in->line_weights, sets_of(*in, (size_t)g),
                            n_sets_of(*in, (size_t)g));
    size_t per = pl.nz * pl.table.nsamp;
    for (size_t q = 0; q < s.size(); ++q) put_cx(s[q], out + 2 * per * q);
  });
}

int oracle_simulate_acquisition_3d_spiral(const mrsim_acquisition_3d_input* in, const mrsim_acquisition* acq,
                                          const mrsim_echo_train* tr, const mrsim_spiral_readout* ro,
                                          const mrsim_kz_options* opts, uint64_t seed, int32_t threads,
                                          double* vols_out, float* mag, float* ph) {
  return guard([&] {
    auto vols = spiral_volumes_o(*in, *acq, *tr, *ro, opts, seed, threads);
    size_t nv = in->n_volumes;
    for (size_t g = 0; g < vols.size(); ++g) {
      if (vols_out) put_cx(vols[g], vols_out + 2 * vols[g].size() * g);
      for (size_t vox = 0; vox < vols[g].size(); ++vox) {
        float re = (float)vols[g][vox].re, im = (float)vols[g][vox].im;
        if (mag) mag[vox * nv + g] = std::sqrt(re * re + im * im);
        if (ph) ph[vox * nv + g] = std::atan2(im, re);
      }
    }
  });
}

// `simulate_acquisition_3d_ge` (kspace3d.rs:732-856): complex volumes [e][g][vox] (FP64) and per
// echo the f32 magnitude / phase at vox * nv + g
int oracle_simulate_acquisition_3d_ge(const mrsim_acquisition_ge_input* in, const mrsim_acquisition* acq,
                                      const mrsim_excitation_train* tr, const mrsim_ge3d_readout* ro, uint64_t seed,
                                      int32_t threads, double* vols_out, float* const* mag, float* const* ph) {
  return guard([&] {
    auto vols = ge_volumes_o(*in, *acq, *tr, *ro, seed, threads);
    size_t nv = in->n_volumes, ne = tr->n_echoes;
    size_t nvox = (size_t)(in->acq_dims[0] * in->acq_dims[1] * in->acq_dims[2]);
    for (size_t e = 0; e < ne; ++e)
      for (size_t g = 0; g < nv; ++g) {
        if (vols_out) put_cx(vols[g][e], vols_out + 2 * nvox * (e * nv + g));
        for (size_t vox = 0; vox < nvox; ++vox) {
          float re = (float)vols[g][e][vox].re, im = (float)vols[g][e][vox].im;
          if (mag) mag[e][vox * nv + g] = std::sqrt(re * re + im * im);
          if (ph) ph[e][vox * nv + g] = std::atan2(im, re);
        }
      }
  });
}

// `reconstruct_coils` (kspace.rs:1291-1298) without a GRAPPA kernel: coils [nc][ny*nx] -> combined
int oracle_reconstruct_coils(const double* coils, int64_t nc, int64_t nx, int64_t ny, const mrsim_acquisition* acq,
                             double* out) {
  return guard([&] {
    std::vector<std::vector<Cx>> k(nc, std::vector<Cx>(nx * ny));
    for (int64_t q = 0; q < nc; ++q)
      for (int64_t i = 0; i < nx * ny; ++i) k[q][i] = {coils[2 * (q * nx * ny + i)], coils[2 * (q * nx * ny + i) + 1]};
    SliceRecon R = reconstruct_coils_full(k, *acq, nx, ny, false, false, false, nullptr);
    put_cx(R.combined, out);
  });
}

}  // extern "C"
