// spiral_host.cpp — host plans of the stack-of-spirals path: the spiral trajectory
// (`spiral_tau_c` / `spiral_trajectory`, reference readout.rs:463-653), the certified time
// segmentation (`tseg::plan`, tseg.rs:38-289) and the CPMG echo amplitudes (`epg_cpmg`,
// epg.rs:47-125).  All FP64 on the host: they are per-series plans of a few thousand numbers that
// the device kernels read.
#include "spiral_host.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>

#include "host_tables.h"
#include "mrsim_internal.h"

namespace mrsim {

// ---- spiral trajectory ------------------------------------------------------------------------
double spiral_tau_c(int nx, int interleaves, double readout_ms, double dwell_ms, double radial_oversampling) {
  auto pos = [](double v) { return std::isfinite(v) && v > 0.0; };
  char buf[512];
  if (interleaves <= 0 || !pos(readout_ms) || !pos(dwell_ms)) {
    std::snprintf(buf, sizeof buf,
                  "a spiral needs interleaves > 0, a positive readout time and a positive dwell time (got %d, %g ms, "
                  "%g ms)",
                  interleaves, readout_ms, dwell_ms);
    fail(buf);
  }
  if (!(std::isfinite(radial_oversampling) && radial_oversampling >= 1.0)) {
    std::snprintf(buf, sizeof buf, "a spiral's radial oversampling must be at least 1 (got %g)", radial_oversampling);
    fail(buf);
  }
  const double k_max = nx / 2.0;
  const double n_turns = radial_oversampling * nx / (2.0 * interleaves);
  const double t = readout_ms;
  const double pi = kTau / 2.0;
  const double dwell_max = t / (2.0 * pi * n_turns * k_max);
  const double kd = k_max * dwell_ms;
  const double den = 1.0 / (kd * kd) - 4.0 * pi * pi * n_turns * n_turns / (t * t);
  if (dwell_ms >= dwell_max || den <= 0.0) {
    std::snprintf(buf, sizeof buf,
                  "a %d x %d spiral of %d interleaves (%g turns each) over %g ms cannot be sampled every %g ms: its "
                  "outer turns alone move more than one cycle/FOV per sample. The dwell time must be below %.6e ms (or "
                  "more interleaves, or a longer readout)",
                  nx, nx, interleaves, n_turns, t, dwell_ms, dwell_max);
    fail(buf);
  }
  const double tau_c = 1.0 / (t * den);
  if (tau_c > t) {
    std::snprintf(buf, sizeof buf,
                  "a %d x %d spiral of %d interleaves sampled every %g ms needs a constant-angular-velocity centre of "
                  "%.6f ms to keep within one cycle/FOV per sample, longer than the %g ms readout: the readout is too "
                  "short for the dwell time",
                  nx, nx, interleaves, dwell_ms, tau_c, t);
    fail(buf);
  }
  return tau_c;
}

SpiralTraj spiral_trajectory(int nx, int ny, int interleaves, double readout_ms, double dwell_ms,
                             double radial_oversampling) {
  if (nx != ny) fail("a spiral readout needs a square in-plane matrix, not " + std::to_string(nx) + " x " + std::to_string(ny));
  SpiralTraj tr;
  tr.tau_c_ms = spiral_tau_c(nx, interleaves, readout_ms, dwell_ms, radial_oversampling);
  const int n = (int)std::floor(readout_ms / dwell_ms * (1.0 + 1e-12));
  tr.interleaves = interleaves;
  tr.k_max = nx / 2.0;
  tr.n_turns = radial_oversampling * nx / (2.0 * interleaves);
  tr.readout_ms = readout_ms;
  tr.tau_ms.resize(n);
  for (int j = 0; j < n; ++j) tr.tau_ms[j] = ((double)j + 0.5) * dwell_ms;
  tr.k.reserve((size_t)n * interleaves * 2);
  const double t = readout_ms, tc = tr.tau_c_ms;
  for (int s = 0; s < interleaves; ++s)
    for (int j = 0; j < n; ++j) {
      const double tau = tr.tau_ms[j];
      const double u = tau < tc ? tau / std::sqrt(tc * t) : std::sqrt(tau / t);
      const double th = kTau * (tr.n_turns * u + (double)s / (double)interleaves);
      tr.k.push_back(tr.k_max * u * std::cos(th));
      tr.k.push_back(tr.k_max * u * std::sin(th));
    }
  return tr;
}

// ---- time segmentation ----------------------------------------------------------------------------
namespace {
constexpr double kBoundTarget = 1e-7;
constexpr double kRemainderTarget = 5e-8;
constexpr int kLMax = 64;
constexpr int kMMax = 80;
constexpr double kMaxPhase = 1e4;
constexpr double kRcond = 1e-13;
const double kPi = 3.141592653589793;
const double kEps = 2.220446049250313e-16;

std::vector<double> cheb(double a, double b, int m) {
  if (b <= a) return {a};
  std::vector<double> v(m + 1);
  for (int k = 0; k <= m; ++k)
    v[k] = 0.5 * (a + b) + 0.5 * (b - a) * std::cos((double)(2 * k + 1) * kPi / (double)(2 * (m + 1)));
  return v;
}
double lebesgue(int m) { return 1.0 + 2.0 / kPi * std::log((double)(m + 1)); }
double remainder(double r, double t, int m, double b_sum) {
  if (r <= 0.0) return 0.0;
  const double x = r * t / 4.0;
  double v = 2.0 * (1.0 + b_sum);
  for (int k = 1; k <= m + 1; ++k) v *= x / (double)k;
  return v;
}

// Truncated SVD by one-sided Jacobi (Hestenes) on the narrower side, kept factored
// (`Lsq`, tseg.rs:108-182).
struct Lsq {
  std::vector<std::vector<double>> left, right;
  std::vector<double> sig;

  static Lsq make(const std::vector<std::vector<double>>& cols) {
    const size_t n = cols.size();
    const size_t m = n ? cols[0].size() : 0;
    if (n > m) {
      std::vector<std::vector<double>> rows(m, std::vector<double>(n));
      for (size_t i = 0; i < m; ++i)
        for (size_t c = 0; c < n; ++c) rows[i][c] = cols[c][i];
      Lsq t = make(rows);
      Lsq o;
      o.left = t.right;
      o.right = t.left;
      o.sig = t.sig;
      return o;
    }
    std::vector<std::vector<double>> u = cols;
    std::vector<std::vector<double>> v(n, std::vector<double>(n, 0.0));
    for (size_t i = 0; i < n; ++i) v[i][i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
      bool rotated = false;
      for (size_t p = 0; p < n; ++p)
        for (size_t q = p + 1; q < n; ++q) {
          double alpha = 0.0, beta = 0.0, gamma = 0.0;
          for (size_t k = 0; k < m; ++k) {
            alpha += u[p][k] * u[p][k];
            beta += u[q][k] * u[q][k];
            gamma += u[p][k] * u[q][k];
          }
          if (gamma == 0.0 || std::fabs(gamma) <= 1e-15 * std::sqrt(alpha) * std::sqrt(beta)) continue;
          rotated = true;
          const double zeta = (beta - alpha) / (2.0 * gamma);
          const double sgn = zeta > 0.0 ? 1.0 : (zeta < 0.0 ? -1.0 : 1.0);
          const double t = sgn / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
          const double c = 1.0 / std::sqrt(1.0 + t * t);
          const double s = c * t;
          for (auto* w : {&u, &v}) {
            auto& P = (*w)[p];
            auto& Q = (*w)[q];
            for (size_t k = 0; k < P.size(); ++k) {
              const double x = P[k], y = Q[k];
              P[k] = c * x - s * y;
              Q[k] = s * x + c * y;
            }
          }
        }
      if (!rotated) break;
    }
    std::vector<double> norms(n);
    double smax = 0.0;
    for (size_t k = 0; k < n; ++k) {
      double a = 0.0;
      for (double x : u[k]) a += x * x;
      norms[k] = std::sqrt(a);
      smax = std::max(smax, norms[k]);
    }
    Lsq out;
    for (size_t k = 0; k < n; ++k)
      if (norms[k] > kRcond * smax && norms[k] > 0.0) {
        std::vector<double> l(u[k].size());
        for (size_t i = 0; i < l.size(); ++i) l[i] = u[k][i] / norms[k];
        out.left.push_back(std::move(l));
        out.right.push_back(v[k]);
        out.sig.push_back(norms[k]);
      }
    return out;
  }

  std::vector<double> solve(const std::vector<double>& y) const {
    std::vector<double> x(right.empty() ? 0 : right[0].size(), 0.0);
    for (size_t k = 0; k < left.size(); ++k) {
      double c = 0.0;
      for (size_t i = 0; i < y.size(); ++i) c += left[k][i] * y[i];
      c /= sig[k];
      for (size_t i = 0; i < x.size(); ++i) x[i] += c * right[k][i];
    }
    return x;
  }
};

struct FitOut {
  std::vector<double> tau_l;
  std::vector<double> b;  // (re, im) pairs, [sample][segment]
  double b_sum = 0.0, err = 0.0;
};

// `fit` (tseg.rs:185-227): least-squares interpolators over the rate grid
FitOut fit(const std::vector<double>& tau, double t, int l, const std::vector<std::pair<double, double>>& rates,
           TsegDevice* dev) {
  FitOut o;
  o.tau_l.resize(l);
  for (int i = 0; i < l; ++i) o.tau_l[i] = l == 1 ? 0.0 : t * (double)i / (double)(l - 1);
  const size_t g = rates.size();
  std::vector<std::vector<double>> cols(2 * l, std::vector<double>(2 * g, 0.0));
  for (int i = 0; i < l; ++i)
    for (size_t k = 0; k < g; ++k) {
      const double mag = std::exp(rates[k].first * o.tau_l[i]);
      const double c = std::cos(rates[k].second * o.tau_l[i]) * mag, s = std::sin(rates[k].second * o.tau_l[i]) * mag;
      cols[i][k] = c;
      cols[i][g + k] = s;
      cols[l + i][k] = -s;
      cols[l + i][g + k] = c;
    }
  Lsq p = Lsq::make(cols);
  if (dev) {  // the per-sample solve and residual on the device; b stays there until accepted
    dev->fit(rates, cols, p.left, p.right, p.sig, l, &o.b_sum, &o.err);
    return o;
  }
  std::vector<double> y(2 * g);
  o.b.reserve(tau.size() * l * 2);
  for (double tj : tau) {
    for (size_t k = 0; k < g; ++k) {
      const double mag = std::exp(rates[k].first * tj);
      y[k] = std::cos(rates[k].second * tj) * mag;
      y[g + k] = std::sin(rates[k].second * tj) * mag;
    }
    auto x = p.solve(y);
    double s = 0.0;
    for (int i = 0; i < l; ++i) {
      o.b.push_back(x[i]);
      o.b.push_back(x[l + i]);
      s += std::hypot(x[i], x[l + i]);
    }
    o.b_sum = std::max(o.b_sum, s);
    for (size_t k = 0; k < g; ++k) {
      double re = y[k], im = y[g + k];
      for (int i = 0; i < 2 * l; ++i) {
        re -= cols[i][k] * x[i];
        im -= cols[i][g + k] * x[i];
      }
      o.err = std::max(o.err, std::hypot(re, im));
    }
  }
  return o;
}
}  // namespace

TsegPlan tseg_plan(const std::vector<double>& tau, double t_ms, const double d[2], const double f[2],
                   TsegDevice* dev) {
  char buf[512];
  if (!(d[0] >= 0.0 && d[1] >= d[0] && f[1] >= f[0])) {
    std::snprintf(buf, sizeof buf, "rate rectangle RateRect { d: [%g, %g], f: [%g, %g] }", d[0], d[1], f[0], f[1]);
    fail(buf);
  }
  for (double x : tau)
    if (!(x >= 0.0 && x <= t_ms)) fail("sample times outside [0, T]");
  const double r_d = d[1] - d[0];
  const double r_f = kTau * (f[1] - f[0]) / 1000.0;
  const double w_max = kTau * std::max(std::fabs(f[0]), std::fabs(f[1])) / 1000.0;
  const double theta = t_ms * std::hypot(d[1], w_max);
  if (std::isnan(theta) || theta > kMaxPhase) {
    std::snprintf(buf, sizeof buf,
                  "the time segmentation's rates (decay up to %.4f 1/ms, off-resonance %.2f..%.2f Hz) reach %.3e rad "
                  "over the %g ms readout, past 1e4: not a fieldmap this model certifies",
                  d[1], f[0], f[1], theta, t_ms);
    fail(buf);
  }
  int l = (int)std::ceil((t_ms / 1000.0) * (f[1] - f[0])) + 2;
  if (dev) dev->set_times(tau);
  for (;;) {
    if (l > kLMax) {
      std::snprintf(buf, sizeof buf,
                    "the time segmentation cannot certify 1e-7 within 64 segments over decay rates %.4f..%.4f 1/ms and "
                    "off-resonance %.2f..%.2f Hz on a %g ms readout",
                    d[0], d[1], f[0], f[1], t_ms);
      fail(buf);
    }
    auto rem_total = [&](int m, double b_sum) {
      const double lam_d = r_d > 0.0 ? lebesgue(m) : 1.0;
      return remainder(r_d, t_ms, m, b_sum) + lam_d * remainder(r_f, t_ms, m, b_sum);
    };
    int m = 1;
    while (m < kMMax && rem_total(m, 0.0) >= kRemainderTarget) ++m;
    for (;;) {
      auto ds = cheb(d[0], d[1], m);
      auto fs = cheb(kTau * f[0] / 1000.0, kTau * f[1] / 1000.0, m);
      std::vector<std::pair<double, double>> rates;
      for (double dd : ds)
        for (double w : fs) rates.emplace_back(-dd, w);
      FitOut o = fit(tau, t_ms, l, rates, dev);
      const double rem = rem_total(m, o.b_sum);
      if (rem >= kRemainderTarget && m < kMMax) {
        ++m;
        continue;
      }
      const double lam_d = r_d > 0.0 ? lebesgue(m) : 1.0;
      const double lam_f = r_f > 0.0 ? lebesgue(m) : 1.0;
      const double delta = 4.0 * kEps * (1.0 + theta);
      const double rounding = (lam_d * lam_f + 1.0) * (1.0 + o.b_sum) * (delta + 2.0 * (double)l * kEps);
      const double bound = lam_d * lam_f * o.err + rem + rounding;
      if (bound < kBoundTarget) {
        TsegPlan p;
        p.l = l;
        p.m = m;
        p.tau_l = o.tau_l;
        if (dev)
          dev->fetch_b(p.b);
        else
          p.b = o.b;
        p.b_sum = o.b_sum;
        p.grid_err = o.err;
        p.bound = bound;
        return p;
      }
      break;
    }
    l *= 2;
  }
}

// ---- EPG ----------------------------------------------------------------------------------------
namespace {
struct Cx {
  double re, im;
};
Cx cadd(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
Cx cmul(Cx a, Cx o) { return {a.re * o.re - a.im * o.im, a.re * o.im + a.im * o.re}; }
Cx cscale(Cx a, double s) { return {a.re * s, a.im * s}; }
}  // namespace

std::vector<double> epg_cpmg(int n_echoes, double esp_ms, double refocusing_deg, double t1_ms, double t2_ms) {
  if (!(esp_ms > 0.0 && std::isfinite(esp_ms))) fail("echo spacing " + std::to_string(esp_ms) + " ms");
  if (!(refocusing_deg > 0.0 && refocusing_deg <= 180.0)) fail("refocusing angle " + std::to_string(refocusing_deg));
  if (!(t1_ms > 0.0 && t2_ms > 0.0)) fail("relaxation times must be positive");
  const int n = 2 * n_echoes + 2;
  std::vector<Cx> fp(n, {0, 0}), fm(n, {0, 0}), z(n, {0, 0});
  z[0] = {1.0, 0.0};
  auto pulse = [&](double alpha, double phi) {  // Weigel eq. 15
    const double ch = std::cos(alpha / 2.0), sh = std::sin(alpha / 2.0);
    const double c2 = ch * ch, s2 = sh * sh, sa = std::sin(alpha), ca = std::cos(alpha);
    auto e = [](double a) { return Cx{std::cos(a), std::sin(a)}; };
    const Cx e2p = e(2.0 * phi), e2m = e(-2.0 * phi), e1p = e(phi), e1m = e(-phi);
    const Cx i = {0.0, 1.0}, mi = {0.0, -1.0};
    for (int k = 0; k < n; ++k) {
      const Cx p = fp[k], m = fm[k], zz = z[k];
      fp[k] = cadd(cadd(cscale(p, c2), cscale(cmul(e2p, m), s2)), cscale(cmul(cmul(mi, e1p), zz), sa));
      fm[k] = cadd(cadd(cscale(cmul(e2m, p), s2), cscale(m, c2)), cscale(cmul(cmul(i, e1m), zz), sa));
      z[k] = cadd(cadd(cscale(cmul(cmul(mi, e1m), p), sa / 2.0), cscale(cmul(cmul(i, e1p), m), sa / 2.0)), cscale(zz, ca));
    }
  };
  auto relax = [&](double e1, double e2) {
    for (int k = 0; k < n; ++k) {
      fp[k] = cscale(fp[k], e2);
      fm[k] = cscale(fm[k], e2);
      z[k] = cscale(z[k], e1);
    }
    z[0] = cadd(z[0], {1.0 - e1, 0.0});
  };
  auto shift = [&]() {
    for (int k = n - 1; k >= 1; --k) fp[k] = fp[k - 1];
    for (int k = 0; k < n - 1; ++k) fm[k] = fm[k + 1];
    fm[n - 1] = {0.0, 0.0};
    fp[0] = {fm[0].re, -fm[0].im};
  };
  auto decay = [](double dt, double t) { return std::isinf(t) ? 1.0 : std::exp(-dt / t); };
  pulse(kPi / 2.0, 0.0);
  const double norm = std::hypot(fp[0].re, fp[0].im);
  const double half = esp_ms / 2.0;
  const double e1 = decay(half, t1_ms), e2 = decay(half, t2_ms);
  const double beta = refocusing_deg * kPi / 180.0;
  std::vector<double> out(n_echoes);
  for (int e = 0; e < n_echoes; ++e) {
    relax(e1, e2);
    shift();
    pulse(beta, kPi / 2.0);
    shift();
    relax(e1, e2);
    const double a = std::hypot(fp[0].re, fp[0].im) / norm;
    out[e] = a == 0.0 ? -INFINITY : std::log(a);
  }
  return out;
}

}  // namespace mrsim
