// spiral.cpp — host side of the device NUFFT pair and spiral forwards: geometry tables (FP64
// deapodization and twiddles), the segmented forward's inputs and plan, and the exact forward.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstring>
#include <string>

#include "driver.h"
#include "host_tables.h"
#include "mrsim_internal.h"
#include "nufft.h"
#include "spiral.h"
#include "spiral_host.h"

namespace mrsim {

int nufft_width(double tol) {  // nufft.rs:48, 165
  int w = (int)std::ceil(-std::log10(tol)) + 1;
  return std::min(16, std::max(2, w));
}

// 1/psi-hat(k) of the modes m_lo .. m_lo + m_out on nf fine cells (`deapodization`, nufft.rs:113-123)
static std::vector<double> deapodization(int nf, int w, double beta, int m_lo, int m_out) {
  const double half = w / 2.0;
  auto psi = [&](double z) { return std::fabs(z) < 1.0 ? std::exp(beta * (std::sqrt(1.0 - z * z) - 1.0)) : 0.0; };
  std::vector<double> c(m_out);
  for (int j = 0; j < m_out; ++j) {
    const double k = (double)(m_lo + j);
    double s = psi(0.0);
    for (double m = 1.0; m < half; m += 1.0) s += 2.0 * psi(m / half) * std::cos(kTau * k * m / nf);
    c[j] = 1.0 / s;
  }
  return c;
}

// e^{-i2pi k/n}, k = 0..n-1, on the device in precision R.
template <class R>
const void* upload_twiddles(DevArena& A, int n, cudaStream_t st) {
  using V = typename Vec2<R>::type;
  std::vector<V> t(n);
  for (int k = 0; k < n; ++k) {
    t[k].x = (R)std::cos(-kTau * k / n);
    t[k].y = (R)std::sin(-kTau * k / n);
  }
  return A.upload(t.data(), t.size() * sizeof(V), st);
}
template const void* upload_twiddles<float>(DevArena&, int, cudaStream_t);
template const void* upload_twiddles<double>(DevArena&, int, cudaStream_t);

template <class R>
NufftGridT<R> make_nufft(DevArena& A, int n0, int n1, int m_lo0, int m_lo1, int m_out0, int m_out1, double tol,
                         cudaStream_t st) {
  using V = typename Vec2<R>::type;
  if (m_out0 <= 0 || m_out1 <= 0 || m_lo0 < -(n0 / 2) || m_lo0 + m_out0 - 1 > n0 / 2 || m_lo1 < -(n1 / 2) ||
      m_lo1 + m_out1 - 1 > n1 / 2)
    fail("mode band must sit inside the coarse Nyquist band");
  const int n_max = sizeof(R) == 8 ? 4096 : 8192;  // the fine-grid line must fit in shared memory
  if (n0 <= 0 || n1 <= 0 || n0 > n_max || n1 > n_max)
    fail("NUFFT period must be in 1.." + std::to_string(n_max));
  NufftGridT<R> g;
  std::memset(&g, 0, sizeof g);
  g.n0 = n0;
  g.n1 = n1;
  g.nf0 = 2 * n0;
  g.nf1 = 2 * n1;
  g.w = nufft_width(tol);
  g.beta = (R)(2.30 * g.w);
  g.m_lo0 = m_lo0;
  g.m_lo1 = m_lo1;
  g.m_out0 = m_out0;
  g.m_out1 = m_out1;
  const double beta = 2.30 * g.w;
  auto cast = [](const std::vector<double>& v) { return std::vector<R>(v.begin(), v.end()); };
  auto c0 = cast(deapodization(g.nf0, g.w, beta, m_lo0, m_out0));
  auto c1 = cast(deapodization(g.nf1, g.w, beta, m_lo1, m_out1));
  g.corr0 = (const R*)A.upload(c0.data(), c0.size() * sizeof(R), st);
  g.corr1 = (const R*)A.upload(c1.data(), c1.size() * sizeof(R), st);
  g.tw0 = (const V*)upload_twiddles<R>(A, g.nf0, st);
  g.tw1 = g.nf1 == g.nf0 ? g.tw0 : (const V*)upload_twiddles<R>(A, g.nf1, st);
  return g;
}
template NufftGridT<float> make_nufft<float>(DevArena&, int, int, int, int, int, int, double, cudaStream_t);
template NufftGridT<double> make_nufft<double>(DevArena&, int, int, int, int, int, int, double, cudaStream_t);

// ---- bins of the deterministic spread ----------------------------------------------------------
namespace {
// The tiles of a fine ring of nf cells (tiles of `tile` cells) that the kernel window of a point
// at period coordinate u can reach: the window's cells m0 .. m0 + w - 1 (m0 as the device forms
// it), widened by a cell each side.  A non-finite position reaches none (its taps are zero).
void window_tiles(double u, int nf, int w, int tile, std::vector<int>& out) {
  out.clear();
  if (!std::isfinite(u)) return;
  const double half = 0.5 * w;
  double p = std::fmod(2.0 * u, (double)nf);
  if (p < 0.0) p += nf;
  const long long m0 = (long long)std::floor(p - half) + 1;
  for (long long m = m0 - 1; m <= m0 + w; ++m) {
    const int c = (int)(((m % nf) + nf) % nf);
    const int t = c / tile;
    if (std::find(out.begin(), out.end(), t) == out.end()) out.push_back(t);
  }
}

// CSR of per-tile point lists in point order (two passes: counts, then fill point by point).
NufftBins upload_bins(DevArena& A, int tiles0, int tiles1, int npts, const std::function<void(int, std::vector<int>&)>& tiles_of,
                      cudaStream_t st) {
  const size_t nt = (size_t)tiles0 * tiles1;
  std::vector<int> start(nt + 1, 0), tl;
  for (int j = 0; j < npts; ++j) {
    tiles_of(j, tl);
    for (int t : tl) ++start[(size_t)t + 1];
  }
  for (size_t t = 0; t < nt; ++t) start[t + 1] += start[t];
  std::vector<int> pts((size_t)start[nt]), cur(start.begin(), start.end() - 1);
  for (int j = 0; j < npts; ++j) {
    tiles_of(j, tl);
    for (int t : tl) pts[(size_t)cur[(size_t)t]++] = j;
  }
  NufftBins b;
  b.tiles0 = tiles0;
  b.tiles1 = tiles1;
  b.start = (const int*)A.upload(start.data(), start.size() * 4, st);
  b.pts = (const int*)A.upload(pts.data(), std::max<size_t>(1, pts.size()) * 4, st);
  return b;
}
}  // namespace

NufftBins nufft_bins2(DevArena& A, int nf0, int nf1, int w, const double* u_host, int npts, cudaStream_t st) {
  const int tiles0 = (nf0 + kSpreadTile - 1) / kSpreadTile, tiles1 = (nf1 + kSpreadTile - 1) / kSpreadTile;
  std::vector<int> t0, t1;
  return upload_bins(A, tiles0, tiles1, npts, [&](int j, std::vector<int>& out) {
    window_tiles(u_host[2 * (size_t)j], nf0, w, kSpreadTile, t0);
    window_tiles(u_host[2 * (size_t)j + 1], nf1, w, kSpreadTile, t1);
    out.clear();
    for (int b : t1)
      for (int a : t0) out.push_back(a + tiles0 * b);
  }, st);
}

NufftBins nufft_bins1(DevArena& A, int nf, int w, const double* pos_host, int npos, cudaStream_t st) {
  const int tiles = (nf + kSpreadTile1 - 1) / kSpreadTile1;
  return upload_bins(A, tiles, 1, npos, [&](int j, std::vector<int>& out) {
    window_tiles(pos_host[j], nf, w, kSpreadTile1, out);
  }, st);
}

// ---- the 1D type-1 NUFFT (`Nufft1::new` / `run`, nufft.rs:41-107) on host buffers, FP64 ---------
void nufft1_host(mrsim_context* ctx, int n, int k_lo, int n_out, double tol, const double* pos, int npos,
                 const double* weights, int nw, double* out) {
  if (!(n_out > 0 && k_lo >= -(n / 2) && k_lo + n_out - 1 <= n / 2))
    fail("output band must sit inside the coarse Nyquist band");
  if (n <= 0 || n > 4096) fail("NUFFT period must be in 1..4096");
  cudaStream_t st = ctx->stream;
  DevArena A;
  Nufft1Grid g;
  g.n = n;
  g.nf = 2 * n;
  g.w = nufft_width(tol);
  g.beta = 2.30 * g.w;
  g.k_lo = k_lo;
  g.n_out = n_out;
  auto corr = deapodization(g.nf, g.w, g.beta, k_lo, n_out);
  g.corr = (const double*)A.upload(corr.data(), corr.size() * 8, st);
  g.tw = (const double2*)upload_twiddles<double>(A, g.nf, st);
  const double* dp = npos > 0 ? (const double*)A.upload(pos, (size_t)npos * 8, st) : nullptr;
  const double2* dw = npos > 0 ? (const double2*)A.upload(weights, (size_t)nw * npos * 16, st) : nullptr;
  double2* dout = (double2*)A.alloc((size_t)nw * n_out * 16);
  double2* work = (double2*)A.alloc((size_t)nw * g.nf * 16);
  const NufftBins bins = nufft_bins1(A, g.nf, g.w, pos, npos, st);
  nufft1_run(g, dp, npos, bins, dw, nw, dout, work, st);
  MRSIM_CUDA(cudaGetLastError());
  MRSIM_CUDA(cudaMemcpyAsync(out, dout, (size_t)nw * n_out * 16, cudaMemcpyDeviceToHost, st));
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

// ---- host-buffer NUFFT pair -----------------------------------------------------------------------
void nufft2_host(mrsim_context* ctx, int type, int n0, int n1, int m_lo0, int m_lo1, int m_out0, int m_out1, double tol,
                 const double* u, int npts, const float* in, int sign, float* out) {
  cudaStream_t st = ctx->stream;
  DevArena A;
  NufftGrid g = make_nufft<float>(A, n0, n1, m_lo0, m_lo1, m_out0, m_out1, tol, st);
  const size_t nm = (size_t)m_out0 * m_out1;
  if (npts == 0) {  // no points: type 2 has no values, type 1 all-zero modes
    if (type == 1) std::memset(out, 0, nm * sizeof(float2));
    MRSIM_CUDA(cudaStreamSynchronize(st));
    return;
  }
  const double* du = (const double*)A.upload(u, (size_t)npts * 2 * 8, st);
  float2* work = (float2*)A.alloc((size_t)g.nf0 * g.nf1 * sizeof(float2));
  if (type == 2) {
    const float2* dm = (const float2*)A.upload(in, nm * sizeof(float2), st);
    float2* dout = (float2*)A.alloc((size_t)npts * sizeof(float2));
    nufft_type2<float>(g, dm, 1, nm, du, npts, dout, npts, work, sign, nullptr, st);
    MRSIM_CUDA(cudaGetLastError());
    MRSIM_CUDA(cudaMemcpyAsync(out, dout, (size_t)npts * sizeof(float2), cudaMemcpyDeviceToHost, st));
  } else {
    const float2* dw = (const float2*)A.upload(in, (size_t)npts * sizeof(float2), st);
    float2* dm = (float2*)A.alloc(nm * sizeof(float2));
    const NufftBins bins = nufft_bins2(A, g.nf0, g.nf1, g.w, u, npts, st);
    nufft_type1<float>(g, du, npts, bins, dw, 1, npts, dm, nm, work, sign, st);
    MRSIM_CUDA(cudaGetLastError());
    MRSIM_CUDA(cudaMemcpyAsync(out, dm, nm * sizeof(float2), cudaMemcpyDeviceToHost, st));
  }
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

// ---- the spiral forwards --------------------------------------------------------------------------
namespace {
struct SliceStatics {
  std::vector<double> amp, phi0, rate;  // spiral.rs:33-57
};

SliceStatics slice_statics(const mrsim_slice_input& inp, const mrsim_acquisition& acq, int coil, int ncoils) {
  const int snx = (int)inp.sim[0], sny = (int)inp.sim[1], nx = (int)inp.acq_matrix[0], ny = (int)inp.acq_matrix[1];
  if (!(snx % nx == 0 && sny % ny == 0)) fail("sim grid must be an integer multiple of the acquired matrix");
  if (acq.echo != MRSIM_ECHO_SPIN) fail("the spiral train is a spin-echo train");
  if (inp.has_eddy_drive) fail("the eddy model is not available for spirals");
  const int ox = snx / nx, oy = sny / ny;
  const double xoff = (ox - 1.0) / 2.0, yoff = (oy - 1.0) / 2.0;
  SliceStatics s;
  const size_t n = (size_t)snx * sny;
  s.amp.resize(n);
  s.phi0.resize(n);
  s.rate.resize(n);
  for (int y = 0; y < sny; ++y)
    for (int x = 0; x < snx; ++x) {
      const size_t i = (size_t)x + (size_t)snx * y;
      s.amp[i] = acq.signal_scale * coil_sensitivity(coil, ncoils, ((double)x - xoff) / ox, ((double)y - yoff) / oy, nx, ny);
      s.phi0[i] = inp.phase0 ? inp.phase0[i] : 0.0;
      s.rate[i] = acq.do_distortions ? (double)inp.fmap[i] : 0.0;
    }
  return s;
}

double decay_rate(const mrsim_slice_input& inp, const mrsim_acquisition& acq, int c, size_t i) {  // spiral.rs:60-68
  const double t2 = inp.t2[c].is_map ? (double)inp.t2[c].map[i] : (double)inp.t2[c].value;
  const double tp = inp.t_inhom ? (inp.t_inhom[c].is_map ? (double)inp.t_inhom[c].map[i] : (double)inp.t_inhom[c].value)
                                : acq.t_inhom;
  return 1.0 / t2 + 1.0 / tp;
}
}  // namespace

void spiral_exact_host(mrsim_context* ctx, const mrsim_slice_input& inp, const mrsim_acquisition& acq, int coil,
                       int ncoils, const double* k, const double* tau_ms, int npts, const double* log_amp,
                       float* out) {
  cudaStream_t st = ctx->stream;
  if (inp.ncomp > 4) fail("the exact spiral forward handles up to 4 compartments");
  SliceStatics s = slice_statics(inp, acq, coil, ncoils);
  if (npts == 0) return;
  const int snx = (int)inp.sim[0], sny = (int)inp.sim[1], nx = (int)inp.acq_matrix[0], ny = (int)inp.acq_matrix[1];
  const size_t n = (size_t)snx * sny;
  const int ncomp = (int)inp.ncomp;
  std::vector<float> amp(n), ph(n), rate(n), comp(std::max<size_t>(1, n * ncomp)), dec(std::max<size_t>(1, n * ncomp));
  for (size_t i = 0; i < n; ++i) {
    amp[i] = (float)s.amp[i];
    double t = s.phi0[i] / kTau;
    t -= std::rint(t);
    ph[i] = (float)t;
    rate[i] = (float)s.rate[i];
    for (int c = 0; c < ncomp; ++c) {
      comp[(size_t)c * n + i] = inp.compartments[c][i];
      dec[(size_t)c * n + i] = (float)decay_rate(inp, acq, c, i);
    }
  }
  DevArena A;
  SpiralExactArgs a;
  std::memset(&a, 0, sizeof a);
  a.k = (const double*)A.upload(k, (size_t)npts * 2 * 8, st);
  a.tau_ms = (const double*)A.upload(tau_ms, (size_t)npts * 8, st);
  a.npts = npts;
  a.snx = snx;
  a.sny = sny;
  a.nx = nx;
  a.ny = ny;
  a.ox = snx / nx;
  a.oy = sny / ny;
  a.sxs = a.ox * (nx / 2);
  a.sys = a.oy * (ny / 2);
  a.xoff = (a.ox - 1.0) / 2.0;
  a.yoff = (a.oy - 1.0) / 2.0;
  a.amp = (const float*)A.upload(amp.data(), n * 4, st);
  a.phase_turns = (const float*)A.upload(ph.data(), n * 4, st);
  a.rate = (const float*)A.upload(rate.data(), n * 4, st);
  a.comp = (const float*)A.upload(comp.data(), comp.size() * 4, st);
  a.decay = (const float*)A.upload(dec.data(), dec.size() * 4, st);
  if (log_amp && acq.do_relaxation) {
    std::vector<float> la(n);
    for (size_t i = 0; i < n; ++i) la[i] = (float)log_amp[i];
    a.log_amp = (const float*)A.upload(la.data(), n * 4, st);
  }
  a.ncomp = ncomp;
  a.relax = acq.do_relaxation ? 1 : 0;
  a.inv_nvox = (float)(1.0 / (double)n);
  float2* dout = (float2*)A.alloc((size_t)npts * sizeof(float2));
  a.out = dout;
  spiral_exact(a, st);
  MRSIM_CUDA(cudaGetLastError());
  MRSIM_CUDA(cudaMemcpyAsync(out, dout, (size_t)npts * sizeof(float2), cudaMemcpyDeviceToHost, st));
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

// `segment_inputs` (spiral.rs:83-103) + `SegmentedForward::new` / `apply` (spiral.rs:154-201).
SegmentedInfo spiral_segmented_host(mrsim_context* ctx, const mrsim_slice_input& inp, const mrsim_acquisition& acq,
                                    int coil, int ncoils, const double* k, const int64_t* tau_idx, int npts,
                                    const double* tau_ms, int ntau, double t_ms, const double rect_d[2],
                                    const double rect_f[2], const double* log_amp, bool decay_inside, float* out) {
  cudaStream_t st = ctx->stream;
  if (inp.ncomp != 1) fail("one compartment per segmented forward");
  const int snx = (int)inp.sim[0], sny = (int)inp.sim[1], nx = (int)inp.acq_matrix[0], ny = (int)inp.acq_matrix[1];
  SliceStatics s = slice_statics(inp, acq, coil, ncoils);
  const size_t n = (size_t)snx * sny;
  std::vector<float2> x(n), rate(n);
  for (size_t i = 0; i < n; ++i) {
    double a = s.amp[i] * (double)inp.compartments[0][i];
    double d = 0.0;
    if (decay_inside && acq.do_relaxation) {
      a *= log_amp ? std::exp(log_amp[i]) : 1.0;
      d = decay_rate(inp, acq, 0, i);
    }
    x[i] = make_float2((float)(a * std::cos(s.phi0[i])), (float)(a * std::sin(s.phi0[i])));
    rate[i] = make_float2((float)(-d), (float)(kTau * s.rate[i] / 1000.0));
  }
  std::vector<double> tau(tau_ms, tau_ms + ntau);
  TsegPlan plan;
  {
    TsegDevice dev(st);
    plan = tseg_plan(tau, t_ms, rect_d, rect_f, &dev);
  }
  SegmentedInfo info;
  info.l = plan.l;
  info.m = plan.m;
  info.bound = plan.bound;
  info.b_sum = plan.b_sum;
  info.grid_err = plan.grid_err;
  if (npts == 0) return info;
  const int L = plan.l;
  const int ox = snx / nx, oy = sny / ny;
  const int sxs = ox * (nx / 2), sys = oy * (ny / 2);
  const double xoff = (ox - 1.0) / 2.0, yoff = (oy - 1.0) / 2.0;
  const double ninv = 1.0 / (double)n;
  std::vector<float2> stat(npts);
  std::vector<int> tidx(npts);
  for (int j = 0; j < npts; ++j) {
    const double ph = -kTau * (k[2 * j] * xoff / snx + k[2 * j + 1] * yoff / sny);
    stat[j] = make_float2((float)(std::cos(ph) * ninv), (float)(std::sin(ph) * ninv));
    if (tau_idx[j] < 0 || tau_idx[j] >= ntau) fail("sample-time index out of range");
    tidx[j] = (int)tau_idx[j];
  }
  DevArena A;
  NufftGrid g = make_nufft<float>(A, snx, sny, -sxs, -sys, snx, sny, 1e-12, st);
  const float2* dx = (const float2*)A.upload(x.data(), n * sizeof(float2), st);
  const float2* drate = (const float2*)A.upload(rate.data(), n * sizeof(float2), st);
  const double* dtl = (const double*)A.upload(plan.tau_l.data(), plan.tau_l.size() * 8, st);
  float2* imgs = (float2*)A.alloc((size_t)L * n * sizeof(float2));
  segment_images(dx, drate, (int)n, dtl, L, imgs, st);
  const double* du = (const double*)A.upload(k, (size_t)npts * 2 * 8, st);
  float2* seg = (float2*)A.alloc((size_t)L * npts * sizeof(float2));
  float2* work = (float2*)A.alloc((size_t)L * g.nf0 * g.nf1 * sizeof(float2));
  nufft_type2<float>(g, imgs, L, n, du, npts, seg, npts, work, 1, nullptr, st);
  const double* db = (const double*)A.upload(plan.b.data(), plan.b.size() * 8, st);
  const float2* dstat = (const float2*)A.upload(stat.data(), stat.size() * sizeof(float2), st);
  const int* dti = (const int*)A.upload(tidx.data(), tidx.size() * 4, st);
  float2* dout = (float2*)A.alloc((size_t)npts * sizeof(float2));
  segment_combine(seg, npts, L, dti, db, dstat, dout, st);
  MRSIM_CUDA(cudaGetLastError());
  MRSIM_CUDA(cudaMemcpyAsync(out, dout, (size_t)npts * sizeof(float2), cudaMemcpyDeviceToHost, st));
  MRSIM_CUDA(cudaStreamSynchronize(st));
  return info;
}

}  // namespace mrsim
