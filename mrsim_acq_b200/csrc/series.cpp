// series.cpp — the per-slice pipeline and the series drivers on the device: forward, spikes and
// noise, GRAPPA calibration and apply, window, inverse DFT, Roemer combine, image-space noise and
// the output layout (reference kspace.rs:1229-1378 and 1665-2215).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>

#include "driver.h"
#include "host_tables.h"
#include "mrsim_internal.h"
#include "noise_kernels.h"
#include "recon_kernels.h"
#include "series.h"
#include "series_parts.h"

namespace mrsim {


// Tables of one acquired geometry for the reconstruction.
ReconTables build_recon_tables(DevArena& A, int nx, int ny, int nc, const mrsim_acquisition& acq, cudaStream_t st) {
  ReconTables T;
  const int xs = nx / 2, ys = ny / 2;
  std::vector<float2> ex(nx), ey(ny);
  for (int m = 0; m < nx; ++m) ex[m] = make_float2((float)std::cos(-kTau * m / nx), (float)std::sin(-kTau * m / nx));
  for (int m = 0; m < ny; ++m) ey[m] = make_float2((float)std::cos(-kTau * m / ny), (float)std::sin(-kTau * m / ny));
  T.ex_tab = (float2*)A.upload(ex.data(), ex.size() * sizeof(float2), st);
  T.ey_tab = (float2*)A.upload(ey.data(), ey.size() * sizeof(float2), st);
  // `coil_sensitivity` on the acquired grid and the Roemer denominator (kspace.rs:1343-1373)
  T.sens_host.assign((size_t)nc * nx * ny, 0.f);
  std::vector<double> ssum((size_t)nx * ny, 0.0);
  for (int q = 0; q < nc; ++q)
    for (int i = 0; i < nx * ny; ++i) {
      double s = coil_sensitivity(q, nc, (double)(i % nx), (double)(i / nx), nx, ny);
      T.sens_host[(size_t)q * nx * ny + i] = (float)s;
      ssum[i] += s * s;
    }
  std::vector<float> inv((size_t)nx * ny);
  for (int i = 0; i < nx * ny; ++i) inv[i] = (float)(1.0 / std::max(ssum[i], 1e-12));
  T.sens = (float*)A.upload(T.sens_host.data(), T.sens_host.size() * 4, st);
  T.inv_ssum = (float*)A.upload(inv.data(), inv.size() * 4, st);
  if (acq.window_kind != MRSIM_WINDOW_NONE) {
    std::vector<float> w((size_t)nx * ny);
    for (int ky = 0; ky < ny; ++ky)
      for (int kx = 0; kx < nx; ++kx)
        w[(size_t)ky * nx + kx] =
            (float)window_at(acq, ((double)kx - xs) / (double)nx, ((double)ky - ys) / (double)ny);
    T.window = (float*)A.upload(w.data(), w.size() * 4, st);
  }
  // the lines GRAPPA synthesises (`GrappaKernel::apply`, kspace.rs:1605-1632)
  const int accel = (int)std::max<int64_t>(acq.accel, 1);
  if (accel > 1) {
    auto acquired = sampling_mask(1, ny, acq);
    std::vector<int4> fills;
    for (int d = 1; d < accel; ++d)
      for (int ky = 0; ky < ny; ++ky) {
        int r = ((ky - ys) % accel + accel) % accel;
        if (r != d || ky < d || ky + accel - d >= ny) continue;
        int s0 = ky - d, s1 = ky - d + accel;
        if (!(acquired[s0] && acquired[s1])) continue;
        fills.push_back(make_int4(ky, d, s0, s1));
      }
    T.n_fills = (int)fills.size();
    if (!fills.empty()) T.fills = (int4*)A.upload(fills.data(), fills.size() * sizeof(int4), st);
  }
  return T;
}

// One batch of forward units: descriptors, statics, plan.
void add_unit(Batch& B, const UnitInputs& in, int snx, int sny, int nx, int ny, int ncomp, int ncoils, bool maps,
              const float* t2u, const float* tiu, const GeoTab& geo, const mrsim_acquisition& acq) {
  const bool eddy = acq.eddy_strength != 0.0 && in.has_eddy;
  const bool eddy_phase = acq.eddy_phase != 0.0 && in.has_eddy;
  UnitDesc u;
  std::memset(&u, 0, sizeof u);
  u.snx = snx;
  u.sny = sny;
  u.nx = nx;
  u.ny = ny;
  u.ncomp = ncomp;
  u.ncoils = ncoils;
  u.n_lines = in.n_lines;
  u.n_rows = ny;
  u.flags = (acq.do_relaxation ? UF_RELAX : 0) | (maps ? UF_MAPS : 0) | (eddy ? UF_EDDY : 0) |
            (acq.do_distortions ? UF_DISTORT : 0) | (acq.echo == MRSIM_ECHO_GRADIENT ? UF_GRADIENT : 0);
  u.z = in.z;
  u.nz = in.nz_full;
  u.comp_stride = in.comp_stride;
  u.map_stride = in.map_stride;
  u.comp = in.comp;
  u.fmap = in.fmap;
  u.phase = in.phase_out;
  u.t2map = in.t2map;
  u.timap = in.timap;
  u.log_amp = in.log_amp;
  u.lines = in.lines;
  u.geo = geo;
  u.signal_scale = (float)acq.signal_scale;
  for (int c = 0; c < kMaxComp; ++c) {
    u.t2u[c] = t2u[c];
    u.tiu[c] = tiu[c];
  }
  if (eddy) {
    const double zc = (double)in.z - (double)(in.nz_full / 2);
    u.eddy_cx = (float)(acq.eddy_strength * in.grad[0]);
    u.eddy_qx = (float)(acq.eddy_quad * in.grad[0]);
    u.eddy_cy = (float)(acq.eddy_strength * in.grad[1]);
    u.eddy_qy = (float)(acq.eddy_quad * in.grad[1]);
    u.eddy_z = (float)(acq.eddy_strength * in.grad[2] * zc + acq.eddy_quad * in.grad[2] * zc * zc);
  }
  u.kspace = in.kspace;
  u.g = in.g;
  B.units.push_back(u);

  StaticDesc sd;
  std::memset(&sd, 0, sizeof sd);
  sd.snx = snx;
  sd.sny = sny;
  sd.nx = nx;
  sd.ny = ny;
  sd.o = snx / nx;
  sd.z = in.z;
  sd.nz_full = in.nz_full;
  sd.flags = (in.phase0 ? 1 : 0) | (eddy_phase ? 2 : 0);
  sd.phase0 = in.phase0;
  if (!in.phase0 && in.phase) {
    sd.global = in.phase->global;
    for (int k = 0; k < 10; ++k) sd.bg[k] = in.phase->background[k];
    for (int k = 0; k < 3; ++k) {
      sd.shot_q[k] = in.shot.q[k];
      sd.shot_dx[k] = in.shot.dx[k];
      sd.shot_rot[k] = in.shot.rot[k];
    }
  }
  for (int i = 0; i < 3; ++i) sd.eddy_phase_coef[i] = acq.eddy_phase * (in.has_eddy ? in.grad[i] : 0.0);
  sd.zc_c = (double)in.z - ((double)in.nz_full - 1.0) / 2.0;
  sd.out = in.phase_out;
  B.statics.push_back(sd);
}

void run_forward(const Batch& B, cudaStream_t st) {
  if (B.units.empty()) return;
  std::unique_ptr<EpiPlan> plan(epi_plan_create(B.units.data(), (int)B.units.size(), B.statics.data(),
                                                (int)B.statics.size()));
  epi_plan_statics(plan.get(), st);
  epi_plan_forward(plan.get(), st);
  MRSIM_CUDA(cudaStreamSynchronize(st));  // the plan's device memory is freed on return
}

// Uniform relaxation weights of a line (kspace.rs:886-903), with T2' from Acquisition::t_inhom
// as f64 when no per-compartment T2' is given.
void lines_for(std::vector<LineRec>& out, const mrsim_acquisition& acq, int nx, int ny, bool eddy, bool uniform,
               int ncomp, const float* t2u, const float* tiu, bool has_tinhom, const LineTimingTab* timing) {
  LineTimingTab lt = timing ? *timing : line_timing(acq, nx, ny);
  auto mask = sampling_mask(nx, ny, acq);
  for (int ky = 0; ky < ny; ++ky) {
    if (!mask[(size_t)nx * ky]) continue;
    LineRec L;
    std::memset(&L, 0, sizeof L);
    L.ky = ky;
    L.row = ky;
    L.pol = lt.polarity[ky] < 0 ? -1 : 1;
    const double t = lt.t_ms[ky] / 1000.0, trf = lt.trf_ms[ky];
    const bool spin = acq.echo == MRSIM_ECHO_SPIN;
    const double tb0 = spin ? t : t + acq.t_echo / 1000.0;
    L.t_hi = (float)tb0;
    L.t_lo = (float)(tb0 - (double)L.t_hi);
    L.t_s = (float)tb0;
    const double inh = spin ? std::fabs(t) * 1000.0 : trf;
    L.inhom_ms = (float)inh;
    L.trf_ms = (float)trf;
    L.decay = eddy ? (float)(std::exp(-lt.tread_ms[ky] / acq.eddy_tau) * t) : 0.f;
    for (int c = 0; c < kMaxComp; ++c) {
      double rel = 1.0;
      if (c < ncomp && uniform && acq.do_relaxation)
        rel = std::exp(-trf / (double)t2u[c] - inh / (has_tinhom ? (double)tiu[c] : acq.t_inhom));
      L.rel[c] = (float)rel;
    }
    out.push_back(L);
  }
}

void run_noise(DevArena& A, const std::vector<NoiseSpec>& specs, const std::vector<int>& rows,
               const std::vector<int>& picks, int nx, int ny, const mrsim_acquisition& acq, cudaStream_t st) {
  const bool do_spikes = acq.n_spikes > 0 && !picks.empty();
  const bool do_noise = acq.noise_variance > 0.0;
  if ((!do_spikes && !do_noise) || rows.empty() || specs.empty()) return;
  const int* d_rows = (const int*)A.upload(rows.data(), rows.size() * 4, st);
  const int* d_picks = do_spikes ? (const int*)A.upload(picks.data(), picks.size() * 4, st) : nullptr;
  std::vector<NoiseJob> jobs(specs.size());
  for (size_t j = 0; j < specs.size(); ++j) {
    NoiseJob& J = jobs[j];
    std::memset(&J, 0, sizeof J);
    J.k = specs[j].k;
    J.rows = d_rows;
    J.picks = d_picks ? d_picks + specs[j].pick_offset : nullptr;
    J.n_rows = (int)rows.size();
    J.nx = nx;
    J.n_picks = do_spikes ? (int)acq.n_spikes : 0;
    J.seed = (specs[j].slice_seed ^ ((uint64_t)specs[j].coil * 0x9E3779B9ull)) | 1ull;
    J.sigma = do_noise ? std::sqrt(acq.noise_variance / (double)((size_t)nx * ny)) : 0.0;
    J.spike_amplitude = acq.spike_amplitude;
  }
  const NoiseJob* d_jobs = (const NoiseJob*)A.upload(jobs.data(), jobs.size() * sizeof(NoiseJob), st);
  auto* d_keys = (unsigned long long*)A.alloc(sizeof(unsigned long long) * jobs.size());
  launch_noise_jobs(d_jobs, (int)jobs.size(), do_spikes, do_noise, (int)rows.size() * nx, d_keys, st);
  MRSIM_CUDA(cudaGetLastError());
}

// The spike sample indices of one slice (`build_coil_kspace_timed` kspace.rs:997-1019).
void spike_picks(std::vector<int>& picks, uint64_t slice_seed, const std::vector<uint8_t>& mask,
                 const mrsim_acquisition& acq) {
  if (acq.n_spikes <= 0) return;
  std::vector<int> acquired;
  for (size_t i = 0; i < mask.size(); ++i)
    if (mask[i]) acquired.push_back((int)i);
  Rng rng(slice_seed ^ 0xA5A5123456789ABCull);
  for (int64_t s = 0; s < acq.n_spikes; ++s)
    picks.push_back(acquired.empty() ? 0 : acquired[(size_t)(rng.next_u64() % (uint64_t)acquired.size())]);
}

// GRAPPA calibration of a batch of reference scans (one per slice): weights [slice][d-1][co][f].
float2* fit_grappa(DevArena& A, const std::vector<float2*>& ref_k, int nx, int ny, int nc,
                   const mrsim_acquisition& acq_ref, int accel, int acs_lines, cudaStream_t st) {
  const int nf = 6 * nc;
  const size_t per_slice = (size_t)(accel - 1) * nc * nf;
  float2* W = (float2*)A.alloc(std::max<size_t>(1, ref_k.size() * per_slice) * sizeof(float2));
  if (accel <= 1 || ref_k.empty()) return W;
  auto lines = sampling_mask(1, ny, acq_ref);
  uint8_t* d_lines = (uint8_t*)A.upload(lines.data(), lines.size(), st);
  const int ys = ny / 2;
  const int acs_half = acs_lines / 2;
  const int acs_lo = std::max(ys - acs_half, 0);
  const int acs_hi = std::min(ys + acs_half, ny - 1);
  std::vector<GrappaSystem> sys;
  const size_t work_n = (size_t)nf * (nf + nc), fs_n = (size_t)2 * nf + (size_t)nc * 2 * nf;
  double2* work = (double2*)A.alloc(ref_k.size() * (accel - 1) * work_n * sizeof(double2));
  double* fscr = (double*)A.alloc(ref_k.size() * (accel - 1) * fs_n * sizeof(double));
  for (size_t s = 0; s < ref_k.size(); ++s)
    for (int d = 1; d < accel; ++d) {
      GrappaSystem g;
      std::memset(&g, 0, sizeof g);
      g.k = ref_k[s];
      g.lines = d_lines;
      g.nx = nx;
      g.ny = ny;
      g.nc = nc;
      g.accel = accel;
      g.d = d;
      g.acs_lo = acs_lo;
      g.acs_hi = acs_hi;
      const size_t idx = s * (accel - 1) + (d - 1);
      g.work = work + idx * work_n;
      g.fscratch = fscr + idx * fs_n;
      g.weights = W + s * per_slice + (size_t)(d - 1) * nc * nf;
      sys.push_back(g);
    }
  const GrappaSystem* d_sys = (const GrappaSystem*)A.upload(sys.data(), sys.size() * sizeof(GrappaSystem), st);
  launch_grappa_fit(d_sys, (int)sys.size(), nc, kGrappaLambda, st);
  MRSIM_CUDA(cudaGetLastError());
  return W;
}

bool uniform_relaxation(const mrsim_t2* t2, const mrsim_t2* ti, int ncomp) {
  bool u = true;
  for (int c = 0; c < ncomp; ++c) u = u && !t2[c].is_map;
  if (ti)
    for (int c = 0; c < ncomp; ++c) u = u && !ti[c].is_map;
  return u;
}


// =============================================================================================
// Per slice (`simulate_slice_with`, kspace.rs:1271-1284)
struct SliceState {
  DevArena A;
  int snx, sny, nx, ny, ncomp, nc;
  float2* k = nullptr;  // [coil][ny][nx]
};

// Forward of one slice with spikes and noise, into `S.k` (device).
static void slice_forward_into(mrsim_context* ctx, SliceState& S, const mrsim_slice_input& inp,
                               const mrsim_acquisition& acq, const LineTimingTab* timing, const double* log_amp) {
  cudaStream_t st = ctx->stream;
  DevArena& A = S.A;
  const int snx = S.snx, sny = S.sny, nx = S.nx, ny = S.ny, ncomp = S.ncomp, nc = S.nc;
  const size_t plane = (size_t)snx * sny;
  const bool uniform = uniform_relaxation(inp.t2, inp.t_inhom, ncomp) && log_amp == nullptr;
  const bool maps = !uniform && acq.do_relaxation;
  float t2u[kMaxComp], tiu[kMaxComp];
  for (int c = 0; c < kMaxComp; ++c) {
    t2u[c] = c < ncomp ? inp.t2[c].value : 1.f;
    tiu[c] = c < ncomp ? (inp.t_inhom ? inp.t_inhom[c].value : (float)acq.t_inhom) : 1.f;
  }
  const bool eddy = acq.eddy_strength != 0.0 && inp.has_eddy_drive;
  std::vector<LineRec> lines;
  lines_for(lines, acq, nx, ny, eddy, uniform, ncomp, t2u, tiu, inp.t_inhom != nullptr, timing);
  std::vector<float> comp(std::max<size_t>(1, (size_t)ncomp * plane));
  for (int c = 0; c < ncomp; ++c) std::memcpy(&comp[(size_t)c * plane], inp.compartments[c], plane * 4);
  UnitInputs ui;
  std::memset(&ui, 0, sizeof ui);
  ui.comp = (const float*)A.upload(comp.data(), comp.size() * 4, st);
  ui.comp_stride = (long long)plane;
  ui.fmap = (const float*)A.upload(inp.fmap, plane * 4, st);
  ui.map_stride = (long long)plane;
  if (maps) {
    auto build = [&](const mrsim_t2* v) -> const float* {
      bool any = false;
      for (int c = 0; c < ncomp; ++c) any = any || v[c].is_map;
      if (!any) return nullptr;
      std::vector<float> m((size_t)ncomp * plane);
      for (int c = 0; c < ncomp; ++c)
        for (size_t i = 0; i < plane; ++i) m[(size_t)c * plane + i] = v[c].is_map ? v[c].map[i] : v[c].value;
      return (const float*)A.upload(m.data(), m.size() * 4, st);
    };
    ui.t2map = build(inp.t2);
    ui.timap = inp.t_inhom ? build(inp.t_inhom) : nullptr;
    if (log_amp) {
      std::vector<float> m(plane);
      for (size_t i = 0; i < plane; ++i) m[i] = (float)log_amp[i];
      ui.log_amp = (const float*)A.upload(m.data(), plane * 4, st);
    }
  }
  ui.lines = (const LineRec*)A.upload(lines.data(), std::max<size_t>(1, lines.size()) * sizeof(LineRec), st);
  ui.n_lines = (int)lines.size();
  S.k = (float2*)A.alloc((size_t)nc * nx * ny * sizeof(float2));
  MRSIM_CUDA(cudaMemsetAsync(S.k, 0, (size_t)nc * nx * ny * sizeof(float2), st));
  ui.kspace = S.k;
  ui.g = (float2*)A.alloc(std::max<size_t>(1, (size_t)nc * lines.size() * snx) * sizeof(float2));
  ui.phase_out = (float*)A.alloc(plane * 4);
  ui.phase0 = inp.phase0 ? (const double*)A.upload(inp.phase0, plane * 8, st) : nullptr;
  mrsim_phase_model zero;
  std::memset(&zero, 0, sizeof zero);
  ui.phase = &zero;
  ui.z = (int)inp.z;
  ui.nz_full = (int)inp.nz;
  ui.has_eddy = inp.has_eddy_drive != 0;
  for (int i = 0; i < 3; ++i) ui.grad[i] = inp.eddy_drive[i];
  GeoTab geo = build_geo(A, snx, sny, nx, ny, nc, acq.ghost_offset, st);
  Batch B;
  add_unit(B, ui, snx, sny, nx, ny, ncomp, nc, maps, t2u, tiu, geo, acq);
  if (!lines.empty()) run_forward(B, st);
  else {
    std::unique_ptr<EpiPlan> plan(epi_plan_create(B.units.data(), 1, B.statics.data(), 1));
    epi_plan_statics(plan.get(), st);
    MRSIM_CUDA(cudaStreamSynchronize(st));
  }
  std::vector<int> rows;
  for (auto& L : lines) rows.push_back(L.ky);
  std::vector<int> picks;
  spike_picks(picks, inp.slice_seed, sampling_mask(nx, ny, acq), acq);
  std::vector<NoiseSpec> specs;
  for (int q = 0; q < nc; ++q) specs.push_back({S.k + (size_t)q * nx * ny, inp.slice_seed, q, 0});
  run_noise(A, specs, rows, picks, nx, ny, acq, st);
}

std::vector<float2> slice_forward2(mrsim_context* ctx, const mrsim_slice_input& inp, const mrsim_acquisition& acq,
                                   const LineTimingTab* timing, const double* log_amp) {
  SliceState S;
  S.snx = (int)inp.sim[0];
  S.sny = (int)inp.sim[1];
  S.nx = (int)inp.acq_matrix[0];
  S.ny = (int)inp.acq_matrix[1];
  S.ncomp = (int)inp.ncomp;
  S.nc = (int)std::max<int64_t>(acq.n_coils, 1);
  slice_forward_into(ctx, S, inp, acq, timing, log_amp);
  std::vector<float2> out((size_t)S.nc * S.nx * S.ny);
  MRSIM_CUDA(cudaMemcpyAsync(out.data(), S.k, out.size() * sizeof(float2), cudaMemcpyDeviceToHost, ctx->stream));
  MRSIM_CUDA(cudaStreamSynchronize(ctx->stream));
  return out;
}

static void check_slice(const mrsim_slice_input& inp, const mrsim_acquisition& acq) {
  if (inp.sim[0] <= 0 || inp.sim[1] <= 0 || inp.acq_matrix[0] <= 0 || inp.acq_matrix[1] <= 0)
    fail("empty simulation grid or acquired matrix");
  if (!(inp.sim[0] % inp.acq_matrix[0] == 0 && inp.sim[1] % inp.acq_matrix[1] == 0))
    fail("sim grid must be an integer multiple of the acquired matrix");
  if (inp.ncomp > kMaxComp) fail("more than 8 compartments");
  if (std::max<int64_t>(acq.n_coils, 1) > kMaxCoils) fail("more than 64 coils");
  if (acq.accel > 1 && inp.acq_matrix[0] > 1024) fail("acquired matrix too wide for the reconstruction");
}

void simulate_slice_full(mrsim_context* ctx, const mrsim_slice_input& inp, const mrsim_acquisition& acq,
                         SliceOutputs& out) {
  check_slice(inp, acq);
  cudaStream_t st = ctx->stream;
  const int nx = (int)inp.acq_matrix[0], ny = (int)inp.acq_matrix[1];
  const int nc = (int)std::max<int64_t>(acq.n_coils, 1);
  const int accel = (int)std::max<int64_t>(acq.accel, 1);
  const size_t per = (size_t)nx * ny;
  SliceState S;
  S.snx = (int)inp.sim[0];
  S.sny = (int)inp.sim[1];
  S.nx = nx;
  S.ny = ny;
  S.ncomp = (int)inp.ncomp;
  S.nc = nc;
  DevArena& A = S.A;
  // GRAPPA: a lone slice fits its own kernel on a reference scan of itself, its noise on the slice
  // seed salted by SEED_SALT_GRAPPA_CAL, without eddy and preparation drives (kspace.rs:1253-1284)
  float2* W = nullptr;
  if (accel > 1) {
    SliceState R;
    R.snx = S.snx;
    R.sny = S.sny;
    R.nx = nx;
    R.ny = ny;
    R.ncomp = S.ncomp;
    R.nc = nc;
    mrsim_slice_input ref = inp;
    ref.has_eddy_drive = 0;
    ref.has_prep_drive = 0;
    ref.slice_seed = inp.slice_seed ^ kSeedSaltGrappaCal;
    mrsim_acquisition acq_ref = acq;
    acq_ref.accel = 1;
    acq_ref.n_spikes = 0;
    slice_forward_into(ctx, R, ref, acq_ref, nullptr, nullptr);
    W = fit_grappa(A, {R.k}, nx, ny, nc, acq_ref, accel, (int)acq.acs_lines, st);
    MRSIM_CUDA(cudaStreamSynchronize(st));  // R's buffers are freed at the end of this scope
  }
  slice_forward_into(ctx, S, inp, acq, nullptr, nullptr);
  if (out.acquired)
    MRSIM_CUDA(cudaMemcpyAsync(out.acquired, S.k, (size_t)nc * per * sizeof(float2), cudaMemcpyDeviceToHost, st));
  ReconTables T = build_recon_tables(A, nx, ny, nc, acq, st);
  ReconJob J;
  std::memset(&J, 0, sizeof J);
  J.k = S.k;
  J.grappa_w = W;
  J.window = T.window;
  J.ex_tab = T.ex_tab;
  J.ey_tab = T.ey_tab;
  J.sens = T.sens;
  J.inv_ssum = T.inv_ssum;
  J.combined = (float2*)A.alloc(per * sizeof(float2));
  if (out.coil_images) J.coil_images = (float2*)A.alloc((size_t)nc * per * sizeof(float2));
  if (out.reconstructed) J.reconstructed = (float2*)A.alloc((size_t)nc * per * sizeof(float2));
  J.nx = nx;
  J.ny = ny;
  J.nc = nc;
  const ReconJob* d_job = (const ReconJob*)A.upload(&J, sizeof J, st);
  if (accel > 1) launch_grappa_apply(d_job, 1, T.fills, T.n_fills, nx, nc, st);
  launch_recon_combine(d_job, 1, nx, ny, out.reconstructed != nullptr, st);
  MRSIM_CUDA(cudaGetLastError());
  MRSIM_CUDA(cudaMemcpyAsync(out.combined, J.combined, per * sizeof(float2), cudaMemcpyDeviceToHost, st));
  if (out.coil_images)
    MRSIM_CUDA(cudaMemcpyAsync(out.coil_images, J.coil_images, (size_t)nc * per * sizeof(float2),
                               cudaMemcpyDeviceToHost, st));
  if (out.reconstructed)
    MRSIM_CUDA(cudaMemcpyAsync(out.reconstructed, J.reconstructed, (size_t)nc * per * sizeof(float2),
                               cudaMemcpyDeviceToHost, st));
  if (out.sensitivities) std::memcpy(out.sensitivities, T.sens_host.data(), T.sens_host.size() * 4);
  if (out.mask) {
    auto m = sampling_mask(nx, ny, acq);
    std::memcpy(out.mask, m.data(), m.size());
  }
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

// =============================================================================================
// The series (`acquire_volumes_complex`, kspace.rs:1851-2125).
namespace {

void validate_t2_volumes(const char* what, const mrsim_t2* vols, int ncomp, size_t nvox) {
  for (int c = 0; c < ncomp; ++c) {
    if (!vols[c].is_map) continue;
    if (!vols[c].map) fail(std::string(what) + " map for compartment " + std::to_string(c) + " is NULL");
    for (size_t i = 0; i < nvox; ++i) {
      float v = vols[c].map[i];
      if (std::isnan(v) || v <= 0.0f) {
        char buf[256];
        std::snprintf(buf, sizeof buf, "%s map for compartment %d: T2 map value %g at index %zu is not strictly positive",
                      what, c, (double)v, i);
        fail(buf);
      }
    }
  }
}

}  // namespace

void acquire_series(mrsim_context* ctx, const mrsim_acquisition_input& in, const mrsim_acquisition& acq,
                    const mrsim_acquisition_options* opts_in, uint64_t excitation_seed, uint64_t receiver_seed,
                    const float* const* images, mrsim_acquisition_output& out, bool mag_phase,
                    SeriesImageCache* cache) {
  mrsim_acquisition_options dflt;
  std::memset(&dflt, 0, sizeof dflt);
  const mrsim_acquisition_options& opts = opts_in ? *opts_in : dflt;
  cudaStream_t st = ctx->stream;
  const int snx = (int)in.sim_dims[0], sny = (int)in.sim_dims[1], nz = (int)in.sim_dims[2];
  const int nx = (int)in.acq_dims[0], ny = (int)in.acq_dims[1], nzo = (int)in.acq_dims[2];
  const int nv = (int)in.n_volumes, ncomp = (int)in.ncomp;
  if (nz != nzo) fail("slice count must match; z is never oversampled");
  if (snx <= 0 || sny <= 0 || nx <= 0 || ny <= 0) fail("empty simulation grid or acquired matrix");
  if (!(snx % nx == 0 && sny % ny == 0)) fail("sim grid must be an integer multiple of the acquired matrix");
  const int o = snx / nx;
  if (o != sny / ny) fail("oversampling must match on both axes");
  if (ncomp > kMaxComp) fail("more than 8 compartments");
  const int nc = (int)std::max<int64_t>(acq.n_coils, 1);
  if (nc > kMaxCoils) fail("more than 64 coils");
  if (nx > 1024) fail("acquired matrix too wide for the reconstruction");
  const size_t plane = (size_t)snx * sny, nvox_sim = plane * nz, per = (size_t)nx * ny;
  const size_t nvox_acq = per * nz;
  if (!in.fmap) fail("fieldmap is not on the simulation grid");
  if (ncomp > 0 && !images) fail("compartment image is not on the simulation grid");
  validate_t2_volumes("T2", in.t2, ncomp, nvox_sim);
  if (in.t_inhom) validate_t2_volumes("T2'", in.t_inhom, ncomp, nvox_sim);
  if (!opts.t_echo_per_volume) {
    validate_acquisition_timing(acq, nx, ny);
  } else {
    for (int g = 0; g < nv; ++g) {
      mrsim_acquisition a = acq;
      a.t_echo = opts.t_echo_per_volume[g];
      try {
        validate_acquisition_timing(a, nx, ny);
      } catch (const Error& e) {
        fail("volume " + std::to_string(g) + ": " + e.what());
      }
    }
  }
  const int nz_full = opts.nz_full > 0 ? (int)opts.nz_full : nz;
  if (opts.slice_z)
    for (int zl = 0; zl < nz; ++zl)
      if (opts.slice_z[zl] < 0 || opts.slice_z[zl] >= nz_full)
        fail("slice_z entries must be below nz_full " + std::to_string(nz_full));
  auto global_z = [&](int zl) { return opts.slice_z ? (int)opts.slice_z[zl] : zl; };
  std::vector<int> captured;
  for (int64_t i = 0; i < opts.n_kspace_slices; ++i) {
    if (opts.kspace_slices[i] < 0 || opts.kspace_slices[i] >= nz)
      fail("kspace_slices index " + std::to_string(opts.kspace_slices[i]) + " out of range for " + std::to_string(nz) +
           " slices");
    captured.push_back((int)opts.kspace_slices[i]);
  }
  DevArena A;
  // ---- inputs on the device (kept in `cache` for a later call with the same arrays)
  const size_t per_comp = nvox_sim * nv;
  const std::vector<const float*> img_from(images, images + (images ? ncomp : 0));
  float* d_img = nullptr;
  if (cache && cache->d_img && cache->from == img_from && cache->n == per_comp * ncomp) {
    d_img = cache->d_img;
  } else {
    float* staging = (float*)A.alloc(std::max<size_t>(1, per_comp * ncomp) * 4);
    for (int c = 0; c < ncomp; ++c) copy_pageable_h2d(ctx, staging + (size_t)c * per_comp, images[c], per_comp * 4, st);
    if (cache) {
      if (cache->d_img && cache->n < per_comp * ncomp) {
        MRSIM_CUDA(cudaStreamSynchronize(st));
        MRSIM_CUDA(cudaFree(cache->d_img));
        cache->d_img = nullptr;
      }
      if (!cache->d_img) {
        MRSIM_CUDA(cudaMalloc(&cache->d_img, std::max<size_t>(1, per_comp * ncomp) * 4));
        cache->n = per_comp * ncomp;
      }
      cache->from = img_from;
      cache->n = per_comp * ncomp;
      d_img = cache->d_img;
    } else {
      d_img = (float*)A.alloc(std::max<size_t>(1, per_comp * ncomp) * 4);
    }
    if (ncomp) launch_series_transpose(staging, d_img, ncomp, nv, nz, (int)plane, st);
  }
  float* d_fmap = (float*)A.upload(in.fmap, nvox_sim * 4, st);
  const bool uniform = uniform_relaxation(in.t2, in.t_inhom, ncomp);
  const bool maps = !uniform && acq.do_relaxation;
  float* d_t2 = nullptr;
  float* d_ti = nullptr;
  if (maps) {
    auto build = [&](const mrsim_t2* v) -> float* {
      bool any = false;
      for (int c = 0; c < ncomp; ++c) any = any || v[c].is_map;
      if (!any) return nullptr;
      std::vector<float> m((size_t)ncomp * nvox_sim);
      for (int c = 0; c < ncomp; ++c)
        for (size_t i = 0; i < nvox_sim; ++i) m[(size_t)c * nvox_sim + i] = v[c].is_map ? v[c].map[i] : v[c].value;
      return (float*)A.upload(m.data(), m.size() * 4, st);
    };
    d_t2 = build(in.t2);
    if (in.t_inhom) d_ti = build(in.t_inhom);
  }
  float t2u[kMaxComp], tiu[kMaxComp];
  for (int c = 0; c < kMaxComp; ++c) {
    t2u[c] = c < ncomp ? in.t2[c].value : 1.f;
    tiu[c] = c < ncomp ? (in.t_inhom ? in.t_inhom[c].value : (float)acq.t_inhom) : 1.f;
  }
  GeoTab geo = build_geo(A, snx, sny, nx, ny, nc, acq.ghost_offset, st);
  ReconTables T = build_recon_tables(A, nx, ny, nc, acq, st);
  const int accel = (int)std::max<int64_t>(acq.accel, 1);

  // echo times: one line table per distinct TE
  std::vector<double> tes;
  if (opts.t_echo_per_volume)
    tes.assign(opts.t_echo_per_volume, opts.t_echo_per_volume + nv);
  else
    tes.push_back(acq.t_echo);
  std::sort(tes.begin(), tes.end());
  tes.erase(std::unique(tes.begin(), tes.end(), [](double a, double b) { return std::memcmp(&a, &b, 8) == 0; }),
            tes.end());
  auto te_index = [&](double te) {
    for (size_t i = 0; i < tes.size(); ++i)
      if (std::memcmp(&tes[i], &te, 8) == 0) return (int)i;
    return 0;
  };
  const bool any_eddy = acq.eddy_strength != 0.0 && in.eddy_drive_set &&
                        std::any_of(in.eddy_drive_set, in.eddy_drive_set + nv, [](int32_t v) { return v != 0; });
  std::vector<LineRec*> d_lines(tes.size());
  std::vector<int> n_lines(tes.size());
  std::vector<int> rows;
  for (size_t t = 0; t < tes.size(); ++t) {
    mrsim_acquisition a = acq;
    a.t_echo = tes[t];
    std::vector<LineRec> L;
    lines_for(L, a, nx, ny, any_eddy, uniform, ncomp, t2u, tiu, in.t_inhom != nullptr, nullptr);
    n_lines[t] = (int)L.size();
    d_lines[t] = (LineRec*)A.upload(L.data(), std::max<size_t>(1, L.size()) * sizeof(LineRec), st);
    if (t == 0)
      for (auto& r : L) rows.push_back(r.ky);
  }
  const int max_lines = *std::max_element(n_lines.begin(), n_lines.end());

  // ---- GRAPPA calibration: one reference scan per slice per distinct echo time
  std::vector<float2*> weights(tes.size(), nullptr);
  if (accel > 1 && nv > 0) {
    float* cal_img = d_img;  // volume 0 of the series (units g = 0 are its first nz units)
    uint64_t cal_seed = receiver_seed;
    if (opts.has_grappa_calibration) {
      float* cstage = (float*)A.alloc(std::max<size_t>(1, nvox_sim * ncomp) * 4);
      for (int c = 0; c < ncomp; ++c)
        MRSIM_CUDA(cudaMemcpyAsync(cstage + (size_t)c * nvox_sim, opts.grappa_calibration_images[c], nvox_sim * 4,
                                   cudaMemcpyHostToDevice, st));
      cal_img = (float*)A.alloc(std::max<size_t>(1, nvox_sim * ncomp) * 4);
      if (ncomp) launch_series_transpose(cstage, cal_img, ncomp, 1, nz, (int)plane, st);
      cal_seed = opts.grappa_calibration_seed;
    }
    for (size_t t = 0; t < tes.size(); ++t) {
      mrsim_acquisition acq_cal = acq;
      acq_cal.t_echo = tes[t];
      acq_cal.accel = 1;
      acq_cal.n_spikes = 0;
      std::vector<LineRec> L;
      lines_for(L, acq_cal, nx, ny, false, uniform, ncomp, t2u, tiu, in.t_inhom != nullptr, nullptr);
      const LineRec* dl = (const LineRec*)A.upload(L.data(), std::max<size_t>(1, L.size()) * sizeof(LineRec), st);
      DevArena C;
      float2* ck = (float2*)C.alloc((size_t)nz * nc * per * sizeof(float2));
      MRSIM_CUDA(cudaMemsetAsync(ck, 0, (size_t)nz * nc * per * sizeof(float2), st));
      float2* cg = (float2*)C.alloc(std::max<size_t>(1, (size_t)nz * nc * L.size() * snx) * sizeof(float2));
      float* cph = (float*)C.alloc(nz * plane * 4);
      Batch B;
      std::vector<NoiseSpec> specs;
      for (int zl = 0; zl < nz; ++zl) {
        UnitInputs ui;
        std::memset(&ui, 0, sizeof ui);
        ui.comp = cal_img + (size_t)zl * ncomp * plane;
        ui.comp_stride = (long long)plane;
        ui.fmap = d_fmap + (size_t)zl * plane;
        ui.t2map = d_t2 ? d_t2 + (size_t)zl * plane : nullptr;
        ui.timap = d_ti ? d_ti + (size_t)zl * plane : nullptr;
        ui.map_stride = (long long)nvox_sim;
        ui.lines = dl;
        ui.n_lines = (int)L.size();
        ui.kspace = ck + (size_t)zl * nc * per;
        ui.g = cg + (size_t)zl * nc * L.size() * snx;
        ui.phase_out = cph + (size_t)zl * plane;
        ui.phase = in.phase;
        ui.z = global_z(zl);
        ui.nz_full = nz_full;
        add_unit(B, ui, snx, sny, nx, ny, ncomp, nc, maps, t2u, tiu, geo, acq_cal);
        const uint64_t seed = ((uint64_t)ui.z * 0x9E37ull) ^ cal_seed ^ kSeedSaltGrappaCal;
        for (int q = 0; q < nc; ++q) specs.push_back({ck + ((size_t)zl * nc + q) * per, seed, q, 0});
      }
      if (!L.empty()) run_forward(B, st);
      std::vector<int> crow;
      for (auto& r : L) crow.push_back(r.ky);
      run_noise(C, specs, crow, {}, nx, ny, acq_cal, st);
      std::vector<float2*> refs;
      for (int zl = 0; zl < nz; ++zl) refs.push_back(ck + (size_t)zl * nc * per);
      weights[t] = fit_grappa(A, refs, nx, ny, nc, acq_cal, accel, (int)acq.acs_lines, st);
      MRSIM_CUDA(cudaStreamSynchronize(st));
    }
  }

  // ---- the series: forward, spikes and noise, in chunks of volumes
  const size_t nf = 6 * (size_t)nc;
  const size_t w_per_slice = (size_t)(accel - 1) * nc * nf;
  const int nsl = (int)captured.size();
  float2* cap_acq = nullptr;
  float2* cap_rec = nullptr;
  float2* cap_img = nullptr;
  float2* cap_comb = nullptr;
  if (nsl) {
    const size_t n = (size_t)nv * nsl * nc * per;
    if (opts.capture_acquired && out.acquired) cap_acq = (float2*)A.alloc(n * sizeof(float2));
    if (opts.capture_reconstructed && out.reconstructed) cap_rec = (float2*)A.alloc(n * sizeof(float2));
    if (opts.capture_coil_images && out.coil_images) cap_img = (float2*)A.alloc(n * sizeof(float2));
    cap_comb = (float2*)A.alloc((size_t)nv * nsl * per * sizeof(float2));
  }
  float* d_re = (float*)A.alloc(std::max<size_t>(1, nvox_acq * nv) * 4);
  float* d_im = (float*)A.alloc(std::max<size_t>(1, nvox_acq * nv) * 4);
  const float* d_sigma = in.noise_sigma ? (const float*)A.upload(in.noise_sigma, nvox_acq * 4, st) : nullptr;
  // chunk the volumes so the scratch stays within a budget
  const size_t bytes_per_unit = (size_t)nc * max_lines * snx * 8 + (size_t)nc * per * 8 * 2 + plane * 4 + per * 8;
  const size_t budget = (size_t)4 << 30;
  int vchunk = (int)std::max<size_t>(1, std::min<size_t>(nv, budget / std::max<size_t>(1, bytes_per_unit * nz)));
  auto mask = sampling_mask(nx, ny, acq);
  std::vector<int> zmap(nz);
  for (int zl = 0; zl < nz; ++zl) zmap[zl] = global_z(zl);
  const int* d_zmap = (const int*)A.upload(zmap.data(), zmap.size() * 4, st);
  for (int g0 = 0; g0 < nv; g0 += vchunk) {
    const int g1 = std::min(nv, g0 + vchunk);
    const int nunit = (g1 - g0) * nz;
    DevArena C;
    float2* ks = (float2*)C.alloc((size_t)nunit * nc * per * sizeof(float2));
    MRSIM_CUDA(cudaMemsetAsync(ks, 0, (size_t)nunit * nc * per * sizeof(float2), st));
    float2* gs = (float2*)C.alloc(std::max<size_t>(1, (size_t)nunit * nc * max_lines * snx) * sizeof(float2));
    float* ph = (float*)C.alloc((size_t)nunit * plane * 4);
    float2* comb = (float2*)C.alloc((size_t)nunit * per * sizeof(float2));
    Batch B;
    std::vector<NoiseSpec> specs;
    std::vector<int> picks;
    std::vector<ReconJob> jobs;
    for (int g = g0; g < g1; ++g) {
      mrsim_acquisition acq_g = acq;
      if (opts.t_echo_per_volume) acq_g.t_echo = opts.t_echo_per_volume[g];
      const int ti = te_index(acq_g.t_echo);
      const bool has_eddy = in.eddy_drive_set && in.eddy_drive_set[g];
      const bool has_prep = in.prep_drive_set && in.prep_drive_set[g];
      for (int zl = 0; zl < nz; ++zl) {
        const int z = global_z(zl);
        const int u = (g - g0) * nz + zl;
        UnitInputs ui;
        std::memset(&ui, 0, sizeof ui);
        ui.comp = d_img + ((size_t)g * nz + zl) * ncomp * plane;
        ui.comp_stride = (long long)plane;
        ui.fmap = d_fmap + (size_t)zl * plane;
        ui.t2map = d_t2 ? d_t2 + (size_t)zl * plane : nullptr;
        ui.timap = d_ti ? d_ti + (size_t)zl * plane : nullptr;
        ui.map_stride = (long long)nvox_sim;
        ui.lines = d_lines[ti];
        ui.n_lines = n_lines[ti];
        ui.kspace = ks + (size_t)u * nc * per;
        ui.g = gs + (size_t)u * nc * max_lines * snx;
        ui.phase_out = ph + (size_t)u * plane;
        ui.phase = in.phase;
        if (in.phase && in.phase->has_prep && has_prep)
          ui.shot = prep_shot(*in.phase, in.prep_drive[4 * g], &in.prep_drive[4 * g + 1], g, z, excitation_seed);
        ui.z = z;
        ui.nz_full = nz_full;
        ui.has_eddy = has_eddy;
        for (int i = 0; i < 3; ++i) ui.grad[i] = has_eddy ? in.eddy_drive[3 * g + i] : 0.0;
        add_unit(B, ui, snx, sny, nx, ny, ncomp, nc, maps, t2u, tiu, geo, acq_g);
        const uint64_t slice_seed = (((uint64_t)g * 0x1000001ull) + (uint64_t)z) * 0x9E37ull ^ receiver_seed;
        const int off = (int)picks.size();
        spike_picks(picks, slice_seed, mask, acq);
        for (int q = 0; q < nc; ++q) specs.push_back({ks + ((size_t)u * nc + q) * per, slice_seed, q, off});
        ReconJob J;
        std::memset(&J, 0, sizeof J);
        J.k = ks + (size_t)u * nc * per;
        J.grappa_w = accel > 1 ? weights[ti] + (size_t)zl * w_per_slice : nullptr;
        J.window = T.window;
        J.ex_tab = T.ex_tab;
        J.ey_tab = T.ey_tab;
        J.sens = T.sens;
        J.inv_ssum = T.inv_ssum;
        J.combined = comb + (size_t)u * per;
        for (int s = 0; s < nsl; ++s)
          if (captured[s] == zl) {
            const size_t base = ((size_t)g * nsl + s) * nc * per;
            if (cap_img) J.coil_images = cap_img + base;
            if (cap_rec) J.reconstructed = cap_rec + base;
          }
        J.nx = nx;
        J.ny = ny;
        J.nc = nc;
        jobs.push_back(J);
      }
    }
    run_forward(B, st);
    run_noise(C, specs, rows, picks, nx, ny, acq, st);
    for (int g = g0; g < g1; ++g)
      for (int s = 0; s < nsl; ++s) {
        const int u = (g - g0) * nz + captured[s];
        if (cap_acq)
          MRSIM_CUDA(cudaMemcpyAsync(cap_acq + ((size_t)g * nsl + s) * nc * per, ks + (size_t)u * nc * per,
                                     (size_t)nc * per * sizeof(float2), cudaMemcpyDeviceToDevice, st));
      }
    const ReconJob* d_jobs = (const ReconJob*)C.upload(jobs.data(), jobs.size() * sizeof(ReconJob), st);
    if (accel > 1) launch_grappa_apply(d_jobs, (int)jobs.size(), T.fills, T.n_fills, nx, nc, st);
    launch_recon_combine(d_jobs, (int)jobs.size(), nx, ny, cap_rec != nullptr, st);
    MRSIM_CUDA(cudaGetLastError());
    for (int g = g0; g < g1; ++g)
      for (int s = 0; s < nsl; ++s)
        MRSIM_CUDA(cudaMemcpyAsync(cap_comb + ((size_t)g * nsl + s) * per, comb + ((size_t)(g - g0) * nz + captured[s]) * per,
                                   per * sizeof(float2), cudaMemcpyDeviceToDevice, st));
    launch_series_output(comb, d_sigma, d_re, d_im, g0, g1, nv, nz, nx, ny, d_zmap, receiver_seed, st, mag_phase);
    MRSIM_CUDA(cudaStreamSynchronize(st));
  }
  copy_pageable_d2h(ctx, out.re, d_re, nvox_acq * nv * 4, st);
  copy_pageable_d2h(ctx, out.im, d_im, nvox_acq * nv * 4, st);
  if (nsl) {
    const size_t n = (size_t)nv * nsl * nc * per;
    if (cap_acq) MRSIM_CUDA(cudaMemcpyAsync(out.acquired, cap_acq, n * sizeof(float2), cudaMemcpyDeviceToHost, st));
    if (cap_rec)
      MRSIM_CUDA(cudaMemcpyAsync(out.reconstructed, cap_rec, n * sizeof(float2), cudaMemcpyDeviceToHost, st));
    if (cap_img)
      MRSIM_CUDA(cudaMemcpyAsync(out.coil_images, cap_img, n * sizeof(float2), cudaMemcpyDeviceToHost, st));
    if (out.combined)
      MRSIM_CUDA(cudaMemcpyAsync(out.combined, cap_comb, (size_t)nv * nsl * per * sizeof(float2),
                                 cudaMemcpyDeviceToHost, st));
    if (out.mask) std::memcpy(out.mask, mask.data(), mask.size());
    if (out.sensitivities) std::memcpy(out.sensitivities, T.sens_host.data(), T.sens_host.size() * 4);
  }
  MRSIM_CUDA(cudaStreamSynchronize(st));
  if (opts.progress)
    for (int g = 0; g < nv; ++g) opts.progress(g + 1, nv, opts.progress_user);
}

}  // namespace mrsim
