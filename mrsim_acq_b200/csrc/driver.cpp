// driver.cpp — host orchestration of the B200 k-space library: context, geometry and line
// tables, the batched forward/adjoint operator of a 2D EPI series, and the per-slice forward.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <thread>
#include <tuple>
#if defined(__SSE2__)
#include <emmintrin.h>
#endif

#include "driver.h"
#include "host_tables.h"
#include "mrsim_internal.h"
#include "noise_kernels.h"
#include "ts_epi.h"

namespace mrsim {

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(MRSIM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

void* workspace(mrsim_context* ctx, int slot, size_t bytes) {
  if ((int)ctx->ws.size() <= slot) ctx->ws.resize(slot + 1);
  DeviceBuffer& b = ctx->ws[slot];
  if (b.n < bytes) {
    if (b.p) MRSIM_CUDA(cudaFree(b.p));
    b.p = nullptr;
    b.n = 0;
    MRSIM_CUDA(cudaMalloc(&b.p, bytes));
    b.n = bytes;
  }
  return b.p;
}

// ---- device memory owned by an object --------------------------------------------------------
void* DevArena::alloc(size_t bytes) {
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  MRSIM_CUDA(cudaMalloc(&p, bytes));
  ptrs.push_back(p);
  return p;
}
void* DevArena::upload(const void* src, size_t bytes, cudaStream_t st) {
  void* p = alloc(bytes);
  if (bytes) MRSIM_CUDA(cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, st));
  return p;
}
DevArena::~DevArena() {
  for (void* p : ptrs) cudaFree(p);
}

// ---- geometry tables -----------------------------------------------------------------------
// ex/ey: the two factors of the Gaussian ring coil sensitivity (`coil_sensitivity`
// kspace.rs:226-237) on the sim grid in acquired-voxel units (xa = (x - xoff)/o); tw: the x-stage
// twiddles e^{i2pi (kx - xs + gh)(x - sxs - xoff)/snx} for gh = +ghost, -ghost (`XStage::new`,
// kspace.rs:1069-1110), with the k.r part from the exact integer index (kx-xs)(2(x-sxs)-(o-1))
// mod 2 snx, stored [pol][x][kx] then transposed [pol][kx][x].
GeoTab build_geo(DevArena& arena, int snx, int sny, int nx, int ny, int ncoils, double ghost, cudaStream_t st) {
  const int ox = snx / nx, oy = sny / ny;
  const double xoff = (ox - 1.0) / 2.0, yoff = (oy - 1.0) / 2.0;
  const int xs = nx / 2, sxs = ox * xs;
  std::vector<float> ex((size_t)ncoils * snx), ey((size_t)ncoils * sny);
  const double sigma = 0.9 * (double)std::max(nx, ny);
  const double r = 0.6 * (double)std::max(nx, ny);
  for (int q = 0; q < ncoils; ++q) {
    if (ncoils <= 1) {
      for (int x = 0; x < snx; ++x) ex[x] = 1.f;
      for (int y = 0; y < sny; ++y) ey[y] = 1.f;
      continue;
    }
    const double ang = kTau * (double)q / (double)ncoils;
    const double px = nx / 2.0 + r * std::cos(ang), py = ny / 2.0 + r * std::sin(ang);
    for (int x = 0; x < snx; ++x) {
      double d = ((double)x - xoff) / ox - px;
      ex[(size_t)q * snx + x] = (float)std::exp(-(d * d) / (2.0 * sigma * sigma));
    }
    for (int y = 0; y < sny; ++y) {
      double d = ((double)y - yoff) / oy - py;
      ey[(size_t)q * sny + y] = (float)std::exp(-(d * d) / (2.0 * sigma * sigma));
    }
  }
  std::vector<float2> tw((size_t)4 * snx * nx);
  const double c = (double)sxs + xoff;
  const long long m2 = 2LL * snx;
  for (int pol = 0; pol < 2; ++pol) {
    const double gh = pol == 0 ? ghost : -ghost;
    for (int x = 0; x < snx; ++x) {
      const long long X = 2LL * (x - sxs) - (ox - 1);
      const double gramp = gh * ((double)x - c) / (double)snx;
      for (int kx = 0; kx < nx; ++kx) {
        long long K = kx - xs;
        double turns = (double)((K * X) % m2) / (double)m2 + gramp;
        turns -= std::rint(turns);
        double ph = kTau * turns;
        float2 v = make_float2((float)std::cos(ph), (float)std::sin(ph));
        tw[(size_t)pol * snx * nx + (size_t)x * nx + kx] = v;
        tw[(size_t)(2 + pol) * snx * nx + (size_t)kx * snx + x] = v;
      }
    }
  }
  GeoTab g;
  g.xf = nullptr;
  if ((snx >= 8 && snx <= kXfftMaxN && (snx & (snx - 1)) == 0) || (snx % 32 == 0 && snx <= 256)) {
    // the factored x-stage: tw[x][kx] = premod_pol(x) * e^{i2pi (kx-xs) x/snx} * post(kx)
    std::vector<float2> xf((size_t)snx / 2 + 2 * (size_t)snx + nx);
    for (int k = 0; k < snx / 2; ++k) {
      const double ph = -kTau * (double)k / (double)snx;
      xf[k] = make_float2((float)std::cos(ph), (float)std::sin(ph));
    }
    for (int pol = 0; pol < 2; ++pol) {
      const double gh = pol == 0 ? ghost : -ghost;
      for (int x = 0; x < snx; ++x) {
        double turns = gh * ((double)x - c) / (double)snx;
        turns -= std::rint(turns);
        xf[(size_t)snx / 2 + (size_t)pol * snx + x] =
            make_float2((float)std::cos(kTau * turns), (float)std::sin(kTau * turns));
      }
    }
    const long long c2 = 2LL * sxs + (ox - 1);  // 2c, an integer
    for (int kx = 0; kx < nx; ++kx) {
      const long long K = kx - xs;
      double turns = -(double)((K * c2) % m2) / (double)m2;
      turns -= std::rint(turns);
      xf[(size_t)snx / 2 + 2 * (size_t)snx + kx] = make_float2((float)std::cos(kTau * turns), (float)std::sin(kTau * turns));
    }
    g.xf = (const float2*)arena.upload(xf.data(), xf.size() * sizeof(float2), st);
  }
  {
    // coil classes of bitwise-equal ey rows
    std::vector<int> cls(ncoils, -1);
    std::vector<float> eyc;
    int ncls = 0;
    for (int q = 0; q < ncoils; ++q) {
      for (int q2 = 0; q2 < q && cls[q] < 0; ++q2)
        if (std::memcmp(&ey[(size_t)q * sny], &ey[(size_t)q2 * sny], sizeof(float) * sny) == 0) cls[q] = cls[q2];
      if (cls[q] < 0) {
        cls[q] = ncls++;
        eyc.insert(eyc.end(), ey.begin() + (size_t)q * sny, ey.begin() + (size_t)(q + 1) * sny);
      }
    }
    g.ncls = ncls;
    g.cls = (const int*)arena.upload(cls.data(), cls.size() * sizeof(int), st);
    g.eyc = (const float*)arena.upload(eyc.data(), eyc.size() * 4, st);
  }
  g.ex = (const float*)arena.upload(ex.data(), ex.size() * 4, st);
  g.ey = (const float*)arena.upload(ey.data(), ey.size() * 4, st);
  g.tw = (const float2*)arena.upload(tw.data(), tw.size() * sizeof(float2), st);
  g.coil_off = ncoils <= 1 ? 0.f : 0.15f;
  return g;
}

// ---- line records --------------------------------------------------------------------------
// One echo's acquired lines, in ky order (the reference loops kyi = 0..ny and skips rows the
// sampling mask drops, kspace.rs:843-846), with the per-line factors of kspace.rs:847-903.
void append_lines(std::vector<LineRec>& out, const mrsim_acquisition& acq, const LineTimingTab& lt, int nx, int ny,
                  int echo, bool eddy, bool uniform, int ncomp, const float* t2u, const float* tiu) {
  auto mask = sampling_mask(nx, ny, acq);
  for (int ky = 0; ky < ny; ++ky) {
    if (!mask[(size_t)nx * ky]) continue;
    LineRec L;
    std::memset(&L, 0, sizeof L);
    L.ky = ky;
    L.row = echo * ny + ky;
    L.pol = lt.polarity[ky] < 0 ? -1 : 1;
    const double t = lt.t_ms[ky] / 1000.0;
    const double trf = lt.trf_ms[ky];
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
      if (c < ncomp && uniform && acq.do_relaxation) rel = std::exp(-trf / (double)t2u[c] - inh / (double)tiu[c]);
      L.rel[c] = (float)rel;
    }
    out.push_back(L);
  }
}

// Zero `n` bytes at `p` with streaming (non-temporal) stores where the ISA has them: the write
// does not first read the lines into the cache, so it takes half the memory traffic of a plain
// memset and leaves the bandwidth to the concurrent device-to-host copies.  Streaming stores are
// weakly ordered: a thread calls stream_fence() once after its last zero_stream, before it ends
// (a fence per call would drain the write-combining buffers on every 512-byte row).
static void zero_stream(char* p, size_t n) {
#if defined(__SSE2__)
  while (n > 0 && ((uintptr_t)p & 15)) {
    *p++ = 0;
    --n;
  }
  const __m128i z = _mm_setzero_si128();
  for (; n >= 64; n -= 64, p += 64) {
    _mm_stream_si128((__m128i*)p, z);
    _mm_stream_si128((__m128i*)(p + 16), z);
    _mm_stream_si128((__m128i*)(p + 32), z);
    _mm_stream_si128((__m128i*)(p + 48), z);
  }
  for (; n >= 16; n -= 16, p += 16) _mm_stream_si128((__m128i*)p, z);
#endif
  std::memset(p, 0, n);
}
static void stream_fence() {
#if defined(__SSE2__)
  _mm_sfence();
#endif
}

// =============================================================================================
// The batched forward/adjoint operator of a 2D EPI series.
EpiOperator::~EpiOperator() {
  ts_plan_destroy(ts);
  for (cudaEvent_t e : events) cudaEventDestroy(e);
  if (copy_stream) cudaStreamDestroy(copy_stream);
  if (upload_stream) cudaStreamDestroy(upload_stream);
}

static void validate_series(const mrsim_acquisition_input& in, const mrsim_acquisition& acq) {
  const int64_t snx = in.sim_dims[0], sny = in.sim_dims[1], nz = in.sim_dims[2];
  const int64_t nx = in.acq_dims[0], ny = in.acq_dims[1], nzo = in.acq_dims[2];
  if (nz != nzo) fail("slice count must match; z is never oversampled");
  if (nx <= 0 || ny <= 0 || snx <= 0 || sny <= 0) fail("empty simulation grid or acquired matrix");
  if (!(snx % nx == 0 && sny % ny == 0)) fail("sim grid must be an integer multiple of the acquired matrix");
  if (snx / nx != sny / ny) fail("oversampling must match on both axes");
  if (in.ncomp > kMaxComp) fail("more than 8 compartments");
  if (std::max<int64_t>(acq.n_coils, 1) > kMaxCoils) fail("more than 64 coils");
  (void)acq;
}

EpiOperator* epi_operator_create(mrsim_context* ctx, const mrsim_acquisition_input& in, const mrsim_acquisition& acq,
                                 const double* echo_times_ms, int64_t n_echoes, const int64_t* slice_z,
                                 int64_t nz_full_in, int grads) {
  validate_series(in, acq);
  std::unique_ptr<EpiOperator> op(new EpiOperator());
  op->ctx = ctx;
  cudaStream_t st = ctx->stream;
  const int snx = (int)in.sim_dims[0], sny = (int)in.sim_dims[1], nz = (int)in.sim_dims[2];
  const int nx = (int)in.acq_dims[0], ny = (int)in.acq_dims[1];
  const int nv = (int)in.n_volumes, ncomp = (int)in.ncomp;
  const int ncoils = (int)std::max<int64_t>(acq.n_coils, 1);
  const int nz_full = nz_full_in > 0 ? (int)nz_full_in : nz;
  std::vector<double> tes;
  if (echo_times_ms && n_echoes > 0)
    tes.assign(echo_times_ms, echo_times_ms + n_echoes);
  else
    tes.push_back(acq.t_echo);
  const int ne = (int)tes.size();
  op->snx = snx;
  op->sny = sny;
  op->nx = nx;
  op->ny = ny;
  op->nz = nz;
  op->nv = nv;
  op->ncomp = ncomp;
  op->ncoils = ncoils;
  op->n_echoes = ne;
  const size_t plane = (size_t)snx * sny;

  bool uniform = true;
  for (int c = 0; c < ncomp; ++c) uniform = uniform && !in.t2[c].is_map;
  if (in.t_inhom)
    for (int c = 0; c < ncomp; ++c) uniform = uniform && !in.t_inhom[c].is_map;
  const bool maps = !uniform && acq.do_relaxation;
  float t2u[kMaxComp], tiu[kMaxComp];
  for (int c = 0; c < kMaxComp; ++c) {
    t2u[c] = c < ncomp ? in.t2[c].value : 1.f;
    tiu[c] = c < ncomp ? (in.t_inhom ? in.t_inhom[c].value : (float)acq.t_inhom) : 1.f;
  }
  // eddy is per volume; lines are built with decay for the eddy case (decay is only read when a
  // unit has UF_EDDY, so one line table serves every volume)
  const bool any_eddy = acq.eddy_strength != 0.0 && in.eddy_drive_set &&
                        std::any_of(in.eddy_drive_set, in.eddy_drive_set + nv, [](int32_t v) { return v != 0; });
  std::vector<LineRec> lines;
  for (int e = 0; e < ne; ++e) {
    mrsim_acquisition a = acq;
    a.t_echo = tes[e];
    validate_acquisition_timing(a, nx, ny);
    LineTimingTab lt = line_timing(a, nx, ny);
    size_t before = lines.size();
    append_lines(lines, a, lt, nx, ny, e, any_eddy, uniform, ncomp, t2u, tiu);
    if (uniform && acq.do_relaxation && !in.t_inhom)
      for (size_t k = before; k < lines.size(); ++k) {
        LineRec& L = lines[k];
        double t = lt.t_ms[L.ky] / 1000.0, trf = lt.trf_ms[L.ky];
        double inh = a.echo == MRSIM_ECHO_SPIN ? std::fabs(t) * 1000.0 : trf;
        for (int c = 0; c < ncomp; ++c) L.rel[c] = (float)std::exp(-trf / (double)t2u[c] - inh / a.t_inhom);
      }
  }
  op->n_lines = (int)lines.size();
  op->acq = acq;
  op->tes = tes;
  op->h_lines = lines;
  op->h_fmap.assign(in.fmap, in.fmap + (size_t)nz * snx * sny);
  for (int c = 0; c < kMaxComp; ++c) {
    op->t2u[c] = t2u[c];
    op->tiu[c] = tiu[c];
  }
  op->maps = maps;
  op->any_eddy = any_eddy;
  {
    // the acquired rows: the same arithmetic progression of ky in every echo?
    std::vector<std::vector<int>> ky(ne);
    for (const LineRec& L : lines) ky[L.row / ny].push_back(L.ky);
    bool ok = !ky.empty() && !ky[0].empty();
    for (int e = 1; e < ne && ok; ++e) ok = ky[e] == ky[0];
    int step = 1;
    if (ok && ky[0].size() > 1) step = ky[0][1] - ky[0][0];
    for (size_t i = 1; ok && i < ky[0].size(); ++i) ok = ky[0][i] - ky[0][i - 1] == step;
    if (ok && step >= 1 && ny % step == 0) {
      op->krow0 = ky[0][0];
      op->krow_step = step;
      op->krow_n = (int)ky[0].size();
    }
  }
  op->samples_per_step = (int64_t)nv * nz * ncoils * (int64_t)lines.size() * nx;

  DevArena& A = op->arena;
  op->d_images = (float*)A.alloc((size_t)nv * nz * ncomp * plane * 4);
  op->d_fmap = (float*)A.upload(in.fmap, (size_t)nz * plane * 4, st);
  if (maps) {
    bool any_t2 = false, any_ti = false;
    for (int c = 0; c < ncomp; ++c) {
      any_t2 = any_t2 || in.t2[c].is_map;
      any_ti = any_ti || (in.t_inhom && in.t_inhom[c].is_map);
    }
    auto build = [&](const mrsim_t2* v) {
      std::vector<float> m((size_t)ncomp * nz * plane);
      for (int c = 0; c < ncomp; ++c)
        for (size_t i = 0; i < (size_t)nz * plane; ++i) m[(size_t)c * nz * plane + i] = v[c].is_map ? v[c].map[i] : v[c].value;
      return (float*)A.upload(m.data(), m.size() * 4, st);
    };
    if (any_t2) op->d_t2 = build(in.t2);
    if (any_ti) op->d_ti = build(in.t_inhom);
  }
  op->geo = build_geo(A, snx, sny, nx, ny, ncoils, acq.ghost_offset, st);
  op->d_lines = (LineRec*)A.upload(lines.data(), std::max<size_t>(1, lines.size()) * sizeof(LineRec), st);
  const size_t nunits = (size_t)nv * nz;
  op->d_phase = (float*)A.alloc(nunits * plane * 4);
  op->d_g = (float2*)A.alloc(std::max<size_t>(1, nunits * ncoils * lines.size() * snx) * sizeof(float2));
  op->kspace_elems = nunits * ncoils * ne * (size_t)ny * nx;
  op->d_kspace = (float2*)A.alloc(op->kspace_elems * sizeof(float2));
  MRSIM_CUDA(cudaMemsetAsync(op->d_kspace, 0, op->kspace_elems * sizeof(float2), st));
  op->d_comp_grad = (float2*)A.alloc(nunits * ncomp * plane * sizeof(float2));
  op->want_fmap = (grads & 1) != 0;
  op->want_r2 = (grads & 2) != 0;
  op->d_fmap_grad = op->want_fmap ? (float*)A.alloc(nunits * plane * 4) : nullptr;
  op->d_r2_grad = op->want_r2 ? (float*)A.alloc(nunits * ncomp * plane * 4) : nullptr;

  std::vector<UnitDesc> units(nunits);
  std::vector<StaticDesc> statics(nunits);
  for (int g = 0; g < nv; ++g) {
    const bool has_eddy = in.eddy_drive_set && in.eddy_drive_set[g];
    const bool eddy = acq.eddy_strength != 0.0 && has_eddy;
    const bool eddy_phase = acq.eddy_phase != 0.0 && has_eddy;
    double grad[3] = {0, 0, 0};
    if (has_eddy)
      for (int i = 0; i < 3; ++i) grad[i] = in.eddy_drive[3 * g + i];
    for (int zl = 0; zl < nz; ++zl) {
      const int z = slice_z ? (int)slice_z[zl] : zl;
      // memory is volume-major (ui); the plan orders units slice-major (pi) so that a range of
      // slices is a range of plan units
      const size_t ui = (size_t)g * nz + zl, pi = (size_t)zl * nv + g;
      UnitDesc& u = units[pi];
      std::memset(&u, 0, sizeof u);
      u.snx = snx;
      u.sny = sny;
      u.nx = nx;
      u.ny = ny;
      u.ncomp = ncomp;
      u.ncoils = ncoils;
      u.n_lines = (int)lines.size();
      u.n_rows = ne * ny;
      u.flags = (acq.do_relaxation ? UF_RELAX : 0) | (maps ? UF_MAPS : 0) | (eddy ? UF_EDDY : 0) |
                (acq.do_distortions ? UF_DISTORT : 0) | (acq.echo == MRSIM_ECHO_GRADIENT ? UF_GRADIENT : 0) |
                (op->want_fmap ? UF_WANT_FMAP_GRAD : 0) | (op->want_r2 ? UF_WANT_R2_GRAD : 0);
      u.z = z;
      u.nz = nz_full;
      u.comp_stride = (long long)plane;
      u.map_stride = (long long)nz * plane;
      u.comp = op->d_images + ui * ncomp * plane;
      u.fmap = op->d_fmap + (size_t)zl * plane;
      u.phase = op->d_phase + ui * plane;
      u.t2map = op->d_t2 ? op->d_t2 + (size_t)zl * plane : nullptr;
      u.timap = op->d_ti ? op->d_ti + (size_t)zl * plane : nullptr;
      u.lines = op->d_lines;
      u.geo = op->geo;
      u.signal_scale = (float)acq.signal_scale;
      for (int c = 0; c < kMaxComp; ++c) {
        u.t2u[c] = t2u[c];
        u.tiu[c] = tiu[c];
      }
      if (eddy) {
        const double zc = (double)z - (double)(nz_full / 2);
        u.eddy_cx = (float)(acq.eddy_strength * grad[0]);
        u.eddy_qx = (float)(acq.eddy_quad * grad[0]);
        u.eddy_cy = (float)(acq.eddy_strength * grad[1]);
        u.eddy_qy = (float)(acq.eddy_quad * grad[1]);
        u.eddy_z = (float)(acq.eddy_strength * grad[2] * zc + acq.eddy_quad * grad[2] * zc * zc);
      }
      u.kspace = op->d_kspace + ui * (size_t)ncoils * ne * ny * nx;
      u.g = op->d_g + ui * (size_t)ncoils * lines.size() * snx;
      u.comp_grad = op->d_comp_grad + ui * ncomp * plane;
      u.fmap_grad = op->d_fmap_grad ? op->d_fmap_grad + ui * plane : nullptr;
      u.r2_grad = op->d_r2_grad ? op->d_r2_grad + ui * ncomp * plane : nullptr;

      StaticDesc& sd = statics[pi];
      std::memset(&sd, 0, sizeof sd);
      sd.snx = snx;
      sd.sny = sny;
      sd.nx = nx;
      sd.ny = ny;
      sd.o = snx / nx;
      sd.z = z;
      sd.nz_full = nz_full;
      sd.flags = eddy_phase ? 2 : 0;
      if (in.phase) {
        sd.global = in.phase->global;
        for (int k = 0; k < 10; ++k) sd.bg[k] = in.phase->background[k];
        const bool has_prep = in.prep_drive_set && in.prep_drive_set[g];
        if (in.phase->has_prep && has_prep) {
          ShotParams sp = prep_shot(*in.phase, in.prep_drive[4 * g], &in.prep_drive[4 * g + 1], g, z, in.seed);
          for (int k = 0; k < 3; ++k) {
            sd.shot_q[k] = sp.q[k];
            sd.shot_dx[k] = sp.dx[k];
            sd.shot_rot[k] = sp.rot[k];
          }
        }
      }
      for (int i = 0; i < 3; ++i) sd.eddy_phase_coef[i] = acq.eddy_phase * grad[i];
      sd.zc_c = (double)z - ((double)nz_full - 1.0) / 2.0;
      sd.out = op->d_phase + ui * plane;
    }
  }
  op->plan.reset(epi_plan_create(units.data(), (int)units.size(), statics.data(), (int)statics.size()));
  if (in.images) upload_series_images(op.get(), in.images);
  MRSIM_CUDA(cudaStreamSynchronize(st));
  return op.release();
}

// Reference layout (per compartment, vox*nv + g with vox = x + snx*(y + sny*z)) to the
// operator's unit-major layout [g][z][c][y][x], on the device.
void upload_series_images(EpiOperator* op, const float* const* host_images) {
  cudaStream_t st = op->ctx->stream;
  const size_t plane = (size_t)op->snx * op->sny;
  const size_t per_comp = (size_t)op->nz * plane * op->nv;
  float* staging = (float*)workspace(op->ctx, 20, per_comp * op->ncomp * 4);
  for (int c = 0; c < op->ncomp; ++c)
    copy_pageable_h2d(op->ctx, staging + (size_t)c * per_comp, host_images[c], per_comp * 4, st);
  launch_series_transpose(staging, op->d_images, op->ncomp, op->nv, op->nz, (int)plane, st);
}

// A new fieldmap (Hz, [z][sny][snx], the creation layout) for the forwards and adjoints queued
// after it: the kernels read the device copy directly, and nothing at creation derives from it.
// With the time-segmented path selected, a fieldmap outside the range its segmentation certified
// rebuilds the segmentation and its tables.
void epi_operator_set_fieldmap(EpiOperator* op, const float* fmap) {
  cudaStream_t st = op->ctx->stream;
  const size_t n = (size_t)op->nz * op->snx * op->sny;
  MRSIM_CUDA(cudaMemcpyAsync(op->d_fmap, fmap, n * 4, cudaMemcpyHostToDevice, st));
  op->h_fmap.assign(fmap, fmap + n);
  MRSIM_CUDA(cudaStreamSynchronize(st));
  if (op->ts && op->acq.do_distortions) {
    const auto mm = std::minmax_element(op->h_fmap.begin(), op->h_fmap.end());
    if (*mm.first < op->ts->fmin || *mm.second > op->ts->fmax) epi_operator_set_segmented(op, op->ts_precision);
  }
}

// Selects the y-stages: 0 the exact per-line phasors, 1 / 2 the time-segmented tensor-core
// contractions in split f16 / split bf16 (built here: segmentation, tables, tensor maps).
void epi_operator_set_segmented(EpiOperator* op, int precision) {
  TsPlan* fresh = precision ? ts_plan_build(*op, precision) : nullptr;
  ts_plan_destroy(op->ts);
  op->ts = fresh;
  op->ts_precision = precision;
}

void epi_operator_forward_units(EpiOperator* op, cudaStream_t st, int u0, int u1) {
  if (op->ts) {
    ts_forward_ystage(*op->ts, *op->plan, st, u0, u1);
    epi_plan_forward_xstage(op->plan.get(), st, u0, u1);
  } else {
    epi_plan_forward(op->plan.get(), st, u0, u1);
  }
}

void epi_operator_adjoint_units(EpiOperator* op, cudaStream_t st, int u0, int u1) {
  if (op->ts) {
    epi_plan_adjoint_xstage(op->plan.get(), st, u0, u1);
    ts_adjoint_ystage(*op->ts, *op->plan, st, u0, u1);
  } else {
    epi_plan_adjoint(op->plan.get(), st, u0, u1);
  }
}

EpiBatch* epi_batch_create(mrsim_context* ctx, int n, const mrsim_acquisition_input* const* inputs,
                           const mrsim_acquisition& acq, const double* echo_times_ms, int64_t n_echoes, int grads) {
  if (n <= 0) fail("a batch needs at least one series");
  std::unique_ptr<EpiBatch> b(new EpiBatch());
  b->ctx = ctx;
  std::vector<UnitDesc> units;
  std::vector<StaticDesc> statics;
  for (int i = 0; i < n; ++i) {
    if (!inputs[i]) fail("series " + std::to_string(i) + " is NULL");
    b->ops.emplace_back(epi_operator_create(ctx, *inputs[i], acq, echo_times_ms, n_echoes, nullptr, 0, grads));
    const EpiPlan& p = *b->ops.back()->plan;
    b->unit0.push_back((int)units.size());
    units.insert(units.end(), p.host_units.begin(), p.host_units.end());
    std::vector<StaticDesc> sd(p.n_statics);
    MRSIM_CUDA(cudaMemcpy(sd.data(), p.d_statics, sizeof(StaticDesc) * sd.size(), cudaMemcpyDeviceToHost));
    statics.insert(statics.end(), sd.begin(), sd.end());
    b->samples += b->ops.back()->samples_per_step;
  }
  b->plan.reset(epi_plan_create(units.data(), (int)units.size(), statics.data(), (int)statics.size()));
  MRSIM_CUDA(cudaStreamSynchronize(ctx->stream));
  return b.release();
}

void epi_batch_forward(EpiBatch* b) {
  epi_plan_statics(b->plan.get(), b->ctx->stream);
  epi_plan_forward(b->plan.get(), b->ctx->stream);
}

void epi_batch_adjoint(EpiBatch* b) { epi_plan_adjoint(b->plan.get(), b->ctx->stream); }

// ---- the autotuner ------------------------------------------------------------------------------
namespace {
std::string tune_key(const EpiOperator& o) {
  char buf[256];
  std::snprintf(buf, sizeof buf, "epi snx%d sny%d nx%d ny%d coils%d comp%d lines%d echoes%d maps%d grads%d%d", o.snx,
                o.sny, o.nx, o.ny, o.ncoils, o.ncomp, o.n_lines, o.n_echoes, o.maps ? 1 : 0, o.want_fmap ? 1 : 0,
                o.want_r2 ? 1 : 0);
  return buf;
}
struct TuneChoice {
  EpiPlanOptions opt;
  int segmented = 0;  // 0 exact, 1 split f16, 2 split bf16
};
std::string describe(const TuneChoice& c) {
  char buf[160];
  std::snprintf(buf, sizeof buf, "classes=%d x=%s adjoint_rows=%d path=%s", c.opt.no_classes ? 0 : 1,
                c.opt.dft_x ? "dft-gemm" : "fft", c.opt.adj_rows, c.segmented == 0 ? "exact" : c.segmented == 1 ? "segmented-f16" : "segmented-bf16");
  return buf;
}
bool parse_choice(const std::string& v, TuneChoice& c) {
  int cls = 1, rows = 0;
  char x[32] = {0}, path[32] = {0};
  if (std::sscanf(v.c_str(), "classes=%d x=%31s adjoint_rows=%d path=%31s", &cls, x, &rows, path) != 4) return false;
  c.opt.no_classes = cls ? 0 : 1;
  c.opt.dft_x = std::string(x) == "dft-gemm" ? 1 : 0;
  c.opt.adj_rows = rows;
  const std::string ps(path);
  c.segmented = ps == "segmented-f16" ? 1 : ps == "segmented-bf16" ? 2 : 0;
  return true;
}
void apply_choice(EpiOperator* op, const TuneChoice& c) {
  op->plan.reset(epi_plan_create(op->plan->host_units.data(), op->plan->n_units, op->plan->host_statics.data(),
                                 (int)op->plan->host_statics.size(), &c.opt));
  epi_operator_set_segmented(op, c.segmented);
}
}  // namespace

std::string epi_operator_tune(EpiOperator* op, const char* cache_path, int flags, double* ms_out) {
  const std::string key = tune_key(*op);
  // the cache: one "key<TAB>choice" line per shape
  std::vector<std::pair<std::string, std::string>> lines;
  if (cache_path) {
    if (FILE* f = std::fopen(cache_path, "r")) {
      char buf[1024];
      while (std::fgets(buf, sizeof buf, f)) {
        std::string l(buf);
        while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
        const size_t t = l.find('\t');
        if (t != std::string::npos) lines.emplace_back(l.substr(0, t), l.substr(t + 1));
      }
      std::fclose(f);
    }
    for (auto& kv : lines) {
      TuneChoice c;
      if (kv.first == key && parse_choice(kv.second, c)) {
        apply_choice(op, c);
        if (ms_out) *ms_out = 0.0;
        return describe(c) + " (cached)";
      }
    }
  }
  cudaStream_t st = op->ctx->stream;
  const bool had_cls = op->plan->fwd_cls || op->plan->adj_cls;
  const bool had_fft = op->plan->xfft;
  bool has_four = false;
  for (int pass = 0; pass < 4; ++pass) has_four = has_four || (op->plan->adjq[pass] && op->plan->adj_ty[pass] == 4);
  std::vector<TuneChoice> cands;
  for (int nc = 0; nc <= (had_cls ? 1 : 0); ++nc)
    for (int dx = 0; dx <= (had_fft ? 1 : 0); ++dx)
      for (int rows : {0, 2}) {
        if (rows == 2 && !has_four) continue;
        TuneChoice c;
        c.opt.no_classes = nc;
        c.opt.dft_x = dx;
        c.opt.adj_rows = rows;
        cands.push_back(c);
        if (flags & 1)
          for (int sg : {1, 2}) {
            TuneChoice t = c;
            t.segmented = sg;
            cands.push_back(t);
          }
      }
  const int u1 = std::min(op->plan->n_units, 2 * 148);
  cudaEvent_t e0, e1;
  MRSIM_CUDA(cudaEventCreate(&e0));
  MRSIM_CUDA(cudaEventCreate(&e1));
  double best_ms = 1e300;
  TuneChoice best;
  for (const TuneChoice& c : cands) {
    try {
      apply_choice(op, c);
    } catch (const Error&) {
      continue;  // not valid for this shape (e.g. the segmented path's preconditions)
    }
    auto pass = [&] {
      epi_plan_statics(op->plan.get(), st, 0, u1);
      epi_operator_forward_units(op, st, 0, u1);
      epi_operator_adjoint_units(op, st, 0, u1);
    };
    pass();
    MRSIM_CUDA(cudaEventRecord(e0, st));
    for (int r = 0; r < 3; ++r) pass();
    MRSIM_CUDA(cudaEventRecord(e1, st));
    MRSIM_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    MRSIM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms / 3.0 < best_ms) {
      best_ms = ms / 3.0;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  apply_choice(op, best);
  if (ms_out) *ms_out = best_ms;
  if (cache_path) {
    bool replaced = false;
    for (auto& kv : lines)
      if (kv.first == key) {
        kv.second = describe(best);
        replaced = true;
      }
    if (!replaced) lines.emplace_back(key, describe(best));
    if (FILE* f = std::fopen(cache_path, "w")) {
      for (auto& kv : lines) std::fprintf(f, "%s\t%s\n", kv.first.c_str(), kv.second.c_str());
      std::fclose(f);
    }
  }
  return describe(best);
}

void epi_operator_forward(EpiOperator* op) {
  cudaStream_t st = op->ctx->stream;
  epi_plan_statics(op->plan.get(), st);
  epi_operator_forward_units(op, st, 0, -1);
}

void epi_operator_adjoint(EpiOperator* op) { epi_operator_adjoint_units(op, op->ctx->stream, 0, -1); }

int epi_operator_segmented_error(EpiOperator* op) { return op->ts ? ts_error(*op->ts, op->ctx->stream) : 0; }

void epi_operator_apply_host(EpiOperator* o, const float* const* images, float* kspace, float* comp_grad,
                             float* fmap_grad, float* r2_grad, bool compact) {
  if (compact && kspace && o->krow_n <= 0)
    fail("the compact k-space layout needs the acquired rows at a uniform stride in every echo");
  cudaStream_t st = o->ctx->stream;
  const int nv = o->nv, nz = o->nz;
  // Groups are boxes of volumes [g0, g1) x slices [z0, z1), each a range of the slice-major plan
  // units: about eight groups of whole slices, or with one slice, about eight groups of volumes.
  struct Box {
    int g0, g1, z0, z1;
  };
  std::vector<Box> boxes;
  if (nz >= 2) {
    const int per = std::max(1, (nz + 7) / 8);
    for (int z0 = 0; z0 < nz; z0 += per) boxes.push_back({0, nv, z0, std::min(nz, z0 + per)});
  } else {
    const int per = std::max(1, (nv + 7) / 8);
    for (int g0 = 0; g0 < nv; g0 += per) boxes.push_back({g0, std::min(nv, g0 + per), 0, nz});
  }
  const int ng = (int)boxes.size();
  for (cudaStream_t* s : {&o->copy_stream, &o->upload_stream})
    if (!*s) MRSIM_CUDA(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
  while ((int)o->events.size() < 3 * ng + 1) {
    cudaEvent_t e;
    MRSIM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    o->events.push_back(e);
  }
  cudaEvent_t* ev = o->events.data();
  cudaStream_t cs = o->copy_stream, us = o->upload_stream;
  const size_t plane = (size_t)o->snx * o->sny;
  const size_t per_comp = (size_t)nz * plane * nv;  // host floats per compartment
  float* staging = images ? (float*)workspace(o->ctx, 20, per_comp * o->ncomp * 4) : nullptr;
  // uploads: by slice groups on their own stream (the reference layout keeps a slice range of
  // every volume contiguous), else all at once
  if (images) {
    MRSIM_CUDA(cudaEventRecord(ev[3 * ng], st));  // earlier work on the compute stream is done first
    MRSIM_CUDA(cudaStreamWaitEvent(us, ev[3 * ng], 0));
    for (int b = 0; b < ng; ++b) {
      const Box& B = boxes[b];
      if (nz >= 2 || b == 0) {
        const size_t f0 = nz >= 2 ? (size_t)B.z0 * plane * nv : 0;
        const size_t nf = nz >= 2 ? (size_t)(B.z1 - B.z0) * plane * nv : per_comp;
        for (int c = 0; c < o->ncomp; ++c)
          MRSIM_CUDA(cudaMemcpyAsync(staging + (size_t)c * per_comp + f0, images[c] + f0, nf * 4,
                                     cudaMemcpyHostToDevice, us));
      }
      MRSIM_CUDA(cudaEventRecord(ev[3 * b], us));
    }
  }
  const EpiPlan* p = o->plan.get();
  epi_plan_statics(p, st);
  for (int b = 0; b < ng; ++b) {
    const Box& B = boxes[b];
    if (images) {
      MRSIM_CUDA(cudaStreamWaitEvent(st, ev[3 * b], 0));
      if (nz >= 2 || b == 0)
        launch_series_transpose(staging, o->d_images, o->ncomp, nv, nz, (int)plane, st, nz >= 2 ? B.z0 : 0,
                                nz >= 2 ? B.z1 : nz);
    }
    const int u0 = B.z0 * nv + B.g0, u1 = (B.z1 - 1) * nv + B.g1;  // slice-major plan units
    epi_operator_forward_units(o, st, u0, u1);
    MRSIM_CUDA(cudaEventRecord(ev[3 * b + 1], st));
    epi_operator_adjoint_units(o, st, u0, u1);
    MRSIM_CUDA(cudaEventRecord(ev[3 * b + 2], st));
  }
  // downloads: the box is nv' rows (volumes) of (z1 - z0) units, pitch nz units
  const size_t kunit = o->kspace_elems / ((size_t)nv * nz);
  auto down = [&](const Box& B, void* host, const void* dev, size_t unit_bytes) {
    const size_t off = ((size_t)B.g0 * nz + B.z0) * unit_bytes, pitch = (size_t)nz * unit_bytes;
    MRSIM_CUDA(cudaMemcpy2DAsync((char*)host + off, pitch, (const char*)dev + off, pitch, (B.z1 - B.z0) * unit_bytes,
                                 B.g1 - B.g0, cudaMemcpyDeviceToHost, cs));
  };
  // k-space: with a strided row pattern only the acquired rows cross PCIe (one pitched 3D copy per
  // volume of a box: rows k0 + s i of every [unit][coil][echo] block of ny rows), and host threads
  // zero the other rows of the output meanwhile
  const int nx = o->nx, ny = o->ny;
  const bool sparse_k = kspace && o->krow_n > 0;
  const size_t row_bytes = (size_t)nx * sizeof(float2), blocks_per_unit = (size_t)o->ncoils * o->n_echoes;
  auto down_k = [&](const Box& B) {
    for (int g = B.g0; g < B.g1; ++g) {
      const size_t off = ((size_t)g * nz + B.z0) * kunit * sizeof(float2) + (size_t)o->krow0 * row_bytes;
      cudaMemcpy3DParms m;
      std::memset(&m, 0, sizeof m);
      m.srcPtr = make_cudaPitchedPtr((char*)o->d_kspace + off, o->krow_step * row_bytes, row_bytes, ny / o->krow_step);
      if (compact) {  // [g][z][coil][echo][acquired row][kx], no rows in between
        const size_t coff = ((size_t)g * nz + B.z0) * blocks_per_unit * o->krow_n * row_bytes;
        m.dstPtr = make_cudaPitchedPtr((char*)kspace + coff, row_bytes, row_bytes, o->krow_n);
      } else {
        m.dstPtr = make_cudaPitchedPtr((char*)kspace + off, o->krow_step * row_bytes, row_bytes, ny / o->krow_step);
      }
      m.extent = make_cudaExtent(row_bytes, o->krow_n, (size_t)(B.z1 - B.z0) * blocks_per_unit);
      m.kind = cudaMemcpyDeviceToHost;
      MRSIM_CUDA(cudaMemcpy3DAsync(&m, cs));
    }
  };
  struct Joiner {
    std::vector<std::thread> t;
    ~Joiner() {
      for (auto& th : t) th.join();
    }
  } zeroers;
  if (sparse_k && !compact) {
    const size_t nblocks = (size_t)nv * nz * blocks_per_unit;
    std::vector<char> acquired(ny, 0);
    for (int i = 0; i < o->krow_n; ++i) acquired[o->krow0 + i * o->krow_step] = 1;
    const int nt = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    for (int t = 0; t < nt; ++t)
      zeroers.t.emplace_back([=]() {
        for (size_t b = nblocks * t / nt; b < nblocks * (t + 1) / nt; ++b) {
          char* blk = (char*)kspace + b * ny * row_bytes;
          for (int y = 0; y < ny;) {  // runs of rows that are not acquired
            if (acquired[y]) {
              ++y;
              continue;
            }
            int y1 = y;
            while (y1 < ny && !acquired[y1]) ++y1;
            zero_stream(blk + (size_t)y * row_bytes, (size_t)(y1 - y) * row_bytes);
            y = y1;
          }
        }
        stream_fence();
      });
  }
  for (int b = 0; b < ng; ++b) {
    const Box& B = boxes[b];
    MRSIM_CUDA(cudaStreamWaitEvent(cs, ev[3 * b + 1], 0));
    if (sparse_k)
      down_k(B);
    else if (kspace)
      down(B, kspace, o->d_kspace, kunit * sizeof(float2));
    MRSIM_CUDA(cudaStreamWaitEvent(cs, ev[3 * b + 2], 0));
    if (comp_grad) down(B, comp_grad, o->d_comp_grad, o->ncomp * plane * sizeof(float2));
    if (fmap_grad && o->d_fmap_grad) down(B, fmap_grad, o->d_fmap_grad, plane * 4);
    if (r2_grad && o->d_r2_grad) down(B, r2_grad, o->d_r2_grad, o->ncomp * plane * 4);
  }
  // the compute stream ends after the copies, so work queued on it later sees them done
  MRSIM_CUDA(cudaEventRecord(ev[3 * ng], cs));
  MRSIM_CUDA(cudaStreamWaitEvent(st, ev[3 * ng], 0));
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

}  // namespace mrsim
