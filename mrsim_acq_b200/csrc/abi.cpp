// abi.cpp — the extern "C" entry points of libmrsim_acq_cuda.so (declared in include/mrsim_acq.h).
// Each converts C++ exceptions into a status code plus a thread-local message.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "driver.h"
#include "motion.h"
#include "nifti.h"
#include "ts_epi.h"
#include "host_tables.h"
#include "mrsim_internal.h"
#include "series.h"
#include "grase3d.h"
#include "spiral3d.h"
#include "host3d.h"
#include "spiral.h"
#include "spiral_host.h"
#include "spiral_recon.h"
#include "spin_history.h"

namespace {
thread_local std::string g_last_error;

template <class F>
int guarded(F&& f) {
  try {
    f();
    return MRSIM_OK;
  } catch (const mrsim::Error& e) {
    g_last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return MRSIM_ERR_NOMEM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return MRSIM_ERR_INVALID;
  }
}

void need(const void* p, const char* what) {
  if (!p) mrsim::fail(std::string(what) + " is NULL");
}

void check_slice_input(const mrsim_slice_input& inp, const mrsim_acquisition& acq) {
  if (inp.sim[0] <= 0 || inp.sim[1] <= 0 || inp.acq_matrix[0] <= 0 || inp.acq_matrix[1] <= 0)
    mrsim::fail("empty simulation grid or acquired matrix");
  if (!(inp.sim[0] % inp.acq_matrix[0] == 0 && inp.sim[1] % inp.acq_matrix[1] == 0))
    mrsim::fail("sim grid must be an integer multiple of the acquired matrix");
  if (inp.ncomp > mrsim::kMaxComp) mrsim::fail("more than 8 compartments");
  if (inp.ncomp > 0 && !inp.compartments) mrsim::fail("compartments is NULL");
  if (!inp.t2 && inp.ncomp > 0) mrsim::fail("t2 is NULL");
  if (!inp.fmap) mrsim::fail("fmap is NULL");
  if (std::max<int64_t>(acq.n_coils, 1) > mrsim::kMaxCoils) mrsim::fail("more than 64 coils");
}

// Runs `f` on the context's device with the context locked.
template <class F>
int on_ctx(mrsim_context* ctx, F&& f) {
  return guarded([&] {
    need(ctx, "context");
    std::lock_guard<std::mutex> lk(ctx->mu);
    MRSIM_CUDA(cudaSetDevice(ctx->device));
    f();
  });
}
}  // namespace

struct mrsim_epi_operator {
  mrsim::EpiOperator* impl;
};

struct mrsim_spiral_recon {
  mrsim::SpiralRecon* impl;
};

struct mrsim_spin_history {
  mrsim::SpinHistoryDev* impl;
};

namespace {
// host (re, im) f64 buffers through the device
template <class F>
int recon_call(mrsim_spiral_recon* rec, const double* in, size_t in_elems, double* out, size_t out_elems, F&& f) {
  if (!rec) return guarded([] { need(nullptr, "reconstruction"); });
  return on_ctx(rec->impl->ctx, [&] {
    need(in, "samples");
    need(out, "out");
    cudaStream_t st = rec->impl->ctx->stream;
    mrsim::DevArena T;
    double2* din = (double2*)T.upload(in, in_elems * 16, st);
    double2* dout = (double2*)T.alloc(out_elems * 16);
    f(din, dout);
    MRSIM_CUDA(cudaMemcpyAsync(out, dout, out_elems * 16, cudaMemcpyDeviceToHost, st));
    MRSIM_CUDA(cudaStreamSynchronize(st));
  });
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" {

int mrsim_abi_version(void) { return MRSIM_ABI_VERSION; }
const char* mrsim_last_error(void) { return g_last_error.c_str(); }

int mrsim_acquisition_default(mrsim_acquisition* acq) {
  return guarded([&] {
    need(acq, "acq");
    *acq = mrsim::acquisition_default();
  });
}

int mrsim_phase_model_hbcd_like(mrsim_phase_model* out) {  // phase.rs:187-195
  return guarded([&] {
    need(out, "out");
    std::memset(out, 0, sizeof *out);
    out->background[1] = 0.13;
    out->background[2] = 0.10;
    out->background[3] = 0.02;
    out->has_prep = 1;
    out->c_q = 0.0425;
    out->sigma_dx = 1.0;
    out->sigma_rot = 2.0e-3;
  });
}

int mrsim_phase_model_none(mrsim_phase_model* out) {  // phase.rs:197-205
  return guarded([&] {
    need(out, "out");
    std::memset(out, 0, sizeof *out);
    out->has_prep = 1;
  });
}

int mrsim_context_create(int device, mrsim_context** out) {
  return guarded([&] {
    need(out, "out");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
      cudaGetLastError();
      throw mrsim::Error(MRSIM_ERR_NOGPU, "no CUDA device: this library runs on the GPU only");
    }
    if (device < 0 || device >= n) mrsim::fail("device index out of range");
    auto* ctx = new mrsim_context();
    ctx->device = device;
    try {
      MRSIM_CUDA(cudaSetDevice(device));
      MRSIM_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    } catch (...) {
      delete ctx;
      throw;
    }
    *out = ctx;
  });
}

int mrsim_context_destroy(mrsim_context* ctx) {
  return guarded([&] {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& b : ctx->ws)
      if (b.p) cudaFree(b.p);
    for (auto& e : ctx->slot_ev)
      if (e) cudaEventDestroy(e);
    if (ctx->host_pinned) cudaFreeHost(ctx->host_pinned);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
  });
}

void* mrsim_context_stream(mrsim_context* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int mrsim_context_synchronize(mrsim_context* ctx) {
  return on_ctx(ctx, [&] { MRSIM_CUDA(cudaStreamSynchronize(ctx->stream)); });
}

int mrsim_sampling_mask(int64_t nx, int64_t ny, const mrsim_acquisition* acq, uint8_t* mask) {
  return guarded([&] {
    need(acq, "acq");
    need(mask, "mask");
    auto m = mrsim::sampling_mask((size_t)nx, (size_t)ny, *acq);
    std::memcpy(mask, m.data(), m.size());
  });
}

int64_t mrsim_pf_skipped_lines(int64_t ny, const mrsim_acquisition* acq) {
  return acq ? (int64_t)mrsim::pf_skipped_lines((size_t)ny, *acq) : -1;
}

int mrsim_line_timing(const mrsim_acquisition* acq, int64_t nx, int64_t ny, double* t_ms, double* trf_ms,
                      double* tread_ms, int8_t* polarity) {
  return guarded([&] {
    need(acq, "acq");
    auto lt = mrsim::line_timing(*acq, (size_t)nx, (size_t)ny);
    if (t_ms) std::memcpy(t_ms, lt.t_ms.data(), (size_t)ny * 8);
    if (trf_ms) std::memcpy(trf_ms, lt.trf_ms.data(), (size_t)ny * 8);
    if (tread_ms) std::memcpy(tread_ms, lt.tread_ms.data(), (size_t)ny * 8);
    if (polarity) std::memcpy(polarity, lt.polarity.data(), (size_t)ny);
  });
}

int mrsim_validate_acquisition_timing(const mrsim_acquisition* acq, int64_t nx, int64_t ny) {
  return guarded([&] {
    need(acq, "acq");
    mrsim::validate_acquisition_timing(*acq, (size_t)nx, (size_t)ny);
  });
}

int mrsim_epi_order(const mrsim_acquisition* acq, int64_t nx, int64_t ny, int64_t* order) {
  return guarded([&] {
    need(acq, "acq");
    need(order, "order");
    auto o = mrsim::epi_order(*acq, (size_t)nx, (size_t)ny);
    std::memcpy(order, o.data(), o.size() * 8);
  });
}

int mrsim_build_coil_kspaces(mrsim_context* ctx, const mrsim_slice_input* inp, const mrsim_acquisition* acq,
                             const double* t_ms, const double* trf_ms, const double* tread_ms, const int8_t* polarity,
                             const double* log_amp, double* out) {
  return on_ctx(ctx, [&] {
    need(inp, "inp");
    need(acq, "acq");
    need(out, "out");
    if (t_ms && !(trf_ms && tread_ms && polarity))
      mrsim::fail("line-timing table must have one entry per phase-encode line");
    mrsim::LineTimingTab lt;
    const int64_t ny = inp->acq_matrix[1];
    if (t_ms) {
      lt.t_ms.assign(t_ms, t_ms + ny);
      lt.trf_ms.assign(trf_ms, trf_ms + ny);
      lt.tread_ms.assign(tread_ms, tread_ms + ny);
      lt.polarity.assign(polarity, polarity + ny);
    }
    check_slice_input(*inp, *acq);
    auto k = mrsim::slice_forward2(ctx, *inp, *acq, t_ms ? &lt : nullptr, log_amp);
    for (size_t i = 0; i < k.size(); ++i) {
      out[2 * i] = (double)k[i].x;
      out[2 * i + 1] = (double)k[i].y;
    }
  });
}

int mrsim_simulate_slice(mrsim_context* ctx, const mrsim_slice_input* inp, const mrsim_acquisition* acq,
                         float* out) {
  return on_ctx(ctx, [&] {
    need(inp, "inp");
    need(acq, "acq");
    need(out, "out");
    check_slice_input(*inp, *acq);
    mrsim::SliceOutputs so;
    so.combined = (float2*)out;
    mrsim::simulate_slice_full(ctx, *inp, *acq, so);
  });
}

int mrsim_simulate_slice_full(mrsim_context* ctx, const mrsim_slice_input* inp, const mrsim_acquisition* acq,
                              float* combined, float* acquired, float* reconstructed, float* coil_images,
                              float* sensitivities, uint8_t* mask) {
  return on_ctx(ctx, [&] {
    need(inp, "inp");
    need(acq, "acq");
    need(combined, "combined");
    check_slice_input(*inp, *acq);
    mrsim::SliceOutputs so;
    so.combined = (float2*)combined;
    so.acquired = (float2*)acquired;
    so.reconstructed = (float2*)reconstructed;
    so.coil_images = (float2*)coil_images;
    so.sensitivities = sensitivities;
    so.mask = mask;
    mrsim::simulate_slice_full(ctx, *inp, *acq, so);
  });
}

int mrsim_simulate_slice_kspace(mrsim_context* ctx, const mrsim_slice_input* inp, const mrsim_acquisition* acq,
                                double* out) {
  return on_ctx(ctx, [&] {
    need(inp, "inp");
    need(acq, "acq");
    need(out, "out");
    check_slice_input(*inp, *acq);
    auto k = mrsim::slice_forward2(ctx, *inp, *acq, nullptr, nullptr);
    const size_t per = (size_t)inp->acq_matrix[0] * inp->acq_matrix[1];
    for (size_t i = 0; i < per; ++i) {
      out[2 * i] = (double)k[i].x;
      out[2 * i + 1] = (double)k[i].y;
    }
  });
}

static void check_series_input(const mrsim_acquisition_input* in, const mrsim_acquisition* acq,
                               bool images = true) {
  need(in, "in");
  need(acq, "acq");
  if (in->ncomp > 0) {
    if (images) need(in->images, "images");
    need(in->t2, "t2");
  }
  need(in->phase, "phase");
}

int mrsim_simulate_acquisition_complex(mrsim_context* ctx, const mrsim_acquisition_input* in,
                                       const mrsim_acquisition* acq, const mrsim_acquisition_options* opts,
                                       mrsim_acquisition_output* out) {
  return on_ctx(ctx, [&] {
    check_series_input(in, acq);
    need(out, "out");
    need(out->re, "out->re");
    need(out->im, "out->im");
    mrsim::acquire_series(ctx, *in, *acq, opts, in->seed, in->seed, in->images, *out);
  });
}

int mrsim_simulate_acquisition_oversampled(mrsim_context* ctx, const mrsim_acquisition_input* in,
                                           const mrsim_acquisition* acq, float* mag, float* phase) {
  return on_ctx(ctx, [&] {
    check_series_input(in, acq);
    need(mag, "mag");
    need(phase, "phase");
    mrsim_acquisition_output out;
    std::memset(&out, 0, sizeof out);
    out.re = mag;  // the device writes magnitude and phase (kspace.rs:1839-1846) in its output pass
    out.im = phase;
    mrsim::acquire_series(ctx, *in, *acq, nullptr, in->seed, in->seed, in->images, out, true);
  });
}

int mrsim_simulate_acquisition_echoes(mrsim_context* ctx, const mrsim_acquisition_input* in,
                                      const float* const* const* images_per_echo, const mrsim_acquisition* acq,
                                      const double* echo_times_ms, int64_t n_echoes,
                                      const float* const* const* grappa_calibration_images,
                                      const uint64_t* grappa_calibration_seeds, float* const* mag,
                                      float* const* phase) {
  return on_ctx(ctx, [&] {
    check_series_input(in, acq, false);
    need(images_per_echo, "images_per_echo");
    need(echo_times_ms, "echo_times_ms");
    need(mag, "mag");
    need(phase, "phase");
    // `simulate_acquisition_echoes` kspace.rs:2152-2215
    for (int64_t e = 0; e + 1 < n_echoes; ++e)
      if (!(echo_times_ms[e] < echo_times_ms[e + 1])) {
        char buf[256];
        std::snprintf(buf, sizeof buf, "echo times must increase strictly: echo %lld at %g ms, echo %lld at %g ms",
                      (long long)e, echo_times_ms[e], (long long)(e + 1), echo_times_ms[e + 1]);
        mrsim::fail(buf);
      }
    if (n_echoes <= 0) mrsim::fail("simulate_acquisition_echoes needs at least one echo");
    mrsim::SeriesImageCache images;  // echoes given the same image arrays upload them once
    for (int64_t e = 0; e < n_echoes; ++e) {
      mrsim_acquisition acq_e = *acq;
      acq_e.t_echo = echo_times_ms[e];
      mrsim_acquisition_options opts;
      std::memset(&opts, 0, sizeof opts);
      if (grappa_calibration_images) {
        opts.has_grappa_calibration = 1;
        opts.grappa_calibration_images = grappa_calibration_images[e];
        opts.grappa_calibration_seed = grappa_calibration_seeds ? grappa_calibration_seeds[e] : in->seed;
      }
      mrsim_acquisition_output out;
      std::memset(&out, 0, sizeof out);
      out.re = mag[e];
      out.im = phase[e];
      mrsim::acquire_series(ctx, *in, acq_e, &opts, in->seed, in->seed ^ mrsim::echo_salt((uint64_t)e),
                            images_per_echo[e], out, true, &images);
    }
  });
}

int mrsim_build_coil_kspaces_noalloc(const mrsim_slice_input* inp, const mrsim_acquisition* acq, void* stream,
                                     float* kspace) {
  return guarded([&] {
    need(inp, "inp");
    need(acq, "acq");
    need(kspace, "kspace");
    check_slice_input(*inp, *acq);
    mrsim::build_coil_kspaces_noalloc(*inp, *acq, (float2*)kspace, (cudaStream_t)stream);
  });
}

int mrsim_epi_operator_create(mrsim_context* ctx, const mrsim_acquisition_input* in, const mrsim_acquisition* acq,
                              const double* echo_times_ms, int64_t n_echoes, const int64_t* slice_z, int64_t nz_full,
                              int32_t grads, mrsim_epi_operator** out) {
  return on_ctx(ctx, [&] {
    need(in, "in");
    need(acq, "acq");
    need(out, "out");
    need(in->fmap, "fmap");
    need(in->t2, "t2");
    auto* op = new mrsim_epi_operator();
    try {
      op->impl = mrsim::epi_operator_create(ctx, *in, *acq, echo_times_ms, n_echoes, slice_z, nz_full, grads);
    } catch (...) {
      delete op;
      throw;
    }
    *out = op;
  });
}

int mrsim_epi_operator_destroy(mrsim_epi_operator* op) {
  return guarded([&] {
    if (!op) return;
    if (op->impl) {
      mrsim_context* ctx = op->impl->ctx;
      std::lock_guard<std::mutex> lk(ctx->mu);
      cudaSetDevice(ctx->device);
      cudaStreamSynchronize(ctx->stream);
      delete op->impl;
    }
    delete op;
  });
}

int64_t mrsim_epi_operator_samples(const mrsim_epi_operator* op) {
  return op && op->impl ? op->impl->samples_per_step : -1;
}

int mrsim_epi_operator_buffers(mrsim_epi_operator* op, float** images, float** kspace, float** comp_grad,
                               float** fmap_grad, float** r2_grad) {
  return guarded([&] {
    need(op, "operator");
    auto* o = op->impl;
    if (images) *images = o->d_images;
    if (kspace) *kspace = (float*)o->d_kspace;
    if (comp_grad) *comp_grad = (float*)o->d_comp_grad;
    if (fmap_grad) *fmap_grad = o->d_fmap_grad;
    if (r2_grad) *r2_grad = o->d_r2_grad;
  });
}

int mrsim_epi_operator_upload_images(mrsim_epi_operator* op, const float* const* images) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] {
    need(images, "images");
    mrsim::upload_series_images(op->impl, images);
  });
}

int mrsim_epi_operator_set_fieldmap(mrsim_epi_operator* op, const float* fmap) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] {
    need(fmap, "fmap");
    mrsim::epi_operator_set_fieldmap(op->impl, fmap);
  });
}

int mrsim_epi_operator_forward(mrsim_epi_operator* op) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] { mrsim::epi_operator_forward(op->impl); });
}

int mrsim_epi_operator_adjoint(mrsim_epi_operator* op) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] { mrsim::epi_operator_adjoint(op->impl); });
}

int mrsim_epi_operator_stage(mrsim_epi_operator* op, int32_t stage) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] {
    const mrsim::EpiPlan* p = op->impl->plan.get();
    cudaStream_t st = op->impl->ctx->stream;
    switch (stage) {
      case 0: mrsim::epi_plan_statics(p, st); break;
      case 1:
        if (op->impl->ts)
          mrsim::ts_forward_ystage(*op->impl->ts, *p, st);
        else
          mrsim::epi_plan_forward_ystage(p, st);
        break;
      case 2: mrsim::epi_plan_forward_xstage(p, st); break;
      case 3: mrsim::epi_plan_adjoint_xstage(p, st); break;
      case 4:
        if (op->impl->ts)
          mrsim::ts_adjoint_ystage(*op->impl->ts, *p, st);
        else
          mrsim::epi_plan_adjoint_ystage(p, st);
        break;
      default: mrsim::fail("stage must be 0..4");
    }
  });
}

int mrsim_epi_operator_set_segmented(mrsim_epi_operator* op, int32_t precision) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] {
    MRSIM_CUDA(cudaStreamSynchronize(op->impl->ctx->stream));
    mrsim::epi_operator_set_segmented(op->impl, precision);
  });
}

int mrsim_epi_operator_segmentation(const mrsim_epi_operator* op, int32_t* n_groups, int32_t* seg_l, double* bound,
                                    int32_t max_groups, double* flops_forward, double* flops_adjoint) {
  return guarded([&] {
    need(op, "operator");
    need(n_groups, "n_groups");
    const mrsim::TsPlan* t = op->impl->ts;
    *n_groups = t ? t->n_groups : 0;
    if (t) {
      for (int g = 0; g < t->n_groups && g < max_groups; ++g) {
        if (seg_l) seg_l[g] = t->L[g];
        if (bound) bound[g] = t->bound[g];
      }
    }
    if (flops_forward) *flops_forward = t ? t->flops_fwd : 0.0;
    if (flops_adjoint) *flops_adjoint = t ? t->flops_adj : 0.0;
  });
}

int mrsim_epi_operator_tune(mrsim_epi_operator* op, const char* cache_path, int32_t flags, char* choice,
                            int64_t choice_cap, double* ms) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] {
    MRSIM_CUDA(cudaStreamSynchronize(op->impl->ctx->stream));
    const std::string c = mrsim::epi_operator_tune(op->impl, cache_path, flags, ms);
    if (choice && choice_cap > 0) {
      const size_t n = std::min<size_t>(c.size(), (size_t)choice_cap - 1);
      std::memcpy(choice, c.data(), n);
      choice[n] = 0;
    }
  });
}

int mrsim_epi_operator_segmented_status(mrsim_epi_operator* op, int32_t* code) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] {
    need(code, "code");
    *code = mrsim::epi_operator_segmented_error(op->impl);
  });
}

int mrsim_probe_fp32_tflops(mrsim_context* ctx, double* tflops) {
  return on_ctx(ctx, [&] {
    need(tflops, "tflops");
    *tflops = mrsim::probe_fp32_tflops(ctx->stream);
  });
}

int mrsim_epi_operator_adjoint_host(mrsim_epi_operator* op, const float* kspace, float* comp_grad, float* fmap_grad,
                                    float* r2_grad) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] {
    need(kspace, "kspace");
    auto* o = op->impl;
    cudaStream_t st = o->ctx->stream;
    const size_t plane = (size_t)o->snx * o->sny, nunits = (size_t)o->nv * o->nz;
    MRSIM_CUDA(cudaMemcpyAsync(o->d_kspace, kspace, o->kspace_elems * sizeof(float2), cudaMemcpyHostToDevice, st));
    mrsim::epi_operator_adjoint(o);
    if (comp_grad)
      MRSIM_CUDA(cudaMemcpyAsync(comp_grad, o->d_comp_grad, nunits * o->ncomp * plane * sizeof(float2),
                                 cudaMemcpyDeviceToHost, st));
    if (fmap_grad && o->d_fmap_grad)
      MRSIM_CUDA(cudaMemcpyAsync(fmap_grad, o->d_fmap_grad, nunits * plane * 4, cudaMemcpyDeviceToHost, st));
    if (r2_grad && o->d_r2_grad)
      MRSIM_CUDA(cudaMemcpyAsync(r2_grad, o->d_r2_grad, nunits * o->ncomp * plane * 4, cudaMemcpyDeviceToHost, st));
    MRSIM_CUDA(cudaStreamSynchronize(st));
  });
}

int mrsim_epi_operator_host_bytes(const mrsim_epi_operator* op, int64_t* upload_bytes, int64_t* download_bytes) {
  return guarded([&] {
    need(op, "operator");
    need(upload_bytes, "upload_bytes");
    need(download_bytes, "download_bytes");
    const auto* o = op->impl;
    const int64_t plane = (int64_t)o->snx * o->sny, units = (int64_t)o->nv * o->nz;
    const int64_t rows = o->krow_n > 0 ? (int64_t)o->krow_n * o->n_echoes : (int64_t)o->n_echoes * o->ny;
    *upload_bytes = units * o->ncomp * plane * 4;
    *download_bytes = units * o->ncoils * rows * o->nx * 8 + units * o->ncomp * plane * 8 +
                      (o->d_fmap_grad ? units * plane * 4 : 0) + (o->d_r2_grad ? units * o->ncomp * plane * 4 : 0);
  });
}

int mrsim_epi_operator_apply_host(mrsim_epi_operator* op, const float* const* images, float* kspace, float* comp_grad,
                                  float* fmap_grad, float* r2_grad) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] {
    mrsim::epi_operator_apply_host(op->impl, images, kspace, comp_grad, fmap_grad, r2_grad);
  });
}

int mrsim_epi_operator_apply_host_compact(mrsim_epi_operator* op, const float* const* images, float* kspace_rows,
                                          float* comp_grad, float* fmap_grad, float* r2_grad) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] {
    mrsim::epi_operator_apply_host(op->impl, images, kspace_rows, comp_grad, fmap_grad, r2_grad, true);
  });
}

int mrsim_epi_operator_acquired_rows(const mrsim_epi_operator* op, int32_t* first, int32_t* step, int32_t* count) {
  return guarded([&] {
    need(op, "operator");
    need(first, "first");
    need(step, "step");
    need(count, "count");
    *first = op->impl->krow0;
    *step = op->impl->krow_step;
    *count = op->impl->krow_n;
  });
}

int mrsim_epi_operator_host_bytes_for(const mrsim_epi_operator* op, int32_t outputs, int64_t* upload_bytes,
                                      int64_t* download_bytes) {
  return guarded([&] {
    need(op, "operator");
    need(upload_bytes, "upload_bytes");
    need(download_bytes, "download_bytes");
    const auto* o = op->impl;
    const int64_t plane = (int64_t)o->snx * o->sny, units = (int64_t)o->nv * o->nz;
    const int64_t rows = o->krow_n > 0 ? (int64_t)o->krow_n * o->n_echoes : (int64_t)o->n_echoes * o->ny;
    *upload_bytes = units * o->ncomp * plane * 4;
    int64_t d = 0;
    if (outputs & 1) d += units * o->ncoils * rows * o->nx * 8;
    if (outputs & 2) d += units * o->ncomp * plane * 8;
    if ((outputs & 4) && o->d_fmap_grad) d += units * plane * 4;
    if ((outputs & 8) && o->d_r2_grad) d += units * o->ncomp * plane * 4;
    *download_bytes = d;
  });
}


// ---- a batch of series of different geometries -----------------------------------------------------
struct mrsim_epi_batch {
  mrsim::EpiBatch* impl;
};

int mrsim_epi_batch_create(mrsim_context* ctx, int32_t n_series, const mrsim_acquisition_input* const* inputs,
                           const mrsim_acquisition* acq, const double* echo_times_ms, int64_t n_echoes,
                           int32_t grads, mrsim_epi_batch** out) {
  return on_ctx(ctx, [&] {
    need(inputs, "inputs");
    need(acq, "acq");
    need(out, "out");
    for (int32_t i = 0; i < n_series; ++i) {
      need(inputs[i], "inputs[i]");
      need(inputs[i]->fmap, "fmap");
      need(inputs[i]->t2, "t2");
    }
    auto* b = new mrsim_epi_batch();
    try {
      b->impl = mrsim::epi_batch_create(ctx, n_series, inputs, *acq, echo_times_ms, n_echoes, grads);
    } catch (...) {
      delete b;
      throw;
    }
    *out = b;
  });
}

int mrsim_epi_batch_destroy(mrsim_epi_batch* b) {
  return guarded([&] {
    if (!b) return;
    if (b->impl) {
      mrsim_context* ctx = b->impl->ctx;
      std::lock_guard<std::mutex> lk(ctx->mu);
      cudaSetDevice(ctx->device);
      cudaStreamSynchronize(ctx->stream);
      delete b->impl;
    }
    delete b;
  });
}

int64_t mrsim_epi_batch_samples(const mrsim_epi_batch* b) { return b && b->impl ? b->impl->samples : 0; }

int mrsim_epi_batch_forward(mrsim_epi_batch* b) {
  if (!b) return guarded([] { need(nullptr, "batch"); });
  return on_ctx(b->impl->ctx, [&] { mrsim::epi_batch_forward(b->impl); });
}

int mrsim_epi_batch_adjoint(mrsim_epi_batch* b) {
  if (!b) return guarded([] { need(nullptr, "batch"); });
  return on_ctx(b->impl->ctx, [&] { mrsim::epi_batch_adjoint(b->impl); });
}

int mrsim_epi_batch_download(mrsim_epi_batch* b, int32_t series, float* kspace, float* comp_grad) {
  if (!b) return guarded([] { need(nullptr, "batch"); });
  return on_ctx(b->impl->ctx, [&] {
    if (series < 0 || series >= (int32_t)b->impl->ops.size()) mrsim::fail("series index out of range");
    const mrsim::EpiOperator* o = b->impl->ops[series].get();
    cudaStream_t st = b->impl->ctx->stream;
    if (kspace)
      MRSIM_CUDA(cudaMemcpyAsync(kspace, o->d_kspace, o->kspace_elems * sizeof(float2), cudaMemcpyDeviceToHost, st));
    if (comp_grad)
      MRSIM_CUDA(cudaMemcpyAsync(comp_grad, o->d_comp_grad,
                                 (size_t)o->nv * o->nz * o->ncomp * o->snx * o->sny * sizeof(float2),
                                 cudaMemcpyDeviceToHost, st));
    MRSIM_CUDA(cudaStreamSynchronize(st));
  });
}

// ---- writing the series ----------------------------------------------------------------------------
int mrsim_write_nifti_4d(const char* path, const int64_t* dims, int64_t nt, const float* data, const double* v2w,
                         double tr_s) {
  return guarded([&] {
    need(path, "path");
    need(dims, "dims");
    need(data, "data");
    need(v2w, "v2w");
    mrsim::write_nifti(path, dims, nt, data, v2w, tr_s, true);
  });
}

int mrsim_write_nifti_3d(const char* path, const int64_t* dims, const float* data, const double* v2w) {
  return guarded([&] {
    need(path, "path");
    need(dims, "dims");
    need(data, "data");
    need(v2w, "v2w");
    mrsim::write_nifti(path, dims, 1, data, v2w, 0.0, false);
  });
}

int mrsim_hires_grid(const double* v2w, const int64_t* dims, int64_t o, double* out_v2w, int64_t* out_dims) {
  return guarded([&] {
    need(v2w, "v2w");
    need(dims, "dims");
    need(out_v2w, "out_v2w");
    need(out_dims, "out_dims");
    mrsim::hires_grid(v2w, dims, o, out_v2w, out_dims);
  });
}

int mrsim_write_complex_4d(const char* out_prefix, const char* suffix, const int64_t* dims, int64_t n_volumes,
                           const float* mag, const float* phase, const double* v2w, const mrsim_sidecar_info* info) {
  return guarded([&] {
    need(out_prefix, "out_prefix");
    need(suffix, "suffix");
    need(dims, "dims");
    need(mag, "mag");
    need(phase, "phase");
    need(v2w, "v2w");
    need(info, "info");
    mrsim::write_complex_4d(out_prefix, suffix, dims, n_volumes, mag, phase, v2w, *info);
  });
}

// ---- image motion -----------------------------------------------------------------------------------
namespace {
// the reference layout of n_volumes volumes: element (x, y, z) of volume g at (x + nx (y + ny z)) nv + g
struct HostSeries {
  long long sx, sy, sz, sg, sc;
};
HostSeries host_strides(const int64_t* dims, int64_t nv) {
  const long long nvox = dims[0] * dims[1] * dims[2];
  return {nv, dims[0] * nv, dims[0] * dims[1] * nv, 1, nvox * nv};
}
void check_dims(const int64_t* dims, int64_t nv) {
  need(dims, "dims");
  if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0 || nv <= 0) mrsim::fail("empty volume or no volumes");
  if (dims[0] * dims[1] * dims[2] >= (1LL << 31)) mrsim::fail("a volume of 2^31 voxels or more");
}
}  // namespace

int mrsim_resample_by_pose(mrsim_context* ctx, const float* src, const int64_t* dims, const double* v2w,
                           const double* pose, float* out) {
  return on_ctx(ctx, [&] {
    need(src, "src");
    need(v2w, "v2w");
    need(pose, "pose");
    need(out, "out");
    check_dims(dims, 1);
    cudaStream_t st = ctx->stream;
    const size_t n = (size_t)(dims[0] * dims[1] * dims[2]);
    mrsim::DevArena A;
    float* in = (float*)A.upload(src, n * 4, st);
    float* o = (float*)A.alloc(n * 4);
    mrsim::resample_poses_device(in, o, dims, 1, 1, 1, dims[0], dims[0] * dims[1], 0, 0, v2w, pose, st, A);
    MRSIM_CUDA(cudaMemcpyAsync(out, o, n * 4, cudaMemcpyDeviceToHost, st));
    MRSIM_CUDA(cudaStreamSynchronize(st));
  });
}

int mrsim_apply_motion(mrsim_context* ctx, float* const* images, int64_t ncomp, const int64_t* dims, int64_t n_volumes,
                       const double* v2w, const double* poses) {
  return on_ctx(ctx, [&] {
    need(images, "images");
    need(v2w, "v2w");
    need(poses, "poses");
    check_dims(dims, n_volumes);
    if (ncomp <= 0) return;
    cudaStream_t st = ctx->stream;
    const HostSeries H = host_strides(dims, n_volumes);
    const size_t per = (size_t)H.sc;
    mrsim::DevArena A;
    float* in = (float*)A.alloc(per * ncomp * 4);
    float* o = (float*)A.alloc(per * ncomp * 4);
    for (int64_t c = 0; c < ncomp; ++c)
      MRSIM_CUDA(cudaMemcpyAsync(in + per * c, images[c], per * 4, cudaMemcpyHostToDevice, st));
    mrsim::resample_poses_device(in, o, dims, (int)n_volumes, (int)ncomp, H.sx, H.sy, H.sz, H.sg, H.sc, v2w, poses,
                                 st, A);
    for (int64_t c = 0; c < ncomp; ++c)
      MRSIM_CUDA(cudaMemcpyAsync(images[c], o + per * c, per * 4, cudaMemcpyDeviceToHost, st));
    MRSIM_CUDA(cudaStreamSynchronize(st));
  });
}

int mrsim_apply_multiband_motion(mrsim_context* ctx, float* const* images, int64_t ncomp, const int64_t* dims,
                                 int64_t n_volumes, const double* v2w, int64_t mb, int32_t interleaved,
                                 const mrsim_dropout_law* law, const mrsim_motion_event* events, int64_t n_events,
                                 const int64_t* slice_z, int64_t nz_full, mrsim_dropped_shot* dropped,
                                 int64_t capacity, int64_t* n_dropped) {
  return on_ctx(ctx, [&] {
    need(images, "images");
    need(v2w, "v2w");
    need(law, "law");
    need(n_dropped, "n_dropped");
    check_dims(dims, n_volumes);
    if (n_events > 0) need(events, "events");
    cudaStream_t st = ctx->stream;
    const HostSeries H = host_strides(dims, n_volumes);
    const size_t per = (size_t)H.sc;
    mrsim::DevArena A;
    float* in = (float*)A.alloc(per * std::max<int64_t>(ncomp, 1) * 4);
    float* o = (float*)A.alloc(per * std::max<int64_t>(ncomp, 1) * 4);
    for (int64_t c = 0; c < ncomp; ++c)
      MRSIM_CUDA(cudaMemcpyAsync(in + per * c, images[c], per * 4, cudaMemcpyHostToDevice, st));
    *n_dropped = mrsim::multiband_device(in, o, dims, (int)n_volumes, (int)ncomp, H.sx, H.sy, H.sz, H.sg, H.sc, v2w,
                                         mb, interleaved != 0, *law, events, n_events, slice_z, nz_full, dropped,
                                         capacity, st, A);
    for (int64_t c = 0; c < ncomp; ++c)
      MRSIM_CUDA(cudaMemcpyAsync(images[c], o + per * c, per * 4, cudaMemcpyDeviceToHost, st));
    MRSIM_CUDA(cudaStreamSynchronize(st));
  });
}

int mrsim_epi_operator_apply_motion(mrsim_epi_operator* op, const double* v2w, const double* poses) {
  if (!op) return guarded([] { need(nullptr, "operator"); });
  return on_ctx(op->impl->ctx, [&] {
    need(v2w, "v2w");
    need(poses, "poses");
    auto* o = op->impl;
    cudaStream_t st = o->ctx->stream;
    const long long plane = (long long)o->snx * o->sny;
    const size_t n = (size_t)o->nv * o->nz * o->ncomp * plane;
    const int64_t dims[3] = {o->snx, o->sny, o->nz};
    // the pre-motion images, then the moved ones back into the operator's buffer
    float* scratch = (float*)mrsim::workspace(o->ctx, 21, n * 4);
    MRSIM_CUDA(cudaMemcpyAsync(scratch, o->d_images, n * 4, cudaMemcpyDeviceToDevice, st));
    mrsim::DevArena A;
    mrsim::resample_poses_device(scratch, o->d_images, dims, o->nv, o->ncomp, 1, o->snx, o->ncomp * plane,
                                 (long long)o->nz * o->ncomp * plane, plane, v2w, poses, st, A);
    MRSIM_CUDA(cudaStreamSynchronize(st));  // the pose tables (in A) are read by the kernel
  });
}

// ---- stack-of-spirals path ------------------------------------------------------------------------
int mrsim_spiral_tau_c(int64_t nx, int64_t interleaves, double readout_ms, double dwell_ms, double radial_oversampling,
                       double* tau_c_ms) {
  return guarded([&] {
    need(tau_c_ms, "tau_c_ms");
    *tau_c_ms = mrsim::spiral_tau_c((int)nx, (int)interleaves, readout_ms, dwell_ms, radial_oversampling);
  });
}

int mrsim_spiral_trajectory(int64_t nx, int64_t ny, int64_t interleaves, double readout_ms, double dwell_ms,
                            double radial_oversampling, int64_t capacity, double* k, double* tau_ms,
                            mrsim_spiral_info* info) {
  return guarded([&] {
    need(info, "info");
    mrsim::SpiralTraj tr =
        mrsim::spiral_trajectory((int)nx, (int)ny, (int)interleaves, readout_ms, dwell_ms, radial_oversampling);
    info->samples = (int64_t)tr.tau_ms.size();
    info->interleaves = tr.interleaves;
    info->k_max = tr.k_max;
    info->n_turns = tr.n_turns;
    info->tau_c_ms = tr.tau_c_ms;
    if (!k && !tau_ms) return;
    if (capacity < info->samples) mrsim::fail("sample capacity below the samples per interleaf");
    if (tau_ms) std::memcpy(tau_ms, tr.tau_ms.data(), tr.tau_ms.size() * 8);
    if (k) std::memcpy(k, tr.k.data(), tr.k.size() * 8);
  });
}

static void tseg_plan_out(mrsim::TsegDevice* dev, const double* tau_ms, int64_t n_tau, double t_ms, const double d[2],
                          const double f[2], int64_t l_capacity, double* tau_l, double* b, mrsim_tseg_info* info) {
    need(d, "d");
    need(f, "f");
    need(info, "info");
    if (n_tau > 0) need(tau_ms, "tau_ms");
    std::vector<double> tau(tau_ms, tau_ms + std::max<int64_t>(0, n_tau));
    mrsim::TsegPlan p = mrsim::tseg_plan(tau, t_ms, d, f, dev);
    info->l = p.l;
    info->m = p.m;
    info->b_sum = p.b_sum;
    info->grid_err = p.grid_err;
    info->bound = p.bound;
    if (!tau_l && !b) return;
    if (l_capacity < p.l) mrsim::fail("segment capacity below the plan's L");
    if (tau_l) std::memcpy(tau_l, p.tau_l.data(), p.tau_l.size() * 8);
    if (b) std::memcpy(b, p.b.data(), p.b.size() * 8);
}

int mrsim_tseg_plan(const double* tau_ms, int64_t n_tau, double t_ms, const double d[2], const double f[2],
                    int64_t l_capacity, double* tau_l, double* b, mrsim_tseg_info* info) {
  return guarded([&] { tseg_plan_out(nullptr, tau_ms, n_tau, t_ms, d, f, l_capacity, tau_l, b, info); });
}

int mrsim_tseg_plan_device(mrsim_context* ctx, const double* tau_ms, int64_t n_tau, double t_ms, const double d[2],
                           const double f[2], int64_t l_capacity, double* tau_l, double* b, mrsim_tseg_info* info) {
  return on_ctx(ctx, [&] {
    mrsim::TsegDevice dev(ctx->stream);
    tseg_plan_out(&dev, tau_ms, n_tau, t_ms, d, f, l_capacity, tau_l, b, info);
  });
}

int mrsim_epg_cpmg(int64_t n_echoes, double esp_ms, double refocusing_deg, double t1_ms, double t2_ms,
                   double* ln_amp) {
  return guarded([&] {
    if (n_echoes < 0) mrsim::fail("negative echo count");
    if (n_echoes > 0) need(ln_amp, "ln_amp");
    auto v = mrsim::epg_cpmg((int)n_echoes, esp_ms, refocusing_deg, t1_ms, t2_ms);
    if (n_echoes > 0) std::memcpy(ln_amp, v.data(), v.size() * 8);
  });
}

int mrsim_nufft_kernel_width(double tol) { return mrsim::nufft_width(tol); }

static void check_nufft(const int64_t n[2], const int64_t m_lo[2], const int64_t m_out[2], int64_t npts, int sign) {
  need(n, "n");
  need(m_lo, "m_lo");
  need(m_out, "m_out");
  for (int a = 0; a < 2; ++a)
    if (n[a] <= 0 || n[a] > 8192) mrsim::fail("NUFFT period must be in 1..8192");
  if (npts < 0 || npts > ((int64_t)1 << 30)) mrsim::fail("NUFFT point count out of range");
  if (sign != 1 && sign != -1) mrsim::fail("NUFFT sign must be +1 or -1");
}

int mrsim_nufft2_type1(mrsim_context* ctx, const int64_t n[2], const int64_t m_lo[2], const int64_t m_out[2],
                       double tol, const double* u, int64_t npts, const float* weights, int32_t sign, float* modes) {
  return on_ctx(ctx, [&] {
    check_nufft(n, m_lo, m_out, npts, sign);
    need(modes, "modes");
    if (npts > 0) {
      need(u, "u");
      need(weights, "weights");
    }
    mrsim::nufft2_host(ctx, 1, (int)n[0], (int)n[1], (int)m_lo[0], (int)m_lo[1], (int)m_out[0], (int)m_out[1], tol, u,
                       (int)npts, weights, sign, modes);
  });
}

int mrsim_nufft2_type2(mrsim_context* ctx, const int64_t n[2], const int64_t m_lo[2], const int64_t m_out[2],
                       double tol, const float* modes, const double* u, int64_t npts, int32_t sign, float* out) {
  return on_ctx(ctx, [&] {
    check_nufft(n, m_lo, m_out, npts, sign);
    need(modes, "modes");
    if (npts > 0) {
      need(u, "u");
      need(out, "out");
    }
    mrsim::nufft2_host(ctx, 2, (int)n[0], (int)n[1], (int)m_lo[0], (int)m_lo[1], (int)m_out[0], (int)m_out[1], tol, u,
                       (int)npts, modes, sign, out);
  });
}

int mrsim_spiral_kspace_exact(mrsim_context* ctx, const mrsim_slice_input* inp, const mrsim_acquisition* acq,
                              int64_t coil, int64_t ncoils, const double* k, const double* tau_ms, int64_t npts,
                              const double* log_amp, float* out) {
  return on_ctx(ctx, [&] {
    need(inp, "inp");
    need(acq, "acq");
    check_slice_input(*inp, *acq);
    if (npts < 0) mrsim::fail("negative sample count");
    if (npts > 0) {
      need(k, "k");
      need(tau_ms, "tau_ms");
      need(out, "out");
    }
    if (coil < 0 || coil >= std::max<int64_t>(ncoils, 1)) mrsim::fail("coil index out of range");
    mrsim::spiral_exact_host(ctx, *inp, *acq, (int)coil, (int)ncoils, k, tau_ms, (int)npts, log_amp, out);
  });
}

int mrsim_spiral_segmented_forward(mrsim_context* ctx, const mrsim_slice_input* inp, const mrsim_acquisition* acq,
                                   int64_t coil, int64_t ncoils, const double* k, const int64_t* tau_idx,
                                   int64_t npts, const double* tau_ms, int64_t n_tau, double t_ms, const double d[2],
                                   const double f[2], const double* log_amp, int32_t decay_inside, float* out,
                                   mrsim_tseg_info* info) {
  return on_ctx(ctx, [&] {
    need(inp, "inp");
    need(acq, "acq");
    need(d, "d");
    need(f, "f");
    check_slice_input(*inp, *acq);
    if (npts < 0 || n_tau < 0) mrsim::fail("negative sample count");
    if (npts > 0) {
      need(k, "k");
      need(tau_idx, "tau_idx");
      need(out, "out");
    }
    if (n_tau > 0) need(tau_ms, "tau_ms");
    if (coil < 0 || coil >= std::max<int64_t>(ncoils, 1)) mrsim::fail("coil index out of range");
    auto r = mrsim::spiral_segmented_host(ctx, *inp, *acq, (int)coil, (int)ncoils, k, tau_idx, (int)npts, tau_ms,
                                          (int)n_tau, t_ms, d, f, log_amp, decay_inside != 0, out);
    if (info) {
      info->l = r.l;
      info->m = r.m;
      info->bound = r.bound;
      info->b_sum = r.b_sum;
      info->grid_err = r.grid_err;
    }
  });
}

int mrsim_spiral_recon_create(mrsim_context* ctx, const double* k, int64_t npts, int64_t n, int32_t window_kind,
                              double window_a, double window_b, int64_t iterations, double kappa,
                              int32_t band_limited, mrsim_spiral_recon** out) {
  return on_ctx(ctx, [&] {
    need(out, "out");
    need(k, "k");
    if (npts <= 0 || npts > ((int64_t)1 << 28)) mrsim::fail("sample count out of range");
    if (iterations > 100000) mrsim::fail("Chebyshev iterations out of range");
    mrsim_acquisition w = mrsim::acquisition_default();
    w.window_kind = window_kind;
    w.window_a = window_a;
    w.window_b = window_b;
    auto* r = new mrsim::SpiralRecon(ctx, k, (int)npts, (int)n, w, (int)iterations, kappa, band_limited != 0);
    *out = new mrsim_spiral_recon{r};
  });
}

int mrsim_spiral_recon_destroy(mrsim_spiral_recon* rec) {
  return guarded([&] {
    if (!rec) return;
    mrsim_context* ctx = rec->impl->ctx;
    std::lock_guard<std::mutex> lk(ctx->mu);
    MRSIM_CUDA(cudaSetDevice(ctx->device));
    delete rec->impl;
    delete rec;
  });
}

int mrsim_spiral_recon_info(const mrsim_spiral_recon* rec, double* lambda_hi, int64_t* power_iterations,
                            double* weights) {
  return guarded([&] {
    need(rec, "reconstruction");
    const mrsim::SpiralRecon* r = rec->impl;
    if (lambda_hi) *lambda_hi = r->lambda_hi;
    if (power_iterations) *power_iterations = r->power_iterations;
    if (weights) std::memcpy(weights, r->w_host.data(), r->w_host.size() * 8);
  });
}

int mrsim_spiral_recon_gridding(mrsim_spiral_recon* rec, const double* samples, int64_t batch, double* out) {
  if (batch <= 0) return guarded([] { mrsim::fail("batch must be positive"); });
  const size_t np = rec ? (size_t)rec->impl->npts : 0, nn = rec ? (size_t)rec->impl->n * rec->impl->n : 0;
  return recon_call(rec, samples, np * batch, out, nn * batch,
                    [&](double2* i, double2* o) { rec->impl->gridding(i, (int)batch, o); });
}

int mrsim_spiral_recon_image(mrsim_spiral_recon* rec, const double* samples, int64_t batch, double* out) {
  if (batch <= 0) return guarded([] { mrsim::fail("batch must be positive"); });
  const size_t np = rec ? (size_t)rec->impl->npts : 0, nn = rec ? (size_t)rec->impl->n * rec->impl->n : 0;
  return recon_call(rec, samples, np * batch, out, nn * batch, [&](double2* i, double2* o) {
    for (int64_t b0 = 0; b0 < batch; b0 += mrsim::kMaxBatch) {
      const int nb = (int)std::min<int64_t>(mrsim::kMaxBatch, batch - b0);
      rec->impl->images(i + b0 * np, nb, o + b0 * nn);
    }
  });
}

int mrsim_spiral_recon_rings(mrsim_spiral_recon* rec, const double* coil_samples, int64_t n_partitions,
                             int64_t ncoils, int64_t ring, const double* zsens, double* out) {
  if (n_partitions <= 0 || ncoils <= 0) return guarded([] { mrsim::fail("partitions and coils must be positive"); });
  const size_t np = rec ? (size_t)rec->impl->npts : 0, nn = rec ? (size_t)rec->impl->n * rec->impl->n : 0;
  return recon_call(rec, coil_samples, np * ncoils * n_partitions, out, nn * n_partitions,
                    [&](double2* i, double2* o) {
                      need(zsens, "zsens");
                      rec->impl->rings(i, (int)n_partitions, (int)ncoils, (int)ring, zsens, o);
                    });
}

// ---- 3D echo trains -------------------------------------------------------------------------------
int mrsim_kz_order(int64_t nz, int32_t order, int64_t* out) {
  return guarded([&] {
    if (nz <= 0) mrsim::fail("nz must be positive");
    need(out, "out");
    auto v = mrsim::kz_order((int)nz, order);
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
  });
}

int mrsim_grase_lines(const mrsim_echo_train* train, const mrsim_grase_readout* ro, int64_t ny, int64_t nz,
                      int64_t* shot, int64_t* echo, double* t_ms, double* trf_ms, int8_t* polarity, int64_t* e_c,
                      int64_t* n_shots) {
  return guarded([&] {
    need(train, "train");
    need(ro, "readout");
    if (ny <= 0 || nz <= 0) mrsim::fail("ny and nz must be positive");
    mrsim::Grase3dTable T = mrsim::grase_lines(*train, *ro, (int)ny, (int)nz);
    for (size_t i = 0; i < T.lines.size(); ++i) {
      if (shot) shot[i] = T.lines[i].shot;
      if (echo) echo[i] = T.lines[i].echo;
      if (t_ms) t_ms[i] = T.lines[i].t_ms;
      if (trf_ms) trf_ms[i] = T.lines[i].trf_ms;
      if (polarity) polarity[i] = T.lines[i].polarity;
    }
    if (e_c) *e_c = T.e_c;
    if (n_shots) *n_shots = T.n_shots;
  });
}

static void check_3d_input(const mrsim_acquisition_3d_input* in, const mrsim_acquisition* acq,
                           const mrsim_echo_train* train, const mrsim_grase_readout* ro) {
  need(in, "input");
  need(acq, "acq");
  need(train, "train");
  need(ro, "readout");
  if (in->n_volumes < 0) mrsim::fail("negative volume count");
  if (in->ncomp > 0 && !in->images) mrsim::fail("compartment image is not on the simulation grid");
  for (int64_t c = 0; c < in->ncomp; ++c)
    if (!in->images[c]) mrsim::fail("compartment image is not on the simulation grid");
}

int mrsim_simulate_acquisition_3d(mrsim_context* ctx, const mrsim_acquisition_3d_input* in,
                                  const mrsim_acquisition* acq, const mrsim_echo_train* train,
                                  const mrsim_grase_readout* ro, uint64_t seed, float* mag, float* phase) {
  return on_ctx(ctx, [&] {
    check_3d_input(in, acq, train, ro);
    need(mag, "mag");
    need(phase, "phase");
    mrsim::grase_acquire(ctx, *in, *acq, *train, *ro, seed, mag, phase);
  });
}

int mrsim_kspace_3d_observed(mrsim_context* ctx, const mrsim_acquisition_3d_input* in, const mrsim_acquisition* acq,
                             const mrsim_echo_train* train, const mrsim_grase_readout* ro, int64_t g, float* out) {
  return on_ctx(ctx, [&] {
    check_3d_input(in, acq, train, ro);
    need(out, "out");
    mrsim::grase_observed(ctx, *in, *acq, *train, *ro, (int)g, out);
  });
}

int mrsim_spiral_lines(const mrsim_echo_train* train, const mrsim_spiral_readout* ro, int64_t nx, int64_t ny,
                       int64_t nz, uint8_t* acquired, int64_t* echo, int64_t* kz_segment, int64_t* band_start,
                       int64_t* e_c, int64_t* n_shots, int64_t* samples_per_interleaf) {
  return guarded([&] {
    need(train, "train");
    need(ro, "readout");
    if (nx <= 0 || ny <= 0 || nz <= 0) mrsim::fail("empty matrix");
    mrsim::Spiral3dTable T = mrsim::spiral_lines(*train, *ro, (int)nx, (int)ny, (int)nz);
    for (int p = 0; p < (int)nz; ++p) {
      if (acquired) acquired[p] = T.acquired[p];
      if (echo) echo[p] = T.echo[p];
      if (kz_segment) kz_segment[p] = T.kz_segment[p];
    }
    if (band_start) *band_start = T.band_start;
    if (e_c) *e_c = T.e_c;
    if (n_shots) *n_shots = T.n_shots;
    if (samples_per_interleaf) *samples_per_interleaf = (int64_t)T.traj.tau_ms.size();
  });
}

static void check_spiral_3d(const mrsim_acquisition_3d_input* in, const mrsim_acquisition* acq,
                            const mrsim_echo_train* train, const mrsim_spiral_readout* ro) {
  need(in, "input");
  need(acq, "acq");
  need(train, "train");
  need(ro, "readout");
  if (in->n_volumes < 0) mrsim::fail("negative volume count");
  if (in->ncomp > 0 && !in->images) mrsim::fail("compartment image is not on the simulation grid");
  for (int64_t c = 0; c < in->ncomp; ++c)
    if (!in->images[c]) mrsim::fail("compartment image is not on the simulation grid");
}

int mrsim_simulate_acquisition_3d_spiral(mrsim_context* ctx, const mrsim_acquisition_3d_input* in,
                                         const mrsim_acquisition* acq, const mrsim_echo_train* train,
                                         const mrsim_spiral_readout* ro, const mrsim_kz_options* kz_opts,
                                         uint64_t seed, float* mag, float* phase) {
  return on_ctx(ctx, [&] {
    check_spiral_3d(in, acq, train, ro);
    need(mag, "mag");
    need(phase, "phase");
    mrsim::spiral3d_acquire(ctx, *in, *acq, *train, *ro, kz_opts, seed, mag, phase);
  });
}

int mrsim_spiral_samples_3d(mrsim_context* ctx, const mrsim_acquisition_3d_input* in, const mrsim_acquisition* acq,
                            const mrsim_echo_train* train, const mrsim_spiral_readout* ro,
                            const mrsim_kz_options* kz_opts, int64_t g, float* out) {
  return on_ctx(ctx, [&] {
    check_spiral_3d(in, acq, train, ro);
    need(out, "out");
    mrsim::spiral3d_samples(ctx, *in, *acq, *train, *ro, kz_opts, (int)g, out);
  });
}

int mrsim_ge3d_lines(const mrsim_excitation_train* train, const mrsim_ge3d_readout* ro, int64_t ny, int64_t nz,
                     int64_t* shot, int64_t* excitation, double* t_ms, int8_t* polarity, int64_t* n_shots,
                     int64_t* n_exc, int64_t* e_c) {
  return guarded([&] {
    need(train, "train");
    need(ro, "readout");
    if (ny <= 0 || nz <= 0) mrsim::fail("ny and nz must be positive");
    mrsim::Ge3dTable T = mrsim::ge3d_lines(*train, *ro, (int)ny, (int)nz);
    for (size_t i = 0; i < T.lines.size(); ++i) {
      if (shot) shot[i] = T.lines[i].shot;
      if (excitation) excitation[i] = T.lines[i].excitation;
      if (t_ms) t_ms[i] = T.lines[i].t_ms;
      if (polarity) polarity[i] = T.lines[i].polarity;
    }
    if (n_shots) *n_shots = T.n_shots;
    if (n_exc) *n_exc = T.n_exc;
    if (e_c) *e_c = T.e_c;
  });
}

int mrsim_simulate_acquisition_3d_ge(mrsim_context* ctx, const mrsim_acquisition_ge_input* in,
                                     const mrsim_acquisition* acq, const mrsim_excitation_train* train,
                                     const mrsim_ge3d_readout* ro, uint64_t seed, float* const* mag,
                                     float* const* phase) {
  return on_ctx(ctx, [&] {
    need(in, "input");
    need(acq, "acq");
    need(train, "train");
    need(ro, "readout");
    if (in->n_volumes < 0) mrsim::fail("negative volume count");
    mrsim::ge_acquire(ctx, *in, *acq, *train, *ro, seed, mag, phase);
  });
}

int mrsim_nufft1(mrsim_context* ctx, int64_t n, int64_t k_lo, int64_t n_out, double tol, const double* pos,
                 int64_t npos, const double* weights, int64_t nw, double* out) {
  return on_ctx(ctx, [&] {
    if (npos < 0 || npos > ((int64_t)1 << 30) || nw <= 0 || nw > 4096) mrsim::fail("NUFFT point or vector count out of range");
    need(out, "out");
    if (npos > 0) {
      need(pos, "pos");
      need(weights, "weights");
    }
    mrsim::nufft1_host(ctx, (int)n, (int)k_lo, (int)n_out, tol, pos, (int)npos, weights, (int)nw, out);
  });
}

int mrsim_check_grase_timing(const mrsim_echo_train* train, const mrsim_grase_readout* ro, int64_t ny, int64_t nz,
                             double t_exc_ms, double tr_ms) {
  return guarded([&] {
    need(train, "train");
    need(ro, "readout");
    std::string e = mrsim::check_grase_timing(*train, mrsim::grase_lines(*train, *ro, (int)ny, (int)nz), t_exc_ms, tr_ms);
    if (!e.empty()) mrsim::fail(e);
  });
}

int mrsim_check_ge3d_timing(const mrsim_excitation_train* train, const mrsim_ge3d_readout* ro, int64_t ny, int64_t nz,
                            double t_exc_ms, double tr_ms) {
  return guarded([&] {
    need(train, "train");
    need(ro, "readout");
    std::string e = mrsim::check_ge3d_timing(*train, mrsim::ge3d_lines(*train, *ro, (int)ny, (int)nz), t_exc_ms, tr_ms);
    if (!e.empty()) mrsim::fail(e);
  });
}

int mrsim_check_spiral_timing(const mrsim_echo_train* train, const mrsim_spiral_readout* ro, int64_t nx, int64_t ny,
                              int64_t nz, double t_exc_ms, double tr_ms, double* end_ms) {
  return guarded([&] {
    need(train, "train");
    need(ro, "readout");
    mrsim::spiral_lines(*train, *ro, (int)nx, (int)ny, (int)nz);  // the table's own checks first
    std::string e = mrsim::check_spiral_timing(*train, ro->readout_ms, t_exc_ms, tr_ms, end_ms);
    if (!e.empty()) mrsim::fail(e);
  });
}

double mrsim_esp_from_echo_time(double te_ms, int64_t e_c, const mrsim_grase_readout* ro, int64_t ny) {
  // `esp_from_echo_time` (readout.rs:286-288): (TE - t(ky = ny/2)) / e_c
  mrsim::GraseBlock b = mrsim::grase_block((int)ny, (int)ro->ky_segments, ro->t_line_ms, ro->reverse_phase != 0);
  return (te_ms - b.t_ms[b.t_ms.size() / 2]) / (double)e_c;
}

double mrsim_spiral_esp_from_echo_time(double te_ms, int64_t e_c) { return te_ms / (double)e_c; }  // readout.rs:702

int mrsim_spiral_segmentation(const mrsim_acquisition_3d_input* in, const mrsim_acquisition* acq,
                              const mrsim_echo_train* train, const mrsim_spiral_readout* ro, int64_t capacity,
                              mrsim_spiral_segmentation_row* rows, int64_t* count) {
  return guarded([&] {
    need(in, "input");
    need(acq, "acq");
    need(train, "train");
    need(ro, "readout");
    need(count, "count");
    auto v = mrsim::spiral_segmentation(*in, *acq, *train, *ro);
    *count = (int64_t)v.size();
    if (!rows) return;
    if (capacity < (int64_t)v.size()) mrsim::fail("row capacity below the segmentations");
    for (size_t i = 0; i < v.size(); ++i)
      rows[i] = mrsim_spiral_segmentation_row{v[i].z, v[i].voxel, v[i].l, v[i].m, v[i].b_sum, v[i].bound};
  });
}

// ---- spin history (spin_history.rs) --------------------------------------------------------------
int mrsim_spin_history_create(mrsim_context* ctx, const int64_t* src_dims, const double* src_v2w, const float* t1,
                              const float* weight, const uint8_t* cls, int64_t n_classes, const int64_t* slab_dims,
                              const double* slab_v2w, const mrsim_pulse* pulses, int64_t n_pulses,
                              mrsim_spin_history** out) {
  return on_ctx(ctx, [&] {
    need(out, "out");
    *out = nullptr;
    need(src_dims, "src_dims");
    need(src_v2w, "src_v2w");
    need(t1, "t1");
    need(weight, "weight");
    need(cls, "cls");
    need(slab_dims, "slab_dims");
    need(slab_v2w, "slab_v2w");
    if (n_pulses > 0) need(pulses, "pulses");
    std::unique_ptr<mrsim::SpinHistoryDev> h(mrsim::spin_history_create(
        ctx, src_dims, src_v2w, t1, weight, cls, n_classes, slab_dims, slab_v2w, pulses, n_pulses));
    *out = new mrsim_spin_history{h.release()};
  });
}

void mrsim_spin_history_destroy(mrsim_spin_history* h) {
  if (!h) return;
  {
    std::lock_guard<std::mutex> lk(h->impl->ctx->mu);
    cudaSetDevice(h->impl->ctx->device);
    cudaStreamSynchronize(h->impl->ctx->stream);  // the batch buffers may still be read
    delete h->impl;
  }
  delete h;
}

int mrsim_spin_history_n_tracked(mrsim_spin_history* h, int64_t* n) {
  return guarded([&] {
    need(h, "spin history");
    need(n, "n");
    *n = h->impl->nt;
  });
}

int mrsim_spin_history_prime(mrsim_spin_history* h, const double* times, const int64_t* slices,
                             const int64_t* offsets, int64_t n_shots, const double* transform) {
  if (!h) return guarded([] { need(nullptr, "spin history"); });
  return on_ctx(h->impl->ctx, [&] {
    if (n_shots <= 0) return;
    need(times, "times");
    need(offsets, "offsets");
    need(transform, "transform");
    std::vector<mrsim_spin_shot> shots((size_t)n_shots);
    for (int64_t s = 0; s < n_shots; ++s) {
      if (offsets[s + 1] < offsets[s]) mrsim::fail("offsets must not decrease");
      if (offsets[s + 1] > offsets[s]) need(slices, "slices");
      mrsim_spin_shot& S = shots[(size_t)s];
      S = mrsim_spin_shot{};
      S.t = times[s];
      std::memcpy(S.transform, transform, sizeof S.transform);
      S.slices = slices ? slices + offsets[s] : nullptr;
      S.n_slices = offsets[s + 1] - offsets[s];
      S.ref.kind = MRSIM_MZREF_NONE;
    }
    mrsim::spin_history_run(*h->impl, shots.data(), n_shots, nullptr);
    MRSIM_CUDA(cudaStreamSynchronize(h->impl->ctx->stream));
  });
}

int mrsim_spin_history_terms_size(mrsim_spin_history* h, const mrsim_spin_shot* shots, int64_t n_shots,
                                  int64_t* n_floats) {
  return guarded([&] {
    need(h, "spin history");
    need(n_floats, "n_floats");
    if (n_shots > 0) need(shots, "shots");
    *n_floats = mrsim::spin_history_terms_size(*h->impl, shots, n_shots);
  });
}

int mrsim_spin_history_excite(mrsim_spin_history* h, const mrsim_spin_shot* shots, int64_t n_shots, float* terms) {
  if (!h) return guarded([] { need(nullptr, "spin history"); });
  return on_ctx(h->impl->ctx, [&] {
    if (n_shots <= 0) return;
    need(shots, "shots");
    const int64_t nf = mrsim::spin_history_terms_size(*h->impl, shots, n_shots);
    if (nf > 0) need(terms, "terms");
    float* d = (float*)h->impl->out_b.get((size_t)std::max<int64_t>(nf, 1) * 4);
    mrsim::spin_history_run(*h->impl, shots, n_shots, d);
    cudaStream_t st = h->impl->ctx->stream;
    if (nf > 0) MRSIM_CUDA(cudaMemcpyAsync(terms, d, (size_t)nf * 4, cudaMemcpyDeviceToHost, st));
    MRSIM_CUDA(cudaStreamSynchronize(st));
    (void)mrsim::spin_history_merges(*h->impl);  // reports a kernel's error status
  });
}

int mrsim_spin_history_excite_device(mrsim_spin_history* h, const mrsim_spin_shot* shots, int64_t n_shots,
                                     float* terms) {
  if (!h) return guarded([] { need(nullptr, "spin history"); });
  return on_ctx(h->impl->ctx, [&] {
    if (n_shots <= 0) return;
    need(shots, "shots");
    mrsim::spin_history_run(*h->impl, shots, n_shots, terms);
  });
}

int mrsim_spin_history_merges(mrsim_spin_history* h, uint64_t* merges) {
  if (!h) return guarded([] { need(nullptr, "spin history"); });
  return on_ctx(h->impl->ctx, [&] {
    need(merges, "merges");
    *merges = mrsim::spin_history_merges(*h->impl);
  });
}

}  // extern "C"
#pragma GCC visibility pop
