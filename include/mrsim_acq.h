/*
 * mrsim_acq.h — C ABI of the B200 k-space acquisition library (libmrsim_acq_cuda.so).
 *
 * The library is a drop-in for the k-space path of the Rust crate `mrsim-acq`: the 2D EPI
 * per-slice exact-DFT forward and its adjoint, GRAPPA calibration and apply, window, inverse DFT,
 * Roemer combine and series drivers; the 3D GRASE, gradient-echo and stack-of-spirals trains; and
 * the spiral pieces (NUFFT pair, certified time segmentation, spiral forwards and
 * reconstruction, trajectory and EPG).  Every entry point cites the reference item it replaces as
 * `file:line` within the reference crate.  A Rust shim behind a `gpu` cargo feature binds these
 * symbols one for one in an `extern "C"` block.
 *
 * Conventions
 *  - Plain pointers and sizes; no C++ or torch types cross the boundary.
 *  - Every function returns an `int` status: 0 = success, non-zero = failure.  On failure
 *    `mrsim_last_error()` returns the message (thread-local), worded like the reference's panic
 *    message for the same input, so the Rust shim can `panic!("{}", msg)` and keep
 *    `#[should_panic]` behaviour.
 *  - Entry points named `*_host` / the series and slice entry points take HOST pointers in the
 *    reference's layouts and copy to and from the device inside the call.  Entry points taking a
 *    `mrsim_epi_batch` take DEVICE pointers and run asynchronously on the context's stream.
 *  - Layouts are the reference's: sim-grid planes `x + snx*y`, volumes `x + snx*(y + sny*z)`,
 *    series images `vox*n_volumes + g`, k-space `kx + nx*ky`, complex values as (re, im) pairs.
 *  - Input pointers are never retained after a call returns.
 */
#ifndef MRSIM_ACQ_H
#define MRSIM_ACQ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MRSIM_ABI_VERSION 1

/* ---- status codes ---------------------------------------------------------------------- */
enum {
  MRSIM_OK = 0,
  MRSIM_ERR_INVALID = 1,   /* an input failed validation (the reference panics or returns Err) */
  MRSIM_ERR_CUDA = 2,      /* a CUDA runtime call failed                                      */
  MRSIM_ERR_NOMEM = 3,     /* device or host allocation failed                                */
  MRSIM_ERR_DEVICE = 4,    /* a kernel reported an error status (bounded wait ran out, ...)   */
  MRSIM_ERR_NOGPU = 5      /* no CUDA device: the library has no CPU fallback                 */
};

/* ---- acquisition parameters: `Acquisition` kspace.rs:166-197, Default kspace.rs:239-267 --- */
enum { MRSIM_PF_FIBERFOX = 0, MRSIM_PF_CONTIGUOUS = 1, MRSIM_PF_SCANNER = 2 }; /* kspace.rs:85 */
enum { MRSIM_WINDOW_NONE = 0, MRSIM_WINDOW_TUKEY = 1, MRSIM_WINDOW_HANN = 2,
       MRSIM_WINDOW_FERMI = 3 };                                               /* kspace.rs:126 */
enum { MRSIM_ECHO_SPIN = 0, MRSIM_ECHO_GRADIENT = 1 };                        /* kspace.rs:207 */

typedef struct mrsim_acquisition {
  double t_line;          /* ms per PE line                                              */
  double t_echo;          /* ms                                                          */
  double t_inhom;         /* ms, T2' used when no per-compartment T2' is given           */
  double signal_scale;
  int32_t reverse_phase;
  int32_t do_distortions;
  int32_t do_relaxation;
  int32_t pf_mode;        /* MRSIM_PF_*                                                  */
  double noise_variance;
  double partial_fourier;
  double ghost_offset;
  double eddy_strength;
  double eddy_quad;
  double eddy_phase;
  double eddy_tau;
  int64_t n_spikes;
  double spike_amplitude;
  int32_t window_kind;    /* MRSIM_WINDOW_*                                              */
  int32_t echo;           /* MRSIM_ECHO_*                                                */
  double window_a;        /* Tukey: alpha; Fermi: radius                                 */
  double window_b;        /* Fermi: width                                                */
  int64_t n_coils;
  int64_t accel;
  int64_t acs_lines;
  uint64_t seed;
} mrsim_acquisition;

/* Fill `acq` with `Acquisition::default()` (kspace.rs:239-267). */
int mrsim_acquisition_default(mrsim_acquisition* acq);

/* ---- per-compartment T2 / T2': `T2Slice` kspace.rs:380-386, `T2Volume` :389-393 ---------- */
typedef struct mrsim_t2 {
  const float* map;       /* NULL = uniform; else a map on the sim slice (or volume)     */
  float value;            /* the uniform value (ms) when map == NULL                     */
  int32_t is_map;
} mrsim_t2;

/* ---- one slice's input: `SliceInput` kspace.rs:458-496 ---------------------------------- */
typedef struct mrsim_slice_input {
  const float* const* compartments; /* ncomp planes, each snx*sny                        */
  int64_t ncomp;
  const mrsim_t2* t2;               /* ncomp                                              */
  const mrsim_t2* t_inhom;          /* ncomp, or NULL = Acquisition::t_inhom              */
  const float* fmap;                /* Hz, snx*sny                                        */
  const double* phase0;             /* radians, snx*sny, or NULL                          */
  int64_t sim[2];                   /* [snx, sny]                                         */
  int64_t acq_matrix[2];            /* [nx, ny]                                           */
  int64_t z;
  int64_t nz;
  int32_t has_eddy_drive;
  int32_t has_prep_drive;
  double eddy_drive[3];
  double prep_magnitude;
  double prep_direction[3];
  uint64_t slice_seed;
} mrsim_slice_input;

/* ---- object phase model: `PhaseModel` phase.rs:130-205 ----------------------------------- */
typedef struct mrsim_phase_model {
  double global;
  double background[10];  /* 1, x, y, z, x^2, y^2, z^2, xy, xz, yz (phase.rs:52)          */
  int32_t has_prep;       /* PrepPhase present                                          */
  int32_t reserved;
  double c_q;
  double sigma_dx;
  double sigma_rot;
} mrsim_phase_model;

/* `PhaseModel::hbcd_like()` phase.rs:187 and `PhaseModel::none()` phase.rs:197. */
int mrsim_phase_model_hbcd_like(mrsim_phase_model* out);
int mrsim_phase_model_none(mrsim_phase_model* out);

/* ---- series input / options / output: kspace.rs:1720-1797 -------------------------------- */
typedef struct mrsim_acquisition_input {
  int64_t sim_dims[3];              /* [snx, sny, nz]                                     */
  int64_t acq_dims[3];              /* [nx, ny, nz]                                       */
  int64_t n_volumes;
  int64_t ncomp;
  const float* const* images;       /* ncomp arrays, each snx*sny*nz*n_volumes, vox*nv+g  */
  const mrsim_t2* t2;               /* ncomp; maps are whole sim volumes                  */
  const float* fmap;                /* snx*sny*nz                                         */
  const mrsim_t2* t_inhom;          /* ncomp or NULL                                      */
  const int32_t* eddy_drive_set;    /* n_volumes flags (Some/None), or NULL = all None    */
  const double* eddy_drive;         /* n_volumes*3                                        */
  const int32_t* prep_drive_set;    /* n_volumes flags, or NULL = all None                */
  const double* prep_drive;         /* n_volumes*4: magnitude, direction[3]               */
  const mrsim_phase_model* phase;
  uint64_t seed;
  const float* noise_sigma;         /* nx*ny*nz or NULL                                   */
} mrsim_acquisition_input;

typedef void (*mrsim_progress_fn)(int64_t done, int64_t total, void* user);

typedef struct mrsim_acquisition_options {
  const int64_t* slice_z;           /* nz entries, or NULL = 0..nz                        */
  int64_t nz_full;                  /* <= 0: acq_dims[2]                                  */
  const int64_t* kspace_slices;     /* local slice indices to capture, or NULL            */
  int64_t n_kspace_slices;
  int32_t capture_acquired;
  int32_t capture_reconstructed;
  int32_t capture_coil_images;
  int32_t has_grappa_calibration;
  const double* t_echo_per_volume;  /* n_volumes, or NULL                                 */
  mrsim_progress_fn progress;       /* called on the calling thread, or NULL              */
  void* progress_user;
  const float* const* grappa_calibration_images; /* ncomp arrays of snx*sny*nz           */
  uint64_t grappa_calibration_seed;
} mrsim_acquisition_options;

typedef struct mrsim_acquisition_output {
  float* re;                        /* nx*ny*nz*n_volumes, (vox*nv + g)                   */
  float* im;
  /* k-space capture (`KspaceCapture` kspace.rs:1767-1788); each may be NULL when not asked. */
  uint8_t* mask;                    /* ny*nx                                              */
  float* sensitivities;             /* n_coils*ny*nx                                      */
  float* acquired;                  /* [vol, slice, coil, ky, kx] (re, im)                */
  float* reconstructed;             /* [vol, slice, coil, ky, kx] (re, im)                */
  float* coil_images;               /* [vol, slice, coil, y, x] (re, im)                  */
  float* combined;                  /* [vol, slice, y, x] (re, im)                        */
} mrsim_acquisition_output;

/* ---- context --------------------------------------------------------------------------- */
typedef struct mrsim_context mrsim_context;

/* One CUDA stream, a device workspace and a plan cache on `device`.  Thread-safe per context:
 * calls on one context are serialised by an internal lock. */
int mrsim_context_create(int device, mrsim_context** out);
int mrsim_context_destroy(mrsim_context* ctx);
/* The context's CUDA stream (a `cudaStream_t`), for callers that enqueue their own work. */
void* mrsim_context_stream(mrsim_context* ctx);
int mrsim_context_synchronize(mrsim_context* ctx);
const char* mrsim_last_error(void);
int mrsim_abi_version(void);

/* ---- host tables, bit-exact with the reference ------------------------------------------ */
/* `sampling_mask` kspace.rs:546-588; mask[kx + nx*ky] = 0/1. */
int mrsim_sampling_mask(int64_t nx, int64_t ny, const mrsim_acquisition* acq, uint8_t* mask);
/* `pf_skipped_lines` kspace.rs:110-116. */
int64_t mrsim_pf_skipped_lines(int64_t ny, const mrsim_acquisition* acq);
/* `LineTiming::for_acquisition` kspace.rs:310-325 (+ `line_times` :271-284). */
int mrsim_line_timing(const mrsim_acquisition* acq, int64_t nx, int64_t ny,
                      double* t_ms, double* trf_ms, double* tread_ms, int8_t* polarity);
/* `validate_acquisition_timing` kspace.rs:411-431: MRSIM_ERR_INVALID with the message. */
int mrsim_validate_acquisition_timing(const mrsim_acquisition* acq, int64_t nx, int64_t ny);
/* `epi_timing` kspace.rs:353-361: order[ny] (acquisition order of ky lines). */
int mrsim_epi_order(const mrsim_acquisition* acq, int64_t nx, int64_t ny, int64_t* order);

/* ---- per-slice entry points (host buffers) ---------------------------------------------- */
/* `build_coil_kspace_timed` kspace.rs:607-1042 for every coil of one slice, timing from
 * `LineTiming::for_acquisition` unless t_ms.. are given (each ny long, or all NULL); log_amp is
 * the 3D voxel-mode log-amplitude (snx*sny) or NULL.  out = n_coils*nx*ny (re, im) f64. */
int mrsim_build_coil_kspaces(mrsim_context* ctx, const mrsim_slice_input* inp,
                             const mrsim_acquisition* acq, const double* t_ms,
                             const double* trf_ms, const double* tread_ms,
                             const int8_t* polarity, const double* log_amp, double* out);

/* `simulate_slice` kspace.rs:1229-1235: GRAPPA (a lone slice fits its kernel on a reference scan
 * of itself), window, inverse DFT, Roemer combine.  out = nx*ny (re, im) f32 pairs. */
int mrsim_simulate_slice(mrsim_context* ctx, const mrsim_slice_input* inp,
                         const mrsim_acquisition* acq, float* out);
/* `simulate_slice_full` kspace.rs:1241-1284 with the `SliceCapture` intermediates (kspace.rs:1184-
 * 1224); combined = nx*ny (re, im) f32; acquired, reconstructed, coil_images = n_coils*nx*ny (re,
 * im) f32; sensitivities = n_coils*nx*ny f32; mask = nx*ny bytes.  Captures may be NULL. */
int mrsim_simulate_slice_full(mrsim_context* ctx, const mrsim_slice_input* inp,
                              const mrsim_acquisition* acq, float* combined, float* acquired,
                              float* reconstructed, float* coil_images, float* sensitivities,
                              uint8_t* mask);
/* `simulate_slice_kspace` kspace.rs:1144-1149: coil 0's acquired k-space, nx*ny (re, im) f64. */
int mrsim_simulate_slice_kspace(mrsim_context* ctx, const mrsim_slice_input* inp,
                                const mrsim_acquisition* acq, double* out);

/* ---- series entry points (host buffers) ------------------------------------------------- */
/* `simulate_acquisition_complex` kspace.rs:1803-1808. */
int mrsim_simulate_acquisition_complex(mrsim_context* ctx, const mrsim_acquisition_input* inp,
                                       const mrsim_acquisition* acq,
                                       const mrsim_acquisition_options* opts,
                                       mrsim_acquisition_output* out);
/* `simulate_acquisition_oversampled` kspace.rs:1687-1714: magnitude and phase (f32). */
int mrsim_simulate_acquisition_oversampled(mrsim_context* ctx, const mrsim_acquisition_input* inp,
                                           const mrsim_acquisition* acq, float* mag, float* phase);
/* `simulate_acquisition_echoes` kspace.rs:2152-2174: images_per_echo[e] holds echo e's ncomp
 * image arrays; grappa_calibration_images[e] (ncomp single volumes) and _seeds[e] are each echo's
 * `GrappaCalibration` or NULL; mag/phase are n_echoes arrays of nx*ny*nz*n_volumes. */
int mrsim_simulate_acquisition_echoes(mrsim_context* ctx, const mrsim_acquisition_input* inp,
                                      const float* const* const* images_per_echo,
                                      const mrsim_acquisition* acq, const double* echo_times_ms,
                                      int64_t n_echoes,
                                      const float* const* const* grappa_calibration_images,
                                      const uint64_t* grappa_calibration_seeds, float* const* mag,
                                      float* const* phase);

/* No counterpart in the reference: a forward that allocates no device memory.  For callers that
 * may not call cudaMalloc while they run (a host whose device memory is all in its own pool or
 * arena, a pipeline that pre-allocates at start-up so no call can stall or fail on allocation).
 * Computes what mrsim_build_coil_kspaces computes with noise_variance = 0 and n_spikes = 0, for
 * uniform T2/T2' (no maps, no log-amplitude), into `kspace` (DEVICE, n_coils*ny*nx (re, im) f32).
 * `inp` is a host struct whose data pointers are DEVICE pointers: the compartment planes
 * contiguous (plane c at compartments[0] + c*snx*sny), fmap, and phase0 (f64) or NULL.  `stream`
 * is a cudaStream_t (NULL: the legacy default stream) of the current device; the call returns
 * when the output is complete.  Intermediates live in static device arrays of ~7.8 MiB held by
 * every GPU that loads the library until exit; limits: n_coils*acquired_lines*snx <= 524288,
 * snx*sny <= 262144, snx*nx <= 65536, n_coils*max(snx,sny) <= 32768, acquired lines <= 1024 —
 * larger inputs fail with MRSIM_ERR_INVALID, and so does a data pointer that is not device (or
 * managed) memory of the current device.  The first call on a device, and the first after that
 * device's context changed (e.g. after cudaDeviceReset), looks up the arrays' addresses
 * (cudaGetSymbolAddress, that device current); make the first call before any stream capture
 * begins.  Each call waits for `stream` before it returns.  Calls share the arrays: calls that
 * overlap on the GPU race and must be serialised. */
int mrsim_build_coil_kspaces_noalloc(const mrsim_slice_input* inp, const mrsim_acquisition* acq,
                                     void* stream, float* kspace);

/* ---- the batched forward / adjoint operator of a 2D EPI series --------------------------- */
/*
 * The series' forward model `build_coil_kspace_timed` (kspace.rs:607-1042, without spikes and
 * noise) over every volume, slice, echo and coil in one batch, and its adjoint.  A unit is one
 * slice of one volume; its line list holds every echo's acquired lines, so the echoes of a
 * volume share one pass over its voxels and the adjoint sums over them.  For each unit
 *   k_q[e][ky][kx] = (1/nvox) sum_{x,y} tw(kx,x) amp_q(x,y) e^{i2pi theta(x,y,ky,e)}
 *                    sum_c rel_c(x,y,ky,e) m_c(x,y)
 * and the adjoint applied to the k-space buffer r writes
 *   comp_grad_c(x,y) = (A^H r)_c(x,y)                      (complex, per compartment)
 *   fmap_grad(x,y)   = dL/d fmap(x,y)    for L = sum |r|^2 with r = A m - d (Hz^-1 units)
 *   r2_grad_c(x,y)   = dL/d R2_c(x,y),   R2 = 1/T2 in 1/ms.
 * The reference has no adjoint; its oracle is the FP64 transpose plus finite differences.
 *
 * Device layouts (all owned by the operator; see mrsim_epi_operator_buffers):
 *   images    [g][z][c][sny][snx] f32            fmap  [z][sny][snx] f32
 *   kspace    [g][z][coil][echo][ny][nx] complex (re, im) f32; un-acquired rows stay zero
 *   comp_grad [g][z][c][sny][snx] complex        fmap_grad [g][z][sny][snx]
 *   r2_grad   [g][z][c][sny][snx]
 * The images of every echo are the same (callers that decay them per echo use one operator per
 * echo).  `in->images` may be NULL at creation; `in->fmap`, T2/T2' maps, drives and the phase
 * model are read at creation.  `grads` bit 0 = fmap_grad, bit 1 = r2_grad.
 */
typedef struct mrsim_epi_operator mrsim_epi_operator;

int mrsim_epi_operator_create(mrsim_context* ctx, const mrsim_acquisition_input* in,
                              const mrsim_acquisition* acq, const double* echo_times_ms,
                              int64_t n_echoes, const int64_t* slice_z, int64_t nz_full,
                              int32_t grads, mrsim_epi_operator** out);
int mrsim_epi_operator_destroy(mrsim_epi_operator* op);
/* Acquired k-space samples one forward produces (every coil, echo, slice and volume). */
int64_t mrsim_epi_operator_samples(const mrsim_epi_operator* op);
/* Device pointers of the operator's buffers (any argument may be NULL). */
int mrsim_epi_operator_buffers(mrsim_epi_operator* op, float** images, float** kspace,
                               float** comp_grad, float** fmap_grad, float** r2_grad);
/* Copy host images (reference layout: ncomp arrays of vox*n_volumes + g) to the device. */
int mrsim_epi_operator_upload_images(mrsim_epi_operator* op, const float* const* images);
/* Replace the fieldmap (Hz, [z][sny][snx] f32 host array, the layout of `in->fmap`) for every
 * forward and adjoint queued after the call, which returns once the copy is done: the update
 * step of a fieldmap fit by gradient descent on fmap_grad.  No reference counterpart (the
 * reference takes its fieldmap per simulation call and has no adjoint). */
int mrsim_epi_operator_set_fieldmap(mrsim_epi_operator* op, const float* fmap);
/* Asynchronous on the context stream: statics + forward into the k-space buffer. */
int mrsim_epi_operator_forward(mrsim_epi_operator* op);
/* Asynchronous: adjoint / VJP of the k-space buffer's current contents. */
int mrsim_epi_operator_adjoint(mrsim_epi_operator* op);
/* One stage of the pair, asynchronous, for per-kernel timing: 0 statics (static phase),
 * 1 forward y-stage, 2 forward x-stage, 3 adjoint x-stage, 4 adjoint y-stage. */
int mrsim_epi_operator_stage(mrsim_epi_operator* op, int32_t stage);
/* FP32 FMA throughput of the context's device (TFLOP/s, a register-resident FMA loop): the
 * denominator of the exact path's roofline, measured because no table of peaks carries it. */
int mrsim_probe_fp32_tflops(mrsim_context* ctx, double* tflops);
/* Synchronous, host buffers: the adjoint / VJP of the given k-space (residual) r, layout of the
 * k-space buffer, (re, im) f32.  Any output may be NULL. */
int mrsim_epi_operator_adjoint_host(mrsim_epi_operator* op, const float* kspace, float* comp_grad,
                                    float* fmap_grad, float* r2_grad);
/* Synchronous, host buffers: upload images, forward, copy k-space to the host, adjoint of that
 * k-space (the residual of zero data), copy the gradients to the host.  Any output may be NULL.
 * Computed in groups of slices (of volumes for a single slice) whose images upload, and whose
 * results copy back, while other groups compute (page-locked host buffers let the copies overlap). */
int mrsim_epi_operator_apply_host(mrsim_epi_operator* op, const float* const* images,
                                  float* kspace, float* comp_grad, float* fmap_grad,
                                  float* r2_grad);
/* The time-segmented y-stages of the pair (a tensor-core form of the exact DFT; no
 * reference counterpart: the reference segments only the spiral forward, `tseg::plan`
 * tseg.rs:230-289 via spiral.rs:141-201).  precision 0 restores the exact per-line phasors;
 * 1 selects contractions in split f16 (hi + lo operands, three products, FP32 accumulation),
 * 2 in split bf16.  The lines of each echo (and side of the spin echo) share a segmentation of
 * the fieldmap phase and the relaxation certified by the reference's planner to 1e-7, so the
 * y-stage becomes dense complex contractions on the tensor cores (tcgen05, TMEM accumulators,
 * TMA-loaded constant tables).  Needs uniform T2 / T2', no eddy-current polynomial, at most 4
 * compartments, sny a multiple of 8, and grads = 0 (the complex-image adjoint only); otherwise
 * MRSIM_ERR_INVALID.  A fieldmap set later outside the certified range rebuilds the tables. */
int mrsim_epi_operator_set_segmented(mrsim_epi_operator* op, int32_t precision);
/* The segmentation in use: groups, per-group segment counts L (max_groups entries) and
 * certified bounds, and the tensor-pipe FLOP of one forward and one adjoint pass (three split
 * products per complex MAC pair).  *n_groups = 0 when the exact path is selected. */
int mrsim_epi_operator_segmentation(const mrsim_epi_operator* op, int32_t* n_groups, int32_t* seg_l,
                                    double* bound, int32_t max_groups, double* flops_forward,
                                    double* flops_adjoint);
/* The autotuner (no reference counterpart): times the plan's tunables on the operator's first
 * units with device events — coil classes on/off, the x-stage as FFTs or as the DFT GEMM, the
 * fixed-coil y-adjoint's rows per thread (4 or 2) and, with flags bit 0, the segmented path in
 * split f16 / bf16 — keeps the fastest, and records it in the text file cache_path (one line per
 * operator shape; NULL: no cache).  A shape found in the cache takes its recorded choice without
 * timing.  The choice is written to `choice` (NUL-terminated, capacity choice_cap) and the timed
 * forward + adjoint of the timed units to *ms (0 when taken from the cache). */
int mrsim_epi_operator_tune(mrsim_epi_operator* op, const char* cache_path, int32_t flags, char* choice,
                            int64_t choice_cap, double* ms);
/* 0, or the code of a wait inside the segmented kernels that gave up (synchronises the stream). */
int mrsim_epi_operator_segmented_status(mrsim_epi_operator* op, int32_t* code);
/* As mrsim_epi_operator_apply_host, with the k-space in the compact layout
 * [g][z][coil][echo][acquired row][kx]: only the acquired rows, k-space row first + step * i of
 * mrsim_epi_operator_acquired_rows, no zero-filled rows (the host writes only what crosses the
 * link).  New API, no reference counterpart: the reference-compatible series entries keep the
 * zero-filled layout of `KspaceCapture` (kspace.rs:1767-1797).  MRSIM_ERR_INVALID when the
 * acquired rows of the echoes are not one uniform stride. */
int mrsim_epi_operator_apply_host_compact(mrsim_epi_operator* op, const float* const* images,
                                          float* kspace_rows, float* comp_grad, float* fmap_grad,
                                          float* r2_grad);
/* The acquired k-space rows of every echo as first + step * i, i < count (count 0: irregular). */
int mrsim_epi_operator_acquired_rows(const mrsim_epi_operator* op, int32_t* first, int32_t* step,
                                     int32_t* count);
/* Bytes a host-buffer call moves with the outputs of `outputs` (bit 0 k-space, 1 comp_grad,
 * 2 fmap_grad, 3 r2_grad): the images up, the acquired k-space rows and the requested gradients
 * down. */
int mrsim_epi_operator_host_bytes_for(const mrsim_epi_operator* op, int32_t outputs,
                                      int64_t* upload_bytes, int64_t* download_bytes);
/* Bytes one mrsim_epi_operator_apply_host call moves between host and device with every input
 * and output given: the images up; the acquired k-space rows (the other rows are zero-filled on
 * the host when the acquired rows form a uniform stride, else every row) and the gradients down. */
int mrsim_epi_operator_host_bytes(const mrsim_epi_operator* op, int64_t* upload_bytes,
                                  int64_t* download_bytes);

/* ---- a batch of series of different geometries --------------------------------------------- */
/* No reference counterpart (the reference runs one series per call): n_series series, each its
 * own geometry (matrix, grid, slice count; the same acquisition and echoes), as one plan, so each
 * stage of a forward or adjoint is one launch over every unit (slice of a volume) of every series,
 * with each unit's own descriptor.  Each series keeps its own buffers in the layouts of
 * mrsim_epi_operator; `grads` as there. */
typedef struct mrsim_epi_batch mrsim_epi_batch;
int mrsim_epi_batch_create(mrsim_context* ctx, int32_t n_series, const mrsim_acquisition_input* const* inputs,
                           const mrsim_acquisition* acq, const double* echo_times_ms, int64_t n_echoes,
                           int32_t grads, mrsim_epi_batch** out);
int mrsim_epi_batch_destroy(mrsim_epi_batch* b);
/* Acquired k-space samples of one forward over every series. */
int64_t mrsim_epi_batch_samples(const mrsim_epi_batch* b);
/* Asynchronous on the context stream: statics + forward of every series; adjoint of every series'
 * k-space buffer. */
int mrsim_epi_batch_forward(mrsim_epi_batch* b);
int mrsim_epi_batch_adjoint(mrsim_epi_batch* b);
/* Synchronous: series i's k-space and complex-image adjoint to host buffers (layouts of
 * mrsim_epi_operator; either may be NULL). */
int mrsim_epi_batch_download(mrsim_epi_batch* b, int32_t series, float* kspace, float* comp_grad);

/* ---- image motion before the forward (motion.rs) -------------------------------------------- */
/* A pose is 6 doubles: rotation (degrees about x, y, z; R = Rz Ry Rx) then translation (mm),
 * `Pose` (motion.rs:43-47).  v2w is the grid's voxel-to-world affine, row-major 4x4.  The
 * resampling backward-maps every output voxel in FP64 in the reference's operation order and
 * samples the source trilinearly (edge voxels extend half a voxel, zero beyond): the results are
 * the reference's bit for bit. */
/* `resample_by_pose` motion.rs:430-460: one volume (x + nx*(y + ny*z)) into `out`. */
int mrsim_resample_by_pose(mrsim_context* ctx, const float* src, const int64_t* dims, const double* v2w,
                           const double* pose, float* out);
/* `apply_motion` motion.rs:466-482: images[c][vox*n_volumes + g] moved in place by poses[g]
 * (n_volumes x 6 doubles). */
int mrsim_apply_motion(mrsim_context* ctx, float* const* images, int64_t ncomp, const int64_t* dims,
                       int64_t n_volumes, const double* v2w, const double* poses);

enum { MRSIM_DROPOUT_UNIFORM = 0, MRSIM_DROPOUT_SCALED = 1, MRSIM_DROPOUT_SCALED_TO = 2 };
/* `DropoutLaw` (motion.rs:625-662): Uniform 1 - severity; Scaled 1 - severity (drive/drive_max),
 * drive < floor exempt; ScaledTo the same with the given max. */
typedef struct mrsim_dropout_law {
  int32_t kind;
  const double* drive;
  int64_t n_drive;
  double floor;
  double max;
} mrsim_dropout_law;
/* `MotionEvent` (motion.rs:608-615). */
typedef struct mrsim_motion_event {
  int64_t volume;
  int64_t shot;
  float severity;
  double jump_mm[3];
  double jump_deg[3];
} mrsim_motion_event;
/* `DroppedShot` (motion.rs:618-624): slices in full-FOV indices (at most 64). */
typedef struct mrsim_dropped_shot {
  int64_t volume;
  int64_t shot;
  float attenuation;
  int64_t n_slices;
  int64_t slices[64];
} mrsim_dropped_shot;
/* `apply_multiband_motion_slab` motion.rs:686-772 (slice_z NULL and nz_full 0: the whole volume,
 * `apply_multiband_motion` motion.rs:666-680): within-volume shot motion and dropout of
 * images[c][vox*n_volumes + g] in place; the dropped shots go to `dropped` (capacity entries),
 * their count to *n_dropped. */
int mrsim_apply_multiband_motion(mrsim_context* ctx, float* const* images, int64_t ncomp, const int64_t* dims,
                                 int64_t n_volumes, const double* v2w, int64_t mb, int32_t interleaved,
                                 const mrsim_dropout_law* law, const mrsim_motion_event* events,
                                 int64_t n_events, const int64_t* slice_z, int64_t nz_full,
                                 mrsim_dropped_shot* dropped, int64_t capacity, int64_t* n_dropped);
/* No reference counterpart: `apply_motion` on an EPI operator's device images (its slab of
 * slices, grid v2w of the sim grid, poses n_volumes x 6), in place; returns when done.  A moved
 * series reaches the forward without crossing the host link. */
int mrsim_epi_operator_apply_motion(mrsim_epi_operator* op, const double* v2w, const double* poses);

/* ---- writing the series (io.rs) ------------------------------------------------------------- */
/* NIfTI-1 with the grid's voxel-to-world affine v2w (row-major 4x4); gzip when the path ends in
 * ".gz".  `write_4d_timed` io.rs:135-146: data (x + nx*(y + ny*z))*nt + t, a 4D header; tr_s > 0
 * puts the repetition time in pixdim[4] and seconds in xyzt_units (`write_4d` io.rs:131: 0). */
int mrsim_write_nifti_4d(const char* path, const int64_t* dims, int64_t nt, const float* data, const double* v2w,
                         double tr_s);
/* `write_3d` io.rs:149-156: one volume x + nx*(y + ny*z), a 3D header. */
int mrsim_write_nifti_3d(const char* path, const int64_t* dims, const float* data, const double* v2w);
/* `hires_grid` io.rs:104-124: the simulation grid of an acquired grid refined in-plane by o. */
int mrsim_hires_grid(const double* v2w, const int64_t* dims, int64_t o, double* out_v2w, int64_t* out_dims);
/* `SidecarInfo` io.rs:162-184. */
typedef struct mrsim_sidecar_info {
  const char* manufacturer;
  const char* phase_encoding_direction; /* "i", "j-", ... for the written voxel frame */
  double total_readout_time;            /* s */
  double echo_time;                     /* s */
  double partial_fourier;
  int64_t accel;
  int64_t mb;
  int32_t has_repetition_time;
  double repetition_time_s;
  const char* b0_field_source;          /* NULL: none */
} mrsim_sidecar_info;
/* `write_complex_4d` io.rs:186-228: <prefix>_part-mag_<suffix>.nii.gz, _part-phase_ (radians) and
 * their .json sidecars; mag / phase as from mrsim_simulate_acquisition_oversampled, whose device
 * output pass splits magnitude and phase. */
int mrsim_write_complex_4d(const char* out_prefix, const char* suffix, const int64_t* dims, int64_t n_volumes,
                           const float* mag, const float* phase, const double* v2w,
                           const mrsim_sidecar_info* info);

/* ---- spin history of slice-selective excitations under head motion (spin_history.rs) -------- */
/* The longitudinal magnetisation of every tracked source voxel (class != MRSIM_SPIN_NO_CLASS), as
 * at most MRSIM_SPIN_MAX_PIECES pieces of its z extent (mz just after each piece's last
 * excitation and that time), stepped through the excitations of a series on the device.  Per
 * excitation and excited slice: num[class][cell] = sum l V w (Mz(t) - mz_ref(T1)) and
 * den[class][cell] = sum l V w mz_ref(T1) over the pieces inside the slice's slab, at the slab
 * cell nearest each voxel's moved centre (`SpinHistory`, spin_history.rs:171-452).  Each sum runs
 * in FP64 in the reference's order (source planes, then voxels, then pieces) and is rounded to
 * f32 once, as the reference does. */
#define MRSIM_SPIN_NO_CLASS 255
#define MRSIM_SPIN_MAX_PIECES 8
enum { MRSIM_PULSE_INVERSION = 0, MRSIM_PULSE_SATURATION = 1 };
/* `Pulse` (spin_history.rs:63-69): Inversion scales Mz by 1 - 2 epsilon; Saturation sets 0. */
typedef struct mrsim_pulse {
  int32_t kind;
  double t;       /* s, on the series clock */
  double epsilon; /* inversion only */
} mrsim_pulse;
/* The reference magnetisation of an excitation, `mz_ref(T1)` (the closure `excite` takes,
 * spin_history.rs:311), as one of:
 *   NONE      the excitation reads no terms (`prime`, spin_history.rs:303-307);
 *   RECOVERY  1 - (1 - a) exp(-b / T1)   (a = 0: saturation recovery over b seconds);
 *   CONSTANT  a where T1 > 0, else b;
 *   REPLAY    Mz at the excitation's time from a just after time b, through the series' pulses
 *             (0 where T1 <= 0): the static head's closed form;
 *   VALUES    values[i] for the i-th tracked voxel in source order (host pointer). */
enum { MRSIM_MZREF_NONE = 0, MRSIM_MZREF_RECOVERY = 1, MRSIM_MZREF_CONSTANT = 2, MRSIM_MZREF_REPLAY = 3,
       MRSIM_MZREF_VALUES = 4 };
typedef struct mrsim_mz_reference {
  int32_t kind;
  double a, b;
  const double* values;
} mrsim_mz_reference;
/* One shot: the excitation's time (s), the head's world-space transform (p' = m p, row-major
 * 4x4), the slab indices it excites, its reference and, optionally, a weight per source voxel
 * (x + nx*(y + ny*z), host pointer) that replaces the source weight for this shot only. */
typedef struct mrsim_spin_shot {
  double t;
  double transform[16];
  const int64_t* slices;
  int64_t n_slices;
  mrsim_mz_reference ref;
  const float* weight;
} mrsim_spin_shot;
typedef struct mrsim_spin_history mrsim_spin_history;
/* `SpinHistory::new` spin_history.rs:254-289: the source grid (dims, voxel-to-world v2w,
 * per-voxel T1 in s, weight and class), the slab grid whose z index is the slice, and the
 * series' pulses in any order.  Every voxel starts fully relaxed. */
int mrsim_spin_history_create(mrsim_context* ctx, const int64_t* src_dims, const double* src_v2w, const float* t1,
                              const float* weight, const uint8_t* cls, int64_t n_classes, const int64_t* slab_dims,
                              const double* slab_v2w, const mrsim_pulse* pulses, int64_t n_pulses,
                              mrsim_spin_history** out);
void mrsim_spin_history_destroy(mrsim_spin_history* h);
/* The number of tracked voxels (the length of a VALUES reference). */
int mrsim_spin_history_n_tracked(mrsim_spin_history* h, int64_t* n);
/* `SpinHistory::prime` spin_history.rs:303-307: shot i excites slices[offsets[i]..offsets[i+1]]
 * at times[i], every shot at `transform`, reading no terms. */
int mrsim_spin_history_prime(mrsim_spin_history* h, const double* times, const int64_t* slices,
                             const int64_t* offsets, int64_t n_shots, const double* transform);
/* The number of floats the terms of `shots` take: sum over the shots that read terms of
 * n_slices * 2 * n_classes * slab_nx * slab_ny. */
int mrsim_spin_history_terms_size(mrsim_spin_history* h, const mrsim_spin_shot* shots, int64_t n_shots,
                                  int64_t* n_floats);
/* `SpinHistory::excite` spin_history.rs:311-315, for n_shots shots in order: the terms of each
 * shot that reads them, packed shot after shot as [slice in shot][num, den][class][x + slab_nx*y]
 * (f32), into the host buffer `terms`.  Returns when done. */
int mrsim_spin_history_excite(mrsim_spin_history* h, const mrsim_spin_shot* shots, int64_t n_shots, float* terms);
/* No reference counterpart: the same with `terms` a device buffer, queued on the context's
 * stream; the call returns once the launches are queued (the host inputs have been copied). */
int mrsim_spin_history_excite_device(mrsim_spin_history* h, const mrsim_spin_shot* shots, int64_t n_shots,
                                     float* terms);
/* `SpinHistory::merges` spin_history.rs:296-301 (synchronises the stream; reports a kernel's
 * error status). */
int mrsim_spin_history_merges(mrsim_spin_history* h, uint64_t* merges);

/* ---- the 3D echo trains (kspace3d.rs, readout.rs:75-322) ----------------------------------- */
enum { MRSIM_KZ_CENTRIC = 0, MRSIM_KZ_LINEAR = 1 };                            /* readout.rs:75 */

/* `EchoTrain` (readout.rs:82-95). */
typedef struct mrsim_echo_train {
  int64_t etl;
  double esp_ms;
  double refocusing_deg;
  int32_t kz_order;        /* MRSIM_KZ_* */
  int32_t reserved;
  int64_t kz_segments;
  double refocusing_time_ms;
} mrsim_echo_train;

/* `Readout3d::Grase` (readout.rs:103-106). */
typedef struct mrsim_grase_readout {
  int64_t ky_segments;
  double t_line_ms;
  int32_t reverse_phase;
  int32_t reserved;
} mrsim_grase_readout;

/* `ShotSet` (kspace3d.rs:59-65): the images one set of shots of one volume saw (per-shot motion),
 * per compartment one simulation-grid volume x + snx*(y + sny*z).  Every line (spiral: every
 * interleave) of a shot in `shots` is computed from these images instead of the volume's own; a
 * shot in several sets takes the first. */
typedef struct mrsim_shot_set {
  const int64_t* shots;
  int64_t n_shots;
  const float* const* images;
} mrsim_shot_set;

/* The inputs of `simulate_acquisition_3d` (kspace3d.rs:549-565): images as the 2D series takes
 * them (ncomp arrays of snx*sny*nz*n_volumes, vox*nv+g); t2 / t1 / t_inhom per compartment over
 * the simulation volume (t1 NULL = infinite; required below 180 degrees of refocusing; t_inhom
 * NULL = Acquisition::t_inhom); `line_weights` = `LineWeights::w` [g][shot][c] or NULL; the
 * in-plane GRAPPA reference scan (`GrappaCalibration`, kspace.rs:1646) when
 * has_grappa_calibration, else the first volume's images and `seed`; `shot_sets` /
 * `n_shot_sets` = the per-shot images (`shot_images: Option<&[Vec<ShotSet>]>`): volume g's sets at
 * shot_sets[g][0 .. n_shot_sets[g]], or both NULL (the reference scan never takes them). */
typedef struct mrsim_acquisition_3d_input {
  int64_t sim_dims[3];
  int64_t acq_dims[3];
  int64_t n_volumes;
  int64_t ncomp;
  const float* const* images;
  const mrsim_t2* t2;
  const mrsim_t2* t1;
  const float* fmap;
  const mrsim_t2* t_inhom;
  const mrsim_phase_model* phase;
  const double* line_weights;
  int32_t has_grappa_calibration;
  int32_t reserved;
  const float* const* grappa_calibration_images;   /* ncomp sim volumes */
  uint64_t grappa_calibration_seed;
  const mrsim_shot_set* const* shot_sets;          /* n_volumes lists, or NULL */
  const int64_t* n_shot_sets;                      /* n_volumes counts, or NULL */
} mrsim_acquisition_3d_input;

/* `kz_order` (readout.rs:167-189). */
int mrsim_kz_order(int64_t nz, int32_t order, int64_t* out);
/* `grase_lines` (readout.rs:283-322): per line p*ny + ky its shot, echo (1-based), t and trf
 * (ms) and polarity (any output may be NULL); e_c and n_shots. */
int mrsim_grase_lines(const mrsim_echo_train* train, const mrsim_grase_readout* ro, int64_t ny,
                      int64_t nz, int64_t* shot, int64_t* echo, double* t_ms, double* trf_ms,
                      int8_t* polarity, int64_t* e_c, int64_t* n_shots);
/* `simulate_acquisition_3d` (kspace3d.rs:549-565) with a GRASE readout, on the device: per
 * volume every compartment's 2D forward (within-echo timing, class or voxel decay), the centred
 * z-DFT, the line weights and sampling, spikes and noise per (volume, partition, coil), the
 * inverse z-DFT, GRAPPA (one kernel per slice from the reference scan) and the 2D reconstruction.
 * mag / phase: f32, vox*nv + g. */
int mrsim_simulate_acquisition_3d(mrsim_context* ctx, const mrsim_acquisition_3d_input* in,
                                  const mrsim_acquisition* acq, const mrsim_echo_train* train,
                                  const mrsim_grase_readout* ro, uint64_t seed, float* mag,
                                  float* phase);
/* `kspace_3d_observed` (kspace3d.rs:439-456): volume g's acquired 3D k-space per coil before
 * spikes and noise, out [coil][(p*ny + ky)*nx + kx] (re, im) f32. */
int mrsim_kspace_3d_observed(mrsim_context* ctx, const mrsim_acquisition_3d_input* in,
                             const mrsim_acquisition* acq, const mrsim_echo_train* train,
                             const mrsim_grase_readout* ro, int64_t g, float* out);

/* ---- the 3D gradient-echo stack-of-EPI train (kspace3d.rs:590-856, readout.rs:356-462) ----- */
/* `ExcitationTrain` (readout.rs:362-369); echo_times_ms strictly increasing, n_echoes >= 1. */
typedef struct mrsim_excitation_train {
  int64_t kz_segments;
  int32_t kz_order;         /* MRSIM_KZ_* */
  int32_t reserved;
  double exc_spacing_ms;
  const double* echo_times_ms;
  int64_t n_echoes;
  double excitation_time_ms;
} mrsim_excitation_train;

/* `Ge3dReadout` (readout.rs:374-379). */
typedef struct mrsim_ge3d_readout {
  int64_t ky_segments;
  double t_line_ms;
  int32_t reverse_phase;
  int32_t reserved;
} mrsim_ge3d_readout;

/* `GeVolume` (kspace3d.rs:592-603): per compartment one sim volume (NULL = a compartment this
 * volume does not use; its weights must be 0), the excitation weights
 * w[(p * ky_segments + sy) * ncomp + c], and the per-shot images (`shot_images`: n_shot_sets
 * sets, each with an image for every compartment the volume uses; 0 / NULL = none; the GRAPPA
 * reference scan never takes them). */
typedef struct mrsim_ge_volume {
  const float* const* images;
  const double* weights;
  const mrsim_shot_set* shot_sets;
  int64_t n_shot_sets;
} mrsim_ge_volume;

/* The `volume` callback: fill *out for volume g (pointers valid until the next call or the end
 * of the acquisition call); return 0, or non-zero to abort with MRSIM_ERR_INVALID.  Called on the
 * calling thread, once per volume (and once more for volume 0 when a GRAPPA reference is needed
 * and none is given). */
typedef int (*mrsim_ge_volume_fn)(int64_t g, void* user, mrsim_ge_volume* out);

typedef struct mrsim_acquisition_ge_input {
  int64_t sim_dims[3];
  int64_t acq_dims[3];
  int64_t n_volumes;
  int64_t ncomp;
  const mrsim_t2* t2;
  const float* fmap;
  const mrsim_t2* t_inhom;            /* ncomp or NULL */
  const mrsim_phase_model* phase;
  mrsim_ge_volume_fn volume;
  void* user;
  const mrsim_ge_volume* reference;   /* the GRAPPA reference scan's volume, or NULL */
} mrsim_acquisition_ge_input;

/* `ge3d_lines` (readout.rs:418-450): per line p*ny + ky its shot, excitation, t (ms) and
 * polarity (any output may be NULL); n_shots, n_exc and e_c (0-based excitation). */
int mrsim_ge3d_lines(const mrsim_excitation_train* train, const mrsim_ge3d_readout* ro, int64_t ny,
                     int64_t nz, int64_t* shot, int64_t* excitation, double* t_ms,
                     int8_t* polarity, int64_t* n_shots, int64_t* n_exc, int64_t* e_c);
/* `simulate_acquisition_3d_ge` (kspace3d.rs:837-856) on the device: per echo e, mag[e] and
 * phase[e] (f32, vox*nv + g). */
int mrsim_simulate_acquisition_3d_ge(mrsim_context* ctx, const mrsim_acquisition_ge_input* in,
                                     const mrsim_acquisition* acq,
                                     const mrsim_excitation_train* train,
                                     const mrsim_ge3d_readout* ro, uint64_t seed,
                                     float* const* mag, float* const* phase);

/* ---- the stack of spirals (kspace3d.rs:858-1569, readout.rs:107-160, 622-700) -------------- */
/* `KzSampling` (readout.rs:107-160). */
typedef struct mrsim_kz_sampling {
  double partial_fourier;  /* (0.5, 1] */
  int64_t accel;           /* >= 1 */
} mrsim_kz_sampling;

/* `Readout3d::Spiral` (readout.rs:103-106). */
typedef struct mrsim_spiral_readout {
  int64_t interleaves;
  double readout_ms;
  double dwell_ms;
  double radial_oversampling;
  mrsim_kz_sampling kz;
} mrsim_spiral_readout;

/* `KzOptions` (kspace3d.rs:1173-1178): coil rings along z, the kz calibration acquisition
 * (images: ncomp sim volumes, read only when kz.accel > 1) and the partial-Fourier recon
 * (0 = ZeroFill, 1 = Pocs). */
typedef struct mrsim_kz_options {
  int64_t coil_rows;
  const float* const* calibration_images;
  uint64_t calibration_seed;
  int32_t pocs;
  int32_t reserved;
} mrsim_kz_options;

/* `spiral_lines` (readout.rs:653-676): per partition acquired (0/1), echo (1-based, 0 = not
 * read) and kz segment; band start, centre echo, shots, and the samples per interleaf. */
int mrsim_spiral_lines(const mrsim_echo_train* train, const mrsim_spiral_readout* ro, int64_t nx,
                       int64_t ny, int64_t nz, uint8_t* acquired, int64_t* echo,
                       int64_t* kz_segment, int64_t* band_start, int64_t* e_c, int64_t* n_shots,
                       int64_t* samples_per_interleaf);
/* `simulate_acquisition_3d_kz` (kspace3d.rs:567-589) with a spiral readout (`spiral_volumes`
 * :1472-1569): per slice the certified time-segmented forward of every compartment and coil
 * element, the centred z-DFT with the rings' z profiles, echo amplitudes and line weights, the
 * noise per (volume, partition, coil), the kz GRAPPA fill from the calibration acquisition, POCS or
 * zero fill along z, the inverse z-DFT and the spiral reconstruction with the ring Roemer
 * combine, on the device.  kz_opts may be NULL (one ring, no kz acceleration).  mag / phase f32
 * at vox*nv + g. */
int mrsim_simulate_acquisition_3d_spiral(mrsim_context* ctx, const mrsim_acquisition_3d_input* in,
                                         const mrsim_acquisition* acq, const mrsim_echo_train* train,
                                         const mrsim_spiral_readout* ro,
                                         const mrsim_kz_options* kz_opts, uint64_t seed,
                                         float* mag, float* phase);
/* `SpiralSegmentation` / `spiral_segmentation` (kspace3d.rs:860-870, 1441-1470): the certified
 * time segmentations a spiral series will use, per slice and mode (class first), or the error
 * naming the slice whose rate rectangle cannot be certified.  Images are not read.  With rows
 * NULL only *count is written.  Planned on the host (no context): the series plans with its fits
 * on the device, which choose the same L and m; b_sum and the bound agree to ~1e-6 relative. */
typedef struct mrsim_spiral_segmentation_row {
  int32_t z, voxel, l, m;
  double b_sum, bound;
} mrsim_spiral_segmentation_row;
int mrsim_spiral_segmentation(const mrsim_acquisition_3d_input* in, const mrsim_acquisition* acq,
                              const mrsim_echo_train* train, const mrsim_spiral_readout* ro,
                              int64_t capacity, mrsim_spiral_segmentation_row* rows,
                              int64_t* count);

/* `SpiralPlan::samples_all` (kspace3d.rs:1047-1060): volume g's samples per coil before noise,
 * out [coil][p*nsamp + j] (re, im) f32 (zero on partitions not read). */
int mrsim_spiral_samples_3d(mrsim_context* ctx, const mrsim_acquisition_3d_input* in,
                            const mrsim_acquisition* acq, const mrsim_echo_train* train,
                            const mrsim_spiral_readout* ro, const mrsim_kz_options* kz_opts,
                            int64_t g, float* out);

/* ---- timing checks of the 3D trains (readout.rs:326-354, 460-500, 706-730) ---------------- */
/* 0 when the train fits its RF and sampling intervals, else MRSIM_ERR_INVALID with the
 * reference's message.  `check_spiral_timing` writes the train's end (ms) to end_ms (may be NULL). */
int mrsim_check_grase_timing(const mrsim_echo_train* train, const mrsim_grase_readout* ro,
                             int64_t ny, int64_t nz, double t_exc_ms, double tr_ms);
int mrsim_check_ge3d_timing(const mrsim_excitation_train* train, const mrsim_ge3d_readout* ro,
                            int64_t ny, int64_t nz, double t_exc_ms, double tr_ms);
int mrsim_check_spiral_timing(const mrsim_echo_train* train, const mrsim_spiral_readout* ro,
                              int64_t nx, int64_t ny, int64_t nz, double t_exc_ms, double tr_ms,
                              double* end_ms);
/* `esp_from_echo_time` (readout.rs:286-288) and `spiral_esp_from_echo_time` (:702-704). */
double mrsim_esp_from_echo_time(double te_ms, int64_t e_c, const mrsim_grase_readout* ro, int64_t ny);
double mrsim_spiral_esp_from_echo_time(double te_ms, int64_t e_c);

/* ---- the stack-of-spirals path: host plans ------------------------------------------------ */
/* `spiral_tau_c` (readout.rs:564-596): the constant-angular-velocity centre region (ms). */
int mrsim_spiral_tau_c(int64_t nx, int64_t interleaves, double readout_ms, double dwell_ms,
                       double radial_oversampling, double* tau_c_ms);

typedef struct mrsim_spiral_info {
  int64_t samples;     /* per interleaf: floor(T / dwell) */
  int64_t interleaves;
  double k_max, n_turns, tau_c_ms;
} mrsim_spiral_info;

/* `spiral_trajectory` (readout.rs:597-620).  Fills `info`; with k / tau_ms non-NULL also writes
 * k [interleaf][sample][2] (cycles/FOV) and tau_ms [sample] ((j + 1/2) dwell) when
 * `capacity` >= samples per interleaf.  Errors carry the reference's messages. */
int mrsim_spiral_trajectory(int64_t nx, int64_t ny, int64_t interleaves, double readout_ms,
                            double dwell_ms, double radial_oversampling, int64_t capacity,
                            double* k, double* tau_ms, mrsim_spiral_info* info);

typedef struct mrsim_tseg_info {
  int64_t l, m;      /* segments, Chebyshev degree */
  double b_sum;      /* max over samples of sum_l |b_l| */
  double grid_err;   /* max residual on the rate grid */
  double bound;      /* certified bound (< 1e-7) */
} mrsim_tseg_info;

/* `tseg::plan` (tseg.rs:230-289) over the rate rectangle d (1/ms) x f (Hz).  With tau_l / b
 * non-NULL and l_capacity >= L: tau_l [L] (ms) and b [n_tau][L][2] (re, im). */
int mrsim_tseg_plan(const double* tau_ms, int64_t n_tau, double t_ms, const double d[2],
                    const double f[2], int64_t l_capacity, double* tau_l, double* b,
                    mrsim_tseg_info* info);
/* The same plan with every fit's per-sample work (right-hand sides over the rate grid, the
 * factored least-squares solve, the residual) on the context's device in FP64; the Jacobi
 * factorisation and the search over L and m stay on the host.  This is the planner the device
 * forwards use.  Same L and m as mrsim_tseg_plan; b_sum and the bound agree to ~1e-6 relative
 * and b to the conditioning of the truncated least-squares problem (CUDA's exp / sin / cos round
 * differently from the host's in the last bit). */
int mrsim_tseg_plan_device(mrsim_context* ctx, const double* tau_ms, int64_t n_tau, double t_ms,
                           const double d[2], const double f[2], int64_t l_capacity, double* tau_l,
                           double* b, mrsim_tseg_info* info);

/* `epg_cpmg` (epg.rs:101-125): ln A_e for e = 1..n_echoes of a CPMG train. */
int mrsim_epg_cpmg(int64_t n_echoes, double esp_ms, double refocusing_deg, double t1_ms,
                   double t2_ms, double* ln_amp);

/* ---- the stack-of-spirals path: device NUFFT pair and spiral forwards ---------------------- */
/* Kernel width of the exponential-of-semicircle NUFFT at tolerance tol (nufft.rs:165). */
int mrsim_nufft_kernel_width(double tol);

/* `Nufft1::new` + `run` (nufft.rs:41-107) on the device in FP64: nw weight vectors (weights
 * [nw][npos] (re, im) f64) at sources `pos` (cells, any real, period n) to the integer frequencies
 * k_lo .. k_lo + n_out (inside [-n/2, n/2]): out [nw][n_out] (re, im) f64,
 * F[k] = sum_j w_j e^{+i2pi k pos_j / n}. */
int mrsim_nufft1(mrsim_context* ctx, int64_t n, int64_t k_lo, int64_t n_out, double tol,
                 const double* pos, int64_t npos, const double* weights, int64_t nw, double* out);

/* `Nufft2::type1` (nufft.rs:225-256) on the device, host buffers: periods n, modes m_lo ..
 * m_lo + m_out per axis (inside [-n/2, n/2]), points u [npts][2] (period-n coordinates),
 * weights [npts] (re, im) f32, sign +1 / -1; modes [m_out1][m_out0] (re, im) f32. */
int mrsim_nufft2_type1(mrsim_context* ctx, const int64_t n[2], const int64_t m_lo[2],
                       const int64_t m_out[2], double tol, const double* u, int64_t npts,
                       const float* weights, int32_t sign, float* modes);
/* `Nufft2::type2` (nufft.rs:259-292): values at the points from modes in type 1's layout. */
int mrsim_nufft2_type2(mrsim_context* ctx, const int64_t n[2], const int64_t m_lo[2],
                       const int64_t m_out[2], double tol, const float* modes, const double* u,
                       int64_t npts, int32_t sign, float* out);

/* `spiral_kspace_exact` (spiral.rs:107-137) on the device: one slice and coil at frequencies
 * k [npts][2] (cycles/FOV) sampled tau_ms [npts] after the echo; log_amp per sim voxel or NULL.
 * Up to 4 compartments.  out [npts] (re, im) f32. */
int mrsim_spiral_kspace_exact(mrsim_context* ctx, const mrsim_slice_input* inp,
                              const mrsim_acquisition* acq, int64_t coil, int64_t ncoils,
                              const double* k, const double* tau_ms, int64_t npts,
                              const double* log_amp, float* out);

/* `SegmentedForward::new` + `apply` with `segment_inputs` (spiral.rs:83-103, 154-201): the
 * time-segmented type-2 NUFFT forward of a one-compartment slice.  Sample j sits at
 * tau_ms[tau_idx[j]]; the plan is certified over d (1/ms) x f (Hz) on [0, t_ms];
 * decay_inside = voxel mode.  `info` (may be NULL) receives the plan's figures. */
int mrsim_spiral_segmented_forward(mrsim_context* ctx, const mrsim_slice_input* inp,
                                   const mrsim_acquisition* acq, int64_t coil, int64_t ncoils,
                                   const double* k, const int64_t* tau_idx, int64_t npts,
                                   const double* tau_ms, int64_t n_tau, double t_ms,
                                   const double d[2], const double f[2], const double* log_amp,
                                   int32_t decay_inside, float* out, mrsim_tseg_info* info);

/* ---- the stack-of-spirals path: the reconstruction ------------------------------------------ */
/*
 * `SpiralRecon` (grid_recon.rs:54-325) of one trajectory k [npts][2] (cycles/FOV) on an n x n
 * image, FP64 on the device: Pipe-Menon weights (10 iterations), the centre normalization, the
 * window (window_kind / window_a / window_b as in mrsim_acquisition), the image band, the power
 * iteration for lambda_hi, then per image `iterations` Chebyshev steps over
 * [lambda_hi / kappa, lambda_hi] and the residual check.  `SpiralRecon::new` is iterations = 80,
 * kappa = 100, band_limited = 1.  Sample and image buffers are host (re, im) f64 pairs.
 */
typedef struct mrsim_spiral_recon mrsim_spiral_recon;

int mrsim_spiral_recon_create(mrsim_context* ctx, const double* k, int64_t npts, int64_t n,
                              int32_t window_kind, double window_a, double window_b,
                              int64_t iterations, double kappa, int32_t band_limited,
                              mrsim_spiral_recon** out);
int mrsim_spiral_recon_destroy(mrsim_spiral_recon* rec);
/* lambda_hi, the power iterations run, and the normalized weights [npts] (any may be NULL). */
int mrsim_spiral_recon_info(const mrsim_spiral_recon* rec, double* lambda_hi,
                            int64_t* power_iterations, double* weights);
/* `gridding` (grid_recon.rs:231): n^2 A^H W d for samples [batch][npts] -> [batch][n*n]. */
int mrsim_spiral_recon_gridding(mrsim_spiral_recon* rec, const double* samples, int64_t batch,
                                double* out);
/* `image` (grid_recon.rs:238-275) of each of `batch` sample sets -> [batch][n*n].  Fails with
 * the reference's message when a residual grows. */
int mrsim_spiral_recon_image(mrsim_spiral_recon* rec, const double* samples, int64_t batch,
                             double* out);
/* `reconstruct_rings` (grid_recon.rs:285-320) of n_partitions partitions at once: coil_samples
 * [partition][coil][npts], zsens [partition][coil], coils in rings of `ring` (coil q is element
 * q % ring); out [partition][n*n].  `reconstruct` is ring = ncoils with zsens all 1. */
int mrsim_spiral_recon_rings(mrsim_spiral_recon* rec, const double* coil_samples,
                             int64_t n_partitions, int64_t ncoils, int64_t ring,
                             const double* zsens, double* out);

#ifdef __cplusplus
}
#endif
#endif /* MRSIM_ACQ_H */
