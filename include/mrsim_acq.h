/*
 * mrsim_acq.h — C ABI of the B200 k-space acquisition library (libmrsim_acq_cuda.so).
 *
 * The library is a drop-in for the 2D EPI k-space path of the Rust crate `mrsim-acq`
 * (per-slice exact-DFT forward, GRAPPA calibration and apply, window, inverse DFT, Roemer
 * combine, series driver).  Every entry point cites the reference item it replaces as
 * `file:line` within the reference crate.  A Rust shim behind a `gpu` cargo feature binds these
 * symbols one for one (see INTEGRATION.md for the `extern "C"` block).
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
/* `simulate_slice` kspace.rs:1229-1235: out = nx*ny (re, im) f32 pairs. */
int mrsim_simulate_slice(mrsim_context* ctx, const mrsim_slice_input* inp,
                         const mrsim_acquisition* acq, float* out);
/* `simulate_slice_kspace` kspace.rs:1144-1149: coil 0's acquired k-space, nx*ny (re, im) f64. */
int mrsim_simulate_slice_kspace(mrsim_context* ctx, const mrsim_slice_input* inp,
                                const mrsim_acquisition* acq, double* out);
/* `build_coil_kspace_timed` kspace.rs:607-1042 for every coil of one slice, timing from
 * `LineTiming::for_acquisition` unless t_ms.. are given (each ny long, or all NULL); log_amp is
 * the 3D voxel-mode log-amplitude (snx*sny) or NULL.  out = n_coils*nx*ny (re, im) f64. */
int mrsim_build_coil_kspaces(mrsim_context* ctx, const mrsim_slice_input* inp,
                             const mrsim_acquisition* acq, const double* t_ms,
                             const double* trf_ms, const double* tread_ms,
                             const int8_t* polarity, const double* log_amp, double* out);

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
 * image arrays; mag/phase are n_echoes arrays of nx*ny*nz*n_volumes. */
int mrsim_simulate_acquisition_echoes(mrsim_context* ctx, const mrsim_acquisition_input* inp,
                                      const float* const* const* images_per_echo,
                                      const mrsim_acquisition* acq, const double* echo_times_ms,
                                      int64_t n_echoes, float* const* mag, float* const* phase);

/* ---- the batched forward / adjoint operator pair (device buffers) ------------------------ */
/*
 * A batch is a list of independent units (one slice of one volume read at one echo), each with
 * its own geometry, so one launch covers uneven matrix sizes.  All pointers are DEVICE pointers.
 * The forward is `build_coil_kspace_timed` (kspace.rs:607-1042) before spikes and noise:
 *   s_q[kx,ky] = (1/nvox) sum_x tw(kx,x) sum_y amp_q(x,y) e^{i2pi a(x,y)} E(x,y,ky)
 *                sum_c rel_c(x,y,ky) m_c(x,y)
 * with E = e^{i2pi(rate*t(ky) + (ky-ys)(y-c)/sny)} times the eddy polynomial factors.
 * The adjoint is its Hermitian transpose with respect to complex compartment images and, on
 * request, the vector-Jacobian products with respect to the fieldmap (Hz) and each compartment's
 * R2 = 1/T2 (1/ms).  The reference has no adjoint; its oracle is the FP64 transpose and central
 * finite differences.
 */
typedef struct mrsim_epi_unit {
  /* geometry */
  int32_t snx, sny, nx, ny;
  int32_t ncomp, ncoils, coil0, n_lines; /* coils coil0..coil0+ncoils-1 of ncoils_total     */
  int32_t ncoils_total;                  /* ring size for coil_sensitivity                 */
  int32_t z, nz;                         /* eddy z-terms                                   */
  int32_t flags;                         /* MRSIM_UNIT_* bits                              */
  /* device inputs */
  const float* comp;          /* ncomp planes of snx*sny (real) — or 2*ncomp (re,im) if  */
                              /* MRSIM_UNIT_COMPLEX_M                                     */
  const float* fmap;          /* snx*sny, Hz                                              */
  const float* phase_turns;   /* snx*sny static phase / (2 pi), or NULL                   */
  const float* t2_map;        /* ncomp planes (ms), only for MAPS units; or NULL           */
  const float* ti_map;        /* ncomp planes (ms), only for MAPS units; or NULL           */
  const float* log_amp;       /* snx*sny or NULL                                          */
  const float* lines;         /* n_lines records of MRSIM_LINE_FLOATS floats (see below)  */
  /* scalars */
  float t2_uniform[4];        /* per compartment (ms) for uniform compartments             */
  float ti_uniform[4];
  float signal_scale;
  float eddy_strength, eddy_quad, eddy_tau;
  float eddy_drive[3];
  float ghost_offset;
  /* device output (forward) / input (adjoint): ncoils*ny*nx (re, im) */
  float* kspace;
  /* adjoint outputs (device): comp_grad ncomp*snx*sny (re,im); fmap_grad, r2_grad ncomp*snx*sny */
  float* comp_grad;
  float* fmap_grad;
  float* r2_grad;
} mrsim_epi_unit;

/* unit flags */
#define MRSIM_UNIT_RELAX      1   /* do_relaxation                                           */
#define MRSIM_UNIT_MAPS       2   /* per-voxel relaxation (a T2/T2' map or log_amp present)   */
#define MRSIM_UNIT_GRADIENT   4   /* gradient echo: T2' decays from the RF                   */
#define MRSIM_UNIT_EDDY       8   /* gradient-model eddy polynomial on                       */
#define MRSIM_UNIT_COMPLEX_M 16   /* compartments are complex (re, im interleaved planes)     */
#define MRSIM_UNIT_WANT_FMAP_GRAD 32
#define MRSIM_UNIT_WANT_R2_GRAD   64
#define MRSIM_UNIT_DISTORT  128   /* do_distortions (rate = fmap)                            */

/* A line record: ky index, t (s, hi and lo split), |t|*1000 (ms), trf (ms), tread (ms),
 * polarity (+1/-1). */
#define MRSIM_LINE_FLOATS 8

/* Forward over every unit of the batch (device pointers, asynchronous on the context stream).
 * `units` is a host array of n_units descriptors. */
int mrsim_epi_forward(mrsim_context* ctx, const mrsim_epi_unit* units, int64_t n_units);
/* Adjoint / VJP over every unit (reads unit.kspace, writes comp_grad and the requested grads). */
int mrsim_epi_adjoint(mrsim_context* ctx, const mrsim_epi_unit* units, int64_t n_units);

#ifdef __cplusplus
}
#endif
#endif /* MRSIM_ACQ_H */
