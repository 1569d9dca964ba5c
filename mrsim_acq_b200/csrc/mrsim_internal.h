// mrsim_internal.h — shared declarations of the B200 k-space library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mrsim_acq.h"

namespace mrsim {

constexpr int kMaxComp = 8;   // compartments per unit handled by the kernels
constexpr int kMaxCoils = 64; // coils per series
constexpr int kXfftMaxN = 2048; // largest power-of-two snx of the FFT x-stage (one CTA holds 2048 points)

// An error carrying the library status code; the ABI layer turns it into (status, message).
struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};
inline void fail(const std::string& m) { throw Error(MRSIM_ERR_INVALID, m); }
void cuda_check(cudaError_t e, const char* what);
#define MRSIM_CUDA(x) ::mrsim::cuda_check((x), #x)

// ---- device-side records ------------------------------------------------------------------
// One acquired line of one echo (the "line table" of `LineTiming`, kspace.rs:292-325, resolved
// per acquisition).  Phase time is split hi+lo so f*t keeps ~1e-9 turn accuracy in FP32.
struct LineRec {
  int ky;         // PE index within the acquired matrix
  int row;        // output row within the unit: echo*ny + ky
  int pol;        // readout polarity +1 / -1 (ghost sign)
  int pad;
  float t_hi;     // phase time t_b0 (s), hi part: spin echo t, gradient echo t + TE/1000
  float t_lo;     // lo part
  float t_s;      // echo time t (s) for the fmap VJP? (= t_hi+t_lo), kept for clarity
  float inhom_ms; // |t|*1000 (spin echo) or trf (gradient echo): the T2' clock
  float trf_ms;   // time from RF: the T2 clock
  float decay;    // eddy decay exp(-tread/tau)*t (0 when the eddy polynomial is off)
  float rel[kMaxComp];  // uniform relaxation weight per compartment for this line (1 if off)
};

// Geometry tables shared by every unit of one (snx, sny, nx, ny, ncoils, ghost) geometry.
struct GeoTab {
  const float* ex;      // [coil][snx]  exp(-(xa-px)^2/(2 s^2)) (1 for a single coil)
  const float* ey;      // [coil][sny]
  const float2* tw;     // [pol 0/1][x][kx]  e^{i2pi (kx-xs+gh)(x-c)/snx}
  float coil_off;       // 0.15 (ring of coils) or 0 (single coil)
  // x-stage FFT tables when snx is a power of two (else NULL): [snx/2] e^{-i2pi k/snx}, then
  // [pol 0/1][x] e^{i2pi gh (x-c)/snx}, then [kx] e^{-i2pi (kx-xs) c/snx}
  const float2* xf;
  // coil classes: coils whose ey rows are bitwise equal share a class (a ring of 8 coils has 5),
  // so sum_q amp_q(x,y) v = sum_d ey_d(y) (sum_{q in d} ex_q v) + off sum v.  ncls = 0: none.
  int ncls;
  const int* cls;     // [coil] class index
  const float* eyc;   // [class][sny] the class rows
};

// One unit of work: one slice of one volume, all echoes.  Device pointers throughout.
struct UnitDesc {
  int snx, sny, nx, ny;
  int ncomp, ncoils, n_lines, n_rows;
  int flags, z, nz, pad0;
  long long comp_stride;   // elements between compartment planes
  long long map_stride;    // elements between compartment map planes
  const float* comp;       // compartment 0 plane (real) — snx*sny
  const float* fmap;       // Hz
  const float* phase;      // static phase in turns (frac), per unit scratch, or NULL
  const float* t2map;      // ms, per compartment plane (NULL: uniform)
  const float* timap;      // ms, per compartment plane (NULL: uniform)
  const float* log_amp;    // snx*sny or NULL
  const LineRec* lines;    // n_lines
  GeoTab geo;
  float signal_scale;
  float t2u[kMaxComp];     // uniform T2 (ms) per compartment (used when a map is absent)
  float tiu[kMaxComp];     // uniform T2' (ms)
  float eddy_cx, eddy_qx, eddy_cy, eddy_qy, eddy_z;  // polynomial coefficients (turns per
                                                     // unit decay): cx*xc + qx*xc^2, ...
  float2* kspace;          // [coil][row][kx]
  float2* g;               // scratch [coil][line][snx] (y-stage out / x-adjoint out)
  float2* comp_grad;       // [comp][snx*sny] adjoint (A^H r per compartment)
  float* fmap_grad;        // [snx*sny]
  float* r2_grad;          // [comp][snx*sny]
};

enum : int {
  UF_RELAX = 1,
  UF_MAPS = 2,
  UF_GRADIENT = 4,
  UF_EDDY = 8,
  UF_WANT_FMAP_GRAD = 32,
  UF_WANT_R2_GRAD = 64,
  UF_DISTORT = 128,
};

// A tile of the x-stage GEMM: up to 32 rows (lines of one readout polarity x coils) by 64 output
// columns of one unit.
struct XTile {
  int unit, q0, nq, nl, col0, pol, pad0, pad1;
  int line[32];
};

// Per-unit static phase inputs for the statics kernel.
struct StaticDesc {
  int snx, sny, nx, ny, o, z, nz_full, flags;  // flags: 1 = phase from phase0, 2 = eddy phase
  const double* phase0;        // explicit phase (radians) or NULL
  double global, bg[10];       // phase model (used when phase0 == NULL)
  double shot_q[3], shot_dx[3], shot_rot[3];
  double eddy_phase_coef[3];   // eddy_phase * gradient
  double zc_c;                 // z - (nz-1)/2 for the eddy object-phase ramp
  float* out;                  // turns, frac in [-0.5, 0.5)
};

// ---- context --------------------------------------------------------------------------------
struct DeviceBuffer {
  void* p = nullptr;
  size_t n = 0;
};

}  // namespace mrsim

struct mrsim_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  // grow-only device workspaces keyed by role
  std::vector<mrsim::DeviceBuffer> ws;
  void* host_pinned = nullptr;  // page-locked staging slots of the pageable copies (host_copy.cpp)
  size_t host_pinned_n = 0;
  std::vector<cudaEvent_t> slot_ev;  // per slot: its last copy
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace mrsim {

// Workspace slot `slot` of at least `bytes` (grow-only, device memory of the context's device).
void* workspace(mrsim_context* ctx, int slot, size_t bytes);

// Large copies between pageable host memory and the device through the context's page-locked
// slots, several host threads at once (host_copy.cpp).  The upload is ordered on `st` like a
// cudaMemcpyAsync; the download returns when `dst` holds the data.
void copy_pageable_h2d(mrsim_context* ctx, void* dst, const void* src, size_t bytes, cudaStream_t st);
void copy_pageable_d2h(mrsim_context* ctx, void* dst, const void* src, size_t bytes, cudaStream_t st);

// ---- the forward/adjoint plan (epi_kernels.cu) -----------------------------------------------
// The plan's tunables (0: the built-in choice), the space the autotuner searches: coil classes
// off (per-coil y- and x-stages), the x-stage as the DFT GEMM instead of the FFTs, and the rows
// per thread of the fixed-coil y-adjoint (2 or 4).
struct EpiPlanOptions {
  int no_classes = 0;
  int dft_x = 0;
  int adj_rows = 0;
};
// Device-resident unit descriptors and tile lists, built once; executing a plan only launches
// kernels on a stream (no host copies, no synchronisation), so it can be captured in a graph.
// The caller zeroes the k-space outputs once: un-acquired rows are never written.
struct EpiPlan {
  int n_units = 0, n_statics = 0;
  std::vector<UnitDesc> host_units;
  UnitDesc* d_units = nullptr;
  StaticDesc* d_statics = nullptr;
  int max_static_n = 0, max_sny = 0, max_snx = 0, max_nx = 0, max_lines = 0, max_coils = 0, qg = 1, nc = 1;
  int max_hchunk = 0;  // max over units of (adjoint h chunk lines x coils)
  int4* d_ytiles[2] = {nullptr, nullptr};
  int n_ytiles[2] = {0, 0};
  void* d_gtiles[2] = {nullptr, nullptr};  // x-stage GEMM tiles: forward, adjoint
  int n_gtiles[2] = {0, 0};
  int4* d_atiles[4] = {nullptr, nullptr, nullptr, nullptr};
  int n_atiles[4] = {0, 0, 0, 0};
  // x-stage as per-row FFTs (every unit has a power-of-two snx and FFT tables): tiles of rows
  bool xfft = false;
  int xfft_e = 0;  // > 0: every unit has snx = 32 * xfft_e and the warp-per-row FFT runs; -1:
                   // every snx is a warp width (32 E, E <= 8) but not one width: per-width launches
  int fe_first[9] = {0}, fe_count[9] = {0};  // xfft_e == -1: the width-E tiles of d_ftiles
  // coil classes in the adjoint: the x-adjoint writes class rows (tiles of 4 lines x 8 coils) and
  // the y-adjoint combines 6 rows instead of 8 coils
  bool adj_cls = false;
  // coil classes in the forward: the y-stage writes the 6 class rows and the x-stage expands them
  // (the same tiles of 4 lines x 8 coils)
  bool fwd_cls = false;
  int4* d_ctiles = nullptr;
  int n_ctiles = 0;
  std::vector<int> c_start;
  int4* d_ftiles = nullptr;
  int n_ftiles = 0;
  // forward y-stage pass (maps) served by the staged-input kernel (8 lines per tile)
  bool fwdq[2] = {false, false};
  // ... and accumulating coil classes: their count plus the coil offset row, or 0
  int fwd_nv[2] = {0, 0};
  // y-adjoint pass (maps | grads << 1) served by the fixed-coil-count kernel: its coil count, or 0
  // for the general kernel
  int adjq[4] = {0, 0, 0, 0};
  // first tile of each unit in each list (n_units + 1 entries; empty: launch whole lists only)
  std::vector<int> y_start[2], a_start[4], f_start, g_start[2];
  // rows per thread of the fixed-coil y-adjoint, per pass
  int adj_ty[4] = {0, 0, 0, 0};
  EpiPlanOptions opt;
  std::vector<StaticDesc> host_statics;
  std::vector<void*> allocs;
  ~EpiPlan();
};
EpiPlan* epi_plan_create(const UnitDesc* units, int n, const StaticDesc* statics, int ns,
                         const EpiPlanOptions* opt = nullptr);
// The x-stage tiles of one unit (dir 0 forward, 1 adjoint); `lines` is a host copy of its table.
void append_xtiles(std::vector<XTile>& out, const UnitDesc& u, int unit_index, const LineRec* lines, int dir);
// Each launcher covers units [u0, u1) of the plan (u1 < 0: every unit).
void epi_plan_statics(const EpiPlan* p, cudaStream_t st, int u0 = 0, int u1 = -1);
void epi_plan_forward(const EpiPlan* p, cudaStream_t st, int u0 = 0, int u1 = -1);
void epi_plan_adjoint(const EpiPlan* p, cudaStream_t st, int u0 = 0, int u1 = -1);
void epi_plan_forward_ystage(const EpiPlan* p, cudaStream_t st, int u0 = 0, int u1 = -1);
void epi_plan_forward_xstage(const EpiPlan* p, cudaStream_t st, int u0 = 0, int u1 = -1);
void epi_plan_adjoint_xstage(const EpiPlan* p, cudaStream_t st, int u0 = 0, int u1 = -1);
void epi_plan_adjoint_ystage(const EpiPlan* p, cudaStream_t st, int u0 = 0, int u1 = -1);
// FP32 FMA throughput probe (misc_kernels.cu): TFLOP/s of a register-resident FMA loop.
double probe_fp32_tflops(cudaStream_t st);

}  // namespace mrsim
