// driver.h — host orchestration objects (see driver.cpp).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "mrsim_internal.h"

namespace mrsim {

struct TsPlan;
void ts_plan_destroy(TsPlan* p);

// Device allocations owned by one object, freed together.
struct DevArena {
  std::vector<void*> ptrs;
  void* alloc(size_t bytes);
  void* upload(const void* src, size_t bytes, cudaStream_t st);
  DevArena() = default;
  DevArena(const DevArena&) = delete;
  DevArena& operator=(const DevArena&) = delete;
  ~DevArena();
};

GeoTab build_geo(DevArena& arena, int snx, int sny, int nx, int ny, int ncoils, double ghost, cudaStream_t st);

// The forward/adjoint operator of a whole 2D EPI series: units (volume, slice) with every
// echo's acquired lines.  Device layouts:
//   images    [g][z][c][sny][snx]            fmap [z][sny][snx]
//   kspace    [g][z][coil][echo][ny][nx]     complex
//   comp_grad [g][z][c][sny][snx]            complex (A^H applied to the k-space buffer)
//   fmap_grad [g][z][sny][snx],  r2_grad [g][z][c][sny][snx]
struct EpiOperator {
  mrsim_context* ctx = nullptr;
  int snx = 0, sny = 0, nx = 0, ny = 0, nz = 0, nv = 0, ncomp = 0, ncoils = 0, n_echoes = 0, n_lines = 0;
  int64_t samples_per_step = 0;
  size_t kspace_elems = 0;
  bool want_fmap = false, want_r2 = false;
  DevArena arena;
  float* d_images = nullptr;
  float* d_fmap = nullptr;
  float* d_t2 = nullptr;
  float* d_ti = nullptr;
  LineRec* d_lines = nullptr;
  GeoTab geo{};
  float* d_phase = nullptr;
  float2* d_g = nullptr;
  float2* d_kspace = nullptr;
  float2* d_comp_grad = nullptr;
  float* d_fmap_grad = nullptr;
  float* d_r2_grad = nullptr;
  std::unique_ptr<EpiPlan> plan;
  // acquired k-space rows of every echo as k0 + s i (i < n) with ny % s == 0, or n = 0: the host
  // call then downloads only those rows and zero-fills the others on the host
  int krow0 = 0, krow_step = 0, krow_n = 0;
  // host-buffer apply: download and upload streams and per-group events, made on first use
  cudaStream_t copy_stream = nullptr, upload_stream = nullptr;
  std::vector<cudaEvent_t> events;
  // what the time-segmented path rebuilds its tables from
  mrsim_acquisition acq{};
  std::vector<double> tes;
  std::vector<LineRec> h_lines;
  std::vector<float> h_fmap;
  float t2u[kMaxComp] = {0}, tiu[kMaxComp] = {0};
  bool maps = false, any_eddy = false;
  // the time-segmented tensor-core y-stages, when selected (mrsim_epi_operator_set_segmented)
  TsPlan* ts = nullptr;
  int ts_precision = 0;
  ~EpiOperator();
};

EpiOperator* epi_operator_create(mrsim_context* ctx, const mrsim_acquisition_input& in, const mrsim_acquisition& acq,
                                 const double* echo_times_ms, int64_t n_echoes, const int64_t* slice_z,
                                 int64_t nz_full, int grads);
void upload_series_images(EpiOperator* op, const float* const* host_images);
void epi_operator_set_fieldmap(EpiOperator* op, const float* fmap);
void epi_operator_forward(EpiOperator* op);
void epi_operator_adjoint(EpiOperator* op);
// plan units [u0, u1) (u1 < 0: all) of the y- and x-stages of either path
void epi_operator_forward_units(EpiOperator* op, cudaStream_t st, int u0, int u1);
void epi_operator_adjoint_units(EpiOperator* op, cudaStream_t st, int u0, int u1);
void epi_operator_set_segmented(EpiOperator* op, int precision);
// Times the plan's tunables (and with flags bit 0 the segmented path) on the operator's first
// units, keeps the fastest, and records it in the cache file (NULL: none) under the operator's
// shape; a shape already in the cache takes its recorded choice without timing.
std::string epi_operator_tune(EpiOperator* op, const char* cache_path, int flags, double* ms);
int epi_operator_segmented_error(EpiOperator* op);
// Forward + adjoint from host images to host k-space and gradients (any output may be NULL),
// pipelined by groups of slices (or of volumes for one slice): a group's images upload, and its
// results copy back, on two more streams while other groups compute.
// compact: k-space as [g][z][coil][echo][acquired row][kx] (the acquired rows only), else the
// reference's zero-filled [g][z][coil][echo][ny][nx]
void epi_operator_apply_host(EpiOperator* op, const float* const* images, float* kspace, float* comp_grad,
                             float* fmap_grad, float* r2_grad, bool compact = false);

// Several series of different geometries (matrix, grid, slice count, coils) in one plan: each
// series keeps its own operator (buffers, tables, line list) and the units of all of them form
// one unit list, so each stage of a forward or adjoint is one launch over every unit.
struct EpiBatch {
  mrsim_context* ctx = nullptr;
  std::vector<std::unique_ptr<EpiOperator>> ops;
  std::vector<int> unit0;  // first plan unit of each series
  std::unique_ptr<EpiPlan> plan;
  int64_t samples = 0;
};
EpiBatch* epi_batch_create(mrsim_context* ctx, int n, const mrsim_acquisition_input* const* inputs,
                           const mrsim_acquisition& acq, const double* echo_times_ms, int64_t n_echoes, int grads);
void epi_batch_forward(EpiBatch* b);
void epi_batch_adjoint(EpiBatch* b);

// noalloc.cu: the forward of one slice with every intermediate in static device arrays.
void build_coil_kspaces_noalloc(const mrsim_slice_input& inp, const mrsim_acquisition& acq, float2* out,
                                cudaStream_t st);

// misc_kernels.cu
// Slices [z0, z1) (z1 < 0: all) of the reference image layout (per compartment [z][y][x][g]) into
// the unit-major layout [g][z][c][y][x].
void launch_series_transpose(const float* staging, float* out, int ncomp, int nv, int nz, int plane, cudaStream_t st,
                             int z0 = 0, int z1 = -1);

}  // namespace mrsim
