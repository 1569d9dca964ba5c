// series_parts.h — building blocks of the device series drivers (defined in series.cpp), shared by
// the 2D series, the per-slice pipeline and the 3D echo-train drivers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "driver.h"
#include "host_tables.h"
#include "mrsim_internal.h"

namespace mrsim {

// Tables of one acquired geometry for the reconstruction.
struct ReconTables {
  float2* ex_tab = nullptr;
  float2* ey_tab = nullptr;
  float* sens = nullptr;
  float* inv_ssum = nullptr;
  float* window = nullptr;
  int4* fills = nullptr;
  int n_fills = 0;
  std::vector<float> sens_host;
};
ReconTables build_recon_tables(DevArena& A, int nx, int ny, int nc, const mrsim_acquisition& acq, cudaStream_t st);

// One forward launch over many units (slices of volumes, or compartments of slices).
struct Batch {
  std::vector<UnitDesc> units;
  std::vector<StaticDesc> statics;
};

struct UnitInputs {
  const float* comp;
  long long comp_stride;
  const float* fmap;
  const float* t2map;
  const float* timap;
  long long map_stride;
  const float* log_amp;
  const LineRec* lines;
  int n_lines;
  float2* kspace;
  float2* g;
  float* phase_out;
  const double* phase0;  // explicit phase (device) or NULL: the phase model
  const mrsim_phase_model* phase;
  ShotParams shot;
  int z, nz_full;
  bool has_eddy;
  double grad[3];
};

void add_unit(Batch& B, const UnitInputs& in, int snx, int sny, int nx, int ny, int ncomp, int ncoils, bool maps,
              const float* t2u, const float* tiu, const GeoTab& geo, const mrsim_acquisition& acq);
void run_forward(const Batch& B, cudaStream_t st);
// Line records of the acquired lines (uniform relaxation weights when `uniform`).
void lines_for(std::vector<LineRec>& out, const mrsim_acquisition& acq, int nx, int ny, bool eddy, bool uniform,
               int ncomp, const float* t2u, const float* tiu, bool has_tinhom, const LineTimingTab* timing);

// spikes + noise for a list of (k-space of one coil) jobs
struct NoiseSpec {
  float2* k;
  uint64_t slice_seed;
  int coil;
  int pick_offset;  // into the picks array, n_spikes per unit
};
void run_noise(DevArena& A, const std::vector<NoiseSpec>& specs, const std::vector<int>& rows,
               const std::vector<int>& picks, int nx, int ny, const mrsim_acquisition& acq, cudaStream_t st);
void spike_picks(std::vector<int>& picks, uint64_t slice_seed, const std::vector<uint8_t>& mask,
                 const mrsim_acquisition& acq);
// GRAPPA calibration of a batch of reference scans (one per slice): weights [slice][d-1][co][f].
float2* fit_grappa(DevArena& A, const std::vector<float2*>& ref_k, int nx, int ny, int nc,
                   const mrsim_acquisition& acq_ref, int accel, int acs_lines, cudaStream_t st);
bool uniform_relaxation(const mrsim_t2* t2, const mrsim_t2* ti, int ncomp);

}  // namespace mrsim
