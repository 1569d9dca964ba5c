// spiral3d.h — the 3D stack-of-spirals acquisition on the device (see spiral3d.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "mrsim_internal.h"
#include "spiral_host.h"

namespace mrsim {

// `Spiral3dTable` / `spiral_lines` (readout.rs:622-676).
struct Spiral3dTable {
  int nz = 0, band_start = 0, kz_segments = 1, e_c = 0, n_shots = 0;
  SpiralTraj traj;
  std::vector<uint8_t> acquired;
  std::vector<int> echo, kz_segment;
};
int kz_band_start(const mrsim_kz_sampling& kz, int nz);
std::vector<uint8_t> kz_acquired(const mrsim_kz_sampling& kz, int nz);
Spiral3dTable spiral_lines(const mrsim_echo_train& train, const mrsim_spiral_readout& ro, int nx, int ny, int nz);
double coil_row_sensitivity(int row, int rows, double z, int nz);

struct SpiralSegmentationRow {
  int z, voxel, l, m;
  double b_sum, bound;
};
std::vector<SpiralSegmentationRow> spiral_segmentation(const mrsim_acquisition_3d_input& in,
                                                       const mrsim_acquisition& acq, const mrsim_echo_train& train,
                                                       const mrsim_spiral_readout& ro);

// `spiral_volumes` (kspace3d.rs:1472-1569) through the f32 magnitude / phase of
// `simulate_acquisition_3d_kz`; host buffers.
void spiral3d_acquire(mrsim_context* ctx, const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                      const mrsim_echo_train& train, const mrsim_spiral_readout& ro, const mrsim_kz_options* opts,
                      uint64_t seed, float* mag, float* ph);
// `SpiralPlan::samples_all` of volume g before noise: [coil][p][nsamp] complex f32 (host).
void spiral3d_samples(mrsim_context* ctx, const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                      const mrsim_echo_train& train, const mrsim_spiral_readout& ro, const mrsim_kz_options* opts,
                      int g, float* out);

}  // namespace mrsim
