// series.h — the per-slice pipeline and the series drivers (see series.cpp).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "host_tables.h"
#include "mrsim_internal.h"

namespace mrsim {

// Host outputs of one slice (any capture may be NULL); complex values as float2 (re, im).
struct SliceOutputs {
  float2* combined = nullptr;       // ny*nx
  float2* acquired = nullptr;       // n_coils*ny*nx
  float2* reconstructed = nullptr;  // n_coils*ny*nx
  float2* coil_images = nullptr;    // n_coils*ny*nx
  float* sensitivities = nullptr;   // n_coils*ny*nx
  uint8_t* mask = nullptr;          // ny*nx
};

// `build_coil_kspace_timed` for every coil of one slice (spikes and noise included), on the device.
std::vector<float2> slice_forward2(mrsim_context* ctx, const mrsim_slice_input& inp, const mrsim_acquisition& acq,
                                   const LineTimingTab* timing, const double* log_amp);
// `simulate_slice_full` (kspace.rs:1241-1284): GRAPPA (own reference scan), recon, combine.
void simulate_slice_full(mrsim_context* ctx, const mrsim_slice_input& inp, const mrsim_acquisition& acq,
                         SliceOutputs& out);
// `acquire_volumes_complex` (kspace.rs:1851-2125) with explicit excitation and receiver seeds;
// `images` overrides in.images (the echoes entry passes each echo's images).  mag_phase: out.re /
// out.im receive the magnitude and phase (kspace.rs:1839-1846), split on the device.
// The device copy of a series' images ([g][z][c][plane], transposed from the reference's
// vox*nv + g), kept across the calls of one entry point that pass the same arrays (the echoes of
// `simulate_acquisition_echoes` when their images are one set).
struct SeriesImageCache {
  std::vector<const float*> from;  // the host arrays the copy was made from
  float* d_img = nullptr;
  size_t n = 0;  // floats
  SeriesImageCache() = default;
  SeriesImageCache(const SeriesImageCache&) = delete;
  SeriesImageCache& operator=(const SeriesImageCache&) = delete;
  ~SeriesImageCache() {
    if (d_img) cudaFree(d_img);
  }
};
void acquire_series(mrsim_context* ctx, const mrsim_acquisition_input& in, const mrsim_acquisition& acq,
                    const mrsim_acquisition_options* opts, uint64_t excitation_seed, uint64_t receiver_seed,
                    const float* const* images, mrsim_acquisition_output& out, bool mag_phase = false,
                    SeriesImageCache* cache = nullptr);

// misc_kernels.cu: combined images -> (re, im) in the series layout vox*nv + g, plus the
// image-space noise of `acquire_volumes_complex` (kspace.rs:2031-2052).
void launch_series_output(const float2* combined, const float* sigma, float* re, float* im, int g0, int g1, int nv,
                          int nz, int nx, int ny, const int* zmap, uint64_t receiver_seed, cudaStream_t st,
                          bool mag_phase = false);

}  // namespace mrsim
