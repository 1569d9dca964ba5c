// noise_kernels.h — device spikes and k-space noise (see noise_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mrsim {

// One coil's k-space of one (unit, echo): k points at row 0 of that echo, layout [ky][kx].
struct NoiseJob {
  float2* k;
  const int* rows;      // acquired ky rows, in mask order (device)
  const int* picks;     // spike sample indices kx + nx*ky (device), n_picks of them
  int n_rows, nx, n_picks, pad;
  uint64_t seed;        // (slice_seed ^ coil*0x9E3779B9) | 1
  double sigma;         // sqrt(noise_variance / (nx*ny)), 0 = no noise
  double spike_amplitude;
};

void launch_noise_jobs(const NoiseJob* d_jobs, int n_jobs, bool spikes, bool noise, int max_samples,
                       unsigned long long* d_keys, cudaStream_t st);

}  // namespace mrsim
