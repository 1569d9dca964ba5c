// noise_kernels.cu — spikes and thermal k-space noise on acquired samples (reference
// kspace.rs:997-1039), on the device.
//
// Noise: the reference draws, for each acquired sample m in mask order, two Box-Muller normals
// from a SplitMix64 stream seeded (slice_seed ^ coil*0x9E3779B9) | 1, i.e. uniform draws 4m..4m+3.
// SplitMix64 is counter-based (draw k = mix(seed + (k+1)*gamma)), so every sample is evaluated
// independently here; the uniform draws are bit-identical to the reference, the FP64
// log/sqrt/cos are CUDA's (within an ulp or two of glibc's).
// Spikes: the sample of largest magnitude (first on ties) of each coil's k-space, scaled by
// spike_amplitude, overwrites the samples the host drew from the slice's spike stream.
#include <cuda_runtime.h>
#include <stdint.h>

#include "noise_kernels.h"

namespace mrsim {

namespace {

__device__ __forceinline__ uint64_t splitmix_draw(uint64_t seed, uint64_t k) {
  uint64_t z = seed + (k + 1ull) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double unit_draw(uint64_t seed, uint64_t k) {
  return ((double)(splitmix_draw(seed, k) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// one CTA per job: argmax |k| over the job's acquired rows (first index on ties)
__global__ void peak_kernel(const NoiseJob* __restrict__ jobs, unsigned long long* __restrict__ keys) {
  const NoiseJob& J = jobs[blockIdx.x];
  const int n = J.n_rows * J.nx;
  unsigned long long best = 0;
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    int r = m / J.nx, kx = m % J.nx;
    int ky = J.rows[r];
    float2 v = J.k[(size_t)ky * J.nx + kx];
    float mag = sqrtf(v.x * v.x + v.y * v.y);
    unsigned idx = (unsigned)(ky * J.nx + kx);
    unsigned long long key = ((unsigned long long)__float_as_uint(mag) << 32) | (0xFFFFFFFFu - idx);
    best = key > best ? key : best;
  }
  __shared__ unsigned long long red[256];
  red[threadIdx.x] = best;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = max(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) keys[blockIdx.x] = red[0];
}

__global__ void spike_kernel(const NoiseJob* __restrict__ jobs, const unsigned long long* __restrict__ keys) {
  const NoiseJob& J = jobs[blockIdx.x];
  if (threadIdx.x != 0 || J.n_picks == 0) return;
  unsigned long long key = keys[blockIdx.x];
  unsigned idx = 0xFFFFFFFFu - (unsigned)(key & 0xFFFFFFFFull);
  float2 peak = (key >> 32) == 0 ? make_float2(0.f, 0.f) : J.k[idx];
  float2 spike = make_float2((float)((double)peak.x * J.spike_amplitude), (float)((double)peak.y * J.spike_amplitude));
  for (int p = 0; p < J.n_picks; ++p) J.k[J.picks[p]] = spike;
}

__global__ void noise_kernel(const NoiseJob* __restrict__ jobs) {
  const NoiseJob& J = jobs[blockIdx.y];
  const int n = J.n_rows * J.nx;
  const uint64_t seed = J.seed;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
    int r = m / J.nx, kx = m % J.nx;
    int ky = J.rows[r];
    uint64_t k = 4ull * (uint64_t)m;
    double u1 = unit_draw(seed, k), u2 = unit_draw(seed, k + 1);
    double u3 = unit_draw(seed, k + 2), u4 = unit_draw(seed, k + 3);
    const double tau = 6.283185307179586;
    double g1 = sqrt(-2.0 * log(u1)) * cos(tau * u2);
    double g2 = sqrt(-2.0 * log(u3)) * cos(tau * u4);
    float2* p = J.k + (size_t)ky * J.nx + kx;
    float2 v = *p;
    v.x = (float)((double)v.x + g1 * J.sigma);
    v.y = (float)((double)v.y + g2 * J.sigma);
    *p = v;
  }
}

}  // namespace

void launch_noise_jobs(const NoiseJob* d_jobs, int n_jobs, bool spikes, bool noise, int max_samples,
                       unsigned long long* d_keys, cudaStream_t st) {
  if (n_jobs <= 0) return;
  if (spikes) {
    peak_kernel<<<n_jobs, 256, 0, st>>>(d_jobs, d_keys);
    spike_kernel<<<n_jobs, 32, 0, st>>>(d_jobs, d_keys);
  }
  if (noise) {
    dim3 grid((max_samples + 255) / 256, n_jobs);
    noise_kernel<<<grid, 256, 0, st>>>(d_jobs);
  }
}

}  // namespace mrsim
