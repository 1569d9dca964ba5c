// misc_kernels.cu — layout changes between the reference's host layouts and the device layouts.
#include <cuda_runtime.h>

#include "driver.h"
#include "series.h"

namespace mrsim {

namespace {
// staging: per compartment c, the reference series layout in[c][vox * nv + g] with
// vox = p + plane * z; out: [g][z][c][p].  One thread per (c, vox) reads nv consecutive values.
__global__ void series_transpose_kernel(const float* __restrict__ in, float* __restrict__ out, int ncomp, int nv,
                                        int nz, int plane, int z0, int z1) {
  const long long nvox = (long long)nz * plane;
  const long long span = (long long)(z1 - z0) * plane;
  const long long total = span * ncomp;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / span);
    const long long vox = (long long)z0 * plane + t % span;
    const int z = (int)(vox / plane), p = (int)(vox % plane);
    const float* src = in + (size_t)c * nvox * nv + (size_t)vox * nv;
    for (int g = 0; g < nv; ++g) out[(((size_t)g * nz + z) * ncomp + c) * plane + p] = src[g];
  }
}
__device__ __forceinline__ double unit_of(uint64_t seed, uint64_t k) {
  uint64_t z = seed + (k + 1ull) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

// One thread per (volume, slice, y, x) of a chunk of volumes [g0, g1).
// mag_phase: write the magnitude sqrt(re^2 + im^2) and phase atan2(im, re) in f32 instead of
// (re, im) (`simulate_acquisition_oversampled`, kspace.rs:1839-1846), in the same pass.
__global__ void series_output_kernel(const float2* __restrict__ comb, const float* __restrict__ sigma,
                                     float* __restrict__ re, float* __restrict__ im, int g0, int g1, int nv, int nz,
                                     int nx, int ny, const int* __restrict__ zmap, uint64_t seed, int mag_phase) {
  const long long per = (long long)nx * ny;
  const long long total = (long long)(g1 - g0) * nz * per;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int g = g0 + (int)(t / (nz * per));
    const int zl = (int)((t / per) % nz);
    const long long p = t % per;
    const float2 c = comb[t];
    float r = c.x, i = c.y;
    const long long vox = p + per * zl;
    if (sigma) {
      const double sd = (double)sigma[vox];
      if (sd > 0.0) {
        const long long vox_g = p + per * zmap[zl];
        const uint64_t s = (seed ^ ((uint64_t)g * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)vox_g * 0xBF58476D1CE4E5B9ull)) |
                           1ull;
        const double tau = 6.283185307179586;
        const double n1 = sqrt(-2.0 * log(unit_of(s, 0))) * cos(tau * unit_of(s, 1));
        const double n2 = sqrt(-2.0 * log(unit_of(s, 2))) * cos(tau * unit_of(s, 3));
        r += (float)(n1 * sd);
        i += (float)(n2 * sd);
      }
    }
    if (mag_phase) {
      re[vox * nv + g] = sqrtf(__fadd_rn(__fmul_rn(r, r), __fmul_rn(i, i)));
      im[vox * nv + g] = atan2f(i, r);
    } else {
      re[vox * nv + g] = r;
      im[vox * nv + g] = i;
    }
  }
}

// Independent FMA chains per thread, all operands in registers: the FP32 pipe's throughput.
__global__ void __launch_bounds__(256) fma_probe_kernel(float* out, int iters, float a, float b) {
  float v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = threadIdx.x * 1e-3f + k;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = fmaf(v[k], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 16; ++k) s += v[k];
  if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the loop live
}
}  // namespace

double probe_fp32_tflops(cudaStream_t st) {
  int dev = 0, sms = 0;
  MRSIM_CUDA(cudaGetDevice(&dev));
  MRSIM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  float* out = nullptr;
  MRSIM_CUDA(cudaMalloc(&out, 256 * sizeof(float)));
  const int blocks = sms * 8, iters = 2048;
  cudaEvent_t e0, e1;
  MRSIM_CUDA(cudaEventCreate(&e0));
  MRSIM_CUDA(cudaEventCreate(&e1));
  fma_probe_kernel<<<blocks, 256, 0, st>>>(out, 256, 0.999f, 1e-3f);
  MRSIM_CUDA(cudaEventRecord(e0, st));
  for (int r = 0; r < 5; ++r) fma_probe_kernel<<<blocks, 256, 0, st>>>(out, iters, 0.999f, 1e-3f);
  MRSIM_CUDA(cudaEventRecord(e1, st));
  MRSIM_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  MRSIM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const double flops = 5.0 * blocks * 256.0 * iters * 16.0 * 2.0;
  return flops / (ms * 1e-3) / 1e12;
}

void launch_series_output(const float2* combined, const float* sigma, float* re, float* im, int g0, int g1, int nv,
                          int nz, int nx, int ny, const int* zmap, uint64_t receiver_seed, cudaStream_t st,
                          bool mag_phase) {
  const long long total = (long long)(g1 - g0) * nz * nx * ny;
  if (total <= 0) return;
  int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  series_output_kernel<<<blocks, 256, 0, st>>>(combined, sigma, re, im, g0, g1, nv, nz, nx, ny, zmap, receiver_seed,
                                                mag_phase ? 1 : 0);
  MRSIM_CUDA(cudaGetLastError());
}

void launch_series_transpose(const float* staging, float* out, int ncomp, int nv, int nz, int plane, cudaStream_t st,
                             int z0, int z1) {
  if (z1 < 0) z1 = nz;
  const long long total = (long long)(z1 - z0) * plane * ncomp;
  if (total <= 0) return;
  int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  series_transpose_kernel<<<blocks, 256, 0, st>>>(staging, out, ncomp, nv, nz, plane, z0, z1);
  MRSIM_CUDA(cudaGetLastError());
}

}  // namespace mrsim
