// misc_kernels.cu — layout changes between the reference's host layouts and the device layouts.
#include <cuda_runtime.h>

#include "driver.h"

namespace mrsim {

namespace {
// staging: per compartment c, the reference series layout in[c][vox * nv + g] with
// vox = p + plane * z; out: [g][z][c][p].  One thread per (c, vox) reads nv consecutive values.
__global__ void series_transpose_kernel(const float* __restrict__ in, float* __restrict__ out, int ncomp, int nv,
                                        int nz, int plane) {
  const long long nvox = (long long)nz * plane;
  const long long total = nvox * ncomp;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(t / nvox);
    const long long vox = t % nvox;
    const int z = (int)(vox / plane), p = (int)(vox % plane);
    const float* src = in + (size_t)c * nvox * nv + (size_t)vox * nv;
    for (int g = 0; g < nv; ++g) out[(((size_t)g * nz + z) * ncomp + c) * plane + p] = src[g];
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

void launch_series_transpose(const float* staging, float* out, int ncomp, int nv, int nz, int plane, cudaStream_t st) {
  const long long total = (long long)nz * plane * ncomp;
  int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  series_transpose_kernel<<<blocks, 256, 0, st>>>(staging, out, ncomp, nv, nz, plane);
  MRSIM_CUDA(cudaGetLastError());
}

}  // namespace mrsim
