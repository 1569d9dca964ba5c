// nufft.h — the device NUFFT pair and the spiral forwards (see nufft_kernels.cu, spiral.cpp).
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace mrsim {

// One NUFFT geometry (`Nufft2::new`, nufft.rs:162-182): periods n, fine grid nf = 2n, modes
// m_lo .. m_lo + m_out per axis; device tables corr (1/psi-hat per mode) and tw (e^{-i2pi k/nf}).
struct NufftGrid {
  int n0, n1, nf0, nf1, w;
  float beta;
  int m_lo0, m_lo1, m_out0, m_out1;
  const float* corr0;
  const float* corr1;
  const float2* tw0;
  const float2* tw1;
};

void nufft_fft2(const NufftGrid& g, float2* grid, int batch, int sign, cudaStream_t st);
// Type 2 (nufft.rs:259-292): out[b][j] = sum_m modes[b][m] e^{sign i2pi (u_j0 m0/n0 + u_j1 m1/n1)},
// optional per-batch scale; `work` holds batch fine grids.
void nufft_type2(const NufftGrid& g, const float2* modes, int batch, size_t mode_stride, const double* u, int npts,
                 float2* out, size_t out_stride, float2* work, int sign, const float* scale, cudaStream_t st);
// Type 1 (nufft.rs:225-256): modes[b][m] = sum_j w[b][j] e^{sign i2pi (...)}.
void nufft_type1(const NufftGrid& g, const double* u, int npts, const float2* wts, int batch, size_t w_stride,
                 float2* modes, size_t mode_stride, float2* work, int sign, cudaStream_t st);

// The exact spiral sum (`spiral_kspace_exact`, spiral.rs:107-137) of one slice and coil.
struct SpiralExactArgs {
  const double* k;        // npts x 2, cycles/FOV
  const double* tau_ms;   // npts
  int npts;
  int snx, sny, nx, ny, ox, oy, sxs, sys;
  double xoff, yoff;
  const float* amp;       // nvox: signal_scale x coil sensitivity
  const float* phase_turns;  // nvox static phase / 2pi, or NULL
  const float* rate;      // nvox off-resonance (Hz), NULL without distortions
  const float* comp;      // ncomp planes
  const float* decay;     // ncomp planes of 1/T2 + 1/T2' (1/ms), read under relaxation
  const float* log_amp;   // nvox or NULL
  int ncomp;              // <= 4
  int relax;
  float inv_nvox;
  float2* out;
};
void spiral_exact(const SpiralExactArgs& a, cudaStream_t st);

void segment_images(const float2* x, const float2* rate, int nvox, const double* tau_l, int L, float2* out,
                    cudaStream_t st);
void segment_combine(const float2* seg, int npts, int L, const int* tau_idx, const double* b, const float2* stat,
                     float2* out, cudaStream_t st);

}  // namespace mrsim
