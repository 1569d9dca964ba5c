// nufft.h — the device NUFFT pair, FFTs and the spiral forwards (see nufft_kernels.cu, spiral.cpp,
// spiral_recon.cpp).
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace mrsim {

template <class R>
struct Vec2;
template <>
struct Vec2<float> {
  using type = float2;
};
template <>
struct Vec2<double> {
  using type = double2;
};

// One NUFFT geometry (`Nufft2::new`, nufft.rs:162-182): periods n, fine grid nf = 2n, modes
// m_lo .. m_lo + m_out per axis; device tables corr (1/psi-hat per mode) and tw (e^{-i2pi k/nf}).
// R = float for the forwards, double for the reconstruction.
template <class R>
struct NufftGridT {
  using V = typename Vec2<R>::type;
  int n0, n1, nf0, nf1, w;
  R beta;
  int m_lo0, m_lo1, m_out0, m_out1;
  const R* corr0;
  const R* corr1;
  const V* tw0;
  const V* tw1;
};
using NufftGrid = NufftGridT<float>;

// In-place 2D FFT of `batch` grids of n0 x n1 (layout c0 + n0 c1, batch stride n0 n1), sign -1 or
// +1, unnormalized; tw0 / tw1 hold e^{-i2pi k/n} for each axis.
template <class V>
void fft2(V* grid, int n0, int n1, const V* tw0, const V* tw1, int batch, int sign, cudaStream_t st);

template <class R>
void nufft_fft2(const NufftGridT<R>& g, typename Vec2<R>::type* grid, int batch, int sign, cudaStream_t st) {
  fft2(grid, g.nf0, g.nf1, g.tw0, g.tw1, batch, sign, st);
}

// Type 2 (nufft.rs:259-292): out[b][j] = sum_m modes[b][m] e^{sign i2pi (u_j0 m0/n0 + u_j1 m1/n1)},
// optional per-batch scale; `work` holds batch fine grids.
template <class R>
void nufft_type2(const NufftGridT<R>& g, const typename Vec2<R>::type* modes, int batch, size_t mode_stride,
                 const double* u, int npts, typename Vec2<R>::type* out, size_t out_stride,
                 typename Vec2<R>::type* work, int sign, const R* scale, cudaStream_t st);
// The deterministic spread's fine-grid tiles and, per tile, the points whose kernel window can
// reach it, in point order (CSR on the device, built on the host from the positions once per
// point set).  A tile is 8 x 8 fine cells in 2D (a cell's scan covers (8 + w)^2 cells of
// windows to use w^2; a 128 x 128 fine grid still gives 256 blocks), 256 cells in 1D.
constexpr int kSpreadTile = 8;
constexpr int kSpreadTile1 = 256;
struct NufftBins {
  int tiles0 = 0, tiles1 = 0;
  const int* start = nullptr;  // tiles0 * tiles1 + 1
  const int* pts = nullptr;
};
struct DevArena;
// 2D points u (npts x 2, period n per axis) on a fine grid of nf0 x nf1 cells, kernel width w
NufftBins nufft_bins2(DevArena& A, int nf0, int nf1, int w, const double* u_host, int npts, cudaStream_t st);
// 1D positions (cells, period n) on a fine grid of nf cells
NufftBins nufft_bins1(DevArena& A, int nf, int w, const double* pos_host, int npos, cudaStream_t st);

// Type 1 (nufft.rs:225-256): modes[b][m] = sum_j w[b][j] e^{sign i2pi (...)}.  The fine grid is
// spread without atomics: each cell sums its points in point order (the reference's order), so
// the result is the same on every run.  `bins` from nufft_bins2 over the same points.
template <class R>
void nufft_type1(const NufftGridT<R>& g, const double* u, int npts, const NufftBins& bins,
                 const typename Vec2<R>::type* wts, int batch, size_t w_stride, typename Vec2<R>::type* modes,
                 size_t mode_stride, typename Vec2<R>::type* work, int sign, cudaStream_t st);

// The 1D type-1 NUFFT (`Nufft1`, nufft.rs:25-112) in FP64: sources at `pos` (cells, period n),
// outputs at integer frequencies k_lo .. k_lo + n_out, F[k] = sum_j w_j e^{+i2pi k pos_j / n}, for
// nw weight vectors sharing the positions.  corr and tw on the device; work holds nw fine grids.
struct Nufft1Grid {
  int n, nf, w, k_lo, n_out;
  double beta;
  const double* corr;
  const double2* tw;
};
void nufft1_run(const Nufft1Grid& g, const double* pos, int npos, const NufftBins& bins, const double2* wts, int nw,
                double2* out, double2* work, cudaStream_t st);

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
