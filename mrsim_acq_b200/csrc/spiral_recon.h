// spiral_recon.h — the device spiral reconstruction (see spiral_recon.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "driver.h"
#include "mrsim_internal.h"
#include "nufft.h"

namespace mrsim {

// grid_recon.rs:36-50
constexpr int kDcfIterations = 10;
constexpr int kLsIterations = 80;
constexpr double kLsKappa = 100.0;
constexpr int kPowerIterations = 1000;
constexpr double kLambdaMargin = 1.1;
constexpr int kMaxBatch = 256;  // images per pass through the Chebyshev loop

struct SpiralRecon {
  mrsim_context* ctx;
  int n, npts, iterations;
  double kappa;
  bool band;
  double lambda_hi = 0.0;
  int power_iterations = 0;
  DevArena A;
  NufftGridT<double> g{};
  NufftBins bins_k;  // the trajectory's spread bins on g
  const double2* tw_n = nullptr;
  const double2* tw_2n = nullptr;
  double* d_k = nullptr;
  double* d_w = nullptr;    // normalized density weights
  double* d_win = nullptr;  // window per sample
  unsigned char* d_keep = nullptr;
  double2* d_tf = nullptr;  // transform of the Toeplitz kernel's circulant, 2n x 2n
  std::vector<double> w_host, k_host;

  struct Scratch {
    double2* pad;
    double2* tmp;
  };

  // `SpiralRecon::with_params` (grid_recon.rs:152-198); the window is win_acq's.
  SpiralRecon(mrsim_context* ctx, const double* k, int npts, int n, const mrsim_acquisition& win_acq,
              int iterations, double kappa, bool band_limited);
  Scratch scratch(DevArena& T, int batch) const;
  void project(double2* x, int batch, cudaStream_t st) const;
  void normal(const double2* x, double2* out, int batch, const Scratch& s, cudaStream_t st) const;
  void sumsq(const double2* v, int batch, double* out, cudaStream_t st) const;
  // device buffers: data [batch][npts], images [batch][n*n]
  void gridding(const double2* d_data, int batch, double2* d_out);
  void images(const double2* d_data, int batch, double2* d_x);
  void rings(const double2* d_coil, int n_part, int ncoils, int ring, const double* zsens, double2* d_out);
};

}  // namespace mrsim
