// spiral.h — host entry points of the device NUFFT pair and spiral forwards (see spiral.cpp).
#pragma once

#include <cstdint>

#include "driver.h"
#include "mrsim_internal.h"
#include "nufft.h"

namespace mrsim {

int nufft_width(double tol);
template <class R>
NufftGridT<R> make_nufft(DevArena& A, int n0, int n1, int m_lo0, int m_lo1, int m_out0, int m_out1, double tol,
                         cudaStream_t st);
template <class R>
const void* upload_twiddles(DevArena& A, int n, cudaStream_t st);
void nufft1_host(mrsim_context* ctx, int n, int k_lo, int n_out, double tol, const double* pos, int npos,
                 const double* weights, int nw, double* out);
void nufft2_host(mrsim_context* ctx, int type, int n0, int n1, int m_lo0, int m_lo1, int m_out0, int m_out1, double tol,
                 const double* u, int npts, const float* in, int sign, float* out);
void spiral_exact_host(mrsim_context* ctx, const mrsim_slice_input& inp, const mrsim_acquisition& acq, int coil,
                       int ncoils, const double* k, const double* tau_ms, int npts, const double* log_amp, float* out);
struct SegmentedInfo {
  int l = 0, m = 0;
  double bound = 0, b_sum = 0, grid_err = 0;
};
SegmentedInfo spiral_segmented_host(mrsim_context* ctx, const mrsim_slice_input& inp, const mrsim_acquisition& acq,
                                    int coil, int ncoils, const double* k, const int64_t* tau_idx, int npts,
                                    const double* tau_ms, int ntau, double t_ms, const double rect_d[2],
                                    const double rect_f[2], const double* log_amp, bool decay_inside, float* out);

}  // namespace mrsim
