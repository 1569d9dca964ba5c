// hermitian_solve.cuh — one CTA solves a dense complex system [H | B] in place (n x (n + nrhs),
// row-major, FP64) by Gaussian elimination with partial pivoting, every right-hand side at once
// (`solve_hermitian`, kspace.rs:1455-1491).  The pivots depend on H alone, so each column of B
// goes through the reference's sequence of operations for that right-hand side; the products and
// sums use the non-contracting FP64 intrinsics, so every value rounds as the reference's separate
// multiply and add do, whatever contraction the including file is compiled with.
#pragma once

#include <cuda_runtime.h>

namespace mrsim {

struct HsCd {
  double re, im;
};
__device__ __forceinline__ HsCd hs_mul(HsCd a, HsCd b) {
  return {__dsub_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im)),
          __dadd_rn(__dmul_rn(a.re, b.im), __dmul_rn(a.im, b.re))};
}
__device__ __forceinline__ double hs_abs(double2 h) {
  return __dsqrt_rn(__dadd_rn(__dmul_rn(h.x, h.x), __dmul_rn(h.y, h.y)));
}
__device__ __forceinline__ HsCd hs_recip(HsCd d) {
  const double m2 = __dadd_rn(__dmul_rn(d.re, d.re), __dmul_rn(d.im, d.im));
  if (m2 < 1e-18) return {0.0, 0.0};
  return {__ddiv_rn(d.re, m2), __ddiv_rn(-d.im, m2)};
}

// W: [n][n + nrhs] in global memory; fre/fim: n doubles each; xs: nrhs * 2n doubles (solution
// scratch); out: [nrhs][n] complex f32.  red_v / red_i: blockDim.x-entry shared arrays.  Every
// thread of the block calls it.
__device__ inline void hermitian_solve_block(double2* W, int n, int nrhs, double* fre, double* fim, double* xs,
                                             float2* out, double* red_v, int* red_i) {
  const int cols = n + nrhs;
  for (int col = 0; col < n; ++col) {
    // pivot: the first row of largest |h[r][col]| among r >= col (the reference keeps `col`
    // unless a later row is strictly larger)
    double best = -1.0;
    int bi = col;
    for (int r = col + (int)threadIdx.x; r < n; r += blockDim.x) {
      const double m = hs_abs(W[(size_t)r * cols + col]);
      if (m > best) {
        best = m;
        bi = r;
      }
    }
    red_v[threadIdx.x] = best;
    red_i[threadIdx.x] = bi;
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = red_v[0];
      int p = red_i[0];
      for (int t = 1; t < (int)blockDim.x; ++t)
        if (red_v[t] > b || (red_v[t] == b && red_i[t] < p)) {
          b = red_v[t];
          p = red_i[t];
        }
      if (!(b > hs_abs(W[(size_t)col * cols + col]))) p = col;
      red_i[0] = p;
    }
    __syncthreads();
    const int piv = red_i[0];
    if (piv != col)
      for (int c = threadIdx.x; c < cols; c += blockDim.x) {
        const double2 a = W[(size_t)col * cols + c];
        W[(size_t)col * cols + c] = W[(size_t)piv * cols + c];
        W[(size_t)piv * cols + c] = a;
      }
    __syncthreads();
    const double2 dd = W[(size_t)col * cols + col];
    const HsCd dinv = hs_recip({dd.x, dd.y});
    for (int r = col + 1 + (int)threadIdx.x; r < n; r += blockDim.x) {
      const double2 h = W[(size_t)r * cols + col];
      const HsCd f = hs_mul({h.x, h.y}, dinv);
      fre[r] = f.re;
      fim[r] = f.im;
    }
    __syncthreads();
    const int rows = n - col - 1, width = cols - col;
    for (int e = threadIdx.x; e < rows * width; e += blockDim.x) {
      const int r = col + 1 + e / width, c = col + e % width;
      const double2 p = W[(size_t)col * cols + c];
      const HsCd s = hs_mul({fre[r], fim[r]}, {p.x, p.y});
      double2 h = W[(size_t)r * cols + c];
      h.x = __dsub_rn(h.x, s.re);
      h.y = __dsub_rn(h.y, s.im);
      W[(size_t)r * cols + c] = h;
    }
    __syncthreads();
  }
  // back substitution, one thread per right-hand side
  for (int q = threadIdx.x; q < nrhs; q += blockDim.x) {
    double* xre = xs + (size_t)q * 2 * n;
    double* xim = xre + n;
    for (int col = n - 1; col >= 0; --col) {
      const double2 b = W[(size_t)col * cols + n + q];
      HsCd s = {b.x, b.y};
      for (int c = col + 1; c < n; ++c) {
        const double2 h = W[(size_t)col * cols + c];
        const HsCd t = hs_mul({h.x, h.y}, {xre[c], xim[c]});
        s.re = __dsub_rn(s.re, t.re);
        s.im = __dsub_rn(s.im, t.im);
      }
      const double2 d = W[(size_t)col * cols + col];
      const HsCd x = hs_mul(s, hs_recip({d.x, d.y}));
      xre[col] = x.re;
      xim[col] = x.im;
    }
    for (int f = 0; f < n; ++f) out[(size_t)q * n + f] = make_float2((float)xre[f], (float)xim[f]);
  }
}

}  // namespace mrsim
