// spiral_recon.cu — the spiral reconstruction on the device, FP64 (reference `SpiralRecon`,
// grid_recon.rs:54-325): Pipe-Menon density weights, the centre normalization, the window, the
// image band, the power iteration for lambda_hi, the Chebyshev semi-iteration of the
// density-weighted least squares, its residual check, and the ring Roemer combine.
//
// The normal operator Q A^H W A Q is applied as what it is, a Toeplitz convolution on the n x n
// grid: (A^H W A x)(X) = sum_X' x(X') T(X - X') with T(d) = n^-4 sum_j w_j e^{-i2pi k_j.d/n},
// |d| < n per axis.  T is one type-1 NUFFT (period 2n, points 2k_j) at setup; each application is
// then a 2n x 2n FFT pair and a pointwise product (circulant embedding), instead of a type-2 and a
// type-1 NUFFT over every sample.  It is the same linear operator as the reference's NUFFT pair
// to the NUFFT's tolerance (1e-12); everything is FP64.  Batches of images (partitions x coil
// elements) share the trajectory and run as one batch through every kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "driver.h"
#include "host_tables.h"
#include "mrsim_internal.h"
#include "nufft.h"
#include "spiral.h"
#include "spiral_recon.h"

namespace mrsim {

namespace {

// in-place line FFTs along one axis of `lines` lines (see fft2); per line CTA, batch on grid.y
template <class V>
__global__ void fft_lines_kernel(V* __restrict__ data, int n, int logn, size_t es, size_t ls, size_t bs,
                                 const V* __restrict__ tw, int sign) {
  extern __shared__ __align__(16) unsigned char fl_smem[];
  V* buf = reinterpret_cast<V*>(fl_smem);
  V* base = data + blockIdx.y * bs + blockIdx.x * ls;
  for (int i = threadIdx.x; i < n; i += blockDim.x) buf[__brev(i) >> (32 - logn)] = base[(size_t)i * es];
  __syncthreads();
  for (int s = 1; s <= logn; ++s) {
    const int m = 1 << s, h = m >> 1;
    for (int t = threadIdx.x; t < n / 2; t += blockDim.x) {
      const int i0 = (t / h) * m + t % h, i1 = i0 + h;
      V w = tw[(size_t)(t % h) * (n / m)];
      if (sign > 0) w.y = -w.y;
      const V a = buf[i0], b = buf[i1];
      const double bx = b.x * w.x - b.y * w.y, by = b.x * w.y + b.y * w.x;
      buf[i0] = make_double2(a.x + bx, a.y + by);
      buf[i1] = make_double2(a.x - bx, a.y - by);
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) base[(size_t)i * es] = buf[i];
}

__global__ void dft_lines_kernel(double2* __restrict__ data, int n, size_t es, size_t ls, size_t bs,
                                 const double2* __restrict__ tw, int sign) {
  extern __shared__ __align__(16) unsigned char dl_smem[];
  double2* buf = reinterpret_cast<double2*>(dl_smem);
  double2* base = data + blockIdx.y * bs + blockIdx.x * ls;
  for (int i = threadIdx.x; i < n; i += blockDim.x) buf[i] = base[(size_t)i * es];
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double ar = 0, ai = 0;
    for (int j = 0; j < n; ++j) {
      double2 w = tw[((long long)j * k) % n];
      if (sign > 0) w.y = -w.y;
      ar = fma(buf[j].x, w.x, fma(-buf[j].y, w.y, ar));
      ai = fma(buf[j].x, w.y, fma(buf[j].y, w.x, ai));
    }
    base[(size_t)k * es] = make_double2(ar, ai);
  }
}

void fft_lines(double2* data, int n, int lines, size_t es, size_t ls, size_t bs, int batch, const double2* tw,
               int sign, cudaStream_t st) {
  const size_t smem = sizeof(double2) * n;
  dim3 g(lines, batch);
  if ((n & (n - 1)) == 0) {
    int logn = 0;
    while ((1 << logn) < n) ++logn;
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(fft_lines_kernel<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    fft_lines_kernel<double2><<<g, std::min(256, std::max(32, n / 2)), smem, st>>>(data, n, logn, es, ls, bs, tw, sign);
  } else {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(dft_lines_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dft_lines_kernel<<<g, std::min(256, n), smem, st>>>(data, n, es, ls, bs, tw, sign);
  }
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// wts[b][j] = d[b][j] * win[j] * w[j] * sc  (win may be NULL: 1)
__global__ void weight_samples_kernel(const double2* __restrict__ d, const double* __restrict__ win,
                                      const double* __restrict__ w, double sc, int npts, double2* __restrict__ out) {
  const int b = blockIdx.y;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npts; j += gridDim.x * blockDim.x) {
    double2 v = d[(size_t)b * npts + j];
    if (win) {
      v.x *= win[j];
      v.y *= win[j];
    }
    out[(size_t)b * npts + j] = make_double2(v.x * w[j] * sc, v.y * w[j] * sc);
  }
}

// zero outside the band and scale by s (between the forward and inverse FFT of the projection)
__global__ void band_mask_kernel(double2* __restrict__ g, const unsigned char* __restrict__ keep, int nn, double s) {
  const int b = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    double2& v = g[(size_t)b * nn + i];
    v = keep[i] ? make_double2(v.x * s, v.y * s) : make_double2(0.0, 0.0);
  }
}

// n x n image -> zero-padded 2n x 2n grid
__global__ void pad_kernel(const double2* __restrict__ x, int n, double2* __restrict__ g) {
  const int b = blockIdx.y, m = 2 * n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m * m; i += gridDim.x * blockDim.x) {
    const int c0 = i % m, c1 = i / m;
    g[(size_t)b * m * m + i] =
        (c0 < n && c1 < n) ? x[(size_t)b * n * n + c0 + (size_t)n * c1] : make_double2(0.0, 0.0);
  }
}

// g *= tf * s (the circulant's transform; s the inverse transform's 1/(2n)^2)
__global__ void toeplitz_mul_kernel(double2* __restrict__ g, const double2* __restrict__ tf, int mm, double s) {
  const int b = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < mm; i += gridDim.x * blockDim.x) {
    const double2 p = cmul(g[(size_t)b * mm + i], tf[i]);
    g[(size_t)b * mm + i] = make_double2(p.x * s, p.y * s);
  }
}

__global__ void crop_kernel(const double2* __restrict__ g, int n, double2* __restrict__ x) {
  const int b = blockIdx.y, m = 2 * n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * n; i += gridDim.x * blockDim.x) {
    const int c0 = i % n, c1 = i / n;
    x[(size_t)b * n * n + i] = g[(size_t)b * m * m + c0 + (size_t)m * c1];
  }
}

// circulant arrangement of T(d), d = -n..n-1 per axis (type-1 layout (d + n) + 2n (d1 + n)):
// position d mod 2n
__global__ void circulant_kernel(const double2* __restrict__ t, int n, double2* __restrict__ c) {
  const int m = 2 * n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m * m; i += gridDim.x * blockDim.x) {
    const int j0 = i % m, j1 = i / m;
    const int c0 = (j0 + n) % m, c1 = (j1 + n) % m;
    c[c0 + (size_t)m * c1] = t[i];
  }
}

// Chebyshev step (grid_recon.rs:256-266): x += dir; r -= nd; dir = dir c1 + r c2
__global__ void cheb_update_kernel(double2* __restrict__ x, double2* __restrict__ r, double2* __restrict__ dir,
                                   const double2* __restrict__ nd, size_t total, double c1, double c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const double2 dv = dir[i];
    double2 xv = x[i];
    xv.x += dv.x;
    xv.y += dv.y;
    x[i] = xv;
    double2 rv = r[i];
    rv.x -= nd[i].x;
    rv.y -= nd[i].y;
    r[i] = rv;
    dir[i] = make_double2(dv.x * c1 + rv.x * c2, dv.y * c1 + rv.y * c2);
  }
}

__global__ void scale_kernel(const double2* __restrict__ a, double s, size_t total, double2* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
    out[i] = make_double2(a[i].x * s, a[i].y * s);
}

// per-batch sum of |v|^2 (one CTA per batch item, fixed order: deterministic)
__global__ void __launch_bounds__(256) sumsq_kernel(const double2* __restrict__ v, int len, double* __restrict__ out) {
  __shared__ double part[256];
  const int b = blockIdx.x;
  double s = 0.0;
  for (int i = threadIdx.x; i < len; i += blockDim.x) {
    const double2 x = v[(size_t)b * len + i];
    s = fma(x.x, x.x, fma(x.y, x.y, s));
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h) part[threadIdx.x] += part[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[b] = part[0];
}

// Pipe-Menon update: w /= |back|
__global__ void pipe_menon_kernel(double* __restrict__ w, const double2* __restrict__ back, int npts) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npts; j += gridDim.x * blockDim.x)
    w[j] /= hypot(back[j].x, back[j].y);
}

__global__ void real_to_complex_kernel(const double* __restrict__ w, double s, int npts, double2* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npts; j += gridDim.x * blockDim.x)
    out[j] = make_double2(w[j] * s, 0.0);
}

// the centre pixel of a constant object's samples: w_j D(kx_j) D(ky_j), D(k) = (1/n) sum_x
// e^{i2pi k (x - n/2)/n} (`dirichlet`, grid_recon.rs:68-75)
__global__ void dirichlet_kernel(const double* __restrict__ k, const double* __restrict__ w, int npts, int n,
                                 double2* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npts; j += gridDim.x * blockDim.x) {
    double2 d[2];
    for (int a = 0; a < 2; ++a) {
      double re = 0.0, im = 0.0;
      for (int x = 0; x < n; ++x) {
        double s, c;
        sincos(6.283185307179586 * k[2 * j + a] * (double)(x - n / 2) / (double)n, &s, &c);
        re += c;
        im += s;
      }
      d[a] = make_double2(re / n, im / n);
    }
    const double2 p = cmul(d[0], d[1]);
    out[j] = make_double2(p.x * w[j], p.y * w[j]);
  }
}

// element data of a ring: out[p][a][j] = sum_r zsens[p][r ring + a] coil[p][r ring + a][j]
__global__ void ring_data_kernel(const double2* __restrict__ coil, const double* __restrict__ zsens, int ncoils,
                                 int ring, int npts, double2* __restrict__ out) {
  const int p = blockIdx.z, a = blockIdx.y, rows = ncoils / ring;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npts; j += gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int r = 0; r < rows; ++r) {
      const int q = r * ring + a;
      const double z = zsens[(size_t)p * ncoils + q];
      const double2 c = coil[((size_t)p * ncoils + q) * npts + j];
      re += c.x * z;
      im += c.y * z;
    }
    out[((size_t)p * ring + a) * npts + j] = make_double2(re, im);
  }
}

// ring Roemer combine (grid_recon.rs:296-320): sum_a img_a s_a / max(sum_a s_a^2 z2_a, 1e-12)
__global__ void ring_combine_kernel(const double2* __restrict__ img, const double* __restrict__ sens,
                                    const double* __restrict__ z2, int ring, int nn, double2* __restrict__ out) {
  const int p = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    double wr = 0.0, wi = 0.0, ss = 0.0;
    for (int a = 0; a < ring; ++a) {
      const double s = sens[(size_t)a * nn + i];
      const double2 v = img[((size_t)p * ring + a) * nn + i];
      wr += v.x * s;
      wi += v.y * s;
      ss += s * s * z2[(size_t)p * ring + a];
    }
    const double d = fmax(ss, 1e-12);
    out[(size_t)p * nn + i] = make_double2(wr / d, wi / d);
  }
}

dim3 grid1(size_t n, int batch = 1) { return dim3((unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 4096)), batch); }

}  // namespace

// ---- SpiralRecon ------------------------------------------------------------------------------------
SpiralRecon::SpiralRecon(mrsim_context* c, const double* k, int npts_, int n_, const mrsim_acquisition& win_acq,
                         int iterations_, double kappa_, bool band_limited)
    : ctx(c), n(n_), npts(npts_), iterations(iterations_), kappa(kappa_), band(band_limited) {
  cudaStream_t st = ctx->stream;
  if (n <= 0 || n > 1024) fail("spiral reconstruction matrix must be in 1..1024");
  if (npts <= 0) fail("a spiral reconstruction needs samples");
  if (iterations < 0 || !(kappa > 1.0)) fail("Chebyshev iterations must be >= 0 and the interval ratio above 1");
  const int h = n / 2;
  g = make_nufft<double>(A, n, n, -h, -h, n, n, 1e-12, st);
  tw_n = (const double2*)upload_twiddles<double>(A, n, st);
  tw_2n = (const double2*)upload_twiddles<double>(A, 2 * n, st);
  k_host.assign(k, k + 2 * (size_t)npts);
  d_k = (double*)A.upload(k, (size_t)npts * 2 * 8, st);
  bins_k = nufft_bins2(A, g.nf0, g.nf1, g.w, k, npts, st);
  d_w = (double*)A.alloc((size_t)npts * 8);
  DevArena T;
  // Pipe-Menon (grid_recon.rs:54-66)
  {
    std::vector<double> ones(npts, 1.0);
    MRSIM_CUDA(cudaMemcpyAsync(d_w, ones.data(), (size_t)npts * 8, cudaMemcpyHostToDevice, st));
    double2* wc = (double2*)T.alloc((size_t)npts * 16);
    double2* img = (double2*)T.alloc((size_t)n * n * 16);
    double2* back = (double2*)T.alloc((size_t)npts * 16);
    double2* work = (double2*)T.alloc((size_t)g.nf0 * g.nf1 * 16);
    for (int it = 0; it < kDcfIterations; ++it) {
      real_to_complex_kernel<<<grid1(npts), 256, 0, st>>>(d_w, 1.0, npts, wc);
      nufft_type1<double>(g, d_k, npts, bins_k, wc, 1, npts, img, (size_t)n * n, work, -1, st);
      nufft_type2<double>(g, img, 1, (size_t)n * n, d_k, npts, back, npts, work, 1, nullptr, st);
      pipe_menon_kernel<<<grid1(npts), 256, 0, st>>>(d_w, back, npts);
    }
    MRSIM_CUDA(cudaGetLastError());
    // the centre normalization: a constant object grids to 1 at the image centre
    dirichlet_kernel<<<grid1(npts), 256, 0, st>>>(d_k, d_w, npts, n, back);
    std::vector<double2> cs(npts);
    MRSIM_CUDA(cudaMemcpyAsync(cs.data(), back, (size_t)npts * 16, cudaMemcpyDeviceToHost, st));
    w_host.resize(npts);
    MRSIM_CUDA(cudaMemcpyAsync(w_host.data(), d_w, (size_t)npts * 8, cudaMemcpyDeviceToHost, st));
    MRSIM_CUDA(cudaStreamSynchronize(st));
    double cre = 0.0;
    for (int j = 0; j < npts; ++j) cre += cs[j].x;
    const double s = 1.0 / cre;
    for (double& x : w_host) x *= s;
    MRSIM_CUDA(cudaMemcpyAsync(d_w, w_host.data(), (size_t)npts * 8, cudaMemcpyHostToDevice, st));
  }
  // window per sample and the band
  {
    std::vector<double> win(npts);
    double radius = 0.0;
    for (int j = 0; j < npts; ++j) {
      win[j] = window_at(win_acq, k[2 * j] / n, k[2 * j + 1] / n);
      radius = std::max(radius, std::hypot(k[2 * j], k[2 * j + 1]));
    }
    d_win = (double*)A.upload(win.data(), (size_t)npts * 8, st);
    if (band) {
      const int half_up = (n + 1) / 2;
      auto sgn = [&](int i) { return i < half_up ? (double)i : (double)i - n; };
      std::vector<unsigned char> keep((size_t)n * n);
      for (int i = 0; i < n * n; ++i) keep[i] = std::hypot(sgn(i % n), sgn(i / n)) <= radius ? 1 : 0;
      d_keep = (unsigned char*)A.upload(keep.data(), keep.size(), st);
    }
  }
  // the Toeplitz kernel: T(d) = sc^2 sum_j w_j e^{-i2pi k_j.d/n}, d = -n..n-1, as a type 1 of
  // period 2n at the points 2k_j; then its circulant's transform
  {
    const int m = 2 * n;
    NufftGridT<double> g2 = make_nufft<double>(T, m, m, -n, -n, m, m, 1e-12, st);
    std::vector<double> u2(2 * (size_t)npts);
    for (size_t i = 0; i < u2.size(); ++i) u2[i] = 2.0 * k[i];
    const double* du2 = (const double*)T.upload(u2.data(), u2.size() * 8, st);
    const double sc = 1.0 / ((double)n * n);
    double2* wc = (double2*)T.alloc((size_t)npts * 16);
    real_to_complex_kernel<<<grid1(npts), 256, 0, st>>>(d_w, sc * sc, npts, wc);
    double2* tmodes = (double2*)T.alloc((size_t)m * m * 16);
    double2* work = (double2*)T.alloc((size_t)g2.nf0 * g2.nf1 * 16);
    const NufftBins bins2 = nufft_bins2(T, g2.nf0, g2.nf1, g2.w, u2.data(), npts, st);
    nufft_type1<double>(g2, du2, npts, bins2, wc, 1, npts, tmodes, (size_t)m * m, work, -1, st);
    d_tf = (double2*)A.alloc((size_t)m * m * 16);
    circulant_kernel<<<grid1((size_t)m * m), 256, 0, st>>>(tmodes, n, d_tf);
    fft_lines(d_tf, m, m, 1, m, (size_t)m * m, 1, tw_2n, -1, st);
    fft_lines(d_tf, m, m, m, 1, (size_t)m * m, 1, tw_2n, -1, st);
    MRSIM_CUDA(cudaGetLastError());
  }
  // the power iteration (grid_recon.rs:178-197) from the reference's fixed pseudo-random start
  {
    uint64_t s = 0x9E3779B97F4A7C15ull;
    auto rnd = [&]() {
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      return (double)(s >> 11) / (double)(1ull << 53) - 0.5;
    };
    std::vector<double2> v0((size_t)n * n);
    for (auto& c : v0) {
      c.x = rnd();
      c.y = rnd();
    }
    Scratch sc = scratch(T, 1);
    double2* v = (double2*)T.upload(v0.data(), v0.size() * 16, st);
    double2* u = (double2*)T.alloc(v0.size() * 16);
    double* d_ss = (double*)T.alloc(16);
    double lam = 0.0, ss[2];
    power_iterations = 0;
    for (int it = 0; it < kPowerIterations; ++it) {
      sumsq_kernel<<<1, 256, 0, st>>>(v, n * n, d_ss);
      normal(v, u, 1, sc, st);
      sumsq_kernel<<<1, 256, 0, st>>>(u, n * n, d_ss + 1);
      MRSIM_CUDA(cudaMemcpyAsync(ss, d_ss, 16, cudaMemcpyDeviceToHost, st));
      MRSIM_CUDA(cudaStreamSynchronize(st));
      const double nv = std::sqrt(ss[0]), nu = std::sqrt(ss[1]);
      const double next = nu / nv;
      scale_kernel<<<grid1((size_t)n * n), 256, 0, st>>>(u, 1.0 / nu, (size_t)n * n, v);
      const bool done = std::fabs(next - lam) <= 1e-10 * next;
      lam = next;
      ++power_iterations;
      if (done) break;
    }
    lambda_hi = kLambdaMargin * lam;
    MRSIM_CUDA(cudaStreamSynchronize(st));
  }
}

SpiralRecon::Scratch SpiralRecon::scratch(DevArena& T, int batch) const {
  Scratch s;
  s.pad = (double2*)T.alloc((size_t)batch * 4 * n * n * 16);
  s.tmp = (double2*)T.alloc((size_t)batch * n * n * 16);
  return s;
}

// Q x (in place on `x`; the identity without a band): FFT, mask, scale 1/n^2, inverse FFT
void SpiralRecon::project(double2* x, int batch, cudaStream_t st) const {
  if (!band) return;
  const size_t nn = (size_t)n * n;
  fft_lines(x, n, n, 1, n, nn, batch, tw_n, -1, st);
  fft_lines(x, n, n, n, 1, nn, batch, tw_n, -1, st);
  band_mask_kernel<<<grid1(nn, batch), 256, 0, st>>>(x, d_keep, (int)nn, 1.0 / (double)nn);
  fft_lines(x, n, n, n, 1, nn, batch, tw_n, 1, st);
  fft_lines(x, n, n, 1, n, nn, batch, tw_n, 1, st);
}

// out = Q A^H W A Q x  (x is left unchanged)
void SpiralRecon::normal(const double2* x, double2* out, int batch, const Scratch& s, cudaStream_t st) const {
  const size_t nn = (size_t)n * n;
  const int m = 2 * n;
  const size_t mm = (size_t)m * m;
  MRSIM_CUDA(cudaMemcpyAsync(s.tmp, x, (size_t)batch * nn * 16, cudaMemcpyDeviceToDevice, st));
  project(s.tmp, batch, st);
  pad_kernel<<<grid1(mm, batch), 256, 0, st>>>(s.tmp, n, s.pad);
  fft_lines(s.pad, m, n, 1, m, mm, batch, tw_2n, -1, st);  // rows n..2n-1 are zero
  fft_lines(s.pad, m, m, m, 1, mm, batch, tw_2n, -1, st);
  toeplitz_mul_kernel<<<grid1(mm, batch), 256, 0, st>>>(s.pad, d_tf, (int)mm, 1.0 / (double)mm);
  fft_lines(s.pad, m, m, m, 1, mm, batch, tw_2n, 1, st);
  fft_lines(s.pad, m, n, 1, m, mm, batch, tw_2n, 1, st);  // only the rows the crop keeps
  crop_kernel<<<grid1(nn, batch), 256, 0, st>>>(s.pad, n, out);
  project(out, batch, st);
}

void SpiralRecon::sumsq(const double2* v, int batch, double* out, cudaStream_t st) const {
  DevArena T;
  double* d = (double*)T.alloc((size_t)batch * 8);
  sumsq_kernel<<<batch, 256, 0, st>>>(v, n * n, d);
  MRSIM_CUDA(cudaMemcpyAsync(out, d, (size_t)batch * 8, cudaMemcpyDeviceToHost, st));
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

// `gridding` (grid_recon.rs:231-236): n^2 A^H W d, no window
void SpiralRecon::gridding(const double2* d_data, int batch, double2* d_out) {
  cudaStream_t st = ctx->stream;
  DevArena T;
  const double sc = 1.0 / ((double)n * n);
  double2* wts = (double2*)T.alloc((size_t)batch * npts * 16);
  weight_samples_kernel<<<grid1(npts, batch), 256, 0, st>>>(d_data, nullptr, d_w, sc, npts, wts);
  double2* work = (double2*)T.alloc((size_t)batch * g.nf0 * g.nf1 * 16);
  nufft_type1<double>(g, d_k, npts, bins_k, wts, batch, npts, d_out, (size_t)n * n, work, -1, st);
  scale_kernel<<<grid1((size_t)batch * n * n), 256, 0, st>>>(d_out, (double)n * n, (size_t)batch * n * n, d_out);
  MRSIM_CUDA(cudaGetLastError());
  MRSIM_CUDA(cudaStreamSynchronize(st));  // T's buffers are freed on return
}

// `image` (grid_recon.rs:238-275) for a batch of sample sets
void SpiralRecon::images(const double2* d_data, int batch, double2* d_x) {
  cudaStream_t st = ctx->stream;
  const size_t nn = (size_t)n * n;
  DevArena T;
  const double sc = 1.0 / ((double)n * n);
  double2* r = (double2*)T.alloc((size_t)batch * nn * 16);
  double2* dir = (double2*)T.alloc((size_t)batch * nn * 16);
  double2* nd = (double2*)T.alloc((size_t)batch * nn * 16);
  {
    DevArena W;
    double2* wts = (double2*)W.alloc((size_t)batch * npts * 16);
    weight_samples_kernel<<<grid1(npts, batch), 256, 0, st>>>(d_data, d_win, d_w, sc, npts, wts);
    double2* work = (double2*)W.alloc((size_t)batch * g.nf0 * g.nf1 * 16);
    nufft_type1<double>(g, d_k, npts, bins_k, wts, batch, npts, r, nn, work, -1, st);
    project(r, batch, st);
    MRSIM_CUDA(cudaStreamSynchronize(st));  // W's buffers are freed on return
  }
  std::vector<double> r0(batch), rn(batch);
  sumsq(r, batch, r0.data(), st);
  const double hi = lambda_hi, lo = lambda_hi / kappa;
  const double theta = (hi + lo) / 2.0, delta = (hi - lo) / 2.0;
  const double sigma1 = theta / delta;
  double rho = 1.0 / sigma1;
  MRSIM_CUDA(cudaMemsetAsync(d_x, 0, (size_t)batch * nn * 16, st));
  scale_kernel<<<grid1((size_t)batch * nn), 256, 0, st>>>(r, 1.0 / theta, (size_t)batch * nn, dir);
  Scratch s = scratch(T, batch);
  for (int it = 0; it < iterations; ++it) {
    normal(dir, nd, batch, s, st);
    const double rho1 = 1.0 / (2.0 * sigma1 - rho);
    cheb_update_kernel<<<grid1((size_t)batch * nn), 256, 0, st>>>(d_x, r, dir, nd, (size_t)batch * nn, rho1 * rho,
                                                                  2.0 * rho1 / delta);
    rho = rho1;
  }
  MRSIM_CUDA(cudaGetLastError());
  sumsq(r, batch, rn.data(), st);
  for (int b = 0; b < batch; ++b) {
    const double a = std::sqrt(r0[b]), z = std::sqrt(rn[b]);
    if (!(z <= (1.0 + 1e-6) * a + 1e-300)) {
      char buf[320];
      std::snprintf(buf, sizeof buf,
                    "spiral reconstruction: the residual grew from %e to %e; the normal operator has an eigenvalue "
                    "above the estimated %e",
                    a, z, lambda_hi);
      fail(buf);
    }
  }
}

// `reconstruct_rings` (grid_recon.rs:285-320) for P partitions at once
void SpiralRecon::rings(const double2* d_coil, int n_part, int ncoils, int ring, const double* zsens,
                        double2* d_out) {
  cudaStream_t st = ctx->stream;
  if (ring < 1 || ncoils % ring != 0) fail("the coils do not divide into rings of " + std::to_string(ring));
  const int rows = ncoils / ring;
  const size_t nn = (size_t)n * n;
  DevArena T;
  double* dz = (double*)T.upload(zsens, (size_t)n_part * ncoils * 8, st);
  std::vector<double> z2((size_t)n_part * ring, 0.0), sens((size_t)ring * nn);
  for (int p = 0; p < n_part; ++p)
    for (int a = 0; a < ring; ++a)
      for (int r = 0; r < rows; ++r) {
        const double z = zsens[(size_t)p * ncoils + r * ring + a];
        z2[(size_t)p * ring + a] += z * z;
      }
  for (int a = 0; a < ring; ++a)
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) sens[(size_t)a * nn + x + (size_t)n * y] = coil_sensitivity(a, ring, x, y, n, n);
  double* dz2 = (double*)T.upload(z2.data(), z2.size() * 8, st);
  double* dsens = (double*)T.upload(sens.data(), sens.size() * 8, st);
  const int batch = n_part * ring;
  double2* data = (double2*)T.alloc((size_t)batch * npts * 16);
  dim3 rg((unsigned)std::min(4096, (npts + 255) / 256), ring, n_part);
  ring_data_kernel<<<rg, 256, 0, st>>>(d_coil, dz, ncoils, ring, npts, data);
  double2* imgs = (double2*)T.alloc((size_t)batch * nn * 16);
  for (int b0 = 0; b0 < batch; b0 += kMaxBatch) {
    const int nb = std::min(kMaxBatch, batch - b0);
    images(data + (size_t)b0 * npts, nb, imgs + (size_t)b0 * nn);
  }
  ring_combine_kernel<<<grid1(nn, n_part), 256, 0, st>>>(imgs, dsens, dz2, ring, (int)nn, d_out);
  MRSIM_CUDA(cudaGetLastError());
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

}  // namespace mrsim
