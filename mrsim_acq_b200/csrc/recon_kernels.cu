// recon_kernels.cu — the reconstruction of one slice's coils on the device (reference
// `reconstruct_coils_full`, kspace.rs:1301-1378): GRAPPA calibration (FP64 normal equations and
// pivoted Gaussian elimination, `GrappaKernel::fit` kspace.rs:1547-1599 + `solve_hermitian`
// :1457-1491), GRAPPA apply (kspace.rs:1605-1632), the radial window (kspace.rs:1327-1342), the
// centred inverse 2D DFT (`inverse_2d`, kspace.rs:1428-1453) and the Roemer combine
// (kspace.rs:1343-1373).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "hermitian_solve.cuh"
#include "recon_kernels.h"

namespace mrsim {

namespace {

// The source feature i of GRAPPA at readout kx: lines s0/s1, readout offsets -1/0/+1 (wrapped),
// every coil; layout (line*3 + point)*nc + coil (`grappa_feature`, kspace.rs:1526-1538).
__device__ __forceinline__ float2 feature(const float2* __restrict__ k, int nx, int ny, int nc, int s0, int s1,
                                          int kx, int i) {
  int ci = i % nc;
  int p = i / nc;
  int li = p / 3, ki = p % 3;
  int kxs = kx + ki - 1;
  kxs = kxs < 0 ? kxs + nx : (kxs >= nx ? kxs - nx : kxs);
  int sl = li == 0 ? s0 : s1;
  return k[(size_t)ci * nx * ny + (size_t)sl * nx + kxs];
}

// One thread per entry of [A^H A | A^H b]: FP64 sums over the reference band in the reference's
// order (band line, then readout point).
__global__ void grappa_normal_kernel(const GrappaSystem* __restrict__ sys) {
  const GrappaSystem& S = sys[blockIdx.y];
  const int nf = 6 * S.nc;
  const int cols = nf + S.nc;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nf * cols) return;
  const int i = e / cols, j = e % cols;
  double ar = 0.0, ai = 0.0;
  for (int b = S.acs_lo; b < S.acs_hi; ++b) {
    const int s0 = b, s1 = b + S.accel, tgt = b + S.d;
    if (s1 > S.acs_hi || tgt > S.acs_hi || !(S.lines[s0] && S.lines[s1] && S.lines[tgt])) continue;
    for (int kx = 0; kx < S.nx; ++kx) {
      const float2 fi = feature(S.k, S.nx, S.ny, S.nc, s0, s1, kx, i);
      float2 fj;
      if (j < nf)
        fj = feature(S.k, S.nx, S.ny, S.nc, s0, s1, kx, j);
      else
        fj = S.k[(size_t)(j - nf) * S.nx * S.ny + (size_t)tgt * S.nx + kx];
      const double xr = fi.x, xi = -(double)fi.y, yr = fj.x, yi = fj.y;
      ar += xr * yr - xi * yi;
      ai += xr * yi + xi * yr;
    }
  }
  S.work[(size_t)i * cols + j] = make_double2(ar, ai);
}

// One CTA per system: scale by the mean diagonal, add the Tikhonov term, then the pivoted
// Gaussian elimination of [H | B] with every right-hand side at once (hermitian_solve.cuh).
__global__ void __launch_bounds__(256) grappa_solve_kernel(const GrappaSystem* __restrict__ sys, double lambda) {
  const GrappaSystem& S = sys[blockIdx.x];
  const int nf = 6 * S.nc, nc = S.nc;
  const int cols = nf + nc;
  double2* W = S.work;
  __shared__ double red_v[256];
  __shared__ int red_i[256];
  __shared__ double s_scale;
  __shared__ int s_zero;
  if (threadIdx.x == 0) {
    double sum = 0.0;
    for (int i = 0; i < nf; ++i) sum += W[(size_t)i * cols + i].x;
    double mean = sum / (double)nf;
    s_zero = !(mean > 0.0);
    s_scale = s_zero ? 0.0 : 1.0 / mean;
  }
  __syncthreads();
  if (s_zero) {
    for (int e = threadIdx.x; e < nc * nf; e += blockDim.x) S.weights[e] = make_float2(0.f, 0.f);
    return;
  }
  const double sc = s_scale;
  for (int e = threadIdx.x; e < nf * cols; e += blockDim.x) {  // (scale, then add: two roundings)
    double2 v = W[e];
    v.x = __dmul_rn(v.x, sc);
    v.y = __dmul_rn(v.y, sc);
    if (e / cols == e % cols) v.x = __dadd_rn(v.x, lambda);
    W[e] = v;
  }
  __syncthreads();
  hermitian_solve_block(W, nf, nc, S.fscratch, S.fscratch + nf, S.fscratch + 2 * nf, S.weights, red_v, red_i);
}

// GRAPPA apply: one thread per (missing line, kx, output coil) of one (unit, echo).
__global__ void grappa_apply_kernel(const ReconJob* __restrict__ jobs, const int4* __restrict__ fills, int n_fills) {
  const ReconJob& J = jobs[blockIdx.y];
  const int nx = J.nx, ny = J.ny, nc = J.nc, nf = 6 * nc;
  const int total = n_fills * nx * nc;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int co = e % nc;
    const int kx = (e / nc) % nx;
    const int4 fl = fills[e / (nc * nx)];  // ky, d, s0, s1
    const float2* w = J.grappa_w + ((size_t)(fl.y - 1) * nc + co) * nf;
    float vr = 0.f, vi = 0.f;
    for (int f = 0; f < nf; ++f) {
      const float2 x = feature(J.k, nx, ny, nc, fl.z, fl.w, kx, f);
      const float2 ww = w[f];
      vr = vr + (ww.x * x.x - ww.y * x.y);
      vi = vi + (ww.x * x.y + ww.y * x.x);
    }
    J.k[(size_t)co * nx * ny + (size_t)fl.x * nx + kx] = make_float2(vr, vi);
  }
}

// Window, inverse DFT and Roemer combine of one (unit, echo): one CTA per block of YB image rows.
// Per coil: h[y][kx] = sum_ky w k[ky][kx] e^{-i2pi (ky-ys)(y-ys)/ny}  (rows y of the block)
//           img[y][x] = sum_kx h[y][kx] e^{-i2pi (kx-xs)(x-xs)/nx}
//           acc[y][x] += s_q(x,y) img[y][x]
// and finally out = acc / max(sum_q s_q^2, 1e-12).  The exponentials come from exact integer
// indices into one table per axis.
__global__ void __launch_bounds__(256) recon_combine_kernel(const ReconJob* __restrict__ jobs, int YB) {
  extern __shared__ float2 sm[];
  const ReconJob& J = jobs[blockIdx.y];
  const int nx = J.nx, ny = J.ny, nc = J.nc;
  const int y0 = blockIdx.x * YB;
  const int ys = ny / 2, xs = nx / 2;
  float2* Ey = sm;              // ny
  float2* Ex = Ey + ny;         // nx
  float2* h = Ex + nx;          // [YB][nx]
  for (int i = threadIdx.x; i < ny; i += blockDim.x) Ey[i] = J.ey_tab[i];
  for (int i = threadIdx.x; i < nx; i += blockDim.x) Ex[i] = J.ex_tab[i];
  const int nout = YB * nx;
  // accumulators: each thread owns outputs o = threadIdx.x + k*blockDim.x
  constexpr int MAXO = 4;  // YB*nx <= 4*256 outputs per CTA (the host picks YB)
  float2 acc[MAXO];
#pragma unroll
  for (int k = 0; k < MAXO; ++k) acc[k] = make_float2(0.f, 0.f);
  __syncthreads();
  for (int q = 0; q < nc; ++q) {
    const float2* kq = J.k + (size_t)q * nx * ny;
    // stage 1
    for (int o = threadIdx.x; o < nout; o += blockDim.x) {
      const int yy = o / nx, kx = o % nx;
      const int y = y0 + yy;
      float hr = 0.f, hi = 0.f;
      if (y < ny) {
        const int yc = y - ys;
        // m = (ky - ys) yc mod ny, stepped: the same table entries without a modulo per term
        const int step = ((yc % ny) + ny) % ny;
        int m = (((-ys * yc) % ny) + ny) % ny;
        for (int ky = 0; ky < ny; ++ky, m = m + step >= ny ? m + step - ny : m + step) {
          float2 v = kq[(size_t)ky * nx + kx];
          if (J.window) {
            float w = J.window[(size_t)ky * nx + kx];
            v.x *= w;
            v.y *= w;
          }
          const float2 t = Ey[m];
          hr = hr + (v.x * t.x - v.y * t.y);
          hi = hi + (v.x * t.y + v.y * t.x);
        }
      }
      h[o] = make_float2(hr, hi);
    }
    __syncthreads();
    // stage 2
#pragma unroll
    for (int k = 0; k < MAXO; ++k) {
      const int o = threadIdx.x + k * blockDim.x;
      if (o >= nout) break;
      const int yy = o / nx, x = o % nx;
      const int y = y0 + yy;
      if (y >= ny) continue;
      const int xc = x - xs;
      float ir = 0.f, ii = 0.f;
      const int step = ((xc % nx) + nx) % nx;
      int m = (((-xs * xc) % nx) + nx) % nx;
      for (int kx = 0; kx < nx; ++kx, m = m + step >= nx ? m + step - nx : m + step) {
        const float2 v = h[yy * nx + kx];
        const float2 t = Ex[m];
        ir = ir + (v.x * t.x - v.y * t.y);
        ii = ii + (v.x * t.y + v.y * t.x);
      }
      if (J.coil_images)
        J.coil_images[(size_t)q * nx * ny + (size_t)y * nx + x] = make_float2(ir, ii);
      const float s = J.sens[(size_t)q * nx * ny + (size_t)y * nx + x];
      acc[k].x = acc[k].x + ir * s;
      acc[k].y = acc[k].y + ii * s;
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < MAXO; ++k) {
    const int o = threadIdx.x + k * blockDim.x;
    if (o >= nout) break;
    const int yy = o / nx, x = o % nx;
    const int y = y0 + yy;
    if (y >= ny) continue;
    const size_t p = (size_t)y * nx + x;
    const float inv = J.inv_ssum[p];
    J.combined[p] = make_float2(acc[k].x * inv, acc[k].y * inv);
  }
}

__global__ void window_copy_kernel(const ReconJob* __restrict__ jobs) {
  const ReconJob& J = jobs[blockIdx.y];
  if (!J.reconstructed) return;  // only the captured slices keep their reconstructed k-space
  const int n = J.nc * J.nx * J.ny;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    float2 v = J.k[e];
    if (J.window) {
      const float w = J.window[e % (J.nx * J.ny)];
      v.x *= w;
      v.y *= w;
    }
    J.reconstructed[e] = v;
  }
}

}  // namespace

void launch_grappa_fit(const GrappaSystem* d_sys, int n_sys, int max_nc, double lambda, cudaStream_t st) {
  if (n_sys <= 0) return;
  const int nf = 6 * max_nc, cols = nf + max_nc;
  dim3 grid((nf * cols + 127) / 128, n_sys);
  grappa_normal_kernel<<<grid, 128, 0, st>>>(d_sys);
  grappa_solve_kernel<<<n_sys, 256, 0, st>>>(d_sys, lambda);
}

void launch_grappa_apply(const ReconJob* d_jobs, int n_jobs, const int4* d_fills, int n_fills, int nx, int nc,
                         cudaStream_t st) {
  if (n_jobs <= 0 || n_fills <= 0) return;
  const int total = n_fills * nx * nc;
  dim3 grid(std::min((total + 255) / 256, 1024), n_jobs);
  grappa_apply_kernel<<<grid, 256, 0, st>>>(d_jobs, d_fills, n_fills);
}

void launch_recon_combine(const ReconJob* d_jobs, int n_jobs, int nx, int ny, bool capture_reconstructed,
                          cudaStream_t st) {
  if (n_jobs <= 0) return;
  if (capture_reconstructed) {
    dim3 g(64, n_jobs);
    window_copy_kernel<<<g, 256, 0, st>>>(d_jobs);
  }
  const int YB = std::max(1, std::min(8, 1024 / nx));
  dim3 grid((ny + YB - 1) / YB, n_jobs);
  size_t smem = sizeof(float2) * (size_t)(ny + nx + YB * nx);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(recon_combine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  recon_combine_kernel<<<grid, 256, smem, st>>>(d_jobs, YB);
}

}  // namespace mrsim
