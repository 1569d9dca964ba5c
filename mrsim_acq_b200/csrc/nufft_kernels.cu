// nufft_kernels.cu — the 2D NUFFT pair of the stack-of-spirals path on the device (reference
// `Nufft2`, nufft.rs:125-299): exponential-of-semicircle kernel exp(beta (sqrt(1 - z^2) - 1)),
// beta = 2.30 w, w = ceil(-log10 tol) + 1 clamped to 2..16, oversampling 2, deapodization by the
// kernel's sampled transform.  Type 1 spreads (tiles, in point order), type 2 interpolates; the fine-grid
// FFT is a shared-memory radix-2 kernel (a direct DFT for lengths that are not powers of two).
// Point positions and kernel offsets are formed in FP64 (the kernel is steep: an FP32 position
// would cost ~1e-5 of relative accuracy); the taps and sums are FP32.
//
// Also the spiral forwards (spiral.rs): the exact sum over voxels at each sample and the
// time-segmented combination of L type-2 transforms.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>

#include "nufft.h"

namespace mrsim {

namespace {

__device__ __forceinline__ int wrap(int m, int n) {
  m %= n;
  return m < 0 ? m + n : m;
}

template <class R>
__device__ __forceinline__ typename Vec2<R>::type mk2(R a, R b);
template <>
__device__ __forceinline__ float2 mk2<float>(float a, float b) {
  return make_float2(a, b);
}
template <>
__device__ __forceinline__ double2 mk2<double>(double a, double b) {
  return make_double2(a, b);
}
__device__ __forceinline__ float es_exp(float x) { return __expf(x); }
__device__ __forceinline__ double es_exp(double x) { return exp(x); }

constexpr int kWMax = 16;

// First fine cell and the w taps of coordinate u (period n) on a fine grid of nf = 2n cells.
template <class R>
__device__ __forceinline__ int es_taps(double u, int nf, int w, R beta, R* k) {
  const double half = 0.5 * w;
  double p = fmod(2.0 * u, (double)nf);
  if (p < 0.0) p += nf;
  const int m0 = (int)floor(p - half) + 1;
  const R ih = (R)(1.0 / half);
#pragma unroll
  for (int i = 0; i < kWMax; ++i) {
    if (i >= w) break;
    const R z = (R)((double)(m0 + i) - p) * ih;
    k[i] = fabs(z) < (R)1 ? es_exp(beta * (sqrt((R)1 - z * z) - (R)1)) : (R)0;
  }
  return m0;
}

template <class R>
__global__ void place_kernel(const NufftGridT<R> g, const typename Vec2<R>::type* __restrict__ modes,
                             typename Vec2<R>::type* __restrict__ grid, int batch, size_t mode_stride,
                             size_t grid_stride, const R* __restrict__ scale) {
  using V = typename Vec2<R>::type;
  const int b = blockIdx.y;
  const int nmodes = g.m_out0 * g.m_out1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nmodes; e += gridDim.x * blockDim.x) {
    const int j0 = e % g.m_out0, j1 = e / g.m_out0;
    const int b0 = wrap(g.m_lo0 + j0, g.nf0), b1 = wrap(g.m_lo1 + j1, g.nf1);
    V v = modes[b * mode_stride + e];
    R s = g.corr0[j0] * g.corr1[j1];
    if (scale) s *= scale[b];
    grid[b * grid_stride + (size_t)b0 + (size_t)g.nf0 * b1] = mk2<R>(v.x * s, v.y * s);
  }
}

template <class R>
__global__ void extract_kernel(const NufftGridT<R> g, const typename Vec2<R>::type* __restrict__ grid,
                               typename Vec2<R>::type* __restrict__ modes, size_t grid_stride, size_t mode_stride) {
  using V = typename Vec2<R>::type;
  const int b = blockIdx.y;
  const int nmodes = g.m_out0 * g.m_out1;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nmodes; e += gridDim.x * blockDim.x) {
    const int j0 = e % g.m_out0, j1 = e / g.m_out0;
    const int b0 = wrap(g.m_lo0 + j0, g.nf0), b1 = wrap(g.m_lo1 + j1, g.nf1);
    const V v = grid[b * grid_stride + (size_t)b0 + (size_t)g.nf0 * b1];
    const R s = g.corr0[j0] * g.corr1[j1];
    modes[b * mode_stride + e] = mk2<R>(v.x * s, v.y * s);
  }
}

// One CTA per line of length n (power of two): stride between elements `es`, between lines
// `ls`; lines = blockIdx.x within batch item blockIdx.y (batch stride `bs`).
template <class V>
__global__ void fft_pow2_kernel(V* __restrict__ data, int n, int logn, size_t es, size_t ls, size_t bs,
                                const V* __restrict__ tw, int sign) {
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V* buf = reinterpret_cast<V*>(fft_smem);
  V* base = data + blockIdx.y * bs + blockIdx.x * ls;
  // bit-reversed load
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int r = __brev(i) >> (32 - logn);
    buf[r] = base[(size_t)i * es];
  }
  __syncthreads();
  for (int s = 1; s <= logn; ++s) {
    const int m = 1 << s, h = m >> 1;
    for (int t = threadIdx.x; t < n / 2; t += blockDim.x) {
      const int grp = t / h, pos = t % h;
      const int i0 = grp * m + pos, i1 = i0 + h;
      V w = tw[(size_t)pos * (n / m)];  // e^{-i 2 pi pos / m}
      if (sign > 0) w.y = -w.y;
      const V a = buf[i0], b = buf[i1];
      V bw;
      bw.x = b.x * w.x - b.y * w.y;
      bw.y = b.x * w.y + b.y * w.x;
      V s0, s1;
      s0.x = a.x + bw.x;
      s0.y = a.y + bw.y;
      s1.x = a.x - bw.x;
      s1.y = a.y - bw.y;
      buf[i0] = s0;
      buf[i1] = s1;
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) base[(size_t)i * es] = buf[i];
}

// Direct DFT of one line (any n), e^{sign i 2 pi j k / n}.
template <class V>
__global__ void dft_line_kernel(V* __restrict__ data, int n, size_t es, size_t ls, size_t bs, const V* __restrict__ tw,
                                int sign) {
  extern __shared__ __align__(16) unsigned char fft_smem[];
  V* buf = reinterpret_cast<V*>(fft_smem);
  V* base = data + blockIdx.y * bs + blockIdx.x * ls;
  for (int i = threadIdx.x; i < n; i += blockDim.x) buf[i] = base[(size_t)i * es];
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    decltype(V().x) ar = 0, ai = 0;
    for (int j = 0; j < n; ++j) {
      V w = tw[((long long)j * k) % n];
      if (sign > 0) w.y = -w.y;
      const V a = buf[j];
      ar = fma(a.x, w.x, fma(-a.y, w.y, ar));
      ai = fma(a.x, w.y, fma(a.y, w.x, ai));
    }
    V o;
    o.x = ar;
    o.y = ai;
    base[(size_t)k * es] = o;  // inputs are in shared memory: no hazard
  }
}

constexpr int kBatchBlock = 4;  // batch items a type-1 or type-2 thread serves with one set of taps

// Type 2: out[j] = sum over the w x w taps of grid, for each point of each batch item; a thread
// serves one point for up to kBatchBlock batch items (blockIdx.y), forming the taps once.  The tap
// loops run to the compile-time bound kWMax (guarded by w), so taps and column indices live in
// registers; a window wraps at most once when the fine grid is at least 2 kWMax wide (else the
// general modulo).
template <class R>
__global__ void __launch_bounds__(128) interp_kernel(const NufftGridT<R> g, const typename Vec2<R>::type* __restrict__ grid,
                                                     const double* __restrict__ u, int npts,
                                                     typename Vec2<R>::type* __restrict__ out, size_t grid_stride,
                                                     size_t out_stride, int batch) {
  using V = typename Vec2<R>::type;
  const int b0 = blockIdx.y * kBatchBlock, nb = min(kBatchBlock, batch - b0);
  const int w = g.w;
  const bool wide = g.nf0 >= 2 * kWMax && g.nf1 >= 2 * kWMax;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npts; j += gridDim.x * blockDim.x) {
    R k0[kWMax], k1[kWMax];
    const int a0 = es_taps<R>(u[2 * j], g.nf0, w, g.beta, k0);
    const int a1 = es_taps<R>(u[2 * j + 1], g.nf1, w, g.beta, k1);
    int col[kWMax];
#pragma unroll
    for (int i0 = 0; i0 < kWMax; ++i0) {
      int c = a0 + i0;
      if (wide) {
        c = c < 0 ? c + g.nf0 : c;
        c = c >= g.nf0 ? c - g.nf0 : c;
      } else {
        c = wrap(c, g.nf0);
      }
      col[i0] = c;
    }
    R re[kBatchBlock], im[kBatchBlock];
#pragma unroll
    for (int q = 0; q < kBatchBlock; ++q) re[q] = im[q] = 0;
#pragma unroll
    for (int i1 = 0; i1 < kWMax; ++i1) {
      if (i1 >= w) break;
      int c1 = a1 + i1;
      if (wide) {
        c1 = c1 < 0 ? c1 + g.nf1 : c1;
        c1 = c1 >= g.nf1 ? c1 - g.nf1 : c1;
      } else {
        c1 = wrap(c1, g.nf1);
      }
      const V* row = grid + (size_t)g.nf0 * c1;
      R rr[kBatchBlock], ri[kBatchBlock];
#pragma unroll
      for (int q = 0; q < kBatchBlock; ++q) rr[q] = ri[q] = 0;
#pragma unroll
      for (int i0 = 0; i0 < kWMax; ++i0) {
        if (i0 >= w) break;
#pragma unroll
        for (int q = 0; q < kBatchBlock; ++q)
          if (q < nb) {
            const V v = __ldg(row + (size_t)(b0 + q) * grid_stride + col[i0]);
            rr[q] = fma(v.x, k0[i0], rr[q]);
            ri[q] = fma(v.y, k0[i0], ri[q]);
          }
      }
#pragma unroll
      for (int q = 0; q < kBatchBlock; ++q) {
        re[q] = fma(rr[q], k1[i1], re[q]);
        im[q] = fma(ri[q], k1[i1], im[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < kBatchBlock; ++q)
      if (q < nb) out[(size_t)(b0 + q) * out_stride + j] = mk2<R>(re[q], im[q]);
  }
}

// The wrapped offset of cell c from a window start a on a ring of n cells, in [0, n).
__device__ __forceinline__ int ring_offset(int c, int a, int n) {
  int d = c - a;
  while (d < 0) d += n;
  while (d >= n) d -= n;
  return d;
}

constexpr int kSpreadChunk = 64;  // points whose taps a spread block holds at a time

// Type 1 spreading without atomics: one block per 8 x 8 tile of the fine grid (one thread per
// cell) and group of up to kBatchBlock batch items (the taps formed once for the group).  The tile's points (nufft_bins2: every point whose window can reach the
// tile, in point order) pass through shared memory in chunks with their taps; each thread adds
// the contributions to its own cell point after point, cell += w_j (k0 k1) as the reference does
// (nufft.rs:236-250), and stores the cell once.  The sum order is fixed, so the grid is the same
// on every run; a window that wraps onto a cell twice (a fine grid narrower than the kernel) adds
// both taps in tap order.
template <class R>
__global__ void __launch_bounds__(kSpreadTile * kSpreadTile)
    spread_tile_kernel(const NufftGridT<R> g, typename Vec2<R>::type* __restrict__ grid, const double* __restrict__ u,
                       const typename Vec2<R>::type* __restrict__ wts, size_t grid_stride, size_t w_stride,
                       const NufftBins bins, int batch) {
  using V = typename Vec2<R>::type;
  __shared__ R sk0[kSpreadChunk][kWMax], sk1[kSpreadChunk][kWMax];
  __shared__ int sa0[kSpreadChunk], sa1[kSpreadChunk];
  __shared__ V sw[kBatchBlock][kSpreadChunk];
  const int b0 = blockIdx.y * kBatchBlock, nb = min(kBatchBlock, batch - b0), tile = blockIdx.x;
  const int c0 = (tile % bins.tiles0) * kSpreadTile + (int)threadIdx.x % kSpreadTile;
  const int c1 = (tile / bins.tiles0) * kSpreadTile + (int)threadIdx.x / kSpreadTile;
  const bool mine = c0 < g.nf0 && c1 < g.nf1;
  const int w = g.w;
  R re[kBatchBlock], im[kBatchBlock];
#pragma unroll
  for (int q = 0; q < kBatchBlock; ++q) re[q] = im[q] = 0;
  const int p0 = bins.start[tile], p1 = bins.start[tile + 1];
  for (int base = p0; base < p1; base += kSpreadChunk) {
    const int n = min(kSpreadChunk, p1 - base);
    if ((int)threadIdx.x < n) {
      const int t = threadIdx.x, j = bins.pts[base + t];
      sa0[t] = es_taps<R>(u[2 * j], g.nf0, w, g.beta, sk0[t]);
      sa1[t] = es_taps<R>(u[2 * j + 1], g.nf1, w, g.beta, sk1[t]);
#pragma unroll
      for (int q = 0; q < kBatchBlock; ++q)
        if (q < nb) sw[q][t] = wts[(size_t)(b0 + q) * w_stride + j];
    }
    __syncthreads();
    if (mine)
      for (int q = 0; q < n; ++q) {
        const int d0 = ring_offset(c0, sa0[q], g.nf0);
        if (d0 >= w) continue;
        const int d1 = ring_offset(c1, sa1[q], g.nf1);
        if (d1 >= w) continue;
        for (int i1 = d1; i1 < w; i1 += g.nf1)
          for (int i0 = d0; i0 < w; i0 += g.nf0) {
            const R v = sk0[q][i0] * sk1[q][i1];
#pragma unroll
            for (int bq = 0; bq < kBatchBlock; ++bq) {
              re[bq] += sw[bq][q].x * v;
              im[bq] += sw[bq][q].y * v;
            }
          }
      }
    __syncthreads();
  }
  if (mine)
#pragma unroll
    for (int q = 0; q < kBatchBlock; ++q)
      if (q < nb) grid[(size_t)(b0 + q) * grid_stride + (size_t)c0 + (size_t)g.nf0 * c1] = mk2<R>(re[q], im[q]);
}

// ---- the 1D type-1 NUFFT (`Nufft1`, nufft.rs:25-112), FP64 --------------------------------------
// Spreading without atomics: one block per 256-cell tile of the fine grid and weight vector, one
// thread per cell; the tile's points (nufft_bins1, in point order) pass through shared memory with
// their taps, and each cell adds g += w_j k_i point after point as the reference does
// (nufft.rs:80-97).
__global__ void __launch_bounds__(kSpreadTile1)
    spread1_tile_kernel(const double* __restrict__ pos, const double2* __restrict__ wts, int npos, int nf, int w,
                        double beta, double2* __restrict__ grid, const NufftBins bins) {
  __shared__ double sk[kSpreadChunk][kWMax];
  __shared__ int sm0[kSpreadChunk];
  __shared__ double2 sw[kSpreadChunk];
  const int q = blockIdx.y, tile = blockIdx.x;
  const int c = tile * kSpreadTile1 + (int)threadIdx.x;
  const bool mine = c < nf;
  double re = 0.0, im = 0.0;
  const int p0 = bins.start[tile], p1 = bins.start[tile + 1];
  for (int base = p0; base < p1; base += kSpreadChunk) {
    const int n = min(kSpreadChunk, p1 - base);
    if ((int)threadIdx.x < n) {
      const int t = threadIdx.x, j = bins.pts[base + t];
      sm0[t] = es_taps<double>(pos[j], nf, w, beta, sk[t]);  // fine position 2 pos on nf = 2n cells
      sw[t] = wts[(size_t)q * npos + j];
    }
    __syncthreads();
    if (mine)
      for (int t = 0; t < n; ++t) {
        const int d = ring_offset(c, sm0[t], nf);
        for (int i = d; i < w; i += nf) {
          re += sw[t].x * sk[t][i];
          im += sw[t].y * sk[t][i];
        }
      }
    __syncthreads();
  }
  if (mine) grid[(size_t)q * nf + c] = make_double2(re, im);
}

__global__ void extract1_kernel(const double2* __restrict__ grid, int nf, int k_lo, int n_out,
                                const double* __restrict__ corr, int nw, double2* __restrict__ out) {
  const int q = blockIdx.y;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n_out; j += gridDim.x * blockDim.x) {
    const double2 v = grid[(size_t)q * nf + wrap(k_lo + j, nf)];
    out[(size_t)q * n_out + j] = make_double2(v.x * corr[j], v.y * corr[j]);
  }
}

// ---- spiral forwards ---------------------------------------------------------------------------
// The exact sum (`spiral_kspace_exact`, spiral.rs:107-137): one thread per sample, voxels staged
// in shared memory in tiles; the k.r + f tau phase in FP64 (nonuniform k), reduced to turns.
constexpr int kTileVox = 256;

__global__ void __launch_bounds__(256) spiral_exact_kernel(const SpiralExactArgs a) {
  __shared__ double sx[kTileVox], sy[kTileVox];
  __shared__ float sr[kTileVox], sph[kTileVox], samp[kTileVox];
  __shared__ float sm[kTileVox][4];
  __shared__ float sd[kTileVox][4];
  __shared__ float sla[kTileVox];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const bool ok = j < a.npts;
  double kx = 0, ky = 0;
  float tau = 0.f;
  if (ok) {
    kx = a.k[2 * j] / a.nx;
    ky = a.k[2 * j + 1] / a.ny;
    tau = (float)a.tau_ms[j];
  }
  const double taus = ok ? a.tau_ms[j] / 1000.0 : 0.0;
  float re = 0.f, im = 0.f;
  const int nvox = a.snx * a.sny;
  for (int v0 = 0; v0 < nvox; v0 += kTileVox) {
    __syncthreads();
    for (int t = threadIdx.x; t < kTileVox; t += blockDim.x) {
      const int i = v0 + t;
      if (i < nvox) {
        const int x = i % a.snx, y = i / a.snx;
        sx[t] = ((double)x - a.sxs - a.xoff) / a.ox;
        sy[t] = ((double)y - a.sys - a.yoff) / a.oy;
        sr[t] = a.rate ? a.rate[i] : 0.f;
        sph[t] = a.phase_turns ? a.phase_turns[i] : 0.f;
        samp[t] = a.amp[i];
        sla[t] = a.log_amp ? a.log_amp[i] : 0.f;
        for (int c = 0; c < 4; ++c) {
          sm[t][c] = c < a.ncomp ? a.comp[(size_t)c * nvox + i] : 0.f;
          sd[t][c] = (a.decay && c < a.ncomp) ? a.decay[(size_t)c * nvox + i] : 0.f;
        }
      } else {
        samp[t] = 0.f;
        sla[t] = 0.f;
        for (int c = 0; c < 4; ++c) sm[t][c] = sd[t][c] = 0.f;
        sx[t] = sy[t] = 0.0;
        sr[t] = sph[t] = 0.f;
      }
    }
    __syncthreads();
    if (!ok) continue;
    const int nt = min(kTileVox, nvox - v0);
    for (int t = 0; t < nt; ++t) {
      // w = sum_c m_c exp(ln A - tau d_c) under relaxation, sum_c m_c otherwise (spiral.rs:75-80)
      float w = 0.f;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (c < a.ncomp) {
          const float e = a.relax ? __expf(sla[t] - tau * sd[t][c]) : 1.f;
          w = fmaf(sm[t][c], e, w);
        }
      }
      if (w == 0.f) continue;
      double th = kx * sx[t] + ky * sy[t] + (double)sr[t] * taus;
      th -= rint(th);
      float thf = (float)th + sph[t];
      thf -= rintf(thf);
      float sn, cs;
      sincospif(2.0f * thf, &sn, &cs);
      const float amp = samp[t] * w;
      re = fmaf(amp, cs, re);
      im = fmaf(amp, sn, im);
    }
  }
  if (ok) a.out[j] = make_float2(re * a.inv_nvox, im * a.inv_nvox);
}

// Segment images: img_l(r) = x(r) e^{rate(r) tau_l} for every segment l (spiral.rs:174-201).
__global__ void segment_images_kernel(const float2* __restrict__ x, const float2* __restrict__ rate, int nvox,
                                      const double* __restrict__ tau_l, int L, float2* __restrict__ out) {
  const int l = blockIdx.y;
  const double tl = tau_l[l];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nvox; i += gridDim.x * blockDim.x) {
    const float2 r = rate[i];
    const float mag = __expf(r.x * (float)tl);
    double th = (double)r.y * tl / 6.283185307179586;
    th -= rint(th);
    float sn, cs;
    sincospif(2.0f * (float)th, &sn, &cs);
    const float2 v = x[i];
    const float er = mag * cs, ei = mag * sn;
    out[(size_t)l * nvox + i] = make_float2(v.x * er - v.y * ei, v.x * ei + v.y * er);
  }
}

// out_j = stat_j * sum_l b[tau_idx_j][l] * seg[l][j]
__global__ void segment_combine_kernel(const float2* __restrict__ seg, int npts, int L, const int* __restrict__ tau_idx,
                                       const double* __restrict__ b, const float2* __restrict__ stat,
                                       float2* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < npts; j += gridDim.x * blockDim.x) {
    const double* bj = b + (size_t)tau_idx[j] * L * 2;
    float re = 0.f, im = 0.f;
    for (int l = 0; l < L; ++l) {
      const float2 v = seg[(size_t)l * npts + j];
      const float br = (float)bj[2 * l], bi = (float)bj[2 * l + 1];
      re = fmaf(br, v.x, fmaf(-bi, v.y, re));
      im = fmaf(br, v.y, fmaf(bi, v.x, im));
    }
    const float2 s = stat[j];
    out[j] = make_float2(re * s.x - im * s.y, re * s.y + im * s.x);
  }
}

}  // namespace

// ---- launchers ------------------------------------------------------------------------------------
template <class V>
void fft2(V* grid, int n0, int n1, const V* tw0, const V* tw1, int batch, int sign, cudaStream_t st) {
  const size_t gs = (size_t)n0 * n1;
  // rows (axis 0, contiguous), then columns (axis 1, stride n0)
  for (int axis = 0; axis < 2; ++axis) {
    const int n = axis == 0 ? n0 : n1;
    if (n == 1) continue;  // a length-1 transform is the identity
    const int lines = axis == 0 ? n1 : n0;
    const size_t es = axis == 0 ? 1 : (size_t)n0;
    const size_t ls = axis == 0 ? (size_t)n0 : 1;
    const V* tw = axis == 0 ? tw0 : tw1;
    const int threads = std::min(256, std::max(32, n / 2));
    dim3 grid_dim(lines, batch);
    const size_t smem = sizeof(V) * n;  // n <= 16384: at most 256 KiB in FP64, refused above 227 KiB
    if ((n & (n - 1)) == 0) {
      int logn = 0;
      while ((1 << logn) < n) ++logn;
      if (smem > 48 * 1024)
        cudaFuncSetAttribute(fft_pow2_kernel<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      fft_pow2_kernel<V><<<grid_dim, threads, smem, st>>>(grid, n, logn, es, ls, gs, tw, sign);
    } else {
      if (smem > 48 * 1024)
        cudaFuncSetAttribute(dft_line_kernel<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      dft_line_kernel<V><<<grid_dim, std::min(256, n), smem, st>>>(grid, n, es, ls, gs, tw, sign);
    }
  }
}
template void fft2<float2>(float2*, int, int, const float2*, const float2*, int, int, cudaStream_t);
template void fft2<double2>(double2*, int, int, const double2*, const double2*, int, int, cudaStream_t);

template <class R>
void nufft_type2(const NufftGridT<R>& g, const typename Vec2<R>::type* modes, int batch, size_t mode_stride,
                 const double* u, int npts, typename Vec2<R>::type* out, size_t out_stride,
                 typename Vec2<R>::type* work, int sign, const R* scale, cudaStream_t st) {
  using V = typename Vec2<R>::type;
  const size_t gs = (size_t)g.nf0 * g.nf1;
  cudaMemsetAsync(work, 0, gs * batch * sizeof(V), st);
  dim3 pg((g.m_out0 * g.m_out1 + 255) / 256, batch);
  place_kernel<R><<<pg, 256, 0, st>>>(g, modes, work, batch, mode_stride, gs, scale);
  nufft_fft2(g, work, batch, sign, st);
  dim3 ig(std::max(1, std::min((npts + 127) / 128, 4096)), (batch + kBatchBlock - 1) / kBatchBlock);
  interp_kernel<R><<<ig, 128, 0, st>>>(g, work, u, npts, out, gs, out_stride, batch);
}

template <class R>
void nufft_type1(const NufftGridT<R>& g, const double* u, int npts, const NufftBins& bins,
                 const typename Vec2<R>::type* wts, int batch, size_t w_stride, typename Vec2<R>::type* modes,
                 size_t mode_stride, typename Vec2<R>::type* work, int sign, cudaStream_t st) {
  const size_t gs = (size_t)g.nf0 * g.nf1;
  // every cell of every tile is written (zero where no point reaches it)
  dim3 sg(bins.tiles0 * bins.tiles1, (batch + kBatchBlock - 1) / kBatchBlock);
  spread_tile_kernel<R><<<sg, kSpreadTile * kSpreadTile, 0, st>>>(g, work, u, wts, gs, w_stride, bins, batch);
  nufft_fft2(g, work, batch, sign, st);
  dim3 eg((g.m_out0 * g.m_out1 + 255) / 256, batch);
  extract_kernel<R><<<eg, 256, 0, st>>>(g, work, modes, gs, mode_stride);
}

template void nufft_type2<float>(const NufftGridT<float>&, const float2*, int, size_t, const double*, int, float2*,
                                 size_t, float2*, int, const float*, cudaStream_t);
template void nufft_type2<double>(const NufftGridT<double>&, const double2*, int, size_t, const double*, int, double2*,
                                  size_t, double2*, int, const double*, cudaStream_t);
template void nufft_type1<float>(const NufftGridT<float>&, const double*, int, const NufftBins&, const float2*, int,
                                 size_t, float2*, size_t, float2*, int, cudaStream_t);
template void nufft_type1<double>(const NufftGridT<double>&, const double*, int, const NufftBins&, const double2*, int,
                                  size_t, double2*, size_t, double2*, int, cudaStream_t);


void nufft1_run(const Nufft1Grid& g, const double* pos, int npos, const NufftBins& bins, const double2* wts, int nw,
                double2* out, double2* work, cudaStream_t st) {
  // every cell of every tile is written (zero where no source reaches it)
  spread1_tile_kernel<<<dim3(bins.tiles0, nw), kSpreadTile1, 0, st>>>(pos, wts, npos, g.nf, g.w, g.beta, work, bins);
  fft2<double2>(work, g.nf, 1, g.tw, g.tw, nw, 1, st);  // the inverse transform (e^{+i}) of each fine grid
  dim3 eg((g.n_out + 255) / 256, nw);
  extract1_kernel<<<eg, 256, 0, st>>>(work, g.nf, g.k_lo, g.n_out, g.corr, nw, out);
}

void spiral_exact(const SpiralExactArgs& a, cudaStream_t st) {
  spiral_exact_kernel<<<(a.npts + 255) / 256, 256, 0, st>>>(a);
}

void segment_images(const float2* x, const float2* rate, int nvox, const double* tau_l, int L, float2* out,
                    cudaStream_t st) {
  dim3 g((nvox + 255) / 256, L);
  segment_images_kernel<<<g, 256, 0, st>>>(x, rate, nvox, tau_l, L, out);
}

void segment_combine(const float2* seg, int npts, int L, const int* tau_idx, const double* b, const float2* stat,
                     float2* out, cudaStream_t st) {
  segment_combine_kernel<<<(npts + 255) / 256, 256, 0, st>>>(seg, npts, L, tau_idx, b, stat, out);
}

}  // namespace mrsim
