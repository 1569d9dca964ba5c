// epi_kernels.cu — the exact-DFT EPI forward operator and its adjoint / VJP, FP32, sm_100a.
//
// The forward restates `build_coil_kspace_timed` (reference kspace.rs:607-1042) without its
// spikes and noise.  For each unit (one slice of one volume, every echo's acquired lines) it
// evaluates, exactly (no time segmentation, no NUFFT),
//
//   g_q[j][x] = s * sum_y amp_q(x,y) * W_j(x,y) * e^{i 2pi theta_j(x,y)}          (y-stage)
//   k_q[row_j][kx] = (1/nvox) sum_x g_q[j][x] * E_j(x) * tw_pol(j)(kx, x)           (x-stage)
//
//   theta_j = a(x,y) + f(x,y) * t_j + (ky_j - ys)(y - sys - yoff)/sny + Py(y)*decay_j
//   W_j     = sum_c rel_cj(x,y) m_c(x,y)
//
// `a` is the static phase in turns (object phase, eddy object-phase ramp), `Py*decay` the y part
// of the separable eddy polynomial (kspace.rs:904-925), E_j its x and z parts, and tw the x-stage
// twiddle of the line's readout polarity (`XStage`, kspace.rs:1052-1140).  The k.r phase of the
// y-DFT is an exact integer index (ky-ys)*(2(y-sys)-(oy-1)) mod 2*sny; f*t is split hi+lo
// (two-product) so the phase keeps ~1e-7 turn accuracy before the MUFU sin/cos of the reduced
// argument.  amp_q(x,y) = ex_q(x)*ey_q(y) + off is `coil_sensitivity` (kspace.rs:226-237)
// factored per axis (the Gaussian is separable).
//
// The adjoint is the Hermitian transpose with respect to complex compartment images, plus the
// vector-Jacobian products of L = sum |k - d|^2 with respect to the fieldmap and each
// compartment's R2 = 1/T2 (the reference has no adjoint; the oracle is the FP64 transpose).
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include "mrsim_internal.h"

namespace mrsim {

namespace {

constexpr float kTwoPiF = 6.28318530717958647692f;

__device__ __forceinline__ float frac_turn(float v) { return v - rintf(v); }

// Phase of voxel value f (Hz) at line time t = t_hi + t_lo (s), in turns, reduced.
__device__ __forceinline__ float ft_turns(float f, float t_hi, float t_lo) {
  float p = f * t_hi;
  float e = fmaf(f, t_hi, -p);      // exact error of the product
  float r = p - rintf(p);           // exact
  return r + fmaf(f, t_lo, e);
}

// ---------------------------------------------------------------------------------------------
// statics: a(x,y) = frac( (phi0 + eddy object phase) / 2pi ) in FP64, stored as f32 turns.
// phi0 = phase0[i] (explicit) or the phase model `PhaseModel::at` (phase.rs:141) sampled by
// `phase_slice` (kspace.rs:1156-1180).
__global__ void statics_kernel(const StaticDesc* descs) {
  const StaticDesc& d = descs[blockIdx.y];
  int n = d.snx * d.sny;
  const double inv_tau = 0.15915494309189533577;
  int ox = d.snx / d.nx, oy = d.sny / d.ny;
  int sxs = ox * (d.nx / 2), sys = oy * (d.ny / 2);
  double xoff = (ox - 1.0) / 2.0, yoff = (oy - 1.0) / 2.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int x = i % d.snx, y = i / d.snx;
    double p0;
    if (d.flags & 1) {
      p0 = d.phase0[i];
    } else {
      double sx = d.snx / 2.0, sy = d.sny / 2.0, off = (d.o - 1.0) / 2.0;
      double r0 = (x - sx - off) / d.o, r1 = (y - sy - off) / d.o, r2 = d.z - d.nz_full / 2.0;
      const double* c = d.bg;
      double bg = c[0] + c[1] * r0 + c[2] * r1 + c[3] * r2 + c[4] * r0 * r0 + c[5] * r1 * r1 + c[6] * r2 * r2 +
                  c[7] * r0 * r1 + c[8] * r0 * r2 + c[9] * r1 * r2;
      double cr0 = d.shot_rot[1] * r2 - d.shot_rot[2] * r1;
      double cr1 = d.shot_rot[2] * r0 - d.shot_rot[0] * r2;
      double cr2 = d.shot_rot[0] * r1 - d.shot_rot[1] * r0;
      double shot = d.shot_q[0] * (d.shot_dx[0] + cr0) + d.shot_q[1] * (d.shot_dx[1] + cr1) +
                    d.shot_q[2] * (d.shot_dx[2] + cr2);
      p0 = d.global + bg + shot;
    }
    if (d.flags & 2) {
      double xc = (x - sxs - xoff) / ox, yc = (y - sys - yoff) / oy;
      p0 += d.eddy_phase_coef[0] * xc + d.eddy_phase_coef[1] * yc + d.eddy_phase_coef[2] * d.zc_c;
    }
    double tt = p0 * inv_tau;
    tt -= rint(tt);
    d.out[i] = (float)tt;
  }
}

// ---------------------------------------------------------------------------------------------
// y-stage of the forward.  One CTA = (unit, T lines, 128 columns, QG coils); one thread per
// column x accumulates T*QG complex sums over every sim row y.
struct Tile {
  int unit, line0, x0, q0;
};

template <int T, int QG, int NC, bool MAPS>
__global__ void __launch_bounds__(128) ystage_kernel(const UnitDesc* __restrict__ units,
                                                     const Tile* __restrict__ tiles) {
  extern __shared__ float smem[];
  const Tile tl = tiles[blockIdx.x];
  const UnitDesc& u = units[tl.unit];
  const int snx = u.snx, sny = u.sny;
  const int ncomp = u.ncomp;
  float* Bt = smem;                 // [sny][T] phase terms per (row, line)
  float* Ey = smem + sny * T;       // [QG][sny]
  __shared__ float rel_s[T][kMaxComp];
  __shared__ float tinh_s[T], trf_s[T];
  __shared__ float thi_s[T], tlo_s[T];

  const int nl = min(T, u.n_lines - tl.line0);
  const int ys = u.ny / 2;
  const int oy = sny / u.ny;
  const int sys = oy * ys;
  // per-CTA tables
  for (int idx = threadIdx.x; idx < sny * T; idx += blockDim.x) {
    int y = idx / T, j = idx % T;
    float v = 0.f;
    if (j < nl) {
      const LineRec& L = u.lines[tl.line0 + j];
      long long K = L.ky - ys;
      long long Y = 2LL * (y - sys) - (oy - 1);
      long long m2 = 2LL * sny;
      long long r = (K * Y) % m2;
      double tv = (double)r / (double)m2;
      if (u.flags & UF_EDDY) {
        double yc = ((double)y - sys - (oy - 1) / 2.0) / oy;
        tv += ((double)u.eddy_cy * yc + (double)u.eddy_qy * yc * yc) * (double)L.decay;
      }
      tv -= rint(tv);
      v = (float)tv;
    }
    Bt[idx] = v;
  }
  for (int idx = threadIdx.x; idx < QG * sny; idx += blockDim.x) {
    int qq = idx / sny, y = idx % sny;
    int q = tl.q0 + qq;
    Ey[idx] = q < u.ncoils ? u.geo.ey[(size_t)q * sny + y] : 0.f;
  }
  if (threadIdx.x < T) {
    int j = threadIdx.x;
    if (j < nl) {
      const LineRec& L = u.lines[tl.line0 + j];
      thi_s[j] = L.t_hi;
      tlo_s[j] = L.t_lo;
      tinh_s[j] = L.inhom_ms;
      trf_s[j] = L.trf_ms;
      for (int c = 0; c < kMaxComp; ++c) rel_s[j][c] = L.rel[c];
    } else {
      thi_s[j] = tlo_s[j] = tinh_s[j] = trf_s[j] = 0.f;
      for (int c = 0; c < kMaxComp; ++c) rel_s[j][c] = 0.f;
    }
  }
  __syncthreads();

  const int x = tl.x0 + threadIdx.x;
  const bool xok = x < snx;
  const int xs_ = xok ? x : 0;
  float exq[QG];
  const float off = u.geo.coil_off;
#pragma unroll
  for (int qq = 0; qq < QG; ++qq) {
    int q = tl.q0 + qq;
    exq[qq] = (xok && q < u.ncoils) ? u.geo.ex[(size_t)q * snx + x] : 0.f;
  }
  float thi[T], tlo[T];
#pragma unroll
  for (int j = 0; j < T; ++j) {
    thi[j] = thi_s[j];
    tlo[j] = tlo_s[j];
  }
  float2 acc[T][QG];
#pragma unroll
  for (int j = 0; j < T; ++j)
#pragma unroll
    for (int qq = 0; qq < QG; ++qq) acc[j][qq] = make_float2(0.f, 0.f);

  const bool distort = (u.flags & UF_DISTORT) != 0;
  const float* __restrict__ comp = u.comp;
  const float* __restrict__ fmap = u.fmap;
  const float* __restrict__ phase = u.phase;
  for (int y = 0; y < sny; ++y) {
    const int i = xs_ + snx * y;
    const float a = phase ? __ldg(phase + i) : 0.f;
    const float f = distort ? __ldg(fmap + i) : 0.f;
    float m[NC];
    float r2[NC], r2i[NC];
    float la = 0.f;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      m[c] = 0.f;
      r2[c] = 0.f;
      r2i[c] = 0.f;
      if (c < ncomp) {
        m[c] = __ldg(comp + (size_t)c * u.comp_stride + i);
        if (MAPS) {
          float t2 = u.t2map ? __ldg(u.t2map + (size_t)c * u.map_stride + i) : u.t2u[c];
          float ti = u.timap ? __ldg(u.timap + (size_t)c * u.map_stride + i) : u.tiu[c];
          r2[c] = 1.0f / t2;
          r2i[c] = 1.0f / ti;
        }
      }
    }
    if (MAPS && u.log_amp) la = __ldg(u.log_amp + i);
    float amp[QG];
#pragma unroll
    for (int qq = 0; qq < QG; ++qq) amp[qq] = fmaf(exq[qq], Ey[qq * sny + y], off);
#pragma unroll
    for (int j = 0; j < T; ++j) {
      float th = a + Bt[y * T + j] + ft_turns(f, thi[j], tlo[j]);
      th = frac_turn(th);
      float sn, cs;
      __sincosf(kTwoPiF * th, &sn, &cs);
      float W = 0.f;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        if (c < ncomp) {
          float r;
          if (MAPS)
            r = __expf(la - trf_s[j] * r2[c] - tinh_s[j] * r2i[c]);
          else
            r = rel_s[j][c];
          W = fmaf(r, m[c], W);
        }
      }
      const float wr = W * cs, wi = W * sn;
#pragma unroll
      for (int qq = 0; qq < QG; ++qq) {
        acc[j][qq].x = fmaf(amp[qq], wr, acc[j][qq].x);
        acc[j][qq].y = fmaf(amp[qq], wi, acc[j][qq].y);
      }
    }
  }
  if (!xok) return;
  const float s = u.signal_scale;
#pragma unroll
  for (int qq = 0; qq < QG; ++qq) {
    int q = tl.q0 + qq;
    if (q >= u.ncoils) break;
#pragma unroll
    for (int j = 0; j < T; ++j) {
      if (j < nl) {
        float2 v = make_float2(acc[j][qq].x * s, acc[j][qq].y * s);
        u.g[((size_t)q * u.n_lines + tl.line0 + j) * snx + x] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// x-stage: k[q][row][kx] = (1/nvox) sum_x g[q][j][x] E_j(x) tw_pol(kx,x), for 8 lines per CTA.
constexpr int XR = 8;

__global__ void __launch_bounds__(128) xstage_kernel(const UnitDesc* __restrict__ units,
                                                     const int4* __restrict__ tiles) {
  extern __shared__ float2 gs[];  // [XR][snx]
  const int4 tl = tiles[blockIdx.x];  // unit, q, line0
  const UnitDesc& u = units[tl.x];
  const int snx = u.snx, nx = u.nx, q = tl.y, line0 = tl.z;
  const int nl = min(XR, u.n_lines - line0);
  const int ox = snx / nx, sxs = ox * (nx / 2);
  const float xoff = (ox - 1.0f) / 2.0f;
  for (int idx = threadIdx.x; idx < XR * snx; idx += blockDim.x) {
    int j = idx / snx, x = idx % snx;
    float2 v = make_float2(0.f, 0.f);
    if (j < nl) {
      v = u.g[((size_t)q * u.n_lines + line0 + j) * snx + x];
      if (u.flags & UF_EDDY) {
        const LineRec& L = u.lines[line0 + j];
        double xc = ((double)x - sxs - xoff) / ox;
        double tv = ((double)u.eddy_cx * xc + (double)u.eddy_qx * xc * xc + (double)u.eddy_z) * (double)L.decay;
        tv -= rint(tv);
        float sn, cs;
        __sincosf(kTwoPiF * (float)tv, &sn, &cs);
        v = make_float2(v.x * cs - v.y * sn, v.x * sn + v.y * cs);
      }
    }
    gs[idx] = v;
  }
  __shared__ int pol_s[XR];
  __shared__ int row_s[XR];
  if (threadIdx.x < XR) {
    int j = threadIdx.x;
    pol_s[j] = j < nl ? (u.lines[line0 + j].pol < 0 ? 1 : 0) : 0;
    row_s[j] = j < nl ? u.lines[line0 + j].row : 0;
  }
  __syncthreads();
  const float inv_n = 1.0f / (float)(snx * u.sny);
  const float2* tw0 = u.geo.tw;
  const float2* tw1 = u.geo.tw + (size_t)snx * nx;
  for (int kx = threadIdx.x; kx < nx; kx += blockDim.x) {
    float2 acc[XR];
#pragma unroll
    for (int j = 0; j < XR; ++j) acc[j] = make_float2(0.f, 0.f);
    for (int x = 0; x < snx; ++x) {
      const float2 a0 = __ldg(tw0 + (size_t)x * nx + kx);
      const float2 a1 = __ldg(tw1 + (size_t)x * nx + kx);
#pragma unroll
      for (int j = 0; j < XR; ++j) {
        const float2 t = pol_s[j] ? a1 : a0;
        const float2 gv = gs[j * snx + x];
        acc[j].x = fmaf(gv.x, t.x, fmaf(-gv.y, t.y, acc[j].x));
        acc[j].y = fmaf(gv.x, t.y, fmaf(gv.y, t.x, acc[j].y));
      }
    }
#pragma unroll
    for (int j = 0; j < XR; ++j)
      if (j < nl)
        u.kspace[((size_t)q * u.n_rows + row_s[j]) * nx + kx] = make_float2(acc[j].x * inv_n, acc[j].y * inv_n);
  }
}

// ---------------------------------------------------------------------------------------------
// x-adjoint: h[q][j][x] = (1/nvox) conj(E_j(x)) sum_kx conj(tw_pol(kx,x)) r[q][row_j][kx].
__global__ void __launch_bounds__(128) xadjoint_kernel(const UnitDesc* __restrict__ units,
                                                       const int4* __restrict__ tiles) {
  extern __shared__ float2 rs[];  // [XR][nx]
  const int4 tl = tiles[blockIdx.x];
  const UnitDesc& u = units[tl.x];
  const int snx = u.snx, nx = u.nx, q = tl.y, line0 = tl.z;
  const int nl = min(XR, u.n_lines - line0);
  const int ox = snx / nx, sxs = ox * (nx / 2);
  const float xoff = (ox - 1.0f) / 2.0f;
  __shared__ int pol_s[XR];
  __shared__ float dec_s[XR];
  if (threadIdx.x < XR) {
    int j = threadIdx.x;
    pol_s[j] = j < nl ? (u.lines[line0 + j].pol < 0 ? 1 : 0) : 0;
    dec_s[j] = j < nl ? u.lines[line0 + j].decay : 0.f;
  }
  for (int idx = threadIdx.x; idx < XR * nx; idx += blockDim.x) {
    int j = idx / nx, kx = idx % nx;
    float2 v = make_float2(0.f, 0.f);
    if (j < nl) v = u.kspace[((size_t)q * u.n_rows + u.lines[line0 + j].row) * nx + kx];
    rs[idx] = v;
  }
  __syncthreads();
  const float inv_n = 1.0f / (float)(snx * u.sny);
  // transposed twiddles follow the forward tables: [pol][kx][x]
  const float2* tt0 = u.geo.tw + (size_t)2 * snx * nx;
  const float2* tt1 = tt0 + (size_t)snx * nx;
  for (int x = threadIdx.x; x < snx; x += blockDim.x) {
    float2 acc[XR];
#pragma unroll
    for (int j = 0; j < XR; ++j) acc[j] = make_float2(0.f, 0.f);
    for (int kx = 0; kx < nx; ++kx) {
      const float2 a0 = __ldg(tt0 + (size_t)kx * snx + x);
      const float2 a1 = __ldg(tt1 + (size_t)kx * snx + x);
#pragma unroll
      for (int j = 0; j < XR; ++j) {
        const float2 t = pol_s[j] ? a1 : a0;
        const float2 r = rs[j * nx + kx];
        // conj(t) * r
        acc[j].x = fmaf(t.x, r.x, fmaf(t.y, r.y, acc[j].x));
        acc[j].y = fmaf(t.x, r.y, fmaf(-t.y, r.x, acc[j].y));
      }
    }
    double xc = ((double)x - sxs - xoff) / ox;
#pragma unroll
    for (int j = 0; j < XR; ++j) {
      if (j >= nl) continue;
      float2 v = make_float2(acc[j].x * inv_n, acc[j].y * inv_n);
      if (u.flags & UF_EDDY) {
        double tv = ((double)u.eddy_cx * xc + (double)u.eddy_qx * xc * xc + (double)u.eddy_z) * (double)dec_s[j];
        tv -= rint(tv);
        float sn, cs;
        __sincosf(kTwoPiF * (float)tv, &sn, &cs);
        // multiply by conj(E) = (cs, -sn)
        v = make_float2(v.x * cs + v.y * sn, v.y * cs - v.x * sn);
      }
      u.g[((size_t)q * u.n_lines + line0 + j) * snx + x] = v;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// y-adjoint: per voxel, over every line j and coil q:
//   H_j = s * sum_q amp_q h_q[j][x];  Z_j = conj(e^{i2pi theta_j}) H_j
//   comp_grad_c = sum_j rel_cj Z_j            (A^H r, complex)
//   fmap_grad   = -4 pi Im( sum_c m_c conj(sum_j t_j rel_cj Z_j) )      (dL/df, Hz)
//   r2_grad_c   = -2 Re( m_c conj(sum_j trf_j rel_cj Z_j) )             (dL/dR2_c, ms)
// One thread per column x and TY consecutive rows.
template <int TY, int NC, bool MAPS, bool GRADS>
__global__ void __launch_bounds__(128) yadjoint_kernel(const UnitDesc* __restrict__ units,
                                                       const int4* __restrict__ tiles) {
  extern __shared__ float smem[];
  const int4 tl = tiles[blockIdx.x];  // unit, y0, x0
  const UnitDesc& u = units[tl.x];
  const int snx = u.snx, sny = u.sny, ncomp = u.ncomp, nlines = u.n_lines, ncoils = u.ncoils;
  const int y0 = tl.y;
  float* Bt = smem;                      // [nlines][TY]
  float* Ey = smem + nlines * TY;        // [ncoils][TY]
  const int ys = u.ny / 2;
  const int oy = sny / u.ny;
  const int sys = oy * ys;
  for (int idx = threadIdx.x; idx < nlines * TY; idx += blockDim.x) {
    int j = idx / TY, ty = idx % TY;
    int y = y0 + ty;
    float v = 0.f;
    if (y < sny) {
      const LineRec& L = u.lines[j];
      long long K = L.ky - ys;
      long long Y = 2LL * (y - sys) - (oy - 1);
      long long m2 = 2LL * sny;
      double tv = (double)((K * Y) % m2) / (double)m2;
      if (u.flags & UF_EDDY) {
        double yc = ((double)y - sys - (oy - 1) / 2.0) / oy;
        tv += ((double)u.eddy_cy * yc + (double)u.eddy_qy * yc * yc) * (double)L.decay;
      }
      tv -= rint(tv);
      v = (float)tv;
    }
    Bt[idx] = v;
  }
  for (int idx = threadIdx.x; idx < ncoils * TY; idx += blockDim.x) {
    int q = idx / TY, ty = idx % TY;
    int y = y0 + ty;
    Ey[idx] = y < sny ? u.geo.ey[(size_t)q * sny + y] : 0.f;
  }
  __syncthreads();
  const int x = tl.z + threadIdx.x;
  if (x >= snx) return;
  const bool distort = (u.flags & UF_DISTORT) != 0;
  float a[TY], f[TY], m[TY][NC], r2[TY][NC], r2i[TY][NC], la[TY];
#pragma unroll
  for (int ty = 0; ty < TY; ++ty) {
    int y = min(y0 + ty, sny - 1);
    int i = x + snx * y;
    a[ty] = u.phase ? u.phase[i] : 0.f;
    f[ty] = distort ? u.fmap[i] : 0.f;
    la[ty] = (MAPS && u.log_amp) ? u.log_amp[i] : 0.f;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      m[ty][c] = (GRADS && c < ncomp) ? u.comp[(size_t)c * u.comp_stride + i] : 0.f;
      r2[ty][c] = r2i[ty][c] = 0.f;
      if (MAPS && c < ncomp) {
        float t2 = u.t2map ? u.t2map[(size_t)c * u.map_stride + i] : u.t2u[c];
        float ti = u.timap ? u.timap[(size_t)c * u.map_stride + i] : u.tiu[c];
        r2[ty][c] = 1.0f / t2;
        r2i[ty][c] = 1.0f / ti;
      }
    }
  }
  float2 cg[TY][NC], U[TY][GRADS ? NC : 1], V[TY][GRADS ? NC : 1];
#pragma unroll
  for (int ty = 0; ty < TY; ++ty)
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      cg[ty][c] = make_float2(0.f, 0.f);
      if (GRADS) U[ty][GRADS ? c : 0] = V[ty][GRADS ? c : 0] = make_float2(0.f, 0.f);
    }
  const float off = u.geo.coil_off;
  const float s = u.signal_scale;
  for (int j = 0; j < nlines; ++j) {
    const LineRec& L = u.lines[j];
    const float thi = L.t_hi, tlo = L.t_lo, trf = L.trf_ms, tinh = L.inhom_ms;
    const float tph = L.t_hi + L.t_lo;
    float rel[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) rel[c] = L.rel[c];
    float2 H[TY];
#pragma unroll
    for (int ty = 0; ty < TY; ++ty) H[ty] = make_float2(0.f, 0.f);
    const float2* hp = u.g + (size_t)j * snx + x;
    for (int q = 0; q < ncoils; ++q) {
      const float2 h = __ldg(hp + (size_t)q * nlines * snx);
      const float exq = __ldg(u.geo.ex + (size_t)q * snx + x);
#pragma unroll
      for (int ty = 0; ty < TY; ++ty) {
        float amp = fmaf(exq, Ey[q * TY + ty], off);
        H[ty].x = fmaf(amp, h.x, H[ty].x);
        H[ty].y = fmaf(amp, h.y, H[ty].y);
      }
    }
#pragma unroll
    for (int ty = 0; ty < TY; ++ty) {
      float th = a[ty] + Bt[j * TY + ty] + ft_turns(f[ty], thi, tlo);
      th = frac_turn(th);
      float sn, cs;
      __sincosf(kTwoPiF * th, &sn, &cs);
      // Z = conj(P) * H * s
      const float zr = s * (cs * H[ty].x + sn * H[ty].y);
      const float zi = s * (cs * H[ty].y - sn * H[ty].x);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        if (c < ncomp) {
          float r;
          if (MAPS)
            r = __expf(la[ty] - trf * r2[ty][c] - tinh * r2i[ty][c]);
          else
            r = rel[c];
          cg[ty][c].x = fmaf(r, zr, cg[ty][c].x);
          cg[ty][c].y = fmaf(r, zi, cg[ty][c].y);
          if (GRADS) {
            const int cc = GRADS ? c : 0;
            float rt = r * tph, rr = r * trf;
            U[ty][cc].x = fmaf(rt, zr, U[ty][cc].x);
            U[ty][cc].y = fmaf(rt, zi, U[ty][cc].y);
            V[ty][cc].x = fmaf(rr, zr, V[ty][cc].x);
            V[ty][cc].y = fmaf(rr, zi, V[ty][cc].y);
          }
        }
      }
    }
  }
  const size_t plane = (size_t)snx * sny;
#pragma unroll
  for (int ty = 0; ty < TY; ++ty) {
    int y = y0 + ty;
    if (y >= sny) break;
    size_t i = (size_t)x + (size_t)snx * y;
    float fg = 0.f;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      if (c >= ncomp) break;
      u.comp_grad[c * plane + i] = cg[ty][c];
      if (GRADS) {
        const int cc = GRADS ? c : 0;
        // Im(m conj(U)) with m real = -m * U.y
        fg += m[ty][c] * U[ty][cc].y;
        if (u.r2_grad) u.r2_grad[c * plane + i] = -2.0f * m[ty][c] * V[ty][cc].x;
      }
    }
    if (GRADS && u.fmap_grad) u.fmap_grad[i] = 4.0f * 3.14159265358979f * fg * (distort ? 1.f : 0.f);
  }
}

template <class K>
void set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) MRSIM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

}  // namespace

// ---- plans and launchers ----------------------------------------------------------------------
namespace {
constexpr int kT = 4;
constexpr int kTY = 4;
}  // namespace

EpiPlan::~EpiPlan() {
  for (void* p : allocs) cudaFree(p);
}

static void* dev_upload(EpiPlan* p, const void* src, size_t bytes) {
  void* d = nullptr;
  if (bytes == 0) return nullptr;
  MRSIM_CUDA(cudaMalloc(&d, bytes));
  p->allocs.push_back(d);
  MRSIM_CUDA(cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice));
  return d;
}

EpiPlan* epi_plan_create(const UnitDesc* hu, int n, const StaticDesc* hs, int ns) {
  EpiPlan* p = new EpiPlan();
  try {
    p->n_units = n;
    p->host_units.assign(hu, hu + n);
    p->d_units = (UnitDesc*)dev_upload(p, hu, sizeof(UnitDesc) * n);
    p->n_statics = ns;
    p->d_statics = (StaticDesc*)dev_upload(p, hs, sizeof(StaticDesc) * ns);
    for (int i = 0; i < ns; ++i) p->max_static_n = std::max(p->max_static_n, hs[i].snx * hs[i].sny);
    int max_coils = 0;
    for (int i = 0; i < n; ++i) {
      max_coils = std::max(max_coils, hu[i].ncoils);
      p->max_sny = std::max(p->max_sny, hu[i].sny);
      p->max_snx = std::max(p->max_snx, hu[i].snx);
      p->max_nx = std::max(p->max_nx, hu[i].nx);
      p->max_lines = std::max(p->max_lines, hu[i].n_lines);
      if (hu[i].ncomp > kMaxComp) fail("a unit has more than 8 compartments");
      if (hu[i].ncoils > kMaxCoils) fail("more than 64 coils");
    }
    p->max_coils = max_coils;
    int max_comp = 0;
    for (int i = 0; i < n; ++i) max_comp = std::max(max_comp, hu[i].ncomp);
    p->nc = max_comp <= 1 ? 1 : max_comp <= 2 ? 2 : max_comp <= 3 ? 3 : max_comp <= 4 ? 4 : 8;
    p->qg = max_coils <= 1 ? 1 : max_coils <= 2 ? 2 : max_coils <= 4 ? 4 : 8;
    for (int pass = 0; pass < 2; ++pass) {
      std::vector<int4> tiles;
      for (int i = 0; i < n; ++i) {
        if (((hu[i].flags & UF_MAPS) != 0) != (pass == 1)) continue;
        for (int l = 0; l < hu[i].n_lines; l += kT)
          for (int x0 = 0; x0 < hu[i].snx; x0 += 128)
            for (int q0 = 0; q0 < hu[i].ncoils; q0 += p->qg) tiles.push_back(make_int4(i, l, x0, q0));
      }
      p->n_ytiles[pass] = (int)tiles.size();
      p->d_ytiles[pass] = (int4*)dev_upload(p, tiles.data(), sizeof(int4) * tiles.size());
    }
    std::vector<int4> xt;
    for (int i = 0; i < n; ++i)
      for (int q = 0; q < hu[i].ncoils; ++q)
        for (int l = 0; l < hu[i].n_lines; l += XR) xt.push_back(make_int4(i, q, l, 0));
    p->n_xtiles = (int)xt.size();
    p->d_xtiles = (int4*)dev_upload(p, xt.data(), sizeof(int4) * xt.size());
    for (int pass = 0; pass < 4; ++pass) {
      bool maps = pass & 1, grads = pass & 2;
      std::vector<int4> yt;
      for (int i = 0; i < n; ++i) {
        bool um = (hu[i].flags & UF_MAPS) != 0;
        bool ug = (hu[i].flags & (UF_WANT_FMAP_GRAD | UF_WANT_R2_GRAD)) != 0;
        if (um != maps || ug != grads) continue;
        for (int y0 = 0; y0 < hu[i].sny; y0 += kTY)
          for (int x0 = 0; x0 < hu[i].snx; x0 += 128) yt.push_back(make_int4(i, y0, x0, 0));
      }
      p->n_atiles[pass] = (int)yt.size();
      p->d_atiles[pass] = (int4*)dev_upload(p, yt.data(), sizeof(int4) * yt.size());
    }
  } catch (...) {
    delete p;
    throw;
  }
  return p;
}

void epi_plan_statics(const EpiPlan* p, cudaStream_t st) {
  if (p->n_statics == 0) return;
  dim3 grid((p->max_static_n + 255) / 256, p->n_statics);
  statics_kernel<<<grid, 256, 0, st>>>(p->d_statics);
  MRSIM_CUDA(cudaGetLastError());
}

void epi_plan_forward(const EpiPlan* p, cudaStream_t st) {
  epi_plan_forward_ystage(p, st);
  epi_plan_forward_xstage(p, st);
}

void epi_plan_adjoint(const EpiPlan* p, cudaStream_t st) {
  epi_plan_adjoint_xstage(p, st);
  epi_plan_adjoint_ystage(p, st);
}

void epi_plan_forward_ystage(const EpiPlan* p, cudaStream_t st) {
  for (int pass = 0; pass < 2; ++pass) {
    if (p->n_ytiles[pass] == 0) continue;
    const bool maps = pass == 1;
    const int QG = p->qg, NCv = p->nc;
    const size_t sm = sizeof(float) * (size_t)p->max_sny * (kT + QG);
    bool launched = false;
#define MRSIM_Y(QGV, NCV, M)                                                            \
  if (QG == QGV && NCv == NCV && maps == M) {                                           \
    auto k = ystage_kernel<kT, QGV, NCV, M>;                                            \
    set_smem(k, sm);                                                                    \
    k<<<(unsigned)p->n_ytiles[pass], 128, sm, st>>>(p->d_units, (const Tile*)p->d_ytiles[pass]); \
    launched = true;                                                                    \
  }
#define MRSIM_YQ(NCV, M) MRSIM_Y(1, NCV, M) MRSIM_Y(2, NCV, M) MRSIM_Y(4, NCV, M) MRSIM_Y(8, NCV, M)
#define MRSIM_YN(M) MRSIM_YQ(1, M) MRSIM_YQ(2, M) MRSIM_YQ(3, M) MRSIM_YQ(4, M) MRSIM_YQ(8, M)
    MRSIM_YN(false) MRSIM_YN(true)
#undef MRSIM_YN
#undef MRSIM_YQ
#undef MRSIM_Y
    if (!launched) fail("no forward kernel instance for this unit shape");
    MRSIM_CUDA(cudaGetLastError());
  }
}

void epi_plan_forward_xstage(const EpiPlan* p, cudaStream_t st) {
  if (p->n_xtiles) {
    size_t sm = sizeof(float2) * XR * p->max_snx;
    set_smem(xstage_kernel, sm);
    xstage_kernel<<<(unsigned)p->n_xtiles, 128, sm, st>>>(p->d_units, p->d_xtiles);
    MRSIM_CUDA(cudaGetLastError());
  }
}

void epi_plan_adjoint_xstage(const EpiPlan* p, cudaStream_t st) {
  if (p->n_xtiles) {
    size_t sm = sizeof(float2) * XR * p->max_nx;
    set_smem(xadjoint_kernel, sm);
    xadjoint_kernel<<<(unsigned)p->n_xtiles, 128, sm, st>>>(p->d_units, p->d_xtiles);
    MRSIM_CUDA(cudaGetLastError());
  }
}

void epi_plan_adjoint_ystage(const EpiPlan* p, cudaStream_t st) {
  for (int pass = 0; pass < 4; ++pass) {
    if (p->n_atiles[pass] == 0) continue;
    const bool maps = pass & 1, grads = (pass & 2) != 0;
    const int NCv = p->nc;
    size_t sm = sizeof(float) * (size_t)kTY * (p->max_lines + p->max_coils);
    bool launched = false;
#define MRSIM_A(NCV, M, G)                                                              \
  if (NCv == NCV && maps == M && grads == G) {                                          \
    auto k = yadjoint_kernel<kTY, NCV, M, G>;                                           \
    set_smem(k, sm);                                                                    \
    k<<<(unsigned)p->n_atiles[pass], 128, sm, st>>>(p->d_units, p->d_atiles[pass]);     \
    launched = true;                                                                    \
  }
#define MRSIM_AN(M, G) MRSIM_A(1, M, G) MRSIM_A(2, M, G) MRSIM_A(3, M, G) MRSIM_A(4, M, G) MRSIM_A(8, M, G)
    MRSIM_AN(false, false) MRSIM_AN(true, false) MRSIM_AN(false, true) MRSIM_AN(true, true)
#undef MRSIM_AN
#undef MRSIM_A
    if (!launched) fail("no adjoint kernel instance for this unit shape");
    MRSIM_CUDA(cudaGetLastError());
  }
}

}  // namespace mrsim
