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
//
// Kernels, in the order a step runs them:
//   statics_kernel                     static phase a(x,y) in turns (FP64 per-slice quadratic)
//   ystage_q_kernel / ystage_kernel    y-stage (staged-input form; per-thread-load fallback);
//                                      with the 8-coil ring it accumulates 5 ey classes + offset
//   xfft_warp_kernel / xfft_kernel /   x-stage: warp-per-row FFT (N = 32..256), shared-memory
//   xgemm_kernel                       radix-2 FFT (other powers of two), DFT GEMM (other widths)
//   yadjoint_q_kernel / yadjoint_kernel  y-adjoint (fixed coil or class count; any coil count)
// The class-mode and packed (f32x2) paths are exact rearrangements: equal ey rows, and lanes that
// round like the scalar operations.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include <cstring>
#include <map>

#include "mrsim_internal.h"

// Template flags select whole code paths (packed or scalar, class or coil accumulators); the paths
// an instance does not take leave loops the front end reports as unreachable.
#pragma nv_diag_suppress 128

namespace mrsim {

namespace {

constexpr float kTwoPiF = 6.28318530717958647692f;

// The reduced phase s + f t in turns (s = static phase + k.r term, |s| <= 1 turn; f the voxel's
// off-resonance in Hz; t = t_hi + t_lo the line time in s, |f t| < 2^22) with one rounding to an
// integer: n = round(s + f t_hi) by adding and subtracting 1.5 * 2^23 (the FMA's rounded value
// serves only to choose n), r = f t_hi - n from one FMA of the exact product (|r| < 2: one rounding
// of at most ulp(1)/2), and
//   theta = (r + s) + f t_lo,   |theta| <= 1/2 + ulps,
// whose last two roundings are at most ulp(1/2)/2 each.
__device__ __forceinline__ float phase_turns(float s, float f, float t_hi, float t_lo) {
  const float nn = __fsub_rn(12582912.0f, __fadd_rn(fmaf(f, t_hi, s), 12582912.0f));  // -n
  return fmaf(f, t_lo, __fadd_rn(fmaf(f, t_hi, nn), s));
}

// Packed FP32 pairs (sm_100 add/sub/mul/fma.rn.f32x2): one instruction for two lanes, each lane
// rounding exactly like the scalar operation, so a packed computation is bitwise the scalar one.
__device__ __forceinline__ unsigned long long pk2(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 upk2(unsigned long long r) {
  float2 d;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(r));
  return d;
}
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)), "l"(pk2(c)));
  return upk2(d);
}
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(d);
}
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(d);
}
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk2(a)), "l"(pk2(b)));
  return upk2(d);
}
__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

// The reduced phase s + f t (s = static phase + k.r term, |s| <= 1 turn, t = t_hi + t_lo) on a pair
// of lanes with one rounding to an integer: n = round(s + f t_hi) (the FMA's rounded value serves
// only to choose n), r = f t_hi - n from one FMA of the exact product (|r| < 2: one rounding of
// at most ulp(1)/2), and
//   theta = (r + s) + f t_lo,   |theta| <= 1/2 + ulps,
// whose last two roundings are at most ulp(1/2)/2 each: six packed operations.
__device__ __forceinline__ float2 phase_turns2(float2 s, float2 f, float2 t_hi, float2 t_lo) {
  const float2 M = dup2(12582912.0f);
  const float2 nn = fsub2(M, fadd2(ffma2(f, t_hi, s), M));  // -n
  const float2 r = ffma2(f, t_hi, nn);
  return ffma2(f, t_lo, fadd2(r, s));
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// cp.async helpers (16-byte copies zero-fill the bytes past src_bytes)
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem_src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait_n() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gmem_src), "r"(src_bytes));
}

// ---------------------------------------------------------------------------------------------
// statics: a(x,y) = frac( (phi0 + eddy object phase) / 2pi ) in FP64, stored as f32 turns.
// phi0 = phase0[i] (explicit) or the phase model `PhaseModel::at` (phase.rs:141) sampled by
// `phase_slice` (kspace.rs:1156-1180).
__global__ void statics_kernel(const StaticDesc* descs) {
  const StaticDesc& d = descs[blockIdx.y];
  const int n = d.snx * d.sny;
  const double inv_tau = 0.15915494309189533577;
  const int ox = d.snx / d.nx, oy = d.sny / d.ny;
  const int sxs = ox * (d.nx / 2), sys = oy * (d.ny / 2);
  const double xoff = (ox - 1.0) / 2.0, yoff = (oy - 1.0) / 2.0;
  const bool explicit_phase = (d.flags & 1) != 0;
  // Within a slice the phase model is a quadratic in (x, y): with r0 = (x - sx - off)/o,
  // r1 = (y - sy - off)/o and r2 the slice coordinate, background + shot term are
  //   A + B r0 + C r1 + D r0^2 + E r1^2 + F r0 r1
  // and the eddy object-phase ramp is affine in x and y.  Each thread forms the six FP64
  // coefficients once and evaluates its voxels by Horner's rule.
  double c00 = 0, cx = 0, cy = 0, cxx = 0, cyy = 0, cxy = 0;
  {
    const double o = d.o, sx = d.snx / 2.0, sy = d.sny / 2.0, off = (o - 1.0) / 2.0;
    const double r2 = d.z - d.nz_full / 2.0;
    const double* c = d.bg;
    double A = 0, B = 0, C = 0, D = 0, E = 0, F = 0;
    if (!explicit_phase) {
      const double* q = d.shot_q;
      const double* dx = d.shot_dx;
      const double* rot = d.shot_rot;
      A = d.global + c[0] + c[3] * r2 + c[6] * r2 * r2 + q[0] * (dx[0] + rot[1] * r2) +
          q[1] * (dx[1] - rot[0] * r2) + q[2] * dx[2];
      B = c[1] + c[8] * r2 + q[1] * rot[2] - q[2] * rot[1];
      C = c[2] + c[9] * r2 - q[0] * rot[2] + q[2] * rot[0];
      D = c[4];
      E = c[5];
      F = c[7];
    }
    // r0 = a0 + x / o, r1 = b0 + y / o
    const double a0 = -(sx + off) / o, b0 = -(sy + off) / o, io = 1.0 / o;
    c00 = A + B * a0 + C * b0 + D * a0 * a0 + E * b0 * b0 + F * a0 * b0;
    cx = (B + 2.0 * D * a0 + F * b0) * io;
    cy = (C + 2.0 * E * b0 + F * a0) * io;
    cxx = D * io * io;
    cyy = E * io * io;
    cxy = F * io * io;
    if (d.flags & 2) {  // + e0 (x - sxs - xoff)/ox + e1 (y - sys - yoff)/oy + e2 zc
      const double* e = d.eddy_phase_coef;
      c00 += -e[0] * (sxs + xoff) / ox - e[1] * (sys + yoff) / oy + e[2] * d.zc_c;
      cx += e[0] / ox;
      cy += e[1] / oy;
    }
  }
  const double* __restrict__ phase0 = d.phase0;
  float* __restrict__ out = d.out;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = i % d.snx, y = i / d.snx;
    double p0 = explicit_phase ? phase0[i] : fma(x, fma(cxx, x, fma(cxy, y, cx)), fma(y, fma(cyy, y, cy), c00));
    if (explicit_phase && (d.flags & 2)) p0 += fma(cx, x, fma(cy, y, c00));
    double tt = p0 * inv_tau;
    tt -= rint(tt);
    out[i] = (float)tt;
  }
}

// ---------------------------------------------------------------------------------------------
// y-stage of the forward.  One CTA = (unit, T lines, 128 columns, QG coils); one thread per
// column x accumulates T*QG complex sums over every sim row y.
struct Tile {
  int unit, line0, x0, q0;
};

template <int T, int QG, int NC, bool MAPS>
__global__ void __launch_bounds__(128, 4) ystage_kernel(const UnitDesc* __restrict__ units,
                                                        const Tile* __restrict__ tiles) {
  // A CTA of 128 threads: one column each, T lines x QG coils per thread.
  constexpr int LG = 1;
  constexpr int TL = LG * T;  // lines per CTA
  static_assert(T == 4, "the phase table is read as float4");
  extern __shared__ __align__(16) float smem[];
  const Tile tl = tiles[blockIdx.x];
  const UnitDesc& u = units[tl.unit];
  const int snx = u.snx, sny = u.sny;
  const int ncomp = u.ncomp;
  float* Bt = smem;                 // [sny][TL] phase terms per (row, line)
  float* Ey = smem + sny * TL;      // [sny][QGP] (QGP = QG rounded up to 4)
  constexpr int QGP = (QG + 3) / 4 * 4;
  __shared__ float rel_s[TL][kMaxComp];
  __shared__ float tinh_s[TL], trf_s[TL];
  __shared__ float thi_s[TL], tlo_s[TL];

  const int nl = min(TL, u.n_lines - tl.line0);
  const int ys = u.ny / 2;
  const int oy = sny / u.ny;
  const int sys = oy * ys;
  for (int idx = threadIdx.x; idx < sny * TL; idx += blockDim.x) {
    const int y = idx / TL, j = idx % TL;
    float v = 0.f;
    if (j < nl) {
      const LineRec& L = u.lines[tl.line0 + j];
      const long long K = L.ky - ys;
      const long long Y = 2LL * (y - sys) - (oy - 1);
      const long long m2 = 2LL * sny;
      double tv = (double)((K * Y) % m2) / (double)m2;
      if (u.flags & UF_EDDY) {
        const double yc = ((double)y - sys - (oy - 1) / 2.0) / oy;
        tv += ((double)u.eddy_cy * yc + (double)u.eddy_qy * yc * yc) * (double)L.decay;
      }
      tv -= rint(tv);
      v = (float)tv;
    }
    Bt[idx] = v;
  }
  for (int idx = threadIdx.x; idx < QGP * sny; idx += blockDim.x) {
    const int y = idx / QGP, qq = idx % QGP;
    const int q = tl.q0 + qq;
    Ey[idx] = (qq < QG && q < u.ncoils) ? u.geo.ey[(size_t)q * sny + y] : 0.f;
  }
  if (threadIdx.x < TL) {
    const int j = threadIdx.x;
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

  const int col = threadIdx.x & 127, lg = threadIdx.x >> 7;
  const int jb = lg * T;  // this thread's first line within the CTA
  const int x = tl.x0 + col;
  const bool xok = x < snx;
  const int xs_ = xok ? x : 0;
  float exq[QG];
  const float off = u.geo.coil_off;
#pragma unroll
  for (int qq = 0; qq < QG; ++qq) {
    const int q = tl.q0 + qq;
    exq[qq] = (xok && q < u.ncoils) ? u.geo.ex[(size_t)q * snx + x] : 0.f;
  }
  float thi[T], tlo[T], relr[T][NC];
#pragma unroll
  for (int j = 0; j < T; ++j) {
    thi[j] = thi_s[jb + j];
    tlo[j] = tlo_s[jb + j];
#pragma unroll
    for (int c = 0; c < NC; ++c) relr[j][c] = rel_s[jb + j][c];
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
  // row y's inputs, prefetched one row ahead
  float na = 0.f, nf = 0.f, nm[NC];
  {
    const int i = xs_;
    na = phase ? __ldg(phase + i) : 0.f;
    nf = distort ? __ldg(fmap + i) : 0.f;
#pragma unroll
    for (int c = 0; c < NC; ++c) nm[c] = c < ncomp ? __ldg(comp + (size_t)c * u.comp_stride + i) : 0.f;
  }
  for (int y = 0; y < sny; ++y) {
    const int i = xs_ + snx * y;
    const float a = na, f = nf;
    float m[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) m[c] = nm[c];
    if (y + 1 < sny) {
      const int i1 = i + snx;
      na = phase ? __ldg(phase + i1) : 0.f;
      nf = distort ? __ldg(fmap + i1) : 0.f;
#pragma unroll
      for (int c = 0; c < NC; ++c) nm[c] = c < ncomp ? __ldg(comp + (size_t)c * u.comp_stride + i1) : 0.f;
    }
    float r2[MAPS ? NC : 1], r2i[MAPS ? NC : 1];
    float la = 0.f;
    if (MAPS) {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        r2[MAPS ? c : 0] = r2i[MAPS ? c : 0] = 0.f;
        if (c < ncomp) {
          const float t2 = u.t2map ? __ldg(u.t2map + (size_t)c * u.map_stride + i) : u.t2u[c];
          const float ti = u.timap ? __ldg(u.timap + (size_t)c * u.map_stride + i) : u.tiu[c];
          r2[MAPS ? c : 0] = 1.0f / t2;
          r2i[MAPS ? c : 0] = 1.0f / ti;
        }
      }
      if (u.log_amp) la = __ldg(u.log_amp + i);
    }
    float amp[QG];
#pragma unroll
    for (int q4 = 0; q4 < QGP; q4 += 4) {
      const float4 e4 = *reinterpret_cast<const float4*>(Ey + y * QGP + q4);
      const float ev[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (q4 + k < QG) amp[q4 + k] = fmaf(exq[q4 + k], ev[k], off);
    }
    const float4 b4 = *reinterpret_cast<const float4*>(Bt + y * TL + jb);
    const float bt[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
    for (int j = 0; j < T; ++j) {
      const float th = phase_turns(a + bt[j], f, thi[j], tlo[j]);
      float sn, cs;
      __sincosf(kTwoPiF * th, &sn, &cs);
      float W = 0.f;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        if (c < ncomp) {
          float r;
          if (MAPS)
            r = __expf(la - trf_s[jb + j] * r2[MAPS ? c : 0] - tinh_s[jb + j] * r2i[MAPS ? c : 0]);
          else
            r = relr[j][c];
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
    const int q = tl.q0 + qq;
    if (q >= u.ncoils) break;
#pragma unroll
    for (int j = 0; j < T; ++j) {
      if (jb + j < nl)
        u.g[((size_t)q * u.n_lines + tl.line0 + jb + j) * snx + x] = make_float2(acc[j][qq].x * s, acc[j][qq].y * s);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// y-stage of the forward with the per-row inputs staged in shared memory (every unit of the plan
// has snx % 4 == 0 and 16-byte aligned input planes).  Same sums as ystage_kernel:
//   * a CTA of 256 threads covers 128 columns x 8 lines (two groups of 4 lines, one column each)
//     x QG coils, so each row's inputs serve 8 lines;
//   * the inputs of RC rows (static phase, fieldmap, compartments, and with voxel maps T2, T2',
//     log amplitude) arrive through a 3-stage ring filled by cooperative 16-byte cp.async, one
//     barrier per RC rows, in place of per-thread global loads one row ahead.
constexpr int kFwdStages = 3;
__host__ __device__ __forceinline__ constexpr int fwdq_planes(int nc, bool maps) { return maps ? 3 + 3 * nc : 2 + nc; }
__host__ __device__ __forceinline__ constexpr int fwdq_rows(int nc, bool maps) {
  return fwdq_planes(nc, maps) <= 5 ? 8 : fwdq_planes(nc, maps) <= 12 ? 4 : 2;
}

// NV > 0: the tile holds every coil of the unit and accumulates coil classes instead of coils
// (NV = classes + 1 for the coil offset): acc_v += ey_v(y) W P, acc_off += W P, and the epilogue
// expands g_q = s (ex_q acc_cls(q) + off acc_off).
// cls_rows (with NV): write the class rows G_v = s T_v and G_off = s off T_off ([v][line][x], the
// layout the class-mode x-stage expands) instead of the coil rows.
template <int QG, int NV, int NC, bool MAPS>
__global__ void __launch_bounds__(256, 2) ystage_q_kernel(const UnitDesc* __restrict__ units,
                                                          const Tile* __restrict__ tiles, int cls_rows) {
  constexpr int T = 4, TL = 8;
  constexpr int NA = NV ? NV : QG;             // accumulators per line
  constexpr int NPL = fwdq_planes(NC, MAPS);
  constexpr int RC = fwdq_rows(NC, MAPS);
  constexpr int STAGE = NPL * RC * 128;        // floats per stage
  constexpr int PIECES = NPL * RC * 32;        // 16-byte pieces per stage
  constexpr int PPT = (PIECES + 255) / 256;
  constexpr int QGP = (NA + 3) / 4 * 4;
  // plane order: 0 static phase, 1 fieldmap, 2.. compartments, then T2, T2' maps and log amplitude
  constexpr int P_COMP = 2, P_T2 = 2 + NC, P_TI = 2 + 2 * NC, P_LA = 2 + 3 * NC;
  extern __shared__ __align__(16) float smem[];
  float* ring = smem;                           // [stage][plane][RC][128]
  float* Bt = ring + kFwdStages * STAGE;        // [sny][TL]
  const Tile tl = tiles[blockIdx.x];
  const UnitDesc& u = units[tl.unit];
  const int snx = u.snx, sny = u.sny, ncomp = u.ncomp;
  float* Ey = Bt + sny * TL;                    // [sny][QGP]: ey per coil, or per class and 1
  __shared__ const float* plane_s[NPL];
  __shared__ float rel_s[TL][kMaxComp];
  __shared__ float tinh_s[TL], trf_s[TL], thi_s[TL], tlo_s[TL];
  const int tid = threadIdx.x;
  const bool distort = (u.flags & UF_DISTORT) != 0;
  if (tid < NPL) {
    const float* pp = nullptr;
    const int k = tid;
    if (k == 0) pp = u.phase;
    else if (k == 1) pp = distort ? u.fmap : nullptr;
    else if (k < P_T2) pp = (k - P_COMP) < ncomp ? u.comp + (size_t)(k - P_COMP) * u.comp_stride : nullptr;
    else if (k < P_TI) pp = ((k - P_T2) < ncomp && u.t2map) ? u.t2map + (size_t)(k - P_T2) * u.map_stride : nullptr;
    else if (k < P_LA) pp = ((k - P_TI) < ncomp && u.timap) ? u.timap + (size_t)(k - P_TI) * u.map_stride : nullptr;
    else pp = u.log_amp;
    plane_s[k] = pp;
  }
  __syncthreads();
  const int x0 = tl.x0;
  const int nch = (sny + RC - 1) / RC;
  auto issue_rows = [&](int c) {
    if (c < nch) {
      float* dst = ring + (c % kFwdStages) * STAGE;
#pragma unroll
      for (int i = 0; i < PPT; ++i) {
        const int k = tid + 256 * i;
        if (PIECES % 256 == 0 || k < PIECES) {
          const int pl = k / (RC * 32), rem = k % (RC * 32);
          const int r = rem >> 5, c4 = (rem & 31) * 4;
          // absent planes (no static phase, no distortion, compartments past ncomp) and rows
          // or columns past the plane zero-fill: the row loop reads every plane unconditionally
          const float* base = plane_s[pl];
          const int y = c * RC + r, xx = x0 + c4;
          const bool ok = base != nullptr && y < sny && xx < snx;
          cp_async16(dst + (pl * RC + r) * 128 + c4, ok ? base + (size_t)y * snx + xx : (const float*)u.g, ok ? 16 : 0);
        }
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int c = 0; c < kFwdStages - 1; ++c) issue_rows(c);

  const int nl = min(TL, u.n_lines - tl.line0);
  const int ys = u.ny / 2;
  const int oy = sny / u.ny;
  const int sys = oy * ys;
  for (int idx = tid; idx < sny * TL; idx += 256) {
    const int y = idx / TL, j = idx % TL;
    float v = 0.f;
    if (j < nl) {
      const LineRec& L = u.lines[tl.line0 + j];
      const long long K = L.ky - ys;
      const long long Y = 2LL * (y - sys) - (oy - 1);
      const long long m2 = 2LL * sny;
      double tv = (double)((K * Y) % m2) / (double)m2;
      if (u.flags & UF_EDDY) {
        const double yc = ((double)y - sys - (oy - 1) / 2.0) / oy;
        tv += ((double)u.eddy_cy * yc + (double)u.eddy_qy * yc * yc) * (double)L.decay;
      }
      tv -= rint(tv);
      v = (float)tv;
    }
    Bt[idx] = v;
  }
  for (int idx = tid; idx < QGP * sny; idx += 256) {
    const int y = idx / QGP, qq = idx % QGP;
    if (NV) {
      const int nc = u.geo.ncls;
      Ey[idx] = qq < nc ? u.geo.eyc[(size_t)qq * sny + y] : (qq == nc ? 1.f : 0.f);
    } else {
      const int q = tl.q0 + qq;
      Ey[idx] = (qq < QG && q < u.ncoils) ? u.geo.ey[(size_t)q * sny + y] : 0.f;
    }
  }
  if (tid < TL) {
    const int j = tid;
    if (j < nl) {
      const LineRec& L = u.lines[tl.line0 + j];
      thi_s[j] = L.t_hi;
      tlo_s[j] = L.t_lo;
      tinh_s[j] = L.inhom_ms;
      trf_s[j] = L.trf_ms;
      for (int c = 0; c < kMaxComp; ++c) rel_s[j][c] = c < ncomp ? L.rel[c] : 0.f;
    } else {
      thi_s[j] = tlo_s[j] = tinh_s[j] = trf_s[j] = 0.f;
      for (int c = 0; c < kMaxComp; ++c) rel_s[j][c] = 0.f;
    }
  }
  __syncthreads();

  const int col = tid & 127, lg = tid >> 7;
  const int jb = lg * T;
  const int x = x0 + col;
  const bool xok = x < snx;
  const float off = u.geo.coil_off;
  float exq[NV ? 1 : QG];
  if (!NV) {
#pragma unroll
    for (int qq = 0; qq < QG; ++qq) {
      const int q = tl.q0 + qq;
      exq[NV ? 0 : qq] = (xok && q < u.ncoils) ? u.geo.ex[(size_t)q * snx + x] : 0.f;
    }
  }
  float thi[T], tlo[T], relr[T][MAPS ? 1 : NC], trf[MAPS ? T : 1], tinh[MAPS ? T : 1];
#pragma unroll
  for (int j = 0; j < T; ++j) {
    thi[j] = thi_s[jb + j];
    tlo[j] = tlo_s[jb + j];
    if (MAPS) {
      trf[MAPS ? j : 0] = trf_s[jb + j];
      tinh[MAPS ? j : 0] = tinh_s[jb + j];
    } else {
#pragma unroll
      for (int c = 0; c < NC; ++c) relr[j][MAPS ? 0 : c] = rel_s[jb + j][c];
    }
  }
  const bool has_t2 = MAPS && plane_s[P_T2] != nullptr, has_ti = MAPS && plane_s[P_TI] != nullptr;
  const bool has_la = MAPS && plane_s[P_LA] != nullptr;
  float2 acc[T][NA];
#pragma unroll
  for (int j = 0; j < T; ++j)
#pragma unroll
    for (int qq = 0; qq < NA; ++qq) acc[j][qq] = make_float2(0.f, 0.f);

  for (int c = 0; c < nch; ++c) {
    cp_async_wait_n<kFwdStages - 2>();
    __syncthreads();  // rows of chunk c landed; every thread is done with chunk c - 1
    issue_rows(c + kFwdStages - 1);
    const float* S = ring + (c % kFwdStages) * STAGE + col;
    const int rn = min(RC, sny - c * RC);
    for (int r = 0; r < rn; ++r) {
      const int y = c * RC + r;
      const float a = S[(0 * RC + r) * 128];
      const float f = S[(1 * RC + r) * 128];
      float m[NC];
#pragma unroll
      for (int cc = 0; cc < NC; ++cc) m[cc] = S[((P_COMP + cc) * RC + r) * 128];
      float r2[MAPS ? NC : 1], r2i[MAPS ? NC : 1];
      float la = 0.f;
      if (MAPS) {
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) {
          r2[MAPS ? cc : 0] = r2i[MAPS ? cc : 0] = 0.f;
          if (cc < ncomp) {
            const float t2 = has_t2 ? S[((P_T2 + cc) * RC + r) * 128] : u.t2u[cc];
            const float ti = has_ti ? S[((P_TI + cc) * RC + r) * 128] : u.tiu[cc];
            r2[MAPS ? cc : 0] = 1.0f / t2;
            r2i[MAPS ? cc : 0] = 1.0f / ti;
          }
        }
        if (has_la) la = S[(P_LA * RC + r) * 128];
      }
      float amp[NA];
#pragma unroll
      for (int q4 = 0; q4 < QGP; q4 += 4) {
        const float4 e4 = *reinterpret_cast<const float4*>(Ey + y * QGP + q4);
        const float ev[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (q4 + k < NA) amp[q4 + k] = NV ? ev[k] : fmaf(exq[NV ? 0 : q4 + k], ev[k], off);
      }
      const float4 b4 = *reinterpret_cast<const float4*>(Bt + y * TL + jb);
      const float bt[4] = {b4.x, b4.y, b4.z, b4.w};
      if (NV && !MAPS) {
        // lines (0, 1) and (2, 3) as packed pairs: the same arithmetic, two lanes per instruction
        const float2 a2 = dup2(a), f2 = dup2(f);
#pragma unroll
        for (int jp = 0; jp < T; jp += 2) {
          float2 th = phase_turns2(fadd2(a2, make_float2(bt[jp], bt[jp + 1])), f2,
                                   make_float2(thi[jp], thi[jp + 1]), make_float2(tlo[jp], tlo[jp + 1]));
          th = fmul2(dup2(kTwoPiF), th);
          float s0, c0, s1, c1;
          __sincosf(th.x, &s0, &c0);
          __sincosf(th.y, &s1, &c1);
          float2 W = fmul2(make_float2(relr[jp][MAPS ? 0 : 0], relr[jp + 1][MAPS ? 0 : 0]), dup2(m[0]));
#pragma unroll
          for (int cc = 1; cc < NC; ++cc)
            W = ffma2(make_float2(relr[jp][MAPS ? 0 : cc], relr[jp + 1][MAPS ? 0 : cc]), dup2(m[cc]), W);
          const float2 w0 = fmul2(dup2(W.x), make_float2(c0, s0)), w1 = fmul2(dup2(W.y), make_float2(c1, s1));
#pragma unroll
          for (int qq = 0; qq < NA - 1; ++qq) {
            acc[jp][qq] = ffma2(dup2(amp[qq]), w0, acc[jp][qq]);
            acc[jp + 1][qq] = ffma2(dup2(amp[qq]), w1, acc[jp + 1][qq]);
          }
          acc[jp][NA - 1] = fadd2(acc[jp][NA - 1], w0);
          acc[jp + 1][NA - 1] = fadd2(acc[jp + 1][NA - 1], w1);
        }
        continue;
      }
#pragma unroll
      for (int j = 0; j < T; ++j) {
        const float th = phase_turns(a + bt[j], f, thi[j], tlo[j]);
        float sn, cs;
        __sincosf(kTwoPiF * th, &sn, &cs);
        float W = 0.f;
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) {
          if (!MAPS || cc < ncomp) {  // class decay: rel and m are 0 past ncomp
            float rr;
            if (MAPS)
              rr = __expf(la - trf[MAPS ? j : 0] * r2[MAPS ? cc : 0] - tinh[MAPS ? j : 0] * r2i[MAPS ? cc : 0]);
            else
              rr = relr[j][MAPS ? 0 : cc];
            W = fmaf(rr, m[cc], W);
          }
        }
        const float wr = W * cs, wi = W * sn;
#pragma unroll
        for (int qq = 0; qq < NA; ++qq) {
          if (NV && qq == NA - 1) {  // the coil-offset row is all ones
            acc[j][qq].x += wr;
            acc[j][qq].y += wi;
          } else if (NV) {
            acc[j][qq] = ffma2(make_float2(amp[qq], amp[qq]), make_float2(wr, wi), acc[j][qq]);
          } else {
            acc[j][qq].x = fmaf(amp[qq], wr, acc[j][qq].x);
            acc[j][qq].y = fmaf(amp[qq], wi, acc[j][qq].y);
          }
        }
      }
    }
  }
  cp_async_wait0();
  if (!xok) return;
  const float s = u.signal_scale;
  if (NV && cls_rows) {
#pragma unroll
    for (int j = 0; j < T; ++j) {
      if (jb + j >= nl) break;
#pragma unroll
      for (int v = 0; v < NA; ++v) {
        const float sv = v == NA - 1 ? s * off : s;
        u.g[((size_t)v * u.n_lines + tl.line0 + jb + j) * snx + x] = make_float2(sv * acc[j][v].x, sv * acc[j][v].y);
      }
    }
    return;
  }
  if (NV) {
    // expand the classes to the unit's coils (all in this tile)
    for (int q = 0; q < u.ncoils; ++q) {
      const int cl = u.geo.cls[q];
      const float e = s * u.geo.ex[(size_t)q * snx + x], o = s * off;
#pragma unroll
      for (int j = 0; j < T; ++j) {
        float2 v = acc[j][0];
#pragma unroll
        for (int k = 1; k < NA - 1; ++k)
          if (cl == k) v = acc[j][k];
        if (jb + j < nl)
          u.g[((size_t)q * u.n_lines + tl.line0 + jb + j) * snx + x] =
              make_float2(fmaf(e, v.x, o * acc[j][NA - 1].x), fmaf(e, v.y, o * acc[j][NA - 1].y));
      }
    }
    return;
  }
#pragma unroll
  for (int qq = 0; qq < QG; ++qq) {
    const int q = tl.q0 + qq;
    if (q >= u.ncoils) break;
#pragma unroll
    for (int j = 0; j < T; ++j) {
      if (jb + j < nl)
        u.g[((size_t)q * u.n_lines + tl.line0 + jb + j) * snx + x] = make_float2(acc[j][qq].x * s, acc[j][qq].y * s);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// y-adjoint: per voxel, over every line j and coil q:
//   H_j = s * sum_q (ex_q ey_q + off) h_q[j][x];   Z_j = conj(e^{i2pi theta_j}) H_j
//   comp_grad_c = sum_j rel_cj Z_j                          (A^H r, complex)
//   fmap_grad   = 4 pi sum_c m_c Im(sum_j t_j rel_cj Z_j)   (dL/dfmap, L = sum |r|^2)
//   r2_grad_c   = -2 m_c Re(sum_j trf_j rel_cj Z_j)         (dL/dR2_c)
// A CTA of 128 threads covers 128 columns x TY rows (one column each).  The line table sits in
// shared memory; h arrives by cp.async in double-buffered chunks of JC lines x every coil.
// The number of lines per h chunk for `ncoils` coils (16 coil-lines per chunk, at least one line).
__host__ __device__ __forceinline__ int adjoint_chunk_lines(int ncoils) { return ncoils >= 16 ? 1 : 16 / ncoils; }

template <int TY, int NC, bool MAPS, bool GRADS>
__global__ void __launch_bounds__(128) yadjoint_kernel(const UnitDesc* __restrict__ units,
                                                       const int4* __restrict__ tiles) {
  extern __shared__ __align__(16) float smem[];
  static_assert(TY == 4, "the row tables are read as float4");
  constexpr int ROWS = TY;
  const int4 tl = tiles[blockIdx.x];  // unit, y0, x0
  const UnitDesc& u = units[tl.x];
  const int snx = u.snx, sny = u.sny, ncomp = u.ncomp, nlines = u.n_lines, ncoils = u.ncoils;
  const int y0 = tl.y;
  const int JC = adjoint_chunk_lines(ncoils);
  // shared layout: h buffers (2 x JC x ncoils x 128 float2), then floats
  float2* hbuf = reinterpret_cast<float2*>(smem);
  float* Bt = reinterpret_cast<float*>(hbuf + 2 * JC * ncoils * 128);  // [nlines][ROWS]
  float* Ey = Bt + nlines * ROWS;                                        // [ncoils][ROWS]
  float* Ex = Ey + ncoils * ROWS;                                        // [ncoils][128], scale folded
  float* Lt = Ex + ncoils * 128;                                         // [nlines][LF] line table
  constexpr int LF = 5 + NC;  // t_hi, t_lo, trf, inhom, t_phase, rel[NC]
  const int ys = u.ny / 2;
  const int oy = sny / u.ny;
  const int sys = oy * ys;
  const int col = threadIdx.x;
  const int x = tl.z + col;
  const bool xok = x < snx;
  const float2* __restrict__ hcol = u.g + (xok ? x : 0);
  const size_t qstride = (size_t)nlines * snx;
  // the first h chunk is in flight while the tables fill
  auto issue_chunk = [&](int c, int buf) {
    const int j0 = c * JC;
    for (int jj = 0; jj < JC; ++jj) {
      const int j = j0 + jj;
      if (j >= nlines) break;
      for (int q = 0; q < ncoils; ++q)
        cp_async8(hbuf + ((size_t)(buf * JC + jj) * ncoils + q) * 128 + col, hcol + q * qstride + (size_t)j * snx);
    }
    cp_async_commit();
  };
  const int nchunks = (nlines + JC - 1) / JC;
  if (nchunks > 0) issue_chunk(0, 0);
  for (int idx = threadIdx.x; idx < nlines * ROWS; idx += blockDim.x) {
    const int j = idx / ROWS, r = idx % ROWS;
    const int y = y0 + r;
    float v = 0.f;
    if (y < sny) {
      const LineRec& L = u.lines[j];
      const long long K = L.ky - ys;
      const long long Y = 2LL * (y - sys) - (oy - 1);
      const long long m2 = 2LL * sny;
      double tv = (double)((K * Y) % m2) / (double)m2;
      if (u.flags & UF_EDDY) {
        const double yc = ((double)y - sys - (oy - 1) / 2.0) / oy;
        tv += ((double)u.eddy_cy * yc + (double)u.eddy_qy * yc * yc) * (double)L.decay;
      }
      tv -= rint(tv);
      v = (float)tv;
    }
    Bt[idx] = v;
  }
  for (int idx = threadIdx.x; idx < ncoils * ROWS; idx += blockDim.x) {
    const int q = idx / ROWS, r = idx % ROWS;
    const int y = y0 + r;
    Ey[idx] = y < sny ? u.geo.ey[(size_t)q * sny + y] : 0.f;
  }
  for (int idx = threadIdx.x; idx < ncoils * 128; idx += blockDim.x) {
    const int q = idx / 128, c = idx % 128;
    const int xx = tl.z + c;
    Ex[idx] = xx < snx ? u.signal_scale * u.geo.ex[(size_t)q * snx + xx] : 0.f;
  }
  for (int j = threadIdx.x; j < nlines; j += blockDim.x) {
    const LineRec& L = u.lines[j];
    float* e = Lt + j * LF;
    e[0] = L.t_hi;
    e[1] = L.t_lo;
    e[2] = L.trf_ms;
    e[3] = L.inhom_ms;
    e[4] = L.t_hi + L.t_lo;
#pragma unroll
    for (int c = 0; c < NC; ++c) e[5 + c] = L.rel[c];
  }
  __syncthreads();
  const bool active = xok && y0 < sny;
  const bool distort = (u.flags & UF_DISTORT) != 0;
  float a[TY], f[TY], r2[TY][MAPS ? NC : 1], r2i[TY][MAPS ? NC : 1], la[TY];
#pragma unroll
  for (int ty = 0; ty < TY; ++ty) {
    const int y = min(y0 + ty, sny - 1);
    const int i = (xok ? x : 0) + snx * y;
    a[ty] = u.phase ? __ldg(u.phase + i) : 0.f;
    f[ty] = distort ? __ldg(u.fmap + i) : 0.f;
    la[ty] = (MAPS && u.log_amp) ? __ldg(u.log_amp + i) : 0.f;
    if (MAPS) {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        r2[ty][MAPS ? c : 0] = r2i[ty][MAPS ? c : 0] = 0.f;
        if (c < ncomp) {
          const float t2 = u.t2map ? __ldg(u.t2map + (size_t)c * u.map_stride + i) : u.t2u[c];
          const float ti = u.timap ? __ldg(u.timap + (size_t)c * u.map_stride + i) : u.tiu[c];
          r2[ty][MAPS ? c : 0] = 1.0f / t2;
          r2i[ty][MAPS ? c : 0] = 1.0f / ti;
        }
      }
    }
  }
  float2 cg[TY][NC];
  float Uy[TY][GRADS ? NC : 1], Vx[TY][GRADS ? NC : 1];
#pragma unroll
  for (int ty = 0; ty < TY; ++ty)
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      cg[ty][c] = make_float2(0.f, 0.f);
      if (GRADS) Uy[ty][GRADS ? c : 0] = Vx[ty][GRADS ? c : 0] = 0.f;
    }
  const float soff = u.signal_scale * u.geo.coil_off;
  for (int c = 0; c < nchunks; ++c) {
    const int buf = c & 1;
    if (c + 1 < nchunks) {
      issue_chunk(c + 1, buf ^ 1);
      cp_async_wait1();
    } else {
      cp_async_wait0();
    }
    // each thread reads back only its own column, which it copied itself: no barrier needed
    const int j0 = c * JC;
    const int jn = min(JC, nlines - j0);
    for (int jj = 0; jj < jn; ++jj) {
      const int j = j0 + jj;
      const float* e = Lt + j * LF;
      const float thi = e[0], tlo = e[1], trf = e[2], tinh = e[3], tph = e[4];
      // (Re, Im) pairs in packed f32x2 arithmetic: each lane rounds as the scalar product, sum and
      // fused multiply-add do, so the sums are bitwise the scalar ones in half the issue slots
      float2 H[TY];
      float2 hs = make_float2(0.f, 0.f);
#pragma unroll
      for (int ty = 0; ty < TY; ++ty) H[ty] = make_float2(0.f, 0.f);
      const float2* hb = hbuf + (size_t)(buf * JC + jj) * ncoils * 128 + col;
#pragma unroll 4
      for (int q = 0; q < ncoils; ++q) {
        const float2 h = hb[q * 128];
        const float ex = Ex[q * 128 + col];
        hs = fadd2(hs, h);
        const float2 uu = fmul2(dup2(ex), h);
        const float4 e4 = *reinterpret_cast<const float4*>(Ey + q * ROWS);
        const float ey[4] = {e4.x, e4.y, e4.z, e4.w};
#pragma unroll
        for (int ty = 0; ty < TY; ++ty) H[ty] = ffma2(dup2(ey[ty]), uu, H[ty]);
      }
      const float hsr = hs.x, hsi = hs.y;
      const float4 b4 = *reinterpret_cast<const float4*>(Bt + j * ROWS);
      const float bt[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
      for (int ty = 0; ty < TY; ++ty) {
        const float hr = fmaf(soff, hsr, H[ty].x), hi = fmaf(soff, hsi, H[ty].y);
        const float th = phase_turns(a[ty] + bt[ty], f[ty], thi, tlo);
        float sn, cs;
        __sincosf(kTwoPiF * th, &sn, &cs);
        const float zr = fmaf(cs, hr, sn * hi);  // Z = conj(P) * H
        const float zi = fmaf(cs, hi, -sn * hr);
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) {
          if (cc < ncomp) {
            float r;
            if (MAPS)
              r = __expf(la[ty] - trf * r2[ty][MAPS ? cc : 0] - tinh * r2i[ty][MAPS ? cc : 0]);
            else
              r = e[5 + cc];
            cg[ty][cc].x = fmaf(r, zr, cg[ty][cc].x);
            cg[ty][cc].y = fmaf(r, zi, cg[ty][cc].y);
            if (GRADS) {
              Uy[ty][GRADS ? cc : 0] = fmaf(r * tph, zi, Uy[ty][GRADS ? cc : 0]);
              Vx[ty][GRADS ? cc : 0] = fmaf(r * trf, zr, Vx[ty][GRADS ? cc : 0]);
            }
          }
        }
      }
    }
  }
  if (!active) return;
  const size_t plane = (size_t)snx * sny;
#pragma unroll
  for (int ty = 0; ty < TY; ++ty) {
    const int y = y0 + ty;
    if (y >= sny) break;
    const size_t i = (size_t)x + (size_t)snx * y;
    float fg = 0.f;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      if (c >= ncomp) break;
      u.comp_grad[c * plane + i] = cg[ty][c];
      if (GRADS) {
        const float m = __ldg(u.comp + (size_t)c * u.comp_stride + i);
        fg = fmaf(m, Uy[ty][GRADS ? c : 0], fg);
        if (u.r2_grad) u.r2_grad[c * plane + i] = -2.0f * m * Vx[ty][GRADS ? c : 0];
      }
    }
    if (GRADS && u.fmap_grad) u.fmap_grad[i] = distort ? 4.0f * 3.14159265358979f * fg : 0.f;
  }
}

// ---------------------------------------------------------------------------------------------
// y-adjoint for a compile-time coil count NQ (every unit of the plan has NQ coils, an even snx and
// 16-byte aligned h rows).  Same sums as yadjoint_kernel, reorganised so the per-(line, voxel)
// work is the coil combination and the phase:
//   * a CTA of 256 threads covers 128 columns x 2*TY rows (two groups of TY rows, one column each;
//     TY = 4 with class decay, 2 with voxel maps, whose rates take the registers);
//   * amp_q(x, y) = s * (ex_q(x) ey_q(y) + off) of the thread's TY rows sits in registers, so the
//     coil combination is 2 FMAs per (coil, row) from one shared load of h per coil;
//   * h arrives through a 3-stage ring of JC-line chunks (every coil, 128 columns) filled by
//     cooperative 16-byte cp.async, one barrier per chunk;
//   * the line table carries rel_cj, rel_cj * t_j and rel_cj * trf_j (class decay), so every
//     accumulator update is one FMA.
constexpr int kAdjStages = 3;
__host__ __device__ __forceinline__ constexpr int adjq_chunk_lines(int nq) { return nq >= 16 ? 1 : 16 / nq; }
__host__ __device__ __forceinline__ constexpr int adjq_line_floats(int nc, bool maps) {
  return ((maps ? 5 : 4 + 3 * nc) + 3) / 4 * 4;
}
// rows per thread: 4 with class decay and up to 3 compartments, else 2 (registers)
__host__ __device__ __forceinline__ constexpr int adjq_rows(int nc, bool maps) { return !maps && nc <= 3 ? 4 : 2; }
// ... the same with coil-class rows (two rows per thread in 80 registers and three CTAs per SM
// measured 30 % slower than four rows: the per-line loads then serve half the rows)
__host__ __device__ __forceinline__ constexpr int adjq_rows_v(int nc, bool maps, bool virt) {
  return adjq_rows(nc, maps);
}


// VIRT: the h rows are the NQ = classes + 1 class rows of the class-mode x-adjoint (scale, ex and
// the coil offset already applied), so amp_v(y) = ey_v(y) for the classes and 1 for the offset row.
template <int NQ, int TY, int NC, bool MAPS, bool GRADS, bool VIRT>
__global__ void __launch_bounds__(256, (VIRT && !MAPS && TY == 2) ? 3 : 2) yadjoint_q_kernel(const UnitDesc* __restrict__ units,
                                                            const int4* __restrict__ tiles) {
  extern __shared__ __align__(16) float smem[];
  static_assert(TY == 2 || TY == 4, "the row phases are read as one float2 / float4");
  constexpr int ROWS = 2 * TY;
  constexpr int JC = adjq_chunk_lines(NQ);
  constexpr int LF = adjq_line_floats(NC, MAPS);
  constexpr int STAGE = JC * NQ * 128;        // float2 per stage
  constexpr int PIECES = JC * NQ * 64;        // 16-byte pieces per stage
  constexpr int PPT = (PIECES + 255) / 256;   // pieces per thread
  const int4 tl = tiles[blockIdx.x];          // unit, y0, x0
  const UnitDesc& u = units[tl.x];
  const int snx = u.snx, sny = u.sny, ncomp = u.ncomp, nlines = u.n_lines;
  const int y0 = tl.y, x0 = tl.z;
  float2* hbuf = reinterpret_cast<float2*>(smem);
  float* Bt = reinterpret_cast<float*>(hbuf + kAdjStages * STAGE);  // [nlines][ROWS]
  // the line tables cover whole chunks (zero entries past nlines), so the packed path runs every
  // line of a chunk without a branch
  const int nlp = (nlines + JC - 1) / JC * JC;
  float* Lt = Bt + nlp * ROWS;                                       // [nlp][LF]
  const int tid = threadIdx.x;
  const int col = tid & 127, rg = tid >> 7;
  const int x = x0 + col;
  const bool xok = x < snx;
  const int nchunks = (nlines + JC - 1) / JC;

  // This thread's 16-byte pieces k = tid + 256 i of a chunk: row r = k / 64 = (line jj, coil q),
  // column pair 2 (k % 64); the destination is float2 2k of the stage.  The source offset of
  // each piece for the chunk's first line (or -1 past snx) sits in a per-thread shared table, so
  // a chunk costs one shared load, a compare and a select per piece.  (The plan keeps
  // NQ * lines * snx below 2^31.)
  __shared__ int ptab[PPT * 256];
  const float2* __restrict__ gsrc = u.g;
#pragma unroll
  for (int i = 0; i < PPT; ++i) {
    const int k = tid + 256 * i;
    if (PIECES % 256 == 0 || k < PIECES) {
      const int r = k >> 6, xx = x0 + (k & 63) * 2;
      ptab[i * 256 + tid] = xx < snx ? ((r % NQ) * nlines + r / NQ) * snx + xx : -1;
    }
  }
  auto issue_chunk = [&](int c, int stage) {
    if (c < nchunks) {
      const int rem = nlines - c * JC, jo = c * JC * snx;
      float2* dst = hbuf + stage * STAGE;
#pragma unroll
      for (int i = 0; i < PPT; ++i) {
        const int k = tid + 256 * i;
        if (PIECES % 256 == 0 || k < PIECES) {
          const int o = ptab[i * 256 + tid];
          const bool ok = o >= 0 && ((tid >> 6) + 4 * i) / NQ < rem;
          cp_async16(dst + 2 * k, gsrc + (ok ? o + jo : 0), ok ? 16 : 0);
        }
      }
    }
    cp_async_commit();
  };
#pragma unroll
  for (int c = 0; c < kAdjStages - 1; ++c) issue_chunk(c, c);

  const int ys = u.ny / 2;
  const int oy = sny / u.ny;
  const int sys = oy * ys;
  for (int idx = tid; idx < nlp * ROWS; idx += 256) {
    const int j = idx / ROWS, r = idx % ROWS;
    const int y = y0 + r;
    float v = 0.f;
    if (y < sny && j < nlines) {
      const LineRec& L = u.lines[j];
      const long long K = L.ky - ys;
      const long long Y = 2LL * (y - sys) - (oy - 1);
      const long long m2 = 2LL * sny;
      double tv = (double)((K * Y) % m2) / (double)m2;
      if (u.flags & UF_EDDY) {
        const double yc = ((double)y - sys - (oy - 1) / 2.0) / oy;
        tv += ((double)u.eddy_cy * yc + (double)u.eddy_qy * yc * yc) * (double)L.decay;
      }
      tv -= rint(tv);
      v = (float)tv;
    }
    Bt[idx] = v;
  }
  for (int j = tid; j < nlp; j += 256) {
    float* e = Lt + j * LF;
    if (j >= nlines) {
#pragma unroll
      for (int k = 0; k < LF; ++k) e[k] = 0.f;
      continue;
    }
    const LineRec& L = u.lines[j];
    const float tph = L.t_hi + L.t_lo;
    e[0] = L.t_hi;
    e[1] = L.t_lo;
    e[2] = L.trf_ms;
    e[3] = L.inhom_ms;
    if (MAPS) {
      e[4] = tph;
    } else {
#pragma unroll
      for (int c = 0; c < NC; ++c) {  // zero weights past ncomp: those accumulators stay 0
        const float r = c < ncomp ? L.rel[c] : 0.f;
        e[4 + c] = r;
        e[4 + NC + c] = r * tph;
        e[4 + 2 * NC + c] = r * L.trf_ms;
      }
    }
  }

  // per-thread constants of its 4 rows
  const bool distort = (u.flags & UF_DISTORT) != 0;
  const int xs_ = xok ? x : 0;
  const float s = u.signal_scale, off = u.geo.coil_off;
  float amp[TY][NQ];
  float a[TY], f[TY];
  float r2[TY][MAPS ? NC : 1], r2i[TY][MAPS ? NC : 1], la[TY];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const float ex = VIRT ? 0.f : u.geo.ex[(size_t)q * snx + xs_];
#pragma unroll
    for (int ty = 0; ty < TY; ++ty) {
      const int y = min(y0 + rg * TY + ty, sny - 1);
      if (VIRT)
        amp[ty][q] = q < NQ - 1 ? u.geo.eyc[(size_t)q * sny + y] : 1.f;
      else
        amp[ty][q] = s * fmaf(ex, u.geo.ey[(size_t)q * sny + y], off);
    }
  }
#pragma unroll
  for (int ty = 0; ty < TY; ++ty) {
    const int y = min(y0 + rg * TY + ty, sny - 1);
    const int i = xs_ + snx * y;
    a[ty] = u.phase ? __ldg(u.phase + i) : 0.f;
    f[ty] = distort ? __ldg(u.fmap + i) : 0.f;
    la[ty] = (MAPS && u.log_amp) ? __ldg(u.log_amp + i) : 0.f;
    if (MAPS) {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        r2[ty][MAPS ? c : 0] = r2i[ty][MAPS ? c : 0] = 0.f;
        if (c < ncomp) {
          const float t2 = u.t2map ? __ldg(u.t2map + (size_t)c * u.map_stride + i) : u.t2u[c];
          const float ti = u.timap ? __ldg(u.timap + (size_t)c * u.map_stride + i) : u.tiu[c];
          r2[ty][MAPS ? c : 0] = 1.0f / t2;
          r2i[ty][MAPS ? c : 0] = 1.0f / ti;
        }
      }
    }
  }
  // PK (class rows, class decay, 4 rows): rows (0, 1) and (2, 3) run as packed f32x2 pairs, with
  // accumulators pcx/pcy/puy/pvx[pair][c] holding the two rows' Re/Im comp sums, t- and trf-sums
  constexpr bool PK = VIRT && !MAPS;
  constexpr int NPR = PK ? TY / 2 : 1;  // row pairs
  float2 pcx[NPR][NC], pcy[NPR][NC], puy[NPR][NC], pvx[NPR][NC];
  if (PK) {
#pragma unroll
    for (int pp = 0; pp < NPR; ++pp)
#pragma unroll
      for (int c = 0; c < NC; ++c) pcx[pp][c] = pcy[pp][c] = puy[pp][c] = pvx[pp][c] = make_float2(0.f, 0.f);
  }
  float2 cg[TY][NC];
  float Uy[TY][GRADS ? NC : 1], Vx[TY][GRADS ? NC : 1];
#pragma unroll
  for (int ty = 0; ty < TY; ++ty)
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      cg[ty][c] = make_float2(0.f, 0.f);
      if (GRADS) Uy[ty][GRADS ? c : 0] = Vx[ty][GRADS ? c : 0] = 0.f;
    }

  int s_use = 0, s_issue = kAdjStages - 1;  // stages of chunk c and of chunk c + stages - 1
  for (int c = 0; c < nchunks; ++c) {
    cp_async_wait_n<kAdjStages - 2>();
    __syncthreads();  // chunk c landed for every thread; every thread is done with chunk c - 1
    issue_chunk(c + kAdjStages - 1, s_issue);
    s_issue = s_issue + 1 == kAdjStages ? 0 : s_issue + 1;
    const float2* hs = hbuf + s_use * STAGE + col;
    s_use = s_use + 1 == kAdjStages ? 0 : s_use + 1;
    const int j0 = c * JC;
#pragma unroll
    for (int jj = 0; jj < JC; ++jj) {
      const int j = j0 + jj;
      if (!PK && j >= nlines) break;  // (the packed path reads the zero entries instead)
      const float* e = Lt + j * LF;
      const float4 e0 = *reinterpret_cast<const float4*>(e);
      const float thi = e0.x, tlo = e0.y, trf = e0.z, tinh = e0.w;
      if (PK) {
        float2 Hx[NPR], Hy[NPR];  // [pair] = rows (2p, 2p + 1); starts from the offset row (amplitude 1)
        {
          const float2 h = hs[(jj * NQ + NQ - 1) * 128];
#pragma unroll
          for (int pp = 0; pp < NPR; ++pp) {
            Hx[pp] = dup2(h.x);
            Hy[pp] = dup2(h.y);
          }
        }
#pragma unroll
        for (int q = 0; q < NQ - 1; ++q) {
          const float2 h = hs[(jj * NQ + q) * 128];
          const float2 hx = dup2(h.x), hy = dup2(h.y);
#pragma unroll
          for (int pp = 0; pp < NPR; ++pp) {
            const float2 am = make_float2(amp[2 * pp][q], amp[(2 * pp + 1) % TY][q]);
            Hx[pp] = ffma2(am, hx, Hx[pp]);
            Hy[pp] = ffma2(am, hy, Hy[pp]);
          }
        }
        float2 btp[NPR];
        if (TY == 4) {
          const float4 b4 = *reinterpret_cast<const float4*>(Bt + j * ROWS + rg * TY);
          btp[0] = make_float2(b4.x, b4.y);
          btp[NPR - 1] = make_float2(b4.z, b4.w);
        } else {
          btp[0] = *reinterpret_cast<const float2*>(Bt + j * ROWS + rg * TY);
        }
        const float2 thi2 = dup2(thi), tlo2 = dup2(tlo);
#pragma unroll
        for (int pp = 0; pp < NPR; ++pp) {
          const int t0 = 2 * pp, t1 = (2 * pp + 1) % TY;
          const float2 bt2 = btp[pp];
          float2 th = phase_turns2(fadd2(make_float2(a[t0], a[t1]), bt2), make_float2(f[t0], f[t1]), thi2, tlo2);
          th = fmul2(dup2(kTwoPiF), th);
          float s0, c0, s1, c1;
          __sincosf(th.x, &s0, &c0);
          __sincosf(th.y, &s1, &c1);
          const float2 cs2 = make_float2(c0, c1), sn2 = make_float2(s0, s1);
          const float2 zr = ffma2(cs2, Hx[pp], fmul2(sn2, Hy[pp]));  // Z = conj(P) H per row
          const float2 zi = ffma2(cs2, Hy[pp], fsub2(dup2(0.f), fmul2(sn2, Hx[pp])));
#pragma unroll
          for (int cc = 0; cc < NC; ++cc) {
            const float2 r = dup2(e[4 + cc]);
            pcx[PK ? pp : 0][cc] = ffma2(r, zr, pcx[PK ? pp : 0][cc]);
            pcy[PK ? pp : 0][cc] = ffma2(r, zi, pcy[PK ? pp : 0][cc]);
            if (GRADS) {
              puy[PK ? pp : 0][cc] = ffma2(dup2(e[4 + NC + cc]), zi, puy[PK ? pp : 0][cc]);
              pvx[PK ? pp : 0][cc] = ffma2(dup2(e[4 + 2 * NC + cc]), zr, pvx[PK ? pp : 0][cc]);
            }
          }
        }
        continue;
      }
      float2 H[TY];
      {
        const float2 h = hs[jj * NQ * 128];
#pragma unroll
        for (int ty = 0; ty < TY; ++ty) H[ty] = make_float2(amp[ty][0] * h.x, amp[ty][0] * h.y);
      }
#pragma unroll
      for (int q = 1; q < NQ; ++q) {
        const float2 h = hs[(jj * NQ + q) * 128];
#pragma unroll
        for (int ty = 0; ty < TY; ++ty) {
          H[ty].x = fmaf(amp[ty][q], h.x, H[ty].x);
          H[ty].y = fmaf(amp[ty][q], h.y, H[ty].y);
        }
      }
      float bt[TY];
      if (TY == 4) {
        const float4 b4 = *reinterpret_cast<const float4*>(Bt + j * ROWS + rg * TY);
        bt[0] = b4.x, bt[1] = b4.y, bt[TY > 2 ? 2 : 0] = b4.z, bt[TY > 3 ? 3 : 0] = b4.w;
      } else {
        const float2 b2 = *reinterpret_cast<const float2*>(Bt + j * ROWS + rg * TY);
        bt[0] = b2.x, bt[1] = b2.y;
      }
      const float tph = MAPS ? e[4] : 0.f;
#pragma unroll
      for (int ty = 0; ty < TY; ++ty) {
        const float th = phase_turns(a[ty] + bt[ty], f[ty], thi, tlo);
        float sn, cs;
        __sincosf(kTwoPiF * th, &sn, &cs);
        const float zr = fmaf(cs, H[ty].x, sn * H[ty].y);  // Z = conj(P) * H
        const float zi = fmaf(cs, H[ty].y, -sn * H[ty].x);
#pragma unroll
        for (int cc = 0; cc < NC; ++cc) {
          if (!MAPS || cc < ncomp) {
            float r, rt, rf;
            if (MAPS) {
              r = __expf(la[ty] - trf * r2[ty][MAPS ? cc : 0] - tinh * r2i[ty][MAPS ? cc : 0]);
              rt = r * tph;
              rf = r * trf;
            } else {
              r = e[4 + cc];
              rt = e[4 + NC + cc];
              rf = e[4 + 2 * NC + cc];
            }
            cg[ty][cc].x = fmaf(r, zr, cg[ty][cc].x);
            cg[ty][cc].y = fmaf(r, zi, cg[ty][cc].y);
            if (GRADS) {
              Uy[ty][GRADS ? cc : 0] = fmaf(rt, zi, Uy[ty][GRADS ? cc : 0]);
              Vx[ty][GRADS ? cc : 0] = fmaf(rf, zr, Vx[ty][GRADS ? cc : 0]);
            }
          }
        }
      }
    }
  }
  cp_async_wait0();
  if (!xok) return;
  if (PK) {
#pragma unroll
    for (int ty = 0; ty < TY; ++ty)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const int pp = PK ? (ty >> 1) % NPR : 0;
        const bool hi = ty & 1;
        cg[ty][c] = make_float2(hi ? pcx[pp][c].y : pcx[pp][c].x, hi ? pcy[pp][c].y : pcy[pp][c].x);
        if (GRADS) {
          Uy[ty][GRADS ? c : 0] = hi ? puy[pp][c].y : puy[pp][c].x;
          Vx[ty][GRADS ? c : 0] = hi ? pvx[pp][c].y : pvx[pp][c].x;
        }
      }
  }
  const size_t plane = (size_t)snx * sny;
#pragma unroll
  for (int ty = 0; ty < TY; ++ty) {
    const int y = y0 + rg * TY + ty;
    if (y >= sny) break;
    const size_t i = (size_t)x + (size_t)snx * y;
    float fg = 0.f;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      if (c >= ncomp) break;
      u.comp_grad[c * plane + i] = cg[ty][c];
      if (GRADS) {
        const float m = __ldg(u.comp + (size_t)c * u.comp_stride + i);
        fg = fmaf(m, Uy[ty][GRADS ? c : 0], fg);
        if (u.r2_grad) u.r2_grad[c * plane + i] = -2.0f * m * Vx[ty][GRADS ? c : 0];
      }
    }
    if (GRADS && u.fmap_grad) u.fmap_grad[i] = distort ? 4.0f * 3.14159265358979f * fg : 0.f;
  }
}

// ---------------------------------------------------------------------------------------------
// x-stage as a register-tiled complex GEMM.  A tile is up to 32 rows (lines of ONE readout polarity
// x coils) by 64 output columns; K runs over the contraction in chunks of 32 staged in shared memory.
//   forward : out[q][row_j][kx] = (1/nvox) sum_x  g[q][j][x] E_j(x)        tw_pol[x][kx]
//   adjoint : h[q][j][x]        = (1/nvox) conj(E_j(x)) sum_kx conj(tw_pol[x][kx]) r[q][row_j][kx]
// Each of 256 threads owns 4 rows x 2 columns.
template <bool ADJ>
__global__ void __launch_bounds__(256) xgemm_kernel(const UnitDesc* __restrict__ units,
                                                    const XTile* __restrict__ tiles) {
  __shared__ float2 As[32][33];   // [row][k]
  __shared__ float2 Bs[32][64];   // [k][col]
  __shared__ int lrow[32], lline[32], lq[32];
  __shared__ float ldec[32];
  const XTile& T = tiles[blockIdx.x];
  const UnitDesc& u = units[T.unit];
  const int snx = u.snx, nx = u.nx;
  const int K = ADJ ? nx : snx;       // contraction length
  const int N = ADJ ? snx : nx;       // output columns
  const int nrows = T.nl * T.nq;
  const int ox = snx / nx, sxs = ox * (nx / 2);
  const double xoff = (ox - 1.0) / 2.0;
  const bool eddy = (u.flags & UF_EDDY) != 0;
  if (threadIdx.x < 32) {
    const int r = threadIdx.x;
    if (r < nrows) {
      const int jj = r / T.nq, qq = r % T.nq;
      const LineRec& L = u.lines[T.line[jj]];
      lrow[r] = L.row;
      lline[r] = T.line[jj];
      lq[r] = T.q0 + qq;
      ldec[r] = L.decay;
    } else {
      lrow[r] = 0;
      lline[r] = 0;
      lq[r] = -1;
      ldec[r] = 0.f;
    }
  }
  __syncthreads();
  // the twiddles of this tile's polarity: forward [x][kx], adjoint [kx][x] (transposed table)
  const float2* tw = u.geo.tw + (size_t)(ADJ ? 2 + T.pol : T.pol) * snx * nx;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 8 row groups of 4
  float2 acc[4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i) acc[i][0] = acc[i][1] = make_float2(0.f, 0.f);
  for (int k0 = 0; k0 < K; k0 += 32) {
    // stage A: 32 rows x 32 k
    for (int e = threadIdx.x; e < 32 * 32; e += 256) {
      const int r = e >> 5, kk = e & 31, k = k0 + kk;
      float2 v = make_float2(0.f, 0.f);
      if (lq[r] >= 0 && k < K) {
        if (!ADJ) {
          v = u.g[((size_t)lq[r] * u.n_lines + lline[r]) * snx + k];
          if (eddy) {
            const double xc = ((double)k - sxs - xoff) / ox;
            double tv = ((double)u.eddy_cx * xc + (double)u.eddy_qx * xc * xc + (double)u.eddy_z) * (double)ldec[r];
            tv -= rint(tv);
            float sn, cs;
            __sincosf(kTwoPiF * (float)tv, &sn, &cs);
            v = make_float2(v.x * cs - v.y * sn, v.x * sn + v.y * cs);
          }
        } else {
          v = u.kspace[((size_t)lq[r] * u.n_rows + lrow[r]) * nx + k];
        }
      }
      As[r][kk] = v;
    }
    // stage B: 32 k x 64 columns
    for (int e = threadIdx.x; e < 32 * 64; e += 256) {
      const int kk = e >> 6, c = e & 63, k = k0 + kk, col = T.col0 + c;
      Bs[kk][c] = (k < K && col < N) ? __ldg(tw + (size_t)k * N + col) : make_float2(0.f, 0.f);
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < 32; ++kk) {
      const float2 b0 = Bs[kk][tx], b1 = Bs[kk][tx + 32];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float2 a = As[ty * 4 + i][kk];
        if (!ADJ) {
          acc[i][0].x = fmaf(a.x, b0.x, fmaf(-a.y, b0.y, acc[i][0].x));
          acc[i][0].y = fmaf(a.x, b0.y, fmaf(a.y, b0.x, acc[i][0].y));
          acc[i][1].x = fmaf(a.x, b1.x, fmaf(-a.y, b1.y, acc[i][1].x));
          acc[i][1].y = fmaf(a.x, b1.y, fmaf(a.y, b1.x, acc[i][1].y));
        } else {  // a * conj(b)
          acc[i][0].x = fmaf(a.x, b0.x, fmaf(a.y, b0.y, acc[i][0].x));
          acc[i][0].y = fmaf(a.y, b0.x, fmaf(-a.x, b0.y, acc[i][0].y));
          acc[i][1].x = fmaf(a.x, b1.x, fmaf(a.y, b1.y, acc[i][1].x));
          acc[i][1].y = fmaf(a.y, b1.x, fmaf(-a.x, b1.y, acc[i][1].y));
        }
      }
    }
    __syncthreads();
  }
  const float inv_n = 1.0f / (float)(snx * u.sny);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = ty * 4 + i;
    if (lq[r] < 0) continue;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int col = T.col0 + tx + 32 * h;
      if (col >= N) continue;
      float2 v = make_float2(acc[i][h].x * inv_n, acc[i][h].y * inv_n);
      if (!ADJ) {
        u.kspace[((size_t)lq[r] * u.n_rows + lrow[r]) * nx + col] = v;
      } else {
        if (eddy) {
          const double xc = ((double)col - sxs - xoff) / ox;
          double tv = ((double)u.eddy_cx * xc + (double)u.eddy_qx * xc * xc + (double)u.eddy_z) * (double)ldec[r];
          tv -= rint(tv);
          float sn, cs;
          __sincosf(kTwoPiF * (float)tv, &sn, &cs);
          v = make_float2(v.x * cs + v.y * sn, v.y * cs - v.x * sn);
        }
        u.g[((size_t)lq[r] * u.n_lines + lline[r]) * snx + col] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------------------------
// x-stage as per-row FFTs when snx = N is a power of two.  The twiddle of the line's polarity
// factors as tw[x][kx] = premod(x) e^{i2pi K x/N} post(kx), K = kx - xs, since
// (K + gh)(x - c) = K x + gh (x - c) - K c, so
//   forward : out[q][row_j][kx] = (1/nvox) post(kx) FFT+[ g[q][j][x] E_j(x) premod(x) ](K mod N)
//   adjoint : h[q][j][x]        = (1/nvox) conj(E_j(x) premod(x)) FFT-[ r[q][row_j][kx] conj(post(kx)) at K mod N ](x)
// (FFT+- : sum e^{+-i2pi k x/N}).  A CTA of 256 threads transforms up to 2048/N rows of one unit
// ([coil][line] order) in shared memory: radix-2 decimation in time from bit-reversed loads.
// Tile = (unit, first row, rows).
template <bool ADJ>
__global__ void __launch_bounds__(256) xfft_kernel(const UnitDesc* __restrict__ units, const int4* __restrict__ tiles) {
  __shared__ __align__(16) float2 buf[kXfftMaxN];
  __shared__ __align__(16) float2 tws[kXfftMaxN / 2];
  __shared__ int rq[256], rline[256], rrow[256], rpol[256];
  __shared__ float rdec[256];
  const int4 t = tiles[blockIdx.x];
  const UnitDesc& u = units[t.x];
  const int r0 = t.y, nr = t.z;
  const int N = u.snx, nx = u.nx, nl = u.n_lines;
  const int logn = 31 - __clz(N), half = N >> 1;
  const int tid = threadIdx.x;
  const float2* __restrict__ xf = u.geo.xf;
  const float2* __restrict__ premod = xf + half;
  const float2* __restrict__ post = xf + half + 2 * N;
  for (int k = tid; k < half; k += 256) tws[k] = xf[k];
  for (int r = tid; r < nr; r += 256) {
    const int R = r0 + r, q = R / nl, j = R % nl;
    const LineRec& L = u.lines[j];
    rq[r] = q;
    rline[r] = j;
    rrow[r] = L.row;
    rpol[r] = L.pol < 0 ? 1 : 0;
    rdec[r] = L.decay;
  }
  __syncthreads();
  const int ox = N / nx, xs = nx / 2, sxs = ox * xs;
  const double xoff = (ox - 1.0) / 2.0;
  const bool eddy = (u.flags & UF_EDDY) != 0;
  // E_j(x) = e^{i2pi (cx xc + qx xc^2 + z) decay_j}: the x and z parts of the eddy polynomial
  auto eddy_factor = [&](int x, float dec) {
    const double xc = ((double)x - sxs - xoff) / ox;
    double tv = ((double)u.eddy_cx * xc + (double)u.eddy_qx * xc * xc + (double)u.eddy_z) * (double)dec;
    tv -= rint(tv);
    float sn, cs;
    __sincosf(kTwoPiF * (float)tv, &sn, &cs);
    return make_float2(cs, sn);
  };
  const float inv_n = 1.0f / (float)(N * u.sny);
  const int kpos = nx - xs;  // K in [-xs, kpos)
  if (!ADJ) {
    for (int e = tid; e < nr * N; e += 256) {
      const int r = e >> logn, x = e & (N - 1);
      const float2 v = u.g[(size_t)(r0 + r) * N + x];
      float2 m = premod[rpol[r] * N + x];
      if (eddy) m = cmul(m, eddy_factor(x, rdec[r]));
      buf[(r << logn) + (__brev(x) >> (32 - logn))] = cmul(v, m);
    }
  } else {
    for (int e = tid; e < nr * N; e += 256) {
      const int r = e >> logn, k = e & (N - 1);
      const int K = k < kpos ? k : k - N;
      const int kx = K + xs;
      float2 v = make_float2(0.f, 0.f);
      if (kx >= 0 && kx < nx) {
        const float2 p = post[kx];
        v = cmul(u.kspace[((size_t)rq[r] * u.n_rows + rrow[r]) * nx + kx], make_float2(p.x, -p.y));
      }
      buf[(r << logn) + (__brev(k) >> (32 - logn))] = v;
    }
  }
  __syncthreads();
  for (int s = 1; s <= logn; ++s) {
    const int h = 1 << (s - 1);
    for (int b = tid; b < nr * half; b += 256) {
      const int r = b >> (logn - 1), bb = b & (half - 1);
      const int pos = bb & (h - 1), grp = bb >> (s - 1);
      const int i0 = (r << logn) + (grp << s) + pos, i1 = i0 + h;
      float2 w = tws[pos << (logn - s)];  // e^{-i2pi pos / 2h}
      if (!ADJ) w.y = -w.y;
      const float2 a = buf[i0], bw = cmul(buf[i1], w);
      buf[i0] = make_float2(a.x + bw.x, a.y + bw.y);
      buf[i1] = make_float2(a.x - bw.x, a.y - bw.y);
    }
    __syncthreads();
  }
  if (!ADJ) {
    for (int e = tid; e < nr * nx; e += 256) {
      const int r = e / nx, kx = e % nx;
      const int k = (kx - xs) & (N - 1);
      const float2 v = cmul(buf[(r << logn) + k], post[kx]);
      u.kspace[((size_t)rq[r] * u.n_rows + rrow[r]) * nx + kx] = make_float2(v.x * inv_n, v.y * inv_n);
    }
  } else {
    for (int e = tid; e < nr * N; e += 256) {
      const int r = e >> logn, x = e & (N - 1);
      float2 m = premod[rpol[r] * N + x];
      if (eddy) m = cmul(m, eddy_factor(x, rdec[r]));
      const float2 v = cmul(buf[e], make_float2(m.x, -m.y));
      u.g[(size_t)(r0 + r) * N + x] = make_float2(v.x * inv_n, v.y * inv_n);
    }
  }
}

// The same x-stage with one warp per row for N = 32 E (E = 1..8, any E), no block barriers: lane t
// holds x[t + 32 m] (m < E).  With n = t + 32 m and k = k1 + E k2, W = e^{+-i2pi/N}:
//   X[k1 + E k2] = sum_t W^{t k1} [ sum_m x[t + 32 m] W^{32 m k1} ] W^{E t k2}
// so each lane does an E-point DFT of its registers (radix-2, unrolled), the twiddles W^{t k1},
// and the 32-point DFTs over t run as five radix-2 decimation-in-frequency stages of lane
// shuffles, which leave X[k1 + E k2] in lane bitrev5(k2).  A per-warp shared row (padded one
// slot in 32) puts the results back in natural order for coalesced stores.
__host__ __device__ constexpr int bitrev_c(int v, int bits) {
  int r = 0;
  for (int b = 0; b < bits; ++b) r |= ((v >> b) & 1) << (bits - 1 - b);
  return r;
}
__host__ __device__ constexpr int log2_c(int v) { return v <= 1 ? 0 : 1 + log2_c(v / 2); }

// CLS (8 coils in 5 classes + offset): a tile is (unit, first line, up to 4 lines) x all 8 coils.
// Adjoint: warp w transforms coil w of each line into shared memory, and the CTA then writes the
// 6 class rows G_v = s sum_{q in v} ex_q h_q, G_off = s off sum_q h_q ([v][line][x] in g) that
// the class-mode y-adjoint combines as sum_v ey_v(y) G_v + G_off.  Forward: the CTA stages the
// tile's class rows from the class-mode y-stage and each row loads g_q = ex_q G_cls(q) + G_off.
template <int E, bool ADJ, bool CLS>
__global__ void __launch_bounds__(256, E <= 4 ? 4 : 2) xfft_warp_kernel(const UnitDesc* __restrict__ units,
                                                           const int4* __restrict__ tiles) {
  constexpr int N = 32 * E, LE = log2_c(E);
  constexpr bool P2 = (E & (E - 1)) == 0;  // E a power of two: radix-2 register DFT, else direct
  constexpr int NP = N + N / 32;  // padded row
  constexpr int RT = 32;          // rows per tile
  static_assert(!CLS || E <= 4, "coil classes: rows of at most 128 points");
  __shared__ __align__(16) float2 hsm[CLS ? 4 * 8 * N : 1];  // [line][coil][x]
  __shared__ int cls_s[8];
  __shared__ __align__(16) float2 tw[N];        // e^{-i2pi j/N}
  __shared__ __align__(16) float2 pm[2 * N];    // premodulation per polarity
  __shared__ __align__(16) float2 pt[N];        // post-twiddle per kx (nx <= N)
  __shared__ __align__(16) float2 rb[8][NP];
  __shared__ int rq[RT], rrow[RT], rpol[RT];
  __shared__ float rdec[RT];
  const int4 t = tiles[blockIdx.x];
  const UnitDesc& u = units[t.x];
  const int r0 = t.y, nr = CLS ? 8 * t.z : t.z;  // CLS: first line, lines
  const int nx = u.nx, nl = u.n_lines, n_rows = u.n_rows;
  // the unit's buffers, read once: the row loop's warp barriers order memory, so the fields would
  // otherwise be loaded again for every row
  float2* const ksp = u.kspace;
  float2* const gbuf = u.g;
  // forward: the 8 coils' ex rows ([q][x]) after the class rows of at most 4 lines (24 N float2)
  float* exs = CLS ? reinterpret_cast<float*>(hsm + 24 * N) : nullptr;
  if (CLS && !ADJ) {  // the tile's class rows, [line][v][x], as 16-byte asynchronous copies issued
                      // first, so that their latency overlaps the table setup (N is even and the
                      // rows of g start on 16-byte boundaries); then the ex rows
    constexpr int HN = N / 2;
    const float4* g4 = reinterpret_cast<const float4*>(gbuf);
    float4* h4 = reinterpret_cast<float4*>(hsm);
    for (int e = threadIdx.x; e < (nr >> 3) * 6 * HN; e += 256) {
      const int jl = e / (6 * HN), v = (e / HN) % 6, x2 = e % HN;
      cp_async16(h4 + e, g4 + ((size_t)v * nl + r0 + jl) * HN + x2, 16);
    }
    cp_async_commit();
    for (int e = threadIdx.x; e < 8 * N; e += 256) exs[e] = u.geo.ex[e];
  }
  const float2* __restrict__ xf = u.geo.xf;
  for (int k = threadIdx.x; k < N / 2; k += 256) {
    const float2 w = xf[k];
    tw[k] = w;
    tw[k + N / 2] = make_float2(-w.x, -w.y);
  }
  // the output side's table carries the 1/(N sny) scale: the post-twiddle in the forward, the
  // premodulation in the adjoint
  const float inv_n = 1.0f / (float)(N * u.sny);
  for (int k = threadIdx.x; k < 2 * N; k += 256) {
    const float2 v = xf[N / 2 + k];
    pm[k] = ADJ ? make_float2(v.x * inv_n, v.y * inv_n) : v;
  }
  for (int k = threadIdx.x; k < nx; k += 256) {
    const float2 v = xf[N / 2 + 2 * N + k];
    pt[k] = ADJ ? v : make_float2(v.x * inv_n, v.y * inv_n);
  }
  if (CLS && threadIdx.x < 8) cls_s[threadIdx.x] = u.geo.cls[threadIdx.x];
  for (int r = threadIdx.x; r < nr; r += 256) {
    const int R = CLS ? (r & 7) * nl + r0 + (r >> 3) : r0 + r;  // CLS: row r = (line r / 8, coil r % 8)
    const LineRec& L = u.lines[R % nl];
    rq[r] = R / nl;
    rrow[r] = L.row;
    rpol[r] = L.pol < 0 ? 1 : 0;
    rdec[r] = L.decay;
  }
  if (CLS && !ADJ) cp_async_wait0();
  __syncthreads();
  // W(j) = e^{sigma i2pi j/N}: sigma = +1 forward, -1 adjoint
  auto W = [&](int j) {
    const float2 w = tw[j];
    return ADJ ? w : make_float2(w.x, -w.y);
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ox = N / nx, xs = nx / 2, sxs = ox * xs;
  const double xoff = (ox - 1.0) / 2.0;
  const bool eddy = (u.flags & UF_EDDY) != 0;
  const int kpos = nx - xs;
  float2* row = rb[warp];
  // premodulation of the line's polarity times E_j(x) = e^{i2pi (cx xc + qx xc^2 + z) decay_j}
  auto modulation = [&](int pol, float dec, int x) {
    float2 md = pm[pol * N + x];
    if (eddy) {
      const double xc = ((double)x - sxs - xoff) / ox;
      double tv = ((double)u.eddy_cx * xc + (double)u.eddy_qx * xc * xc + (double)u.eddy_z) * (double)dec;
      tv -= rint(tv);
      float sn, cs;
      __sincosf(kTwoPiF * (float)tv, &sn, &cs);
      md = cmul(md, make_float2(cs, sn));
    }
    return md;
  };
  // adjoint: the k-space samples of the warp's next row are loaded while the current row transforms
  // (zero outside the acquired kx)
  float2 pre[ADJ ? E : 1];
  auto fetch = [&](int r) {
    const float2* kr = ksp + ((size_t)rq[r] * n_rows + rrow[r]) * nx;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int n = lane + 32 * m;
      const int kx = (n < kpos ? n : n - N) + xs;
      pre[ADJ ? m : 0] = kx >= 0 && kx < nx ? kr[kx] : make_float2(0.f, 0.f);
    }
  };
  if (ADJ && warp < nr) fetch(warp);
  for (int r = warp; r < nr; r += 8) {
    const int R = CLS ? (r & 7) * nl + r0 + (r >> 3) : r0 + r, q = rq[r], orow = rrow[r], pol = rpol[r];
    const float dec = rdec[r];
    float2 b[E];
    if (!ADJ && CLS) {
      const int jl = r >> 3, c = cls_s[q];
      const float2* cr = hsm + (jl * 6) * N;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int x = lane + 32 * m;
        const float ex = exs[q * N + x];
        const float2 gv = cr[c * N + x], go = cr[5 * N + x];
        b[P2 ? bitrev_c(m, LE) : m] = cmul(make_float2(fmaf(ex, gv.x, go.x), fmaf(ex, gv.y, go.y)), modulation(pol, dec, x));
      }
    } else if (!ADJ) {
      const float2* gr = gbuf + (size_t)R * N;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int x = lane + 32 * m;
        b[P2 ? bitrev_c(m, LE) : m] = cmul(gr[x], modulation(pol, dec, x));
      }
    } else {
      float2 cur[E];
#pragma unroll
      for (int m = 0; m < E; ++m) cur[m] = pre[ADJ ? m : 0];
      if (r + 8 < nr) fetch(r + 8);
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int n = lane + 32 * m;
        const int kx = (n < kpos ? n : n - N) + xs;
        float2 v = make_float2(0.f, 0.f);
        if (kx >= 0 && kx < nx) {
          const float2 p = pt[kx];
          v = cmul(cur[m], make_float2(p.x, -p.y));
        }
        b[P2 ? bitrev_c(m, LE) : m] = v;
      }
    }
    // E-point DFT of the registers: decimation in time from bit-reversed order, or for E not a
    // power of two the direct sum Y[k1] = sum_m b[m] W^{32 (m k1 mod E)}
    if (!P2) {
      float2 y[E];
#pragma unroll
      for (int k1 = 0; k1 < E; ++k1) {
        y[k1] = b[0];
#pragma unroll
        for (int m = 1; m < E; ++m) {
          const float2 v = (m * k1) % E == 0 ? b[m] : cmul(b[m], W(32 * ((m * k1) % E)));
          y[k1] = make_float2(y[k1].x + v.x, y[k1].y + v.y);
        }
      }
#pragma unroll
      for (int k1 = 0; k1 < E; ++k1) b[k1] = y[k1];
    }
#pragma unroll
    for (int len = 2; len <= (P2 ? E : 1); len <<= 1) {
#pragma unroll
      for (int i = 0; i < E; i += len) {
#pragma unroll
        for (int p = 0; p < len / 2; ++p) {
          float2 v = b[i + p + len / 2];
          const int j = p * (E / len) * 32;
          if (4 * j == N)  // W(N/4) = sigma i exactly
            v = ADJ ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
          else if (p != 0)
            v = cmul(v, W(j));
          const float2 a = b[i + p];
          b[i + p] = make_float2(a.x + v.x, a.y + v.y);
          b[i + p + len / 2] = make_float2(a.x - v.x, a.y - v.y);
        }
      }
    }
#pragma unroll
    for (int k1 = 1; k1 < E; ++k1) b[k1] = cmul(b[k1], W(lane * k1));
    // 32-point DFTs across the lanes: radix-2 decimation in frequency.  The last two stages'
    // twiddles are exact: 1 at h = 1, and 1 or W(N/4) = sigma i (a swap and a sign) at h = 2.
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) {
      const bool up = (lane & h) != 0;
      const float sg = up ? -1.f : 1.f;
      const float2 w = h >= 4 && up ? W((lane & (h - 1)) * (N / (2 * h))) : make_float2(1.f, 0.f);
      const bool quarter = h == 2 && up && (lane & 1);
#pragma unroll
      for (int k1 = 0; k1 < E; ++k1) {
        const float ox_ = __shfl_xor_sync(0xffffffffu, b[k1].x, h);
        const float oy_ = __shfl_xor_sync(0xffffffffu, b[k1].y, h);
        const float2 v = make_float2(fmaf(sg, b[k1].x, ox_), fmaf(sg, b[k1].y, oy_));
        if (h >= 4)
          b[k1] = cmul(v, w);
        else if (h == 2)  // times sigma i: -i for the adjoint (e^{-i pi/2}), +i for the forward
          b[k1] = quarter ? (ADJ ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x)) : v;
        else
          b[k1] = v;
      }
    }
    const int k2 = __brev(lane) >> 27;
#pragma unroll
    for (int k1 = 0; k1 < E; ++k1) {
      const int k = k1 + E * k2;
      row[k + (k >> 5)] = b[k1];
    }
    __syncwarp();
    if (!ADJ) {
      float2* out = ksp + ((size_t)q * n_rows + orow) * nx;
      for (int kx = lane; kx < nx; kx += 32) {
        const int k = ((kx - xs) % N + N) % N;
        out[kx] = cmul(row[k + (k >> 5)], pt[kx]);
      }
    } else {
      float2* gr = CLS ? hsm + ((r >> 3) * 8 + (r & 7)) * N : gbuf + (size_t)R * N;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int x = lane + 32 * m;
        const float2 md = modulation(pol, dec, x);
        gr[x] = cmul(row[x + (x >> 5)], make_float2(md.x, -md.y));
      }
    }
    __syncwarp();
  }
  if (CLS && ADJ) {
    __syncthreads();
    const float s = u.signal_scale, so = s * u.geo.coil_off;
    float* sex = reinterpret_cast<float*>(&rb[0][0]);  // s ex_q(x), [q][x], in the free reorder rows
    for (int e = threadIdx.x; e < 8 * N; e += 256) sex[e] = s * u.geo.ex[e];
    __syncthreads();
    const int nj = nr >> 3;
    for (int e = threadIdx.x; e < nj * N; e += 256) {
      const int jl = e / N, x = e % N;
      float2 G[6];
#pragma unroll
      for (int v = 0; v < 6; ++v) G[v] = make_float2(0.f, 0.f);
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float2 h = hsm[(jl * 8 + q) * N + x];
        const float ex = sex[q * N + x];
        const int c = cls_s[q];
#pragma unroll
        for (int v = 0; v < 5; ++v)
          if (c == v) {
            G[v].x = fmaf(ex, h.x, G[v].x);
            G[v].y = fmaf(ex, h.y, G[v].y);
          }
        G[5].x += h.x;
        G[5].y += h.y;
      }
      G[5] = make_float2(so * G[5].x, so * G[5].y);
#pragma unroll
      for (int v = 0; v < 6; ++v) gbuf[((size_t)v * nl + r0 + jl) * N + x] = G[v];
    }
  }
}

template <class K>
void set_smem(K kernel, size_t bytes) {
  // past 48 KB of static + dynamic shared memory the launch needs the dynamic opt-in
  cudaFuncAttributes fa;
  MRSIM_CUDA(cudaFuncGetAttributes(&fa, kernel));
  if (bytes + fa.sharedSizeBytes > 48 * 1024)
    MRSIM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

}  // namespace

// ---- plans and launchers ----------------------------------------------------------------------
void append_xtiles(std::vector<XTile>& out, const UnitDesc& u, int unit_index, const LineRec* lines, int dir) {
  const int nl = u.n_lines, nc = u.ncoils;
  const int N = dir == 0 ? u.nx : u.snx;
  const int nq = std::min(nc, 32);
  const int lines_per_tile = std::max(1, 32 / nq);
  for (int pol = 0; pol < 2; ++pol) {
    std::vector<int> group;
    for (int l = 0; l < nl; ++l)
      if ((lines[l].pol < 0 ? 1 : 0) == pol) group.push_back(l);
    for (size_t g0 = 0; g0 < group.size(); g0 += lines_per_tile)
      for (int q0 = 0; q0 < nc; q0 += nq)
        for (int c0 = 0; c0 < N; c0 += 64) {
          XTile t;
          std::memset(&t, 0, sizeof t);
          t.unit = unit_index;
          t.q0 = q0;
          t.nq = std::min(nq, nc - q0);
          t.nl = (int)std::min<size_t>(lines_per_tile, group.size() - g0);
          t.col0 = c0;
          t.pol = pol;
          for (int k = 0; k < t.nl; ++k) t.line[k] = group[g0 + k];
          out.push_back(t);
        }
  }
}

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

EpiPlan* epi_plan_create(const UnitDesc* hu, int n, const StaticDesc* hs, int ns, const EpiPlanOptions* opt) {
  EpiPlan* p = new EpiPlan();
  try {
    if (opt) p->opt = *opt;
    p->n_units = n;
    p->host_units.assign(hu, hu + n);
    p->host_statics.assign(hs, hs + ns);
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
    for (int i = 0; i < n; ++i)
      p->max_hchunk = std::max(p->max_hchunk, adjoint_chunk_lines(hu[i].ncoils) * hu[i].ncoils);
    int max_comp = 0;
    for (int i = 0; i < n; ++i) max_comp = std::max(max_comp, hu[i].ncomp);
    p->nc = max_comp <= 1 ? 1 : max_comp <= 2 ? 2 : max_comp <= 3 ? 3 : max_comp <= 4 ? 4 : 8;
    p->qg = max_coils <= 1 ? 1 : max_coils <= 2 ? 2 : max_coils <= 4 ? 4 : 8;
    // the staged-input forward serves a pass when every unit has snx % 4 == 0 and 16-byte aligned
    // input planes (cooperative 16-byte copies)
    auto al16 = [](const void* q) { return ((uintptr_t)q & 15) == 0; };
    for (int pass = 0; pass < 2; ++pass) {
      bool ok = true;
      for (int i = 0; i < n; ++i) {
        const UnitDesc& u = hu[i];
        if (((u.flags & UF_MAPS) != 0) != (pass == 1)) continue;
        ok = ok && (u.snx % 4) == 0 && al16(u.phase) && al16(u.fmap) && al16(u.comp) && al16(u.t2map) &&
             al16(u.timap) && al16(u.log_amp) && (u.ncomp <= 1 || u.comp_stride % 4 == 0) &&
             (u.ncomp <= 1 || (u.map_stride % 4) == 0);
      }
      // eight coils with voxel maps (four or more compartments) or eight compartments take more
      // registers than the 256-thread CTA leaves: those shapes keep the per-thread-load kernel
      if (p->qg == 8 && (p->nc == 8 || (pass == 1 && p->nc >= 4))) ok = false;
      p->fwdq[pass] = ok;
      // coil classes: every unit with the same 8 coils in 5 classes (the ring) -> 6 accumulators
      bool cl = ok && n > 0 && p->qg == 8 && (pass == 0 || p->nc <= 3);
      for (int i = 0; i < n && cl; ++i) {
        const UnitDesc& u = hu[i];
        if (((u.flags & UF_MAPS) != 0) != (pass == 1)) continue;
        cl = u.ncoils == 8 && u.geo.ncls == 5 && u.geo.coil_off != 0.f && u.geo.cls && u.geo.eyc;
      }
      p->fwd_nv[pass] = (cl && !p->opt.no_classes) ? 6 : 0;
    }
    for (int pass = 0; pass < 2; ++pass) {
      std::vector<int4> tiles;
      const int step = p->fwdq[pass] ? 8 : kT;
      p->y_start[pass].assign(n + 1, 0);
      for (int i = 0; i < n; ++i) {
        p->y_start[pass][i] = (int)tiles.size();
        if (((hu[i].flags & UF_MAPS) != 0) != (pass == 1)) continue;
        for (int l = 0; l < hu[i].n_lines; l += step)
          for (int x0 = 0; x0 < hu[i].snx; x0 += 128)
            for (int q0 = 0; q0 < hu[i].ncoils; q0 += p->qg) tiles.push_back(make_int4(i, l, x0, q0));
      }
      p->y_start[pass][n] = (int)tiles.size();
      p->n_ytiles[pass] = (int)tiles.size();
      p->d_ytiles[pass] = (int4*)dev_upload(p, tiles.data(), sizeof(int4) * tiles.size());
    }
    // x-stage as per-row FFTs when every unit has a power-of-two snx with FFT tables
    p->xfft = n > 0 && !p->opt.dft_x;
    for (int i = 0; i < n; ++i) {
      const int N = hu[i].snx;
      const bool pow2 = N >= 8 && N <= kXfftMaxN && (N & (N - 1)) == 0, warp = N % 32 == 0 && N <= 256;
      if (hu[i].geo.xf == nullptr || !(pow2 || warp) || hu[i].nx > N) p->xfft = false;
    }
    if (p->xfft) {
      const int N0 = hu[0].snx;
      p->xfft_e = (N0 % 32 == 0 && N0 <= 256) ? N0 / 32 : 0;
      bool all_warp = true;
      for (int i = 0; i < n; ++i) {
        if (hu[i].snx != N0) p->xfft_e = 0;
        all_warp = all_warp && hu[i].snx % 32 == 0 && hu[i].snx <= 256;
      }
      // every row a warp width but not one width (a batch of 128, 192 and 256): the warp FFT once
      // per width over that width's tiles
      if (p->xfft_e == 0 && all_warp) p->xfft_e = -1;
      // otherwise the shared-memory radix-2 FFT serves, which needs every row length to be a power
      // of two; failing that, the DFT GEMM
      if (p->xfft_e == 0)
        for (int i = 0; i < n; ++i) {
          const int N = hu[i].snx;
          if (!(N >= 8 && N <= kXfftMaxN && (N & (N - 1)) == 0)) p->xfft = false;
        }
    }
    if (p->xfft && p->xfft_e < 0) {
      // one list ordered by width, no per-unit ranges (such a plan runs whole)
      std::vector<int4> ft;
      for (int E = 1; E <= 8; ++E) {
        p->fe_first[E] = (int)ft.size();
        for (int i = 0; i < n; ++i) {
          if (hu[i].snx != 32 * E) continue;
          const int rows = hu[i].ncoils * hu[i].n_lines;
          for (int r0 = 0; r0 < rows; r0 += 32) ft.push_back(make_int4(i, r0, std::min(32, rows - r0), 0));
        }
        p->fe_count[E] = (int)ft.size() - p->fe_first[E];
      }
      p->f_start.clear();
      p->n_ftiles = (int)ft.size();
      p->d_ftiles = (int4*)dev_upload(p, ft.data(), sizeof(int4) * ft.size());
    } else if (p->xfft) {
      std::vector<int4> ft;
      p->f_start.assign(n + 1, 0);
      for (int i = 0; i < n; ++i) {
        p->f_start[i] = (int)ft.size();
        const int rows = hu[i].ncoils * hu[i].n_lines;
        const int per = p->xfft_e ? 32 : std::min(256, kXfftMaxN / hu[i].snx);
        for (int r0 = 0; r0 < rows; r0 += per) ft.push_back(make_int4(i, r0, std::min(per, rows - r0), 0));
      }
      p->f_start[n] = (int)ft.size();
      p->n_ftiles = (int)ft.size();
      p->d_ftiles = (int4*)dev_upload(p, ft.data(), sizeof(int4) * ft.size());
    }
    // coil classes through the forward x-stage: every unit's y-stage runs in class mode and the
    // rows have at most 128 points
    {
      bool fc = p->xfft && p->xfft_e >= 1 && p->xfft_e <= 4 && n > 0;
      for (int pass = 0; pass < 2 && fc; ++pass) {
        bool any = false;
        for (int i = 0; i < n && !any; ++i) any = ((hu[i].flags & UF_MAPS) != 0) == (pass == 1);
        if (any && p->fwd_nv[pass] != 6) fc = false;
      }
      p->fwd_cls = fc;
    }
    // x-stage GEMM tiles, from host copies of the line tables (one copy per distinct table)
    std::map<const LineRec*, std::vector<LineRec>> host_lines;
    for (int dir = 0; dir < 2 && !p->xfft; ++dir) {
      std::vector<XTile> xt;
      p->g_start[dir].assign(n + 1, 0);
      for (int i = 0; i < n; ++i) {
        p->g_start[dir][i] = (int)xt.size();
        const int nl = hu[i].n_lines;
        if (nl == 0) continue;
        auto it = host_lines.find(hu[i].lines);
        if (it == host_lines.end()) {
          std::vector<LineRec> L(nl);
          MRSIM_CUDA(cudaMemcpy(L.data(), hu[i].lines, sizeof(LineRec) * nl, cudaMemcpyDeviceToHost));
          it = host_lines.emplace(hu[i].lines, std::move(L)).first;
        }
        append_xtiles(xt, hu[i], i, it->second.data(), dir);
      }
      p->g_start[dir][n] = (int)xt.size();
      p->n_gtiles[dir] = (int)xt.size();
      p->d_gtiles[dir] = dev_upload(p, xt.data(), sizeof(XTile) * xt.size());
    }
    // the fixed-coil-count y-adjoint serves a pass when every unit has the same coil count (1, 2,
    // 4 or 8), an even snx and 16-byte aligned h rows (cooperative 16-byte copies)
    int nq_all = n > 0 ? hu[0].ncoils : 0;
    for (int i = 0; i < n; ++i)
      if (hu[i].ncoils != nq_all || (hu[i].snx & 1) || ((uintptr_t)hu[i].g & 15) ||
          (long long)hu[i].ncoils * hu[i].n_lines * hu[i].snx >= (1LL << 31))
        nq_all = 0;
    if (nq_all != 1 && nq_all != 2 && nq_all != 4 && nq_all != 8) nq_all = 0;
    // coil classes in the adjoint: every unit has the 8-coil ring (5 classes + offset), rows of
    // at most 128 points in the warp FFT, and the fixed-count y-adjoint for its shape
    {
      bool cl = n > 0 && p->xfft && p->xfft_e >= 1 && p->xfft_e <= 4 && p->nc <= 4 && nq_all == 8;
      for (int i = 0; i < n && cl; ++i) {
        const UnitDesc& u = hu[i];
        cl = u.ncoils == 8 && u.geo.ncls == 5 && u.geo.coil_off != 0.f && u.geo.cls && u.geo.eyc;
      }
      p->adj_cls = cl && !p->opt.no_classes;
    }
    for (int pass = 0; pass < 4; ++pass) {
      bool maps = pass & 1, grads = pass & 2;
      p->adjq[pass] = p->adj_cls ? 6 : (maps && p->nc == 8) ? 0 : nq_all;
      // rows per thread: the built-in choice, or 2 where 4 would be (the tunable)
      int ty = adjq_rows_v(p->nc, maps, p->adj_cls);
      if (p->opt.adj_rows == 2 && ty == 4) ty = 2;
      p->adj_ty[pass] = ty;
      const int step = p->adjq[pass] ? 2 * ty : kTY;
      std::vector<int4> yt;
      p->a_start[pass].assign(n + 1, 0);
      for (int i = 0; i < n; ++i) {
        p->a_start[pass][i] = (int)yt.size();
        bool um = (hu[i].flags & UF_MAPS) != 0;
        bool ug = (hu[i].flags & (UF_WANT_FMAP_GRAD | UF_WANT_R2_GRAD)) != 0;
        if (um != maps || ug != grads) continue;
        for (int y0 = 0; y0 < hu[i].sny; y0 += step)
          for (int x0 = 0; x0 < hu[i].snx; x0 += 128) yt.push_back(make_int4(i, y0, x0, 0));
      }
      p->a_start[pass][n] = (int)yt.size();
      p->n_atiles[pass] = (int)yt.size();
      p->d_atiles[pass] = (int4*)dev_upload(p, yt.data(), sizeof(int4) * yt.size());
    }
    if (p->adj_cls || p->fwd_cls) {  // the class x-stage tiles: 4 lines x the 8 coils
      std::vector<int4> ct;
      p->c_start.assign(n + 1, 0);
      for (int i = 0; i < n; ++i) {
        p->c_start[i] = (int)ct.size();
        for (int j0 = 0; j0 < hu[i].n_lines; j0 += 4) ct.push_back(make_int4(i, j0, std::min(4, hu[i].n_lines - j0), 0));
      }
      p->c_start[n] = (int)ct.size();
      p->n_ctiles = (int)ct.size();
      p->d_ctiles = (int4*)dev_upload(p, ct.data(), sizeof(int4) * ct.size());
    }
  } catch (...) {
    delete p;
    throw;
  }
  return p;
}

namespace {
// The tiles of units [u0, u1) in a list with per-unit starts `start` (empty: the whole list).
struct TileRange {
  int t0, n;
};
TileRange tile_range(const std::vector<int>& start, int n_tiles, int u0, int u1) {
  if (start.empty() || (u0 == 0 && (u1 < 0 || u1 == (int)start.size() - 1))) return {0, n_tiles};
  if (u1 < 0) u1 = (int)start.size() - 1;
  if (u0 < 0 || u0 > u1 || u1 >= (int)start.size()) fail("unit range outside the plan");
  return {start[u0], start[u1] - start[u0]};
}
}  // namespace

void epi_plan_statics(const EpiPlan* p, cudaStream_t st, int u0, int u1) {
  if (u1 < 0) u1 = p->n_statics;
  if (u0 < 0 || u0 > u1 || u1 > p->n_statics) fail("unit range outside the plan");
  if (u1 == u0) return;
  dim3 grid(std::min(8, (p->max_static_n + 255) / 256), u1 - u0);  // a few voxels per thread
  statics_kernel<<<grid, 256, 0, st>>>(p->d_statics + u0);
  MRSIM_CUDA(cudaGetLastError());
}

void epi_plan_forward(const EpiPlan* p, cudaStream_t st, int u0, int u1) {
  epi_plan_forward_ystage(p, st, u0, u1);
  epi_plan_forward_xstage(p, st, u0, u1);
}

void epi_plan_adjoint(const EpiPlan* p, cudaStream_t st, int u0, int u1) {
  epi_plan_adjoint_xstage(p, st, u0, u1);
  epi_plan_adjoint_ystage(p, st, u0, u1);
}

void epi_plan_forward_ystage(const EpiPlan* p, cudaStream_t st, int u0, int u1) {
  for (int pass = 0; pass < 2; ++pass) {
    const TileRange R = tile_range(p->y_start[pass], p->n_ytiles[pass], u0, u1);
    if (R.n == 0) continue;
    const Tile* tiles = (const Tile*)p->d_ytiles[pass] + R.t0;
    const bool maps = pass == 1;
    const int QG = p->qg, NCv = p->nc;
    if (p->fwdq[pass]) {
      const size_t smq = sizeof(float) * ((size_t)kFwdStages * fwdq_planes(NCv, maps) * fwdq_rows(NCv, maps) * 128 +
                                          (size_t)p->max_sny * (8 + (QG + 3) / 4 * 4));
      bool launched = false;
      const int NVv = p->fwd_nv[pass];
#define MRSIM_YF(QGV, NVV, NCV, M)                                                      \
  if (QG == QGV && NVv == NVV && NCv == NCV && maps == M) {                             \
    auto k = ystage_q_kernel<QGV, NVV, NCV, M>;                                         \
    set_smem(k, smq);                                                                   \
    k<<<(unsigned)R.n, 256, smq, st>>>(p->d_units, tiles, p->fwd_cls ? 1 : 0);          \
    launched = true;                                                                    \
  }
#define MRSIM_YFQ(NCV, M) MRSIM_YF(1, 0, NCV, M) MRSIM_YF(2, 0, NCV, M) MRSIM_YF(4, 0, NCV, M) MRSIM_YF(8, 0, NCV, M)
#define MRSIM_YFN(M) MRSIM_YFQ(1, M) MRSIM_YFQ(2, M) MRSIM_YFQ(3, M) MRSIM_YFQ(4, M) MRSIM_YFQ(8, M)
      MRSIM_YFN(false) MRSIM_YFN(true)
      MRSIM_YF(8, 6, 1, false) MRSIM_YF(8, 6, 2, false) MRSIM_YF(8, 6, 3, false) MRSIM_YF(8, 6, 4, false)
      MRSIM_YF(8, 6, 1, true) MRSIM_YF(8, 6, 2, true) MRSIM_YF(8, 6, 3, true)
#undef MRSIM_YFN
#undef MRSIM_YFQ
#undef MRSIM_YF
      if (!launched) fail("no forward kernel instance for this unit shape");
      MRSIM_CUDA(cudaGetLastError());
      continue;
    }
    const size_t sm = sizeof(float) * (size_t)p->max_sny * (kT + (QG + 3) / 4 * 4);
    bool launched = false;
#define MRSIM_Y(QGV, NCV, M)                                                            \
  if (QG == QGV && NCv == NCV && maps == M) {                                           \
    auto k = ystage_kernel<kT, QGV, NCV, M>;                                            \
    set_smem(k, sm);                                                                    \
    k<<<(unsigned)R.n, 128, sm, st>>>(p->d_units, tiles);                               \
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

namespace {
void launch_xstage(const EpiPlan* p, cudaStream_t st, int u0, int u1, bool adj) {
  if ((adj && p->adj_cls) || (!adj && p->fwd_cls)) {
    const TileRange R = tile_range(p->c_start, p->n_ctiles, u0, u1);
    if (R.n == 0) return;
    const int4* tiles = p->d_ctiles + R.t0;
    const unsigned g = (unsigned)R.n;
#define MRSIM_XC(ADJ)                                                                             \
  switch (p->xfft_e) {                                                                            \
    case 1: xfft_warp_kernel<1, ADJ, true><<<g, 256, 0, st>>>(p->d_units, tiles); break;          \
    case 2: xfft_warp_kernel<2, ADJ, true><<<g, 256, 0, st>>>(p->d_units, tiles); break;          \
    case 3: xfft_warp_kernel<3, ADJ, true><<<g, 256, 0, st>>>(p->d_units, tiles); break;          \
    default: xfft_warp_kernel<4, ADJ, true><<<g, 256, 0, st>>>(p->d_units, tiles); break;         \
  }
    if (adj) {
      MRSIM_XC(true)
    } else {
      MRSIM_XC(false)
    }
#undef MRSIM_XC
    MRSIM_CUDA(cudaGetLastError());
    return;
  }
  if (p->xfft && p->xfft_e < 0) {
    if (!(u0 == 0 && (u1 < 0 || u1 == p->n_units))) fail("a plan of mixed row widths runs its units whole");
    for (int E = 1; E <= 8; ++E) {
      if (p->fe_count[E] == 0) continue;
      const int4* tiles = p->d_ftiles + p->fe_first[E];
      const unsigned g = (unsigned)p->fe_count[E];
#define MRSIM_XE(ADJ)                                                                               \
  switch (E) {                                                                                      \
    case 1: xfft_warp_kernel<1, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;           \
    case 2: xfft_warp_kernel<2, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;           \
    case 3: xfft_warp_kernel<3, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;           \
    case 4: xfft_warp_kernel<4, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;           \
    case 5: xfft_warp_kernel<5, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;           \
    case 6: xfft_warp_kernel<6, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;           \
    case 7: xfft_warp_kernel<7, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;           \
    default: xfft_warp_kernel<8, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;          \
  }
      if (adj) {
        MRSIM_XE(true)
      } else {
        MRSIM_XE(false)
      }
#undef MRSIM_XE
      MRSIM_CUDA(cudaGetLastError());
    }
    return;
  }
  if (p->xfft) {
    const TileRange R = tile_range(p->f_start, p->n_ftiles, u0, u1);
    if (R.n == 0) return;
    const int4* tiles = p->d_ftiles + R.t0;
    const unsigned g = (unsigned)R.n;
#define MRSIM_XF(ADJ)                                                                             \
  switch (p->xfft_e) {                                                                            \
    case 1: xfft_warp_kernel<1, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;         \
    case 2: xfft_warp_kernel<2, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;         \
    case 3: xfft_warp_kernel<3, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;         \
    case 4: xfft_warp_kernel<4, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;         \
    case 5: xfft_warp_kernel<5, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;         \
    case 6: xfft_warp_kernel<6, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;         \
    case 7: xfft_warp_kernel<7, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;         \
    case 8: xfft_warp_kernel<8, ADJ, false><<<g, 256, 0, st>>>(p->d_units, tiles); break;         \
    default: xfft_kernel<ADJ><<<g, 256, 0, st>>>(p->d_units, tiles);                              \
  }
    if (adj) {
      MRSIM_XF(true)
    } else {
      MRSIM_XF(false)
    }
#undef MRSIM_XF
    MRSIM_CUDA(cudaGetLastError());
    return;
  }
  const int dir = adj ? 1 : 0;
  const TileRange R = tile_range(p->g_start[dir], p->n_gtiles[dir], u0, u1);
  if (R.n == 0) return;
  const XTile* tiles = (const XTile*)p->d_gtiles[dir] + R.t0;
  if (adj)
    xgemm_kernel<true><<<(unsigned)R.n, 256, 0, st>>>(p->d_units, tiles);
  else
    xgemm_kernel<false><<<(unsigned)R.n, 256, 0, st>>>(p->d_units, tiles);
  MRSIM_CUDA(cudaGetLastError());
}
}  // namespace

void epi_plan_forward_xstage(const EpiPlan* p, cudaStream_t st, int u0, int u1) { launch_xstage(p, st, u0, u1, false); }

void epi_plan_adjoint_xstage(const EpiPlan* p, cudaStream_t st, int u0, int u1) { launch_xstage(p, st, u0, u1, true); }

void epi_plan_adjoint_ystage(const EpiPlan* p, cudaStream_t st, int u0, int u1) {
  for (int pass = 0; pass < 4; ++pass) {
    const TileRange R = tile_range(p->a_start[pass], p->n_atiles[pass], u0, u1);
    if (R.n == 0) continue;
    const int4* tiles = p->d_atiles[pass] + R.t0;
    const bool maps = pass & 1, grads = (pass & 2) != 0;
    const int NCv = p->nc;
    if (p->adjq[pass]) {
      const int NQv = p->adjq[pass];
      const int TYv = p->adj_ty[pass];
      const size_t smq = sizeof(float2) * (size_t)kAdjStages * adjq_chunk_lines(NQv) * NQv * 128 +
                         sizeof(float) * (size_t)(p->max_lines + adjq_chunk_lines(NQv)) *
                             (2 * TYv + adjq_line_floats(NCv, maps));
      bool launched = false;
      const bool virt = p->adj_cls;
      // the built-in rows per thread, and 2 rows where the built-in choice is 4
#define MRSIM_AQV(NQV, NCV, M, G, V)                                                    \
  if (NQv == NQV && NCv == NCV && maps == M && grads == G && virt == V) {               \
    if (TYv == adjq_rows_v(NCV, M, V)) {                                                \
      auto k = yadjoint_q_kernel<NQV, adjq_rows_v(NCV, M, V), NCV, M, G, V>;            \
      set_smem(k, smq);                                                                 \
      k<<<(unsigned)R.n, 256, smq, st>>>(p->d_units, tiles);                            \
      launched = true;                                                                  \
    } else if (adjq_rows_v(NCV, M, V) == 4 && TYv == 2) {                               \
      auto k = yadjoint_q_kernel<NQV, 2, NCV, M, G, V>;                                 \
      set_smem(k, smq);                                                                 \
      k<<<(unsigned)R.n, 256, smq, st>>>(p->d_units, tiles);                            \
      launched = true;                                                                  \
    }                                                                                   \
  }
#define MRSIM_AQ(NQV, NCV, M, G) MRSIM_AQV(NQV, NCV, M, G, false)
#define MRSIM_AQC(NCV, M, G) MRSIM_AQ(1, NCV, M, G) MRSIM_AQ(2, NCV, M, G) MRSIM_AQ(4, NCV, M, G) MRSIM_AQ(8, NCV, M, G)
#define MRSIM_AQN(M, G) MRSIM_AQC(1, M, G) MRSIM_AQC(2, M, G) MRSIM_AQC(3, M, G) MRSIM_AQC(4, M, G)
#define MRSIM_AQK(M, G) MRSIM_AQV(6, 1, M, G, true) MRSIM_AQV(6, 2, M, G, true) MRSIM_AQV(6, 3, M, G, true) \
  MRSIM_AQV(6, 4, M, G, true)
      MRSIM_AQN(false, false) MRSIM_AQN(true, false) MRSIM_AQN(false, true) MRSIM_AQN(true, true)
      MRSIM_AQC(8, false, false) MRSIM_AQC(8, false, true)
      MRSIM_AQK(false, false) MRSIM_AQK(true, false) MRSIM_AQK(false, true) MRSIM_AQK(true, true)
#undef MRSIM_AQK
#undef MRSIM_AQN
#undef MRSIM_AQC
#undef MRSIM_AQ
#undef MRSIM_AQV
      if (!launched) fail("no adjoint kernel instance for this unit shape");
      MRSIM_CUDA(cudaGetLastError());
      continue;
    }
    size_t sm = sizeof(float2) * (size_t)2 * p->max_hchunk * 128 +
                sizeof(float) * ((size_t)kTY * (p->max_lines + p->max_coils) + 128 * (size_t)p->max_coils +
                                 (size_t)p->max_lines * (5 + NCv));
    bool launched = false;
#define MRSIM_A(NCV, M, G)                                                              \
  if (NCv == NCV && maps == M && grads == G) {                                          \
    auto k = yadjoint_kernel<kTY, NCV, M, G>;                                           \
    set_smem(k, sm);                                                                    \
    k<<<(unsigned)R.n, 128, sm, st>>>(p->d_units, tiles);                               \
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
