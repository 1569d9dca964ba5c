// ts_epi.cu — the time-segmented EPI forward / adjoint on the tensor cores (tcgen05, sm_100a).
//
// The exact operator (epi_kernels.cu) evaluates, per unit (slice, volume) and acquired line j,
//   g_v[j][x] = s sv sum_y ey_v(y) e^{i2pi (a + kr_j(y))} sum_c rel_cj m_c e^{i2pi f t_j}
// with a fresh phasor per (line, voxel).  Here the time dependence is segmented with the
// reference's certified plan (`tseg::plan`, tseg.rs:230-289, the same certificate the spiral
// forward uses, spiral.rs:141-201): the acquired lines are cut into groups over which every
// factor is an exponential in the line time — an echo, split at t = 0 for the spin echo's |t| —
// and with tau_j = t_j - t_first (ms), z_c = -(d_c - d_lo) + i 2pi f / 1000,
//   rel_cj e^{i2pi f t_j} = w_j e^{A_c} e^{i2pi f t_first} e^{z_c tau_j},  w_j = e^{-d_lo tau_j}
//                         ~ w_j sum_l b_l(tau_j) alpha_cl e^{i2pi f (t_first + tau_l/1000)}
// (alpha_cl = e^{A_c - (d_c - d_lo) tau_l}), certified to 1e-7 over the rectangle of rates
// d in [0, max d_c - d_lo], f in the fieldmap's range.  Per group the y-stage becomes one
// complex contraction over K = (node l, row y):
//   G[x, (j, v)] = sum_{l, y} P_l(x, y) B[(l, y), (j, v)],
//   P_l(x, y) = e^{i2pi (a + f t_l)} sum_c alpha_cl m_c            (the segment images)
//   B[(l, y), (j, v)] = s sv ey_v(y) e^{i2pi kr_j(y)} b_l(tau_j) w_j (a constant table)
// run as a real GEMM (re/im interleaved along K and N) in split precision: each operand is
// hi + lo in f16 (or bf16) and D = Ahi Bhi + Alo Bhi + Ahi Blo accumulates in FP32 in TMEM.
// The adjoint is the transposed contraction H[x, (l, y)] = sum_{(j, v)} G[x, (j, v)] conj(B~)
// followed by comp_grad_c(x, y) = sum_l alpha_cl e^{-i2pi (a + f t_l)} H[x, (l, y)].
//
// Kernels:
//   ts_forward_kernel   producers (8 warps) write P into 128-byte-swizzled shared tiles, a TMA
//                       warp loads the B tiles (cp.async.bulk.tensor), an MMA warp issues
//                       tcgen05.mma into double-buffered TMEM accumulators, 4 epilogue warps
//                       read them (tcgen05.ld) and write the class rows the x-stage expands
//   ts_gconvert_kernel  the x-adjoint's class rows (or coil rows, combined into classes) to
//                       split f16/bf16 K-major rows, with a per-unit power-of-two scale
//   ts_adjoint_kernel   TMA loads of both operands, tcgen05.mma, and 8 epilogue warps forming
//                       comp_grad from the TMEM accumulators (phasors on the CUDA cores)
//   ts_scale_kernel     the per-unit power-of-two input scale of the f16 forward
//   ts_expand_kernel    class rows to coil rows when the x-stage runs per coil
// Coverage: uniform relaxation (no voxel maps), no eddy-current polynomial (its time profile is
// not an exponential in t), at most 4 compartments; everything else of the exact operator.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "driver.h"
#include "host_tables.h"
#include "mrsim_internal.h"
#include "sm100_ptx.h"
#include "spiral_host.h"
#include "ts_epi.h"

namespace mrsim {

using namespace sm100;

namespace {

constexpr float kTwoPiF = 6.28318530717958647692f;
constexpr int kStages = 2;       // operand stages of A (and of everything in the adjoint)
constexpr int kMaxBStages = 3;   // stages of the forward's constant B tiles, when they fit
constexpr int kStageA = 32768;   // A hi + lo: 128 rows x 128 bytes each
constexpr int kNodeFloats = 6;   // per node in shared memory: t_hi, t_lo, alpha[4]

// error codes written to the plan's device flag
enum : int { TS_ERR_FULL_A = 1, TS_ERR_FULL_B = 2, TS_ERR_EMPTY = 3, TS_ERR_ACC_FULL = 4, TS_ERR_ACC_EMPTY = 5,
             TS_ERR_DRAIN = 6 };

__device__ __forceinline__ float phase_turns(float s, float f, float t_hi, float t_lo) {
  // s + f (t_hi + t_lo) reduced to |theta| <= 1/2: n = round(s + f t_hi) by the 1.5 * 2^23 trick,
  // r = f t_hi - n from one FMA of the exact product, theta = (r + s) + f t_lo
  const float nn = __fsub_rn(12582912.0f, __fadd_rn(fmaf(f, t_hi, s), 12582912.0f));
  return fmaf(f, t_lo, __fadd_rn(fmaf(f, t_hi, nn), s));
}

template <int DT>
struct Split;
template <>
struct Split<0> {  // f16
  static __device__ __forceinline__ uint32_t pack(float a, float b) {
    __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
  }
  static __device__ __forceinline__ float2 unpack(uint32_t u) {
    __half2 h = *reinterpret_cast<__half2*>(&u);
    return __half22float2(h);
  }
};
template <>
struct Split<1> {  // bf16
  static __device__ __forceinline__ uint32_t pack(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
  }
  static __device__ __forceinline__ float2 unpack(uint32_t u) {
    __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162*>(&u);
    return __bfloat1622float2(h);
  }
};
// (re, im) -> hi pair and lo pair: hi = round(v), lo = round(v - hi)
template <int DT>
__device__ __forceinline__ void split2(float re, float im, uint32_t& hi, uint32_t& lo) {
  hi = Split<DT>::pack(re, im);
  const float2 h = Split<DT>::unpack(hi);
  lo = Split<DT>::pack(re - h.x, im - h.y);
}

// No memory clobber: the compiler may keep computing the next values across these stores; the
// async-proxy fence that publishes the tile (a volatile asm with a memory clobber) stays after them.
__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d));
}

struct TsSmem {
  uint32_t a0, b0;      // shared addresses of stage 0 of A and B
  uint32_t b_stage;     // bytes per B stage (hi + lo)
};

// ---------------------------------------------------------------------------------------------
// forward y-stage
template <int DT, int NC>
__global__ void __launch_bounds__(448, 1) ts_forward_kernel(const __grid_constant__ TsFwdParams P) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t b_stage = 2u * (uint32_t)P.np_max * 128u;
  const int SB = P.b_stages;  // B stages (A has kStages): the constant tiles prefetched further ahead
  unsigned char* sA = smem;
  unsigned char* sB = sA + kStages * kStageA;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + SB * b_stage);
  uint64_t* full_a = bars;                   // [kStages]
  uint64_t* empty_a = full_a + kStages;      // [kStages]
  uint64_t* full_b = empty_a + kStages;      // [kMaxBStages]
  uint64_t* empty_b = full_b + kMaxBStages;  // [kMaxBStages]
  uint64_t* acc_full = empty_b + kMaxBStages;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* drain = acc_empty + 2;
  uint32_t* tmem_base_s = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_s = reinterpret_cast<volatile int*>(tmem_base_s + 1);
  // every group's node times and compartment weights: [group][l][t_hi, t_lo, alpha 0..3]
  float* nodes = reinterpret_cast<float*>(tmem_base_s + 4);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_a[s], 8);
      mbar_init(&empty_a[s], 1);
    }
    for (int s = 0; s < SB; ++s) {
      mbar_init(&full_b[s], 1);
      mbar_init(&empty_b[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 4);
    }
    mbar_init(drain, 1);
    *abort_s = 0;
    fence_mbar_init();
  }
  for (int e = threadIdx.x; e < P.n_groups * kTsMaxL; e += blockDim.x) {
    const int g = e / kTsMaxL, l = e % kTsMaxL;
    const TsGroupDev& G = P.groups[g];
    float* d = nodes + (size_t)e * kNodeFloats;
    d[0] = G.t_hi[l];
    d[1] = G.t_lo[l];
    for (int cc = 0; cc < 4; ++cc) d[2 + cc] = G.alpha[l][cc];
  }
  if (warp == 13) {
    tmem_alloc(tmem_base_s, 512);
    tmem_relinquish();
  }
  if (warp == 12 && lane == 0)
    for (int g = 0; g < P.n_groups; ++g) tma_prefetch_map(&P.bmap[g]);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_base_s;
  const int n_items = P.n_items;

  if (warp < 8) {
    // ---- producers: the segment images P_l(x, y), split, into the swizzled A tiles ----------
    const int r = 32 * (warp & 3) + lane, kh = warp >> 2;
    const uint32_t a0 = smem_u32(sA);
    uint32_t c = 0;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
      const int ui = P.u0 + it / P.snx_tiles;
      const UnitDesc& u = P.units[ui];
      const int snx = u.snx, sny = u.sny;
      const int x = (it % P.snx_tiles) * 128 + r;
      const bool xok = x < snx;
      const float scale = P.unit_scale ? P.unit_scale[ui] : 1.f;
      const bool distort = (u.flags & UF_DISTORT) != 0;
      const int ny8 = sny / 8;
      // this thread's four rows of the chunk: y = 8 y8 + 4 kh + k
      float ca[4], cf[4], cm[4][NC], na[4], nf[4], nm[4][NC];
      auto load_rows = [&](int y8, float (&a)[4], float (&f)[4], float (&m)[4][NC]) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const size_t i = (size_t)(y8 * 8 + 4 * kh + k) * snx + x;
          a[k] = (xok && u.phase) ? __ldg(u.phase + i) : 0.f;
          f[k] = (xok && distort) ? __ldg(u.fmap + i) : 0.f;
#pragma unroll
          for (int cc = 0; cc < NC; ++cc)
            m[k][cc] = (xok && cc < u.ncomp) ? __ldg(u.comp + (size_t)cc * u.comp_stride + i) * scale : 0.f;
        }
      };
      load_rows(0, na, nf, nm);
      for (int g = 0; g < P.n_groups; ++g) {
        const TsGroupDev& G = P.groups[g];
        const int LQ = G.Lp >> 2;
        for (int kb = 0; kb < G.kb_f; ++kb, ++c) {
          const int y8 = kb / LQ, lq = kb - y8 * LQ;
          if (lq == 0) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              ca[k] = na[k];
              cf[k] = nf[k];
#pragma unroll
              for (int cc = 0; cc < NC; ++cc) cm[k][cc] = nm[k][cc];
            }
            load_rows(y8 + 1 < ny8 ? y8 + 1 : 0, na, nf, nm);  // the next chunk in sequence
          }
          const int s = c % kStages;
          if (!__all_sync(0xffffffffu, mbar_wait(&empty_a[s], ((c / kStages) & 1) ^ 1, abort_s, P.err, TS_ERR_EMPTY)))
            goto done;
          {
            // K within the block: (l % 4) 16 + yy 2 + re/im, so node l's rows 4 kh .. 4 kh + 3 are
            // 16-byte chunk 2 (l % 4) + kh
            const uint32_t hi0 = a0 + s * kStageA, lo0 = hi0 + kStageA / 2;
            // the block's four nodes, read together
            float th4[4], tl4[4], al4[4][NC];
#pragma unroll
            for (int dl = 0; dl < 4; ++dl) {
              const float* nd = nodes + ((size_t)g * kTsMaxL + 4 * lq + dl) * kNodeFloats;
              th4[dl] = nd[0];
              tl4[dl] = nd[1];
#pragma unroll
              for (int cc = 0; cc < NC; ++cc) al4[dl][cc] = nd[2 + cc];
            }
#pragma unroll
            for (int dl = 0; dl < 4; ++dl) {
              const float th = th4[dl], tl = tl4[dl];
              float al[NC];
#pragma unroll
              for (int cc = 0; cc < NC; ++cc) al[cc] = al4[dl][cc];
              uint32_t hv[4], lv[4];
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const float t = phase_turns(ca[k], cf[k], th, tl);
                float sn, cs;
                __sincosf(kTwoPiF * t, &sn, &cs);
                float W = 0.f;
#pragma unroll
                for (int cc = 0; cc < NC; ++cc) W = fmaf(al[cc], cm[k][cc], W);
                split2<DT>(W * cs, W * sn, hv[k], lv[k]);
              }
              const int ch = 2 * dl + kh;
              st_shared_v4(hi0 + sw128_offset(r, ch), hv[0], hv[1], hv[2], hv[3]);
              st_shared_v4(lo0 + sw128_offset(r, ch), lv[0], lv[1], lv[2], lv[3]);
            }
          }
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) mbar_arrive(&full_a[s]);
        }
      }
    }
  } else if (warp < 12) {
    // ---- epilogue: TMEM accumulators to class rows ------------------------------------------
    const int q = warp - 8, r = 32 * q + lane;
    uint32_t gc = 0;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
      const int ui = P.u0 + it / P.snx_tiles;
      const UnitDesc& u = P.units[ui];
      const int snx = u.snx;
      const int x = (it % P.snx_tiles) * 128 + r;
      const bool xok = x < snx;
      const float scale = P.unit_scale ? P.unit_scale[ui] : 1.f;
      float2* out = P.cls_out ? P.cls_out + (size_t)ui * P.cls_unit_stride : u.g;
      for (int g = 0; g < P.n_groups; ++g, ++gc) {
        const TsGroupDev& G = P.groups[g];
        const int b = gc & 1;
        if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[b], (gc >> 1) & 1, abort_s, P.err, TS_ERR_ACC_FULL)))
          goto done;
        tc_fence_after();
        const float osc = G.out_scale_f / scale;
        const uint32_t ta = tmem + (uint32_t)(b * 256) + ((uint32_t)(32 * q) << 16);
        for (int col = 0; col < G.np_f; col += 8) {
          float v[8];
          tmem_ld8(ta + (uint32_t)col, v);
#pragma unroll
          for (int p = 0; p < 4; ++p) {
            const int n2 = (col >> 1) + p, jl = n2 / P.na, vv = n2 - jl * P.na;
            if (jl < G.n_j && xok)
              out[((size_t)vv * u.n_lines + G.lines[jl]) * snx + x] = make_float2(v[2 * p] * osc, v[2 * p + 1] * osc);
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acc_empty[b]);
      }
    }
  } else if (warp == 12) {
    // ---- TMA: the constant B tiles ------------------------------------------------------------
    if (lane == 0) {
      uint32_t c = 0;
      for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        for (int g = 0; g < P.n_groups; ++g) {
          const TsGroupDev& G = P.groups[g];
          for (int kb = 0; kb < G.kb_f; ++kb, ++c) {
            const int s = c % SB;
            if (!mbar_wait(&empty_b[s], ((c / SB) & 1) ^ 1, abort_s, P.err, TS_ERR_EMPTY)) goto tma_done;
            mbar_arrive_expect_tx(&full_b[s], 2u * (uint32_t)G.np_f * 128u);
            unsigned char* bh = sB + s * b_stage;
            tma_load_2d(bh, &P.bmap[g], kb * 64, 0, &full_b[s]);
            tma_load_2d(bh + (size_t)P.np_max * 128, &P.bmap[g], kb * 64, G.np_f, &full_b[s]);
          }
        }
      }
    tma_done:
      // loads still in flight (after an abort) land before the CTA leaves
      for (uint32_t k = c > (uint32_t)SB ? c - SB : 0; k < c; ++k)
        mbar_wait(&full_b[k % SB], (k / SB) & 1, abort_s, nullptr, 0);
    }
    __syncwarp();
  } else {
    // ---- MMA issue -----------------------------------------------------------------------------
    if (lane == 0) {
      uint32_t c = 0, gc = 0;
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
      for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        for (int g = 0; g < P.n_groups; ++g, ++gc) {
          const TsGroupDev& G = P.groups[g];
          const int b = gc & 1;
          if (!mbar_wait(&acc_empty[b], ((gc >> 1) & 1) ^ 1, abort_s, P.err, TS_ERR_ACC_EMPTY)) goto mma_done;
          tc_fence_after();
          const uint32_t d = tmem + (uint32_t)(b * 256);
          const uint32_t idesc = idesc_f16(128, G.np_f, DT);
          for (int kb = 0; kb < G.kb_f; ++kb, ++c) {
            const int s = c % kStages, sb = c % SB;
            if (!mbar_wait(&full_a[s], (c / kStages) & 1, abort_s, P.err, TS_ERR_FULL_A)) goto mma_done;
            if (!mbar_wait(&full_b[sb], (c / SB) & 1, abort_s, P.err, TS_ERR_FULL_B)) goto mma_done;
            tc_fence_after();
            const uint64_t ah = sw128_desc(a0 + s * kStageA), al = sw128_desc(a0 + s * kStageA + kStageA / 2);
            const uint64_t bh = sw128_desc(b0 + sb * b_stage), bl = sw128_desc(b0 + sb * b_stage + P.np_max * 128);
#pragma unroll
            for (int k = 0; k < 4; ++k) umma_f16(d, ah + 2 * k, bh + 2 * k, idesc, (kb | k) != 0);
#pragma unroll
            for (int k = 0; k < 4; ++k) umma_f16(d, al + 2 * k, bh + 2 * k, idesc, 1);
#pragma unroll
            for (int k = 0; k < 4; ++k) umma_f16(d, ah + 2 * k, bl + 2 * k, idesc, 1);
            umma_commit(&empty_a[s]);
            umma_commit(&empty_b[sb]);
          }
          umma_commit(&acc_full[b]);
        }
      }
    mma_done:
      // every MMA this thread issued completes before the TMEM is released
      umma_commit(drain);
      mbar_wait(drain, 0, abort_s, P.err, TS_ERR_DRAIN);
    }
    __syncwarp();
  }
done:
  tc_fence_before();
  __syncthreads();
  if (warp == 13) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ---------------------------------------------------------------------------------------------
// The x-adjoint's rows as split K-major operand rows: Gs[unit * snx_pad + x][ka0_g + (j NA + v) 2
// + ri] for each group, zero past a group's lines and past snx; with a per-unit power-of-two
// scale that puts the largest magnitude near 2^8 (f16), or 1 (bf16).
template <int DT>
__global__ void __launch_bounds__(256) ts_gconvert_kernel(TsConvParams P) {
  const int ui = P.u0 + blockIdx.x;
  const UnitDesc& u = P.units[ui];
  const int snx = u.snx, nl = u.n_lines, na = P.na;
  const float s = u.signal_scale, so = s * u.geo.coil_off;
  // G(v, line, x): a class row, read directly or formed from the coil rows
  auto gval = [&](int v, int line, int x) -> float2 {
    if (P.class_rows) return u.g[((size_t)v * nl + line) * snx + x];
    float2 acc = make_float2(0.f, 0.f);
    if (v == na - 1) {
      for (int qq = 0; qq < u.ncoils; ++qq) {
        const float2 h = u.g[((size_t)qq * nl + line) * snx + x];
        acc.x += h.x;
        acc.y += h.y;
      }
      return make_float2(so * acc.x, so * acc.y);
    }
    for (int qq = 0; qq < u.ncoils; ++qq) {
      if (u.geo.cls[qq] != v) continue;
      const float2 h = u.g[((size_t)qq * nl + line) * snx + x];
      const float e = u.geo.ex[(size_t)qq * snx + x];
      acc.x = fmaf(e, h.x, acc.x);
      acc.y = fmaf(e, h.y, acc.y);
    }
    return make_float2(s * acc.x, s * acc.y);
  };
  __shared__ float red[256];
  float scale = 1.f;
  if (DT == 0) {
    float mx = 0.f;
    for (int g = 0; g < P.n_groups; ++g) {
      const TsGroupDev& G = P.groups[g];
      const int n = G.n_j * na * snx;
      for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const int x = e % snx, p = e / snx, jl = p / na, v = p - jl * na;
        const float2 w = gval(v, G.lines[jl], x);
        mx = fmaxf(mx, fmaxf(fabsf(w.x), fabsf(w.y)));
      }
    }
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
      if (threadIdx.x < k) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + k]);
      __syncthreads();
    }
    mx = red[0];
    scale = mx > 0.f ? exp2f(8.f - ceilf(log2f(mx))) : 1.f;
  }
  if (threadIdx.x == 0) P.unit_scale[ui] = scale;
  const int kc_total = P.kp_total / 8;  // 16-byte chunks per row
  const int n = P.snx_pad * kc_total;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const int x = e % P.snx_pad, kc = e / P.snx_pad;
    const int k0 = kc * 8;
    int g = 0;
    while (g + 1 < P.n_groups && k0 >= P.groups[g + 1].ka0) ++g;
    const TsGroupDev& G = P.groups[g];
    uint32_t hv[4], lv[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int p = (k0 - G.ka0) / 2 + i, jl = p / na, v = p - jl * na;
      float2 w = make_float2(0.f, 0.f);
      if (x < snx && jl < G.n_j) w = gval(v, G.lines[jl], x);
      split2<DT>(w.x * scale, w.y * scale, hv[i], lv[i]);
    }
    const size_t off = ((size_t)ui * P.snx_pad + x) * P.kp_total + k0;
    *reinterpret_cast<uint4*>(P.gs_hi + off) = make_uint4(hv[0], hv[1], hv[2], hv[3]);
    *reinterpret_cast<uint4*>(P.gs_lo + off) = make_uint4(lv[0], lv[1], lv[2], lv[3]);
  }
}

// ---------------------------------------------------------------------------------------------
// adjoint y-stage
template <int DT, int NC>
__global__ void __launch_bounds__(320, 1) ts_adjoint_kernel(const __grid_constant__ TsAdjParams P) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t b_stage = 2u * (uint32_t)P.np_max * 128u;
  unsigned char* sA = smem;
  unsigned char* sB = sA + kStages * kStageA;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + kStages * b_stage);
  uint64_t* full = bars;
  uint64_t* empty = bars + kStages;
  uint64_t* acc_full = bars + 2 * kStages;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* drain = acc_empty + 2;
  uint32_t* tmem_base_s = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_s = reinterpret_cast<volatile int*>(tmem_base_s + 1);
  // every group's node times and adjoint weights: [group][l][t_hi, t_lo, alpha_adj 0..3]
  float* nodes = reinterpret_cast<float*>(tmem_base_s + 4);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int e = threadIdx.x; e < P.n_groups * kTsMaxL; e += blockDim.x) {
    const int g = e / kTsMaxL, l = e % kTsMaxL;
    const TsGroupDev& G = P.groups[g];
    float* d = nodes + (size_t)e * kNodeFloats;
    d[0] = G.t_hi[l];
    d[1] = G.t_lo[l];
    for (int cc = 0; cc < 4; ++cc) d[2 + cc] = G.alpha_adj[l][cc];
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&acc_full[b], 1);
      mbar_init(&acc_empty[b], 8);
    }
    mbar_init(drain, 1);
    *abort_s = 0;
    fence_mbar_init();
  }
  if (warp == 9) {
    tmem_alloc(tmem_base_s, 512);
    tmem_relinquish();
  }
  if (warp == 8 && lane == 0) {
    tma_prefetch_map(&P.amap_hi);
    tma_prefetch_map(&P.amap_lo);
    for (int g = 0; g < P.n_groups; ++g) tma_prefetch_map(&P.bmap[g]);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_base_s;
  const int n_items = P.n_items, nyc = P.nyc, YC = P.yc, YH = YC / 2;

  if (warp < 8) {
    // ---- epilogue: H -> comp_grad ------------------------------------------------------------
    const int q = warp & 3, h = warp >> 2, r = 32 * q + lane;
    uint32_t gc = 0;
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
      const int ui = P.u0 + it / P.snx_tiles;
      const UnitDesc& u = P.units[ui];
      const int snx = u.snx;
      const size_t plane = (size_t)snx * u.sny;
      const int x = (it % P.snx_tiles) * 128 + r;
      const bool xok = x < snx;
      const bool distort = (u.flags & UF_DISTORT) != 0;
      const float inv = 1.f / P.unit_scale[ui];
      for (int yc = 0; yc < nyc; ++yc) {
        float a[4], f[4];
        float2 acc[4][NC];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int y = yc * YC + h * YH + k;
          const bool ok = xok && k < YH;
          const size_t i = (size_t)y * snx + x;
          a[k] = (ok && u.phase) ? __ldg(u.phase + i) : 0.f;
          f[k] = (ok && distort) ? __ldg(u.fmap + i) : 0.f;
#pragma unroll
          for (int cc = 0; cc < NC; ++cc) acc[k][cc] = make_float2(0.f, 0.f);
        }
        for (int g = 0; g < P.n_groups; ++g, ++gc) {
          const TsGroupDev& G = P.groups[g];
          const int b = gc & 1;
          if (!__all_sync(0xffffffffu, mbar_wait(&acc_full[b], (gc >> 1) & 1, abort_s, P.err, TS_ERR_ACC_FULL)))
          goto done;
          tc_fence_after();
          const uint32_t ta = tmem + (uint32_t)(b * 256) + ((uint32_t)(32 * q) << 16);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            if (k >= YH) break;
            const int yy = h * YH + k;
            for (int l0 = 0; l0 < G.Lp; l0 += 4) {
              float v[8];
              tmem_ld8(ta + (uint32_t)((yy * G.Lp + l0) * 2), v);
#pragma unroll
              for (int p = 0; p < 4; ++p) {
                const int l = l0 + p;
                if (l >= G.L) break;
                const float* nd = nodes + ((size_t)g * kTsMaxL + l) * kNodeFloats;
                const float t = phase_turns(a[k], f[k], nd[0], nd[1]);
                float sn, cs;
                __sincosf(kTwoPiF * t, &sn, &cs);
                const float hr = v[2 * p], hi = v[2 * p + 1];
                const float zr = fmaf(cs, hr, sn * hi), zi = fmaf(cs, hi, -sn * hr);
#pragma unroll
                for (int cc = 0; cc < NC; ++cc) {
                  const float w = nd[2 + cc];
                  acc[k][cc].x = fmaf(w, zr, acc[k][cc].x);
                  acc[k][cc].y = fmaf(w, zi, acc[k][cc].y);
                }
              }
            }
          }
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[b]);
        }
        if (xok) {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            if (k >= YH) break;
            const int y = yc * YC + h * YH + k;
#pragma unroll
            for (int cc = 0; cc < NC; ++cc)
              if (cc < u.ncomp)
                u.comp_grad[(size_t)cc * plane + (size_t)y * snx + x] = make_float2(acc[k][cc].x * inv, acc[k][cc].y * inv);
          }
        }
      }
    }
  } else if (warp == 8) {
    // ---- TMA: the k-space rows (A) and the constant table (B) ----------------------------------
    if (lane == 0) {
      uint32_t c = 0;
      for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const int ui = P.u0 + it / P.snx_tiles;
        const int row = ui * P.snx_pad + (it % P.snx_tiles) * 128;
        for (int yc = 0; yc < nyc; ++yc)
          for (int g = 0; g < P.n_groups; ++g) {
            const TsGroupDev& G = P.groups[g];
            for (int kb = 0; kb < G.kp_a / 64; ++kb, ++c) {
              const int s = c % kStages;
              if (!mbar_wait(&empty[s], ((c / kStages) & 1) ^ 1, abort_s, P.err, TS_ERR_EMPTY)) goto tma_done;
              mbar_arrive_expect_tx(&full[s], (uint32_t)kStageA + 2u * (uint32_t)G.np_a * 128u);
              unsigned char* ad = sA + s * kStageA;
              tma_load_2d(ad, &P.amap_hi, G.ka0 + kb * 64, row, &full[s]);
              tma_load_2d(ad + kStageA / 2, &P.amap_lo, G.ka0 + kb * 64, row, &full[s]);
              unsigned char* bd = sB + s * b_stage;
              tma_load_2d(bd, &P.bmap[g], kb * 64, (yc * 2) * G.np_a, &full[s]);
              tma_load_2d(bd + (size_t)P.np_max * 128, &P.bmap[g], kb * 64, (yc * 2 + 1) * G.np_a, &full[s]);
            }
          }
      }
    tma_done:
      for (uint32_t k = c > kStages ? c - kStages : 0; k < c; ++k)
        mbar_wait(&full[k % kStages], (k / kStages) & 1, abort_s, nullptr, 0);
    }
    __syncwarp();
  } else {
    // ---- MMA issue -----------------------------------------------------------------------------
    if (lane == 0) {
      uint32_t c = 0, gc = 0;
      const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
      for (int it = blockIdx.x; it < n_items; it += gridDim.x)
        for (int yc = 0; yc < nyc; ++yc)
          for (int g = 0; g < P.n_groups; ++g, ++gc) {
            const TsGroupDev& G = P.groups[g];
            const int b = gc & 1;
            if (!mbar_wait(&acc_empty[b], ((gc >> 1) & 1) ^ 1, abort_s, P.err, TS_ERR_ACC_EMPTY)) goto mma_done;
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(b * 256);
            const uint32_t idesc = idesc_f16(128, G.np_a, DT);
            const int nkb = G.kp_a / 64;
            for (int kb = 0; kb < nkb; ++kb, ++c) {
              const int s = c % kStages;
              if (!mbar_wait(&full[s], (c / kStages) & 1, abort_s, P.err, TS_ERR_FULL_A)) goto mma_done;
              tc_fence_after();
              const uint64_t ah = sw128_desc(a0 + s * kStageA), al = sw128_desc(a0 + s * kStageA + kStageA / 2);
              const uint64_t bh = sw128_desc(b0 + s * b_stage), bl = sw128_desc(b0 + s * b_stage + P.np_max * 128);
#pragma unroll
              for (int k = 0; k < 4; ++k) umma_f16(d, ah + 2 * k, bh + 2 * k, idesc, (kb | k) != 0);
#pragma unroll
              for (int k = 0; k < 4; ++k) umma_f16(d, al + 2 * k, bh + 2 * k, idesc, 1);
#pragma unroll
              for (int k = 0; k < 4; ++k) umma_f16(d, ah + 2 * k, bl + 2 * k, idesc, 1);
              umma_commit(&empty[s]);
            }
            umma_commit(&acc_full[b]);
          }
    mma_done:
      umma_commit(drain);
      mbar_wait(drain, 0, abort_s, P.err, TS_ERR_DRAIN);
    }
    __syncwarp();
  }
done:
  tc_fence_before();
  __syncthreads();
  if (warp == 9) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// Per unit: the f16 forward's input scale, a power of two putting max_voxel sum_c amax_c |m_c|
// near 2^8.
__global__ void __launch_bounds__(256) ts_scale_kernel(const UnitDesc* __restrict__ units, int u0, TsAmax amax,
                                                       float* __restrict__ out) {
  const int ui = u0 + blockIdx.x;
  const UnitDesc& u = units[ui];
  const size_t n = (size_t)u.snx * u.sny;
  float mx = 0.f;
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) {
    float w = 0.f;
    for (int c = 0; c < u.ncomp; ++c) w = fmaf(amax.v[c], fabsf(__ldg(u.comp + (size_t)c * u.comp_stride + i)), w);
    mx = fmaxf(mx, w);
  }
  __shared__ float red[256];
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + k]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[ui] = red[0] > 0.f ? exp2f(8.f - ceilf(log2f(red[0]))) : 1.f;
}

// Class rows (scratch) to the unit's coil rows: g_q = ex_q G_cls(q) + G_off.
__global__ void __launch_bounds__(256) ts_expand_kernel(const UnitDesc* __restrict__ units, int u0, int na,
                                                        const float2* __restrict__ cls, long long cls_stride) {
  const int ui = u0 + blockIdx.y;
  const UnitDesc& u = units[ui];
  const int snx = u.snx, nl = u.n_lines;
  const float2* C = cls + (size_t)ui * cls_stride;
  const int n = nl * snx;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const int line = e / snx, x = e - line * snx;
    const float2 off = C[((size_t)(na - 1) * nl + line) * snx + x];
    for (int qq = 0; qq < u.ncoils; ++qq) {
      const float2 t = C[((size_t)u.geo.cls[qq] * nl + line) * snx + x];
      const float ex = u.geo.ex[(size_t)qq * snx + x];
      u.g[((size_t)qq * nl + line) * snx + x] = make_float2(fmaf(ex, t.x, off.x), fmaf(ex, t.y, off.y));
    }
  }
}

// ---- host ---------------------------------------------------------------------------------------
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiled)f;
  });
  if (!fn) fail("the driver does not provide cuTensorMapEncodeTiled");
  return fn;
}

// A 2D map over a row-major [rows][cols] array of 16-bit elements, tiles of 64 columns (128
// bytes, swizzled) by box_rows rows.
CUtensorMap make_map(const void* base, int dt, uint64_t cols, uint64_t rows, uint32_t box_rows) {
  CUtensorMap m;
  std::memset(&m, 0, sizeof m);
  if (((uintptr_t)base & 15) || (cols * 2) % 16 || box_rows == 0 || box_rows > 256)
    fail("segmented path: a table violates the tensor-map alignment rules");
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {cols * 2};
  const cuuint32_t box[2] = {64, box_rows};
  const cuuint32_t es[2] = {1, 1};
  CUresult r = encode_fn()(&m, dt == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                           const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail("segmented path: cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return m;
}

uint16_t to16(double v, int dt) {
  if (dt == 0) {
    __half h = __float2half_rn((float)v);
    return *reinterpret_cast<uint16_t*>(&h);
  }
  __nv_bfloat16 h = __float2bfloat16_rn((float)v);
  return *reinterpret_cast<uint16_t*>(&h);
}
double from16(uint16_t u, int dt) {
  if (dt == 0) {
    __half h = *reinterpret_cast<__half*>(&u);
    return (double)__half2float(h);
  }
  __nv_bfloat16 h = *reinterpret_cast<__nv_bfloat16*>(&u);
  return (double)__bfloat162float(h);
}

// A power of two putting the largest |entry| near 2^8.
double pow2_scale(double mx) { return mx > 0 ? std::ldexp(1.0, 8 - (int)std::ceil(std::log2(mx))) : 1.0; }

}  // namespace

// ---------------------------------------------------------------------------------------------
TsPlan::~TsPlan() = default;

void ts_plan_destroy(TsPlan* p) { delete p; }

TsPlan* ts_plan_build(const EpiOperator& op, int precision) {
  if (precision != 1 && precision != 2) fail("segmented path: precision must be 1 (split f16) or 2 (split bf16)");
  const int dt = precision == 1 ? 0 : 1;
  const EpiPlan& ep = *op.plan;
  if (op.maps) fail("the segmented path needs uniform T2 and T2' (voxel maps make the decay rates per voxel)");
  if (op.any_eddy)
    fail("the segmented path does not model the eddy-current polynomial (its time profile is not an exponential)");
  if (op.ncomp > 4) fail("the segmented path handles at most 4 compartments");
  if (op.want_fmap || op.want_r2)
    fail("the segmented path computes the complex-image adjoint only: create the operator with grads = 0");
  if (op.sny % 8) fail("the segmented path needs sny a multiple of 8");
  std::unique_ptr<TsPlan> tp(new TsPlan());
  TsPlan& T = *tp;
  T.dt = dt;
  const int snx = op.snx, sny = op.sny, nx = op.nx, ny = op.ny, ncomp = op.ncomp;
  const mrsim_acquisition& acq = op.acq;
  cudaStream_t st = op.ctx->stream;
  TsegDevice fitdev(st);  // the segmentation fits' per-sample work

  // coil classes (the geometry's bitwise-equal ey rows) plus the offset row
  std::vector<float> eyc((size_t)op.geo.ncls * sny);
  MRSIM_CUDA(cudaMemcpy(eyc.data(), op.geo.eyc, eyc.size() * 4, cudaMemcpyDeviceToHost));
  const int ncls = op.geo.ncls, na = ncls + 1;
  T.na = na;
  const double sig = acq.signal_scale, off = op.geo.coil_off;

  // the fieldmap range the segmentation must certify
  double fmin = 0, fmax = 0;
  if (acq.do_distortions && !op.h_fmap.empty()) {
    fmin = *std::min_element(op.h_fmap.begin(), op.h_fmap.end());
    fmax = *std::max_element(op.h_fmap.begin(), op.h_fmap.end());
  }
  T.fmin = fmin;
  T.fmax = fmax;

  // ---- groups: echo x sign of t (spin echo), lines in table order ------------------------------
  struct Line {
    int idx, ky;
    double t_s, tb0, trf, inh;
  };
  std::vector<std::vector<Line>> groups;
  for (int e = 0; e < op.n_echoes; ++e) {
    mrsim_acquisition a = acq;
    a.t_echo = op.tes[e];
    LineTimingTab lt = line_timing(a, nx, ny);
    std::vector<Line> neg, pos;
    for (int i = 0; i < (int)op.h_lines.size(); ++i) {
      const LineRec& L = op.h_lines[i];
      if (L.row / ny != e) continue;
      Line l;
      l.idx = i;
      l.ky = L.ky;
      l.t_s = lt.t_ms[L.ky] / 1000.0;
      l.trf = lt.trf_ms[L.ky];
      const bool spin = acq.echo == MRSIM_ECHO_SPIN;
      l.tb0 = spin ? l.t_s : l.t_s + a.t_echo / 1000.0;
      l.inh = spin ? std::fabs(l.t_s) * 1000.0 : l.trf;
      (spin && l.t_s < 0 ? neg : pos).push_back(l);
    }
    // at most 256 output columns per group: n_j NA 2 <= 256
    const int cap = std::max(1, std::min(kTsMaxLines, 256 / (2 * na)));
    for (auto* v : {&neg, &pos}) {
      if (v->empty()) continue;
      for (size_t i0 = 0; i0 < v->size(); i0 += cap)
        groups.emplace_back(v->begin() + i0, v->begin() + std::min(v->size(), i0 + (size_t)cap));
    }
  }
  if ((int)groups.size() > kTsMaxGroups)
    fail("the segmented path supports at most " + std::to_string(kTsMaxGroups) + " line groups");
  T.n_groups = (int)groups.size();

  const int ys = ny / 2, oy = sny / ny, sys = oy * ys;
  const long long m2 = 2LL * sny;
  T.groups_h.resize(T.n_groups);
  std::vector<std::vector<double>> bre(T.n_groups), bim(T.n_groups);  // complex B[(l,y)][(j,v)]
  int np_max_f = 16, L_min_yc = 1 << 30;
  int ka = 0;
  T.flops_fwd = T.flops_adj = 0;
  for (int g = 0; g < T.n_groups; ++g) {
    const std::vector<Line>& gl = groups[g];
    TsGroupDev& G = T.groups_h[g];
    std::memset(&G, 0, sizeof G);
    const int nj = (int)gl.size();
    G.n_j = nj;
    double tmin = gl[0].t_s, tmax = gl[0].t_s;
    int imin = 0;
    for (int j = 0; j < nj; ++j) {
      if (gl[j].t_s < tmin) {
        tmin = gl[j].t_s;
        imin = j;
      }
      tmax = std::max(tmax, gl[j].t_s);
    }
    const double Tms = (tmax - tmin) * 1000.0;
    std::vector<double> tau(nj);
    for (int j = 0; j < nj; ++j) tau[j] = std::min(Tms, std::max(0.0, (gl[j].t_s - tmin) * 1000.0));
    // relaxation as e^{A_c - d_c tau}: trf and the T2' clock are affine in tau within a group
    const double trf0 = gl[imin].trf, inh0 = gl[imin].inh;
    double sigma = 1.0;
    if (acq.echo == MRSIM_ECHO_SPIN && tmin < 0) sigma = -1.0;
    for (int j = 0; j < nj; ++j) {
      if (std::fabs(gl[j].trf - (trf0 + tau[j])) > 1e-6 || std::fabs(gl[j].inh - (inh0 + sigma * tau[j])) > 1e-6)
        fail("the segmented path needs line times affine within an echo");
    }
    double dc[kMaxComp] = {0}, Ac[kMaxComp] = {0};
    for (int c = 0; c < ncomp; ++c) {
      if (acq.do_relaxation) {
        const double t2 = (double)op.t2u[c], ti = (double)op.tiu[c];
        const bool spin = acq.echo == MRSIM_ECHO_SPIN;
        dc[c] = 1.0 / t2 + (spin ? sigma : 1.0) / ti;
        Ac[c] = -trf0 / t2 - inh0 / ti;
      }
    }
    double dlo = dc[0], dhi = dc[0];
    for (int c = 1; c < ncomp; ++c) {
      dlo = std::min(dlo, dc[c]);
      dhi = std::max(dhi, dc[c]);
    }
    // the certified segmentation (one node when the group is a single instant)
    TsegPlan plan;
    if (Tms <= 0.0 || nj == 1) {
      plan.l = 1;
      plan.tau_l = {0.0};
      plan.b.assign((size_t)nj * 2, 0.0);
      for (int j = 0; j < nj; ++j) plan.b[2 * j] = 1.0;
      plan.bound = 0.0;
    } else {
      const double d[2] = {0.0, dhi - dlo}, f[2] = {fmin, fmax};
      plan = tseg_plan(tau, Tms, d, f, &fitdev);
    }
    if (plan.l > kTsMaxL) fail("the segmented path supports at most 32 segments per group");
    G.L = plan.l;
    G.Lp = (plan.l + 3) / 4 * 4;
    T.L.push_back(plan.l);
    T.bound.push_back(plan.bound);
    for (int l = 0; l < G.Lp; ++l) {
      const double tl = l < plan.l ? plan.tau_l[l] : plan.tau_l[plan.l - 1];
      const double tb = gl[imin].tb0 + tl / 1000.0;
      G.t_hi[l] = (float)tb;
      G.t_lo[l] = (float)(tb - (double)G.t_hi[l]);
      for (int c = 0; c < kMaxComp; ++c)
        G.alpha[l][c] = (c < ncomp && l < plan.l) ? (float)std::exp(Ac[c] - (dc[c] - dlo) * tl) : 0.f;
    }
    for (int j = 0; j < nj; ++j) G.lines[j] = gl[j].idx;
    G.np_f = std::max(16, (nj * na * 2 + 15) / 16 * 16);
    G.kb_f = (sny / 8) * (G.Lp / 4);
    G.kp_a = std::max(64, (nj * na * 2 + 63) / 64 * 64);
    G.ka0 = ka;
    ka += G.kp_a;
    np_max_f = std::max(np_max_f, G.np_f);
    L_min_yc = std::min(L_min_yc, 256 / (2 * G.Lp));
    // the complex table B[(l, y)][(j, v)] = sv ey_v(y) e^{i2pi kr_j(y)} b_l(tau_j) w_j
    auto& br = bre[g];
    auto& bi = bim[g];
    br.assign((size_t)G.Lp * sny * nj * na, 0.0);
    bi.assign(br.size(), 0.0);
    for (int j = 0; j < nj; ++j) {
      const double w = std::exp(-dlo * tau[j]);
      const long long K = gl[j].ky - ys;
      for (int y = 0; y < sny; ++y) {
        const long long Y = 2LL * (y - sys) - (oy - 1);
        double tv = (double)((K * Y) % m2) / (double)m2;
        tv -= std::rint(tv);
        const double er = std::cos(kTau * tv), ei = std::sin(kTau * tv);
        for (int l = 0; l < plan.l; ++l) {
          const double pr = plan.b[((size_t)j * plan.l + l) * 2], pi = plan.b[((size_t)j * plan.l + l) * 2 + 1];
          const double cr = (er * pr - ei * pi) * w, ci = (er * pi + ei * pr) * w;
          for (int v = 0; v < na; ++v) {
            const double ey = v < ncls ? (double)eyc[(size_t)v * sny + y] : 1.0;
            const size_t o = (((size_t)l * sny + y) * nj + j) * na + v;
            br[o] = ey * cr;
            bi[o] = ey * ci;
          }
        }
      }
    }
    T.flops_fwd += 2.0 * 128.0 * (double)G.np_f * (double)G.kb_f * 64.0 * 3.0;
  }
  T.np_max_f = np_max_f;
  T.kp_total = ka;
  int yc = 8;
  while (yc > 2 && yc > L_min_yc) yc /= 2;
  if (yc > L_min_yc || sny % yc) fail("the segmented path found no y chunk for these segment counts");
  T.yc = yc;
  T.nyc = sny / yc;
  int np_max_a = 16;
  for (auto& G : T.groups_h) {
    G.yc = yc;
    G.np_a = yc * G.Lp * 2;
    np_max_a = std::max(np_max_a, G.np_a);
    T.flops_adj += 2.0 * 128.0 * (double)G.np_a * (double)G.kp_a * 3.0 * T.nyc;
  }
  T.np_max_a = np_max_a;
  T.snx_tiles = (snx + 127) / 128;
  T.snx_pad = T.snx_tiles * 128;
  const double units = (double)ep.n_units * T.snx_tiles;
  T.flops_fwd *= units;
  T.flops_adj *= units;

  // ---- split 16-bit tables in the K-major layouts the kernels load ----------------------------
  DevArena& A = T.arena;
  std::vector<void*> fwd_tabs(T.n_groups), adj_tabs(T.n_groups);
  for (int g = 0; g < T.n_groups; ++g) {
    TsGroupDev& G = T.groups_h[g];
    const int nj = G.n_j, Lp = G.Lp;
    const auto& br = bre[g];
    const auto& bi = bim[g];
    // forward: rows n = (j NA + v) 2 + ro (hi rows, then lo rows), K = kb 64 + (l % 4) 16 + yy 2 + ri
    const size_t Kf = (size_t)G.kb_f * 64;
    double mxf = 0;
    for (size_t i = 0; i < br.size(); ++i) mxf = std::max(mxf, std::max(std::fabs(br[i]), std::fabs(bi[i])) * sig *
                                                                    std::max(1.0, off));
    const double tsf = pow2_scale(mxf);
    G.out_scale_f = (float)(1.0 / tsf);
    std::vector<uint16_t> tf((size_t)2 * G.np_f * Kf, 0);
    for (int j = 0; j < nj; ++j)
      for (int v = 0; v < na; ++v) {
        const double sv = sig * (v == na - 1 ? off : 1.0) * tsf;
        for (int y = 0; y < sny; ++y)
          for (int l = 0; l < Lp; ++l) {
            const size_t o = (((size_t)l * sny + y) * nj + j) * na + v;
            const double cr = br[o] * sv, ci = bi[o] * sv;
            const size_t kb = (size_t)(y / 8) * (Lp / 4) + l / 4;
            const size_t k = kb * 64 + (l % 4) * 16 + (y % 8) * 2;
            const double e[2][2] = {{cr, -ci}, {ci, cr}};  // [ro][ri]
            for (int ro = 0; ro < 2; ++ro)
              for (int ri = 0; ri < 2; ++ri) {
                const size_t n = (size_t)(j * na + v) * 2 + ro;
                const uint16_t hi = to16(e[ro][ri], dt);
                tf[n * Kf + k + ri] = hi;
                tf[((size_t)G.np_f + n) * Kf + k + ri] = to16(e[ro][ri] - from16(hi, dt), dt);
              }
          }
      }
    fwd_tabs[g] = A.upload(tf.data(), tf.size() * 2, st);
    T.fmaps.push_back(make_map(fwd_tabs[g], dt, Kf, (uint64_t)2 * G.np_f, (uint32_t)G.np_f));
    // adjoint: per y chunk, rows n = (yy Lp + l) 2 + ro (hi rows, then lo rows), K = (j NA + v) 2 + ri
    double mxa = 0;
    for (size_t i = 0; i < br.size(); ++i) mxa = std::max(mxa, std::max(std::fabs(br[i]), std::fabs(bi[i])));
    const double tsa = pow2_scale(mxa);
    for (int l = 0; l < kTsMaxL; ++l)
      for (int c = 0; c < kMaxComp; ++c) G.alpha_adj[l][c] = (float)(G.alpha[l][c] / tsa);
    const size_t Ka = (size_t)G.kp_a;
    std::vector<uint16_t> ta((size_t)T.nyc * 2 * G.np_a * Ka, 0);
    for (int ycx = 0; ycx < T.nyc; ++ycx)
      for (int yy = 0; yy < yc; ++yy) {
        const int y = ycx * yc + yy;
        for (int l = 0; l < Lp; ++l)
          for (int j = 0; j < nj; ++j)
            for (int v = 0; v < na; ++v) {
              const size_t o = (((size_t)l * sny + y) * nj + j) * na + v;
              const double cr = br[o] * tsa, ci = -bi[o] * tsa;  // conj
              const double e[2][2] = {{cr, -ci}, {ci, cr}};     // [ro][ri]
              const size_t k = (size_t)(j * na + v) * 2;
              for (int ro = 0; ro < 2; ++ro)
                for (int ri = 0; ri < 2; ++ri) {
                  const size_t n = (size_t)(yy * Lp + l) * 2 + ro;
                  const uint16_t hi = to16(e[ro][ri], dt);
                  ta[((size_t)(ycx * 2) * G.np_a + n) * Ka + k + ri] = hi;
                  ta[((size_t)(ycx * 2 + 1) * G.np_a + n) * Ka + k + ri] = to16(e[ro][ri] - from16(hi, dt), dt);
                }
            }
      }
    adj_tabs[g] = A.upload(ta.data(), ta.size() * 2, st);
    T.amaps.push_back(make_map(adj_tabs[g], dt, Ka, (uint64_t)T.nyc * 2 * G.np_a, (uint32_t)G.np_a));
  }
  // compartment-wise largest alpha (the f16 input scale)
  for (int c = 0; c < kMaxComp; ++c) {
    T.amax.v[c] = 0.f;
    for (auto& G : T.groups_h)
      for (int l = 0; l < G.L; ++l) T.amax.v[c] = std::max(T.amax.v[c], G.alpha[l][c]);
  }
  T.d_groups = (TsGroupDev*)A.upload(T.groups_h.data(), T.groups_h.size() * sizeof(TsGroupDev), st);
  const size_t nu = (size_t)ep.n_units;
  T.d_scale_f = (float*)A.alloc(nu * 4);
  T.d_scale_a = (float*)A.alloc(nu * 4);
  T.d_gs_hi = (uint16_t*)A.alloc(nu * T.snx_pad * (size_t)T.kp_total * 2);
  T.d_gs_lo = (uint16_t*)A.alloc(nu * T.snx_pad * (size_t)T.kp_total * 2);
  T.gs_hi_map = make_map(T.d_gs_hi, dt, (uint64_t)T.kp_total, (uint64_t)nu * T.snx_pad, 128);
  T.gs_lo_map = make_map(T.d_gs_lo, dt, (uint64_t)T.kp_total, (uint64_t)nu * T.snx_pad, 128);
  T.fwd_cls = ep.fwd_cls;
  T.adj_cls = ep.adj_cls;
  if (!T.fwd_cls) {
    T.cls_stride = (long long)na * op.n_lines * snx;
    T.d_cls = (float2*)A.alloc(nu * (size_t)T.cls_stride * sizeof(float2));
  }
  T.d_err = (int*)A.alloc(sizeof(int));
  MRSIM_CUDA(cudaMemsetAsync(T.d_err, 0, sizeof(int), st));
  int dev = 0;
  MRSIM_CUDA(cudaGetDevice(&dev));
  MRSIM_CUDA(cudaDeviceGetAttribute(&T.n_sms, cudaDevAttrMultiProcessorCount, dev));
  MRSIM_CUDA(cudaStreamSynchronize(st));
  return tp.release();
}

namespace {
template <class K>
void opt_in(K kernel, size_t bytes) {
  MRSIM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}
// bytes of dynamic shared memory: alignment slack, A and B stages, barriers, the node table
size_t ts_smem(int np_max, int b_stages, int n_groups) {
  return 1024 + (size_t)kStages * kStageA + (size_t)b_stages * 2 * np_max * 128 + 16 * 8 + 16 +
         (size_t)n_groups * kTsMaxL * kNodeFloats * 4;
}
constexpr size_t kSmemLimit = 232448;  // 227 KB per CTA
}  // namespace

void ts_forward_ystage(const TsPlan& T, const EpiPlan& ep, cudaStream_t st, int u0, int u1) {
  if (u1 < 0) u1 = ep.n_units;
  const int nu = u1 - u0;
  if (nu <= 0) return;
  if (T.dt == 0) ts_scale_kernel<<<nu, 256, 0, st>>>(ep.d_units, u0, T.amax, T.d_scale_f);
  TsFwdParams P;
  std::memset(&P, 0, sizeof P);
  for (int g = 0; g < T.n_groups; ++g) P.bmap[g] = T.fmaps[g];
  P.units = ep.d_units;
  P.groups = T.d_groups;
  P.unit_scale = T.dt == 0 ? T.d_scale_f : nullptr;
  P.cls_out = T.fwd_cls ? nullptr : T.d_cls;
  P.cls_unit_stride = T.cls_stride;
  P.err = T.d_err;
  P.n_items = nu * T.snx_tiles;
  P.n_groups = T.n_groups;
  P.na = T.na;
  P.snx_tiles = T.snx_tiles;
  P.np_max = T.np_max_f;
  P.u0 = u0;
  P.b_stages = ts_smem(T.np_max_f, 3, T.n_groups) <= kSmemLimit ? 3 : 2;
  const size_t sm = ts_smem(T.np_max_f, P.b_stages, T.n_groups);
  const unsigned grid = (unsigned)std::min(P.n_items, T.n_sms);
  const int nc = ep.nc;
#define MRSIM_TSF(DT, NC)                           \
  {                                                 \
    auto k = ts_forward_kernel<DT, NC>;             \
    opt_in(k, sm);                                  \
    k<<<grid, 448, sm, st>>>(P);                    \
  }
  if (T.dt == 0) {
    if (nc <= 1) MRSIM_TSF(0, 1) else if (nc == 2) MRSIM_TSF(0, 2) else if (nc == 3) MRSIM_TSF(0, 3) else MRSIM_TSF(0, 4)
  } else {
    if (nc <= 1) MRSIM_TSF(1, 1) else if (nc == 2) MRSIM_TSF(1, 2) else if (nc == 3) MRSIM_TSF(1, 3) else MRSIM_TSF(1, 4)
  }
#undef MRSIM_TSF
  MRSIM_CUDA(cudaGetLastError());
  if (!T.fwd_cls) {
    dim3 g2((unsigned)std::min(64, (ep.max_lines * ep.max_snx + 255) / 256), (unsigned)nu);
    ts_expand_kernel<<<g2, 256, 0, st>>>(ep.d_units, u0, T.na, T.d_cls, T.cls_stride);
    MRSIM_CUDA(cudaGetLastError());
  }
}

void ts_adjoint_ystage(const TsPlan& T, const EpiPlan& ep, cudaStream_t st, int u0, int u1) {
  if (u1 < 0) u1 = ep.n_units;
  const int nu = u1 - u0;
  if (nu <= 0) return;
  TsConvParams C;
  std::memset(&C, 0, sizeof C);
  C.units = ep.d_units;
  C.groups = T.d_groups;
  C.unit_scale = T.d_scale_a;
  C.gs_hi = T.d_gs_hi;
  C.gs_lo = T.d_gs_lo;
  C.n_groups = T.n_groups;
  C.na = T.na;
  C.kp_total = T.kp_total;
  C.snx_pad = T.snx_pad;
  C.class_rows = T.adj_cls ? 1 : 0;
  C.u0 = u0;
  if (T.dt == 0)
    ts_gconvert_kernel<0><<<nu, 256, 0, st>>>(C);
  else
    ts_gconvert_kernel<1><<<nu, 256, 0, st>>>(C);
  MRSIM_CUDA(cudaGetLastError());
  TsAdjParams P;
  std::memset(&P, 0, sizeof P);
  P.amap_hi = T.gs_hi_map;
  P.amap_lo = T.gs_lo_map;
  for (int g = 0; g < T.n_groups; ++g) P.bmap[g] = T.amaps[g];
  P.units = ep.d_units;
  P.groups = T.d_groups;
  P.unit_scale = T.d_scale_a;
  P.err = T.d_err;
  P.n_items = nu * T.snx_tiles;
  P.n_groups = T.n_groups;
  P.snx_tiles = T.snx_tiles;
  P.snx_pad = T.snx_pad;
  P.np_max = T.np_max_a;
  P.nyc = T.nyc;
  P.yc = T.yc;
  P.u0 = u0;
  const size_t sm = ts_smem(T.np_max_a, kStages, T.n_groups);
  const unsigned grid = (unsigned)std::min(P.n_items, T.n_sms);
  const int nc = ep.nc;
#define MRSIM_TSA(DT, NC)                           \
  {                                                 \
    auto k = ts_adjoint_kernel<DT, NC>;             \
    opt_in(k, sm);                                  \
    k<<<grid, 320, sm, st>>>(P);                    \
  }
  if (T.dt == 0) {
    if (nc <= 1) MRSIM_TSA(0, 1) else if (nc == 2) MRSIM_TSA(0, 2) else if (nc == 3) MRSIM_TSA(0, 3) else MRSIM_TSA(0, 4)
  } else {
    if (nc <= 1) MRSIM_TSA(1, 1) else if (nc == 2) MRSIM_TSA(1, 2) else if (nc == 3) MRSIM_TSA(1, 3) else MRSIM_TSA(1, 4)
  }
#undef MRSIM_TSA
  MRSIM_CUDA(cudaGetLastError());
}

int ts_error(const TsPlan& T, cudaStream_t st) {
  int e = 0;
  MRSIM_CUDA(cudaMemcpyAsync(&e, T.d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MRSIM_CUDA(cudaStreamSynchronize(st));
  return e;
}

}  // namespace mrsim
