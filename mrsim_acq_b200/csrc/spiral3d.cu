// spiral3d.cu — the 3D stack-of-spirals acquisition on the device (reference `spiral_volumes`,
// kspace3d.rs:1472-1569, with `SpiralPlan` :907-1067, `spiral_plan` :1069-1137,
// `coil_row_sensitivity` :1139-1150, `pocs_along_z` :1201-1259, `KzGrappa` :1261-1389,
// `spiral_noise` :1391-1404, `kz_calibrate` :1406-1439; the tables `spiral_lines` /
// `spiral_kz_order` / `KzSampling`, readout.rs:107-160, 653-700).
//
// Per volume and slice, one batch of segment images (every coil element x compartment source x
// segment), one batched type-2 NUFFT and one combination kernel give every element's samples;
// one kernel forms the z-DFT with the rings' z profiles, echo amplitudes and line weights for
// every coil; the noise runs on the (volume, partition, coil) streams; the kz GRAPPA kernel is
// fitted once (normal equations accumulated and solved in FP64 on the device) and
// applied by one kernel; the inverse z-DFT feeds the FP64 spiral reconstruction of every slice.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <map>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "driver.h"
#include "hermitian_solve.cuh"
#include "host3d.h"
#include "host_tables.h"
#include "mrsim_internal.h"
#include "noise_kernels.h"
#include "nufft.h"
#include "spiral.h"
#include "spiral3d.h"
#include "spiral_host.h"
#include "spiral_recon.h"

namespace mrsim {

// ---- tables -----------------------------------------------------------------------------------------
int kz_band_start(const mrsim_kz_sampling& kz, int nz) {  // readout.rs:128-142
  if (!(std::isfinite(kz.partial_fourier) && kz.partial_fourier > 0.5 && kz.partial_fourier <= 1.0)) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "partial Fourier along kz must be in (0.5, 1], got %g", kz.partial_fourier);
    fail(buf);
  }
  if (kz.accel < 1) fail("the kz acceleration must be at least 1");
  const int kept = std::min(nz, (int)std::round((double)nz * kz.partial_fourier));
  return nz - kept;
}

std::vector<uint8_t> kz_acquired(const mrsim_kz_sampling& kz, int nz) {  // readout.rs:145-150
  const int lo = kz_band_start(kz, nz), c = nz / 2;
  std::vector<uint8_t> a(nz);
  for (int p = 0; p < nz; ++p) {
    const int64_t r = ((int64_t)(p - c) % kz.accel + kz.accel) % kz.accel;
    a[p] = p >= lo && r == 0;
  }
  return a;
}

Spiral3dTable spiral_lines(const mrsim_echo_train& train, const mrsim_spiral_readout& ro, int nx, int ny, int nz) {
  Spiral3dTable T;
  T.traj = spiral_trajectory(nx, ny, (int)ro.interleaves, ro.readout_ms, ro.dwell_ms, ro.radial_oversampling);
  T.acquired = kz_acquired(ro.kz, nz);
  T.band_start = kz_band_start(ro.kz, nz);
  std::vector<int> order;
  for (int p : kz_order(nz, train.kz_order))
    if (T.acquired[p]) order.push_back(p);
  const bool full = ro.kz.partial_fourier >= 1.0 && ro.kz.accel <= 1;
  char buf[320];
  if (train.kz_segments <= 0 || order.size() % (size_t)train.kz_segments != 0) {
    if (full)
      std::snprintf(buf, sizeof buf, "%d partitions do not divide into %lld kz segments", nz, (long long)train.kz_segments);
    else
      std::snprintf(buf, sizeof buf,
                    "the %zu partitions read (of %d: partial Fourier %g and acceleration %lld along kz) do not divide "
                    "into %lld kz segments",
                    order.size(), nz, ro.kz.partial_fourier, (long long)ro.kz.accel, (long long)train.kz_segments);
    fail(buf);
  }
  if ((size_t)train.etl != order.size() / (size_t)train.kz_segments) {
    if (full)
      std::snprintf(buf, sizeof buf, "echo train length %lld is not %d partitions / %lld kz segments",
                    (long long)train.etl, nz, (long long)train.kz_segments);
    else
      std::snprintf(buf, sizeof buf, "echo train length %lld is not the %zu partitions read (of %d) / %lld kz segments",
                    (long long)train.etl, order.size(), nz, (long long)train.kz_segments);
    fail(buf);
  }
  T.nz = nz;
  T.echo.assign(nz, 0);
  T.kz_segment.assign(nz, 0);
  for (size_t n = 0; n < order.size(); ++n) {
    T.echo[order[n]] = (int)(n / (size_t)train.kz_segments) + 1;
    T.kz_segment[order[n]] = (int)(n % (size_t)train.kz_segments);
  }
  T.kz_segments = (int)train.kz_segments;
  T.e_c = T.echo[nz / 2];
  T.n_shots = (int)ro.interleaves * (int)train.kz_segments;
  return T;
}

double coil_row_sensitivity(int row, int rows, double z, int nz) {  // kspace3d.rs:1139-1150
  if (rows <= 1) return 1.0;
  const double centre = (double)nz * ((double)row + 0.5) / (double)rows - 0.5;
  const double sigma = 0.6 * (double)nz / (double)rows;
  return std::exp(-(z - centre) * (z - centre) / (2.0 * sigma * sigma)) + 0.15;
}

namespace {

constexpr uint64_t kSeedSaltKzcal = 0x4B5A43414C00ull;  // "KZCAL" (kspace3d.rs:1171)
constexpr double kKzLambda = 1e-8;
constexpr int kKzSources = 4;
constexpr int kPocsIterations = 10;

// ---- kernels ------------------------------------------------------------------------------------------
struct SegSlot {
  const float* comp;     // compartment plane (this volume, this slice)
  const float* la;       // ln A_e plane (voxel sources) or NULL
  const float* decay;    // 1/T2 + 1/T2' plane (voxel sources) or NULL
  const float* amp;      // signal_scale x element sensitivity
  int plan;              // 0 class, 1 voxel
  int pad;
};

// seg[slot][l][i] = amp m [e^{ln A}] cis(phi0) e^{-d tau_l} cis(2 pi f tau_l / 1000)
__global__ void seg_images_kernel(const SegSlot* __restrict__ slots, const float2* __restrict__ cis0,
                                  const float* __restrict__ fmap, const double* __restrict__ tau_l0,
                                  const double* __restrict__ tau_l1, int L0, int L1, int nvox,
                                  float2* __restrict__ out, const int* __restrict__ slot_base) {
  const int s = blockIdx.y;
  const SegSlot S = slots[s];
  const int L = S.plan ? L1 : L0;
  const double* tl = S.plan ? tau_l1 : tau_l0;
  float2* o = out + (size_t)slot_base[s] * nvox;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nvox; i += gridDim.x * blockDim.x) {
    float a = S.amp[i] * S.comp[i];
    if (S.la) a *= __expf(S.la[i]);
    const float2 c0 = cis0[i];
    const float2 x = make_float2(c0.x * a, c0.y * a);
    const float d = S.decay ? S.decay[i] : 0.f;
    const float f = fmap ? fmap[i] : 0.f;
    for (int l = 0; l < L; ++l) {
      const double t = tl[l];
      const float mag = __expf(-d * (float)t);
      double th = (double)f * t / 1000.0;
      th -= rint(th);
      float sn, cs;
      sincospif(2.0f * (float)th, &sn, &cs);
      const float er = mag * cs, ei = mag * sn;
      o[(size_t)l * nvox + i] = make_float2(x.x * er - x.y * ei, x.x * ei + x.y * er);
    }
  }
}

// k2[slot][j] = stat_j sum_l b[j % ns][l] seg_out[slot][l][j]
__global__ void seg_combine_kernel(const float2* __restrict__ seg, const int* __restrict__ slot_base,
                                   const int* __restrict__ slot_plan, const double* __restrict__ b0,
                                   const double* __restrict__ b1, int L0, int L1, int ns, int nsamp,
                                   const float2* __restrict__ stat, float2* __restrict__ k2,
                                   const size_t* __restrict__ k2_off) {
  const int s = blockIdx.y;
  const int plan = slot_plan[s];
  const int L = plan ? L1 : L0;
  const double* b = plan ? b1 : b0;
  const float2* sg = seg + (size_t)slot_base[s] * nsamp;
  float2* out = k2 + k2_off[s];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nsamp; j += gridDim.x * blockDim.x) {
    const double* bj = b + (size_t)(j % ns) * L * 2;
    float re = 0.f, im = 0.f;
    for (int l = 0; l < L; ++l) {
      const float2 v = sg[(size_t)l * nsamp + j];
      const float br = (float)bj[2 * l], bi = (float)bj[2 * l + 1];
      re += br * v.x - bi * v.y;
      im += br * v.y + bi * v.x;
    }
    const float2 st = stat[j];
    out[j] = make_float2(re * st.x - im * st.y, re * st.y + im * st.x);
  }
}

struct ZArgs {
  const float2* k2;       // [a][src][z][nsamp]
  float2* out;            // [q][p][nsamp]
  const float2* zkq;      // [row][p][z]
  const int* src;         // [c][p]
  const float* wc;        // [c][p][ns]
  const float* lw;        // [g][shot][c] or NULL
  const int* kzseg;       // [p]
  const unsigned char* acquired;  // [p]
  const int* shot_var;    // [shot]: the image variant the shot saw (0: the volume's own), or NULL
  int nz, nsamp, ns, ncomp, nsrc, ring, kz_segments, n_shots, g;
};

// coil q = r ring + a: out[q][p][j] = sum_c lw (w_c sum_z k2[var(shot)][a][src][z][j] zkq[r][p][z]), var
// the images the sample's shot saw (`samples_rings` kspace3d.rs:1028-1051)
__global__ void spiral_zdft_kernel(const ZArgs a) {
  const int p = blockIdx.y, q = blockIdx.z;
  const int r = q / a.ring, e = q % a.ring;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < a.nsamp; j += gridDim.x * blockDim.x) {
    float2 v = make_float2(0.f, 0.f);
    if (a.acquired[p]) {
      const int shot = (j / a.ns) * a.kz_segments + a.kzseg[p];
      for (int c = 0; c < a.ncomp; ++c) {
        const int s = a.src[c * a.nz + p];
        const int var = a.shot_var ? a.shot_var[shot] : 0;
        const float2* K = a.k2 + ((size_t)((var * a.ring + e) * a.nsrc + s) * a.nz) * a.nsamp + j;
        float ar = 0.f, ai = 0.f;
        for (int z = 0; z < a.nz; ++z) {
          const float2 k = K[(size_t)z * a.nsamp];
          const float2 w = a.zkq[((size_t)r * a.nz + p) * a.nz + z];
          ar += k.x * w.x - k.y * w.y;
          ai += k.x * w.y + k.y * w.x;
        }
        const float wc = a.wc[((size_t)c * a.nz + p) * a.ns + j % a.ns];
        ar *= wc;
        ai *= wc;
        const float l = a.lw ? a.lw[((size_t)a.g * a.n_shots + shot) * a.ncomp + c] : 1.f;
        v.x += ar * l;
        v.y += ai * l;
      }
    }
    a.out[((size_t)q * a.nz + p) * a.nsamp + j] = v;
  }
}

// FP64 normal equations of the kz kernel: G = F^H [F | B] over rows (t, j); F rows are the
// sources' samples of every coil, B the targets'.  One CTA accumulates a block of rows into a
// partial [nfeat][nfeat + nc] result; partials are summed on the host in a fixed order.
struct KzFitArgs {
  const float2* k;     // [q][p][nsamp] calibration samples
  const int* t_list;   // target partitions with every source in the band
  const int* offs;     // nsrc offsets
  int n_t, nsrc, nc, nz, nsamp;
  double2* partial;    // [block][nfeat][nfeat + nc]
};

__global__ void __launch_bounds__(256) kz_normal_kernel(const KzFitArgs a) {
  extern __shared__ __align__(16) unsigned char kz_smem[];
  const int nfeat = a.nsrc * a.nc, ncol = nfeat + a.nc;
  constexpr int kRows = 16;
  double2* fr = reinterpret_cast<double2*>(kz_smem);  // [kRows][ncol]
  const long long total = (long long)a.n_t * a.nsamp;
  const int nent = nfeat * ncol;
  constexpr int kPer = 24;  // entries per thread (nfeat <= 64, nc <= 64: 64 x 128 / 256 = 32 max)
  double2 acc[kPer];
#pragma unroll
  for (int e = 0; e < kPer; ++e) acc[e] = make_double2(0.0, 0.0);
  for (long long r0 = (long long)blockIdx.x * kRows; r0 < total; r0 += (long long)gridDim.x * kRows) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < kRows * ncol; idx += blockDim.x) {
      const int rr = idx / ncol, col = idx % ncol;
      const long long row = r0 + rr;
      double2 v = make_double2(0.0, 0.0);
      if (row < total) {
        const int t = a.t_list[row / a.nsamp];
        const int j = (int)(row % a.nsamp);
        int p, q;
        if (col < nfeat) {
          p = t + a.offs[col / a.nc];
          q = col % a.nc;
        } else {
          p = t;
          q = col - nfeat;
        }
        const float2 s = a.k[((size_t)q * a.nz + p) * a.nsamp + j];
        v = make_double2((double)s.x, (double)s.y);
      }
      fr[rr * ncol + col] = v;
    }
    __syncthreads();
    for (int e = 0; e < kPer; ++e) {
      const int ent = threadIdx.x + e * blockDim.x;
      if (ent >= nent) break;
      const int i = ent / ncol, jj = ent % ncol;
      double re = acc[e].x, im = acc[e].y;
      for (int rr = 0; rr < kRows; ++rr) {
        const double2 fi = fr[rr * ncol + i], fj = fr[rr * ncol + jj];
        re = fma(fi.x, fj.x, fma(fi.y, fj.y, re));  // conj(fi) fj
        im = fma(fi.x, fj.y, fma(-fi.y, fj.x, im));
      }
      acc[e] = make_double2(re, im);
    }
  }
  for (int e = 0; e < kPer; ++e) {
    const int ent = threadIdx.x + e * blockDim.x;
    if (ent >= nent) break;
    a.partial[(size_t)blockIdx.x * nent + ent] = acc[e];
  }
}

// The kz kernel's system (`KzGrappa::fit`, kspace3d.rs:1299-1362): the blocks' partial normal
// equations summed in block order, scaled by nfeat / trace, the Tikhonov term added to the
// diagonal, then every target coil's weights by pivoted elimination (hermitian_solve.cuh).  One
// CTA; status 1 when the trace is not positive (an empty calibration).
struct KzSolveArgs {
  const double2* partial;  // [blocks][nfeat][ncol], ncol = nfeat + nc
  double2* W;              // [nfeat][ncol]
  double* scratch;         // 2 nfeat + nc * 2 nfeat
  float2* out;             // [nc][nfeat]
  int* status;
  double lambda;
  int blocks, nfeat, nc;
};

__global__ void __launch_bounds__(256) kz_solve_kernel(const KzSolveArgs a) {
  __shared__ double red_v[256];
  __shared__ int red_i[256];
  __shared__ double s_scale;
  __shared__ int s_bad;
  const int nf = a.nfeat, ncol = nf + a.nc;
  const size_t n_el = (size_t)nf * ncol;
  for (size_t e = threadIdx.x; e < n_el; e += blockDim.x) {
    double2 g = make_double2(0.0, 0.0);
    for (int b = 0; b < a.blocks; ++b) {
      const double2 p = a.partial[(size_t)b * n_el + e];
      g.x = __dadd_rn(g.x, p.x);
      g.y = __dadd_rn(g.y, p.y);
    }
    a.W[e] = g;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double trace = 0.0;
    for (int i = 0; i < nf; ++i) trace = __dadd_rn(trace, a.W[(size_t)i * ncol + i].x);
    s_bad = !(trace > 0.0);
    s_scale = s_bad ? 0.0 : __ddiv_rn((double)nf, trace);
    if (s_bad) *a.status = 1;
  }
  __syncthreads();
  if (s_bad) return;
  const double sc = s_scale;
  for (size_t e = threadIdx.x; e < n_el; e += blockDim.x) {
    double2 v = a.W[e];
    v.x = __dmul_rn(v.x, sc);
    v.y = __dmul_rn(v.y, sc);
    if ((int)(e / ncol) == (int)(e % ncol)) v.x = __dadd_rn(v.x, a.lambda);
    a.W[e] = v;
  }
  __syncthreads();
  hermitian_solve_block(a.W, nf, a.nc, a.scratch, a.scratch + nf, a.scratch + 2 * nf, a.out, red_v, red_i);
}

struct KzFillJob {
  int p, nsrc, woff, pad;
  int src[kKzSources];
};

// k[qt][p][j] = sum_s sum_qs w[qt][s nc + qs] k[qs][src_s][j]
__global__ void kz_fill_kernel(float2* __restrict__ k, const KzFillJob* __restrict__ jobs,
                               const float2* __restrict__ w, int nc, int nz, int nsamp) {
  const KzFillJob J = jobs[blockIdx.y];
  const int qt = blockIdx.z;
  const int nfeat = J.nsrc * nc;
  const float2* W = w + J.woff + (size_t)qt * nfeat;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nsamp; j += gridDim.x * blockDim.x) {
    float re = 0.f, im = 0.f;
    for (int s = 0; s < J.nsrc; ++s)
      for (int qs = 0; qs < nc; ++qs) {
        const float2 wv = W[s * nc + qs];
        const float2 v = k[((size_t)qs * nz + J.src[s]) * nsamp + j];
        re += wv.x * v.x - wv.y * v.y;
        im += wv.x * v.y + wv.y * v.x;
      }
    k[((size_t)qt * nz + J.p) * nsamp + j] = make_float2(re, im);
  }
}

// slices[z][q][j] = (1/nz) sum_p k[q][p][j] conj(zk[p][z])   (FP64 out for the reconstruction)
__global__ void spiral_izdft_kernel(const float2* __restrict__ k, const float2* __restrict__ zk, int nz, int nc,
                                    int nsamp, double2* __restrict__ out) {
  const int z = blockIdx.y, q = blockIdx.z;
  const float inv = 1.0f / (float)nz;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nsamp; j += gridDim.x * blockDim.x) {
    float ar = 0.f, ai = 0.f;
    for (int p = 0; p < nz; ++p) {
      const float2 v = k[((size_t)q * nz + p) * nsamp + j];
      const float2 e = zk[p * nz + z];
      ar += v.x * e.x + v.y * e.y;
      ai += v.y * e.x - v.x * e.y;
    }
    out[((size_t)z * nc + q) * nsamp + j] = make_double2((double)(ar * inv), (double)(ai * inv));
  }
}

// samples of partitions p >= lo, f32 -> FP64 in [q][p][nsamp] order for the per-partition images
__global__ void to_double_kernel(const float2* __restrict__ in, size_t n, double2* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = make_double2((double)in[i].x, (double)in[i].y);
}

// POCS along z (`pocs_along_z` kspace3d.rs:1201-1259) per (coil, in-plane voxel); h [q][p][nn]
// (zero below lo), out [q][z][nn]; zk FP64 [p][z].
__global__ void pocs_kernel(const double2* __restrict__ h, int lo, const double2* __restrict__ zk, int nz, int nn,
                            int nc, double2* __restrict__ out) {
  const int q = blockIdx.y;
  const int c = nz / 2;
  const int m = min(c - lo, nz - 1 - c);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    double2 k[64], unit[64], x[64];
    for (int p = 0; p < nz; ++p) k[p] = p >= lo ? h[((size_t)q * nz + p) * nn + i] : make_double2(0.0, 0.0);
    for (int z = 0; z < nz; ++z) {  // the low-resolution image's phase
      double re = 0.0, im = 0.0;
      for (int p = 0; p < nz; ++p) {
        const double d = fabs((double)p - (double)c);
        const double hw = d > (double)m ? 0.0 : 0.5 * (1.0 + cos(3.141592653589793 * d / ((double)m + 1.0)));
        const double2 lv = make_double2(k[p].x * hw, k[p].y * hw);
        const double2 e = zk[p * nz + z];
        re += lv.x * e.x + lv.y * e.y;
        im += lv.y * e.x - lv.x * e.y;
      }
      re /= nz;
      im /= nz;
      const double a = hypot(re, im);
      unit[z] = a > 0.0 ? make_double2(re / a, im / a) : make_double2(1.0, 0.0);
    }
    for (int it = 0; it < kPocsIterations; ++it) {
      for (int z = 0; z < nz; ++z) {
        double re = 0.0, im = 0.0;
        for (int p = 0; p < nz; ++p) {
          const double2 e = zk[p * nz + z];
          re += k[p].x * e.x + k[p].y * e.y;
          im += k[p].y * e.x - k[p].x * e.y;
        }
        const double a = hypot(re / nz, im / nz);
        x[z] = make_double2(unit[z].x * a, unit[z].y * a);
      }
      for (int p = 0; p < lo; ++p) {
        double re = 0.0, im = 0.0;
        for (int z = 0; z < nz; ++z) {
          const double2 e = zk[p * nz + z];
          re += x[z].x * e.x - x[z].y * e.y;
          im += x[z].x * e.y + x[z].y * e.x;
        }
        k[p] = make_double2(re, im);
      }
    }
    for (int z = 0; z < nz; ++z) {
      double re = 0.0, im = 0.0;
      for (int p = 0; p < nz; ++p) {
        const double2 e = zk[p * nz + z];
        re += k[p].x * e.x + k[p].y * e.y;
        im += k[p].y * e.x - k[p].x * e.y;
      }
      out[((size_t)q * nz + z) * nn + i] = make_double2(re / nz, im / nz);
    }
  }
}

// Roemer over coils of the POCS images: sum_q img s_q / max(sum_q s_q^2, 1e-12), s_q the in-plane
// element profile times the ring's z factor
__global__ void pocs_combine_kernel(const double2* __restrict__ img, const double* __restrict__ sens,
                                    const double* __restrict__ zs, int nc, int ring, int nz, int nn,
                                    double2* __restrict__ out) {
  const int z = blockIdx.y;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
    double wr = 0.0, wi = 0.0, ss = 0.0;
    for (int q = 0; q < nc; ++q) {
      const double s = sens[(size_t)(q % ring) * nn + i] * zs[(size_t)q * nz + z];
      const double2 v = img[((size_t)q * nz + z) * nn + i];
      wr += v.x * s;
      wi += v.y * s;
      ss += s * s;
    }
    const double d = fmax(ss, 1e-12);
    out[(size_t)z * nn + i] = make_double2(wr / d, wi / d);
  }
}

__global__ void volume_output_d_kernel(const double2* __restrict__ vol, int g, int nv, size_t nvox,
                                       float* __restrict__ mag, float* __restrict__ ph) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nvox; i += (size_t)gridDim.x * blockDim.x) {
    const float re = (float)vol[i].x, im = (float)vol[i].y;
    mag[i * nv + g] = sqrtf(re * re + im * im);
    ph[i * nv + g] = atan2f(im, re);
  }
}

dim3 g3(size_t n, int y, int z) {
  return dim3((unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 1024)), (unsigned)y, (unsigned)z);
}


}  // namespace

// ---- the plan ----------------------------------------------------------------------------------------
// Per slice, the off-resonance interval (Hz) and the decay interval (1/ms) of its voxel-mode
// compartments (`spiral_rects` kspace3d.rs:876-905).
struct SliceRect {
  int z;
  double f[2], d[2];
  bool has_d;
};

static std::vector<SliceRect> spiral_rects(const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                                           const std::vector<CompMode>& modes, size_t plane, int nz) {
  std::vector<SliceRect> out;
  for (int z = 0; z < nz; ++z) {
    SliceRect r;
    r.z = z;
    r.f[0] = r.f[1] = 0.0;
    r.d[0] = r.d[1] = 0.0;
    r.has_d = false;
    if (acq.do_distortions) {
      float lo = INFINITY, hi = -INFINITY;
      for (size_t i = 0; i < plane; ++i) {
        lo = std::min(lo, in.fmap[(size_t)z * plane + i]);
        hi = std::max(hi, in.fmap[(size_t)z * plane + i]);
      }
      r.f[0] = lo;
      r.f[1] = hi;
    }
    for (size_t c = 0; c < modes.size(); ++c) {
      if (!modes[c].voxel) continue;
      for (size_t i = (size_t)z * plane; i < (size_t)(z + 1) * plane; ++i) {
        const double t2 = in.t2[c].is_map ? (double)in.t2[c].map[i] : (double)in.t2[c].value;
        const double tp = in.t_inhom ? (in.t_inhom[c].is_map ? (double)in.t_inhom[c].map[i]
                                                              : (double)in.t_inhom[c].value)
                                     : acq.t_inhom;
        const double v = 1.0 / t2 + 1.0 / tp;
        if (!r.has_d) {
          r.d[0] = r.d[1] = v;
          r.has_d = true;
        } else {
          r.d[0] = std::min(r.d[0], v);
          r.d[1] = std::max(r.d[1], v);
        }
      }
    }
    out.push_back(r);
  }
  return out;
}

// `spiral_segmentation` (kspace3d.rs:1441-1470): per slice and mode the certified plan's figures.
std::vector<SpiralSegmentationRow> spiral_segmentation(const mrsim_acquisition_3d_input& in,
                                                       const mrsim_acquisition& acq, const mrsim_echo_train& train,
                                                       const mrsim_spiral_readout& ro) {
  const int nz = (int)in.sim_dims[2];
  const size_t plane = (size_t)in.sim_dims[0] * in.sim_dims[1];
  if (!in.fmap) fail("fieldmap is not on the simulation grid");
  if (in.ncomp > 0 && !in.t2) fail("t2 is NULL");
  Spiral3dTable T = spiral_lines(train, ro, (int)in.acq_dims[0], (int)in.acq_dims[1], nz);
  auto modes = resolve_modes(in.t2, in.t1, in.t_inhom, (int)in.ncomp, acq, train, plane * nz);
  bool any_class = false;
  for (auto& m : modes) any_class = any_class || !m.voxel;
  std::vector<SpiralSegmentationRow> out;
  for (const SliceRect& r : spiral_rects(in, acq, modes, plane, nz)) {
    auto add = [&](bool voxel, const double* d) {
      TsegPlan p;
      try {
        p = tseg_plan(T.traj.tau_ms, T.traj.readout_ms, d, r.f);
      } catch (const Error& e) {
        fail("slice " + std::to_string(r.z) + ": " + e.what());
      }
      out.push_back({r.z, voxel ? 1 : 0, p.l, p.m, p.b_sum, p.bound});
    };
    const double zero[2] = {0.0, 0.0};
    if (any_class) add(false, zero);
    if (r.has_d) add(true, r.d);
  }
  return out;
}

struct SpiralPlan3 {
  int snx, sny, nz, n, o, ncomp, nc, rows, ring, ns, nsamp;
  size_t plane, nvox;
  Spiral3dTable table;
  std::vector<CompMode> modes;
  bool any_class = false, any_voxel = false;
  std::vector<TsegPlan> class_plan, voxel_plan;  // per slice (empty if the mode is unused)
  std::vector<float2> zk;
  std::vector<double2> zk_d;
  struct Src {
    int c, e;
  };
  std::vector<Src> srcs;
  std::vector<int> src_of;     // [c][p]
  std::vector<float> wc;       // [c][p][ns]
  std::vector<double> zsens;   // [q][z]
  std::vector<float2> cis0;    // [z][plane]: e^{i phi0}
  std::vector<float2> stat;    // [nsamp]
  std::vector<int64_t> tau_idx;
};

static void build_sources(SpiralPlan3& P, const mrsim_acquisition& acq) {
  P.srcs.clear();
  P.src_of.assign((size_t)P.ncomp * P.nz, 0);
  P.wc.assign((size_t)P.ncomp * P.nz * P.ns, 1.f);
  int emax = 0;
  for (int e : P.table.echo) emax = std::max(emax, e);
  for (int c = 0; c < P.ncomp; ++c) {
    const CompMode& m = P.modes[c];
    if (!m.voxel) {
      const int s = (int)P.srcs.size();
      P.srcs.push_back({c, 0});
      for (int p = 0; p < P.nz; ++p) {
        P.src_of[(size_t)c * P.nz + p] = s;
        if (!P.table.acquired[p] || !acq.do_relaxation) continue;
        for (int j = 0; j < P.ns; ++j)
          P.wc[((size_t)c * P.nz + p) * P.ns + j] =
              (float)line_weight(m.ln_a[P.table.echo[p] - 1], P.table.traj.tau_ms[j], m.t2_ms, m.t2p_ms);
      }
    } else {
      for (int e = 1; e <= emax; ++e) {
        bool used = false;
        for (int p = 0; p < P.nz; ++p) used = used || (P.table.acquired[p] && P.table.echo[p] == e);
        if (!used) continue;
        const int s = (int)P.srcs.size();
        P.srcs.push_back({c, e});
        for (int p = 0; p < P.nz; ++p)
          if (P.table.acquired[p] && P.table.echo[p] == e) P.src_of[(size_t)c * P.nz + p] = s;
      }
    }
  }
}

static SpiralPlan3 make_spiral_plan(const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                                    const mrsim_echo_train& train, const mrsim_spiral_readout& ro, int rows,
                                    cudaStream_t st) {
  SpiralPlan3 P;
  P.nc = (int)std::max<int64_t>(acq.n_coils, 1);
  if (P.nc > kMaxCoils) fail("more than 64 coils");
  if (rows < 1 || P.nc % rows != 0)
    fail(std::to_string(P.nc) + " coils do not divide into " + std::to_string(rows) + " rings along z");
  P.rows = rows;
  P.ring = P.nc / rows;
  P.snx = (int)in.sim_dims[0];
  P.sny = (int)in.sim_dims[1];
  P.nz = (int)in.sim_dims[2];
  const int nx = (int)in.acq_dims[0], ny = (int)in.acq_dims[1];
  if (P.nz != (int)in.acq_dims[2]) fail("partition count must match; z is never oversampled");
  if (P.snx <= 0 || P.sny <= 0 || nx <= 0 || ny <= 0 || P.nz <= 0) fail("empty simulation grid or acquired matrix");
  if (!(P.snx % nx == 0 && P.sny % ny == 0)) fail("sim grid must be an integer multiple of the acquired matrix");
  P.o = P.snx / nx;
  if (P.o != P.sny / ny) fail("oversampling must match on both axes");
  if (P.nz > 64) fail("at most 64 partitions");
  P.n = nx;
  P.ncomp = (int)in.ncomp;
  if (P.ncomp > kMaxComp) fail("more than 8 compartments");
  P.plane = (size_t)P.snx * P.sny;
  P.nvox = P.plane * P.nz;
  if (!in.fmap) fail("fieldmap is not on the simulation grid");
  if (P.ncomp > 0 && (!in.images || !in.t2)) fail("compartment image is not on the simulation grid");
  if (acq.echo != MRSIM_ECHO_SPIN) fail("the 3D echo trains are spin-echo trains");
  if (acq.eddy_strength != 0.0 || acq.eddy_quad != 0.0 || acq.eddy_phase != 0.0)
    fail("the eddy model is not available in 3D (an echo-dependent eddy evolution breaks the z factorization)");
  if (acq.accel > 1) fail("GRAPPA has no spiral meaning in this model");
  if (!(acq.partial_fourier >= 1.0))
    fail("in-plane partial Fourier has no spiral meaning in this model (along kz it is the readout's KzSampling)");
  if (acq.ghost_offset != 0.0) fail("Nyquist ghosting has no spiral meaning in this model");
  if (acq.n_spikes != 0) fail("spikes have no spiral meaning in this model");
  P.table = spiral_lines(train, ro, nx, ny, P.nz);
  P.ns = (int)P.table.traj.tau_ms.size();
  P.nsamp = P.ns * (int)ro.interleaves;
  P.modes = resolve_modes(in.t2, in.t1, in.t_inhom, P.ncomp, acq, train, P.nvox);
  for (auto& m : P.modes) (m.voxel ? P.any_voxel : P.any_class) = true;
  build_sources(P, acq);
  P.class_plan.resize(P.nz);
  P.voxel_plan.resize(P.nz);
  // per-slice certified segmentations: each distinct rate rectangle planned once (slices that
  // share one get the same plan bit for bit), the distinct ones on up to 16 host threads, each
  // with its fits' per-sample work on the device on a stream of its own; the first failure in
  // slice order is the one reported, as a sequential plan would report it
  std::vector<double> tau(P.table.traj.tau_ms);
  std::vector<std::array<double, 4>> keys;
  std::vector<int> cls_of(P.nz, -1), vox_of(P.nz, -1);
  auto key_of = [&](const double d[2], const double f[2]) {
    const std::array<double, 4> k{d[0], d[1], f[0], f[1]};
    for (size_t i = 0; i < keys.size(); ++i)
      if (keys[i] == k) return (int)i;
    keys.push_back(k);
    return (int)keys.size() - 1;
  };
  for (const SliceRect& r : spiral_rects(in, acq, P.modes, P.plane, P.nz)) {
    const double zero[2] = {0.0, 0.0};
    if (P.any_class) cls_of[r.z] = key_of(zero, r.f);
    if (r.has_d) vox_of[r.z] = key_of(r.d, r.f);
  }
  std::vector<TsegPlan> plans(keys.size());
  std::vector<std::exception_ptr> errs(keys.size());
  int dev_id = 0;
  MRSIM_CUDA(cudaGetDevice(&dev_id));
  std::atomic<int> next{0};
  std::mutex setup_mu;
  std::exception_ptr setup_err;  // a worker that could not set up its stream
  auto worker = [&] {
    cudaStream_t ws = nullptr;
    try {
      MRSIM_CUDA(cudaSetDevice(dev_id));
      MRSIM_CUDA(cudaStreamCreateWithFlags(&ws, cudaStreamNonBlocking));
      TsegDevice dev(ws);
      for (int i; (i = next.fetch_add(1)) < (int)keys.size();) {
        try {
          const double d[2] = {keys[i][0], keys[i][1]}, f[2] = {keys[i][2], keys[i][3]};
          plans[i] = tseg_plan(tau, P.table.traj.readout_ms, d, f, &dev);
        } catch (...) {
          errs[i] = std::current_exception();
        }
      }
    } catch (...) {
      std::lock_guard<std::mutex> lk(setup_mu);
      if (!setup_err) setup_err = std::current_exception();
    }
    if (ws) cudaStreamDestroy(ws);
  };
  const int nt = (int)std::min<size_t>(keys.size(), std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
  if (nt <= 1) {
    worker();
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t) pool.emplace_back(worker);
    for (auto& t : pool) t.join();
  }
  if (setup_err) std::rethrow_exception(setup_err);
  for (auto& e : errs)
    if (e) std::rethrow_exception(e);
  for (int z = 0; z < P.nz; ++z) {
    if (cls_of[z] >= 0) P.class_plan[z] = plans[cls_of[z]];
    if (vox_of[z] >= 0) P.voxel_plan[z] = plans[vox_of[z]];
  }
  // the centred z-DFT kernel, the ring z profiles, the object phase, the half-cell phase
  const double zs = (double)(P.nz / 2);
  P.zk.resize((size_t)P.nz * P.nz);
  P.zk_d.resize((size_t)P.nz * P.nz);
  for (int p = 0; p < P.nz; ++p)
    for (int z = 0; z < P.nz; ++z) {
      const double th = kTau * ((double)p - zs) * ((double)z - zs) / (double)P.nz;
      P.zk[(size_t)p * P.nz + z] = make_float2((float)std::cos(th), (float)std::sin(th));
      P.zk_d[(size_t)p * P.nz + z] = make_double2(std::cos(th), std::sin(th));
    }
  P.zsens.resize((size_t)P.nc * P.nz);
  for (int q = 0; q < P.nc; ++q)
    for (int z = 0; z < P.nz; ++z) P.zsens[(size_t)q * P.nz + z] = coil_row_sensitivity(q / P.ring, rows, z, P.nz);
  P.cis0.resize(P.nvox);
  mrsim_phase_model pm;
  std::memset(&pm, 0, sizeof pm);
  if (in.phase) pm = *in.phase;
  for (int z = 0; z < P.nz; ++z) {  // `phase_slice` with a zero shot (kspace.rs:1156-1180)
    const double sx = P.snx / 2.0, sy = P.sny / 2.0, off = (P.o - 1.0) / 2.0, r2 = z - P.nz / 2.0;
    for (int y = 0; y < P.sny; ++y)
      for (int x = 0; x < P.snx; ++x) {
        const double r0 = (x - sx - off) / P.o, r1 = (y - sy - off) / P.o;
        const double* c = pm.background;
        const double bg = c[0] + c[1] * r0 + c[2] * r1 + c[3] * r2 + c[4] * r0 * r0 + c[5] * r1 * r1 + c[6] * r2 * r2 +
                          c[7] * r0 * r1 + c[8] * r0 * r2 + c[9] * r1 * r2;
        const double ph = pm.global + bg;
        P.cis0[(size_t)z * P.plane + x + (size_t)P.snx * y] = make_float2((float)std::cos(ph), (float)std::sin(ph));
      }
  }
  const int sxs = P.o * (nx / 2), sys = P.o * (ny / 2);
  (void)sxs;
  (void)sys;
  const double xoff = (P.o - 1.0) / 2.0, yoff = (P.o - 1.0) / 2.0, ninv = 1.0 / (double)P.plane;
  const std::vector<double>& k = P.table.traj.k;
  P.stat.resize(P.nsamp);
  P.tau_idx.resize(P.nsamp);
  for (int j = 0; j < P.nsamp; ++j) {  // `SegmentedForward::new` (spiral.rs:159-170)
    const double ph = -kTau * (k[2 * j] * xoff / P.snx + k[2 * j + 1] * yoff / P.sny);
    P.stat[j] = make_float2((float)(std::cos(ph) * ninv), (float)(std::sin(ph) * ninv));
    P.tau_idx[j] = j % P.ns;
  }
  return P;
}

// Device inputs of one acquisition's images (all volumes), plus per-element amplitudes.
struct SpiralInputs {
  float* img = nullptr;    // [g][z][c][plane]
  float* fmap = nullptr;   // [nvox] (with distortions) or NULL
  float* decay = nullptr;  // [c][nvox] 1/T2 + 1/T2' of voxel compartments
  float* lna = nullptr;    // [c][e][nvox]
  float* amp = nullptr;    // [a][plane]
  float2* cis0 = nullptr;  // [z][plane]
};

static SpiralInputs upload_spiral_inputs(DevArena& A, const SpiralPlan3& P, const mrsim_acquisition_3d_input& in,
                                         const float* const* images, int nv, const mrsim_acquisition& acq,
                                         cudaStream_t st) {
  SpiralInputs I;
  const size_t per_comp = P.nvox * nv;
  float* staging = (float*)A.alloc(std::max<size_t>(1, per_comp * P.ncomp) * 4);
  for (int c = 0; c < P.ncomp; ++c)
    MRSIM_CUDA(cudaMemcpyAsync(staging + (size_t)c * per_comp, images[c], per_comp * 4, cudaMemcpyHostToDevice, st));
  I.img = (float*)A.alloc(std::max<size_t>(1, per_comp * P.ncomp) * 4);
  if (P.ncomp) launch_series_transpose(staging, I.img, P.ncomp, nv, P.nz, (int)P.plane, st);
  if (acq.do_distortions) I.fmap = (float*)A.upload(in.fmap, P.nvox * 4, st);
  if (P.any_voxel) {
    int etl = 0;
    for (auto& m : P.modes)
      if (m.voxel) etl = (int)m.maps.size();
    std::vector<float> d((size_t)P.ncomp * P.nvox, 0.f), la((size_t)P.ncomp * etl * P.nvox, 0.f);
    for (int c = 0; c < P.ncomp; ++c) {
      if (!P.modes[c].voxel) continue;
      for (size_t i = 0; i < P.nvox; ++i) {
        const double t2 = in.t2[c].is_map ? (double)in.t2[c].map[i] : (double)in.t2[c].value;
        const double tp = in.t_inhom ? (in.t_inhom[c].is_map ? (double)in.t_inhom[c].map[i]
                                                              : (double)in.t_inhom[c].value)
                                     : acq.t_inhom;
        d[(size_t)c * P.nvox + i] = (float)(1.0 / t2 + 1.0 / tp);
      }
      for (int e = 0; e < etl; ++e)
        for (size_t i = 0; i < P.nvox; ++i)
          la[((size_t)c * etl + e) * P.nvox + i] = (float)P.modes[c].maps[e][i];
    }
    I.decay = (float*)A.upload(d.data(), d.size() * 4, st);
    I.lna = (float*)A.upload(la.data(), la.size() * 4, st);
  }
  std::vector<float> amp((size_t)P.ring * P.plane);
  const double xoff = (P.o - 1.0) / 2.0, yoff = (P.o - 1.0) / 2.0;
  for (int a = 0; a < P.ring; ++a)
    for (int y = 0; y < P.sny; ++y)
      for (int x = 0; x < P.snx; ++x)
        amp[(size_t)a * P.plane + x + (size_t)P.snx * y] =
            (float)(acq.signal_scale *
                    coil_sensitivity(a, P.ring, ((double)x - xoff) / P.o, ((double)y - yoff) / P.o, P.n, P.n));
  I.amp = (float*)A.upload(amp.data(), amp.size() * 4, st);
  I.cis0 = (float2*)A.upload(P.cis0.data(), P.cis0.size() * sizeof(float2), st);
  return I;
}

// One volume's per-shot images (`ShotSet`, kspace3d.rs:59-65): variant 0 the volume's own
// images, variant v > 0 its set v - 1; per shot the variant it saw (the first set holding it).
struct SpiralVariants {
  int nvar = 1;
  std::vector<std::vector<const float*>> img;  // [v][c] device sim volumes (v > 0)
  const int* d_shot_var = nullptr;             // [n_shots], or NULL without sets
};

static SpiralVariants spiral_sets(DevArena& A, const SpiralPlan3& P, const mrsim_acquisition_3d_input& in, int g,
                                  cudaStream_t st, bool upload = true) {
  SpiralVariants V;
  if (!in.shot_sets || !in.n_shot_sets || in.n_shot_sets[g] <= 0) return V;
  const mrsim_shot_set* sets = in.shot_sets[g];
  const int64_t n = in.n_shot_sets[g];
  if (!sets) fail("volume " + std::to_string(g) + ": its shot sets are NULL");
  V.nvar = (int)n + 1;
  V.img.assign((size_t)V.nvar, std::vector<const float*>(P.ncomp, nullptr));
  std::vector<int> var((size_t)P.table.n_shots, 0);
  for (int64_t i = n - 1; i >= 0; --i) {  // descending, so the first set holding a shot wins
    const mrsim_shot_set& S = sets[i];
    if (S.n_shots > 0 && !S.shots) fail("volume " + std::to_string(g) + ": a shot set's shots are NULL");
    for (int64_t j = 0; j < S.n_shots; ++j) {
      if (S.shots[j] < 0 || S.shots[j] >= P.table.n_shots)
        fail("a shot index beyond the train's " + std::to_string(P.table.n_shots));
      var[(size_t)S.shots[j]] = (int)i + 1;
    }
    for (int c = 0; c < P.ncomp; ++c) {
      if (!S.images || !S.images[c]) fail("shot images are not per compartment");
      if (upload) V.img[(size_t)i + 1][c] = (const float*)A.upload(S.images[c], P.nvox * 4, st);
    }
  }
  if (upload) V.d_shot_var = (const int*)A.upload(var.data(), var.size() * 4, st);
  return V;
}

// Every coil's samples of volume g before noise: out [q][p][nsamp].
static void spiral_samples(const SpiralPlan3& P, const SpiralInputs& I, int g, const float* d_lw, float2* out,
                           cudaStream_t st, const SpiralVariants* V = nullptr) {
  const int nsrc = (int)P.srcs.size(), nz = P.nz, nsamp = P.nsamp, ring = P.ring;
  const int nvar = V ? V->nvar : 1;
  DevArena C;
  NufftGrid grid = make_nufft<float>(C, P.snx, P.sny, -P.o * (P.n / 2), -P.o * (P.n / 2), P.snx, P.sny, 1e-12, st);
  const double* d_k = (const double*)C.upload(P.table.traj.k.data(), P.table.traj.k.size() * 8, st);
  const float2* d_stat = (const float2*)C.upload(P.stat.data(), P.stat.size() * sizeof(float2), st);
  float2* k2 = (float2*)C.alloc((size_t)nvar * ring * nsrc * nz * nsamp * sizeof(float2));
  MRSIM_CUDA(cudaMemsetAsync(k2, 0, (size_t)nvar * ring * nsrc * nz * nsamp * sizeof(float2), st));
  // per slice: slots (a, s) with their plans
  int Lmax = 1;
  for (int z = 0; z < nz; ++z) Lmax = std::max({Lmax, P.class_plan[z].l, P.voxel_plan[z].l});
  const int nslot = nvar * ring * nsrc;
  float2* seg = (float2*)C.alloc((size_t)nslot * Lmax * P.plane * sizeof(float2));
  float2* segout = (float2*)C.alloc((size_t)nslot * Lmax * nsamp * sizeof(float2));
  float2* work = (float2*)C.alloc((size_t)nslot * Lmax * grid.nf0 * grid.nf1 * sizeof(float2));
  SegSlot* d_slots = (SegSlot*)C.alloc((size_t)nslot * sizeof(SegSlot));
  int* d_base = (int*)C.alloc((size_t)nslot * 4);
  int* d_plan = (int*)C.alloc((size_t)nslot * 4);
  size_t* d_off = (size_t*)C.alloc((size_t)nslot * sizeof(size_t));
  for (int z = 0; z < nz; ++z) {
    const TsegPlan& pc = P.class_plan[z];
    const TsegPlan& pv = P.voxel_plan[z];
    std::vector<SegSlot> slots(nslot);
    std::vector<int> base(nslot), plan(nslot);
    std::vector<size_t> off(nslot);
    int tot = 0;
    for (int v = 0; v < nvar; ++v)
    for (int a = 0; a < ring; ++a)
      for (int s = 0; s < nsrc; ++s) {
        const int i = (v * ring + a) * nsrc + s;
        const SpiralPlan3::Src& S = P.srcs[s];
        const bool voxel = P.modes[S.c].voxel;
        SegSlot& sl = slots[i];
        std::memset(&sl, 0, sizeof sl);
        sl.comp = v > 0 ? V->img[(size_t)v][S.c] + (size_t)z * P.plane
                        : I.img + (((size_t)g * nz + z) * P.ncomp + S.c) * P.plane;
        sl.amp = I.amp + (size_t)a * P.plane;
        sl.plan = voxel ? 1 : 0;
        if (voxel) {
          const int etl = (int)P.modes[S.c].maps.size();
          sl.la = I.lna + ((size_t)S.c * etl + (S.e - 1)) * P.nvox + (size_t)z * P.plane;
          sl.decay = I.decay + (size_t)S.c * P.nvox + (size_t)z * P.plane;
        }
        base[i] = tot;
        plan[i] = sl.plan;
        tot += voxel ? pv.l : pc.l;
        off[i] = ((((size_t)v * ring + a) * nsrc + s) * nz + z) * nsamp;
      }
    if (tot == 0) continue;
    MRSIM_CUDA(cudaMemcpyAsync(d_slots, slots.data(), slots.size() * sizeof(SegSlot), cudaMemcpyHostToDevice, st));
    MRSIM_CUDA(cudaMemcpyAsync(d_base, base.data(), base.size() * 4, cudaMemcpyHostToDevice, st));
    MRSIM_CUDA(cudaMemcpyAsync(d_plan, plan.data(), plan.size() * 4, cudaMemcpyHostToDevice, st));
    MRSIM_CUDA(cudaMemcpyAsync(d_off, off.data(), off.size() * sizeof(size_t), cudaMemcpyHostToDevice, st));
    DevArena Z;
    const double* tl0 = pc.l ? (const double*)Z.upload(pc.tau_l.data(), pc.tau_l.size() * 8, st) : nullptr;
    const double* tl1 = pv.l ? (const double*)Z.upload(pv.tau_l.data(), pv.tau_l.size() * 8, st) : nullptr;
    const double* b0 = pc.l ? (const double*)Z.upload(pc.b.data(), pc.b.size() * 8, st) : nullptr;
    const double* b1 = pv.l ? (const double*)Z.upload(pv.b.data(), pv.b.size() * 8, st) : nullptr;
    seg_images_kernel<<<g3(P.plane, nslot, 1), 256, 0, st>>>(d_slots, I.cis0 + (size_t)z * P.plane,
                                                             I.fmap ? I.fmap + (size_t)z * P.plane : nullptr, tl0, tl1,
                                                             pc.l, pv.l, (int)P.plane, seg, d_base);
    nufft_type2<float>(grid, seg, tot, P.plane, d_k, nsamp, segout, nsamp, work, 1, nullptr, st);
    seg_combine_kernel<<<g3(nsamp, nslot, 1), 256, 0, st>>>(segout, d_base, d_plan, b0, b1, pc.l, pv.l, P.ns, nsamp,
                                                            d_stat, k2, d_off);
    MRSIM_CUDA(cudaGetLastError());
    MRSIM_CUDA(cudaStreamSynchronize(st));  // Z's tables are freed at the end of the iteration
  }
  // the z-DFT with the rings' profiles, amplitudes and line weights
  std::vector<float2> zkq((size_t)P.rows * nz * nz);
  for (int r = 0; r < P.rows; ++r)
    for (int p = 0; p < nz; ++p)
      for (int z = 0; z < nz; ++z) {
        float2 v = P.zk[(size_t)p * nz + z];
        if (P.rows > 1) {
          const double s = coil_row_sensitivity(r, P.rows, z, nz);
          const double2 d = P.zk_d[(size_t)p * nz + z];
          v = make_float2((float)(d.x * s), (float)(d.y * s));
        }
        zkq[((size_t)r * nz + p) * nz + z] = v;
      }
  std::vector<int> kzseg(P.table.kz_segment.begin(), P.table.kz_segment.end());
  std::vector<unsigned char> acq_p(P.table.acquired.begin(), P.table.acquired.end());
  ZArgs za;
  za.k2 = k2;
  za.out = out;
  za.zkq = (const float2*)C.upload(zkq.data(), zkq.size() * sizeof(float2), st);
  za.src = (const int*)C.upload(P.src_of.data(), std::max<size_t>(1, P.src_of.size()) * 4, st);
  za.wc = (const float*)C.upload(P.wc.data(), std::max<size_t>(1, P.wc.size()) * 4, st);
  za.lw = d_lw;
  za.kzseg = (const int*)C.upload(kzseg.data(), kzseg.size() * 4, st);
  za.acquired = (const unsigned char*)C.upload(acq_p.data(), acq_p.size(), st);
  za.nz = nz;
  za.nsamp = nsamp;
  za.ns = P.ns;
  za.ncomp = P.ncomp;
  za.nsrc = nsrc;
  za.ring = ring;
  za.kz_segments = P.table.kz_segments;
  za.n_shots = P.table.n_shots;
  za.g = g;
  za.shot_var = V ? V->d_shot_var : nullptr;
  spiral_zdft_kernel<<<g3(nsamp, nz, P.nc), 256, 0, st>>>(za);
  MRSIM_CUDA(cudaGetLastError());
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

// `spiral_noise` (kspace3d.rs:1391-1404) on the acquired partitions of every coil
static void spiral_noise(DevArena& A, const SpiralPlan3& P, const std::vector<uint8_t>& acquired, float2* k, int g,
                         uint64_t seed, double sigma, cudaStream_t st) {
  if (!(sigma > 0.0)) return;
  std::vector<NoiseJob> jobs;
  const int zero_row = 0;
  const int* d_row = (const int*)A.upload(&zero_row, 4, st);
  for (int q = 0; q < P.nc; ++q)
    for (int p = 0; p < P.nz; ++p) {
      if (!acquired[p]) continue;
      const uint64_t pseed = (((uint64_t)g * 0x1000001ull) + (uint64_t)p) * 0x9E37ull ^ seed ^ kSeedSalt3d;
      NoiseJob J;
      std::memset(&J, 0, sizeof J);
      J.k = k + ((size_t)q * P.nz + p) * P.nsamp;
      J.rows = d_row;
      J.n_rows = 1;
      J.nx = P.nsamp;
      J.seed = (pseed ^ ((uint64_t)q * 0x9E3779B9ull)) | 1ull;
      J.sigma = sigma;
      jobs.push_back(J);
    }
  if (jobs.empty()) return;
  const NoiseJob* d_jobs = (const NoiseJob*)A.upload(jobs.data(), jobs.size() * sizeof(NoiseJob), st);
  launch_noise_jobs(d_jobs, (int)jobs.size(), false, true, P.nsamp, nullptr, st);
  MRSIM_CUDA(cudaGetLastError());
}

// `KzGrappa` (kspace3d.rs:1261-1389): the targets of the accelerated table, the fit on the
// calibration samples and the fill.
struct KzKernel {
  struct Target {
    int p, d;
    unsigned pat;
  };
  std::vector<Target> targets;
  std::map<std::pair<int, unsigned>, std::pair<int, int>> where;  // (d, pat) -> (offset into w, nsrc)
  std::vector<float2> w;
};

static std::vector<KzKernel::Target> kz_targets(const Spiral3dTable& T, int accel) {
  std::vector<KzKernel::Target> out;
  const int64_t c = T.nz / 2;
  for (int p = T.band_start; p < T.nz; ++p) {
    if (T.acquired[p]) continue;
    const int d = (int)((((int64_t)p - c) % accel + accel) % accel);
    const int64_t offs[kKzSources] = {-d - accel, -d, accel - d, 2 * accel - d};
    unsigned pat = 0;
    for (int s = 0; s < kKzSources; ++s) {
      const int64_t src = p + offs[s];
      if (src >= 0 && src < T.nz && T.acquired[src]) pat |= 1u << s;
    }
    out.push_back({p, d, pat});
  }
  return out;
}

static KzKernel kz_fit(mrsim_context* ctx, const Spiral3dTable& T, int accel, const float2* d_cal, int nc, int nsamp) {
  cudaStream_t st = ctx->stream;
  KzKernel K;
  K.targets = kz_targets(T, accel);
  const int nz = T.nz, lo = T.band_start;
  for (const auto& tg : K.targets) {
    if (tg.pat == 0) {
      char buf[256];
      std::snprintf(buf, sizeof buf,
                    "partition %d of the partial-Fourier band has no acquired partition within the kernel's reach: %d "
                    "partitions are too few for a kz acceleration of %d",
                    tg.p, nz, accel);
      fail(buf);
    }
    const auto key = std::make_pair(tg.d, tg.pat);
    if (K.where.count(key)) continue;
    const int64_t all[kKzSources] = {-tg.d - accel, -tg.d, accel - tg.d, 2 * accel - tg.d};
    std::vector<int> offs;
    for (int s = 0; s < kKzSources; ++s)
      if (tg.pat & (1u << s)) offs.push_back((int)all[s]);
    const int nsrc = (int)offs.size(), nfeat = nsrc * nc, ncol = nfeat + nc;
    std::vector<int> tl;
    for (int t = lo; t < nz; ++t) {
      bool ok = true;
      for (int o : offs) ok = ok && t + o >= lo && t + o < nz;
      if (ok) tl.push_back(t);
    }
    if (tl.empty()) {
      std::string os;
      for (size_t i = 0; i < offs.size(); ++i) os += (i ? ", " : "") + std::to_string(offs[i]);
      fail("the calibration band (" + std::to_string(nz - lo) +
           " partitions) holds no partition with the kernel's sources at offsets [" + os +
           "]: too few partitions for a kz acceleration of " + std::to_string(accel));
    }
    if (nfeat * ncol > 24 * 256) fail("too many coils for the kz kernel (at most 16 x 4 sources)");
    DevArena A;
    KzFitArgs a;
    a.k = d_cal;
    a.t_list = (const int*)A.upload(tl.data(), tl.size() * 4, st);
    a.offs = (const int*)A.upload(offs.data(), offs.size() * 4, st);
    a.n_t = (int)tl.size();
    a.nsrc = nsrc;
    a.nc = nc;
    a.nz = nz;
    a.nsamp = nsamp;
    const int blocks = 296;
    a.partial = (double2*)A.alloc((size_t)blocks * nfeat * ncol * sizeof(double2));
    const size_t smem = (size_t)16 * ncol * sizeof(double2);
    kz_normal_kernel<<<blocks, 256, smem, st>>>(a);
    MRSIM_CUDA(cudaGetLastError());
    KzSolveArgs sa;
    sa.partial = a.partial;
    sa.W = (double2*)A.alloc((size_t)nfeat * ncol * sizeof(double2));
    sa.scratch = (double*)A.alloc((size_t)(2 * nfeat + nc * 2 * nfeat) * sizeof(double));
    sa.out = (float2*)A.alloc((size_t)nc * nfeat * sizeof(float2));
    sa.status = (int*)A.alloc(sizeof(int));
    sa.lambda = kKzLambda;
    sa.blocks = blocks;
    sa.nfeat = nfeat;
    sa.nc = nc;
    MRSIM_CUDA(cudaMemsetAsync(sa.status, 0, sizeof(int), st));
    kz_solve_kernel<<<1, 256, 0, st>>>(sa);
    MRSIM_CUDA(cudaGetLastError());
    int status = 0;
    const int woff = (int)K.w.size();
    K.w.resize(K.w.size() + (size_t)nc * nfeat);
    MRSIM_CUDA(cudaMemcpyAsync(&status, sa.status, sizeof(int), cudaMemcpyDeviceToHost, st));
    MRSIM_CUDA(cudaMemcpyAsync(K.w.data() + woff, sa.out, (size_t)nc * nfeat * sizeof(float2), cudaMemcpyDeviceToHost,
                               st));
    MRSIM_CUDA(cudaStreamSynchronize(st));
    if (status) fail("the kz calibration acquisition is empty: its images give no signal");
    K.where[key] = std::make_pair(woff, nsrc);
  }
  return K;
}

static void kz_fill(mrsim_context* ctx, const KzKernel& K, int accel, float2* d_k, int nc, int nz, int nsamp) {
  cudaStream_t st = ctx->stream;
  if (K.targets.empty()) return;
  DevArena A;
  std::vector<KzFillJob> jobs;
  for (const auto& tg : K.targets) {
    auto it = K.where.find(std::make_pair(tg.d, tg.pat));
    if (it == K.where.end()) continue;
    KzFillJob J;
    std::memset(&J, 0, sizeof J);
    J.p = tg.p;
    J.woff = it->second.first;
    const int64_t all[kKzSources] = {-tg.d - accel, -tg.d, accel - tg.d, 2 * accel - tg.d};
    for (int s = 0; s < kKzSources; ++s)
      if (tg.pat & (1u << s)) J.src[J.nsrc++] = (int)(tg.p + all[s]);
    jobs.push_back(J);
  }
  // every target reads only acquired partitions: one launch fills them all
  const KzFillJob* d_jobs = (const KzFillJob*)A.upload(jobs.data(), jobs.size() * sizeof(KzFillJob), st);
  const float2* d_w = (const float2*)A.upload(K.w.data(), K.w.size() * sizeof(float2), st);
  kz_fill_kernel<<<g3(nsamp, (int)jobs.size(), nc), 256, 0, st>>>(d_k, d_jobs, d_w, nc, nz, nsamp);
  MRSIM_CUDA(cudaGetLastError());
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

// ---- the entry points ----------------------------------------------------------------------------------
void spiral3d_samples(mrsim_context* ctx, const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                      const mrsim_echo_train& train, const mrsim_spiral_readout& ro, const mrsim_kz_options* opts,
                      int g, float* out) {
  cudaStream_t st = ctx->stream;
  const int rows = opts ? (int)opts->coil_rows : 1;
  SpiralPlan3 P = make_spiral_plan(in, acq, train, ro, rows, st);
  if (g < 0 || g >= (int)in.n_volumes) fail("volume index out of range");
  DevArena A;
  SpiralInputs I = upload_spiral_inputs(A, P, in, in.images, (int)in.n_volumes, acq, st);
  const float* d_lw = nullptr;
  if (in.line_weights) {
    std::vector<float> lw((size_t)in.n_volumes * P.table.n_shots * P.ncomp);
    for (size_t i = 0; i < lw.size(); ++i) lw[i] = (float)in.line_weights[i];
    d_lw = (const float*)A.upload(lw.data(), std::max<size_t>(1, lw.size()) * 4, st);
  }
  float2* k = (float2*)A.alloc((size_t)P.nc * P.nz * P.nsamp * sizeof(float2));
  for (int h = 0; h < (int)in.n_volumes; ++h) (void)spiral_sets(A, P, in, h, st, false);  // every volume's sets checked
  const SpiralVariants V = spiral_sets(A, P, in, g, st);
  spiral_samples(P, I, g, d_lw, k, st, &V);
  copy_pageable_d2h(ctx, out, k, (size_t)P.nc * P.nz * P.nsamp * sizeof(float2), st);
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

void spiral3d_acquire(mrsim_context* ctx, const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                      const mrsim_echo_train& train, const mrsim_spiral_readout& ro, const mrsim_kz_options* opts,
                      uint64_t seed, float* mag, float* ph) {
  cudaStream_t st = ctx->stream;
  const int rows = opts ? (int)opts->coil_rows : 1;
  SpiralPlan3 P = make_spiral_plan(in, acq, train, ro, rows, st);
  const int nv = (int)in.n_volumes, nz = P.nz, nc = P.nc, n = P.n, nsamp = P.nsamp;
  const double sigma = std::sqrt(acq.noise_variance / (double)((size_t)n * n));
  DevArena A;
  for (int g = 0; g < nv; ++g) (void)spiral_sets(A, P, in, g, st, false);  // every volume's sets checked first
  SpiralInputs I = upload_spiral_inputs(A, P, in, in.images, nv, acq, st);
  const float* d_lw = nullptr;
  if (in.line_weights) {
    std::vector<float> lw((size_t)nv * P.table.n_shots * P.ncomp);
    for (size_t i = 0; i < lw.size(); ++i) lw[i] = (float)in.line_weights[i];
    d_lw = (const float*)A.upload(lw.data(), std::max<size_t>(1, lw.size()) * 4, st);
  }
  // the kz kernel from the calibration acquisition (`kz_calibrate` kspace3d.rs:1406-1439)
  KzKernel kzk;
  const int accel = (int)ro.kz.accel;
  if (accel > 1) {
    if (!opts) fail("a stack of spirals accelerated along kz needs its KzOptions (coil rings, calibration)");
    if (rows < accel)
      fail("a kz acceleration of " + std::to_string(accel) + " needs at least as many coil rings along z, not " +
           std::to_string(rows));
    if (!opts->calibration_images) fail("the kz calibration images are not one simulation-grid volume per compartment");
    mrsim_spiral_readout cro = ro;
    cro.kz.accel = 1;
    const int n_cal = [&] {
      int c = 0;
      for (uint8_t a : kz_acquired(cro.kz, nz)) c += a;
      return c;
    }();
    if (n_cal % (int)train.kz_segments != 0)
      fail("the kz calibration train reads " + std::to_string(n_cal) + " partitions, which do not divide into " +
           std::to_string(train.kz_segments) + " kz segments");
    mrsim_echo_train ctr = train;
    ctr.etl = n_cal / train.kz_segments;
    SpiralPlan3 Pc = P;  // same segmentations, z-DFT and coils; the calibration train's table and amplitudes
    Pc.table = spiral_lines(ctr, cro, n, n, nz);
    Pc.modes = resolve_modes(in.t2, in.t1, in.t_inhom, P.ncomp, acq, ctr, P.nvox);
    build_sources(Pc, acq);
    DevArena C;
    SpiralInputs Ic = upload_spiral_inputs(C, Pc, in, opts->calibration_images, 1, acq, st);
    float2* ck = (float2*)C.alloc((size_t)nc * nz * nsamp * sizeof(float2));
    spiral_samples(Pc, Ic, 0, nullptr, ck, st);
    spiral_noise(C, Pc, Pc.table.acquired, ck, 0, opts->calibration_seed ^ kSeedSaltKzcal, sigma, st);
    kzk = kz_fit(ctx, P.table, accel, ck, nc, nsamp);
  }
  const bool pocs = ro.kz.partial_fourier < 1.0 && P.table.band_start > 0 && opts && opts->pocs;
  SpiralRecon rec(ctx, P.table.traj.k.data(), nsamp, n, acq, kLsIterations, kLsKappa, true);
  const size_t nn = (size_t)n * n;
  float* d_mag = (float*)A.alloc(std::max<size_t>(1, nn * nz * nv) * 4);
  float* d_ph = (float*)A.alloc(std::max<size_t>(1, nn * nz * nv) * 4);
  std::vector<double> zs_zq((size_t)nz * nc);  // [z][q] for the ring combine
  for (int z = 0; z < nz; ++z)
    for (int q = 0; q < nc; ++q) zs_zq[(size_t)z * nc + q] = P.zsens[(size_t)q * nz + z];
  const float2* d_zk = (const float2*)A.upload(P.zk.data(), P.zk.size() * sizeof(float2), st);
  for (int g = 0; g < nv; ++g) {
    DevArena C;
    float2* k = (float2*)C.alloc((size_t)nc * nz * nsamp * sizeof(float2));
    const SpiralVariants V = spiral_sets(C, P, in, g, st);
    spiral_samples(P, I, g, d_lw, k, st, &V);
    spiral_noise(C, P, P.table.acquired, k, g, seed, sigma, st);
    if (accel > 1) kz_fill(ctx, kzk, accel, k, nc, nz, nsamp);
    double2* vol = (double2*)C.alloc(nn * nz * sizeof(double2));
    if (pocs) {
      // every coil's partitions of the band reconstructed in-plane, completed along z, combined
      const int lo = P.table.band_start;
      const size_t nb = (size_t)(nz - lo);
      double2* hs = (double2*)C.alloc((size_t)nc * nb * nsamp * sizeof(double2));
      for (int q = 0; q < nc; ++q)
        to_double_kernel<<<1024, 256, 0, st>>>(k + ((size_t)q * nz + lo) * nsamp, nb * nsamp,
                                              hs + (size_t)q * nb * nsamp);
      double2* h = (double2*)C.alloc((size_t)nc * nz * nn * sizeof(double2));
      MRSIM_CUDA(cudaMemsetAsync(h, 0, (size_t)nc * nz * nn * sizeof(double2), st));
      double2* himg = (double2*)C.alloc((size_t)nc * nb * nn * sizeof(double2));
      for (size_t b0 = 0; b0 < (size_t)nc * nb; b0 += kMaxBatch) {
        const int cnt = (int)std::min<size_t>(kMaxBatch, (size_t)nc * nb - b0);
        rec.images(hs + b0 * nsamp, cnt, himg + b0 * nn);
      }
      for (int q = 0; q < nc; ++q)
        MRSIM_CUDA(cudaMemcpyAsync(h + ((size_t)q * nz + lo) * nn, himg + (size_t)q * nb * nn, nb * nn * sizeof(double2),
                                   cudaMemcpyDeviceToDevice, st));
      double2* img = (double2*)C.alloc((size_t)nc * nz * nn * sizeof(double2));
      const double2* d_zkd = (const double2*)C.upload(P.zk_d.data(), P.zk_d.size() * sizeof(double2), st);
      pocs_kernel<<<g3(nn, nc, 1), 128, 0, st>>>(h, lo, d_zkd, nz, (int)nn, nc, img);
      std::vector<double> sens((size_t)P.ring * nn);
      for (int a = 0; a < P.ring; ++a)
        for (int y = 0; y < n; ++y)
          for (int x = 0; x < n; ++x) sens[(size_t)a * nn + x + (size_t)n * y] = coil_sensitivity(a, P.ring, x, y, n, n);
      const double* d_sens = (const double*)C.upload(sens.data(), sens.size() * 8, st);
      const double* d_zs = (const double*)C.upload(P.zsens.data(), P.zsens.size() * 8, st);
      pocs_combine_kernel<<<g3(nn, nz, 1), 256, 0, st>>>(img, d_sens, d_zs, nc, P.ring, nz, (int)nn, vol);
      MRSIM_CUDA(cudaGetLastError());
    } else {
      double2* sl = (double2*)C.alloc((size_t)nz * nc * nsamp * sizeof(double2));
      spiral_izdft_kernel<<<g3(nsamp, nz, nc), 256, 0, st>>>(k, d_zk, nz, nc, nsamp, sl);
      MRSIM_CUDA(cudaGetLastError());
      rec.rings(sl, nz, nc, P.ring, zs_zq.data(), vol);
    }
    volume_output_d_kernel<<<1024, 256, 0, st>>>(vol, g, nv, nn * nz, d_mag, d_ph);
    MRSIM_CUDA(cudaGetLastError());
    MRSIM_CUDA(cudaStreamSynchronize(st));
  }
  copy_pageable_d2h(ctx, mag, d_mag, nn * nz * nv * 4, st);
  copy_pageable_d2h(ctx, ph, d_ph, nn * nz * nv * 4, st);
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

}  // namespace mrsim
