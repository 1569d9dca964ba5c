// motion.cu — rigid image motion on the device: `resample_by_pose` (motion.rs:430-460),
// `apply_motion` (motion.rs:466-482) and `apply_multiband_motion(_slab)` (motion.rs:666-772), the
// image preparation that runs before the k-space forward.  Each output voxel is backward-mapped
// through the pose in FP64 in the reference's operation order (no contracted multiply-adds) and
// sampled trilinearly in FP64 from the f32 source (`trilinear`, motion.rs:390-410), so the
// result equals the reference's bit for bit.  The operator variant resamples an EPI operator's
// device images in place, so moved series reach the forward without a host round trip.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <vector>

#include "driver.h"
#include "motion.h"
#include "mrsim_internal.h"

namespace mrsim {

namespace {

// The backward map of one pose (world mm): hv = linv (Rt (lin p + origin - c - t) + c - origin).
struct PoseMap {
  double lin[9], rt[9], linv[9];
  double origin[3], c[3], t[3];
  int moved;  // 0: the identity pose or a singular grid (the source is copied)
  int pad;
};

__device__ __forceinline__ void matvec_rn(const double* m, double x, double y, double z, double* o) {
  // ((m0 x + m1 y) + m2 z), each product and sum rounded once
  for (int r = 0; r < 3; ++r)
    o[r] = __dadd_rn(__dadd_rn(__dmul_rn(m[3 * r], x), __dmul_rn(m[3 * r + 1], y)), __dmul_rn(m[3 * r + 2], z));
}

// Element (x, y, z) of one volume: base + x sx + y sy + z sz.
struct VolView {
  const float* base;
  long long sx, sy, sz;
};

__device__ __forceinline__ double lerp_rn(double a, double b, double t) { return __dadd_rn(a, __dmul_rn(__dsub_rn(b, a), t)); }

__device__ float trilinear_dev(const VolView& v, int nx, int ny, int nz, double px, double py, double pz) {
  if (px < -0.5 || px > (double)nx - 0.5 || py < -0.5 || py > (double)ny - 0.5 || pz < -0.5 || pz > (double)nz - 0.5)
    return 0.0f;
  const double x = px < 0.0 ? 0.0 : (px > (double)(nx - 1) ? (double)(nx - 1) : px);
  const double y = py < 0.0 ? 0.0 : (py > (double)(ny - 1) ? (double)(ny - 1) : py);
  const double z = pz < 0.0 ? 0.0 : (pz > (double)(nz - 1) ? (double)(nz - 1) : pz);
  const int x0 = (int)floor(x), y0 = (int)floor(y), z0 = (int)floor(z);
  const int x1 = min(x0 + 1, nx - 1), y1 = min(y0 + 1, ny - 1), z1 = min(z0 + 1, nz - 1);
  const double fx = __dsub_rn(x, (double)x0), fy = __dsub_rn(y, (double)y0), fz = __dsub_rn(z, (double)z0);
  auto at = [&](int xi, int yi, int zi) { return (double)__ldg(v.base + xi * v.sx + yi * v.sy + zi * v.sz); };
  const double c00 = lerp_rn(at(x0, y0, z0), at(x1, y0, z0), fx);
  const double c10 = lerp_rn(at(x0, y1, z0), at(x1, y1, z0), fx);
  const double c01 = lerp_rn(at(x0, y0, z1), at(x1, y0, z1), fx);
  const double c11 = lerp_rn(at(x0, y1, z1), at(x1, y1, z1), fx);
  return (float)lerp_rn(lerp_rn(c00, c10, fy), lerp_rn(c01, c11, fy), fz);
}

__device__ float resample_voxel(const PoseMap& P, const VolView& v, int nx, int ny, int nz, int x, int y, int z) {
  double w[3], pr[3], hv[3];
  matvec_rn(P.lin, (double)x, (double)y, (double)z, w);
  const double d0 = __dsub_rn(__dsub_rn(__dadd_rn(w[0], P.origin[0]), P.c[0]), P.t[0]);
  const double d1 = __dsub_rn(__dsub_rn(__dadd_rn(w[1], P.origin[1]), P.c[1]), P.t[1]);
  const double d2 = __dsub_rn(__dsub_rn(__dadd_rn(w[2], P.origin[2]), P.c[2]), P.t[2]);
  matvec_rn(P.rt, d0, d1, d2, pr);
  matvec_rn(P.linv, __dsub_rn(__dadd_rn(pr[0], P.c[0]), P.origin[0]), __dsub_rn(__dadd_rn(pr[1], P.c[1]), P.origin[1]),
            __dsub_rn(__dadd_rn(pr[2], P.c[2]), P.origin[2]), hv);
  return trilinear_dev(v, nx, ny, nz, hv[0], hv[1], hv[2]);
}

// Every (voxel, volume, compartment) of a batch: out[c] (volume g) = volume g of in[c] resampled by
// pose g (a copy where the pose does not move).  The layouts are strided views:
//   element (x, y, z) of volume g, compartment c at base_c + x sx + y sy + z sz + g sg + c sc.
struct BatchLayout {
  const float* in;
  float* out;
  long long sx, sy, sz, sg, sc;
};

__global__ void resample_batch_kernel(BatchLayout L, const PoseMap* __restrict__ poses, int nx, int ny, int nz, int nv,
                                      int ncomp) {
  const long long nvox = (long long)nx * ny * nz;
  const long long total = nvox * nv * ncomp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    // voxel fastest, then volume, then compartment
    const long long vox = e % nvox;
    const int g = (int)((e / nvox) % nv), c = (int)(e / (nvox * nv));
    const int x = (int)(vox % nx), y = (int)((vox / nx) % ny), z = (int)(vox / ((long long)nx * ny));
    const long long off = x * L.sx + y * L.sy + z * L.sz + g * L.sg + c * L.sc;
    const PoseMap& P = poses[g];
    if (!P.moved) {
      L.out[off] = L.in[off];
      continue;
    }
    VolView v{L.in + g * L.sg + c * L.sc, L.sx, L.sy, L.sz};
    L.out[off] = resample_voxel(P, v, nx, ny, nz, x, y, z);
  }
}

// The multiband pass over one batch: for each (voxel, affected volume, compartment) the slice's
// shot decides the pose (resampled from the pre-motion input) and the attenuation factors,
// multiplied in event order.
struct ShotTables {
  const int* volume;        // [n_aff] the volume of each affected entry
  const int* shot_of_z;     // [nz] local slice -> shot (-1: none)
  const int* pose_index;    // [n_aff][n_shots] index into poses, -1 for the identity
  const int* fac_start;     // [n_aff][n_shots + 1] offsets into factors
  const float* factors;
  int n_shots;
};

__global__ void multiband_kernel(BatchLayout L, ShotTables S, const PoseMap* __restrict__ poses, int nx, int ny, int nz,
                                 int n_aff, int ncomp) {
  const long long nvox = (long long)nx * ny * nz;
  const long long total = nvox * n_aff * ncomp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long vox = e % nvox;
    const int a = (int)((e / nvox) % n_aff), c = (int)(e / (nvox * n_aff));
    const int g = S.volume[a];
    const int x = (int)(vox % nx), y = (int)((vox / nx) % ny), z = (int)(vox / ((long long)nx * ny));
    const long long off = x * L.sx + y * L.sy + z * L.sz + g * L.sg + c * L.sc;
    const int k = S.shot_of_z[z];
    float v = L.in[off];
    if (k >= 0) {
      const int pi = S.pose_index[a * S.n_shots + k];
      if (pi >= 0) {
        VolView vv{L.in + g * L.sg + c * L.sc, L.sx, L.sy, L.sz};
        v = resample_voxel(poses[pi], vv, nx, ny, nz, x, y, z);
      }
      const int f0 = S.fac_start[a * (S.n_shots + 1) + k], f1 = S.fac_start[a * (S.n_shots + 1) + k + 1];
      for (int f = f0; f < f1; ++f) v *= S.factors[f];
    }
    L.out[off] = v;
  }
}

// ---- host ------------------------------------------------------------------------------------
using M3 = std::array<std::array<double, 3>, 3>;

M3 matmul3(const M3& a, const M3& b) {
  M3 o{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) o[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
  return o;
}

// `mat::rotation_zyx_deg` (mat.rs:69-75): Rz Ry Rx, angles in degrees
M3 rotation_zyx_deg(double rx, double ry, double rz) {
  rx *= M_PI / 180.0;  // f64::to_radians
  ry *= M_PI / 180.0;
  rz *= M_PI / 180.0;
  M3 X = {{{1.0, 0.0, 0.0}, {0.0, std::cos(rx), -std::sin(rx)}, {0.0, std::sin(rx), std::cos(rx)}}};
  M3 Y = {{{std::cos(ry), 0.0, std::sin(ry)}, {0.0, 1.0, 0.0}, {-std::sin(ry), 0.0, std::cos(ry)}}};
  M3 Z = {{{std::cos(rz), -std::sin(rz), 0.0}, {std::sin(rz), std::cos(rz), 0.0}, {0.0, 0.0, 1.0}}};
  return matmul3(Z, matmul3(Y, X));
}

bool pose_identity(const double* p) {
  for (int i = 0; i < 6; ++i)
    if (p[i] != 0.0) return false;
  return true;
}

}  // namespace

// The backward map of `pose` (rot_deg[3], trans_mm[3]) on a grid: what `resample_by_pose` forms
// before its voxel loop (fov_center motion.rs:412-418, mat::inverse3 mat.rs:78-103).
static PoseMap make_pose_map(const int64_t* dims, const double* v2w, const double* pose) {
  PoseMap P;
  std::memset(&P, 0, sizeof P);
  if (pose_identity(pose)) return P;
  const double m[9] = {v2w[0], v2w[1], v2w[2], v2w[4], v2w[5], v2w[6], v2w[8], v2w[9], v2w[10]};
  const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                     m[2] * (m[3] * m[7] - m[4] * m[6]);
  if (std::fabs(det) < 1e-18) return P;
  const double inv = 1.0 / det;
  const double li[9] = {(m[4] * m[8] - m[5] * m[7]) * inv, (m[2] * m[7] - m[1] * m[8]) * inv,
                        (m[1] * m[5] - m[2] * m[4]) * inv, (m[5] * m[6] - m[3] * m[8]) * inv,
                        (m[0] * m[8] - m[2] * m[6]) * inv, (m[2] * m[3] - m[0] * m[5]) * inv,
                        (m[3] * m[7] - m[4] * m[6]) * inv, (m[1] * m[6] - m[0] * m[7]) * inv,
                        (m[0] * m[4] - m[1] * m[3]) * inv};
  const double hx = ((double)dims[0] - 1.0) / 2.0, hy = ((double)dims[1] - 1.0) / 2.0, hz = ((double)dims[2] - 1.0) / 2.0;
  const double cx = m[0] * hx + m[1] * hy + m[2] * hz, cy = m[3] * hx + m[4] * hy + m[5] * hz,
               cz = m[6] * hx + m[7] * hy + m[8] * hz;
  const M3 R = rotation_zyx_deg(pose[0], pose[1], pose[2]);
  for (int i = 0; i < 9; ++i) {
    P.lin[i] = m[i];
    P.linv[i] = li[i];
  }
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) P.rt[3 * r + c] = R[c][r];
  P.origin[0] = v2w[3];
  P.origin[1] = v2w[7];
  P.origin[2] = v2w[11];
  P.c[0] = cx + v2w[3];
  P.c[1] = cy + v2w[7];
  P.c[2] = cz + v2w[11];
  for (int i = 0; i < 3; ++i) P.t[i] = pose[3 + i];
  P.moved = 1;
  return P;
}

static unsigned grid_for(long long n) { return (unsigned)std::max(1LL, std::min((n + 255) / 256, 148LL * 32)); }

void resample_poses_device(const float* in, float* out, const int64_t* dims, int nv, int ncomp, long long sx,
                           long long sy, long long sz, long long sg, long long sc, const double* v2w,
                           const double* poses, cudaStream_t st, DevArena& arena) {
  std::vector<PoseMap> maps(nv);
  for (int g = 0; g < nv; ++g) maps[g] = make_pose_map(dims, v2w, poses + 6 * (size_t)g);
  const PoseMap* d = (const PoseMap*)arena.upload(maps.data(), maps.size() * sizeof(PoseMap), st);
  BatchLayout L{in, out, sx, sy, sz, sg, sc};
  const long long n = dims[0] * dims[1] * dims[2] * (long long)nv * ncomp;
  resample_batch_kernel<<<grid_for(n), 256, 0, st>>>(L, d, (int)dims[0], (int)dims[1], (int)dims[2], nv, ncomp);
  MRSIM_CUDA(cudaGetLastError());
}

// `slice_schedule` motion.rs:486-500
std::vector<std::vector<int64_t>> slice_schedule(int64_t nz, int64_t mb, bool interleaved) {
  mb = std::max<int64_t>(mb, 1);
  const int64_t ng = nz / mb;
  if (ng == 0) {
    std::vector<int64_t> all(nz);
    for (int64_t z = 0; z < nz; ++z) all[z] = z;
    return {all};
  }
  std::vector<int64_t> order;
  for (int64_t g = 0; g < ng; g += interleaved ? 2 : 1) order.push_back(g);
  if (interleaved)
    for (int64_t g = 1; g < ng; g += 2) order.push_back(g);
  std::vector<std::vector<int64_t>> out;
  for (int64_t gi : order) {
    std::vector<int64_t> s;
    for (int64_t j = 0; j < mb; ++j)
      if (gi + j * ng < nz) s.push_back(gi + j * ng);
    out.push_back(s);
  }
  return out;
}

// `DropoutLaw::attenuation` motion.rs:641-662
float dropout_attenuation(const mrsim_dropout_law& law, int64_t volume, float severity) {
  if (law.kind == MRSIM_DROPOUT_UNIFORM) return 1.0f - severity;
  const double d = (law.drive && volume < law.n_drive) ? law.drive[volume] : 0.0;
  if (law.kind == MRSIM_DROPOUT_SCALED) {
    double dmax = 0.0;
    for (int64_t i = 0; i < law.n_drive; ++i) dmax = std::fmax(dmax, law.drive[i]);
    if (d < law.floor || dmax <= 0.0) return 1.0f;
    return 1.0f - severity * (float)(d / dmax);
  }
  if (d < law.floor || law.max <= 0.0) return 1.0f;
  return 1.0f - severity * (float)(d / law.max);
}

int64_t multiband_device(const float* in, float* out, const int64_t* dims, int nv, int ncomp, long long sx, long long sy,
                         long long sz, long long sg, long long sc, const double* v2w, int64_t mb, bool interleaved,
                         const mrsim_dropout_law& law, const mrsim_motion_event* events, int64_t n_events,
                         const int64_t* slice_z, int64_t nz_full, mrsim_dropped_shot* dropped, int64_t capacity,
                         cudaStream_t st, DevArena& arena) {
  const int64_t nz = dims[2];
  if (nz_full <= 0) nz_full = nz;
  if (slice_z)
    for (int64_t i = 0; i < nz; ++i)
      if (slice_z[i] < 0 || slice_z[i] >= nz_full) fail("slice_z names a slice outside the full volume");
  const auto full = slice_schedule(nz_full, mb, interleaved);
  const int n_shots = (int)full.size();
  std::vector<int> shot_of_z(nz, -1);
  for (int k = 0; k < n_shots; ++k)
    for (int64_t zg : full[k]) {
      int64_t local = -1;
      if (!slice_z) {
        if (zg < nz) local = zg;
      } else {
        for (int64_t i = 0; i < nz; ++i)
          if (slice_z[i] == zg) {
            local = i;
            break;
          }
      }
      if (local >= 0) shot_of_z[local] = k;
    }
  std::vector<int> vol, pose_index, fac_start;
  std::vector<float> factors;
  std::vector<PoseMap> maps;
  int64_t nd = 0;
  for (int64_t g = 0; g < nv; ++g) {
    std::vector<int64_t> evs;
    for (int64_t e = 0; e < n_events; ++e)
      if (events[e].volume == g && events[e].shot < n_shots && events[e].shot >= 0) evs.push_back(e);
    if (evs.empty()) continue;
    vol.push_back((int)g);
    double cum[6] = {0, 0, 0, 0, 0, 0};
    for (int k = 0; k < n_shots; ++k) {
      for (int64_t e : evs)
        if (events[e].shot == k)
          for (int i = 0; i < 3; ++i) {
            cum[3 + i] += events[e].jump_mm[i];
            cum[i] += events[e].jump_deg[i];
          }
      if (pose_identity(cum)) {
        pose_index.push_back(-1);
      } else {
        pose_index.push_back((int)maps.size());
        maps.push_back(make_pose_map(dims, v2w, cum));
        if (!maps.back().moved) pose_index.back() = -1;
      }
    }
    // factors per shot in event order
    std::vector<std::vector<float>> per(n_shots);
    for (int64_t e : evs) {
      const float a = dropout_attenuation(law, g, events[e].severity);
      per[events[e].shot].push_back(a);
      if (dropped && nd < capacity) {
        mrsim_dropped_shot& d = dropped[nd];
        std::memset(&d, 0, sizeof d);
        d.volume = g;
        d.shot = events[e].shot;
        d.attenuation = a;
        d.n_slices = (int64_t)std::min<size_t>(full[d.shot].size(), 64);
        for (int64_t i = 0; i < d.n_slices; ++i) d.slices[i] = full[d.shot][i];
      }
      ++nd;
    }
    for (int k = 0; k < n_shots; ++k) {
      fac_start.push_back((int)factors.size());
      factors.insert(factors.end(), per[k].begin(), per[k].end());
    }
    fac_start.push_back((int)factors.size());
  }
  if (dropped && nd > capacity) fail("the dropped-shot list needs " + std::to_string(nd) + " entries, capacity " +
                                     std::to_string(capacity));
  const long long nvox = dims[0] * dims[1] * dims[2];
  if (in != out) {  // volumes without events are copied
    BatchLayout L{in, out, sx, sy, sz, sg, sc};
    std::vector<PoseMap> ident(nv);
    std::memset(ident.data(), 0, ident.size() * sizeof(PoseMap));
    const PoseMap* d = (const PoseMap*)arena.upload(ident.data(), ident.size() * sizeof(PoseMap), st);
    resample_batch_kernel<<<grid_for(nvox * nv * ncomp), 256, 0, st>>>(L, d, (int)dims[0], (int)dims[1], (int)dims[2],
                                                                       nv, ncomp);
    MRSIM_CUDA(cudaGetLastError());
  }
  if (!vol.empty()) {
    ShotTables S;
    S.volume = (const int*)arena.upload(vol.data(), vol.size() * 4, st);
    S.shot_of_z = (const int*)arena.upload(shot_of_z.data(), shot_of_z.size() * 4, st);
    S.pose_index = (const int*)arena.upload(pose_index.data(), pose_index.size() * 4, st);
    S.fac_start = (const int*)arena.upload(fac_start.data(), fac_start.size() * 4, st);
    S.factors = factors.empty() ? nullptr : (const float*)arena.upload(factors.data(), factors.size() * 4, st);
    S.n_shots = n_shots;
    const PoseMap* d =
        maps.empty() ? nullptr : (const PoseMap*)arena.upload(maps.data(), maps.size() * sizeof(PoseMap), st);
    BatchLayout L{in, out, sx, sy, sz, sg, sc};
    multiband_kernel<<<grid_for(nvox * (long long)vol.size() * ncomp), 256, 0, st>>>(
        L, S, d, (int)dims[0], (int)dims[1], (int)dims[2], (int)vol.size(), ncomp);
    MRSIM_CUDA(cudaGetLastError());
  }
  return nd;
}

}  // namespace mrsim
