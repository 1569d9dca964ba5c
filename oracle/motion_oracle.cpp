// motion_oracle.cpp — TEST INFRASTRUCTURE ONLY: an FP64 C++ restatement of the reference's image
// motion (Rust `mrsim-acq` src/motion.rs and src/mat.rs), the parity checker of the device
// resampling.  Nothing in the product links, loads or calls it.  Compiled with -ffp-contract=off
// (Rust never fuses multiply-adds) into liboracle, the reference's operation order kept so the
// results are the reference's bit for bit; pinned by the reference's own motion tests
// (tests/test_oracle_motion.py).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using V3 = std::array<double, 3>;
using M3 = std::array<std::array<double, 3>, 3>;

// `mat::matvec` mat.rs:39-45
V3 matvec(const M3& m, const V3& v) {
  return {m[0][0] * v[0] + m[0][1] * v[1] + m[0][2] * v[2], m[1][0] * v[0] + m[1][1] * v[1] + m[1][2] * v[2],
          m[2][0] * v[0] + m[2][1] * v[1] + m[2][2] * v[2]};
}
// `mat::matmul` mat.rs:47-55
M3 matmul(const M3& a, const M3& b) {
  M3 o{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) o[i][j] = a[i][0] * b[0][j] + a[i][1] * b[1][j] + a[i][2] * b[2][j];
  return o;
}
// `mat::transpose` mat.rs:57-65
M3 transpose(const M3& a) {
  M3 o{};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) o[i][j] = a[j][i];
  return o;
}
double to_radians(double d) { return d * (M_PI / 180.0); }
// `mat::rotation_zyx_deg` mat.rs:69-75: Rz Ry Rx
M3 rotation_zyx_deg(double rx, double ry, double rz) {
  rx = to_radians(rx);
  ry = to_radians(ry);
  rz = to_radians(rz);
  M3 X = {{{1.0, 0.0, 0.0}, {0.0, std::cos(rx), -std::sin(rx)}, {0.0, std::sin(rx), std::cos(rx)}}};
  M3 Y = {{{std::cos(ry), 0.0, std::sin(ry)}, {0.0, 1.0, 0.0}, {-std::sin(ry), 0.0, std::cos(ry)}}};
  M3 Z = {{{std::cos(rz), -std::sin(rz), 0.0}, {std::sin(rz), std::cos(rz), 0.0}, {0.0, 0.0, 1.0}}};
  return matmul(Z, matmul(Y, X));
}
// `mat::inverse3` mat.rs:78-103 (adjugate / determinant; false if |det| < 1e-18)
bool inverse3(const M3& m, M3& out) {
  const double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                     m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                     m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
  if (std::fabs(det) < 1e-18) return false;
  const double inv = 1.0 / det;
  out = {{{(m[1][1] * m[2][2] - m[1][2] * m[2][1]) * inv, (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * inv,
           (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * inv},
          {(m[1][2] * m[2][0] - m[1][0] * m[2][2]) * inv, (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * inv,
           (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * inv},
          {(m[1][0] * m[2][1] - m[1][1] * m[2][0]) * inv, (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * inv,
           (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * inv}}};
  return true;
}
double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

// `trilinear` motion.rs:390-410
float trilinear(const float* vol, const int64_t* dims, const V3& p) {
  const int64_t nx = dims[0], ny = dims[1], nz = dims[2];
  auto outside = [](double c, int64_t n) { return c < -0.5 || c > (double)n - 0.5; };
  if (outside(p[0], nx) || outside(p[1], ny) || outside(p[2], nz)) return 0.0f;
  const double x = clampd(p[0], 0.0, (double)(nx - 1)), y = clampd(p[1], 0.0, (double)(ny - 1)),
               z = clampd(p[2], 0.0, (double)(nz - 1));
  const int64_t x0 = (int64_t)std::floor(x), y0 = (int64_t)std::floor(y), z0 = (int64_t)std::floor(z);
  const int64_t x1 = std::min(x0 + 1, nx - 1), y1 = std::min(y0 + 1, ny - 1), z1 = std::min(z0 + 1, nz - 1);
  const double fx = x - (double)x0, fy = y - (double)y0, fz = z - (double)z0;
  auto at = [&](int64_t xi, int64_t yi, int64_t zi) { return (double)vol[xi + nx * (yi + ny * zi)]; };
  auto lerp = [](double a, double b, double t) { return a + (b - a) * t; };
  const double c00 = lerp(at(x0, y0, z0), at(x1, y0, z0), fx);
  const double c10 = lerp(at(x0, y1, z0), at(x1, y1, z0), fx);
  const double c01 = lerp(at(x0, y0, z1), at(x1, y0, z1), fx);
  const double c11 = lerp(at(x0, y1, z1), at(x1, y1, z1), fx);
  return (float)lerp(lerp(c00, c10, fy), lerp(c01, c11, fy), fz);
}

M3 linear3(const double* v) { return {{{v[0], v[1], v[2]}, {v[4], v[5], v[6]}, {v[8], v[9], v[10]}}}; }

// `fov_center` motion.rs:412-418
V3 fov_center(const int64_t* dims, const double* v2w) {
  const M3 lin = linear3(v2w);
  const V3 c = matvec(lin, {((double)dims[0] - 1.0) / 2.0, ((double)dims[1] - 1.0) / 2.0, ((double)dims[2] - 1.0) / 2.0});
  return {c[0] + v2w[3], c[1] + v2w[7], c[2] + v2w[11]};
}

bool is_identity(const double* pose) {
  for (int i = 0; i < 6; ++i)
    if (pose[i] != 0.0) return false;
  return true;
}

// `resample_by_pose` motion.rs:430-460 (pose = rot_deg[3], trans_mm[3])
std::vector<float> resample_by_pose(const float* src, const int64_t* dims, const double* v2w, const double* pose) {
  const int64_t nx = dims[0], ny = dims[1], nz = dims[2], nvox = nx * ny * nz;
  if (is_identity(pose)) return std::vector<float>(src, src + nvox);
  const M3 lin = linear3(v2w);
  const V3 origin = {v2w[3], v2w[7], v2w[11]};
  M3 linv;
  if (!inverse3(lin, linv)) return std::vector<float>(src, src + nvox);
  const V3 c = fov_center(dims, v2w);
  const M3 rt = transpose(rotation_zyx_deg(pose[0], pose[1], pose[2]));
  const V3 t = {pose[3], pose[4], pose[5]};
  std::vector<float> out(nvox, 0.0f);
  for (int64_t z = 0; z < nz; ++z)
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t x = 0; x < nx; ++x) {
        const V3 w = matvec(lin, {(double)x, (double)y, (double)z});
        const V3 wv = {w[0] + origin[0], w[1] + origin[1], w[2] + origin[2]};
        const V3 d = {wv[0] - c[0] - t[0], wv[1] - c[1] - t[1], wv[2] - c[2] - t[2]};
        const V3 pr = matvec(rt, d);
        const V3 hv = matvec(linv, {pr[0] + c[0] - origin[0], pr[1] + c[1] - origin[1], pr[2] + c[2] - origin[2]});
        out[x + nx * (y + ny * z)] = trilinear(src, dims, hv);
      }
  return out;
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
  if (interleaved) {
    for (int64_t g = 0; g < ng; g += 2) order.push_back(g);
    for (int64_t g = 1; g < ng; g += 2) order.push_back(g);
  } else {
    for (int64_t g = 0; g < ng; ++g) order.push_back(g);
  }
  std::vector<std::vector<int64_t>> out;
  for (int64_t gi : order) {
    std::vector<int64_t> s;
    for (int64_t j = 0; j < mb; ++j)
      if (gi + j * ng < nz) s.push_back(gi + j * ng);
    out.push_back(s);
  }
  return out;
}

// `DropoutLaw::attenuation` motion.rs:641-662 (kind 0 Uniform, 1 Scaled, 2 ScaledTo)
float attenuation(int kind, const double* drive, int64_t n_drive, double floor_, double max_, int64_t volume,
                  float severity) {
  if (kind == 0) return 1.0f - severity;
  const double d = volume < n_drive ? drive[volume] : 0.0;
  if (kind == 1) {
    double dmax = 0.0;
    for (int64_t i = 0; i < n_drive; ++i) dmax = std::fmax(dmax, drive[i]);
    if (d < floor_ || dmax <= 0.0) return 1.0f;
    return 1.0f - severity * (float)(d / dmax);
  }
  if (d < floor_ || max_ <= 0.0) return 1.0f;
  return 1.0f - severity * (float)(d / max_);
}

}  // namespace

extern "C" {

int oracle_motion_trilinear(const float* vol, const int64_t* dims, const double* p, float* out) {
  *out = trilinear(vol, dims, {p[0], p[1], p[2]});
  return 0;
}

int oracle_resample_by_pose(const float* src, const int64_t* dims, const double* v2w, const double* pose, float* out) {
  auto r = resample_by_pose(src, dims, v2w, pose);
  std::memcpy(out, r.data(), r.size() * sizeof(float));
  return 0;
}

// `apply_motion` motion.rs:466-482: images[c][vox * ngrad + g], in place
int oracle_apply_motion(float* const* images, int64_t ncomp, const int64_t* dims, int64_t ngrad, const double* v2w,
                        const double* poses) {
  const int64_t nvox = dims[0] * dims[1] * dims[2];
  for (int64_t g = 0; g < ngrad; ++g) {
    const double* pose = poses + 6 * g;
    if (is_identity(pose)) continue;
    for (int64_t c = 0; c < ncomp; ++c) {
      std::vector<float> src(nvox);
      for (int64_t v = 0; v < nvox; ++v) src[v] = images[c][v * ngrad + g];
      auto moved = resample_by_pose(src.data(), dims, v2w, pose);
      for (int64_t v = 0; v < nvox; ++v) images[c][v * ngrad + g] = moved[v];
    }
  }
  return 0;
}

// `apply_multiband_motion_slab` motion.rs:686-772, in place; events as parallel arrays.  Writes
// the dropped shots as (volume, shot, attenuation) into the given arrays (capacity n_events)
// and their count to *n_dropped.
int oracle_apply_multiband_motion(float* const* images, int64_t ncomp, const int64_t* dims, int64_t ngrad,
                                  const double* v2w, int64_t mb, int32_t interleaved, int32_t law_kind,
                                  const double* drive, int64_t n_drive, double floor_, double max_,
                                  const int64_t* ev_volume, const int64_t* ev_shot, const float* ev_severity,
                                  const double* ev_jump_mm, const double* ev_jump_deg, int64_t n_events,
                                  const int64_t* slice_z, int64_t nz_full, int64_t* dropped_volume,
                                  int64_t* dropped_shot, float* dropped_atten, int64_t* n_dropped) {
  const int64_t nx = dims[0], ny = dims[1], nz = dims[2], nvox = nx * ny * nz;
  if (nz_full <= 0) nz_full = nz;
  auto full = slice_schedule(nz_full, mb, interleaved != 0);
  std::vector<std::vector<int64_t>> sched;
  for (auto& shot : full) {
    std::vector<int64_t> loc;
    for (int64_t zg : shot) {
      if (!slice_z) {
        if (zg < nz) loc.push_back(zg);
      } else {
        for (int64_t i = 0; i < nz; ++i)
          if (slice_z[i] == zg) {
            loc.push_back(i);
            break;
          }
      }
    }
    sched.push_back(loc);
  }
  const int64_t n_shots = (int64_t)sched.size();
  auto at3 = [&](int64_t x, int64_t y, int64_t z) { return x + nx * (y + ny * z); };
  int64_t nd = 0;
  for (int64_t g = 0; g < ngrad; ++g) {
    std::vector<int64_t> evs;
    for (int64_t e = 0; e < n_events; ++e)
      if (ev_volume[e] == g && ev_shot[e] < n_shots) evs.push_back(e);
    if (evs.empty()) continue;
    std::vector<std::array<double, 6>> shot_pose(n_shots);
    std::array<double, 6> cum = {0, 0, 0, 0, 0, 0};
    for (int64_t k = 0; k < n_shots; ++k) {
      for (int64_t e : evs)
        if (ev_shot[e] == k)
          for (int i = 0; i < 3; ++i) {
            cum[3 + i] += ev_jump_mm[3 * e + i];
            cum[i] += ev_jump_deg[3 * e + i];
          }
      shot_pose[k] = cum;
    }
    bool any = false;
    for (auto& p : shot_pose) any = any || !is_identity(p.data());
    if (any)
      for (int64_t c = 0; c < ncomp; ++c) {
        std::vector<float> orig(nvox);
        for (int64_t v = 0; v < nvox; ++v) orig[v] = images[c][v * ngrad + g];
        for (int64_t k = 0; k < n_shots; ++k) {
          if (is_identity(shot_pose[k].data())) continue;
          auto rs = resample_by_pose(orig.data(), dims, v2w, shot_pose[k].data());
          for (int64_t z : sched[k])
            for (int64_t y = 0; y < ny; ++y)
              for (int64_t x = 0; x < nx; ++x) images[c][at3(x, y, z) * ngrad + g] = rs[at3(x, y, z)];
        }
      }
    for (int64_t e : evs) {
      const float a = attenuation(law_kind, drive, n_drive, floor_, max_, g, ev_severity[e]);
      for (int64_t c = 0; c < ncomp; ++c)
        for (int64_t z : sched[ev_shot[e]])
          for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) images[c][at3(x, y, z) * ngrad + g] *= a;
      dropped_volume[nd] = g;
      dropped_shot[nd] = ev_shot[e];
      dropped_atten[nd] = a;
      ++nd;
    }
  }
  *n_dropped = nd;
  return 0;
}

}  // extern "C"
