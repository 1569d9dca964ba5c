// spin_history_oracle.cpp — TEST INFRASTRUCTURE ONLY: an FP64 C++ restatement of the reference's
// spin history (Rust `mrsim-acq` src/spin_history.rs), the parity checker of the device spin
// history.  Nothing in the product links, loads or calls it.  Compiled with -ffp-contract=off
// (Rust never fuses multiply-adds) into liboracle; the reference's operation order is kept (f32
// piece edges and magnetisations, f64 times and terms, the plane-ordered f64 sums rounded to f32
// once).  Pinned by the reference's own spin-history tests, restated in
// tests/test_oracle_spin_history.py (known answers: the double-excitation dip, the skip, the
// presaturation reference, merges).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/mrsim_acq.h"

namespace {

constexpr int kMaxPieces = MRSIM_SPIN_MAX_PIECES;  // `MAX_PIECES` spin_history.rs:37
constexpr double kSnap = 1e-6;                     // `SNAP` spin_history.rs:40
constexpr uint8_t kNoClass = MRSIM_SPIN_NO_CLASS;  // `NO_CLASS` spin_history.rs:34

using M4 = std::array<std::array<double, 4>, 4>;

struct Pulse {
  int kind;  // MRSIM_PULSE_*
  double t, eps;
};

// `replay` spin_history.rs:232-251: Mz at t_to from mz just after t_from, through the pulses in
// (t_from, t_to] (sorted by time); 0 when T1 <= 0.
double replay(double mz, double t_from, double t_to, double t1, const Pulse* P, size_t np) {
  if (t1 <= 0.0) return 0.0;
  auto recover = [&](double m, double dt) { return std::isinf(dt) ? 1.0 : 1.0 - (1.0 - m) * std::exp(-dt / t1); };
  size_t lo = 0, hi = np;  // partition_point(p.t <= t_from)
  while (lo < hi) {
    const size_t mid = (lo + hi) / 2;
    if (P[mid].t <= t_from)
      lo = mid + 1;
    else
      hi = mid;
  }
  double m = mz, t = t_from;
  for (size_t i = lo; i < np; ++i) {
    const double tp = P[i].t;
    if (tp > t_to) break;
    m = recover(m, tp - t);
    m = P[i].kind == MRSIM_PULSE_INVERSION ? m * (1.0 - 2.0 * P[i].eps) : 0.0;
    t = tp;
  }
  return recover(m, t_to - t);
}

// `Pieces` spin_history.rs:87-165: piece i covers [start[i], start[i+1]) of the voxel's [0, 1).
struct Pieces {
  int n = 1;
  float start[kMaxPieces];
  float mz[kMaxPieces];
  double t[kMaxPieces];
  static Pieces relaxed() {
    Pieces p;
    for (int i = 0; i < kMaxPieces; ++i) {
      p.start[i] = 0.0f;
      p.mz[i] = 1.0f;
      p.t[i] = -std::numeric_limits<double>::infinity();
    }
    p.n = 1;
    return p;
  }
  float end(int i) const { return i + 1 < n ? start[i + 1] : 1.0f; }
  bool split(float u) {
    int i = -1;
    for (int k = 0; k < n; ++k)
      if (start[k] < u && u < end(k)) {
        i = k;
        break;
      }
    if (i < 0) return true;
    if (n == kMaxPieces) return false;
    for (int j = n - 1; j >= i + 1; --j) {
      start[j + 1] = start[j];
      mz[j + 1] = mz[j];
      t[j + 1] = t[j];
    }
    start[i + 1] = u;
    mz[i + 1] = mz[i];
    t[i + 1] = t[i];
    ++n;
    return true;
  }
  bool has_edge(float u) const {
    for (int i = 0; i < n; ++i)
      if (start[i] == u) return true;
    return false;
  }
  void remove(int i) {
    for (int j = i; j < n - 1; ++j) {
      start[j] = start[j + 1];
      mz[j] = mz[j + 1];
      t[j] = t[j + 1];
    }
    --n;
  }
  void coalesce() {
    int i = 1;
    while (i < n) {
      if (mz[i] == mz[i - 1] && t[i] == t[i - 1])
        remove(i);
      else
        ++i;
    }
  }
};

// `merge_closest` spin_history.rs:426-452
void merge_closest(Pieces& pc, double t1, const Pulse* P, size_t np, const float* protect, int nprot) {
  const int n = pc.n;
  auto len = [&](int i) { return (double)(pc.end(i) - pc.start[i]); };
  auto cost = [&](int i) {
    const double d = (double)std::fabs(pc.mz[i] - pc.mz[i - 1]) + std::fmin(std::fabs(pc.t[i] - pc.t[i - 1]), 1e6);
    return d * len(i) * len(i - 1) / (len(i) + len(i - 1));
  };
  int best = -1;
  double best_cost = 0.0;
  for (int i = 1; i < n; ++i) {
    bool prot = false;
    for (int q = 0; q < nprot; ++q)
      if (protect[q] == pc.start[i]) prot = true;
    if (prot) continue;
    const double c = cost(i);
    if (best < 0 || c < best_cost) {
      best = i;
      best_cost = c;
    }
  }
  if (best < 0) throw std::runtime_error("a full voxel has an unprotected edge to merge");
  const float la = pc.end(best - 1) - pc.start[best - 1], lb = pc.end(best) - pc.start[best];
  const double ta = pc.t[best - 1], tb = pc.t[best];
  const double t = std::fmax(ta, tb);
  auto at = [&](float mz, double from) { return from == t ? (double)mz : replay((double)mz, from, t, t1, P, np); };
  const double ma = at(pc.mz[best - 1], ta), mb = at(pc.mz[best], tb);
  pc.mz[best - 1] = (float)((ma * (double)la + mb * (double)lb) / (double)(la + lb));
  pc.t[best - 1] = t;
  pc.remove(best);
}

// `Pieces::cut` spin_history.rs:115-131
uint64_t cut(Pieces& pc, float u0, float u1, double t1, const Pulse* P, size_t np) {
  auto needs = [&]() {
    int c = 0;
    for (float u : {u0, u1})
      if (u > 0.0f && u < 1.0f && !pc.has_edge(u)) ++c;
    return c;
  };
  uint64_t merges = 0;
  const float prot[2] = {u0, u1};
  while (pc.n + needs() > kMaxPieces) {
    ++merges;
    merge_closest(pc, t1, P, np, prot, 2);
  }
  for (float u : {u0, u1})
    if (u > 0.0f && u < 1.0f) pc.split(u);
  return merges;
}

double det3(const M4& m) {
  return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
         m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}
// `affine_inverse` spin_history.rs:196-207 with `mat::inverse3` (mat.rs:78-103), `matvec` (mat.rs:39-45)
M4 affine_inverse(const M4& m) {
  const double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                     m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                     m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
  if (std::fabs(det) < 1e-18) throw std::runtime_error("an invertible grid affine");
  const double inv = 1.0 / det;
  const double li[3][3] = {{(m[1][1] * m[2][2] - m[1][2] * m[2][1]) * inv, (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * inv,
                            (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * inv},
                           {(m[1][2] * m[2][0] - m[1][0] * m[2][2]) * inv, (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * inv,
                            (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * inv},
                           {(m[1][0] * m[2][1] - m[1][1] * m[2][0]) * inv, (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * inv,
                            (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * inv}};
  double it[3];
  for (int r = 0; r < 3; ++r) it[r] = li[r][0] * m[0][3] + li[r][1] * m[1][3] + li[r][2] * m[2][3];
  M4 o{};
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) o[r][c] = li[r][c];
    o[r][3] = -it[r];
  }
  o[3] = {0.0, 0.0, 0.0, 1.0};
  return o;
}
// `mul4` spin_history.rs:209-217: a left-to-right sum from zero
M4 mul4(const M4& a, const M4& b) {
  M4 c{};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s = s + a[i][k] * b[k][j];
      c[i][j] = s;
    }
  return c;
}
// `apply4` spin_history.rs:219-225
std::array<double, 3> apply4(const M4& m, double x, double y, double z) {
  return {m[0][0] * x + m[0][1] * y + m[0][2] * z + m[0][3], m[1][0] * x + m[1][1] * y + m[1][2] * z + m[1][3],
          m[2][0] * x + m[2][1] * y + m[2][2] * z + m[2][3]};
}
double col_norm(const M4& m, int c) { return std::sqrt(m[0][c] * m[0][c] + m[1][c] * m[1][c] + m[2][c] * m[2][c]); }
M4 to_m4(const double* a) {
  M4 m{};
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) m[r][c] = a[4 * r + c];
  return m;
}

struct Plane {
  int64_t z;
  int64_t first;  // tracked index of the plane's first voxel (source order)
  std::vector<std::pair<int64_t, int64_t>> xy;
  std::vector<float> t1, weight;
  std::vector<uint8_t> cls;
  std::vector<Pieces> pieces;
};

// `SpinHistory` spin_history.rs:171-422
struct History {
  M4 v2w{}, w2v_slab{};
  int64_t n_classes = 0;
  int64_t sdims[3] = {0, 0, 0};
  std::vector<Pulse> pulses;
  std::vector<Plane> planes;
  int64_t src_nx = 0, src_ny = 0, n_tracked = 0;
  double vox_len = 0, vox_vol = 0;
  uint64_t merges = 0;

  double reference(const mrsim_mz_reference& r, double t1, double t_now, int64_t tracked) const {
    switch (r.kind) {
      case MRSIM_MZREF_RECOVERY:
        return 1.0 - (1.0 - r.a) * std::exp(-r.b / t1);
      case MRSIM_MZREF_CONSTANT:
        return t1 > 0.0 ? r.a : r.b;
      case MRSIM_MZREF_REPLAY:
        return replay(r.a, r.b, t_now, t1, pulses.data(), pulses.size());
      case MRSIM_MZREF_VALUES:
        return r.values[tracked];
      default:
        throw std::runtime_error("unknown reference kind");
    }
  }

  // `SpinHistory::step` spin_history.rs:317-420 (planes in order: the plane-ordered sums are the
  // reference's with or without `par`)
  void step(const mrsim_spin_shot& shot, float* terms) {
    const int64_t snx = sdims[0], sny = sdims[1], snz = sdims[2], cells = snx * sny;
    const M4 m = mul4(w2v_slab, mul4(to_m4(shot.transform), v2w));
    std::vector<int64_t> in_shot(snz, -1);
    for (int64_t k = 0; k < shot.n_slices; ++k) {
      const int64_t z = shot.slices[k];
      if (z < 0 || z >= snz)
        throw std::runtime_error("slice " + std::to_string(z) + " is outside the " + std::to_string(snz) + " slabs");
      in_shot[z] = k;
    }
    const bool read = shot.ref.kind != MRSIM_MZREF_NONE;
    const double len = vox_len, vol = vox_vol;
    const Pulse* P = pulses.data();
    const size_t np = pulses.size();
    std::vector<double> acc(read ? (size_t)shot.n_slices * 2 * n_classes * cells : 0, 0.0);
    for (Plane& pl : planes) {
      double lo = std::numeric_limits<double>::infinity(), hi = -std::numeric_limits<double>::infinity();
      const double cx[4] = {-0.5, (double)src_nx - 0.5, -0.5, (double)src_nx - 0.5};
      const double cy[4] = {-0.5, -0.5, (double)src_ny - 0.5, (double)src_ny - 0.5};
      for (int c = 0; c < 4; ++c) {
        const auto p = apply4(m, cx[c], cy[c], (double)pl.z);
        lo = std::fmin(lo, p[2]);
        hi = std::fmax(hi, p[2]);
      }
      lo = lo - len / 2.0;
      hi = hi + len / 2.0;
      const int64_t k0 = (int64_t)std::fmax(std::floor(lo + 0.5), 0.0);
      const int64_t k1 = (int64_t)std::fmin(std::floor(hi + 0.5), (double)snz - 1.0);
      bool any = false;
      for (int64_t k = k0; k <= k1; ++k)
        if (in_shot[k] >= 0) any = true;
      if (k1 < k0 || !any) continue;
      for (size_t j = 0; j < pl.xy.size(); ++j) {
        const int64_t x = pl.xy[j].first, y = pl.xy[j].second;
        const auto p = apply4(m, (double)x, (double)y, (double)pl.z);
        const double a = p[2] - len / 2.0;
        const double ka = std::floor(a + 0.5), kb = std::floor(a + len + 0.5);
        const double t1 = (double)pl.t1[j];
        const double w_src =
            shot.weight ? (double)shot.weight[x + src_nx * (y + src_ny * pl.z)] : (double)pl.weight[j];
        const double r = read ? reference(shot.ref, t1, shot.t, pl.first + (int64_t)j) : 0.0;
        int64_t cell = -1;
        {
          const double qx = std::round(p[0]), qy = std::round(p[1]);
          if (qx >= 0.0 && qy >= 0.0 && qx < (double)snx && qy < (double)sny)
            cell = (int64_t)qx + snx * (int64_t)qy;
        }
        Pieces& pc = pl.pieces[j];
        for (double k = ka; k <= kb; k += 1.0) {
          if (!(k >= 0.0 && (int64_t)k < snz && in_shot[(int64_t)k] >= 0)) continue;
          auto snap = [](double u) -> float { return u < kSnap ? 0.0f : u > 1.0 - kSnap ? 1.0f : (float)u; };
          const float u0 = snap((k - 0.5 - a) / len);
          const float u1 = snap((k + 0.5 - a) / len);
          if (!(u1 > u0)) continue;
          merges += cut(pc, u0, u1, t1, P, np);
          bool have = false;
          float cm = 0;
          double ct = 0, cv = 0;
          const int64_t kk = in_shot[(int64_t)k];
          for (int i = 0; i < pc.n; ++i) {
            const float s = pc.start[i], e = pc.end(i);
            if (s < u0 || e > u1) continue;
            double mz_t;
            if (have && cm == pc.mz[i] && ct == pc.t[i]) {
              mz_t = cv;
            } else {
              mz_t = replay((double)pc.mz[i], pc.t[i], shot.t, t1, P, np);
              have = true;
              cm = pc.mz[i];
              ct = pc.t[i];
              cv = mz_t;
            }
            if (read && cell >= 0) {
              const double f = (double)(e - s) * vol * w_src;
              const size_t base = ((size_t)kk * 2 * n_classes + pl.cls[j]) * cells + cell;
              acc[base] += f * (mz_t - r);
              acc[base + (size_t)n_classes * cells] += f * r;
            }
            pc.mz[i] = 0.0f;
            pc.t[i] = shot.t;
          }
          pc.coalesce();
        }
      }
    }
    if (read)
      for (size_t i = 0; i < acc.size(); ++i) terms[i] = (float)acc[i];
  }
};

void copy_err(const std::exception& e, char* err, int64_t n) {
  if (err && n > 0) {
    std::strncpy(err, e.what(), (size_t)n - 1);
    err[n - 1] = 0;
  }
}

}  // namespace

extern "C" {

// The piece list of one voxel, for the reference's piece tests.
typedef struct oracle_pieces {
  int32_t n;
  int32_t pad;
  float start[kMaxPieces];
  float mz[kMaxPieces];
  double t[kMaxPieces];
} oracle_pieces;

static Pieces from_c(const oracle_pieces* p) {
  Pieces q;
  q.n = p->n;
  std::memcpy(q.start, p->start, sizeof q.start);
  std::memcpy(q.mz, p->mz, sizeof q.mz);
  std::memcpy(q.t, p->t, sizeof q.t);
  return q;
}
static void to_c(const Pieces& q, oracle_pieces* p) {
  p->n = q.n;
  std::memcpy(p->start, q.start, sizeof q.start);
  std::memcpy(p->mz, q.mz, sizeof q.mz);
  std::memcpy(p->t, q.t, sizeof q.t);
}
static std::vector<Pulse> sorted_pulses(const mrsim_pulse* pulses, int64_t np) {
  std::vector<Pulse> v;
  for (int64_t i = 0; i < np; ++i) v.push_back({pulses[i].kind, pulses[i].t, pulses[i].epsilon});
  // `sort_by(total_cmp)` spin_history.rs:257: stable, -0 before +0
  std::stable_sort(v.begin(), v.end(), [](const Pulse& a, const Pulse& b) {
    if (a.t == b.t) return std::signbit(a.t) && !std::signbit(b.t);
    return a.t < b.t;
  });
  return v;
}

void oracle_pieces_relaxed(oracle_pieces* p) { to_c(Pieces::relaxed(), p); }
int oracle_pieces_split(oracle_pieces* p, float u) {
  Pieces q = from_c(p);
  const bool ok = q.split(u);
  to_c(q, p);
  return ok ? 1 : 0;
}
int oracle_pieces_has_edge(const oracle_pieces* p, float u) { return from_c(p).has_edge(u) ? 1 : 0; }
void oracle_pieces_coalesce(oracle_pieces* p) {
  Pieces q = from_c(p);
  q.coalesce();
  to_c(q, p);
}
uint64_t oracle_pieces_cut(oracle_pieces* p, float u0, float u1, double t1, const mrsim_pulse* pulses, int64_t np) {
  const auto P = sorted_pulses(pulses, np);
  Pieces q = from_c(p);
  const uint64_t m = cut(q, u0, u1, t1, P.data(), P.size());
  to_c(q, p);
  return m;
}
void oracle_pieces_merge_closest(oracle_pieces* p, double t1, const mrsim_pulse* pulses, int64_t np,
                                 const float* protect, int32_t nprot) {
  const auto P = sorted_pulses(pulses, np);
  Pieces q = from_c(p);
  merge_closest(q, t1, P.data(), P.size(), protect, nprot);
  to_c(q, p);
}
double oracle_spin_replay(double mz, double t_from, double t_to, double t1, const mrsim_pulse* pulses, int64_t np) {
  const auto P = sorted_pulses(pulses, np);
  return replay(mz, t_from, t_to, t1, P.data(), P.size());
}

// `SpinHistory::new` spin_history.rs:254-289; NULL (message in err) on invalid input.
void* oracle_spin_new(const int64_t* dims, const double* v2w, const float* t1, const float* weight,
                      const uint8_t* cls, int64_t n_classes, const int64_t* slab_dims, const double* slab_v2w,
                      const mrsim_pulse* pulses, int64_t np, char* err, int64_t errlen) {
  try {
    std::unique_ptr<History> h(new History());
    const int64_t nx = dims[0], ny = dims[1], nz = dims[2];
    h->pulses = sorted_pulses(pulses, np);
    for (int64_t z = 0; z < nz; ++z) {
      Plane pl;
      pl.z = z;
      pl.first = h->n_tracked;
      for (int64_t y = 0; y < ny; ++y)
        for (int64_t x = 0; x < nx; ++x) {
          const int64_t i = x + nx * (y + ny * z);
          const uint8_t c = cls[i];
          if (c == kNoClass) continue;
          if ((int64_t)c >= n_classes)
            throw std::runtime_error("class " + std::to_string(c) + " of voxel " + std::to_string(i) +
                                     " is not below " + std::to_string(n_classes));
          pl.xy.push_back({x, y});
          pl.t1.push_back(t1[i]);
          pl.weight.push_back(weight[i]);
          pl.cls.push_back(c);
          pl.pieces.push_back(Pieces::relaxed());
        }
      h->n_tracked += (int64_t)pl.xy.size();
      if (!pl.xy.empty()) h->planes.push_back(std::move(pl));
    }
    h->v2w = to_m4(v2w);
    const M4 s = to_m4(slab_v2w);
    h->vox_len = col_norm(h->v2w, 2) / col_norm(s, 2);
    h->vox_vol = std::fabs(det3(h->v2w)) / std::fabs(det3(s));
    h->w2v_slab = affine_inverse(s);
    h->n_classes = n_classes;
    for (int i = 0; i < 3; ++i) h->sdims[i] = slab_dims[i];
    h->src_nx = nx;
    h->src_ny = ny;
    return h.release();
  } catch (const std::exception& e) {
    copy_err(e, err, errlen);
    return nullptr;
  }
}

// One `step` (prime: ref.kind NONE, terms unused; excite: terms as the library packs them,
// [slice in shot][num, den][class][cell]).  0 on success.
int oracle_spin_step(void* h, const mrsim_spin_shot* shot, float* terms, char* err, int64_t errlen) {
  try {
    static_cast<History*>(h)->step(*shot, terms);
    return 0;
  } catch (const std::exception& e) {
    copy_err(e, err, errlen);
    return 1;
  }
}
uint64_t oracle_spin_merges(void* h) { return static_cast<History*>(h)->merges; }
int64_t oracle_spin_n_tracked(void* h) { return static_cast<History*>(h)->n_tracked; }
void oracle_spin_free(void* h) { delete static_cast<History*>(h); }

}  // extern "C"
