// spin_history.cu — the spin history of slice-selective excitations under head motion
// (`SpinHistory`, spin_history.rs:171-452 of the reference crate) with its state resident on the
// device.
//
// State.  Every tracked source voxel (class != 255) keeps its z extent as at most 8 pieces
// (f32 start and Mz, f64 time of the last excitation), structure-of-arrays in source order with
// the piece slots slot-major, so a warp of neighbouring voxels reads and writes each slot
// coalesced.  The history of one voxel depends on nothing but its own pieces, so one thread owns
// one voxel for a whole batch of shots: it loads the pieces once, steps them through every shot
// of the batch in registers and local memory (L1), and stores them once.
//
// Terms.  Per shot, every voxel of an active source plane writes one record: its slab cell (the
// cell nearest its moved centre, or -1) and its contributions (slice in the shot, l V w (Mz -
// mz_ref), l V w mz_ref), in the reference's order (slabs ascending, pieces ascending).  A
// second kernel gathers each output (shot, slice, class, cell), a tile of cells per block: the
// block stages the cells' candidate source voxels in shared memory, and each thread walks the
// voxels whose moved centre can round to its cell and whose z extent can reach the slab (the box
// of the cell's preimage, z then y then x ascending, which is the reference's plane-then-voxel
// order) and adds their matching contributions in FP64, then rounds once to f32.  The sums are the
// reference's, added in the reference's order: no atomics, the same bits on every run.
//
// Arithmetic.  The file is compiled without multiply-add contraction (build.py), so every f64
// expression rounds as the reference's does; f32 piece edges and magnetisations as in the
// reference.  `exp` is CUDA's (within 1 ulp of the correctly rounded value).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>

#include "spin_history.h"

namespace mrsim {

void* GrowBuf::get(size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (bytes > n) {
    if (p) MRSIM_CUDA(cudaFree(p));
    p = nullptr;
    n = 0;
    MRSIM_CUDA(cudaMalloc(&p, bytes));
    n = bytes;
  }
  return p;
}
GrowBuf::~GrowBuf() {
  if (p) cudaFree(p);
}

SpinHistoryDev::~SpinHistoryDev() {
  for (void* p : allocs) cudaFree(p);
  for (int b = 0; b < 2; ++b) {
    if (pin_ev[b]) cudaEventSynchronize(pin_ev[b]);
    if (pin[b]) cudaFreeHost(pin[b]);
    if (pin_ev[b]) cudaEventDestroy(pin_ev[b]);
  }
}

namespace {

constexpr int kPieces = MRSIM_SPIN_MAX_PIECES;
constexpr double kSnap = 1e-6;  // a slab edge this close to a voxel's end is the end

// ---- piece arithmetic (the reference's `Pieces`, `replay`, `merge_closest`) ------------------
__device__ __forceinline__ double recover(double m, double dt, double t1) {
  return isinf(dt) ? 1.0 : 1.0 - (1.0 - m) * exp(-dt / t1);
}

// Mz at t_to from mz just after t_from through the pulses in (t_from, t_to] (`replay`
// spin_history.rs:232-251).
__device__ double replay(double mz, double t_from, double t_to, double t1, const SpinPulseDev* __restrict__ P,
                         int np) {
  if (t1 <= 0.0) return 0.0;
  int lo = 0, hi = np;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (P[mid].t <= t_from)
      lo = mid + 1;
    else
      hi = mid;
  }
  double m = mz, t = t_from;
  for (int i = lo; i < np; ++i) {
    const double tp = P[i].t;
    if (tp > t_to) break;
    m = recover(m, tp - t, t1);
    m = P[i].kind == MRSIM_PULSE_INVERSION ? m * (1.0 - 2.0 * P[i].eps) : 0.0;
    t = tp;
  }
  return recover(m, t_to - t, t1);
}

struct Pieces {
  int n;
  float start[kPieces];
  float mz[kPieces];
  double t[kPieces];
  __device__ float end(int i) const { return i + 1 < n ? start[i + 1] : 1.0f; }
  __device__ bool has_edge(float u) const {
    bool e = false;
    for (int i = 0; i < n; ++i) e |= start[i] == u;
    return e;
  }
  __device__ void split(float u) {
    int i = -1;
    for (int k = 0; k < n; ++k)
      if (i < 0 && start[k] < u && u < end(k)) i = k;
    if (i < 0 || n == kPieces) return;
    for (int j = n - 1; j >= i + 1; --j) {
      start[j + 1] = start[j];
      mz[j + 1] = mz[j];
      t[j + 1] = t[j];
    }
    start[i + 1] = u;
    mz[i + 1] = mz[i];
    t[i + 1] = t[i];
    ++n;
  }
  __device__ void remove(int i) {
    for (int j = i; j < n - 1; ++j) {
      start[j] = start[j + 1];
      mz[j] = mz[j + 1];
      t[j] = t[j + 1];
    }
    --n;
  }
  __device__ void coalesce() {
    int i = 1;
    while (i < n) {
      if (mz[i] == mz[i - 1] && t[i] == t[i - 1])
        remove(i);
      else
        ++i;
    }
  }
};

// A full voxel: the neighbouring pair whose merge averages least (state difference times the
// pair's reduced length), never removing the edge u0 or u1, becomes its length-weighted mean at
// the later of the two times (`merge_closest` spin_history.rs:426-452).
__device__ void merge_closest(Pieces& pc, double t1, const SpinPulseDev* __restrict__ P, int np, float u0, float u1) {
  int best = -1;
  double best_cost = 0.0;
  for (int i = 1; i < pc.n; ++i) {
    if (pc.start[i] == u0 || pc.start[i] == u1) continue;
    const double li = (double)(pc.end(i) - pc.start[i]), lj = (double)(pc.end(i - 1) - pc.start[i - 1]);
    const double d = (double)fabsf(pc.mz[i] - pc.mz[i - 1]) + fmin(fabs(pc.t[i] - pc.t[i - 1]), 1e6);
    const double c = d * li * lj / (li + lj);
    if (best < 0 || c < best_cost) {
      best = i;
      best_cost = c;
    }
  }
  if (best < 0) return;  // a full voxel has seven edges and at most two are protected
  const float la = pc.end(best - 1) - pc.start[best - 1], lb = pc.end(best) - pc.start[best];
  const double ta = pc.t[best - 1], tb = pc.t[best];
  const double t = fmax(ta, tb);
  const double ma = ta == t ? (double)pc.mz[best - 1] : replay((double)pc.mz[best - 1], ta, t, t1, P, np);
  const double mb = tb == t ? (double)pc.mz[best] : replay((double)pc.mz[best], tb, t, t1, P, np);
  pc.mz[best - 1] = (float)((ma * (double)la + mb * (double)lb) / (double)(la + lb));
  pc.t[best - 1] = t;
  pc.remove(best);
}

// Make u0 and u1 edges, merging first while the voxel lacks room (`Pieces::cut`
// spin_history.rs:115-131); returns the merges.
__device__ unsigned cut(Pieces& pc, float u0, float u1, double t1, const SpinPulseDev* __restrict__ P, int np) {
  unsigned merges = 0;
  for (int guard = 0; guard < kPieces; ++guard) {
    const int needs = (u0 > 0.0f && u0 < 1.0f && !pc.has_edge(u0)) + (u1 > 0.0f && u1 < 1.0f && !pc.has_edge(u1));
    if (pc.n + needs <= kPieces) break;
    ++merges;
    merge_closest(pc, t1, P, np, u0, u1);
  }
  if (u0 > 0.0f && u0 < 1.0f) pc.split(u0);
  if (u1 > 0.0f && u1 < 1.0f) pc.split(u1);
  return merges;
}

__device__ __forceinline__ float snap(double u) { return u < kSnap ? 0.0f : u > 1.0 - kSnap ? 1.0f : (float)u; }

struct StepArgs {
  const SpinShotDev* shots;
  int n_shots;
  const int* tabs;
  const double* values;
  const float* weights;
  const uint32_t* flat;
  const float* t1;
  const float* w;
  uint8_t* pn;
  float* pstart;
  float* pmz;
  double* pt;
  const SpinPulseDev* pulses;
  int np;
  const int* plane_first;
  int* rec_cell;
  uint8_t* rec_cnt;
  double* ent_num;
  double* ent_den;
  int16_t* ent_kk;
  long long n_rec;
  int maxc, nk_max, ncls;
  const uint8_t* cls;
  long long nt;
  int nx, ny, snx, sny, snz;
  double len, half_len, vol;
  unsigned long long* merges;
  int* err;
};

// One thread per tracked voxel: the voxel's pieces through every shot of the batch
// (`SpinHistory::step` spin_history.rs:317-420, the per-voxel body).
__global__ void __launch_bounds__(128) spin_step_kernel(StepArgs A) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.nt) return;
  const uint32_t f = A.flat[i];
  const int x = (int)(f % (uint32_t)A.nx);
  const int y = (int)((f / (uint32_t)A.nx) % (uint32_t)A.ny);
  const int z = (int)(f / ((uint32_t)A.nx * (uint32_t)A.ny));
  const int pf = A.plane_first[z];
  const double t1 = (double)A.t1[i];
  Pieces pc;
  pc.n = 0;
  bool loaded = false, dirty = false;
  unsigned long long merges = 0;
  for (int s = 0; s < A.n_shots; ++s) {
    const SpinShotDev& S = A.shots[s];
    const int base = A.tabs[S.plane_tab + z];
    if (base < 0) continue;  // the voxel's plane does not reach the shot's slabs
    if (!loaded) {
      pc.n = A.pn[i];
      for (int q = 0; q < pc.n; ++q) {
        pc.start[q] = A.pstart[q * A.nt + i];
        pc.mz[q] = A.pmz[q * A.nt + i];
        pc.t[q] = A.pt[q * A.nt + i];
      }
      loaded = true;
    }
    const double X = (double)x, Y = (double)y, Z = (double)z;
    const double p0 = S.m[0] * X + S.m[1] * Y + S.m[2] * Z + S.m[3];
    const double p1 = S.m[4] * X + S.m[5] * Y + S.m[6] * Z + S.m[7];
    const double p2 = S.m[8] * X + S.m[9] * Y + S.m[10] * Z + S.m[11];
    const double a = p2 - A.half_len;
    const double ka = floor(a + 0.5), kb = floor(a + A.len + 0.5);
    const bool reads = S.ref_kind != MRSIM_MZREF_NONE;
    const double w_src = S.weight >= 0 ? (double)A.weights[S.weight + f] : (double)A.w[i];
    double r = 0.0;
    switch (S.ref_kind) {
      case MRSIM_MZREF_RECOVERY:
        r = 1.0 - (1.0 - S.ref_a) * exp(-S.ref_b / t1);
        break;
      case MRSIM_MZREF_CONSTANT:
        r = t1 > 0.0 ? S.ref_a : S.ref_b;
        break;
      case MRSIM_MZREF_REPLAY:
        r = replay(S.ref_a, S.ref_b, S.t, t1, A.pulses, A.np);
        break;
      case MRSIM_MZREF_VALUES:
        r = A.values[S.values + i];
        break;
      default:
        break;
    }
    int cell = -1;
    {
      const double qx = round(p0), qy = round(p1);
      if (qx >= 0.0 && qy >= 0.0 && qx < (double)A.snx && qy < (double)A.sny) cell = (int)qx + A.snx * (int)qy;
    }
    const long long rec = S.rec + base + (i - pf);
    int cnt = 0;
    double k = ka;
    for (int it = 0; it < A.nk_max && k <= kb; ++it, k += 1.0) {
      if (!(k >= 0.0 && k < (double)A.snz)) continue;
      const int kk = A.tabs[S.in_shot + (int)k];
      if (kk < 0) continue;
      const float u0 = snap((k - 0.5 - a) / A.len);
      const float u1 = snap((k + 0.5 - a) / A.len);
      if (!(u1 > u0)) continue;
      merges += cut(pc, u0, u1, t1, A.pulses, A.np);
      dirty = true;
      bool have = false;
      float cm = 0.0f;
      double ct = 0.0, cv = 0.0;
      for (int q = 0; q < pc.n; ++q) {
        const float s0 = pc.start[q], e0 = pc.end(q);
        if (s0 < u0 || e0 > u1) continue;
        double mz_t;
        if (have && cm == pc.mz[q] && ct == pc.t[q]) {
          mz_t = cv;
        } else {
          mz_t = replay((double)pc.mz[q], pc.t[q], S.t, t1, A.pulses, A.np);
          have = true;
          cm = pc.mz[q];
          ct = pc.t[q];
          cv = mz_t;
        }
        if (reads && cell >= 0) {
          if (cnt < A.maxc) {
            const double fr = (double)(e0 - s0) * A.vol * w_src;
            const long long e = (long long)cnt * A.n_rec + rec;
            A.ent_num[e] = fr * (mz_t - r);
            A.ent_den[e] = fr * r;
            A.ent_kk[e] = (int16_t)kk;
            ++cnt;
          } else {
            atomicCAS(A.err, 0, 1);  // more contributions than the bound allows: not reachable
          }
        }
        pc.mz[q] = 0.0f;
        pc.t[q] = S.t;
      }
      pc.coalesce();
    }
    if (reads) {
      A.rec_cell[rec] = cell >= 0 ? cell * A.ncls + A.cls[i] : -1;
      A.rec_cnt[rec] = (uint8_t)cnt;
    }
  }
  if (dirty) {
    A.pn[i] = (uint8_t)pc.n;
    for (int q = 0; q < pc.n; ++q) {
      A.pstart[q * A.nt + i] = pc.start[q];
      A.pmz[q * A.nt + i] = pc.mz[q];
      A.pt[q * A.nt + i] = pc.t[q];
    }
  }
  if (merges) atomicAdd(A.merges, merges);
}

constexpr int kTileX = 16, kTileY = 8;  // slab cells of one gather block (one thread each)
constexpr int kStageCap = 5632;          // source voxels a gather block stages (44 KiB of shared memory)
constexpr int kStagePlanes = 256;        // source planes of a staged box whose tables the block keeps

struct GatherArgs {
  const SpinShotDev* shots;
  const int* tabs;
  const long long* bcum;  // n_read + 1 cumulative block counts
  const int* oshot;       // the batch index of each reading shot
  int n_read;
  const int* idx;
  const int* plane_first;
  const uint8_t* cls;
  const int* rec_cell;
  const uint8_t* rec_cnt;
  const double* ent_num;
  const double* ent_den;
  const int16_t* ent_kk;
  long long n_rec;
  int nx, ny, nz, snx, sny, ncls, tiles_x, tiles;
  long long cells;
  double half_len;
  float* terms;
};

// The source voxel box (inclusive, clamped to the grid) holding every voxel whose moved centre can
// round into slab cells [x0, x1] x [y0, y1] and whose z extent can reach slab k: the corners of
// that slab box mapped by the shot's inverse (a singular transform has a NaN inverse, and the box
// is then the whole grid).
__device__ __forceinline__ void preimage_box(const SpinShotDev& S, int x0, int x1, int y0, int y1, int k,
                                             double half_len, const int (&ext)[3], int (&b0)[3], int (&b1)[3]) {
  constexpr double d = 1e-3;
  double blo[3] = {INFINITY, INFINITY, INFINITY}, bhi[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
  for (int corner = 0; corner < 8; ++corner) {
    const double sx = (corner & 1) ? x1 + 0.5 + d : x0 - 0.5 - d;
    const double sy = (corner & 2) ? y1 + 0.5 + d : y0 - 0.5 - d;
    const double sz = k + ((corner & 4) ? 0.5 + half_len + d : -0.5 - half_len - d);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const double v = S.minv[4 * r] * sx + S.minv[4 * r + 1] * sy + S.minv[4 * r + 2] * sz + S.minv[4 * r + 3];
      blo[r] = isnan(v) ? -INFINITY : fmin(blo[r], v);
      bhi[r] = isnan(v) ? INFINITY : fmax(bhi[r], v);
    }
  }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    b0[r] = (int)fmax(0.0, floor(blo[r]));
    b1[r] = (int)fmin((double)(ext[r] - 1), ceil(bhi[r]));
  }
}

// One block per tile of 16 x 8 slab cells of one (reading shot, slice, class), one thread per
// cell.  The block stages the tile's source-voxel box in shared memory (each voxel's cell, or -1
// when it is untracked, of another class or in a plane the shot does not reach, and its record),
// then every thread walks its own cell's box from there (z, then y, then x: the reference's
// plane-then-voxel order) and adds the contributions of the voxels that round to its cell in
// FP64, rounding once to f32 (spin_history.rs:407-419).  A box too large to stage (a strongly
// rotated head on fine slabs) is walked in global memory instead, in the same order.
__global__ void __launch_bounds__(kTileX * kTileY) spin_gather_kernel(GatherArgs A) {
  __shared__ int key[kStageCap];
  __shared__ int roff[kStageCap];
  const long long b = blockIdx.x;
  int lo = 0, hi = A.n_read;  // the reading shot holding block b
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (A.bcum[mid] <= b)
      lo = mid;
    else
      hi = mid;
  }
  const SpinShotDev& S = A.shots[A.oshot[lo]];
  const long long local = b - A.bcum[lo];
  const int tile = (int)(local % A.tiles);
  const int c = (int)((local / A.tiles) % A.ncls);
  const int kk = (int)(local / ((long long)A.tiles * A.ncls));
  const int k = A.tabs[S.slices + kk];
  const int tx0 = (tile % A.tiles_x) * kTileX, ty0 = (tile / A.tiles_x) * kTileY;
  const int tx1 = min(tx0 + kTileX, A.snx) - 1, ty1 = min(ty0 + kTileY, A.sny) - 1;
  const int ext[3] = {A.nx, A.ny, A.nz};
  int B0[3], B1[3];
  preimage_box(S, tx0, tx1, ty0, ty1, k, A.half_len, ext, B0, B1);
  const int bx = max(B1[0] - B0[0] + 1, 0), by = max(B1[1] - B0[1] + 1, 0), bz = max(B1[2] - B0[2] + 1, 0);
  const long long total = (long long)bx * by * bz;
  const bool staged = total <= kStageCap;
  // the box's planes: their first record in the shot (or -1) and first tracked voxel
  __shared__ int pbase[kStagePlanes], pfirst[kStagePlanes];
  const bool planes_fit = bz <= kStagePlanes;
  if (staged && planes_fit) {
    for (int zz = threadIdx.x; zz < bz; zz += blockDim.x) {
      pbase[zz] = A.tabs[S.plane_tab + B0[2] + zz];
      pfirst[zz] = A.plane_first[B0[2] + zz];
    }
  }
  __syncthreads();
  const int want_key0 = c;  // keys are cell * n_classes + class
  if (staged) {
    // one warp per (y, z) row of the box, lanes across x (no division per voxel), four rows in
    // flight per warp: their tracked indices are loaded together, then their records' keys and
    // counts together, so the two dependent round trips overlap across the rows
    constexpr int kRows = 4;
    const int lane = (int)threadIdx.x & 31, warp = (int)threadIdx.x >> 5, n_warps = (int)blockDim.x >> 5;
    const int n_rows = by * bz;
    for (int row0 = warp; row0 < n_rows; row0 += kRows * n_warps)
      for (int xx = lane; xx < bx; xx += 32) {
        int t[kRows], base[kRows], pf[kRows];
#pragma unroll
        for (int u = 0; u < kRows; ++u) {
          const int row = row0 + u * n_warps;
          t[u] = -1;
          base[u] = -1;
          pf[u] = 0;
          if (row < n_rows) {
            const int zz = row / by, yy = row - zz * by;
            const int z = B0[2] + zz, y = B0[1] + yy;
            base[u] = planes_fit ? pbase[zz] : A.tabs[S.plane_tab + z];
            pf[u] = planes_fit ? pfirst[zz] : A.plane_first[z];
            if (base[u] >= 0) t[u] = A.idx[(long long)A.nx * (y + (long long)A.ny * z) + B0[0] + xx];
          }
        }
        int kv[kRows], pk[kRows];
#pragma unroll
        for (int u = 0; u < kRows; ++u) {
          kv[u] = -1;
          pk[u] = 0;
          if (t[u] >= 0) {
            const int ro = base[u] + (t[u] - pf[u]);
            kv[u] = A.rec_cell[S.rec + ro];
            pk[u] = (ro << 6) | (int)A.rec_cnt[S.rec + ro];
          }
        }
#pragma unroll
        for (int u = 0; u < kRows; ++u) {
          const int row = row0 + u * n_warps;
          if (row < n_rows) {
            key[row * bx + xx] = kv[u];
            roff[row * bx + xx] = pk[u];
          }
        }
      }
  }
  __syncthreads();
  const int cx = tx0 + (int)threadIdx.x % kTileX, cy = ty0 + (int)threadIdx.x / kTileX;
  if (cx > tx1 || cy > ty1) return;
  const int cell = cx + A.snx * cy;
  const int want = cell * A.ncls + want_key0;
  int b0[3], b1[3];
  preimage_box(S, cx, cx, cy, cy, k, A.half_len, ext, b0, b1);
  double num = 0.0, den = 0.0;
  if (staged) {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      b0[r] = max(b0[r], B0[r]);
      b1[r] = min(b1[r], B1[r]);
    }
    // the matching records are collected eight at a time and their first entries loaded
    // together (the additions keep the source order: record after record, entry after entry)
    constexpr int kBatch = 8;
    long long mrec[kBatch];
    int mcnt[kBatch];
    int nm = 0;
    auto flush = [&]() {
      double en[kBatch], ed[kBatch];
      int ek[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        ek[u] = -1;
        en[u] = ed[u] = 0.0;
        if (u < nm && mcnt[u] > 0) {
          ek[u] = A.ent_kk[mrec[u]];
          en[u] = A.ent_num[mrec[u]];
          ed[u] = A.ent_den[mrec[u]];
        }
      }
#pragma unroll
      for (int u = 0; u < kBatch; ++u) {
        if (u >= nm) continue;
        if (ek[u] == kk) {
          num += en[u];
          den += ed[u];
        }
        for (int q = 1; q < mcnt[u]; ++q) {
          const long long j = (long long)q * A.n_rec + mrec[u];
          if (A.ent_kk[j] == kk) {
            num += A.ent_num[j];
            den += A.ent_den[j];
          }
        }
      }
      nm = 0;
    };
    for (int z = b0[2]; z <= b1[2]; ++z)
      for (int y = b0[1]; y <= b1[1]; ++y) {
        const int er = bx * ((y - B0[1]) + by * (z - B0[2])) - B0[0];
        for (int x = b0[0]; x <= b1[0]; ++x) {
          const int e = er + x;
          if (key[e] != want) continue;
          const long long rec = S.rec + (roff[e] >> 6);
          const int cnt = roff[e] & 63;
#pragma unroll
          for (int u = 0; u < kBatch; ++u)
            if (u == nm) {
              mrec[u] = rec;
              mcnt[u] = cnt;
            }
          if (++nm == kBatch) flush();
        }
      }
    flush();
  } else {
    for (int z = b0[2]; z <= b1[2]; ++z) {
      const int base = A.tabs[S.plane_tab + z];
      if (base < 0) continue;
      const int pf = A.plane_first[z];
      for (int y = b0[1]; y <= b1[1]; ++y)
        for (int x = b0[0]; x <= b1[0]; ++x) {
          const int t = A.idx[x + A.nx * (y + A.ny * z)];
          if (t < 0) continue;
          const long long rec = S.rec + base + (t - pf);
          if (A.rec_cell[rec] != want) continue;
          const int cnt = A.rec_cnt[rec];
          for (int q = 0; q < cnt; ++q) {
            const long long j = (long long)q * A.n_rec + rec;
            if (A.ent_kk[j] == kk) {
              num += A.ent_num[j];
              den += A.ent_den[j];
            }
          }
        }
    }
  }
  float* o = A.terms + S.out + ((long long)kk * 2 * A.ncls + c) * A.cells + cell;
  o[0] = (float)num;
  o[(long long)A.ncls * A.cells] = (float)den;
}

__global__ void spin_init_kernel(uint8_t* pn, float* pstart, float* pmz, double* pt, long long nt) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  pn[i] = 1;
  for (int q = 0; q < kPieces; ++q) {
    pstart[q * nt + i] = 0.0f;
    pmz[q * nt + i] = 1.0f;
    pt[q * nt + i] = -INFINITY;
  }
}

// ---- host geometry (the reference's f64 order; host code is compiled without contraction) ----
using M4 = double[4][4];
void to_m4(const double* a, M4 m) {
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) m[r][c] = a[4 * r + c];
}
// `mul4` spin_history.rs:209-217
void mul4(const M4 a, const M4 b, M4 c) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = 0.0;
      for (int k = 0; k < 4; ++k) s = s + a[i][k] * b[k][j];
      c[i][j] = s;
    }
}
double det3(const M4 m) {
  return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
         m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
}
// the affine inverse by the adjugate (`affine_inverse` spin_history.rs:196-207, `mat::inverse3`
// mat.rs:78-103); false when |det| < 1e-18
bool affine_inverse(const M4 m, M4 o) {
  const double det = det3(m);
  if (!(std::fabs(det) >= 1e-18)) return false;
  const double inv = 1.0 / det;
  const double li[3][3] = {{(m[1][1] * m[2][2] - m[1][2] * m[2][1]) * inv, (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * inv,
                            (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * inv},
                           {(m[1][2] * m[2][0] - m[1][0] * m[2][2]) * inv, (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * inv,
                            (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * inv},
                           {(m[1][0] * m[2][1] - m[1][1] * m[2][0]) * inv, (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * inv,
                            (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * inv}};
  for (int r = 0; r < 3; ++r) {
    const double it = li[r][0] * m[0][3] + li[r][1] * m[1][3] + li[r][2] * m[2][3];
    for (int c = 0; c < 3; ++c) o[r][c] = li[r][c];
    o[r][3] = -it;
  }
  o[3][0] = o[3][1] = o[3][2] = 0.0;
  o[3][3] = 1.0;
  return true;
}
double col_norm(const M4 m, int c) { return std::sqrt(m[0][c] * m[0][c] + m[1][c] * m[1][c] + m[2][c] * m[2][c]); }
double apply_z(const M4 m, double x, double y, double z) { return m[2][0] * x + m[2][1] * y + m[2][2] * z + m[2][3]; }

template <class T>
T* dalloc(SpinHistoryDev& h, size_t n) {
  void* p = nullptr;
  MRSIM_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  h.allocs.push_back(p);
  return (T*)p;
}

// Bytes of one record: cell, count and the entries.
size_t record_bytes(int maxc) { return 4 + 1 + (size_t)maxc * (8 + 8 + 2); }

}  // namespace

SpinHistoryDev* spin_history_create(mrsim_context* ctx, const int64_t* src_dims, const double* src_v2w,
                                    const float* t1, const float* weight, const uint8_t* cls, int64_t n_classes,
                                    const int64_t* slab_dims, const double* slab_v2w, const mrsim_pulse* pulses,
                                    int64_t n_pulses) {
  for (int i = 0; i < 3; ++i)
    if (src_dims[i] <= 0 || slab_dims[i] <= 0) fail("empty source grid or slab grid");
  const int64_t nv = src_dims[0] * src_dims[1] * src_dims[2];
  if (nv >= (1LL << 31)) fail("a source grid of 2^31 voxels or more");
  if (n_classes <= 0 || n_classes > 255) fail("n_classes must be in 1..255");
  // record keys are cell * n_classes + class in an int
  if (slab_dims[0] * slab_dims[1] * n_classes >= (1LL << 31) || slab_dims[2] > 32767) fail("slab grid too large");
  for (int64_t i = 0; i < n_pulses; ++i)
    if (pulses[i].kind != MRSIM_PULSE_INVERSION && pulses[i].kind != MRSIM_PULSE_SATURATION)
      fail("unknown pulse kind");
  std::unique_ptr<SpinHistoryDev> H(new SpinHistoryDev());
  SpinHistoryDev& h = *H;
  h.ctx = ctx;
  h.nx = src_dims[0];
  h.ny = src_dims[1];
  h.nz = src_dims[2];
  h.nv = nv;
  h.snx = slab_dims[0];
  h.sny = slab_dims[1];
  h.snz = slab_dims[2];
  h.ncls = (int)n_classes;
  std::memcpy(h.v2w, src_v2w, sizeof h.v2w);
  M4 sv, sw, src;
  to_m4(slab_v2w, sv);
  to_m4(src_v2w, src);
  if (!affine_inverse(sv, sw)) fail("an invertible grid affine");
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) h.w2v_slab[4 * r + c] = sw[r][c];
  h.len = col_norm(src, 2) / col_norm(sv, 2);
  h.vol = std::fabs(det3(src)) / std::fabs(det3(sv));
  if (!(h.len > 0.0) || !std::isfinite(h.len)) fail("a source voxel of zero z length");
  // the slabs one voxel reaches, and the contributions one voxel makes in a shot: 7 inner edges
  // plus one piece per slab reached
  const double nk = std::floor(h.len) + 2.0;
  if (nk > 48.0) fail("a source voxel reaches more than 48 slabs");
  h.maxc = 7 + (int)nk;
  // tracked voxels in source order (`SpinHistory::new` spin_history.rs:262-283)
  std::vector<uint32_t> flat;
  std::vector<float> t1t, wt;
  std::vector<uint8_t> ct;
  std::vector<int> idx((size_t)nv, -1);
  h.plane_first.assign((size_t)h.nz + 1, 0);
  for (int64_t z = 0; z < h.nz; ++z) {
    h.plane_first[z] = (int)flat.size();
    for (int64_t y = 0; y < h.ny; ++y)
      for (int64_t x = 0; x < h.nx; ++x) {
        const int64_t i = x + h.nx * (y + h.ny * z);
        const uint8_t c = cls[i];
        if (c == MRSIM_SPIN_NO_CLASS) continue;
        if ((int64_t)c >= n_classes)
          fail("class " + std::to_string(c) + " of voxel " + std::to_string(i) + " is not below " +
               std::to_string(n_classes));
        idx[i] = (int)flat.size();
        flat.push_back((uint32_t)i);
        t1t.push_back(t1[i]);
        wt.push_back(weight[i]);
        ct.push_back(c);
      }
  }
  h.plane_first[h.nz] = (int)flat.size();
  h.nt = (int64_t)flat.size();
  for (int64_t i = 0; i < n_pulses; ++i) h.pulses.push_back({pulses[i].t, pulses[i].epsilon, pulses[i].kind, 0});
  // `sort_by(total_cmp)` spin_history.rs:257: stable by time, -0 before +0
  std::stable_sort(h.pulses.begin(), h.pulses.end(), [](const SpinPulseDev& a, const SpinPulseDev& b) {
    if (a.t == b.t) return std::signbit(a.t) && !std::signbit(b.t);
    return a.t < b.t;
  });
  cudaStream_t st = ctx->stream;
  const size_t nt = (size_t)h.nt;
  h.d_flat = dalloc<uint32_t>(h, nt);
  h.d_t1 = dalloc<float>(h, nt);
  h.d_w = dalloc<float>(h, nt);
  h.d_cls = dalloc<uint8_t>(h, nt);
  h.d_n = dalloc<uint8_t>(h, nt);
  h.d_start = dalloc<float>(h, nt * kPieces);
  h.d_mz = dalloc<float>(h, nt * kPieces);
  h.d_t = dalloc<double>(h, nt * kPieces);
  h.d_idx = dalloc<int>(h, (size_t)nv);
  h.d_plane_first = dalloc<int>(h, h.plane_first.size());
  h.d_pulses = dalloc<SpinPulseDev>(h, h.pulses.size());
  h.d_merges = dalloc<unsigned long long>(h, 1);
  h.d_err = dalloc<int>(h, 1);
  if (nt) {
    MRSIM_CUDA(cudaMemcpyAsync(h.d_flat, flat.data(), nt * 4, cudaMemcpyHostToDevice, st));
    MRSIM_CUDA(cudaMemcpyAsync(h.d_t1, t1t.data(), nt * 4, cudaMemcpyHostToDevice, st));
    MRSIM_CUDA(cudaMemcpyAsync(h.d_w, wt.data(), nt * 4, cudaMemcpyHostToDevice, st));
    MRSIM_CUDA(cudaMemcpyAsync(h.d_cls, ct.data(), nt, cudaMemcpyHostToDevice, st));
    spin_init_kernel<<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(h.d_n, h.d_start, h.d_mz, h.d_t, (long long)nt);
    MRSIM_CUDA(cudaGetLastError());
  }
  MRSIM_CUDA(cudaMemcpyAsync(h.d_idx, idx.data(), (size_t)nv * 4, cudaMemcpyHostToDevice, st));
  MRSIM_CUDA(cudaMemcpyAsync(h.d_plane_first, h.plane_first.data(), h.plane_first.size() * 4,
                             cudaMemcpyHostToDevice, st));
  if (!h.pulses.empty())
    MRSIM_CUDA(cudaMemcpyAsync(h.d_pulses, h.pulses.data(), h.pulses.size() * sizeof(SpinPulseDev),
                               cudaMemcpyHostToDevice, st));
  MRSIM_CUDA(cudaMemsetAsync(h.d_merges, 0, 8, st));
  MRSIM_CUDA(cudaMemsetAsync(h.d_err, 0, 4, st));
  for (int b = 0; b < 2; ++b) MRSIM_CUDA(cudaEventCreateWithFlags(&h.pin_ev[b], cudaEventDisableTiming));
  MRSIM_CUDA(cudaStreamSynchronize(st));  // the host staging vectors go out of scope
  return H.release();
}

int64_t spin_history_terms_size(const SpinHistoryDev& h, const mrsim_spin_shot* shots, int64_t n) {
  int64_t total = 0;
  for (int64_t s = 0; s < n; ++s)
    if (shots[s].ref.kind != MRSIM_MZREF_NONE) total += shots[s].n_slices * 2 * (int64_t)h.ncls * h.snx * h.sny;
  return total;
}

void spin_history_run(SpinHistoryDev& h, const mrsim_spin_shot* shots, int64_t n, float* terms) {
  const int64_t cells = h.snx * h.sny;
  // validate every shot before any work (the reference panics before stepping)
  for (int64_t s = 0; s < n; ++s) {
    const mrsim_spin_shot& S = shots[s];
    if (S.n_slices < 0 || (S.n_slices > 0 && !S.slices)) fail("slices is NULL");
    if (S.ref.kind < MRSIM_MZREF_NONE || S.ref.kind > MRSIM_MZREF_VALUES) fail("unknown reference kind");
    if (S.ref.kind == MRSIM_MZREF_VALUES && !S.ref.values && h.nt > 0) fail("reference values are NULL");
    if (S.ref.kind != MRSIM_MZREF_NONE && S.n_slices > 0 && !terms) fail("terms is NULL");
    for (int64_t k = 0; k < S.n_slices; ++k)
      if (S.slices[k] < 0 || S.slices[k] >= h.snz)
        fail("slice " + std::to_string(S.slices[k]) + " is outside the " + std::to_string(h.snz) + " slabs");
  }
  if (n == 0) return;
  cudaStream_t st = h.ctx->stream;
  M4 v2w, w2v_slab;
  to_m4(h.v2w, v2w);
  to_m4(h.w2v_slab, w2v_slab);
  const size_t rec_budget = std::max<size_t>(1, ((size_t)1 << 30) / record_bytes(h.maxc));  // records per batch
  const size_t w_budget = ((size_t)1 << 30) / 4;  // override weights per batch
  const int tiles_x = (int)((h.snx + kTileX - 1) / kTileX);
  const long long tiles = (long long)tiles_x * ((h.sny + kTileY - 1) / kTileY);
  long long out_off = 0;
  int64_t s0 = 0;
  while (s0 < n) {
    // one batch: shots [s0, s1) with their records and override weights within the budgets
    std::vector<SpinShotDev> sd;
    std::vector<int> tabs;
    std::vector<double> values;
    std::vector<float> weights;
    std::vector<long long> ocum{0};
    std::vector<int> oshot;
    long long n_rec = 0;
    bool any_active = false;
    int64_t s1 = s0;
    for (; s1 < n; ++s1) {
      const mrsim_spin_shot& S = shots[s1];
      const bool reads = S.ref.kind != MRSIM_MZREF_NONE;
      SpinShotDev D{};
      M4 T, TM, m, minv;
      to_m4(S.transform, T);
      mul4(T, v2w, TM);
      mul4(w2v_slab, TM, m);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) D.m[4 * r + c] = m[r][c];
      const bool inv_ok = affine_inverse(m, minv);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 4; ++c) D.minv[4 * r + c] = inv_ok ? minv[r][c] : std::nan("");
      // the slab table and the active planes (the reference's per-plane reach test,
      // spin_history.rs:340-360)
      std::vector<int> in_shot((size_t)h.snz, -1);
      for (int64_t k = 0; k < S.n_slices; ++k) in_shot[(size_t)S.slices[k]] = (int)k;
      std::vector<int> plane((size_t)h.nz, -1);
      long long shot_recs = 0;
      bool shot_active = false;
      for (int64_t z = 0; z < h.nz; ++z) {
        const int cnt = h.plane_first[z + 1] - h.plane_first[z];
        if (cnt == 0) continue;
        double lo = std::numeric_limits<double>::infinity(), hi = -std::numeric_limits<double>::infinity();
        const double cx[4] = {-0.5, (double)h.nx - 0.5, -0.5, (double)h.nx - 0.5};
        const double cy[4] = {-0.5, -0.5, (double)h.ny - 0.5, (double)h.ny - 0.5};
        for (int c = 0; c < 4; ++c) {
          const double pz = apply_z(m, cx[c], cy[c], (double)z);
          lo = std::fmin(lo, pz);
          hi = std::fmax(hi, pz);
        }
        lo = lo - h.len / 2.0;
        hi = hi + h.len / 2.0;
        const double k0d = std::fmax(std::floor(lo + 0.5), 0.0);
        const double k1d = std::fmin(std::floor(hi + 0.5), (double)h.snz - 1.0);
        if (!(k1d >= k0d)) continue;
        bool any = false;
        for (int64_t k = (int64_t)k0d; k <= (int64_t)k1d; ++k) any |= in_shot[(size_t)k] >= 0;
        if (!any) continue;
        plane[(size_t)z] = (int)shot_recs;
        shot_recs += cnt;
        shot_active = true;
      }
      const bool has_w = S.weight != nullptr;
      if (s1 > s0 && ((reads && (size_t)(n_rec + shot_recs) > rec_budget) ||
                      (has_w && weights.size() + (size_t)h.nv > w_budget)))
        break;
      any_active |= shot_active;
      D.t = S.t;
      D.ref_kind = S.ref.kind;
      D.ref_a = S.ref.a;
      D.ref_b = S.ref.b;
      D.n_slices = (int)S.n_slices;
      D.values = -1;
      if (S.ref.kind == MRSIM_MZREF_VALUES) {
        D.values = (long long)values.size();
        values.insert(values.end(), S.ref.values, S.ref.values + h.nt);
      }
      D.weight = -1;
      if (has_w) {
        D.weight = (long long)weights.size();
        weights.insert(weights.end(), S.weight, S.weight + h.nv);
      }
      D.plane_tab = (int)tabs.size();
      tabs.insert(tabs.end(), plane.begin(), plane.end());
      D.in_shot = (int)tabs.size();
      tabs.insert(tabs.end(), in_shot.begin(), in_shot.end());
      D.slices = (int)tabs.size();
      for (int64_t k = 0; k < S.n_slices; ++k) tabs.push_back((int)S.slices[k]);
      D.rec = -1;
      D.out = -1;
      if (reads) {
        D.rec = n_rec;
        n_rec += shot_recs;
        D.out = out_off;
        out_off += S.n_slices * 2 * (long long)h.ncls * cells;
        if (S.n_slices > 0) {
          ocum.push_back(ocum.back() + S.n_slices * (long long)h.ncls * tiles);
          oshot.push_back((int)sd.size());
        }
      }
      sd.push_back(D);
    }
    // the batch's tables packed into the next pinned staging blob (waiting only for the copy out
    // of it two batches ago) and uploaded in one asynchronous copy
    auto a16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    const size_t o_tabs = a16(sd.size() * sizeof(SpinShotDev));
    const size_t o_vals = a16(o_tabs + tabs.size() * 4);
    const size_t o_w = a16(o_vals + values.size() * 8);
    const size_t o_cum = a16(o_w + weights.size() * 4);
    const size_t o_osh = a16(o_cum + ocum.size() * 8);
    const size_t blob = a16(o_osh + oshot.size() * 4);
    const int pb = h.pin_i;
    h.pin_i ^= 1;
    MRSIM_CUDA(cudaEventSynchronize(h.pin_ev[pb]));
    if (h.pin_n[pb] < blob) {
      if (h.pin[pb]) MRSIM_CUDA(cudaFreeHost(h.pin[pb]));
      h.pin[pb] = nullptr;
      h.pin_n[pb] = 0;
      MRSIM_CUDA(cudaHostAlloc(&h.pin[pb], blob, cudaHostAllocDefault));
      h.pin_n[pb] = blob;
    }
    char* hb = (char*)h.pin[pb];
    std::memcpy(hb, sd.data(), sd.size() * sizeof(SpinShotDev));
    if (!tabs.empty()) std::memcpy(hb + o_tabs, tabs.data(), tabs.size() * 4);
    if (!values.empty()) std::memcpy(hb + o_vals, values.data(), values.size() * 8);
    if (!weights.empty()) std::memcpy(hb + o_w, weights.data(), weights.size() * 4);
    std::memcpy(hb + o_cum, ocum.data(), ocum.size() * 8);
    if (!oshot.empty()) std::memcpy(hb + o_osh, oshot.data(), oshot.size() * 4);
    char* db = (char*)h.blob_b.get(blob);
    MRSIM_CUDA(cudaMemcpyAsync(db, hb, blob, cudaMemcpyHostToDevice, st));
    MRSIM_CUDA(cudaEventRecord(h.pin_ev[pb], st));
    const SpinShotDev* d_shots = (const SpinShotDev*)db;
    const int* d_tabs = (const int*)(db + o_tabs);
    const double* d_values = (const double*)(db + o_vals);
    const float* d_weights = (const float*)(db + o_w);
    // a staged record is addressed by 25 bits (its count in the other 6 of an int)
    if (n_rec >= (1LL << 25)) fail("more than 2^25 voxels in reach of one shot");
    const size_t nr = (size_t)std::max<long long>(n_rec, 1);
    int* d_rec_cell = (int*)h.rec_cell_b.get(nr * 4);
    uint8_t* d_rec_cnt = (uint8_t*)h.rec_cnt_b.get(nr);
    double* d_num = (double*)h.ent_num_b.get(nr * h.maxc * 8);
    double* d_den = (double*)h.ent_den_b.get(nr * h.maxc * 8);
    int16_t* d_kk = (int16_t*)h.ent_kk_b.get(nr * h.maxc * 2);
    if (any_active && h.nt > 0) {
      StepArgs A{};
      A.shots = d_shots;
      A.n_shots = (int)sd.size();
      A.tabs = d_tabs;
      A.values = d_values;
      A.weights = d_weights;
      A.flat = h.d_flat;
      A.t1 = h.d_t1;
      A.w = h.d_w;
      A.pn = h.d_n;
      A.pstart = h.d_start;
      A.pmz = h.d_mz;
      A.pt = h.d_t;
      A.pulses = h.d_pulses;
      A.np = (int)h.pulses.size();
      A.plane_first = h.d_plane_first;
      A.rec_cell = d_rec_cell;
      A.rec_cnt = d_rec_cnt;
      A.ent_num = d_num;
      A.ent_den = d_den;
      A.ent_kk = d_kk;
      A.n_rec = (long long)nr;
      A.maxc = h.maxc;
      A.ncls = h.ncls;
      A.cls = h.d_cls;
      A.nk_max = (int)(std::floor(h.len) + 2.0);
      A.nt = h.nt;
      A.nx = (int)h.nx;
      A.ny = (int)h.ny;
      A.snx = (int)h.snx;
      A.sny = (int)h.sny;
      A.snz = (int)h.snz;
      A.len = h.len;
      A.half_len = h.len / 2.0;
      A.vol = h.vol;
      A.merges = h.d_merges;
      A.err = h.d_err;
      spin_step_kernel<<<(unsigned)((h.nt + 127) / 128), 128, 0, st>>>(A);
      MRSIM_CUDA(cudaGetLastError());
    }
    if (!oshot.empty()) {
      const long long n_blocks = ocum.back();
      GatherArgs G{};
      G.shots = d_shots;
      G.tabs = d_tabs;
      G.bcum = (const long long*)(db + o_cum);
      G.oshot = (const int*)(db + o_osh);
      G.n_read = (int)oshot.size();
      G.idx = h.d_idx;
      G.plane_first = h.d_plane_first;
      G.cls = h.d_cls;
      G.rec_cell = d_rec_cell;
      G.rec_cnt = d_rec_cnt;
      G.ent_num = d_num;
      G.ent_den = d_den;
      G.ent_kk = d_kk;
      G.n_rec = (long long)nr;
      G.nx = (int)h.nx;
      G.ny = (int)h.ny;
      G.nz = (int)h.nz;
      G.snx = (int)h.snx;
      G.sny = (int)h.sny;
      G.ncls = h.ncls;
      G.tiles_x = tiles_x;
      G.tiles = (int)tiles;
      G.cells = cells;
      G.half_len = h.len / 2.0;
      G.terms = terms;
      if (n_blocks >= (1LL << 31)) fail("too many terms in one batch");
      spin_gather_kernel<<<(unsigned)n_blocks, kTileX * kTileY, 0, st>>>(G);
      MRSIM_CUDA(cudaGetLastError());
    }
    // the next batch's copies and launches follow these on the stream (a buffer that must grow is
    // freed by cudaFree, which waits for the device)
    s0 = s1;
  }
}

uint64_t spin_history_merges(SpinHistoryDev& h) {
  cudaStream_t st = h.ctx->stream;
  unsigned long long m = 0;
  int err = 0;
  MRSIM_CUDA(cudaMemcpyAsync(&m, h.d_merges, 8, cudaMemcpyDeviceToHost, st));
  MRSIM_CUDA(cudaMemcpyAsync(&err, h.d_err, 4, cudaMemcpyDeviceToHost, st));
  MRSIM_CUDA(cudaStreamSynchronize(st));
  if (err) throw Error(MRSIM_ERR_DEVICE, "spin history: a voxel made more contributions than its bound");
  return m;
}

}  // namespace mrsim
