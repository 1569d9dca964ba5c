// grase3d.cu — the 3D GRASE echo-train acquisition on the device (reference
// `simulate_acquisition_3d_complex_cal`, kspace3d.rs:483-547, with `Plan::compartments` /
// `Plan::kspace` :125-232, `partitions_to_slices` :235-281, `reconstruct_slices` :283-297 and
// `grappa_kernels_3d` :310-325).
//
// Per chunk of volumes, one batched forward launch computes every needed 2D k-space: one unit per
// (volume, compartment, slice) for class compartments (relaxation off, the decay a line weight)
// and per (volume, compartment, echo, slice) for voxel compartments (ln A_e and the T2/T2' maps
// inside the forward).  Then one kernel forms the centred z-DFT, the class and line weights, the
// compartment sum and the sampling per (volume, coil, partition, line, column); the spikes and
// noise run on the (volume, partition, coil) streams; one kernel applies the inverse z-DFT
// (1/nz) into per-slice coil k-spaces, and the 2D reconstruction (GRAPPA apply, window, inverse
// DFT, Roemer) runs on all slices of the chunk at once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "driver.h"
#include "grase3d.h"
#include "host3d.h"
#include "host_tables.h"
#include "mrsim_internal.h"
#include "recon_kernels.h"
#include "series_parts.h"

namespace mrsim {

namespace {

struct ZdftArgs {
  const float2* K;        // [gl][src][z][q][ky][kx]
  float2* out;            // [gl][q][p][ky][kx]
  const float2* zk;       // [p][z]
  const int* src;         // [c][p]: source index of compartment c at partition p
  const float* wc;        // [c][p][ky]: class line weight (1 for voxel compartments)
  const float* lw;        // [g][shot][c] or NULL
  const int* shot;        // [p][ky]
  const unsigned char* row_acquired;  // [ky]
  const int* line_var;    // [gl][p][ky]: the image variant a line reads (0: the volume's own), or NULL
  int nx, ny, nz, nc, ncomp, nsrc, n_shots, g0, nvar;
};

// out = sampling * sum_c lw(g, shot, c) * (w_c(p, ky) * sum_z K[var(p, ky)][src(c, p)][z] zk[p][z]), var
// the images the line's shot saw (`Plan::kspace` kspace3d.rs:206-232)
__global__ void grase_zdft_kernel(const ZdftArgs a) {
  const int per = a.nx * a.ny;
  const int p = blockIdx.y;
  const int gq = blockIdx.z;  // gl * nc + q
  const int gl = gq / a.nc, q = gq % a.nc;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < per; i += gridDim.x * blockDim.x) {
    const int ky = i / a.nx;
    float2 v = make_float2(0.f, 0.f);
    if (a.row_acquired[ky]) {
      for (int c = 0; c < a.ncomp; ++c) {
        const int s = a.src[c * a.nz + p];
        const int var = a.line_var ? a.line_var[((size_t)gl * a.nz + p) * a.ny + ky] : 0;
        const float2* Kc =
            a.K + ((size_t)((gl * a.nvar + var) * a.nsrc + s) * a.nz) * a.nc * per + (size_t)q * per + i;
        float ar = 0.f, ai = 0.f;
        for (int z = 0; z < a.nz; ++z) {
          const float2 k = Kc[(size_t)z * a.nc * per];
          const float2 e = a.zk[p * a.nz + z];
          ar += k.x * e.x - k.y * e.y;
          ai += k.x * e.y + k.y * e.x;
        }
        const float w = a.wc[((size_t)c * a.nz + p) * a.ny + ky];
        ar *= w;
        ai *= w;
        const float l = a.lw ? a.lw[((size_t)(a.g0 + gl) * a.n_shots + a.shot[p * a.ny + ky]) * a.ncomp + c] : 1.f;
        v.x += ar * l;
        v.y += ai * l;
      }
    }
    a.out[(((size_t)gl * a.nc + q) * a.nz + p) * per + i] = v;
  }
}

// slices[gl][z][q] = (1/nz) sum_p k3[gl][q][p] conj(zk[p][z])
__global__ void grase_izdft_kernel(const float2* __restrict__ k3, const float2* __restrict__ zk, int nx, int ny,
                                   int nz, int nc, float2* __restrict__ slices) {
  const int per = nx * ny;
  const int z = blockIdx.y;
  const int gq = blockIdx.z, gl = gq / nc, q = gq % nc;
  const float inv = 1.0f / (float)nz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < per; i += gridDim.x * blockDim.x) {
    float ar = 0.f, ai = 0.f;
    for (int p = 0; p < nz; ++p) {
      const float2 k = k3[(((size_t)gl * nc + q) * nz + p) * per + i];
      const float2 e = zk[p * nz + z];
      ar += k.x * e.x + k.y * e.y;
      ai += k.y * e.x - k.x * e.y;
    }
    slices[(((size_t)gl * nz + z) * nc + q) * per + i] = make_float2(ar * inv, ai * inv);
  }
}

// combined [gl][z][ny][nx] -> magnitude / phase at vox * nv + g
__global__ void volume_output_kernel(const float2* __restrict__ comb, int g0, int ngl, int nv, size_t nvox,
                                     float* __restrict__ mag, float* __restrict__ ph) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)ngl * nvox;
       i += (size_t)gridDim.x * blockDim.x) {
    const int gl = (int)(i / nvox);
    const size_t vox = i % nvox;
    const float2 c = comb[i];
    const size_t o = vox * nv + (g0 + gl);
    mag[o] = sqrtf(c.x * c.x + c.y * c.y);
    ph[o] = atan2f(c.y, c.x);
  }
}

dim3 grid3(size_t per, int y, int z) {
  return dim3((unsigned)std::max<size_t>(1, std::min<size_t>((per + 255) / 256, 1024)), (unsigned)y, (unsigned)z);
}

}  // namespace

// ---- the plan --------------------------------------------------------------------------------------
struct GrasePlan {
  int snx, sny, nz, nx, ny, o, ncomp, nc, etl;
  size_t plane, nvox;
  Grase3dTable table;
  LineTimingTab within;
  std::vector<CompMode> modes;
  std::vector<uint8_t> mask;
  std::vector<float2> zk;
  // sources: class compartment c -> one; voxel compartment c -> one per echo that reads a partition
  struct Src {
    int c, e;  // e = 0 for class
  };
  std::vector<Src> srcs;
  std::vector<int> src_of;  // [c][p]
  std::vector<float> wc;    // [c][p][ky]
  std::vector<int> shot;    // [p][ky]: the index of the line weights (GRASE's shot, GE's excitation)
  int n_shots = 0;
  std::vector<int> set_shot;  // [p][ky]: the shot whose images the line reads (`ShotSet` membership)
  int n_set_shots = 0;
  std::vector<char> used;   // per compartment
};

static GrasePlan make_plan(const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                           const mrsim_echo_train& train, const mrsim_grase_readout& ro) {
  GrasePlan P;
  P.snx = (int)in.sim_dims[0];
  P.sny = (int)in.sim_dims[1];
  P.nz = (int)in.sim_dims[2];
  P.nx = (int)in.acq_dims[0];
  P.ny = (int)in.acq_dims[1];
  if (P.nz != (int)in.acq_dims[2]) fail("partition count must match; z is never oversampled");
  if (P.snx <= 0 || P.sny <= 0 || P.nx <= 0 || P.ny <= 0 || P.nz <= 0) fail("empty simulation grid or acquired matrix");
  if (!(P.snx % P.nx == 0 && P.sny % P.ny == 0)) fail("sim grid must be an integer multiple of the acquired matrix");
  P.o = P.snx / P.nx;
  if (P.o != P.sny / P.ny) fail("oversampling must match on both axes");
  P.ncomp = (int)in.ncomp;
  if (P.ncomp > kMaxComp) fail("more than 8 compartments");
  P.nc = (int)std::max<int64_t>(acq.n_coils, 1);
  if (P.nc > kMaxCoils) fail("more than 64 coils");
  if (P.nx > 1024) fail("acquired matrix too wide for the reconstruction");
  P.plane = (size_t)P.snx * P.sny;
  P.nvox = P.plane * P.nz;
  if (!in.fmap) fail("fieldmap is not on the simulation grid");
  if (P.ncomp > 0 && (!in.images || !in.t2)) fail("compartment image is not on the simulation grid");
  if (acq.echo != MRSIM_ECHO_SPIN) fail("the 3D echo trains are spin-echo trains");
  if (acq.eddy_strength != 0.0 || acq.eddy_quad != 0.0 || acq.eddy_phase != 0.0)
    fail("the eddy model is not available in 3D (an echo-dependent eddy evolution breaks the z factorization)");
  if (!(acq.partial_fourier >= 1.0 || acq.pf_mode != MRSIM_PF_SCANNER))
    fail("Scanner partial Fourier is defined by the 2D EPI train; the 3D readouts take FiberfoxCompatible or "
         "Contiguous");
  if ((ro.reverse_phase != 0) != (acq.reverse_phase != 0))
    fail("the readout's phase-encode sign must be the acquisition's");
  P.table = grase_lines(train, ro, P.ny, P.nz);
  P.within.t_ms = P.table.block.t_ms;
  P.within.trf_ms = P.table.block.t_ms;
  P.within.tread_ms = P.table.block.t_ms;
  P.within.polarity = P.table.block.polarity;
  P.etl = (int)train.etl;
  P.shot.resize((size_t)P.nz * P.ny);
  for (int p = 0; p < P.nz; ++p)
    for (int ky = 0; ky < P.ny; ++ky) P.shot[(size_t)p * P.ny + ky] = P.table.line(p, ky).shot;
  P.n_shots = P.table.n_shots;
  P.set_shot = P.shot;
  P.n_set_shots = P.n_shots;
  P.used.assign(P.ncomp, 1);
  P.modes = resolve_modes(in.t2, in.t1, in.t_inhom, P.ncomp, acq, train, P.nvox);
  P.mask = sampling_mask(P.nx, P.ny, acq);
  const double zs = (double)(P.nz / 2);
  P.zk.resize((size_t)P.nz * P.nz);
  for (int p = 0; p < P.nz; ++p)
    for (int z = 0; z < P.nz; ++z) {
      const double th = kTau * ((double)p - zs) * ((double)z - zs) / (double)P.nz;  // `zkernel` kspace3d.rs:90-101
      P.zk[(size_t)p * P.nz + z] = make_float2((float)std::cos(th), (float)std::sin(th));
    }
  P.src_of.assign((size_t)P.ncomp * P.nz, 0);
  P.wc.assign((size_t)P.ncomp * P.nz * P.ny, 1.f);
  for (int c = 0; c < P.ncomp; ++c) {
    const CompMode& m = P.modes[c];
    if (!m.voxel) {
      const int s = (int)P.srcs.size();
      P.srcs.push_back({c, 0});
      for (int p = 0; p < P.nz; ++p) {
        P.src_of[(size_t)c * P.nz + p] = s;
        for (int ky = 0; ky < P.ny; ++ky) {
          const GraseLine& L = P.table.line(p, ky);
          P.wc[((size_t)c * P.nz + p) * P.ny + ky] =
              acq.do_relaxation ? (float)line_weight(m.ln_a[L.echo - 1], L.t_ms, m.t2_ms, m.t2p_ms) : 1.f;
        }
      }
    } else {
      int emax = 0;
      for (auto& L : P.table.lines) emax = std::max(emax, L.echo);
      for (int e = 1; e <= emax; ++e) {
        bool used = false;
        for (int p = 0; p < P.nz; ++p) used = used || P.table.line(p, 0).echo == e;
        if (!used) continue;
        const int s = (int)P.srcs.size();
        P.srcs.push_back({c, e});
        for (int p = 0; p < P.nz; ++p)
          if (P.table.line(p, 0).echo == e) P.src_of[(size_t)c * P.nz + p] = s;
      }
    }
  }
  return P;
}

// The device-resident inputs of one acquisition (images of every volume on the device, unit-major).
struct GraseInputs {
  float* img = nullptr;    // [g][z][c][plane]
  float* fmap = nullptr;   // [z][plane]
  float* t2 = nullptr;     // [c][nvox] (voxel compartments' values), or NULL
  float* ti = nullptr;
  float* lna = nullptr;    // [c][e][nvox] for voxel compartments
  int nv = 0;
};

static GraseInputs upload_inputs(DevArena& A, const GrasePlan& P, const mrsim_acquisition_3d_input& in,
                                 const float* const* images, int nv, const mrsim_acquisition& acq, cudaStream_t st) {
  GraseInputs I;
  I.nv = nv;
  const size_t per_comp = P.nvox * nv;
  float* staging = (float*)A.alloc(std::max<size_t>(1, per_comp * P.ncomp) * 4);
  for (int c = 0; c < P.ncomp; ++c)
    MRSIM_CUDA(cudaMemcpyAsync(staging + (size_t)c * per_comp, images[c], per_comp * 4, cudaMemcpyHostToDevice, st));
  I.img = (float*)A.alloc(std::max<size_t>(1, per_comp * P.ncomp) * 4);
  if (P.ncomp) launch_series_transpose(staging, I.img, P.ncomp, nv, P.nz, (int)P.plane, st);
  I.fmap = (float*)A.upload(in.fmap, P.nvox * 4, st);
  bool any_voxel = false;
  for (auto& m : P.modes) any_voxel = any_voxel || m.voxel;
  if (any_voxel) {
    std::vector<float> t2((size_t)P.ncomp * P.nvox, 1.f), ti((size_t)P.ncomp * P.nvox, 1.f);
    std::vector<float> la((size_t)P.ncomp * P.etl * P.nvox, 0.f);
    for (int c = 0; c < P.ncomp; ++c) {
      if (!P.modes[c].voxel) continue;
      for (size_t i = 0; i < P.nvox; ++i) {
        t2[(size_t)c * P.nvox + i] = in.t2[c].is_map ? in.t2[c].map[i] : in.t2[c].value;
        ti[(size_t)c * P.nvox + i] =
            in.t_inhom ? (in.t_inhom[c].is_map ? in.t_inhom[c].map[i] : in.t_inhom[c].value) : (float)acq.t_inhom;
      }
      for (int e = 0; e < P.etl; ++e)
        for (size_t i = 0; i < P.nvox; ++i)
          la[((size_t)c * P.etl + e) * P.nvox + i] = (float)P.modes[c].maps[e][i];
    }
    I.t2 = (float*)A.upload(t2.data(), t2.size() * 4, st);
    I.ti = (float*)A.upload(ti.data(), ti.size() * 4, st);
    I.lna = (float*)A.upload(la.data(), la.size() * 4, st);
  }
  return I;
}

// Per-shot images of the volumes of a chunk (`ShotSet`, kspace3d.rs:59-65): variant 0 is each
// volume's own images, variant v > 0 its set v - 1 (one device volume per used compartment);
// per volume and line the variant the line reads (the first set holding its shot).
struct ShotVariants {
  int nvar = 1;
  std::vector<std::vector<const float*>> img;  // [gl * nvar + v][c] (v > 0; NULL: no such set)
  const int* d_line_var = nullptr;             // [gl][p][ky], or NULL when no volume has sets
};

// The sets of volumes g0..g1 (`sets[gl]`, `n_sets[gl]`): checked (shots inside the train, an
// image for every compartment the volume uses), uploaded, and the line table built.
static ShotVariants upload_sets(DevArena& A, const GrasePlan& P, const std::vector<const mrsim_shot_set*>& sets,
                                const std::vector<int64_t>& n_sets, int first_g, cudaStream_t st, bool upload = true) {
  ShotVariants V;
  const int ngl = (int)sets.size();
  int64_t most = 0;
  for (int gl = 0; gl < ngl; ++gl) most = std::max<int64_t>(most, sets[gl] ? n_sets[gl] : 0);
  if (most == 0) return V;
  V.nvar = (int)most + 1;
  V.img.assign((size_t)ngl * V.nvar, std::vector<const float*>(P.ncomp, nullptr));
  std::vector<int> line_var((size_t)ngl * P.nz * P.ny, 0);
  for (int gl = 0; gl < ngl; ++gl) {
    if (!sets[gl]) continue;
    for (int64_t i = 0; i < n_sets[gl]; ++i) {
      const mrsim_shot_set& S = sets[gl][i];
      if (S.n_shots > 0 && !S.shots) fail("volume " + std::to_string(first_g + gl) + ": a shot set's shots are NULL");
      for (int64_t j = 0; j < S.n_shots; ++j)
        if (S.shots[j] < 0 || S.shots[j] >= P.n_set_shots)
          fail("a shot index beyond the train's " + std::to_string(P.n_set_shots));
      for (int c = 0; c < P.ncomp; ++c) {
        if (!P.used[c]) {
          if (S.images && S.images[c])
            fail("volume " + std::to_string(first_g + gl) + ": shot images are not the volume's compartments");
          continue;
        }
        if (!S.images || !S.images[c])
          fail("volume " + std::to_string(first_g + gl) + ": shot images are not the volume's compartments");
        if (upload) V.img[(size_t)gl * V.nvar + i + 1][c] = (const float*)A.upload(S.images[c], P.nvox * 4, st);
      }
    }
    for (size_t l = 0; l < P.set_shot.size() && upload; ++l) {
      const int64_t shot = P.set_shot[l];
      for (int64_t i = 0; i < n_sets[gl]; ++i) {
        const mrsim_shot_set& S = sets[gl][i];
        if (std::find(S.shots, S.shots + S.n_shots, shot) != S.shots + S.n_shots) {
          line_var[(size_t)gl * P.set_shot.size() + l] = (int)i + 1;
          break;
        }
      }
    }
  }
  if (upload) V.d_line_var = (const int*)A.upload(line_var.data(), line_var.size() * 4, st);
  return V;
}

// The 3D input's sets of volumes g0..g1.
static ShotVariants input_sets(DevArena& A, const GrasePlan& P, const mrsim_acquisition_3d_input& in, int g0, int g1,
                               cudaStream_t st, bool upload = true) {
  std::vector<const mrsim_shot_set*> sets;
  std::vector<int64_t> n;
  for (int g = g0; g < g1; ++g) {
    const bool has = in.shot_sets && in.n_shot_sets && in.n_shot_sets[g] > 0;
    if (has && !in.shot_sets[g]) fail("volume " + std::to_string(g) + ": its shot sets are NULL");
    sets.push_back(has ? in.shot_sets[g] : nullptr);
    n.push_back(has ? in.n_shot_sets[g] : 0);
  }
  return upload_sets(A, P, sets, n, g0, st, upload);
}
// The most image variants any volume needs (1 + its sets).
static int most_variants(const mrsim_acquisition_3d_input& in) {
  int64_t most = 0;
  if (in.shot_sets && in.n_shot_sets)
    for (int64_t g = 0; g < in.n_volumes; ++g) most = std::max<int64_t>(most, in.n_shot_sets[g]);
  return (int)most + 1;
}

// The acquired 3D k-space (before spikes and noise) of volumes g0..g1 into k3 [gl][q][p][ky][kx].
static void grase_kspace(const GrasePlan& P, const GraseInputs& I, const mrsim_acquisition& acq,
                         const mrsim_phase_model* phase, const float* d_lw, int g0, int g1,
                         const std::vector<uint8_t>& mask, float2* k3, cudaStream_t st,
                         const ShotVariants* V = nullptr) {
  const int ngl = g1 - g0, nsrc = (int)P.srcs.size(), nz = P.nz, nc = P.nc;
  const int nvar = V ? V->nvar : 1;
  const size_t per = (size_t)P.nx * P.ny;
  DevArena C;
  mrsim_acquisition norel = acq;
  norel.do_relaxation = 0;
  norel.noise_variance = 0.0;
  norel.n_spikes = 0;
  mrsim_acquisition rel = norel;
  rel.do_relaxation = 1;
  float one[kMaxComp];
  for (int c = 0; c < kMaxComp; ++c) one[c] = 1.f;
  std::vector<LineRec> Lc, Lv;
  lines_for(Lc, norel, P.nx, P.ny, false, true, 1, one, one, false, &P.within);
  lines_for(Lv, rel, P.nx, P.ny, false, false, 1, one, one, false, &P.within);
  const int n_lines = (int)Lc.size();
  const LineRec* dLc = (const LineRec*)C.upload(Lc.data(), std::max<size_t>(1, Lc.size()) * sizeof(LineRec), st);
  const LineRec* dLv = (const LineRec*)C.upload(Lv.data(), std::max<size_t>(1, Lv.size()) * sizeof(LineRec), st);
  const size_t nunit = (size_t)ngl * nvar * nsrc * nz;
  float2* K = (float2*)C.alloc(std::max<size_t>(1, nunit * nc * per) * sizeof(float2));
  MRSIM_CUDA(cudaMemsetAsync(K, 0, nunit * nc * per * sizeof(float2), st));
  float2* gs = (float2*)C.alloc(std::max<size_t>(1, nunit * nc * std::max(n_lines, 1) * P.snx) * sizeof(float2));
  float* ph = (float*)C.alloc(std::max<size_t>(1, nunit * P.plane) * 4);
  GeoTab geo = build_geo(C, P.snx, P.sny, P.nx, P.ny, nc, acq.ghost_offset, st);
  mrsim_phase_model zero;
  std::memset(&zero, 0, sizeof zero);
  Batch Bc, Bv;
  for (int gl = 0; gl < ngl; ++gl)
    for (int var = 0; var < nvar; ++var)
    for (int s = 0; s < nsrc; ++s)
      for (int z = 0; z < nz; ++z) {
        const GrasePlan::Src& S = P.srcs[s];
        const size_t u = (((size_t)gl * nvar + var) * nsrc + s) * nz + z;
        const float* set_img = var > 0 ? V->img[(size_t)gl * nvar + var][S.c] : nullptr;
        if (var > 0 && !set_img) continue;  // a volume with fewer sets, or a compartment it does not use
        UnitInputs ui;
        std::memset(&ui, 0, sizeof ui);
        ui.comp = var > 0 ? set_img + (size_t)z * P.plane
                          : I.img + (((size_t)(g0 + gl) * nz + z) * P.ncomp + S.c) * P.plane;
        ui.comp_stride = (long long)P.plane;
        ui.fmap = I.fmap + (size_t)z * P.plane;
        ui.map_stride = (long long)P.nvox;
        ui.kspace = K + u * nc * per;
        ui.g = gs + u * nc * std::max(n_lines, 1) * P.snx;
        ui.phase_out = ph + u * P.plane;
        ui.phase = phase ? phase : &zero;
        ui.z = z;
        ui.nz_full = nz;
        const CompMode& m = P.modes[S.c];
        if (!P.used[S.c]) continue;
        if (!m.voxel) {
          ui.lines = dLc;
          ui.n_lines = n_lines;
          add_unit(Bc, ui, P.snx, P.sny, P.nx, P.ny, 1, nc, false, one, one, geo, norel);
        } else {
          ui.t2map = I.t2 + (size_t)S.c * P.nvox + (size_t)z * P.plane;
          ui.timap = I.ti + (size_t)S.c * P.nvox + (size_t)z * P.plane;
          ui.log_amp = S.e > 0 ? I.lna + ((size_t)S.c * P.etl + (S.e - 1)) * P.nvox + (size_t)z * P.plane : nullptr;
          ui.lines = dLv;
          ui.n_lines = n_lines;
          add_unit(Bv, ui, P.snx, P.sny, P.nx, P.ny, 1, nc, true, one, one, geo, rel);
        }
      }
  if (n_lines > 0) {
    run_forward(Bc, st);
    run_forward(Bv, st);
  }
  // the z-DFT, weights, compartment sum and sampling
  std::vector<unsigned char> rows(P.ny);
  for (int ky = 0; ky < P.ny; ++ky) rows[ky] = mask[(size_t)ky * P.nx] ? 1 : 0;
  const std::vector<int>& shot = P.shot;
  ZdftArgs a;
  a.K = K;
  a.out = k3;
  a.zk = (const float2*)C.upload(P.zk.data(), P.zk.size() * sizeof(float2), st);
  a.src = (const int*)C.upload(P.src_of.data(), std::max<size_t>(1, P.src_of.size()) * 4, st);
  a.wc = (const float*)C.upload(P.wc.data(), std::max<size_t>(1, P.wc.size()) * 4, st);
  a.lw = d_lw;
  a.shot = (const int*)C.upload(shot.data(), shot.size() * 4, st);
  a.row_acquired = (const unsigned char*)C.upload(rows.data(), rows.size(), st);
  a.nx = P.nx;
  a.ny = P.ny;
  a.nz = nz;
  a.nc = nc;
  a.ncomp = P.ncomp;
  a.nsrc = nsrc;
  a.n_shots = P.n_shots;
  a.g0 = g0;
  a.line_var = V ? V->d_line_var : nullptr;
  a.nvar = nvar;
  grase_zdft_kernel<<<grid3(per, nz, ngl * nc), 256, 0, st>>>(a);
  MRSIM_CUDA(cudaGetLastError());
  MRSIM_CUDA(cudaStreamSynchronize(st));  // C's buffers are freed on return
}

// spikes and noise per (volume, partition, coil) (`partitions_to_slices` kspace3d.rs:235-262)
static void grase_noise(DevArena& A, const GrasePlan& P, float2* k3, int g0, int g1, uint64_t seed,
                        const std::vector<uint8_t>& mask, const mrsim_acquisition& acq, cudaStream_t st) {
  if (acq.n_spikes <= 0 && !(acq.noise_variance > 0.0)) return;
  const size_t per = (size_t)P.nx * P.ny;
  std::vector<int> acquired, rows;
  for (size_t i = 0; i < per; ++i)
    if (mask[i]) acquired.push_back((int)i);
  for (int ky = 0; ky < P.ny; ++ky)
    if (mask[(size_t)ky * P.nx]) rows.push_back(ky);
  std::vector<NoiseSpec> specs;
  std::vector<int> picks;
  for (int g = g0; g < g1; ++g)
    for (int p = 0; p < P.nz; ++p) {
      const uint64_t pseed = (((uint64_t)g * 0x1000001ull) + (uint64_t)p) * 0x9E37ull ^ seed ^ kSeedSalt3d;
      for (int q = 0; q < P.nc; ++q) {
        const int off = (int)picks.size();
        if (acq.n_spikes > 0) {  // `spike_picks` kspace3d.rs:327-332: a stream per coil
          Rng rng(pseed ^ 0xA5A5123456789ABCull ^ ((uint64_t)q * 0xC2B2AE3D27D4EB4Full));
          for (int64_t s = 0; s < acq.n_spikes; ++s)
            picks.push_back(acquired.empty() ? 0 : acquired[(size_t)(rng.next_u64() % (uint64_t)acquired.size())]);
        }
        specs.push_back({k3 + (((size_t)(g - g0) * P.nc + q) * P.nz + p) * per, pseed, q, off});
      }
    }
  run_noise(A, specs, rows, picks, P.nx, P.ny, acq, st);
  MRSIM_CUDA(cudaGetLastError());
}

void grase_observed(mrsim_context* ctx, const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                    const mrsim_echo_train& train, const mrsim_grase_readout& ro, int g, float* out) {
  cudaStream_t st = ctx->stream;
  GrasePlan P = make_plan(in, acq, train, ro);
  if (g < 0 || g >= (int)in.n_volumes) fail("volume index out of range");
  DevArena A;
  GraseInputs I = upload_inputs(A, P, in, in.images, (int)in.n_volumes, acq, st);
  const float* d_lw = nullptr;
  if (in.line_weights) {
    std::vector<float> lw((size_t)in.n_volumes * P.table.n_shots * P.ncomp);
    for (size_t i = 0; i < lw.size(); ++i) lw[i] = (float)in.line_weights[i];
    d_lw = (const float*)A.upload(lw.data(), lw.size() * 4, st);
  }
  const size_t per = (size_t)P.nx * P.ny;
  float2* k3 = (float2*)A.alloc((size_t)P.nc * P.nz * per * sizeof(float2));
  ShotVariants V = input_sets(A, P, in, g, g + 1, st);
  grase_kspace(P, I, acq, in.phase, d_lw, g, g + 1, P.mask, k3, st, &V);
  copy_pageable_d2h(ctx, out, k3, (size_t)P.nc * P.nz * per * sizeof(float2), st);
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

void grase_acquire(mrsim_context* ctx, const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                   const mrsim_echo_train& train, const mrsim_grase_readout& ro, uint64_t seed, float* mag,
                   float* ph) {
  cudaStream_t st = ctx->stream;
  GrasePlan P = make_plan(in, acq, train, ro);
  const int nv = (int)in.n_volumes, nz = P.nz, nc = P.nc, nx = P.nx, ny = P.ny;
  const size_t per = (size_t)nx * ny;
  const int accel = (int)std::max<int64_t>(acq.accel, 1);
  const int nvar = most_variants(in);
  DevArena A;
  if (nvar > 1) (void)input_sets(A, P, in, 0, nv, st, false);  // every volume's sets checked before any work
  GraseInputs I = upload_inputs(A, P, in, in.images, nv, acq, st);
  const float* d_lw = nullptr;
  if (in.line_weights) {
    std::vector<float> lw((size_t)nv * P.table.n_shots * P.ncomp);
    for (size_t i = 0; i < lw.size(); ++i) lw[i] = (float)in.line_weights[i];
    d_lw = (const float*)A.upload(lw.data(), std::max<size_t>(1, lw.size()) * 4, st);
  }
  const float2* d_zk = (const float2*)A.upload(P.zk.data(), P.zk.size() * sizeof(float2), st);
  // GRAPPA: one kernel per slice, fitted on the reference scan (`grappa_kernels_3d`)
  float2* W = nullptr;
  const size_t w_per_slice = (size_t)(accel - 1) * nc * 6 * nc;
  if (accel > 1 && nv > 0) {
    mrsim_acquisition acq_cal = acq;
    acq_cal.accel = 1;
    acq_cal.n_spikes = 0;
    GrasePlan Pc = make_plan(in, acq_cal, train, ro);
    DevArena C;
    const float* const* cal_images = in.images;
    int cal_nv = nv;
    uint64_t cal_seed = seed;
    if (in.has_grappa_calibration) {
      if (!in.grappa_calibration_images) fail("the GRAPPA calibration images are NULL");
      cal_images = in.grappa_calibration_images;
      cal_nv = 1;
      cal_seed = in.grappa_calibration_seed;
    }
    GraseInputs Ic = upload_inputs(C, Pc, in, cal_images, cal_nv, acq_cal, st);
    float2* k3 = (float2*)C.alloc((size_t)nc * nz * per * sizeof(float2));
    grase_kspace(Pc, Ic, acq_cal, in.phase, nullptr, 0, 1, Pc.mask, k3, st);
    grase_noise(C, Pc, k3, 0, 1, cal_seed ^ kSeedSaltGrappaCal, Pc.mask, acq_cal, st);
    float2* sl = (float2*)C.alloc((size_t)nz * nc * per * sizeof(float2));
    grase_izdft_kernel<<<grid3(per, nz, nc), 256, 0, st>>>(k3, d_zk, nx, ny, nz, nc, sl);
    std::vector<float2*> refs;
    for (int z = 0; z < nz; ++z) refs.push_back(sl + (size_t)z * nc * per);
    W = fit_grappa(A, refs, nx, ny, nc, acq_cal, accel, (int)acq.acs_lines, st);
    MRSIM_CUDA(cudaStreamSynchronize(st));
  }
  ReconTables T = build_recon_tables(A, nx, ny, nc, acq, st);
  float* d_mag = (float*)A.alloc(std::max<size_t>(1, per * nz * nv) * 4);
  float* d_ph = (float*)A.alloc(std::max<size_t>(1, per * nz * nv) * 4);
  // chunks of volumes within a scratch budget
  const size_t nsrc = P.srcs.size();
  const size_t bytes_per_vol = ((nsrc * nz * nc * per * 8) * 2 + nsrc * nz * (size_t)nc * ny * P.snx * 8) * nvar +
                               (size_t)(nvar - 1) * P.ncomp * P.nvox * 4 + (size_t)nc * nz * per * 8 * 2 +
                               (size_t)nz * per * 8;
  const size_t budget = (size_t)4 << 30;
  const int vchunk = (int)std::max<size_t>(1, std::min<size_t>(std::max(nv, 1), budget / std::max<size_t>(1, bytes_per_vol)));
  for (int g0 = 0; g0 < nv; g0 += vchunk) {
    const int g1 = std::min(nv, g0 + vchunk), ngl = g1 - g0;
    DevArena C;
    float2* k3 = (float2*)C.alloc((size_t)ngl * nc * nz * per * sizeof(float2));
    ShotVariants V = input_sets(C, P, in, g0, g1, st);
    grase_kspace(P, I, acq, in.phase, d_lw, g0, g1, P.mask, k3, st, &V);
    grase_noise(C, P, k3, g0, g1, seed, P.mask, acq, st);
    float2* sl = (float2*)C.alloc((size_t)ngl * nz * nc * per * sizeof(float2));
    grase_izdft_kernel<<<grid3(per, nz, ngl * nc), 256, 0, st>>>(k3, d_zk, nx, ny, nz, nc, sl);
    float2* comb = (float2*)C.alloc((size_t)ngl * nz * per * sizeof(float2));
    std::vector<ReconJob> jobs;
    for (int gl = 0; gl < ngl; ++gl)
      for (int z = 0; z < nz; ++z) {
        ReconJob J;
        std::memset(&J, 0, sizeof J);
        J.k = sl + ((size_t)gl * nz + z) * nc * per;
        J.grappa_w = W ? W + (size_t)z * w_per_slice : nullptr;
        J.window = T.window;
        J.ex_tab = T.ex_tab;
        J.ey_tab = T.ey_tab;
        J.sens = T.sens;
        J.inv_ssum = T.inv_ssum;
        J.combined = comb + ((size_t)gl * nz + z) * per;
        J.nx = nx;
        J.ny = ny;
        J.nc = nc;
        jobs.push_back(J);
      }
    const ReconJob* d_jobs = (const ReconJob*)C.upload(jobs.data(), jobs.size() * sizeof(ReconJob), st);
    if (accel > 1) launch_grappa_apply(d_jobs, (int)jobs.size(), T.fills, T.n_fills, nx, nc, st);
    launch_recon_combine(d_jobs, (int)jobs.size(), nx, ny, false, st);
    volume_output_kernel<<<1024, 256, 0, st>>>(comb, g0, ngl, nv, per * nz, d_mag, d_ph);
    MRSIM_CUDA(cudaGetLastError());
    MRSIM_CUDA(cudaStreamSynchronize(st));
  }
  copy_pageable_d2h(ctx, mag, d_mag, per * nz * nv * 4, st);
  copy_pageable_d2h(ctx, ph, d_ph, per * nz * nv * 4, st);
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

// ---- the 3D gradient-echo train (`simulate_acquisition_3d_ge_complex`, kspace3d.rs:732-835) -------
// Per echo: the 2D forward with gradient-echo formation at t_echo = TE_e, its line timing
// t = the block's, trf = TE_e + t; class compartments (uniform T2, T2') take the decay
// exp(-(TE_e + t)(1/T2 + 1/T2')) as a line weight, the others decay inside the forward.  The
// per-excitation weights w[(p ky_segments + sy) ncomp + c] enter as the z-DFT's line weights.
namespace {

struct GeVolumeData {
  std::vector<const float*> images;  // ncomp (NULL = unused)
  std::vector<double> weights;
  const mrsim_shot_set* sets = nullptr;  // `shot_images` (the reference scan takes none)
  int64_t n_sets = 0;
};

GeVolumeData fetch_ge_volume(const mrsim_acquisition_ge_input& in, int g, int n_exc_lines) {
  mrsim_ge_volume v;
  std::memset(&v, 0, sizeof v);
  if (!in.volume) fail("the volume callback is NULL");
  if (in.volume(g, in.user, &v) != 0) fail("volume " + std::to_string(g) + ": the volume callback failed");
  GeVolumeData d;
  d.images.assign((size_t)in.ncomp, nullptr);
  if (in.ncomp > 0 && !v.images) fail("volume " + std::to_string(g) + ": no compartment images");
  for (int c = 0; c < (int)in.ncomp; ++c) d.images[c] = v.images[c];
  if (!v.weights) fail("volume " + std::to_string(g) + ": weights are not (partition, ky segment, compartment)");
  d.weights.assign(v.weights, v.weights + n_exc_lines);
  if (v.n_shot_sets > 0) {
    if (!v.shot_sets) fail("volume " + std::to_string(g) + ": its shot sets are NULL");
    d.sets = v.shot_sets;
    d.n_sets = v.n_shot_sets;
  }
  for (int c = 0; c < (int)in.ncomp; ++c)
    if (!d.images[c])
      for (int x = 0; x < n_exc_lines / std::max<int>(1, (int)in.ncomp); ++x)
        if (d.weights[(size_t)x * in.ncomp + c] != 0.0)
          fail("volume " + std::to_string(g) + ": compartment " + std::to_string(c) +
               " has no image but a nonzero weight");
  return d;
}

}  // namespace

static GrasePlan make_ge_plan(const mrsim_acquisition_ge_input& in, const mrsim_acquisition& acq,
                              const mrsim_excitation_train& train, const mrsim_ge3d_readout& ro, Ge3dTable& table) {
  GrasePlan P;
  P.snx = (int)in.sim_dims[0];
  P.sny = (int)in.sim_dims[1];
  P.nz = (int)in.sim_dims[2];
  P.nx = (int)in.acq_dims[0];
  P.ny = (int)in.acq_dims[1];
  if (P.nz != (int)in.acq_dims[2]) fail("partition count must match; z is never oversampled");
  if (P.snx <= 0 || P.sny <= 0 || P.nx <= 0 || P.ny <= 0 || P.nz <= 0) fail("empty simulation grid or acquired matrix");
  if (!(P.snx % P.nx == 0 && P.sny % P.ny == 0)) fail("sim grid must be an integer multiple of the acquired matrix");
  P.o = P.snx / P.nx;
  if (P.o != P.sny / P.ny) fail("oversampling must match on both axes");
  P.ncomp = (int)in.ncomp;
  if (P.ncomp > kMaxComp) fail("more than 8 compartments");
  P.nc = (int)std::max<int64_t>(acq.n_coils, 1);
  if (P.nc > kMaxCoils) fail("more than 64 coils");
  if (P.nx > 1024) fail("acquired matrix too wide for the reconstruction");
  P.plane = (size_t)P.snx * P.sny;
  P.nvox = P.plane * P.nz;
  if (!in.fmap) fail("fieldmap is not on the simulation grid");
  if (P.ncomp > 0 && !in.t2) fail("t2 has 0 entries for " + std::to_string(P.ncomp) + " compartments");
  if (acq.echo != MRSIM_ECHO_GRADIENT) fail("the 3D gradient-echo train is a gradient-echo acquisition");
  if (acq.eddy_strength != 0.0 || acq.eddy_quad != 0.0 || acq.eddy_phase != 0.0)
    fail("the eddy model is not available in 3D (an excitation-dependent eddy evolution breaks the z factorization)");
  if (!(acq.partial_fourier >= 1.0)) fail("partial Fourier is not available on the 3D gradient-echo train");
  if ((ro.reverse_phase != 0) != (acq.reverse_phase != 0))
    fail("the readout's phase-encode sign must be the acquisition's");
  if (train.n_echoes < 1 || !train.echo_times_ms) fail("a 3D gradient-echo train needs at least one echo time");
  table = ge3d_lines(train, ro, P.ny, P.nz);
  P.etl = 0;
  P.shot.resize((size_t)P.nz * P.ny);
  const int kys = (int)ro.ky_segments;
  for (int p = 0; p < P.nz; ++p)
    for (int ky = 0; ky < P.ny; ++ky) P.shot[(size_t)p * P.ny + ky] = p * kys + ky % kys;
  P.n_shots = P.nz * kys;
  P.set_shot.resize((size_t)P.nz * P.ny);
  for (int p = 0; p < P.nz; ++p)
    for (int ky = 0; ky < P.ny; ++ky) P.set_shot[(size_t)p * P.ny + ky] = table.line(p, ky).shot;
  P.n_set_shots = table.n_shots;
  P.used.assign(P.ncomp, 1);
  P.modes.resize(P.ncomp);
  for (int c = 0; c < P.ncomp; ++c) {
    const mrsim_t2 ti = in.t_inhom ? in.t_inhom[c] : mrsim_t2{nullptr, (float)acq.t_inhom, 0};
    CompMode& m = P.modes[c];
    if (!in.t2[c].is_map && !ti.is_map) {
      m.t2_ms = in.t2[c].value;
      m.t2p_ms = ti.value;
    } else if (acq.do_relaxation) {
      m.voxel = true;  // decay inside the forward; no echo amplitudes on a gradient-echo train
    } else {
      m.t2_ms = INFINITY;
      m.t2p_ms = INFINITY;
    }
  }
  P.mask = sampling_mask(P.nx, P.ny, acq);
  const double zs = (double)(P.nz / 2);
  P.zk.resize((size_t)P.nz * P.nz);
  for (int p = 0; p < P.nz; ++p)
    for (int z = 0; z < P.nz; ++z) {
      const double th = kTau * ((double)p - zs) * ((double)z - zs) / (double)P.nz;
      P.zk[(size_t)p * P.nz + z] = make_float2((float)std::cos(th), (float)std::sin(th));
    }
  P.src_of.assign((size_t)P.ncomp * P.nz, 0);
  for (int c = 0; c < P.ncomp; ++c) {
    P.srcs.push_back({c, 0});
    for (int p = 0; p < P.nz; ++p) P.src_of[(size_t)c * P.nz + p] = c;
  }
  P.within.t_ms = table.block.t_ms;
  P.within.tread_ms = table.block.t_ms;
  P.within.polarity = table.block.polarity;
  return P;
}

// The plan of echo e: the line timing at TE_e and the class decay weights.
static void ge_echo(GrasePlan& P, const mrsim_acquisition& acq, double te) {
  P.within.trf_ms.resize(P.ny);
  for (int ky = 0; ky < P.ny; ++ky) P.within.trf_ms[ky] = te + P.within.t_ms[ky];
  P.wc.assign((size_t)P.ncomp * P.nz * P.ny, 1.f);
  for (int c = 0; c < P.ncomp; ++c) {
    const CompMode& m = P.modes[c];
    if (m.voxel || !acq.do_relaxation) continue;
    for (int ky = 0; ky < P.ny; ++ky) {
      const double trf = te + P.within.t_ms[ky];  // `ge_line_weight` kspace3d.rs:607-612
      const double d2 = std::isinf(m.t2_ms) ? 0.0 : trf / m.t2_ms;
      const double dp = std::isinf(m.t2p_ms) ? 0.0 : trf / m.t2p_ms;
      const float w = (float)std::exp(-d2 - dp);
      for (int p = 0; p < P.nz; ++p) P.wc[((size_t)c * P.nz + p) * P.ny + ky] = w;
    }
  }
}

// One volume's inputs (images of the compartments it uses, voxel maps) and its weights.
static GraseInputs upload_ge_volume(DevArena& A, const GrasePlan& P, const mrsim_acquisition_ge_input& in,
                                    const GeVolumeData& v, const mrsim_acquisition& acq, const float** d_lw,
                                    cudaStream_t st) {
  GraseInputs I;
  I.nv = 1;
  I.img = (float*)A.alloc(std::max<size_t>(1, P.nvox * P.ncomp) * 4);
  MRSIM_CUDA(cudaMemsetAsync(I.img, 0, std::max<size_t>(1, P.nvox * P.ncomp) * 4, st));
  for (int c = 0; c < P.ncomp; ++c) {
    if (!v.images[c]) continue;
    for (int z = 0; z < P.nz; ++z)  // [z][c][plane]
      MRSIM_CUDA(cudaMemcpyAsync(I.img + ((size_t)z * P.ncomp + c) * P.plane, v.images[c] + (size_t)z * P.plane,
                                 P.plane * 4, cudaMemcpyHostToDevice, st));
  }
  I.fmap = (float*)A.upload(in.fmap, P.nvox * 4, st);
  bool any_voxel = false;
  for (auto& m : P.modes) any_voxel = any_voxel || m.voxel;
  if (any_voxel) {
    std::vector<float> t2((size_t)P.ncomp * P.nvox, 1.f), ti((size_t)P.ncomp * P.nvox, 1.f);
    for (int c = 0; c < P.ncomp; ++c) {
      if (!P.modes[c].voxel) continue;
      for (size_t i = 0; i < P.nvox; ++i) {
        t2[(size_t)c * P.nvox + i] = in.t2[c].is_map ? in.t2[c].map[i] : in.t2[c].value;
        ti[(size_t)c * P.nvox + i] =
            in.t_inhom ? (in.t_inhom[c].is_map ? in.t_inhom[c].map[i] : in.t_inhom[c].value) : (float)acq.t_inhom;
      }
    }
    I.t2 = (float*)A.upload(t2.data(), t2.size() * 4, st);
    I.ti = (float*)A.upload(ti.data(), ti.size() * 4, st);
  }
  std::vector<float> lw(v.weights.begin(), v.weights.end());
  *d_lw = (const float*)A.upload(lw.data(), std::max<size_t>(1, lw.size()) * 4, st);
  return I;
}

void ge_acquire(mrsim_context* ctx, const mrsim_acquisition_ge_input& in, const mrsim_acquisition& acq,
                const mrsim_excitation_train& train, const mrsim_ge3d_readout& ro, uint64_t seed, float* const* mag,
                float* const* ph) {
  cudaStream_t st = ctx->stream;
  Ge3dTable table;
  GrasePlan P = make_ge_plan(in, acq, train, ro, table);
  const int nv = (int)in.n_volumes, nz = P.nz, nc = P.nc, nx = P.nx, ny = P.ny;
  const int n_echoes = (int)train.n_echoes, n_exc_lines = nz * (int)ro.ky_segments * P.ncomp;
  const size_t per = (size_t)nx * ny;
  const int accel = (int)std::max<int64_t>(acq.accel, 1);
  for (int e = 0; e < n_echoes; ++e) {
    if (!mag || !ph || !mag[e] || !ph[e]) fail("an output buffer of echo " + std::to_string(e) + " is NULL");
    if (e > 0 && !(train.echo_times_ms[e] > train.echo_times_ms[e - 1]))
      fail("the echo times must increase strictly");
  }
  DevArena A;
  const float2* d_zk = (const float2*)A.upload(P.zk.data(), P.zk.size() * sizeof(float2), st);
  ReconTables T = build_recon_tables(A, nx, ny, nc, acq, st);
  const size_t w_per_slice = (size_t)(accel - 1) * nc * 6 * nc;
  // GRAPPA: per echo, one kernel per slice from the reference scan (`reference`, else volume 0)
  std::vector<float2*> W(n_echoes, nullptr);
  if (accel > 1 && nv > 0) {
    GeVolumeData ref;
    if (in.reference) {
      ref.images.assign(in.reference->images, in.reference->images + in.ncomp);
      ref.weights.assign(in.reference->weights, in.reference->weights + n_exc_lines);
    } else {
      ref = fetch_ge_volume(in, 0, n_exc_lines);
      ref.sets = nullptr;  // `GeVolume { shot_images: None, .. }` (kspace3d.rs:775)
      ref.n_sets = 0;
    }
    mrsim_acquisition acq_cal = acq;
    acq_cal.accel = 1;
    acq_cal.n_spikes = 0;
    GrasePlan Pc = P;
    Pc.mask = sampling_mask(nx, ny, acq_cal);
    for (int c = 0; c < P.ncomp; ++c) Pc.used[c] = ref.images[c] != nullptr;
    DevArena C;
    const float* d_lw = nullptr;
    GraseInputs Ic = upload_ge_volume(C, Pc, in, ref, acq, &d_lw, st);
    for (int e = 0; e < n_echoes; ++e) {
      const double te = train.echo_times_ms[e];
      ge_echo(Pc, acq_cal, te);
      mrsim_acquisition ae = acq_cal;
      ae.t_echo = te;
      float2* k3 = (float2*)C.alloc((size_t)nc * nz * per * sizeof(float2));
      grase_kspace(Pc, Ic, ae, in.phase, d_lw, 0, 1, Pc.mask, k3, st);
      grase_noise(C, Pc, k3, 0, 1, (seed ^ echo_salt((uint64_t)e)) ^ kSeedSaltGrappaCal, Pc.mask, acq_cal, st);
      float2* sl = (float2*)C.alloc((size_t)nz * nc * per * sizeof(float2));
      grase_izdft_kernel<<<grid3(per, nz, nc), 256, 0, st>>>(k3, d_zk, nx, ny, nz, nc, sl);
      std::vector<float2*> refs;
      for (int z = 0; z < nz; ++z) refs.push_back(sl + (size_t)z * nc * per);
      W[e] = fit_grappa(A, refs, nx, ny, nc, acq_cal, accel, (int)acq.acs_lines, st);
      MRSIM_CUDA(cudaStreamSynchronize(st));
    }
  }
  std::vector<float*> d_mag(n_echoes), d_ph(n_echoes);
  for (int e = 0; e < n_echoes; ++e) {
    d_mag[e] = (float*)A.alloc(std::max<size_t>(1, per * nz * nv) * 4);
    d_ph[e] = (float*)A.alloc(std::max<size_t>(1, per * nz * nv) * 4);
  }
  for (int g = 0; g < nv; ++g) {
    GeVolumeData v = fetch_ge_volume(in, g, n_exc_lines);
    GrasePlan Pg = P;
    for (int c = 0; c < P.ncomp; ++c) Pg.used[c] = v.images[c] != nullptr;
    DevArena C;
    const float* d_lw = nullptr;
    GraseInputs I = upload_ge_volume(C, Pg, in, v, acq, &d_lw, st);
    const ShotVariants V = upload_sets(C, Pg, {v.sets}, {v.n_sets}, g, st);
    for (int e = 0; e < n_echoes; ++e) {
      const double te = train.echo_times_ms[e];
      ge_echo(Pg, acq, te);
      mrsim_acquisition ae = acq;
      ae.t_echo = te;
      DevArena E;
      float2* k3 = (float2*)E.alloc((size_t)nc * nz * per * sizeof(float2));
      grase_kspace(Pg, I, ae, in.phase, d_lw, 0, 1, Pg.mask, k3, st, &V);
      // the noise and spikes of echo e on its own streams (echo 0 unsalted)
      grase_noise(E, Pg, k3, g, g + 1, seed ^ echo_salt((uint64_t)e), Pg.mask, acq, st);
      float2* sl = (float2*)E.alloc((size_t)nz * nc * per * sizeof(float2));
      grase_izdft_kernel<<<grid3(per, nz, nc), 256, 0, st>>>(k3, d_zk, nx, ny, nz, nc, sl);
      float2* comb = (float2*)E.alloc((size_t)nz * per * sizeof(float2));
      std::vector<ReconJob> jobs;
      for (int z = 0; z < nz; ++z) {
        ReconJob J;
        std::memset(&J, 0, sizeof J);
        J.k = sl + (size_t)z * nc * per;
        J.grappa_w = W[e] ? W[e] + (size_t)z * w_per_slice : nullptr;
        J.window = T.window;
        J.ex_tab = T.ex_tab;
        J.ey_tab = T.ey_tab;
        J.sens = T.sens;
        J.inv_ssum = T.inv_ssum;
        J.combined = comb + (size_t)z * per;
        J.nx = nx;
        J.ny = ny;
        J.nc = nc;
        jobs.push_back(J);
      }
      const ReconJob* d_jobs = (const ReconJob*)E.upload(jobs.data(), jobs.size() * sizeof(ReconJob), st);
      if (accel > 1) launch_grappa_apply(d_jobs, (int)jobs.size(), T.fills, T.n_fills, nx, nc, st);
      launch_recon_combine(d_jobs, (int)jobs.size(), nx, ny, false, st);
      volume_output_kernel<<<1024, 256, 0, st>>>(comb, g, 1, nv, per * nz, d_mag[e], d_ph[e]);
      MRSIM_CUDA(cudaGetLastError());
      MRSIM_CUDA(cudaStreamSynchronize(st));
    }
  }
  for (int e = 0; e < n_echoes; ++e) {
    copy_pageable_d2h(ctx, mag[e], d_mag[e], per * nz * nv * 4, st);
    copy_pageable_d2h(ctx, ph[e], d_ph[e], per * nz * nv * 4, st);
  }
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

}  // namespace mrsim
