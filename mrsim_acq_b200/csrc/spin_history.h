// spin_history.h — the spin history of slice-selective excitations under head motion on the device
// (see spin_history.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "mrsim_internal.h"

namespace mrsim {

// A grow-only device buffer.
struct GrowBuf {
  void* p = nullptr;
  size_t n = 0;
  void* get(size_t bytes);
  ~GrowBuf();
};

struct SpinPulseDev {
  double t, eps;
  int kind, pad;
};

// One shot of a batch as the kernels read it.
struct SpinShotDev {
  double m[12];     // source voxel -> slab voxel coordinates (rows 0..2 of the 4x4)
  double minv[12];  // slab voxel -> source voxel coordinates
  double t;         // the excitation's time (s)
  double ref_a, ref_b;
  int ref_kind;     // MRSIM_MZREF_*
  int n_slices;
  long long values; // first value of a VALUES reference in the batch's value buffer, or -1
  long long weight; // first weight of the shot's weight override in the batch's weight buffer, or -1
  long long rec;    // first record of the shot (reading shots)
  long long out;    // first float of the shot's terms (reading shots)
  int plane_tab;    // the shot's plane table: per source plane its first record offset, or -1
  int in_shot;      // the shot's slab table: per slab its index in the shot, or -1
  int slices;       // the shot's slice list
  int pad;
};

// The device state of one series' history.
struct SpinHistoryDev {
  mrsim_context* ctx = nullptr;
  int64_t nx = 0, ny = 0, nz = 0, nv = 0, nt = 0, snx = 0, sny = 0, snz = 0;
  int ncls = 0, maxc = 0;
  double v2w[16], w2v_slab[16];
  double len = 0, vol = 0;
  std::vector<int> plane_first;      // nz + 1: tracked index of each plane's first voxel
  std::vector<SpinPulseDev> pulses;  // sorted by time
  // resident state, tracked voxels in source order (SoA; pieces slot-major: slot s of voxel i at
  // s * nt + i)
  uint32_t* d_flat = nullptr;
  float* d_t1 = nullptr;
  float* d_w = nullptr;
  uint8_t* d_cls = nullptr;
  uint8_t* d_n = nullptr;
  float* d_start = nullptr;
  float* d_mz = nullptr;
  double* d_t = nullptr;
  int* d_idx = nullptr;          // per source voxel: its tracked index, or -1
  int* d_plane_first = nullptr;  // nz + 1
  SpinPulseDev* d_pulses = nullptr;
  unsigned long long* d_merges = nullptr;
  int* d_err = nullptr;
  std::vector<void*> allocs;
  // per-batch buffers
  GrowBuf blob_b, rec_cell_b, rec_cnt_b, ent_num_b, ent_den_b, ent_kk_b, out_b;
  // two pinned host blobs that stage a batch's tables, used in turn; each is rewritten only once
  // the copy out of it (its event) has completed, so the host prepares batch n+1 while the device
  // still runs batch n
  void* pin[2] = {nullptr, nullptr};
  size_t pin_n[2] = {0, 0};
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
  int pin_i = 0;
  ~SpinHistoryDev();
};

SpinHistoryDev* spin_history_create(mrsim_context* ctx, const int64_t* src_dims, const double* src_v2w,
                                    const float* t1, const float* weight, const uint8_t* cls, int64_t n_classes,
                                    const int64_t* slab_dims, const double* slab_v2w, const mrsim_pulse* pulses,
                                    int64_t n_pulses);
// floats of the terms of `shots`
int64_t spin_history_terms_size(const SpinHistoryDev& h, const mrsim_spin_shot* shots, int64_t n);
// the shots in order on the context's stream, the packed terms into device memory `terms`
void spin_history_run(SpinHistoryDev& h, const mrsim_spin_shot* shots, int64_t n, float* terms);
// merges so far (synchronises; throws on a kernel's error status)
uint64_t spin_history_merges(SpinHistoryDev& h);

}  // namespace mrsim
