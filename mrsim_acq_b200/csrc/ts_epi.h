// ts_epi.h — the time-segmented tensor-core EPI operator pair (see ts_epi.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "driver.h"
#include "mrsim_internal.h"

namespace mrsim {

constexpr int kTsMaxGroups = 16;  // line groups (echo x side of the echo, split to <= 256 outputs)
constexpr int kTsMaxL = 32;       // segments per group (padded to a multiple of 4)
constexpr int kTsMaxLines = 32;   // lines per group

// One group of lines sharing a certified segmentation (device copy; read by every kernel).
struct TsGroupDev {
  int n_j;    // lines
  int Lp, L;  // segments, padded to a multiple of 4, and the plan's count
  int np_f;   // forward output columns (j, v, re/im), a multiple of 16 (<= 256)
  int kb_f;   // forward 64-wide K blocks: (sny / 8) (Lp / 4)
  int kp_a;   // adjoint K (j, v, re/im) padded to a multiple of 64
  int ka0;    // first K column of the group in the adjoint operand rows
  int np_a;   // adjoint output columns per y chunk: yc Lp 2
  int yc;
  int pad[3];
  int lines[kTsMaxLines];          // line-table indices
  float t_hi[kTsMaxL], t_lo[kTsMaxL];  // node phase times t_first + tau_l / 1000 (s), hi + lo
  float alpha[kTsMaxL][kMaxComp];      // e^{A_c - (d_c - d_lo) tau_l}
  float alpha_adj[kTsMaxL][kMaxComp];  // alpha over the adjoint table's scale
  float out_scale_f;                   // 1 / the forward table's scale
  float pad2[3];
};

struct TsAmax {
  float v[kMaxComp];
};

struct TsFwdParams {
  CUtensorMap bmap[kTsMaxGroups];
  const UnitDesc* units;
  const TsGroupDev* groups;
  const float* unit_scale;   // per plan unit (f16 input scale) or NULL
  float2* cls_out;           // class-row scratch when the x-stage runs per coil, else NULL (u.g)
  long long cls_unit_stride;
  int* err;
  int n_items, n_groups, na, snx_tiles, np_max, u0, b_stages;
};

struct TsAdjParams {
  CUtensorMap amap_hi, amap_lo;
  CUtensorMap bmap[kTsMaxGroups];
  const UnitDesc* units;
  const TsGroupDev* groups;
  const float* unit_scale;
  int* err;
  int n_items, n_groups, snx_tiles, snx_pad, np_max, nyc, yc, u0;
};

struct TsConvParams {
  const UnitDesc* units;
  const TsGroupDev* groups;
  float* unit_scale;
  uint16_t* gs_hi;
  uint16_t* gs_lo;
  int n_groups, na, kp_total, snx_pad, class_rows, u0;
};

// Host plan: groups, certified segmentations, split tables and tensor maps, scratch.
struct TsPlan {
  int dt = 0;  // 0 split f16, 1 split bf16
  int n_groups = 0, na = 0, np_max_f = 0, np_max_a = 0, yc = 0, nyc = 0, kp_total = 0, snx_pad = 0, snx_tiles = 0;
  int n_sms = 148;
  double fmin = 0, fmax = 0;              // the fieldmap range certified
  double flops_fwd = 0, flops_adj = 0;    // tensor-pipe FLOP per full pass (3 split products)
  std::vector<int> L;
  std::vector<double> bound;
  std::vector<TsGroupDev> groups_h;
  TsGroupDev* d_groups = nullptr;
  std::vector<CUtensorMap> fmaps, amaps;
  CUtensorMap gs_hi_map, gs_lo_map;
  uint16_t* d_gs_hi = nullptr;
  uint16_t* d_gs_lo = nullptr;
  float* d_scale_f = nullptr;
  float* d_scale_a = nullptr;
  float2* d_cls = nullptr;
  long long cls_stride = 0;
  int* d_err = nullptr;
  TsAmax amax;
  bool fwd_cls = false, adj_cls = false;
  DevArena arena;
  ~TsPlan();
};

TsPlan* ts_plan_build(const EpiOperator& op, int precision);
void ts_forward_ystage(const TsPlan& T, const EpiPlan& ep, cudaStream_t st, int u0 = 0, int u1 = -1);
// the x-adjoint's rows must be in the unit scratch (epi_plan_adjoint_xstage) before this runs
void ts_adjoint_ystage(const TsPlan& T, const EpiPlan& ep, cudaStream_t st, int u0 = 0, int u1 = -1);
// the kernels' error code (0: none; otherwise a wait that gave up), synchronising the stream
int ts_error(const TsPlan& T, cudaStream_t st);

}  // namespace mrsim
