// spiral_host.h — host plans of the stack-of-spirals path (see spiral_host.cpp).
#pragma once

#include <cuda_runtime.h>

#include <utility>
#include <vector>

namespace mrsim {

struct SpiralTraj {
  int interleaves = 0;
  double k_max = 0, n_turns = 0, readout_ms = 0, tau_c_ms = 0;
  std::vector<double> tau_ms;  // per sample, (j + 1/2) dwell
  std::vector<double> k;       // [interleaf][sample][2] cycles/FOV
};

// `spiral_tau_c` readout.rs:564-596 and `spiral_trajectory` readout.rs:597-620.
double spiral_tau_c(int nx, int interleaves, double readout_ms, double dwell_ms, double radial_oversampling);
SpiralTraj spiral_trajectory(int nx, int ny, int interleaves, double readout_ms, double dwell_ms,
                             double radial_oversampling);

// `tseg::plan` tseg.rs:230-289: certified segmentation of exp(z tau) over the rectangle
// d in [d0, d1] (1/ms), f in [f0, f1] (Hz).
struct TsegPlan {
  int l = 0, m = 0;
  std::vector<double> tau_l;  // segment times (ms)
  std::vector<double> b;      // [sample][segment] (re, im)
  double b_sum = 0, grid_err = 0, bound = 0;
};

// The per-sample half of every fit of a plan on the device (tseg_fit.cu, FP64): right-hand
// sides, factored solve and residual for all sample times at once; the factorisation and the
// search over L and m stay on the host.  One object serves the plans of one call on one stream.
class TsegDevice {
 public:
  explicit TsegDevice(cudaStream_t st);
  ~TsegDevice();
  TsegDevice(const TsegDevice&) = delete;
  TsegDevice& operator=(const TsegDevice&) = delete;
  void set_times(const std::vector<double>& tau);
  // one fit over the rate grid: the maxima b_sum and err; b stays on the device
  void fit(const std::vector<std::pair<double, double>>& rates, const std::vector<std::vector<double>>& cols,
           const std::vector<std::vector<double>>& left, const std::vector<std::vector<double>>& right,
           const std::vector<double>& sig, int l, double* b_sum, double* err);
  // the last fit's b, [sample][segment] (re, im)
  void fetch_b(std::vector<double>& b) const;

 private:
  struct Bufs;
  cudaStream_t st_;
  Bufs* d_;
  int n_tau_ = 0, l_ = 0;
};

// With `dev` the fits' per-sample work runs on the device (the product's path); without it on
// the host (planning without a GPU, and the host reference of the device fit).
TsegPlan tseg_plan(const std::vector<double>& tau, double t_ms, const double d[2], const double f[2],
                   TsegDevice* dev = nullptr);

// `epg_cpmg` epg.rs:101-125: ln A_e, e = 1..n_echoes.
std::vector<double> epg_cpmg(int n_echoes, double esp_ms, double refocusing_deg, double t1_ms, double t2_ms);

}  // namespace mrsim
