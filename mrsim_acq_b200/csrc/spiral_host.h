// spiral_host.h — host plans of the stack-of-spirals path (see spiral_host.cpp).
#pragma once

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
TsegPlan tseg_plan(const std::vector<double>& tau, double t_ms, const double d[2], const double f[2]);

// `epg_cpmg` epg.rs:101-125: ln A_e, e = 1..n_echoes.
std::vector<double> epg_cpmg(int n_echoes, double esp_ms, double refocusing_deg, double t1_ms, double t2_ms);

}  // namespace mrsim
