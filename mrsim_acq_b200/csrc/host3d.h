// host3d.h — host tables of the 3D echo trains (see host3d.cpp).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "mrsim_acq.h"

namespace mrsim {

// `kz_order` (readout.rs:167-189): partitions in the order the train reads them.
std::vector<int> kz_order(int nz, int order);

// `GraseBlock` / `grase_block` (readout.rs:191-221).
struct GraseBlock {
  std::vector<double> t_ms;
  std::vector<int8_t> polarity;
  std::vector<int> segment;
  int epi = 0;
  double t_line_ms = 0;
};
GraseBlock grase_block(int ny, int ky_segments, double t_line_ms, bool reverse_phase);

// `GraseLine` / `Grase3dTable` / `grase_lines` (readout.rs:223-322), lines indexed p * ny + ky.
struct GraseLine {
  int shot, echo;
  double t_ms, trf_ms;
  int8_t polarity;
};
struct Grase3dTable {
  int ny = 0, nz = 0, e_c = 0, n_shots = 0;
  std::vector<GraseLine> lines;
  GraseBlock block;
  const GraseLine& line(int p, int ky) const { return lines[(size_t)p * ny + ky]; }
};
int centre_echo(const mrsim_echo_train& train, int nz);
Grase3dTable grase_lines(const mrsim_echo_train& train, const mrsim_grase_readout& ro, int ny, int nz);

// `Ge3dLine` / `Ge3dTable` / `ge3d_lines` (readout.rs:381-450), lines indexed p * ny + ky.
struct Ge3dLine {
  int shot, excitation;
  double t_ms;
  int8_t polarity;
};
struct Ge3dTable {
  int ny = 0, nz = 0, n_shots = 0, n_exc = 0, e_c = 0;
  std::vector<Ge3dLine> lines;
  GraseBlock block;
  const Ge3dLine& line(int p, int ky) const { return lines[(size_t)p * ny + ky]; }
};
Ge3dTable ge3d_lines(const mrsim_excitation_train& train, const mrsim_ge3d_readout& ro, int ny, int nz);

// `resolve_modes` (kspace3d.rs:388-432): per compartment, class (ln A per echo, uniform T2/T2')
// or voxel (ln A_e maps per echo over the simulation volume).
struct CompMode {
  bool voxel = false;
  std::vector<double> ln_a;        // class: etl values
  double t2_ms = 0, t2p_ms = 0;    // class
  std::vector<std::vector<double>> maps;  // voxel: [echo][vox]
};
std::vector<CompMode> resolve_modes(const mrsim_t2* t2, const mrsim_t2* t1, const mrsim_t2* t_inhom, int ncomp,
                                    const mrsim_acquisition& acq, const mrsim_echo_train& train, size_t nvox);

// `line_weight` (kspace3d.rs:83-88): exp(ln_a - t/T2 - |t|/T2'), infinite times meaning no decay.
double line_weight(double ln_a, double t_ms, double t2_ms, double t2p_ms);

// The timing checks of the trains (readout.rs:326-354, 460-500, 706-730): an empty string when
// the train fits, else the reference's message.  check_spiral_timing writes the train's end.
std::string check_grase_timing(const mrsim_echo_train& train, const Grase3dTable& t, double t_exc_ms, double tr_ms);
std::string check_ge3d_timing(const mrsim_excitation_train& train, const Ge3dTable& t, double t_exc_ms, double tr_ms);
std::string check_spiral_timing(const mrsim_echo_train& train, double readout_ms, double t_exc_ms, double tr_ms,
                                double* end_ms);

constexpr uint64_t kSeedSalt3d = 0x334452454144ull;  // "3DREAD" (kspace3d.rs:42)

}  // namespace mrsim
