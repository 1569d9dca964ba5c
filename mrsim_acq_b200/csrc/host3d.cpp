// host3d.cpp — host tables of the 3D echo trains: kz order, the GRASE block and line table
// (readout.rs:167-322), and the decay-mode resolution of the 3D path (kspace3d.rs:83-88,
// 388-432).  FP64 on the host; the device reads the tables these produce.
#include "host3d.h"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <algorithm>
#include <utility>

#include "mrsim_internal.h"
#include "spiral_host.h"

namespace mrsim {

std::vector<int> kz_order(int nz, int order) {
  std::vector<int> out;
  if (order == MRSIM_KZ_LINEAR) {
    for (int p = 0; p < nz; ++p) out.push_back(p);
    return out;
  }
  const int c = nz / 2;
  out.push_back(c);
  for (int d = 1; (int)out.size() < nz; ++d) {
    if (c + d < nz) out.push_back(c + d);
    if (d <= c && (int)out.size() < nz) out.push_back(c - d);
  }
  return out;
}

GraseBlock grase_block(int ny, int ky_segments, double t_line_ms, bool reverse_phase) {
  if (ky_segments <= 0 || ny % ky_segments != 0)
    fail(std::to_string(ny) + " phase-encode lines do not divide into " + std::to_string(ky_segments) +
         " ky segments");
  GraseBlock b;
  b.epi = ny / ky_segments;
  b.t_line_ms = t_line_ms;
  b.t_ms.resize(ny);
  b.polarity.resize(ny);
  b.segment.resize(ny);
  for (int ky = 0; ky < ny; ++ky) {
    const int sy = ky % ky_segments, j = ky / ky_segments;
    const int a = reverse_phase ? j : b.epi - 1 - j;  // acquisition index within the block
    b.t_ms[ky] = ((double)a - ((double)b.epi - 1.0) / 2.0) * t_line_ms;
    b.polarity[ky] = a % 2 == 1 ? -1 : 1;
    b.segment[ky] = sy;
  }
  return b;
}

int centre_echo(const mrsim_echo_train& train, int nz) {
  auto order = kz_order(nz, train.kz_order);
  int n = 0;
  while (order[n] != nz / 2) ++n;
  if (train.kz_segments <= 0 || nz % train.kz_segments != 0)
    fail(std::to_string(nz) + " partitions do not divide into " + std::to_string(train.kz_segments) + " kz segments");
  return n / (int)train.kz_segments + 1;
}

Grase3dTable grase_lines(const mrsim_echo_train& train, const mrsim_grase_readout& ro, int ny, int nz) {
  Grase3dTable T;
  T.block = grase_block(ny, (int)ro.ky_segments, ro.t_line_ms, ro.reverse_phase != 0);
  const int kzs = (int)train.kz_segments;
  if (kzs <= 0 || nz % kzs != 0)
    fail(std::to_string(nz) + " partitions do not divide into " + std::to_string(train.kz_segments) + " kz segments");
  if (train.etl != nz / kzs)
    fail("echo train length " + std::to_string(train.etl) + " is not " + std::to_string(nz) + " partitions / " +
         std::to_string(kzs) + " kz segments");
  auto order = kz_order(nz, train.kz_order);
  T.ny = ny;
  T.nz = nz;
  T.lines.assign((size_t)ny * nz, GraseLine{0, 0, 0.0, 0.0, 0});
  std::vector<char> seen((size_t)ny * nz, 0);
  for (int sy = 0; sy < (int)ro.ky_segments; ++sy)
    for (int sz = 0; sz < kzs; ++sz) {
      const int shot = sy * kzs + sz;
      for (int e = 1; e <= (int)train.etl; ++e) {
        const int p = order[sz + kzs * (e - 1)];
        for (int j = 0; j < T.block.epi; ++j) {
          const int ky = sy + (int)ro.ky_segments * j;
          const size_t i = (size_t)p * ny + ky;
          if (seen[i]) fail("line (" + std::to_string(p) + ", " + std::to_string(ky) + ") read twice");
          seen[i] = 1;
          const double t = T.block.t_ms[ky];
          T.lines[i] = GraseLine{shot, e, t, (double)e * train.esp_ms + t, T.block.polarity[ky]};
        }
      }
    }
  for (char s : seen)
    if (!s) fail("a line was never read");
  T.e_c = centre_echo(train, nz);
  T.n_shots = (int)ro.ky_segments * kzs;
  return T;
}

Ge3dTable ge3d_lines(const mrsim_excitation_train& train, const mrsim_ge3d_readout& ro, int ny, int nz) {
  if (nz < 2) fail("a 3D gradient-echo train on " + std::to_string(nz) + " partition is a 2D readout");
  Ge3dTable T;
  T.block = grase_block(ny, (int)ro.ky_segments, ro.t_line_ms, ro.reverse_phase != 0);
  const int kzs = (int)train.kz_segments;
  if (kzs <= 0 || nz % kzs != 0)
    fail(std::to_string(nz) + " partitions do not divide into " + std::to_string(train.kz_segments) + " kz segments");
  T.n_exc = nz / kzs;
  auto order = kz_order(nz, train.kz_order);
  T.ny = ny;
  T.nz = nz;
  T.lines.assign((size_t)ny * nz, Ge3dLine{0, 0, 0.0, 0});
  std::vector<char> seen((size_t)ny * nz, 0);
  for (int sy = 0; sy < (int)ro.ky_segments; ++sy)
    for (int sz = 0; sz < kzs; ++sz) {
      const int shot = sy * kzs + sz;
      for (int j = 0; j < T.n_exc; ++j) {
        const int p = order[sz + kzs * j];
        for (int i = 0; i < T.block.epi; ++i) {
          const int ky = sy + (int)ro.ky_segments * i;
          const size_t at = (size_t)p * ny + ky;
          if (seen[at]) fail("line (" + std::to_string(p) + ", " + std::to_string(ky) + ") read twice");
          seen[at] = 1;
          T.lines[at] = Ge3dLine{shot, j, T.block.t_ms[ky], T.block.polarity[ky]};
        }
      }
    }
  for (char s : seen)
    if (!s) fail("a line was never read");
  int n_c = 0;
  while (order[n_c] != nz / 2) ++n_c;
  T.n_shots = (int)ro.ky_segments * kzs;
  T.e_c = n_c / kzs;
  return T;
}

namespace {
std::string fmt(const char* f, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, f);
  std::vsnprintf(buf, sizeof buf, f, ap);
  va_end(ap);
  return buf;
}
double block_extent(const GraseBlock& b) {
  double m = 0.0;
  for (double t : b.t_ms) m = std::max(m, std::fabs(t));
  return m;
}
}  // namespace

std::string check_grase_timing(const mrsim_echo_train& train, const Grase3dTable& t, double t_exc_ms, double tr_ms) {
  const double t_line = t.block.t_line_ms, extent = block_extent(t.block), half = train.esp_ms / 2.0;
  const double need = extent + t_line / 2.0 + train.refocusing_time_ms / 2.0;
  if (need > half + 1e-9)
    return fmt("the %d-line EPI block reaches %.4f ms from its echo (lines of %.4f ms), and with half the %.3f ms "
               "refocusing time needs %.4f ms, more than half the echo spacing (%.4f ms of %.4f ms). Fewer lines per "
               "block (more ky segments, a smaller matrix), shorter lines, or a longer echo spacing would fit: the echo "
               "spacing must be at least %.4f ms",
               t.block.epi, extent + t_line / 2.0, t_line, train.refocusing_time_ms, need, half, train.esp_ms,
               2.0 * need);
  if (half - train.refocusing_time_ms / 2.0 <= 0.0)
    return fmt("the first refocusing pulse (%.3f ms long, centred %.4f ms after the excitation) overlaps the excitation",
               train.refocusing_time_ms, half);
  const double last = t_exc_ms + (double)train.etl * train.esp_ms + extent + t_line / 2.0;
  if (last > tr_ms + 1e-9)
    return fmt("the echo train ends at %.4f ms (excitation at %.4f ms, %lld echoes of %.4f ms), after the %.4f ms "
               "repetition",
               last, t_exc_ms, (long long)train.etl, train.esp_ms, tr_ms);
  return "";
}

std::string check_ge3d_timing(const mrsim_excitation_train& train, const Ge3dTable& t, double t_exc_ms, double tr_ms) {
  const double* tes = train.echo_times_ms;
  const int n = (int)train.n_echoes;
  if (n < 1 || !tes) return "a 3D gradient-echo train needs at least one echo time";
  const double half = block_extent(t.block) + t.block.t_line_ms / 2.0, pulse = train.excitation_time_ms / 2.0;
  auto lo = [&](int e) { return tes[e] - half; };
  auto hi = [&](int e) { return tes[e] + half; };
  if (lo(0) < pulse - 1e-9)
    return fmt("echo 1 at %.4f ms: its %d-line block starts %.4f ms after the excitation, inside the excitation pulse "
               "(half of %.3f ms); a later echo time or a shorter block would fit",
               tes[0], t.block.epi, lo(0), train.excitation_time_ms);
  for (int e = 1; e < n; ++e)
    if (lo(e) < hi(e - 1) - 1e-9)
      return fmt("echo %d at %.4f ms and echo %d at %.4f ms: their blocks of %.4f ms each side overlap", e, tes[e - 1],
                 e + 1, tes[e], half);
  const double end = hi(n - 1);
  if (t.n_exc > 1 && end > train.exc_spacing_ms - pulse + 1e-9)
    return fmt("the last echo's block ends %.4f ms after its excitation, after the next excitation pulse starts at "
               "%.4f ms (excitation spacing %.4f ms, pulse %.3f ms): the spacing must be at least %.4f ms",
               end, train.exc_spacing_ms - pulse, train.exc_spacing_ms, train.excitation_time_ms, end + pulse);
  const double last = t_exc_ms + ((double)t.n_exc - 1.0) * train.exc_spacing_ms + end;
  if (last > tr_ms + 1e-9)
    return fmt("the train ends at %.4f ms (%d excitations %.4f ms apart from %.4f ms), after the %.4f ms repetition",
               last, t.n_exc, train.exc_spacing_ms, t_exc_ms, tr_ms);
  return "";
}

std::string check_spiral_timing(const mrsim_echo_train& train, double readout_ms, double t_exc_ms, double tr_ms,
                                double* end_ms) {
  const double t = readout_ms, half = train.esp_ms / 2.0, need = t + train.refocusing_time_ms / 2.0;
  if (need > half + 1e-9)
    return fmt("the %g ms spiral with half the %.3f ms refocusing time needs %.4f ms after its echo, more than half the "
               "echo spacing (%.4f ms of %.4f ms): it would run into the next refocusing pulse. A shorter spiral (more "
               "interleaves) or a longer echo spacing would fit: the echo spacing must be at least %.4f ms",
               t, train.refocusing_time_ms, need, half, train.esp_ms, 2.0 * need);
  if (half - train.refocusing_time_ms / 2.0 <= 0.0)
    return fmt("the first refocusing pulse (%.3f ms long, centred %.4f ms after the excitation) overlaps the excitation",
               train.refocusing_time_ms, half);
  const double last = t_exc_ms + (double)train.etl * train.esp_ms + t;
  if (last > tr_ms + 1e-9)
    return fmt("the echo train ends at %.4f ms (excitation at %.4f ms, %lld echoes of %.4f ms, a %g ms spiral), after "
               "the %.4f ms repetition",
               last, t_exc_ms, (long long)train.etl, train.esp_ms, t, tr_ms);
  if (end_ms) *end_ms = last;
  return "";
}

double line_weight(double ln_a, double t_ms, double t2_ms, double t2p_ms) {
  const double d2 = std::isinf(t2_ms) ? 0.0 : t_ms / t2_ms;
  const double dp = std::isinf(t2p_ms) ? 0.0 : std::fabs(t_ms) / t2p_ms;
  return std::exp(ln_a - d2 - dp);
}

std::vector<CompMode> resolve_modes(const mrsim_t2* t2, const mrsim_t2* t1, const mrsim_t2* t_inhom, int ncomp,
                                    const mrsim_acquisition& acq, const mrsim_echo_train& train, size_t nvox) {
  const bool needs_t1 = acq.do_relaxation && train.refocusing_deg != 180.0;
  if (needs_t1 && !t1) fail("refocusing below 180 degrees needs T1 (stimulated echoes)");
  const int etl = (int)train.etl;
  std::map<std::pair<uint32_t, uint32_t>, std::vector<double>> cache;
  auto bits = [](float v) {
    uint32_t b;
    std::memcpy(&b, &v, 4);
    return b;
  };
  auto epg = [&](float t1v, float t2v) -> const std::vector<double>& {
    auto key = std::make_pair(bits(t1v), bits(t2v));
    auto it = cache.find(key);
    if (it == cache.end())
      it = cache.emplace(key, epg_cpmg(etl, train.esp_ms, train.refocusing_deg, (double)t1v, (double)t2v)).first;
    return it->second;
  };
  std::vector<CompMode> modes(ncomp);
  for (int c = 0; c < ncomp; ++c) {
    const mrsim_t2 t1c = t1 ? t1[c] : mrsim_t2{nullptr, INFINITY, 0};
    const mrsim_t2 tic = t_inhom ? t_inhom[c] : mrsim_t2{nullptr, (float)acq.t_inhom, 0};
    CompMode& m = modes[c];
    if (!t2[c].is_map && !t1c.is_map && !tic.is_map) {
      m.ln_a = epg(t1c.value, t2[c].value);
      m.t2_ms = t2[c].value;
      m.t2p_ms = tic.value;
    } else if (!acq.do_relaxation) {
      m.ln_a.assign(etl, 0.0);
      m.t2_ms = INFINITY;
      m.t2p_ms = INFINITY;
    } else {
      m.voxel = true;
      m.maps.assign(etl, std::vector<double>(nvox, 0.0));
      for (size_t i = 0; i < nvox; ++i) {
        const float a = t1c.is_map ? t1c.map[i] : t1c.value;
        const float b = t2[c].is_map ? t2[c].map[i] : t2[c].value;
        const std::vector<double>& la = epg(a, b);
        for (int e = 0; e < etl; ++e) m.maps[e][i] = la[e];
      }
    }
  }
  return modes;
}

}  // namespace mrsim
