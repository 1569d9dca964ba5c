// nifti.cpp — the series writer after the path: NIfTI-1 volumes with the acquisition affine and
// the BIDS `part-mag` / `part-phase` pair with JSON sidecars (reference io.rs:102-228), and the
// simulation grid's affine (`hires_grid`, io.rs:104-124).
//
// The reference writes through the third-party `nifti` crate (0.17; its source is not part of the
// reference tree).  This is an own writer of the published NIfTI-1 single-file format: a 348-byte
// little-endian header, four zero extension bytes, the float32 data at vox_offset 352, gzip when
// the name ends in .gz (zlib).  The header carries what the reference sets (`header_for_grid`,
// io.rs:84-100): pixdim 1..3 the affine's column norms, pixdim 4 the repetition time when given,
// xyzt_units mm (| s), qform and sform from the affine with code 1 (scanner anatomical); the
// qform quaternion follows the standard's matrix-to-quaternion conversion.
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "mrsim_internal.h"
#include "nifti.h"

namespace mrsim {

namespace {

#pragma pack(push, 1)
struct Nifti1Header {
  int32_t sizeof_hdr;
  char data_type[10];
  char db_name[18];
  int32_t extents;
  int16_t session_error;
  char regular;
  char dim_info;
  int16_t dim[8];
  float intent_p1, intent_p2, intent_p3;
  int16_t intent_code;
  int16_t datatype;
  int16_t bitpix;
  int16_t slice_start;
  float pixdim[8];
  float vox_offset;
  float scl_slope, scl_inter;
  int16_t slice_end;
  char slice_code;
  char xyzt_units;
  float cal_max, cal_min;
  float slice_duration;
  float toffset;
  int32_t glmax, glmin;
  char descrip[80];
  char aux_file[24];
  int16_t qform_code, sform_code;
  float quatern_b, quatern_c, quatern_d;
  float qoffset_x, qoffset_y, qoffset_z;
  float srow_x[4], srow_y[4], srow_z[4];
  char intent_name[16];
  char magic[4];
};
#pragma pack(pop)
static_assert(sizeof(Nifti1Header) == 348, "NIfTI-1 header is 348 bytes");

// The quaternion of the rotation part of an affine (columns divided by their norms; a left-handed
// frame flips the third column and sets qfac = -1), by the NIfTI-1 standard's construction.
void affine_to_quatern(const double* v2w, double& b, double& c, double& d, double& qfac) {
  double r[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i][j] = v2w[4 * i + j];
  for (int j = 0; j < 3; ++j) {
    double n = std::sqrt(r[0][j] * r[0][j] + r[1][j] * r[1][j] + r[2][j] * r[2][j]);
    if (n == 0.0) {
      for (int i = 0; i < 3; ++i) r[i][j] = i == j ? 1.0 : 0.0;
      continue;
    }
    for (int i = 0; i < 3; ++i) r[i][j] /= n;
  }
  const double det = r[0][0] * (r[1][1] * r[2][2] - r[1][2] * r[2][1]) -
                     r[0][1] * (r[1][0] * r[2][2] - r[1][2] * r[2][0]) +
                     r[0][2] * (r[1][0] * r[2][1] - r[1][1] * r[2][0]);
  qfac = 1.0;
  if (det < 0.0) {
    qfac = -1.0;
    for (int i = 0; i < 3; ++i) r[i][2] = -r[i][2];
  }
  double a = r[0][0] + r[1][1] + r[2][2] + 1.0;
  if (a > 0.5) {
    a = 0.5 * std::sqrt(a);
    b = 0.25 * (r[2][1] - r[1][2]) / a;
    c = 0.25 * (r[0][2] - r[2][0]) / a;
    d = 0.25 * (r[1][0] - r[0][1]) / a;
  } else {
    const double xd = 1.0 + r[0][0] - (r[1][1] + r[2][2]), yd = 1.0 + r[1][1] - (r[0][0] + r[2][2]),
                 zd = 1.0 + r[2][2] - (r[0][0] + r[1][1]);
    if (xd > 1.0) {
      b = 0.5 * std::sqrt(xd);
      c = 0.25 * (r[0][1] + r[1][0]) / b;
      d = 0.25 * (r[0][2] + r[2][0]) / b;
      a = 0.25 * (r[2][1] - r[1][2]) / b;
    } else if (yd > 1.0) {
      c = 0.5 * std::sqrt(yd);
      b = 0.25 * (r[0][1] + r[1][0]) / c;
      d = 0.25 * (r[1][2] + r[2][1]) / c;
      a = 0.25 * (r[0][2] - r[2][0]) / c;
    } else {
      d = 0.5 * std::sqrt(zd);
      b = 0.25 * (r[0][2] + r[2][0]) / d;
      c = 0.25 * (r[1][2] + r[2][1]) / d;
      a = 0.25 * (r[1][0] - r[0][1]) / d;
    }
    if (a < 0.0) {
      b = -b;
      c = -c;
      d = -d;
    }
  }
}

Nifti1Header header_for(const int64_t* dims, int64_t nt, const double* v2w, double tr_s, bool four) {
  Nifti1Header h;
  std::memset(&h, 0, sizeof h);
  h.sizeof_hdr = 348;
  h.regular = 'r';
  h.dim[0] = four ? 4 : 3;
  for (int i = 0; i < 3; ++i) h.dim[1 + i] = (int16_t)dims[i];
  h.dim[4] = (int16_t)(four ? nt : 1);
  for (int i = 5; i < 8; ++i) h.dim[i] = 1;
  h.datatype = 16;  // float32
  h.bitpix = 32;
  double b = 0, c = 0, d = 0, qfac = 1;
  affine_to_quatern(v2w, b, c, d, qfac);
  auto col_norm = [&](int j) {
    return (float)std::sqrt(std::pow(v2w[j], 2) + std::pow(v2w[4 + j], 2) + std::pow(v2w[8 + j], 2));
  };
  h.pixdim[0] = (float)qfac;
  h.pixdim[1] = col_norm(0);
  h.pixdim[2] = col_norm(1);
  h.pixdim[3] = col_norm(2);
  h.pixdim[4] = tr_s > 0.0 ? (float)tr_s : 0.0f;
  h.vox_offset = 352.0f;
  h.scl_slope = 1.0f;
  h.xyzt_units = tr_s > 0.0 ? (2 | 8) : 2;  // NIFTI_UNITS_MM (| NIFTI_UNITS_SEC)
  h.qform_code = 1;
  h.sform_code = 1;
  h.quatern_b = (float)b;
  h.quatern_c = (float)c;
  h.quatern_d = (float)d;
  h.qoffset_x = (float)v2w[3];
  h.qoffset_y = (float)v2w[7];
  h.qoffset_z = (float)v2w[11];
  for (int j = 0; j < 4; ++j) {
    h.srow_x[j] = (float)v2w[j];
    h.srow_y[j] = (float)v2w[4 + j];
    h.srow_z[j] = (float)v2w[8 + j];
  }
  std::memcpy(h.magic, "n+1\0", 4);
  return h;
}

bool ends_with(const std::string& s, const char* suf) {
  const size_t n = std::strlen(suf);
  return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

void write_bytes(const std::string& path, const std::vector<char>& bytes) {
  if (ends_with(path, ".gz")) {
    gzFile f = gzopen(path.c_str(), "wb");
    if (!f) fail("cannot open " + path + " for writing");
    size_t off = 0;
    while (off < bytes.size()) {
      const unsigned n = (unsigned)std::min<size_t>(bytes.size() - off, 1u << 30);
      if (gzwrite(f, bytes.data() + off, n) != (int)n) {
        gzclose(f);
        fail("write failed: " + path);
      }
      off += n;
    }
    if (gzclose(f) != Z_OK) fail("write failed: " + path);
    return;
  }
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) fail("cannot open " + path + " for writing");
  const bool ok = std::fwrite(bytes.data(), 1, bytes.size(), f) == bytes.size();
  if (std::fclose(f) != 0 || !ok) fail("write failed: " + path);
}

std::string fmt(const char* f, double v) {
  char buf[64];
  std::snprintf(buf, sizeof buf, f, v);
  return buf;
}

// Rust's `{}` for an f64: the shortest representation that round-trips, with no exponent for
// the magnitudes a sidecar holds ("0.75", "1", "0.5").
std::string rust_float(double v) {
  if (v == std::floor(v) && std::fabs(v) < 1e15) return fmt("%.0f", v);
  for (int p = 1; p <= 17; ++p) {
    std::string s = fmt(("%." + std::to_string(p) + "f").c_str(), v);
    if (std::strtod(s.c_str(), nullptr) == v) return s;
  }
  return fmt("%.17g", v);
}

}  // namespace

// `write_4d_timed` io.rs:135-146 (data (x + nx (y + ny z)) nt + t; tr_s <= 0: no time step) and,
// with four = false and nt = 1, `write_3d` io.rs:149-156.
void write_nifti(const std::string& path, const int64_t* dims, int64_t nt, const float* data, const double* v2w,
                 double tr_s, bool four) {
  if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0 || nt <= 0) fail("empty volume");
  for (int i = 0; i < 3; ++i)
    if (dims[i] > 32767) fail("NIfTI-1 dimensions are at most 32767");
  if (nt > 32767) fail("NIfTI-1 dimensions are at most 32767");
  const Nifti1Header h = header_for(dims, nt, v2w, tr_s, four);
  const size_t nvox = (size_t)(dims[0] * dims[1] * dims[2]);
  std::vector<char> bytes(352 + nvox * nt * 4, 0);
  std::memcpy(bytes.data(), &h, sizeof h);
  // NIfTI stores x fastest, then y, z, t: transpose the volume-innermost layout
  float* out = reinterpret_cast<float*>(bytes.data() + 352);
  for (int64_t t = 0; t < nt; ++t)
    for (size_t v = 0; v < nvox; ++v) out[(size_t)t * nvox + v] = data[v * nt + t];
  write_bytes(path, bytes);
}

// `hires_grid` io.rs:104-124: in-plane columns divided by o, origin shifted by half the
// difference of the coarse and fine voxels.
void hires_grid(const double* v2w, const int64_t* dims, int64_t o, double* out_v2w, int64_t* out_dims) {
  if (o <= 0) fail("oversampling factor must be positive");
  const double f = (double)o;
  double m[16];
  std::memcpy(m, v2w, sizeof m);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 2; ++c) m[4 * r + c] /= f;
  for (int r = 0; r < 3; ++r)
    m[4 * r + 3] = v2w[4 * r + 3] - 0.5 * v2w[4 * r] * (1.0 - 1.0 / f) - 0.5 * v2w[4 * r + 1] * (1.0 - 1.0 / f);
  std::memcpy(out_v2w, m, sizeof m);
  out_dims[0] = dims[0] * o;
  out_dims[1] = dims[1] * o;
  out_dims[2] = dims[2];
}

// `write_complex_4d` io.rs:186-228: the part-mag / part-phase NIfTIs and their JSON sidecars.
void write_complex_4d(const std::string& prefix, const std::string& suffix, const int64_t* dims, int64_t nv,
                      const float* mag, const float* phase, const double* v2w, const mrsim_sidecar_info& info) {
  const double tr = info.has_repetition_time ? info.repetition_time_s : 0.0;
  write_nifti(prefix + "_part-mag_" + suffix + ".nii.gz", dims, nv, mag, v2w, tr, true);
  write_nifti(prefix + "_part-phase_" + suffix + ".nii.gz", dims, nv, phase, v2w, tr, true);
  const std::string ped = info.phase_encoding_direction ? info.phase_encoding_direction : "";
  const int pe_axis = ped.empty() ? 1 : (ped[0] == 'i' ? 0 : (ped[0] == 'k' ? 2 : 1));
  const int64_t span = std::max<int64_t>(dims[pe_axis] - 1, 1);
  const double ees = info.total_readout_time / (double)span;
  std::string b0src;
  if (info.b0_field_source) b0src = std::string(",\n  \"B0FieldSource\": \"") + info.b0_field_source + "\"";
  const std::string common = std::string("  \"Manufacturer\": \"") + (info.manufacturer ? info.manufacturer : "") +
                             "\",\n  \"PhaseEncodingDirection\": \"" + ped + "\",\n  \"TotalReadoutTime\": " +
                             fmt("%.6f", info.total_readout_time) + ",\n  \"EffectiveEchoSpacing\": " +
                             fmt("%.8f", ees) + ",\n  \"EchoTime\": " + fmt("%.4f", info.echo_time) +
                             ",\n  \"PartialFourier\": " + rust_float(info.partial_fourier) +
                             ",\n  \"ParallelReductionFactorInPlane\": " + std::to_string(info.accel) +
                             ",\n  \"MultibandAccelerationFactor\": " + std::to_string(info.mb) + b0src;
  auto text = [](const std::string& s) { return std::vector<char>(s.begin(), s.end()); };
  write_bytes(prefix + "_part-mag_" + suffix + ".json",
              text("{\n" + common + ",\n  \"ImageComparison\": \"magnitude\"\n}\n"));
  write_bytes(prefix + "_part-phase_" + suffix + ".json",
              text("{\n" + common + ",\n  \"ImageComparison\": \"phase\",\n  \"Units\": \"rad\"\n}\n"));
}

}  // namespace mrsim
