// nifti.h — the series writer (see nifti.cpp).
#pragma once

#include <stdint.h>

#include <string>

#include "mrsim_internal.h"

namespace mrsim {

void write_nifti(const std::string& path, const int64_t* dims, int64_t nt, const float* data, const double* v2w,
                 double tr_s, bool four);
void hires_grid(const double* v2w, const int64_t* dims, int64_t o, double* out_v2w, int64_t* out_dims);
void write_complex_4d(const std::string& prefix, const std::string& suffix, const int64_t* dims, int64_t nv,
                      const float* mag, const float* phase, const double* v2w, const mrsim_sidecar_info& info);

}  // namespace mrsim
