// motion.h — rigid image motion on the device (see motion.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "driver.h"
#include "mrsim_internal.h"

namespace mrsim {

// Every volume g (pose g: rot_deg[3], trans_mm[3] at poses + 6 g) of every compartment of `in`
// resampled into `out` (different buffers); element (x, y, z) of volume g, compartment c at
// x sx + y sy + z sz + g sg + c sc.  Per-pose tables go to `arena`.
void resample_poses_device(const float* in, float* out, const int64_t* dims, int nv, int ncomp, long long sx,
                           long long sy, long long sz, long long sg, long long sc, const double* v2w,
                           const double* poses, cudaStream_t st, DevArena& arena);
// `apply_multiband_motion_slab` (motion.rs:686-772) from `in` into `out` (different buffers, the
// same strided layout); returns the number of dropped shots (written to `dropped` up to capacity).
int64_t multiband_device(const float* in, float* out, const int64_t* dims, int nv, int ncomp, long long sx, long long sy,
                         long long sz, long long sg, long long sc, const double* v2w, int64_t mb, bool interleaved,
                         const mrsim_dropout_law& law, const mrsim_motion_event* events, int64_t n_events,
                         const int64_t* slice_z, int64_t nz_full, mrsim_dropped_shot* dropped, int64_t capacity,
                         cudaStream_t st, DevArena& arena);
std::vector<std::vector<int64_t>> slice_schedule(int64_t nz, int64_t mb, bool interleaved);

}  // namespace mrsim
