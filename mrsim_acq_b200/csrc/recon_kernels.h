// recon_kernels.h — device reconstruction of a slice's coils (see recon_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mrsim {

// One GRAPPA calibration system: one slice's reference scan, one offset d in 1..accel-1.
struct GrappaSystem {
  const float2* k;         // reference-scan k-space [coil][ny][nx]
  const uint8_t* lines;    // ny acquired-line flags of the reference scan (device)
  int nx, ny, nc, accel, d, acs_lo, acs_hi, pad;
  double2* work;           // nf*(nf+nc) FP64 complex: [A^H A | A^H b]
  double* fscratch;        // 2*nf + nc*2*nf FP64
  float2* weights;         // out: [nc][nf] complex f32 for this d
};

// One (unit, echo) to reconstruct.
struct ReconJob {
  float2* k;                // [coil][ny][nx], GRAPPA fills it in place
  const float2* grappa_w;   // [d-1][co][6 nc] for this slice and echo time, or NULL
  const float* window;      // [ny][nx] or NULL
  const float2* ex_tab;     // e^{-i 2 pi m / nx}, m = 0..nx-1
  const float2* ey_tab;     // e^{-i 2 pi m / ny}
  const float* sens;        // [coil][ny][nx] coil sensitivities on the acquired grid
  const float* inv_ssum;    // [ny][nx] 1 / max(sum_q s_q^2, 1e-12)
  float2* coil_images;      // capture [coil][ny][nx] or NULL
  float2* reconstructed;    // capture [coil][ny][nx] or NULL
  float2* combined;         // out [ny][nx]
  int nx, ny, nc, pad;
};

void launch_grappa_fit(const GrappaSystem* d_sys, int n_sys, int max_nc, double lambda, cudaStream_t st);
// fills: (ky, d, s0, s1) of every line GRAPPA synthesises (the same for every job of the launch)
void launch_grappa_apply(const ReconJob* d_jobs, int n_jobs, const int4* d_fills, int n_fills, int nx, int nc,
                         cudaStream_t st);
void launch_recon_combine(const ReconJob* d_jobs, int n_jobs, int nx, int ny, bool capture_reconstructed,
                          cudaStream_t st);

}  // namespace mrsim
