// grase3d.h — the 3D GRASE echo-train acquisition on the device (see grase3d.cu).
#pragma once

#include "mrsim_internal.h"

namespace mrsim {

// `simulate_acquisition_3d` (kspace3d.rs:483-547, 549-589) with a GRASE readout: mag / phase at
// vox * nv + g (host buffers).
void grase_acquire(mrsim_context* ctx, const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                   const mrsim_echo_train& train, const mrsim_grase_readout& ro, uint64_t seed, float* mag,
                   float* ph);
// `kspace_3d_observed` (kspace3d.rs:439-456): volume g, [coil][p][ky][kx] complex f32 (host).
void grase_observed(mrsim_context* ctx, const mrsim_acquisition_3d_input& in, const mrsim_acquisition& acq,
                    const mrsim_echo_train& train, const mrsim_grase_readout& ro, int g, float* out);

// `simulate_acquisition_3d_ge` (kspace3d.rs:732-856): per echo e, mag[e] / ph[e] at vox * nv + g.
void ge_acquire(mrsim_context* ctx, const mrsim_acquisition_ge_input& in, const mrsim_acquisition& acq,
                const mrsim_excitation_train& train, const mrsim_ge3d_readout& ro, uint64_t seed, float* const* mag,
                float* const* ph);

}  // namespace mrsim
