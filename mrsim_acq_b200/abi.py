"""ctypes mirror of include/mrsim_acq.h and the loader of libmrsim_acq_cuda.so.

The structures here are the C ABI's, field for field.  The library is loaded from this package
directory (it is built in-tree by `build.py`); there is no CPU fallback: loading fails loudly if
the shared object is missing, and every compute entry point needs a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import pathlib

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libmrsim_acq_cuda.so"

c_f32p = C.POINTER(C.c_float)
c_f64p = C.POINTER(C.c_double)


class Acquisition_(C.Structure):
    """`mrsim_acquisition` — `Acquisition` (reference kspace.rs:166-197)."""

    _fields_ = [
        ("t_line", C.c_double), ("t_echo", C.c_double), ("t_inhom", C.c_double), ("signal_scale", C.c_double),
        ("reverse_phase", C.c_int32), ("do_distortions", C.c_int32), ("do_relaxation", C.c_int32),
        ("pf_mode", C.c_int32),
        ("noise_variance", C.c_double), ("partial_fourier", C.c_double), ("ghost_offset", C.c_double),
        ("eddy_strength", C.c_double), ("eddy_quad", C.c_double), ("eddy_phase", C.c_double),
        ("eddy_tau", C.c_double), ("n_spikes", C.c_int64), ("spike_amplitude", C.c_double),
        ("window_kind", C.c_int32), ("echo", C.c_int32), ("window_a", C.c_double), ("window_b", C.c_double),
        ("n_coils", C.c_int64), ("accel", C.c_int64), ("acs_lines", C.c_int64), ("seed", C.c_uint64),
    ]


class T2_(C.Structure):
    """`mrsim_t2` — `T2Slice` / `T2Volume` (kspace.rs:380-393)."""

    _fields_ = [("map", c_f32p), ("value", C.c_float), ("is_map", C.c_int32)]


class SliceInput_(C.Structure):
    """`mrsim_slice_input` — `SliceInput` (kspace.rs:458-496)."""

    _fields_ = [
        ("compartments", C.POINTER(c_f32p)), ("ncomp", C.c_int64), ("t2", C.POINTER(T2_)),
        ("t_inhom", C.POINTER(T2_)), ("fmap", c_f32p), ("phase0", c_f64p), ("sim", C.c_int64 * 2),
        ("acq_matrix", C.c_int64 * 2), ("z", C.c_int64), ("nz", C.c_int64), ("has_eddy_drive", C.c_int32),
        ("has_prep_drive", C.c_int32), ("eddy_drive", C.c_double * 3), ("prep_magnitude", C.c_double),
        ("prep_direction", C.c_double * 3), ("slice_seed", C.c_uint64),
    ]


class PhaseModel_(C.Structure):
    """`mrsim_phase_model` — `PhaseModel` (phase.rs:130-205)."""

    _fields_ = [
        ("global_", C.c_double), ("background", C.c_double * 10), ("has_prep", C.c_int32),
        ("reserved", C.c_int32), ("c_q", C.c_double), ("sigma_dx", C.c_double), ("sigma_rot", C.c_double),
    ]


class DropoutLaw_(C.Structure):
    _fields_ = [("kind", C.c_int32), ("drive", c_f64p), ("n_drive", C.c_int64), ("floor", C.c_double),
                ("max", C.c_double)]


class MotionEvent_(C.Structure):
    _fields_ = [("volume", C.c_int64), ("shot", C.c_int64), ("severity", C.c_float), ("jump_mm", C.c_double * 3),
                ("jump_deg", C.c_double * 3)]


class DroppedShot_(C.Structure):
    _fields_ = [("volume", C.c_int64), ("shot", C.c_int64), ("attenuation", C.c_float), ("n_slices", C.c_int64),
                ("slices", C.c_int64 * 64)]


class SidecarInfo_(C.Structure):
    _fields_ = [("manufacturer", C.c_char_p), ("phase_encoding_direction", C.c_char_p),
                ("total_readout_time", C.c_double), ("echo_time", C.c_double), ("partial_fourier", C.c_double),
                ("accel", C.c_int64), ("mb", C.c_int64), ("has_repetition_time", C.c_int32),
                ("repetition_time_s", C.c_double), ("b0_field_source", C.c_char_p)]


class AcquisitionInput_(C.Structure):
    """`mrsim_acquisition_input` — `AcquisitionInput` (kspace.rs:1720-1740)."""

    _fields_ = [
        ("sim_dims", C.c_int64 * 3), ("acq_dims", C.c_int64 * 3), ("n_volumes", C.c_int64), ("ncomp", C.c_int64),
        ("images", C.POINTER(c_f32p)), ("t2", C.POINTER(T2_)), ("fmap", c_f32p), ("t_inhom", C.POINTER(T2_)),
        ("eddy_drive_set", C.POINTER(C.c_int32)), ("eddy_drive", c_f64p),
        ("prep_drive_set", C.POINTER(C.c_int32)), ("prep_drive", c_f64p),
        ("phase", C.POINTER(PhaseModel_)), ("seed", C.c_uint64), ("noise_sigma", c_f32p),
    ]


PROGRESS_FN = C.CFUNCTYPE(None, C.c_int64, C.c_int64, C.c_void_p)


class AcquisitionOptions_(C.Structure):
    """`mrsim_acquisition_options` — `AcquisitionOptions` (kspace.rs:1744-1762)."""

    _fields_ = [
        ("slice_z", C.POINTER(C.c_int64)), ("nz_full", C.c_int64), ("kspace_slices", C.POINTER(C.c_int64)),
        ("n_kspace_slices", C.c_int64), ("capture_acquired", C.c_int32), ("capture_reconstructed", C.c_int32),
        ("capture_coil_images", C.c_int32), ("has_grappa_calibration", C.c_int32),
        ("t_echo_per_volume", c_f64p), ("progress", PROGRESS_FN), ("progress_user", C.c_void_p),
        ("grappa_calibration_images", C.POINTER(c_f32p)), ("grappa_calibration_seed", C.c_uint64),
    ]


class AcquisitionOutput_(C.Structure):
    """`mrsim_acquisition_output` — `AcquisitionOutput` + `KspaceCapture` (kspace.rs:1767-1797)."""

    _fields_ = [
        ("re", c_f32p), ("im", c_f32p), ("mask", C.POINTER(C.c_uint8)), ("sensitivities", c_f32p),
        ("acquired", c_f32p), ("reconstructed", c_f32p), ("coil_images", c_f32p), ("combined", c_f32p),
    ]


class SpiralInfo_(C.Structure):
    """`mrsim_spiral_info` — the scalars of `SpiralTrajectory` (readout.rs:463-560)."""

    _fields_ = [("samples", C.c_int64), ("interleaves", C.c_int64), ("k_max", C.c_double),
                ("n_turns", C.c_double), ("tau_c_ms", C.c_double)]


class TsegInfo_(C.Structure):
    """`mrsim_tseg_info` — the scalars of `TsegPlan` (tseg.rs:60-75)."""

    _fields_ = [("l", C.c_int64), ("m", C.c_int64), ("b_sum", C.c_double), ("grid_err", C.c_double),
                ("bound", C.c_double)]


class EchoTrain_(C.Structure):
    """`mrsim_echo_train` — `EchoTrain` (readout.rs:82-95)."""

    _fields_ = [("etl", C.c_int64), ("esp_ms", C.c_double), ("refocusing_deg", C.c_double), ("kz_order", C.c_int32),
                ("reserved", C.c_int32), ("kz_segments", C.c_int64), ("refocusing_time_ms", C.c_double)]


class GraseReadout_(C.Structure):
    """`mrsim_grase_readout` — `Readout3d::Grase` (readout.rs:103-106)."""

    _fields_ = [("ky_segments", C.c_int64), ("t_line_ms", C.c_double), ("reverse_phase", C.c_int32),
                ("reserved", C.c_int32)]


class ShotSet_(C.Structure):
    """`mrsim_shot_set` — `ShotSet` (kspace3d.rs:59-65)."""

    _fields_ = [("shots", C.POINTER(C.c_int64)), ("n_shots", C.c_int64), ("images", C.POINTER(c_f32p))]


class Acquisition3dInput_(C.Structure):
    """`mrsim_acquisition_3d_input` — the inputs of `simulate_acquisition_3d` (kspace3d.rs:549)."""

    _fields_ = [
        ("sim_dims", C.c_int64 * 3), ("acq_dims", C.c_int64 * 3), ("n_volumes", C.c_int64), ("ncomp", C.c_int64),
        ("images", C.POINTER(c_f32p)), ("t2", C.POINTER(T2_)), ("t1", C.POINTER(T2_)), ("fmap", c_f32p),
        ("t_inhom", C.POINTER(T2_)), ("phase", C.POINTER(PhaseModel_)), ("line_weights", c_f64p),
        ("has_grappa_calibration", C.c_int32), ("reserved", C.c_int32),
        ("grappa_calibration_images", C.POINTER(c_f32p)), ("grappa_calibration_seed", C.c_uint64),
        ("shot_sets", C.POINTER(C.POINTER(ShotSet_))), ("n_shot_sets", C.POINTER(C.c_int64)),
    ]


class ExcitationTrain_(C.Structure):
    """`mrsim_excitation_train` — `ExcitationTrain` (readout.rs:362-369)."""

    _fields_ = [("kz_segments", C.c_int64), ("kz_order", C.c_int32), ("reserved", C.c_int32),
                ("exc_spacing_ms", C.c_double), ("echo_times_ms", c_f64p), ("n_echoes", C.c_int64),
                ("excitation_time_ms", C.c_double)]


class Ge3dReadout_(C.Structure):
    """`mrsim_ge3d_readout` — `Ge3dReadout` (readout.rs:374-379)."""

    _fields_ = [("ky_segments", C.c_int64), ("t_line_ms", C.c_double), ("reverse_phase", C.c_int32),
                ("reserved", C.c_int32)]


class GeVolume_(C.Structure):
    """`mrsim_ge_volume` — `GeVolume` (kspace3d.rs:592-603)."""

    _fields_ = [("images", C.POINTER(c_f32p)), ("weights", c_f64p), ("shot_sets", C.POINTER(ShotSet_)),
                ("n_shot_sets", C.c_int64)]


GE_VOLUME_FN = C.CFUNCTYPE(C.c_int, C.c_int64, C.c_void_p, C.POINTER(GeVolume_))


class AcquisitionGeInput_(C.Structure):
    """`mrsim_acquisition_ge_input` — the inputs of `simulate_acquisition_3d_ge` (kspace3d.rs:837)."""

    _fields_ = [
        ("sim_dims", C.c_int64 * 3), ("acq_dims", C.c_int64 * 3), ("n_volumes", C.c_int64), ("ncomp", C.c_int64),
        ("t2", C.POINTER(T2_)), ("fmap", c_f32p), ("t_inhom", C.POINTER(T2_)), ("phase", C.POINTER(PhaseModel_)),
        ("volume", GE_VOLUME_FN), ("user", C.c_void_p), ("reference", C.POINTER(GeVolume_)),
    ]


class KzSampling_(C.Structure):
    """`mrsim_kz_sampling` — `KzSampling` (readout.rs:107-160)."""

    _fields_ = [("partial_fourier", C.c_double), ("accel", C.c_int64)]


class SpiralReadout_(C.Structure):
    """`mrsim_spiral_readout` — `Readout3d::Spiral` (readout.rs:103-106)."""

    _fields_ = [("interleaves", C.c_int64), ("readout_ms", C.c_double), ("dwell_ms", C.c_double),
                ("radial_oversampling", C.c_double), ("kz", KzSampling_)]


class KzOptions_(C.Structure):
    """`mrsim_kz_options` — `KzOptions` (kspace3d.rs:1173-1178)."""

    _fields_ = [("coil_rows", C.c_int64), ("calibration_images", C.POINTER(c_f32p)), ("calibration_seed", C.c_uint64),
                ("pocs", C.c_int32), ("reserved", C.c_int32)]


class SpiralSegmentationRow_(C.Structure):
    """`mrsim_spiral_segmentation_row` — `SpiralSegmentation` (kspace3d.rs:860-870)."""

    _fields_ = [("z", C.c_int32), ("voxel", C.c_int32), ("l", C.c_int32), ("m", C.c_int32), ("b_sum", C.c_double),
                ("bound", C.c_double)]


class Pulse_(C.Structure):
    _fields_ = [("kind", C.c_int32), ("t", C.c_double), ("epsilon", C.c_double)]


class MzReference_(C.Structure):
    _fields_ = [("kind", C.c_int32), ("a", C.c_double), ("b", C.c_double), ("values", c_f64p)]


class SpinShot_(C.Structure):
    _fields_ = [("t", C.c_double), ("transform", C.c_double * 16), ("slices", C.POINTER(C.c_int64)),
                ("n_slices", C.c_int64), ("ref", MzReference_), ("weight", c_f32p)]


class LibraryMissing(RuntimeError):
    pass


_lib = None


def _declare(lib):
    P = C.c_void_p
    sigs = {
        "mrsim_abi_version": (C.c_int, []),
        "mrsim_last_error": (C.c_char_p, []),
        "mrsim_acquisition_default": (C.c_int, [C.POINTER(Acquisition_)]),
        "mrsim_phase_model_hbcd_like": (C.c_int, [C.POINTER(PhaseModel_)]),
        "mrsim_phase_model_none": (C.c_int, [C.POINTER(PhaseModel_)]),
        "mrsim_context_create": (C.c_int, [C.c_int, C.POINTER(P)]),
        "mrsim_context_destroy": (C.c_int, [P]),
        "mrsim_context_stream": (P, [P]),
        "mrsim_context_synchronize": (C.c_int, [P]),
        "mrsim_sampling_mask": (C.c_int, [C.c_int64, C.c_int64, C.POINTER(Acquisition_), C.POINTER(C.c_uint8)]),
        "mrsim_pf_skipped_lines": (C.c_int64, [C.c_int64, C.POINTER(Acquisition_)]),
        "mrsim_line_timing": (C.c_int, [C.POINTER(Acquisition_), C.c_int64, C.c_int64, c_f64p, c_f64p, c_f64p,
                                        C.POINTER(C.c_int8)]),
        "mrsim_validate_acquisition_timing": (C.c_int, [C.POINTER(Acquisition_), C.c_int64, C.c_int64]),
        "mrsim_epi_order": (C.c_int, [C.POINTER(Acquisition_), C.c_int64, C.c_int64, C.POINTER(C.c_int64)]),
        "mrsim_build_coil_kspaces": (C.c_int, [P, C.POINTER(SliceInput_), C.POINTER(Acquisition_), c_f64p, c_f64p,
                                               c_f64p, C.POINTER(C.c_int8), c_f64p, c_f64p]),
        "mrsim_simulate_slice": (C.c_int, [P, C.POINTER(SliceInput_), C.POINTER(Acquisition_), c_f32p]),
        "mrsim_simulate_slice_full": (C.c_int, [P, C.POINTER(SliceInput_), C.POINTER(Acquisition_), c_f32p, c_f32p,
                                                c_f32p, c_f32p, c_f32p, C.POINTER(C.c_uint8)]),
        "mrsim_simulate_slice_kspace": (C.c_int, [P, C.POINTER(SliceInput_), C.POINTER(Acquisition_), c_f64p]),
        "mrsim_simulate_acquisition_complex": (C.c_int, [P, C.POINTER(AcquisitionInput_), C.POINTER(Acquisition_),
                                                         C.POINTER(AcquisitionOptions_),
                                                         C.POINTER(AcquisitionOutput_)]),
        "mrsim_simulate_acquisition_oversampled": (C.c_int, [P, C.POINTER(AcquisitionInput_),
                                                             C.POINTER(Acquisition_), c_f32p, c_f32p]),
        "mrsim_simulate_acquisition_echoes": (C.c_int, [P, C.POINTER(AcquisitionInput_),
                                                        C.POINTER(C.POINTER(c_f32p)), C.POINTER(Acquisition_),
                                                        c_f64p, C.c_int64, C.POINTER(C.POINTER(c_f32p)),
                                                        C.POINTER(C.c_uint64), C.POINTER(c_f32p),
                                                        C.POINTER(c_f32p)]),
        "mrsim_build_coil_kspaces_noalloc": (C.c_int, [C.POINTER(SliceInput_), C.POINTER(Acquisition_), P, c_f32p]),
        "mrsim_epi_operator_create": (C.c_int, [P, C.POINTER(AcquisitionInput_), C.POINTER(Acquisition_), c_f64p,
                                                C.c_int64, C.POINTER(C.c_int64), C.c_int64, C.c_int32,
                                                C.POINTER(P)]),
        "mrsim_epi_operator_destroy": (C.c_int, [P]),
        "mrsim_epi_operator_samples": (C.c_int64, [P]),
        "mrsim_epi_operator_buffers": (C.c_int, [P] + [C.POINTER(c_f32p)] * 5),
        "mrsim_epi_operator_upload_images": (C.c_int, [P, C.POINTER(c_f32p)]),
        "mrsim_epi_operator_set_fieldmap": (C.c_int, [P, c_f32p]),
        "mrsim_epi_operator_forward": (C.c_int, [P]),
        "mrsim_epi_operator_adjoint": (C.c_int, [P]),
        "mrsim_epi_operator_stage": (C.c_int, [P, C.c_int32]),
        "mrsim_probe_fp32_tflops": (C.c_int, [P, C.POINTER(C.c_double)]),
        "mrsim_epi_operator_adjoint_host": (C.c_int, [P, c_f32p, c_f32p, c_f32p, c_f32p]),
        "mrsim_epi_operator_apply_host": (C.c_int, [P, C.POINTER(c_f32p), c_f32p, c_f32p, c_f32p, c_f32p]),
        "mrsim_epi_operator_host_bytes": (C.c_int, [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "mrsim_epi_operator_set_segmented": (C.c_int, [P, C.c_int32]),
        "mrsim_resample_by_pose": (C.c_int, [P, c_f32p, C.POINTER(C.c_int64), c_f64p, c_f64p, c_f32p]),
        "mrsim_apply_motion": (C.c_int, [P, C.POINTER(c_f32p), C.c_int64, C.POINTER(C.c_int64), C.c_int64, c_f64p,
                                         c_f64p]),
        "mrsim_apply_multiband_motion": (C.c_int, [P, C.POINTER(c_f32p), C.c_int64, C.POINTER(C.c_int64), C.c_int64,
                                                   c_f64p, C.c_int64, C.c_int32, C.POINTER(DropoutLaw_),
                                                   C.POINTER(MotionEvent_), C.c_int64, C.POINTER(C.c_int64), C.c_int64,
                                                   C.POINTER(DroppedShot_), C.c_int64, C.POINTER(C.c_int64)]),
        "mrsim_epi_operator_apply_motion": (C.c_int, [P, c_f64p, c_f64p]),
        "mrsim_epi_batch_create": (C.c_int, [P, C.c_int32, C.POINTER(C.POINTER(AcquisitionInput_)),
                                             C.POINTER(Acquisition_), c_f64p, C.c_int64, C.c_int32, C.POINTER(P)]),
        "mrsim_epi_batch_destroy": (C.c_int, [P]),
        "mrsim_epi_batch_samples": (C.c_int64, [P]),
        "mrsim_epi_batch_forward": (C.c_int, [P]),
        "mrsim_epi_batch_adjoint": (C.c_int, [P]),
        "mrsim_epi_batch_download": (C.c_int, [P, C.c_int32, c_f32p, c_f32p]),
        "mrsim_write_nifti_4d": (C.c_int, [C.c_char_p, C.POINTER(C.c_int64), C.c_int64, c_f32p, c_f64p, C.c_double]),
        "mrsim_write_nifti_3d": (C.c_int, [C.c_char_p, C.POINTER(C.c_int64), c_f32p, c_f64p]),
        "mrsim_hires_grid": (C.c_int, [c_f64p, C.POINTER(C.c_int64), C.c_int64, c_f64p, C.POINTER(C.c_int64)]),
        "mrsim_spin_history_create": (C.c_int, [P, C.POINTER(C.c_int64), c_f64p, c_f32p, c_f32p,
                                                C.POINTER(C.c_uint8), C.c_int64, C.POINTER(C.c_int64), c_f64p,
                                                C.POINTER(Pulse_), C.c_int64, C.POINTER(P)]),
        "mrsim_spin_history_destroy": (None, [P]),
        "mrsim_spin_history_n_tracked": (C.c_int, [P, C.POINTER(C.c_int64)]),
        "mrsim_spin_history_prime": (C.c_int, [P, c_f64p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_int64,
                                               c_f64p]),
        "mrsim_spin_history_terms_size": (C.c_int, [P, C.POINTER(SpinShot_), C.c_int64, C.POINTER(C.c_int64)]),
        "mrsim_spin_history_excite": (C.c_int, [P, C.POINTER(SpinShot_), C.c_int64, c_f32p]),
        "mrsim_spin_history_excite_device": (C.c_int, [P, C.POINTER(SpinShot_), C.c_int64, P]),
        "mrsim_spin_history_merges": (C.c_int, [P, C.POINTER(C.c_uint64)]),
        "mrsim_write_complex_4d": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_int64), C.c_int64, c_f32p, c_f32p,
                                             c_f64p, C.POINTER(SidecarInfo_)]),
        "mrsim_epi_operator_apply_host_compact": (C.c_int, [P, C.POINTER(c_f32p), c_f32p, c_f32p, c_f32p, c_f32p]),
        "mrsim_epi_operator_acquired_rows": (C.c_int, [P] + [C.POINTER(C.c_int32)] * 3),
        "mrsim_epi_operator_host_bytes_for": (C.c_int, [P, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "mrsim_epi_operator_segmentation": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32), c_f64p,
                                                      C.c_int32, c_f64p, c_f64p]),
        "mrsim_epi_operator_segmented_status": (C.c_int, [P, C.POINTER(C.c_int32)]),
        "mrsim_epi_operator_tune": (C.c_int, [P, C.c_char_p, C.c_int32, C.c_char_p, C.c_int64,
                                              C.POINTER(C.c_double)]),
        "mrsim_spiral_tau_c": (C.c_int, [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, c_f64p]),
        "mrsim_spiral_trajectory": (C.c_int, [C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double,
                                              C.c_int64, c_f64p, c_f64p, C.POINTER(SpiralInfo_)]),
        "mrsim_tseg_plan": (C.c_int, [c_f64p, C.c_int64, C.c_double, c_f64p, c_f64p, C.c_int64, c_f64p, c_f64p,
                                      C.POINTER(TsegInfo_)]),
        "mrsim_tseg_plan_device": (C.c_int, [P, c_f64p, C.c_int64, C.c_double, c_f64p, c_f64p, C.c_int64, c_f64p,
                                             c_f64p, C.POINTER(TsegInfo_)]),
        "mrsim_epg_cpmg": (C.c_int, [C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double, c_f64p]),
        "mrsim_nufft_kernel_width": (C.c_int, [C.c_double]),
        "mrsim_nufft1": (C.c_int, [P, C.c_int64, C.c_int64, C.c_int64, C.c_double, c_f64p, C.c_int64, c_f64p,
                                   C.c_int64, c_f64p]),
        "mrsim_nufft2_type1": (C.c_int, [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                         C.c_double, c_f64p, C.c_int64, c_f32p, C.c_int32, c_f32p]),
        "mrsim_nufft2_type2": (C.c_int, [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                         C.c_double, c_f32p, c_f64p, C.c_int64, C.c_int32, c_f32p]),
        "mrsim_spiral_kspace_exact": (C.c_int, [P, C.POINTER(SliceInput_), C.POINTER(Acquisition_), C.c_int64,
                                                C.c_int64, c_f64p, c_f64p, C.c_int64, c_f64p, c_f32p]),
        "mrsim_spiral_segmented_forward": (C.c_int, [P, C.POINTER(SliceInput_), C.POINTER(Acquisition_), C.c_int64,
                                                     C.c_int64, c_f64p, C.POINTER(C.c_int64), C.c_int64, c_f64p,
                                                     C.c_int64, C.c_double, c_f64p, c_f64p, c_f64p, C.c_int32,
                                                     c_f32p, C.POINTER(TsegInfo_)]),
        "mrsim_kz_order": (C.c_int, [C.c_int64, C.c_int32, C.POINTER(C.c_int64)]),
        "mrsim_grase_lines": (C.c_int, [C.POINTER(EchoTrain_), C.POINTER(GraseReadout_), C.c_int64, C.c_int64,
                                        C.POINTER(C.c_int64), C.POINTER(C.c_int64), c_f64p, c_f64p,
                                        C.POINTER(C.c_int8), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "mrsim_simulate_acquisition_3d": (C.c_int, [P, C.POINTER(Acquisition3dInput_), C.POINTER(Acquisition_),
                                                    C.POINTER(EchoTrain_), C.POINTER(GraseReadout_), C.c_uint64,
                                                    c_f32p, c_f32p]),
        "mrsim_kspace_3d_observed": (C.c_int, [P, C.POINTER(Acquisition3dInput_), C.POINTER(Acquisition_),
                                               C.POINTER(EchoTrain_), C.POINTER(GraseReadout_), C.c_int64, c_f32p]),
        "mrsim_ge3d_lines": (C.c_int, [C.POINTER(ExcitationTrain_), C.POINTER(Ge3dReadout_), C.c_int64, C.c_int64,
                                       C.POINTER(C.c_int64), C.POINTER(C.c_int64), c_f64p, C.POINTER(C.c_int8),
                                       C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "mrsim_simulate_acquisition_3d_ge": (C.c_int, [P, C.POINTER(AcquisitionGeInput_), C.POINTER(Acquisition_),
                                                       C.POINTER(ExcitationTrain_), C.POINTER(Ge3dReadout_),
                                                       C.c_uint64, C.POINTER(c_f32p), C.POINTER(c_f32p)]),
        "mrsim_check_grase_timing": (C.c_int, [C.POINTER(EchoTrain_), C.POINTER(GraseReadout_), C.c_int64, C.c_int64,
                                               C.c_double, C.c_double]),
        "mrsim_check_ge3d_timing": (C.c_int, [C.POINTER(ExcitationTrain_), C.POINTER(Ge3dReadout_), C.c_int64,
                                              C.c_int64, C.c_double, C.c_double]),
        "mrsim_check_spiral_timing": (C.c_int, [C.POINTER(EchoTrain_), C.POINTER(SpiralReadout_), C.c_int64, C.c_int64,
                                                C.c_int64, C.c_double, C.c_double, c_f64p]),
        "mrsim_esp_from_echo_time": (C.c_double, [C.c_double, C.c_int64, C.POINTER(GraseReadout_), C.c_int64]),
        "mrsim_spiral_esp_from_echo_time": (C.c_double, [C.c_double, C.c_int64]),
        "mrsim_spiral_segmentation": (C.c_int, [C.POINTER(Acquisition3dInput_), C.POINTER(Acquisition_),
                                                C.POINTER(EchoTrain_), C.POINTER(SpiralReadout_), C.c_int64,
                                                C.POINTER(SpiralSegmentationRow_), C.POINTER(C.c_int64)]),
        "mrsim_spiral_lines": (C.c_int, [C.POINTER(EchoTrain_), C.POINTER(SpiralReadout_), C.c_int64, C.c_int64,
                                         C.c_int64, C.POINTER(C.c_uint8), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                         C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                         C.POINTER(C.c_int64)]),
        "mrsim_simulate_acquisition_3d_spiral": (C.c_int, [P, C.POINTER(Acquisition3dInput_), C.POINTER(Acquisition_),
                                                           C.POINTER(EchoTrain_), C.POINTER(SpiralReadout_),
                                                           C.POINTER(KzOptions_), C.c_uint64, c_f32p, c_f32p]),
        "mrsim_spiral_samples_3d": (C.c_int, [P, C.POINTER(Acquisition3dInput_), C.POINTER(Acquisition_),
                                              C.POINTER(EchoTrain_), C.POINTER(SpiralReadout_), C.POINTER(KzOptions_),
                                              C.c_int64, c_f32p]),
        "mrsim_spiral_recon_create": (C.c_int, [P, c_f64p, C.c_int64, C.c_int64, C.c_int32, C.c_double, C.c_double,
                                                C.c_int64, C.c_double, C.c_int32, C.POINTER(P)]),
        "mrsim_spiral_recon_destroy": (C.c_int, [P]),
        "mrsim_spiral_recon_info": (C.c_int, [P, c_f64p, C.POINTER(C.c_int64), c_f64p]),
        "mrsim_spiral_recon_gridding": (C.c_int, [P, c_f64p, C.c_int64, c_f64p]),
        "mrsim_spiral_recon_image": (C.c_int, [P, c_f64p, C.c_int64, c_f64p]),
        "mrsim_spiral_recon_rings": (C.c_int, [P, c_f64p, C.c_int64, C.c_int64, C.c_int64, c_f64p, c_f64p]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def lib():
    """The loaded library (raises LibraryMissing if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise LibraryMissing(f"{LIB_PATH} is missing: run `python mrsim_acq_b200/build.py` "
                                 "(the k-space path has no CPU fallback)")
        _lib = _declare(C.CDLL(str(LIB_PATH)))
    return _lib


class MrsimError(RuntimeError):
    """A non-zero status from the library; the message is the reference's panic text."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def check(status: int):
    if status != 0:
        raise MrsimError(status, lib().mrsim_last_error().decode())
    return status


def declared_symbols() -> list[str]:
    """Every function name include/mrsim_acq.h declares (parsed from the header)."""
    import re
    text = (HERE.parent / "include" / "mrsim_acq.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(mrsim_\w+)\s*\(", text, re.M)))
