"""B200-native k-space acquisition path of mrsim-acq: CUDA kernels for sm_100a behind a C ABI.

`api` mirrors the reference crate's names (Acquisition, SliceInput, T2, PhaseModel,
sampling_mask, LineTiming, build_coil_kspaces, EpiOperator); `abi` is the ctypes layer over
include/mrsim_acq.h; `build` compiles libmrsim_acq_cuda.so in-tree.
"""
from .abi import LibraryMissing, MrsimError, lib  # noqa: F401
from .api import (Acquisition, AcquisitionInput, AcquisitionOptions, Context, EchoFormation, EpiOperator, KspaceWindow, LineTiming,  # noqa: F401
                  PartialFourierMode, PhaseModel, SliceInput, T2, build_coil_kspaces, default_context,
                  epi_order, pf_skipped_lines, sampling_mask, simulate_acquisition_complex,
                  simulate_acquisition_echoes, simulate_acquisition_oversampled, simulate_slice,
                  simulate_slice_full, simulate_slice_kspace, validate_acquisition_timing)
