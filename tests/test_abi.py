"""The C ABI library without a GPU: it loads, exports every declared symbol, and its host tables
(sampling mask, line timing, acquisition order, timing validation) equal the oracle's bit for bit."""
import ctypes as C
import itertools

import numpy as np
import pytest

from mrsim_acq_b200 import abi, api
from mrsim_acq_b200.api import Acquisition, PartialFourierMode
from oracle import oracle


def test_library_exports_every_declared_symbol():
    lib = abi.lib()
    declared = abi.declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert lib.mrsim_abi_version() == 1


def _configs():
    for pf, mode, rev, accel in itertools.product((1.0, 0.75, 0.8, 0.625), list(PartialFourierMode), (False, True),
                                                  (1, 2, 3)):
        yield Acquisition(partial_fourier=pf, pf_mode=mode, reverse_phase=rev, accel=accel, t_line=0.5, t_echo=30.0)


@pytest.mark.parametrize("nx,ny", [(17, 70), (16, 40), (8, 9), (64, 64), (64, 48), (1, 1), (3, 2)])
def test_sampling_mask_and_timing_match_the_oracle(nx, ny):
    for acq in _configs():
        assert np.array_equal(api.sampling_mask(nx, ny, acq), oracle.sampling_mask(nx, ny, acq))
        lt = api.LineTiming.for_acquisition(acq, nx, ny)
        t, trf, tread, pol = oracle.line_timing(acq, nx, ny)
        for a, b in ((lt.t_ms, t), (lt.trf_ms, trf), (lt.tread_ms, tread)):
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
        assert np.array_equal(lt.polarity, pol)
        o = np.zeros(ny, np.int64)
        oracle.lib().oracle_epi_order(C.byref(acq.to_c()), nx, ny, o.ctypes.data_as(C.POINTER(C.c_int64)))
        assert np.array_equal(api.epi_order(nx, ny, acq), o)
        assert api.pf_skipped_lines(ny, acq) == oracle.lib().oracle_pf_skipped_lines(ny, C.byref(acq.to_c()))


def test_scanner_pf_keeps_round_ny_pf_lines():
    """kspace.rs:4011: Scanner PF keeps exactly round(ny*pf) consecutive lines and skips the first
    lines of the train (high ky, or low ky when reversed)."""
    for ny, pf in [(64, 0.75), (40, 0.8), (9, 0.625)]:
        for rev in (False, True):
            acq = Acquisition(partial_fourier=pf, pf_mode=PartialFourierMode.Scanner, reverse_phase=rev)
            rows = np.nonzero(api.sampling_mask(4, ny, acq)[:, 0])[0]
            assert len(rows) == round(ny * pf)
            assert rows[-1] - rows[0] + 1 == len(rows)
            assert (rows[0] == 0) != rev or (rows[-1] == ny - 1) == rev


def test_negative_trf_is_rejected_with_the_reference_message():
    """kspace.rs:3702: a readout that starts before the excitation is an error."""
    acq = Acquisition(t_echo=10.0, t_line=1.0)
    with pytest.raises(abi.MrsimError, match=r"trf = .* ms <= 0 on an acquired line"):
        api.validate_acquisition_timing(acq, 64, 64)
    assert oracle.lib().oracle_validate_acquisition_timing(C.byref(acq.to_c()), 64, 64) != 0
    api.validate_acquisition_timing(Acquisition(), 64, 64)


def test_no_cpu_fallback_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(abi.MrsimError, match="no CUDA device"):
        api.Context(0)
