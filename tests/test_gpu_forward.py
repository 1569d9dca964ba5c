"""GPU parity of the FP32 exact-DFT forward (`build_coil_kspace_timed`, kspace.rs:607-1042)
against the FP64 oracle, through the C ABI.  Tolerance: relative L2 <= 1e-5 against FP64."""
import numpy as np
import pytest

from mrsim_acq_b200 import api
from oracle import oracle
from tests import cases

pytestmark = pytest.mark.gpu
TOL = 1e-5


def rel_l2(a, b):
    n = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (n if n > 0 else 1.0)


@pytest.mark.parametrize("idx", range(39))
def test_golden_slices_forward_matches_the_oracle(idx, gpu_ctx):
    name, inp, acq = cases.golden_cases()[idx]
    got = api.build_coil_kspaces(inp, acq, ctx=gpu_ctx)
    nc = max(acq.n_coils, 1)
    for q in range(nc):
        want = oracle.build_coil_kspace(inp, acq, q, nc)
        assert rel_l2(got[q], want) <= TOL, f"{name} coil {q}: rel-L2 {rel_l2(got[q], want):.2e}"


@pytest.mark.parametrize("idx", range(48))
def test_forward_matches_the_literal_sum(idx, gpu_ctx):
    name, inp, acq, coil, ncoils = cases.literal_sum_cases()[idx]
    got = api.build_coil_kspaces(inp, acq.replace(n_coils=ncoils), ctx=gpu_ctx)[coil]
    want = oracle.reference_coil_kspace(inp, acq.replace(n_coils=ncoils), coil, ncoils)
    assert rel_l2(got, want) <= TOL, f"{name}: {rel_l2(got, want):.2e}"


def test_eddy_known_answer_case(gpu_ctx):
    from tests.test_oracle import eddy_known_answer_case
    inp, acq = eddy_known_answer_case()
    got = api.simulate_slice_kspace(inp, acq, ctx=gpu_ctx)
    want = oracle.build_coil_kspace(inp, acq, 0, 1)
    assert rel_l2(got, want) <= TOL


def test_timing_override_and_log_amp(gpu_ctx):
    """The 3D drivers' entry: an explicit line table and a voxel log-amplitude (kspace.rs:600-606)."""
    name, inp, acq = cases.golden_cases()[11]  # maps, 17x70 o2
    nx, ny = inp.acq_matrix
    t, trf, tread, pol = oracle.line_timing(acq, nx, ny)
    t = t * 0.9 + 0.1
    timing = api.LineTiming(t, trf + 3.0, tread, pol)
    la = np.linspace(-0.2, 0.1, inp.sim[0] * inp.sim[1])
    got = api.build_coil_kspaces(inp, acq, timing=timing, log_amp=la, ctx=gpu_ctx)[0]
    want = oracle.build_coil_kspace(inp, acq, 0, 1, timing=timing, log_amp=la)
    assert rel_l2(got, want) <= TOL


def test_spikes_land_on_the_oracle_samples(gpu_ctx):
    """kspace.rs:3265: spikes overwrite acquired samples with a fraction of the peak."""
    name, inp, acq = cases.golden_cases()[1]
    acq = acq.replace(n_spikes=3, spike_amplitude=0.5, partial_fourier=0.75)
    got = api.build_coil_kspaces(inp, acq, ctx=gpu_ctx)[0]
    want = oracle.build_coil_kspace(inp, acq, 0, 1)
    assert rel_l2(got, want) <= TOL


def test_empty_slice_gives_zero_kspace(gpu_ctx):
    name, inp, acq = cases.golden_cases()[14]
    inp.compartments = [np.zeros_like(c) for c in inp.compartments]
    got = api.build_coil_kspaces(inp, acq, ctx=gpu_ctx)
    assert np.all(got == 0)


@pytest.mark.parametrize("idx", [0, 11, 20, 33])
def test_eight_ring_coils_match_the_oracle(idx, gpu_ctx):
    """Eight ring coils put the per-slice forward on the coil-class kernels (5 classes of equal
    ey rows + the coil offset, class rows through the x-stage); every coil against the oracle."""
    name, inp, acq = cases.golden_cases()[idx]
    acq = acq.replace(n_coils=8, accel=1, acs_lines=0)
    got = api.build_coil_kspaces(inp, acq, ctx=gpu_ctx)
    for q in range(8):
        want = oracle.build_coil_kspace(inp, acq, q, 8)
        assert rel_l2(got[q], want) <= TOL, f"{name} coil {q}: rel-L2 {rel_l2(got[q], want):.2e}"
