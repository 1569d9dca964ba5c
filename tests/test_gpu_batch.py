"""A batch of series of different geometries as one plan (`mrsim_epi_batch`): scans of 16, 24 and
32 lines on 2x grids (the precision-at-scale configuration's 64/96/128 mix, scaled down) with
uneven slice counts 3, 2 and 4, one launch per stage over every unit; every series' k-space and
complex-image adjoint against the FP64 oracle (relative L2 <= 1e-5) and equal to the series run
alone.  A second mix, scans of 32, 48 and 64 (rows of 64, 96 and 128 points: every one a warp-FFT
width, but not one width), runs the warp FFT once per width in the batch, as each series alone
does."""
import numpy as np
import pytest

from mrsim_acq_b200 import api
from mrsim_acq_b200.api import Acquisition, PartialFourierMode, PhaseModel
from oracle import oracle
from tests import cases

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))


MIXES = [(((16, 3), (24, 2), (32, 4)), 8, 1e-6), (((32, 2), (48, 1), (64, 2)), 4, 5e-6)]


@pytest.mark.parametrize("mix,coils,alone_tol", MIXES)
def test_mixed_geometry_batch_matches_the_oracle(gpu_ctx, mix, coils, alone_tol):
    acq = Acquisition(n_coils=coils, accel=2, partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner, t_line=0.5,
                      t_echo=30.0, ghost_offset=0.05)
    tes = [30.0, 50.0]
    series = []
    for n, nz in mix:
        s = cases.series_case(nx=n, ny=n, nz=nz, o=2, nv=2, ncomp=3)
        s.update(phase=PhaseModel.hbcd_like(), seed=42)
        series.append(s)
    b = api.EpiBatch(series, acq, echo_times_ms=tes, grads=0, ctx=gpu_ctx)
    assert b.samples == sum(cases_samples(s, acq, tes) for s in series)
    b.forward()
    b.adjoint()
    for i, s in enumerate(series):
        got = b.download(i)
        kw = dict(t_inhom=s["t_inhom"], phase=s["phase"], seed=42)
        want = oracle.series_forward(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"], acq,
                                     echo_times_ms=tes, **kw)
        assert rel_l2(got["kspace"], want) <= 1e-5, i
        adj = oracle.series_adjoint(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"], acq,
                                    got["kspace"].astype(np.complex128), echo_times_ms=tes, **kw)
        assert rel_l2(got["comp_grad"], adj["comp_grad"]) <= 1e-5, i
        op = api.EpiOperator(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["t2"], s["fmap"], acq, images=s["images"],
                             echo_times_ms=tes, grads=0, ctx=gpu_ctx, **kw)
        alone = op.apply_host(None)
        op.close()
        assert rel_l2(got["kspace"], alone["kspace"]) <= alone_tol, i
    b.close()


def cases_samples(s, acq, tes):
    nx, ny, nz = s["acq_dims"]
    rows = int(api.sampling_mask(nx, ny, acq).reshape(ny, nx)[:, 0].sum())
    return s["n_volumes"] * nz * acq.n_coils * len(tes) * rows * nx
