"""The autotuner (`mrsim_epi_operator_tune`): it times the plan's tunables (coil classes, x-stage
FFT or DFT GEMM, the y-adjoint's rows per thread, optionally the segmented path), keeps the
fastest, records it in its cache file, and a second operator of the same shape takes the cached
choice; the tuned operator still matches the FP64 oracle."""
import numpy as np
import pytest

from mrsim_acq_b200 import api
from mrsim_acq_b200.api import Acquisition, PartialFourierMode, PhaseModel
from oracle import oracle
from tests import cases

pytestmark = pytest.mark.gpu


def _case():
    s = cases.series_case(nx=32, ny=32, nz=3, o=2, nv=4, ncomp=3)
    acq = Acquisition(n_coils=8, accel=2, partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner, t_line=0.5,
                      t_echo=30.0, ghost_offset=0.05)
    return s, acq, [20.0, 40.0], dict(t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42)


@pytest.mark.parametrize("segmented", [False, True])
def test_tuned_operator_matches_the_oracle_and_caches(gpu_ctx, tmp_path, segmented):
    s, acq, tes, kw = _case()
    cache = tmp_path / "tune.txt"

    def make():
        return api.EpiOperator(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["t2"], s["fmap"], acq,
                               images=s["images"], echo_times_ms=tes, grads=0, ctx=gpu_ctx, **kw)

    op = make()
    r = op.tune(cache, segmented=segmented)
    assert r["ms"] > 0 and "path=" in r["choice"] and "(cached)" not in r["choice"]
    out = op.apply_host(None)
    op.close()
    want = oracle.series_forward(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"], acq,
                                 echo_times_ms=tes, **kw)
    e = np.linalg.norm(out["kspace"] - want) / np.linalg.norm(want)
    print(r, f"rel-L2 {e:.2e}")
    assert e <= 1e-5
    assert cache.read_text().count("\t") == 1
    op2 = make()
    r2 = op2.tune(cache, segmented=segmented)
    assert r2["choice"] == r["choice"] + " (cached)" and r2["ms"] == 0.0
    out2 = op2.apply_host(None)
    op2.close()
    assert np.array_equal(out2["kspace"], out["kspace"])
