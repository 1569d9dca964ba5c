"""The time-segmented tensor-core operator pair (tcgen05 contractions in split f16 / bf16) against
the FP64 oracle's exact forward and adjoint (relative L2 <= 1e-5, the bar of every FP32 result).

The reference segments only the spiral forward (`tseg::plan`, tseg.rs:230-289); here its
certificate segments the EPI lines of each echo (split at the spin echo) so that the y-stage is
a dense contraction.  Cases: the small series shape with the 8-coil ring (the class-row
x-stage), a 4-coil series (coil rows: the class rows are expanded / combined around the
contractions), the benchmark's 64x64-on-128x128 geometry, the differentiation grid (192-point
rows, lines split into groups of at most 256 outputs), the gradient echo, the adjoint identity,
and the refusals."""
import numpy as np
import pytest

from mrsim_acq_b200 import api
from mrsim_acq_b200.abi import MrsimError
from mrsim_acq_b200.api import T2, Acquisition, EchoFormation, PartialFourierMode, PhaseModel
from oracle import oracle
from tests import cases

pytestmark = pytest.mark.gpu
TOL = 1e-5


def rel_l2(a, b):
    n = np.linalg.norm(np.ravel(b))
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / (n if n > 0 else 1.0)


def _case(nx=16, o=2, nv=2, nz=2, coils=8, tes=(15.0, 35.0, 55.0), echo=EchoFormation.Spin, ncomp=3):
    s = cases.series_case(nx=nx, ny=nx, nz=nz, o=o, nv=nv, ncomp=ncomp)
    acq = Acquisition(n_coils=coils, accel=2, partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner, t_line=0.5,
                      t_echo=30.0, ghost_offset=0.05, signal_scale=100.0, echo=echo)
    kw = dict(t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42)
    return s, acq, list(tes), kw


def _run(s, acq, tes, kw, ctx, precision):
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=0, ctx=ctx, **kw)
    op.set_segmented(precision)
    info = op.segmentation()
    out = op.apply_host(None)
    status = op.segmented_status()
    op.close()
    assert status == 0, f"a segmented kernel gave up a wait (code {status})"
    want = oracle.series_forward(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"], acq,
                                 echo_times_ms=tes, **kw)
    ef = rel_l2(out["kspace"], want)
    adj = oracle.series_adjoint(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"], acq,
                                out["kspace"].astype(np.complex128), echo_times_ms=tes, **kw)
    ea = rel_l2(out["comp_grad"], adj["comp_grad"])
    print(f"{precision}: L {info['L']}, bound {max(info['bound']):.1e}, forward rel-L2 {ef:.2e}, adjoint {ea:.2e}")
    return ef, ea, info


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_class_rows_series_matches_the_oracle(precision, gpu_ctx):
    s, acq, tes, kw = _case()
    ef, ea, info = _run(s, acq, tes, kw, gpu_ctx, precision)
    assert max(info["bound"]) < 1e-7
    assert ef <= TOL and ea <= TOL, (ef, ea)


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_coil_rows_series_matches_the_oracle(precision, gpu_ctx):
    s, acq, tes, kw = _case(coils=4, tes=(20.0, 40.0))
    ef, ea, _ = _run(s, acq, tes, kw, gpu_ctx, precision)
    assert ef <= TOL and ea <= TOL, (ef, ea)


def test_gradient_echo_matches_the_oracle(gpu_ctx):
    s, acq, tes, kw = _case(tes=(20.0, 30.0), echo=EchoFormation.Gradient, ncomp=2)
    ef, ea, _ = _run(s, acq, tes, kw, gpu_ctx, "f16")
    assert ef <= TOL and ea <= TOL, (ef, ea)


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_benchmark_geometry_matches_the_oracle(precision, gpu_ctx):
    """64x64 on 128x128, 8 coils, 3 compartments, echoes 15/35/55 ms, two slices of one volume."""
    s, acq, tes, kw = _case(nx=64, nv=1, nz=2)
    ef, ea, info = _run(s, acq, tes, kw, gpu_ctx, precision)
    assert ef <= TOL and ea <= TOL, (ef, ea)


def test_differentiation_grid_matches_the_oracle(gpu_ctx):
    """96x96 on 192x192 (192-point rows: the per-coil x-stage), 8 coils, 2 compartments, one
    echo whose second half splits into two line groups."""
    s, acq, tes, kw = _case(nx=96, nv=1, nz=2, tes=(30.0,), ncomp=2)
    ef, ea, info = _run(s, acq, tes, kw, gpu_ctx, "f16")
    assert len(info["L"]) >= 3
    assert ef <= TOL and ea <= TOL, (ef, ea)


def test_adjoint_identity(gpu_ctx):
    """<A x, y> = <x, A^H y> for the segmented pair itself (split f16)."""
    s, acq, tes, kw = _case()
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=0, ctx=gpu_ctx, **kw)
    op.set_segmented("f16")
    Ax = op.apply_host(None)["kspace"].astype(np.complex128)
    rng = np.random.default_rng(3)
    y = (rng.standard_normal(Ax.shape) + 1j * rng.standard_normal(Ax.shape)) * (Ax != 0)
    cg = op.adjoint_host(y.astype(np.complex64))["comp_grad"].astype(np.complex128)
    op.close()
    snx, sny, nz = s["sim_dims"]
    nv, nc = s["n_volumes"], len(s["t2"])
    x = np.stack([s["images"][c].reshape(nz, sny, snx, nv) for c in range(nc)])
    x = np.transpose(x, (4, 1, 0, 2, 3))
    lhs, rhs = np.vdot(y, Ax), np.vdot(cg, x)
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs), (lhs, rhs)


def test_exact_path_restored(gpu_ctx):
    s, acq, tes, kw = _case(nv=1, nz=1)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 1, s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=0, ctx=gpu_ctx, **kw)
    op.set_segmented("f16")
    op.set_segmented("exact")
    assert op.segmentation()["L"] == []
    out = op.apply_host(None)
    op.close()
    want = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], s["fmap"], acq,
                                 echo_times_ms=tes, **kw)
    assert rel_l2(out["kspace"], want) <= TOL


def test_refusals(gpu_ctx):
    s, acq, tes, kw = _case(nv=1, nz=1)

    def make(acq=acq, grads=0, t2=s["t2"]):
        return api.EpiOperator(s["sim_dims"], s["acq_dims"], 1, t2, s["fmap"], acq, images=s["images"],
                               echo_times_ms=tes, grads=grads, ctx=gpu_ctx, **kw)

    with pytest.raises(MrsimError, match="grads = 0"):
        make(grads=1).set_segmented("f16")
    with pytest.raises(MrsimError, match="uniform T2"):
        snx, sny, _ = s["sim_dims"]
        make(t2=[T2.of_map(np.full(snx * sny, 70.0, np.float32))] + s["t2"][1:]).set_segmented("f16")
    kw2 = dict(kw, eddy_drive=[(0.5, -0.4, 0.7)])
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 1, s["t2"], s["fmap"], acq.replace(eddy_strength=2.0),
                         images=s["images"], echo_times_ms=tes, grads=0, ctx=gpu_ctx, **kw2)
    with pytest.raises(MrsimError, match="eddy-current polynomial"):
        op.set_segmented("f16")
