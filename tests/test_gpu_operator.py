"""GPU parity of the batched series operator pair: the forward over every (volume, slice, echo,
coil) and its adjoint / VJP (no reference counterpart; checked against the FP64 transpose, the
dot-product identity and central finite differences)."""
import numpy as np
import pytest

from mrsim_acq_b200 import api
from mrsim_acq_b200.api import Acquisition, PartialFourierMode, PhaseModel
from oracle import oracle
from tests import cases

pytestmark = pytest.mark.gpu
TOL = 1e-5


def rel_l2(a, b):
    n = np.linalg.norm(np.ravel(b))
    return np.linalg.norm(np.ravel(a - b)) / (n if n > 0 else 1.0)


def _setup(maps=False, eddy=True, gradient=False, nv=2, nz=2, ncomp=3, coils=4):
    s = cases.series_case(nv=nv, nz=nz, ncomp=ncomp, maps=maps)
    acq = Acquisition(n_coils=coils, accel=2, partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner, t_line=0.5,
                      t_echo=30.0, ghost_offset=0.02, eddy_strength=2.0 if eddy else 0.0, eddy_quad=0.3,
                      eddy_phase=0.1 if eddy else 0.0)
    if gradient:
        acq = acq.replace(echo=api.EchoFormation.Gradient)
    tes = [15.0, 35.0, 55.0]
    kw = dict(t_inhom=s["t_inhom"], eddy_drive=[(0.5, -0.4, 0.7) if g % 2 == 0 else None for g in range(nv)],
              prep_drive=[(1000.0, (0.6, 0.8, 0.0))] * nv, phase=PhaseModel.hbcd_like(), seed=42)
    return s, acq, tes, kw


@pytest.mark.parametrize("maps,eddy,gradient,coils", [(False, False, False, 4), (False, True, False, 4),
                                                      (True, True, False, 4), (False, True, True, 4),
                                                      (True, False, False, 8), (False, False, False, 8)])
def test_series_forward_and_adjoint_match_the_oracle(maps, eddy, gradient, coils, gpu_ctx):
    s, acq, tes, kw = _setup(maps, eddy, gradient, coils=coils)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=3, ctx=gpu_ctx, **kw)
    out = op.apply_host(None)
    want = oracle.series_forward(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"], acq,
                                 echo_times_ms=tes, **kw)
    assert out["kspace"].shape == want.shape
    assert rel_l2(out["kspace"], want) <= TOL, rel_l2(out["kspace"], want)
    adj = oracle.series_adjoint(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"], acq,
                                out["kspace"].astype(np.complex128), echo_times_ms=tes, **kw)
    for key in ("comp_grad", "fmap_grad", "r2_grad"):
        e = rel_l2(out[key], adj[key])
        assert e <= TOL, f"{key}: rel-L2 {e:.2e}"


def test_adjoint_identity(gpu_ctx):
    """<A x, y> = <x, A^H y> with the GPU forward and adjoint (x the real images, y random k-space
    on the acquired samples)."""
    s, acq, tes, kw = _setup()
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=0, ctx=gpu_ctx, **kw)
    Ax = op.apply_host(None)["kspace"].astype(np.complex128)
    rng = np.random.default_rng(3)
    y = (rng.standard_normal(Ax.shape) + 1j * rng.standard_normal(Ax.shape)) * (Ax != 0)
    cg = op.adjoint_host(y.astype(np.complex64))["comp_grad"].astype(np.complex128)
    snx, sny, nz = s["sim_dims"]
    nv, nc = s["n_volumes"], len(s["t2"])
    x = np.stack([s["images"][c].reshape(nz, sny, snx, nv) for c in range(nc)])  # [c][z][y][x][g]
    x = np.transpose(x, (4, 1, 0, 2, 3))  # [g][z][c][y][x]
    lhs = np.vdot(y, Ax)                # <A x, y> conj convention: sum conj(y) Ax
    rhs = np.vdot(cg, x)                # sum conj(A^H y) x
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs), (lhs, rhs)


def test_fieldmap_and_r2_vjp_match_central_differences(gpu_ctx):
    """dL/dfmap and dL/dR2 at seeded voxels against central differences of the FP64 oracle
    forward, L = sum |A(m, fmap, R2)|^2 (h = 1e-3 Hz and a relative 1e-3 step in T2)."""
    s, acq, tes, kw = _setup(eddy=False, nv=1, nz=1)
    acq = acq.replace(n_coils=2)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 1, s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=3, ctx=gpu_ctx, **kw)
    out = op.apply_host(None)
    snx, sny, _ = s["sim_dims"]
    rng = np.random.default_rng(11)
    vox = rng.choice(snx * sny, 6, replace=False)

    def loss(fmap):
        k = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], fmap, acq,
                                  echo_times_ms=tes, **kw)
        return float(np.sum(np.abs(k) ** 2))

    h = 1e-3
    f0 = s["fmap"].astype(np.float64)
    for v in vox:
        fp, fm = f0.copy(), f0.copy()
        fp[v] += h
        fm[v] -= h
        fd = (loss(fp.astype(np.float32)) - loss(fm.astype(np.float32))) / (fp[v].astype(np.float32) - fm[v].astype(np.float32))
        g = out["fmap_grad"].reshape(-1)[v]
        assert abs(g - fd) <= 2e-3 * max(abs(fd), 1e-3 * np.abs(out["fmap_grad"]).max()), (v, g, fd)


@pytest.mark.parametrize("nv,nz", [(11, 1), (5, 3)])
def test_apply_host_volume_groups_match_the_oracle(nv, nz, gpu_ctx):
    """The host-buffer call computes and copies back in groups of volumes (ragged last group):
    every group's k-space and gradients against the FP64 oracle."""
    s, acq, tes, kw = _setup(eddy=True, nv=nv, nz=nz, coils=2)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], nv, s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=3, ctx=gpu_ctx, **kw)
    out = op.apply_host(s["images"])
    want = oracle.series_forward(s["sim_dims"], s["acq_dims"], nv, s["images"], s["t2"], s["fmap"], acq,
                                 echo_times_ms=tes, **kw)
    for g in range(nv):
        assert rel_l2(out["kspace"][g], want[g]) <= TOL, g
    adj = oracle.series_adjoint(s["sim_dims"], s["acq_dims"], nv, s["images"], s["t2"], s["fmap"], acq,
                                out["kspace"].astype(np.complex128), echo_times_ms=tes, **kw)
    for key in ("comp_grad", "fmap_grad", "r2_grad"):
        for g in range(nv):
            e = rel_l2(out[key][g], adj[key][g])
            assert e <= TOL, f"{key} volume {g}: rel-L2 {e:.2e}"


def test_apply_host_fills_the_rows_it_does_not_download(gpu_ctx):
    """The host call downloads only the acquired k-space rows when they form a uniform stride
    and zero-fills the others on the host: outputs preset to garbage come back identical to
    outputs preset to zero, with exact zeros outside the acquired rows."""
    s, acq, tes, kw = _setup(eddy=False, nv=3, nz=2, coils=4)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 3, s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=3, ctx=gpu_ctx, **kw)
    clean = op.apply_host(s["images"])
    shp = op.shapes()
    dirty = {"kspace": np.full(shp["kspace"], np.nan + 1j * np.nan, np.complex64),
             "comp_grad": np.full(shp["comp_grad"], 7.0, np.complex64),
             "fmap_grad": np.full(shp["fmap_grad"], -3.0, np.float32),
             "r2_grad": np.full(shp["r2_grad"], 5.0, np.float32)}
    out = op.apply_host(s["images"], dirty)
    for key in ("kspace", "comp_grad", "fmap_grad", "r2_grad"):
        assert np.array_equal(out[key], clean[key]), key
    mask = api.sampling_mask(s["acq_dims"][0], s["acq_dims"][1], acq).reshape(s["acq_dims"][1], -1)[:, 0]
    assert np.all(out["kspace"][..., ~mask.astype(bool), :] == 0)
    up, down = op.host_bytes()
    assert up == sum(a.nbytes for a in s["images"])
    rows = int(mask.sum()) * len(tes)
    kbytes = 3 * 2 * 4 * rows * s["acq_dims"][0] * 8
    assert down == kbytes + sum(clean[k].nbytes for k in ("comp_grad", "fmap_grad", "r2_grad"))


@pytest.mark.parametrize("nx,ny,pf,tes", [(16, 16, 0.625, (15.0, 35.0, 55.0)), (12, 12, 0.75, (20.0, 40.0))])
def test_coil_classes_odd_lines_and_dft_widths_match_the_oracle(nx, ny, pf, tes, gpu_ctx):
    """Eight ring coils run the coil-class kernels: an odd number of acquired lines per unit (the
    adjoint's last line chunk is half empty) and a 24-point sim width (no power of two: the
    x-stage is the DFT GEMM while the forward still accumulates coil classes)."""
    s = cases.series_case(nx=nx, ny=ny, nv=2, nz=2, ncomp=3)
    acq = Acquisition(n_coils=8, accel=2, partial_fourier=pf, pf_mode=PartialFourierMode.Scanner, t_line=0.5,
                      t_echo=30.0, ghost_offset=0.02)
    kw = dict(t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 2, s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=list(tes), grads=3, ctx=gpu_ctx, **kw)
    out = op.apply_host(None)
    want = oracle.series_forward(s["sim_dims"], s["acq_dims"], 2, s["images"], s["t2"], s["fmap"], acq,
                                 echo_times_ms=list(tes), **kw)
    assert rel_l2(out["kspace"], want) <= TOL
    adj = oracle.series_adjoint(s["sim_dims"], s["acq_dims"], 2, s["images"], s["t2"], s["fmap"], acq,
                                out["kspace"].astype(np.complex128), echo_times_ms=list(tes), **kw)
    for key in ("comp_grad", "fmap_grad", "r2_grad"):
        e = rel_l2(out[key], adj[key])
        assert e <= TOL, f"{key}: rel-L2 {e:.2e}"


@pytest.mark.parametrize("coils,eddy", [(8, False), (4, True)])
def test_128_point_rows_match_the_oracle(coils, eddy, gpu_ctx):
    """The bench's width (64 acquired columns on 128 sim columns): the x-stage runs as 16 x 8 FFTs
    (into coil-class rows for the 8-coil adjoint), with and without the eddy x/z factor."""
    s = cases.series_case(nx=64, ny=64, nv=1, nz=1, ncomp=3)
    acq = Acquisition(n_coils=coils, accel=2, partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner, t_line=0.5,
                      t_echo=30.0, ghost_offset=0.05, eddy_strength=2.0 if eddy else 0.0, eddy_quad=0.3)
    tes = [15.0, 35.0, 55.0]
    kw = dict(t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42,
              eddy_drive=[(0.5, -0.4, 0.7)] if eddy else None)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 1, s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=3, ctx=gpu_ctx, **kw)
    out = op.apply_host(None)
    want = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], s["fmap"], acq,
                                 echo_times_ms=tes, **kw)
    assert rel_l2(out["kspace"], want) <= TOL
    adj = oracle.series_adjoint(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], s["fmap"], acq,
                                out["kspace"].astype(np.complex128), echo_times_ms=tes, **kw)
    for key in ("comp_grad", "fmap_grad", "r2_grad"):
        e = rel_l2(out[key], adj[key])
        assert e <= TOL, f"{key}: rel-L2 {e:.2e}"


def test_96_lines_per_unit_match_the_oracle(gpu_ctx):
    """Full Fourier with R = 2 and three echoes: 96 lines per unit.  The class-mode y-adjoint then
    takes ~45 KB of dynamic shared memory next to its 3 KB static piece table, over 48 KB together,
    which its launch must opt into."""
    s = cases.series_case(nx=64, ny=64, nv=1, nz=1, ncomp=3)
    acq = Acquisition(n_coils=8, accel=2, partial_fourier=1.0, t_line=0.5, t_echo=30.0, ghost_offset=0.05)
    tes = [20.0, 55.0, 90.0]  # a full-Fourier train reads from 15.25 ms before its echo
    kw = dict(t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 1, s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=3, ctx=gpu_ctx, **kw)
    assert op.samples == 1 * 1 * 3 * 32 * 8 * 64
    out = op.apply_host(None)
    want = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], s["fmap"], acq,
                                 echo_times_ms=tes, **kw)
    assert rel_l2(out["kspace"], want) <= TOL
    adj = oracle.series_adjoint(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], s["fmap"], acq,
                                out["kspace"].astype(np.complex128), echo_times_ms=tes, **kw)
    for key in ("comp_grad", "fmap_grad", "r2_grad"):
        e = rel_l2(out[key], adj[key])
        assert e <= TOL, f"{key}: rel-L2 {e:.2e}"


@pytest.mark.parametrize("nx,coils", [(48, 8), (80, 4), (96, 8)])
def test_rows_of_32e_points_match_the_oracle(nx, coils, gpu_ctx):
    """Sim widths 96, 160 and 192 (32 E with E = 3, 5, 6 -- 192 is the differentiation config's
    grid): the warp FFT's E-point register DFT is a direct sum, the 96-point rows also go through
    the coil-class x-stages."""
    s = cases.series_case(nx=nx, ny=nx, nv=1, nz=1, ncomp=3)
    acq = Acquisition(n_coils=coils, accel=2, partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner, t_line=0.5,
                      t_echo=30.0, ghost_offset=0.05, eddy_strength=2.0, eddy_quad=0.3)
    tes = [15.0, 35.0]
    kw = dict(t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42, eddy_drive=[(0.5, -0.4, 0.7)])
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 1, s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=3, ctx=gpu_ctx, **kw)
    out = op.apply_host(None)
    want = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], s["fmap"], acq,
                                 echo_times_ms=tes, **kw)
    assert rel_l2(out["kspace"], want) <= TOL
    adj = oracle.series_adjoint(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], s["fmap"], acq,
                                out["kspace"].astype(np.complex128), echo_times_ms=tes, **kw)
    for key in ("comp_grad", "fmap_grad", "r2_grad"):
        e = rel_l2(out[key], adj[key])
        assert e <= TOL, f"{key}: rel-L2 {e:.2e}"


def test_compact_host_layout_is_the_acquired_rows(gpu_ctx):
    """The compact host call returns exactly the acquired rows of the zero-filled layout, and the
    byte query counts what each call moves."""
    s, acq, tes, kw = _setup(eddy=False, nv=3, nz=2, coils=4)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=3, ctx=gpu_ctx, **kw)
    full = op.apply_host(s["images"])
    first, step, count = op.acquired_rows()
    assert count > 0
    kshape = full["kspace"].shape[:4] + (count, full["kspace"].shape[5])
    comp = op.apply_host_compact(s["images"], {"kspace": np.zeros(kshape, np.complex64), "comp_grad": None,
                                               "fmap_grad": None, "r2_grad": None})
    rows = first + step * np.arange(count)
    assert np.array_equal(comp["kspace"], full["kspace"][:, :, :, :, rows, :])
    up, down_all = op.host_bytes_for()
    _, down_k = op.host_bytes_for(comp_grad=False, fmap_grad=False, r2_grad=False)
    assert down_k == comp["kspace"].nbytes and up == sum(a.nbytes for a in s["images"])
    assert down_all == down_k + full["comp_grad"].nbytes + full["fmap_grad"].nbytes + full["r2_grad"].nbytes
    op.close()
