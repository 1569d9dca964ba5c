"""GPU parity at the geometries and coil counts of every benchmark configuration.

Each case runs the CUDA path at a configuration's own shape and checks it against the FP64
oracle (relative L2 <= 1e-5):

- precision at scale: scan 128x128 on a 256x256 grid, 32 ring coils, 3 compartments (the per-coil
  kernels: a ring of 32 takes no coil-class path), two slices of one volume;
- a 16-coil ring on the 64x64 / 128x128 series grid with three echoes (9 distinct ey classes);
- the differentiation workload at its full 16 slices (96x96 on 192x192, 8 coils): forward and
  adjoint, and the complex-image VJP against central differences of the FP64 loss at 8 voxels;
- the stack-of-spirals in-plane forward at its full trajectory (32 interleaves x 2048 samples,
  4 us dwell, 8.192 ms readout, +-80 Hz fieldmap, 64x64 on a 128x128 grid, certified time
  segmentation) for two coils of the 8-coil ring; the FP64 exact sum is evaluated on a stated
  subset (every 16th sample: 4096 samples across all interleaves and readout times), the device
  computes all 65,536.
"""

import numpy as np
import pytest

from mrsim_acq_b200 import api
from mrsim_acq_b200 import spiral as S
from mrsim_acq_b200.api import T2, Acquisition, PartialFourierMode, PhaseModel, SliceInput
from oracle import oracle
from tests import cases

pytestmark = pytest.mark.gpu
TOL = 1e-5


def rel_l2(a, b):
    n = np.linalg.norm(np.ravel(b))
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / (n if n > 0 else 1.0)


def _pair(s, acq, tes, kw, ctx, grads=3):
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=grads, ctx=ctx, **kw)
    out = op.apply_host(None)
    op.close()
    want = oracle.series_forward(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"], acq,
                                 echo_times_ms=tes, **kw)
    assert out["kspace"].shape == want.shape
    e = rel_l2(out["kspace"], want)
    assert e <= TOL, f"forward rel-L2 {e:.2e}"
    adj = oracle.series_adjoint(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"], acq,
                                out["kspace"].astype(np.complex128), echo_times_ms=tes, **kw)
    errs = {"kspace": e}
    for key in ("comp_grad", "fmap_grad", "r2_grad")[:grads]:
        e = rel_l2(out[key], adj[key])
        errs[key] = e
        assert e <= TOL, f"{key}: rel-L2 {e:.2e}"
    return errs


def test_precision_at_scale_geometry_32_coils(gpu_ctx):
    """128x128 on 256x256, 32 ring coils, 3 compartments, all 128 lines (a 64 ms train), TE 40 ms."""
    s = cases.series_case(nx=128, ny=128, nz=2, o=2, nv=1, ncomp=3)
    acq = Acquisition(n_coils=32, t_line=0.5, t_echo=40.0, ghost_offset=0.02)
    kw = dict(t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42)
    print("32 coils, 256 grid:", _pair(s, acq, [40.0], kw, gpu_ctx))


def test_sixteen_coil_ring_on_the_series_grid(gpu_ctx):
    """64x64 on 128x128, 16 ring coils, GRAPPA R=2 sampling, PF 6/8 Scanner, echoes 15/35/55 ms."""
    s = cases.series_case(nx=64, ny=64, nz=2, o=2, nv=1, ncomp=3)
    acq = Acquisition(n_coils=16, accel=2, partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner, t_line=0.5,
                      t_echo=30.0, ghost_offset=0.05)
    kw = dict(t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42)
    print("16 coils:", _pair(s, acq, [15.0, 35.0, 55.0], kw, gpu_ctx))


def _diff_case(nz):
    s = cases.series_case(nx=96, ny=96, nv=1, nz=nz, ncomp=2)
    acq = Acquisition(n_coils=8, accel=2, partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner, t_line=0.5,
                      t_echo=30.0)
    kw = dict(t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42)
    return s, acq, [30.0], kw


def test_differentiation_workload_all_16_slices(gpu_ctx):
    s, acq, tes, kw = _diff_case(16)
    print("differentiation, 16 slices:", _pair(s, acq, tes, kw, gpu_ctx))


def test_complex_image_vjp_matches_central_differences(gpu_ctx):
    """dL/dRe m + i dL/dIm m = 2 A^H (A m - s_obs) at 8 seeded voxels of the differentiation grid
    (one slice), against central differences of the FP64 loss with h = 1e-3: along Re m by
    perturbing the image itself, along Im m with the oracle's response to a unit impulse
    (L(m +- i h e_v) = ||r +- i h A e_v||^2, A linear in m)."""
    s, acq, tes, kw = _diff_case(1)
    snx, sny, _ = s["sim_dims"]
    rng = np.random.default_rng(5)
    sobs = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, [0.9 * im for im in s["images"]], s["t2"],
                                 s["fmap"] + 3.0, acq, echo_times_ms=tes, **kw)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 1, s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=tes, grads=1, ctx=gpu_ctx, **kw)
    k = op.apply_host(None)["kspace"]
    g = op.adjoint_host((k - sobs).astype(np.complex64))["comp_grad"].reshape(2, sny * snx)
    op.close()
    r = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], s["fmap"], acq,
                              echo_times_ms=tes, **kw) - sobs
    mag = np.asarray(s["images"][0], np.float64)
    h = 1e-3
    for v in rng.choice(np.flatnonzero(mag > 0.2 * mag.max()), 8, replace=False):
        c = int(v % 2)
        ims_p = [np.array(im, np.float64) for im in s["images"]]
        ims_m = [np.array(im, np.float64) for im in s["images"]]
        ims_p[c][v] += h
        ims_m[c][v] -= h
        lp = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, [a.astype(np.float32) for a in ims_p], s["t2"],
                                   s["fmap"], acq, echo_times_ms=tes, **kw) - sobs
        lm = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, [a.astype(np.float32) for a in ims_m], s["t2"],
                                   s["fmap"], acq, echo_times_ms=tes, **kw) - sobs
        step = float(np.float32(s["images"][c][v] + h)) - float(np.float32(s["images"][c][v] - h))
        fd_re = (np.sum(np.abs(lp) ** 2) - np.sum(np.abs(lm) ** 2)) / step
        imp = [np.zeros(snx * sny, np.float32) for _ in s["images"]]
        imp[c][v] = 1.0
        a = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, imp, s["t2"], s["fmap"], acq, echo_times_ms=tes,
                                  **kw)
        fd_im = (np.sum(np.abs(r + 1j * h * a) ** 2) - np.sum(np.abs(r - 1j * h * a) ** 2)) / (2 * h)
        got = 2.0 * complex(g[c][v])
        scale = 2.0 * np.abs(g).max()
        assert abs(got.real - fd_re) <= 2e-3 * max(abs(fd_re), 1e-3 * scale), (v, got, fd_re)
        assert abs(got.imag - fd_im) <= 2e-3 * max(abs(fd_im), 1e-3 * scale), (v, got, fd_im)


def test_stack_of_spirals_in_plane_forward_at_full_trajectory(gpu_ctx):
    n, o = 64, 2
    sg = n * o
    tr = S.spiral_trajectory(n, n, 32, 8.192, 0.004, 1.2)
    ns = len(tr.tau_ms)
    assert ns == 2048 and len(tr.k.reshape(-1, 2)) == 32 * 2048
    k = tr.k.reshape(-1, 2)
    tau_idx = np.arange(len(k)) % ns
    x, y = np.meshgrid(np.arange(sg), np.arange(sg))
    u, v = (x + 0.5) / sg, (y + 0.5) / sg
    blob = lambda cx, cy, w: np.exp(-((u - cx) ** 2 + (v - cy) ** 2) / (2 * w * w))
    img = (blob(0.42, 0.47, 0.12) + 0.6 * blob(0.6, 0.58, 0.07)).astype(np.float32).ravel()
    fmap = (80.0 * blob(0.35, 0.4, 0.15) - 80.0 * blob(0.66, 0.62, 0.12)).astype(np.float32).ravel()
    inp = SliceInput(compartments=[img], t2=[T2.uniform(80.0)], t_inhom=[T2.uniform(40.0)], fmap=fmap, sim=(sg, sg),
                     acq_matrix=(n, n), phase0=(0.4 * u - 0.7 * v * v).ravel())
    acq = Acquisition(do_relaxation=True, do_distortions=True, noise_variance=0.0, n_spikes=0, n_coils=8,
                      signal_scale=1.0)
    rect = S.RateRect((0.0, 0.0), (float(fmap.min()), float(fmap.max())))
    sub = np.arange(0, len(k), 16)
    taus = tr.tau_ms[tau_idx]
    for q in (0, 3):
        got, info = S.spiral_segmented_forward(inp, acq, q, 8, k, tau_idx, tr.tau_ms, 8.192, rect, None, False,
                                               ctx=gpu_ctx)
        assert info["bound"] < 1e-7
        got = got * np.exp(-taus / 80.0 - taus / 40.0)
        want = oracle.spiral_kspace_exact(inp, acq, q, 8, k[sub], taus[sub], None)
        e = rel_l2(got[sub], want)
        print(f"spiral coil {q}: L = {info['l']}, rel-L2 on {len(sub)} samples {e:.2e}")
        assert e <= TOL
        assert np.abs(got[sub] - want).max() <= 5e-6 * np.abs(want).max()
