"""The differentiation workload on the GPU operator: scan 96x96 on a 192x192 grid, 8 coils.  The loss
is L = ||A(m, fmap, R2) - s_obs||^2 with s_obs simulated by the FP64 oracle from a perturbed ground
truth (the fieldmap plus a seeded smooth field of 20 Hz RMS, R2 of one compartment +-10 %).  Its
VJPs are checked against central differences of the oracle's loss at 64 seeded voxels, and the
fieldmap gradient drives 200 steps of gradient descent through `EpiOperator.set_fieldmap`.  (The
workload has 16 slices; one and two slices keep the FP64 differences to seconds.)"""
import multiprocessing

import numpy as np
import pytest

from mrsim_acq_b200 import api
from mrsim_acq_b200.api import T2, Acquisition, PartialFourierMode, PhaseModel
from oracle import oracle
from tests import cases

pytestmark = pytest.mark.gpu


def smooth_field(rng, shape, sigma_px, rms):
    """A seeded Gaussian random field: white noise low-passed by a Gaussian of sigma_px pixels per
    slice, scaled to the given RMS."""
    nz, ny, nx = shape
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.fftfreq(nx)[None, :]
    g = np.exp(-2.0 * (np.pi * sigma_px) ** 2 * (kx ** 2 + ky ** 2))
    out = np.stack([np.real(np.fft.ifft2(np.fft.fft2(rng.standard_normal((ny, nx))) * g)) for _ in range(nz)])
    return out * (rms / np.sqrt(np.mean(out ** 2)))


def _case(nz):
    s = cases.series_case(nx=96, ny=96, nv=1, nz=nz, ncomp=2)
    acq = Acquisition(n_coils=8, accel=2, partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner, t_line=0.5,
                      t_echo=30.0)
    kw = dict(t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42)
    return s, acq, [30.0], kw


_WORKER = {}


def _worker_init(s, acq, tes, kw, sobs):
    _WORKER.update(s=s, acq=acq, tes=tes, kw=kw, sobs=sobs)


def _oracle_loss(args):
    """L = sum |A_FP64(images, t2, fmap) - s_obs|^2 (runs in a spawned worker)."""
    t2, fmap = args
    w = _WORKER
    k = oracle.series_forward(w["s"]["sim_dims"], w["s"]["acq_dims"], 1, w["s"]["images"], t2, fmap, w["acq"],
                              echo_times_ms=w["tes"], **w["kw"])
    return float(np.sum(np.abs(k - w["sobs"]) ** 2))


def test_vjps_match_central_differences_at_64_voxels(gpu_ctx):
    """dL/dfmap and dL/dR2 (compartment 0, a T2 map) of the GPU adjoint against central
    differences of the FP64 oracle's loss (h = 1e-3 Hz; a relative 1e-3 step in R2) at 64 seeded
    voxels inside the object."""
    s, acq, tes, kw = _case(1)
    snx, sny, nz = s["sim_dims"]
    rng = np.random.default_rng(21)
    r2_0 = 1.0 / 80.0
    t2_model = [T2.of_map(np.full(snx * sny, 80.0, np.float32)), s["t2"][1]]
    r2_true = r2_0 * (1.0 + 0.1 * np.clip(smooth_field(rng, (1, sny, snx), 10.0, 0.6), -1, 1)).ravel()
    t2_true = [T2.of_map((1.0 / r2_true).astype(np.float32)), s["t2"][1]]
    f0 = s["fmap"].astype(np.float32)
    f_true = (f0 + smooth_field(rng, (1, sny, snx), 8.0, 20.0).ravel()).astype(np.float32)
    sobs = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, s["images"], t2_true, f_true, acq,
                                 echo_times_ms=tes, **kw)

    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 1, t2_model, f0, acq, images=s["images"],
                         echo_times_ms=tes, grads=3, ctx=gpu_ctx, **kw)
    shp = op.shapes()
    k = op.apply_host(None, {"kspace": np.zeros(shp["kspace"], np.complex64), "comp_grad": None,
                             "fmap_grad": None, "r2_grad": None})["kspace"]
    g = op.adjoint_host((k - sobs).astype(np.complex64))
    op.close()
    gf = g["fmap_grad"].reshape(-1).astype(np.float64)
    gr = g["r2_grad"].reshape(2, -1)[0].astype(np.float64)

    mag = sum(np.asarray(a, np.float64) for a in s["images"])
    vox = rng.choice(np.flatnonzero(mag > 0.3 * mag.max()), 64, replace=False)
    h = 1e-3
    jobs = []
    for v in vox:
        for sgn in (1.0, -1.0):
            f = f0.copy()
            f[v] = np.float32(f0[v] + sgn * h)
            jobs.append((t2_model, f))
    for v in vox:
        for sgn in (1.0, -1.0):
            m = np.full(snx * sny, 80.0, np.float32)
            m[v] = np.float32(1.0 / (r2_0 * (1.0 + sgn * h)))
            jobs.append(([T2.of_map(m), s["t2"][1]], f0))
    with multiprocessing.get_context("spawn").Pool(min(16, multiprocessing.cpu_count()), _worker_init,
                                                   (s, acq, tes, kw, sobs)) as pool:
        L = np.array(pool.map(_oracle_loss, jobs))
    n = len(vox)
    for i, v in enumerate(vox):
        df = float(np.float32(f0[v] + h)) - float(np.float32(f0[v] - h))
        fd = (L[2 * i] - L[2 * i + 1]) / df
        assert abs(gf[v] - fd) <= 2e-3 * max(abs(fd), 1e-3 * np.abs(gf).max()), ("fmap", v, gf[v], fd)
        r2p = 1.0 / float(np.float32(1.0 / (r2_0 * (1.0 + h))))
        r2m = 1.0 / float(np.float32(1.0 / (r2_0 * (1.0 - h))))
        fd = (L[2 * n + 2 * i] - L[2 * n + 2 * i + 1]) / (r2p - r2m)
        assert abs(gr[v] - fd) <= 2e-3 * max(abs(fd), 1e-3 * np.abs(gr).max()), ("r2", v, gr[v], fd)


def test_fieldmap_descent_on_the_differentiation_grid(gpu_ctx):
    """200 steps of gradient descent on the fieldmap (step halved on a rise, grown by 1.3 on a
    fall) from the unperturbed map toward the perturbed truth, with R2 left at its unperturbed
    value: the loss falls by at least 20x and the fieldmap error inside the object by at least half."""
    s, acq, tes, kw = _case(2)
    snx, sny, nz = s["sim_dims"]
    rng = np.random.default_rng(7)
    f0 = s["fmap"].astype(np.float32)
    f_true = (f0 + smooth_field(rng, (nz, sny, snx), 8.0, 20.0).ravel()).astype(np.float32)
    t2_true = [T2.uniform(80.0 * 1.1), T2.uniform(250.0 * 0.9)]
    sobs = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, s["images"], t2_true, f_true, acq,
                                 echo_times_ms=tes, **kw).astype(np.complex64)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 1, s["t2"], f0, acq, images=s["images"],
                         echo_times_ms=tes, grads=1, ctx=gpu_ctx, **kw)
    shp = op.shapes()
    kout = {"kspace": np.zeros(shp["kspace"], np.complex64), "comp_grad": None, "fmap_grad": None, "r2_grad": None}

    def loss_grad(f):
        op.set_fieldmap(f)
        r = op.apply_host(None, kout)["kspace"] - sobs
        g = op.adjoint_host(r)["fmap_grad"].reshape(-1).astype(np.float64)
        return float(np.sum(np.abs(r.astype(np.complex128)) ** 2)), g

    mag = sum(np.asarray(a, np.float64) for a in s["images"])
    inside = mag > 0.3 * mag.max()
    f = f0.copy()
    L, g = loss_grad(f)
    L0, e0 = L, float(np.sqrt(np.mean((f - f_true)[inside] ** 2)))
    alpha = 1.0  # Hz: the largest change of one step
    for _ in range(200):
        while True:
            fn = (f - (alpha / np.abs(g).max()) * g).astype(np.float32)
            Ln, gn = loss_grad(fn)
            if Ln < L or alpha < 1e-6:
                break
            alpha *= 0.5
        if Ln < L:
            f, L, g = fn, Ln, gn
            alpha *= 1.3
    op.close()
    e1 = float(np.sqrt(np.mean((f - f_true)[inside] ** 2)))
    print(f"fieldmap descent: loss {L0:.4g} -> {L:.4g} ({L / L0:.3g}), error {e0:.3g} -> {e1:.3g} Hz")
    assert L <= L0 / 20, (L0, L)
    assert e1 <= 0.5 * e0, (e0, e1)
