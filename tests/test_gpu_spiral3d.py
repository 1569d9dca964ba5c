"""The device stack-of-spirals acquisition against the FP64 oracle (exact in-plane sums; its
restatement is pinned by tests/test_oracle_spiral3d.py).  The device uses the certified
time-segmented forward (1e-7) in FP32 and the FP64 reconstruction: rel-L2 <= 1e-5 on the samples
before noise and on the reconstructed volumes, across class and voxel decay, line weights, noise,
coil rings along z, partial Fourier (zero fill and POCS) and kz acceleration; and the refusals."""
from __future__ import annotations

import numpy as np
import pytest

from cases3d import blobs, train
from mrsim_acq_b200 import kspace3d as K3
from mrsim_acq_b200.abi import MrsimError
from mrsim_acq_b200.api import Acquisition, KspaceWindow, PhaseModel, T2
from oracle import oracle as O
from test_oracle_spiral3d import kz_train, spiral_fmap, spiral_ro

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def case(name):
    n, nz, o, ncomp, nv = 16, 4, 2, 2, 2
    s = n * o
    nvox = s * s * nz
    images = blobs(s, s, nz, nv, ncomp)
    fmap = spiral_fmap(s, s, nz)
    t2 = [T2.uniform(80.0), T2.uniform(120.0)]
    t1 = [T2.uniform(1300.0), T2.uniform(1600.0)]
    ti = None
    acq = Acquisition(do_relaxation=True, do_distortions=True, n_coils=2, signal_scale=100.0)
    tr = train(nz, 2, esp_ms=12.0, b=130.0)
    ro = spiral_ro()
    lw, kzo, phase = None, None, PhaseModel.none()
    if name == "norelax":
        acq = acq.replace(do_relaxation=False)
        t1 = None
        tr = train(nz, 1, esp_ms=12.0)
    elif name == "voxel":
        i = np.arange(nvox)
        t2 = [T2.of_map((60.0 + 40.0 * (i % s) / s).astype(np.float32)), T2.uniform(120.0)]
        ti = [T2.uniform(40.0), T2.of_map((50.0 + 20.0 * (i // (s * s)) / nz).astype(np.float32))]
    elif name == "weights":
        tab = K3.spiral_lines(tr, ro, n, n, nz)
        w = np.array([0.6 + 0.1 * ((g * 7 + sh * 3 + c) % 5) for g in range(nv) for sh in range(tab.n_shots)
                      for c in range(ncomp)])
        lw = K3.LineWeights(tab.n_shots, ncomp, w)
    elif name == "noise":
        acq = acq.replace(noise_variance=9.0, window=KspaceWindow.hann())
    elif name == "rings":
        acq = acq.replace(n_coils=4)
        kzo = K3.KzOptions(coil_rows=2)
        phase = PhaseModel.hbcd_like()
    return dict(sim=[s, s, nz], acqd=[n, n, nz], nv=nv, images=images, t2=t2, t1=t1, fmap=fmap, ti=ti, acq=acq, tr=tr,
                ro=ro, lw=lw, kzo=kzo, phase=phase)


CASES = ["norelax", "class", "voxel", "weights", "noise", "rings"]


@pytest.mark.parametrize("name", CASES)
def test_samples_match_the_oracle(gpu_ctx, name):
    c = case(name)
    args = (c["sim"], c["acqd"], c["nv"], c["images"], c["t2"], c["t1"], c["fmap"], c["ti"], c["acq"], c["tr"], c["ro"])
    got = K3.spiral_samples_3d(*args, line_weights=c["lw"], phase=c["phase"], g=1, kz_opts=c["kzo"], ctx=gpu_ctx)
    want = O.spiral_samples_3d(*args, line_weights=c["lw"], phase=c["phase"], g=1, kz_opts=c["kzo"])
    assert rel_l2(got, want) <= 1e-5, name


@pytest.mark.parametrize("name", CASES)
def test_volumes_match_the_oracle(gpu_ctx, name):
    c = case(name)
    args = (c["sim"], c["acqd"], c["nv"], c["images"], c["t2"], c["t1"], c["fmap"], c["ti"], c["acq"], c["tr"], c["ro"])
    mag, ph = K3.simulate_acquisition_3d(*args, line_weights=c["lw"], phase=c["phase"], seed=7, kz_opts=c["kzo"],
                                         ctx=gpu_ctx)
    vols, omag, _ = O.simulate_acquisition_3d_spiral(*args, line_weights=c["lw"], phase=c["phase"], seed=7,
                                                     kz_opts=c["kzo"])
    z = mag.astype(np.float64) * np.exp(1j * ph.astype(np.float64))
    assert rel_l2(z, vols.T.ravel()) <= 1e-5, name


def _kz_case(kz, rows, pocs=False, noise=0.0):
    n, nz, o, ncomp, nv = 16, 12, 2, 2, 1
    s = n * o
    images = blobs(s, s, nz, nv, ncomp)
    nplane = s * s
    for ci, im in enumerate(images):
        im *= (1.0 - 0.7 * ci)
        z = (np.arange(len(im)) // nv) // nplane
        im *= np.array([1.0, 0.3, 1.4, 0.8, 0.1, 1.2, 0.6, 1.5, 0.2, 0.9, 1.3, 0.5], np.float32)[z % 12]
    cal = blobs(s, s, nz, 1, ncomp)
    fmap = spiral_fmap(s, s, nz)
    t2 = [T2.uniform(80.0), T2.uniform(110.0)]
    acq = Acquisition(do_relaxation=False, do_distortions=True, n_coils=rows, noise_variance=noise, signal_scale=100.0)
    kzo = K3.KzOptions(coil_rows=rows, calibration_images=cal, calibration_seed=1, pocs=pocs)
    return ([s, s, nz], [n, n, nz], nv, images, t2, None, fmap, None, acq, kz_train(nz, kz),
            spiral_ro(kz.partial_fourier, kz.accel)), kzo


@pytest.mark.parametrize("pf,accel,rows,pocs,noise", [(1.0, 2, 4, False, 0.0), (0.75, 2, 4, False, 4.0),
                                                       (0.75, 1, 2, True, 0.0), (1.0, 3, 6, False, 0.0)])
def test_kz_acceleration_and_pocs_match_the_oracle(gpu_ctx, pf, accel, rows, pocs, noise):
    args, kzo = _kz_case(K3.KzSampling(pf, accel), rows, pocs, noise)
    mag, ph = K3.simulate_acquisition_3d(*args, phase=PhaseModel.none(), seed=3, kz_opts=kzo, ctx=gpu_ctx)
    vols, _, _ = O.simulate_acquisition_3d_spiral(*args, phase=PhaseModel.none(), seed=3, kz_opts=kzo)
    z = mag.astype(np.float64) * np.exp(1j * ph.astype(np.float64))
    assert rel_l2(z, vols.T.ravel()) <= 1e-5


def test_refusals(gpu_ctx):
    c = case("class")
    base = (c["sim"], c["acqd"], c["nv"], c["images"], c["t2"], c["t1"], c["fmap"], None)

    def run(acq, ro=c["ro"], kzo=None, tr=c["tr"]):
        return K3.simulate_acquisition_3d(*base, acq, tr, ro, kz_opts=kzo, ctx=gpu_ctx)

    a = c["acq"]
    with pytest.raises(MrsimError, match="GRAPPA has no spiral meaning"):
        run(a.replace(accel=2))
    with pytest.raises(MrsimError, match="in-plane partial Fourier"):
        run(a.replace(partial_fourier=0.75))
    with pytest.raises(MrsimError, match="Nyquist ghosting"):
        run(a.replace(ghost_offset=0.05))
    with pytest.raises(MrsimError, match="spikes have no spiral meaning"):
        run(a.replace(n_spikes=2))
    with pytest.raises(MrsimError, match="do not divide into 3 rings"):
        run(a, kzo=K3.KzOptions(coil_rows=3))
    kz = K3.KzSampling(1.0, 2)
    with pytest.raises(MrsimError, match="needs its KzOptions"):
        run(a, ro=spiral_ro(1.0, 2), tr=kz_train(4, kz, 130.0))
    with pytest.raises(MrsimError, match="at least as many coil rings"):
        run(a, ro=spiral_ro(1.0, 2), tr=kz_train(4, kz, 130.0), kzo=K3.KzOptions(coil_rows=1, calibration_images=c["images"]))


@pytest.mark.parametrize("name", ["class", "voxel", "rings"])
def test_spiral_shot_images_match_the_oracle(gpu_ctx, name):
    """Per-shot images on the stack of spirals: volume 1's shot 1 sees shifted images, shots 2 and
    3 scaled ones; samples and volumes against the oracle."""
    c = case(name)
    s, _, nz = c["sim"]
    nv = c["nv"]

    def sets(g):
        own = [im[g::nv].reshape(nz, s, s) for im in c["images"]]
        return [K3.ShotSet([1], [np.roll(x, 1, axis=2).ravel() * np.float32(1.1) for x in own]),
                K3.ShotSet([2, 3], [x.ravel() * np.float32(0.75) for x in own])]

    si = [[], sets(1)]
    args = (c["sim"], c["acqd"], nv, c["images"], c["t2"], c["t1"], c["fmap"], c["ti"], c["acq"], c["tr"], c["ro"])
    got = K3.spiral_samples_3d(*args, line_weights=c["lw"], phase=c["phase"], g=1, kz_opts=c["kzo"], ctx=gpu_ctx,
                               shot_images=si)
    want = O.spiral_samples_3d(*args, line_weights=c["lw"], phase=c["phase"], g=1, kz_opts=c["kzo"], shot_images=si)
    assert rel_l2(got, want) <= 1e-5, name
    mag, ph = K3.simulate_acquisition_3d(*args, line_weights=c["lw"], phase=c["phase"], seed=7, kz_opts=c["kzo"],
                                         ctx=gpu_ctx, shot_images=si)
    vols, _, _ = O.simulate_acquisition_3d_spiral(*args, line_weights=c["lw"], phase=c["phase"], seed=7,
                                                  kz_opts=c["kzo"], shot_images=si)
    z = mag.astype(np.float64) * np.exp(1j * ph.astype(np.float64))
    assert rel_l2(z, vols.T.ravel()) <= 1e-5, name
