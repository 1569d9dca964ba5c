"""The device 3D GRASE acquisition against the FP64 oracle (whose restatement is pinned by
tests/test_oracle_3d.py): the observed 3D k-space and the reconstructed volumes across class and
voxel decay, EPG trains below 180 degrees, line weights, GRAPPA, spikes and noise, the phase model,
reversed phase encoding and partial Fourier; and the refusals with the reference's messages.
FP32 device arithmetic: rel-L2 <= 1e-5 against FP64."""
from __future__ import annotations

import math

import numpy as np
import pytest

from cases3d import blobs, grase, train
from mrsim_acq_b200 import kspace3d as K3
from mrsim_acq_b200.abi import MrsimError
from mrsim_acq_b200.api import Acquisition, EchoFormation, KspaceWindow, PartialFourierMode, PhaseModel, T2
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def case(name):
    nx, ny, nz, o, nv, ncomp = 16, 16, 6, 2, 2, 2
    snx, sny = nx * o, ny * o
    nvox = snx * sny * nz
    images = blobs(snx, sny, nz, nv, ncomp)
    i = np.arange(nvox)
    fmap = (30.0 * np.sin(TAU_ * (i % snx) / snx) + 10.0 * ((i // snx) % sny) / sny).astype(np.float32)
    t2 = [T2.uniform(80.0), T2.uniform(250.0)]
    t1 = [T2.uniform(1330.0), T2.uniform(4000.0)]
    ti = None
    lw = None
    acq = Acquisition(do_relaxation=True, do_distortions=True, n_coils=2, signal_scale=100.0)
    tr, ro = train(nz, 2, b=150.0), grase(2)
    phase = PhaseModel.none()
    if name == "voxel":
        t2 = [T2.of_map((60.0 + 40.0 * (i % snx) / snx).astype(np.float32)), T2.uniform(250.0)]
        ti = [T2.uniform(40.0), T2.of_map((50.0 + 20.0 * (i // (snx * sny)) / nz).astype(np.float32))]
    elif name == "weights":
        tab = K3.grase_lines(tr, ro, ny, nz)
        w = np.array([0.6 + 0.1 * ((g * 7 + s * 3 + c) % 5) for g in range(nv) for s in range(tab.n_shots)
                      for c in range(ncomp)])
        lw = K3.LineWeights(tab.n_shots, ncomp, w)
    elif name == "grappa":
        acq = acq.replace(n_coils=4, accel=2, acs_lines=8, window=KspaceWindow.hann())
    elif name == "noise":
        acq = acq.replace(noise_variance=4.0, n_spikes=3, spike_amplitude=2.0)
    elif name == "phase":
        phase = PhaseModel.hbcd_like()
        tr = train(nz, 1, K3.KzOrder.Linear, b=130.0)
        ro = grase(4)
    elif name == "reverse_pf":
        acq = acq.replace(reverse_phase=True, partial_fourier=0.75, pf_mode=int(PartialFourierMode.Contiguous),
                          ghost_offset=0.05)
        ro = grase(2, 0.5, True)
    elif name == "norelax":
        acq = acq.replace(do_relaxation=False)
        t1 = None
    return dict(sim=[snx, sny, nz], acqd=[nx, ny, nz], nv=nv, images=images, t2=t2, t1=t1, fmap=fmap, ti=ti, acq=acq,
                tr=tr, ro=ro, lw=lw, phase=phase)


TAU_ = 2.0 * math.pi
CASES = ["class", "voxel", "weights", "grappa", "noise", "phase", "reverse_pf", "norelax"]


@pytest.mark.parametrize("name", CASES)
def test_observed_kspace_matches_the_oracle(gpu_ctx, name):
    c = case(name)
    args = (c["sim"], c["acqd"], c["nv"], c["images"], c["t2"], c["t1"], c["fmap"], c["ti"], c["acq"], c["tr"], c["ro"])
    for g in range(c["nv"]):
        got = K3.kspace_3d_observed(*args, line_weights=c["lw"], phase=c["phase"], g=g, ctx=gpu_ctx)
        want = O.kspace_3d_observed(*args, line_weights=c["lw"], phase=c["phase"], g=g)
        assert rel_l2(got, want) <= 1e-5, (name, g)


@pytest.mark.parametrize("name", CASES)
def test_volumes_match_the_oracle(gpu_ctx, name):
    c = case(name)
    args = (c["sim"], c["acqd"], c["nv"], c["images"], c["t2"], c["t1"], c["fmap"], c["ti"], c["acq"], c["tr"], c["ro"])
    mag, ph = K3.simulate_acquisition_3d(*args, line_weights=c["lw"], phase=c["phase"], seed=42, ctx=gpu_ctx)
    vols, omag, oph = O.simulate_acquisition_3d(*args, line_weights=c["lw"], phase=c["phase"], seed=42)
    z = mag.astype(np.float64) * np.exp(1j * ph.astype(np.float64))
    want = vols.T.ravel()
    assert rel_l2(z, want) <= 1e-5, name
    assert np.abs(mag - omag).max() <= 1e-5 * np.abs(omag).max()


def test_grappa_calibration_scan(gpu_ctx):
    c = case("grappa")
    cal = [blobs(32, 32, 6, 1, 2)[k] * 1.3 for k in range(2)]
    args = (c["sim"], c["acqd"], c["nv"], c["images"], c["t2"], c["t1"], c["fmap"], c["ti"], c["acq"], c["tr"], c["ro"])
    mag, ph = K3.simulate_acquisition_3d(*args, seed=5, grappa_calibration=(cal, 77), ctx=gpu_ctx)
    vols, _, _ = O.simulate_acquisition_3d(*args, seed=5, grappa_calibration=(cal, 77))
    assert rel_l2(mag * np.exp(1j * ph.astype(np.float64)), vols.T.ravel()) <= 1e-5


def test_refusals(gpu_ctx):
    c = case("class")
    base = (c["sim"], c["acqd"], c["nv"], c["images"], c["t2"])

    def run(acq=None, t1=c["t1"], tr=c["tr"], ro=c["ro"]):
        return K3.simulate_acquisition_3d(*base, t1, c["fmap"], None, acq or c["acq"], tr, ro, ctx=gpu_ctx)

    with pytest.raises(MrsimError, match="needs T1"):
        run(t1=None)
    with pytest.raises(MrsimError, match="Scanner partial Fourier"):
        run(c["acq"].replace(partial_fourier=0.75, pf_mode=int(PartialFourierMode.Scanner)))
    with pytest.raises(MrsimError, match="eddy model"):
        run(c["acq"].replace(eddy_strength=0.1))
    with pytest.raises(MrsimError, match="spin-echo trains"):
        run(c["acq"].replace(echo=int(EchoFormation.Gradient)))
    with pytest.raises(MrsimError, match="phase-encode sign"):
        run(ro=grase(2, 0.5, True))
    with pytest.raises(MrsimError, match="echo train length"):
        run(tr=K3.EchoTrain(etl=5, esp_ms=20.0, refocusing_deg=150.0, kz_segments=2))


def moved_sets(images, nv, snx, sny, nz, g):
    """Two shot sets of volume g: shot 1 sees the volume shifted by a voxel along x and scaled,
    shots 0 and 1 see it scaled the other way (shot 1 takes the first set)."""
    own = [im[g::nv].reshape(nz, sny, snx) for im in images]
    a = [np.roll(v, 1, axis=2).ravel() * np.float32(1.1) for v in own]
    b = [v.ravel() * np.float32(0.8) for v in own]
    return [K3.ShotSet([1], a), K3.ShotSet([0, 1], b)]


@pytest.mark.parametrize("name", ["class", "voxel", "grappa", "noise"])
def test_shot_images_match_the_oracle(gpu_ctx, name):
    """Per-shot images (`ShotSet`): volume 0 with two overlapping sets, volume 1 with none; the
    observed k-space and the reconstructed volumes against the oracle."""
    c = case(name)
    snx, sny, nz = c["sim"]
    sets = [moved_sets(c["images"], c["nv"], snx, sny, nz, 0), []]
    args = (c["sim"], c["acqd"], c["nv"], c["images"], c["t2"], c["t1"], c["fmap"], c["ti"], c["acq"], c["tr"], c["ro"])
    for g in range(c["nv"]):
        got = K3.kspace_3d_observed(*args, line_weights=c["lw"], phase=c["phase"], g=g, ctx=gpu_ctx,
                                    shot_images=sets)
        want = O.kspace_3d_observed(*args, line_weights=c["lw"], phase=c["phase"], g=g, shot_images=sets)
        assert rel_l2(got, want) <= 1e-5, (name, g)
    mag, ph = K3.simulate_acquisition_3d(*args, line_weights=c["lw"], phase=c["phase"], seed=11, ctx=gpu_ctx,
                                         shot_images=sets)
    vols, _, _ = O.simulate_acquisition_3d(*args, line_weights=c["lw"], phase=c["phase"], seed=11, shot_images=sets)
    z = mag.astype(np.float64) * np.exp(1j * ph.astype(np.float64))
    assert rel_l2(z, vols.T.ravel()) <= 1e-5, name


def test_shot_images_double_exactly_their_lines_on_the_device(gpu_ctx):
    """Doubled images for shot 1 double exactly (bit for bit: a power-of-two scale commutes with
    every rounding) the device's lines of shot 1 and leave the others unchanged."""
    c = case("class")
    snx, sny, nz = c["sim"]
    args = (c["sim"], c["acqd"], c["nv"], c["images"], c["t2"], c["t1"], c["fmap"], c["ti"], c["acq"], c["tr"], c["ro"])
    full = K3.kspace_3d_observed(*args, phase=c["phase"], g=0, ctx=gpu_ctx)
    doubled = [2.0 * im[0::c["nv"]] for im in c["images"]]
    moved = K3.kspace_3d_observed(*args, phase=c["phase"], g=0, ctx=gpu_ctx,
                                  shot_images=[[K3.ShotSet([1], doubled)], []])
    shot = K3.grase_lines(c["tr"], c["ro"], c["acqd"][1], nz).shot.reshape(nz, c["acqd"][1])
    sel = np.broadcast_to((shot == 1)[None, :, :, None], full.shape)
    assert np.array_equal(moved[sel], 2.0 * full[sel])
    assert np.array_equal(moved[~sel], full[~sel])
    with pytest.raises(MrsimError, match="a shot index beyond the train's"):
        K3.kspace_3d_observed(*args, phase=c["phase"], g=0, ctx=gpu_ctx, shot_images=[[K3.ShotSet([99], doubled)], []])
