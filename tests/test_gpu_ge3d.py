"""The device 3D gradient-echo train against the FP64 oracle (whose restatement is pinned by
tests/test_oracle_ge3d.py): echoes, class and voxel decay, excitation weights across partitions
and segments, an unused compartment, spikes and noise on per-echo streams, GRAPPA with and without
a reference volume, the phase model and reversed phase encoding; and the refusals.  FP32 device
arithmetic: rel-L2 <= 1e-5 against FP64."""
from __future__ import annotations

import numpy as np
import pytest

from cases3d import blobs
from mrsim_acq_b200 import kspace3d as K3
from mrsim_acq_b200.abi import MrsimError
from mrsim_acq_b200.api import KspaceWindow, PhaseModel, T2
from oracle import oracle as O
from test_oracle_ge3d import ge_acq, ge_train3, ge_volume, varying_fmap

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def case(name):
    nx = ny = 12
    nz, o, nv, ncomp = 4, 2, 2, 2
    snx, sny = nx * o, ny * o
    nvox = snx * sny * nz
    imgs = blobs(snx, sny, nz, nv, ncomp)
    per_vol = [[im[g::nv].copy() for im in imgs] for g in range(nv)]
    fmap = varying_fmap(snx, sny, nz)
    t2 = [T2.uniform(80.0), T2.uniform(120.0)]
    ti = None
    acq = ge_acq(2)
    tr = ge_train3(2, [12.0, 30.0])
    ro = K3.Ge3dReadout(2, 0.4)
    phase = PhaseModel.none()
    kys = 2
    w = lambda g: (lambda p, sy, c: 0.5 + 0.1 * p + 0.05 * sy + 0.2 * c + 0.03 * g)
    ref = None
    if name == "voxel":
        i = np.arange(nvox)
        t2 = [T2.of_map((60.0 + 40.0 * (i % snx) / snx).astype(np.float32)), T2.uniform(120.0)]
        ti = [T2.uniform(40.0), T2.of_map((50.0 + 20.0 * (i // (snx * sny)) / nz).astype(np.float32))]
    elif name == "unused":
        per_vol = [[v[0], None] for v in per_vol]
        w = lambda g: (lambda p, sy, c: 0.0 if c == 1 else 0.7 + 0.1 * p)
    elif name == "noise":
        acq = acq.replace(noise_variance=0.5, n_spikes=2)
    elif name == "grappa":
        acq = acq.replace(n_coils=4, accel=2, acs_lines=6, window=KspaceWindow.hann())
    elif name == "grappa_ref":
        acq = acq.replace(n_coils=4, accel=2, acs_lines=6)
        ref = ge_volume([im * 1.2 for im in per_vol[0]], nz, kys, lambda p, sy, c: 1.0)
    elif name == "phase":
        phase = PhaseModel.hbcd_like()
        acq = acq.replace(reverse_phase=True, ghost_offset=0.05)
        ro = K3.Ge3dReadout(2, 0.4, True)
    vol = lambda g: ge_volume(per_vol[g], nz, kys, w(g))
    return dict(args=([snx, sny, nz], [nx, ny, nz], nv, t2, fmap, ti, acq, tr, ro, vol), phase=phase, ref=ref)


CASES = ["class", "voxel", "unused", "noise", "grappa", "grappa_ref", "phase"]


@pytest.mark.parametrize("name", CASES)
def test_ge3d_matches_the_oracle(gpu_ctx, name):
    c = case(name)
    got = K3.simulate_acquisition_3d_ge(*c["args"], phase=c["phase"], seed=77, reference=c["ref"], ctx=gpu_ctx)
    want, _ = O.simulate_acquisition_3d_ge(*c["args"], phase=c["phase"], seed=77, reference=c["ref"])
    for e, (mag, ph) in enumerate(got):
        z = mag.astype(np.float64) * np.exp(1j * ph.astype(np.float64))
        nv = c["args"][2]
        assert rel_l2(z, want[e].T.ravel()) <= 1e-5, (name, e)


def test_ge3d_echo_zero_is_the_one_echo_call(gpu_ctx):
    c = case("noise")
    snx_sny_nz, acq_dims, nv, t2, fmap, ti, acq, tr, ro, vol = c["args"]
    two = K3.simulate_acquisition_3d_ge(snx_sny_nz, acq_dims, nv, t2, fmap, ti, acq, ge_train3(2, [12.0, 30.0]), ro, vol,
                                        seed=77, ctx=gpu_ctx)
    one = K3.simulate_acquisition_3d_ge(snx_sny_nz, acq_dims, nv, t2, fmap, ti, acq, ge_train3(2, [12.0]), ro, vol,
                                        seed=77, ctx=gpu_ctx)
    assert np.array_equal(two[0][0], one[0][0]) and np.array_equal(two[0][1], one[0][1])


def test_ge3d_refusals(gpu_ctx):
    c = case("class")
    sim, acqd, nv, t2, fmap, ti, acq, tr, ro, vol = c["args"]

    def run(acq=acq, tr=tr, ro=ro, vol=vol):
        return K3.simulate_acquisition_3d_ge(sim, acqd, nv, t2, fmap, ti, acq, tr, ro, vol, ctx=gpu_ctx)

    with pytest.raises(MrsimError, match="gradient-echo acquisition"):
        run(acq.replace(echo=0))
    with pytest.raises(MrsimError, match="partial Fourier is not available"):
        run(acq.replace(partial_fourier=0.75))
    with pytest.raises(MrsimError, match="eddy model"):
        run(acq.replace(eddy_strength=0.1))
    with pytest.raises(MrsimError, match="phase-encode sign"):
        run(ro=K3.Ge3dReadout(2, 0.4, True))
    with pytest.raises(MrsimError, match="increase strictly"):
        run(tr=ge_train3(2, [30.0, 12.0]))
    bad = lambda g: K3.GeVolume([vol(g).images[0], None], vol(g).weights)
    with pytest.raises(MrsimError, match="no image but a nonzero weight"):
        run(vol=bad)


@pytest.mark.parametrize("name", ["class", "voxel", "unused", "grappa"])
def test_ge3d_shot_images_match_the_oracle(gpu_ctx, name):
    """`GeVolume::shot_images`: volume 0's shot 1 sees shifted images, shots 2 and 3 scaled ones
    (a compartment the volume does not use has no set image either); the GRAPPA reference scan
    takes none."""
    c = case(name)
    sim, acqd, nv, t2, fmap, ti, acq, tr, ro, vol = c["args"]
    snx, sny, nz = sim

    def with_sets(g):
        v = vol(g)
        if g != 0:
            return v
        own = [None if im is None else np.asarray(im).reshape(nz, sny, snx) for im in v.images]
        a = [None if x is None else np.roll(x, 1, axis=1).ravel() * np.float32(1.2) for x in own]
        b = [None if x is None else x.ravel() * np.float32(0.7) for x in own]
        return K3.GeVolume(v.images, v.weights, [K3.ShotSet([1], a), K3.ShotSet([2, 3], b)])

    args = (sim, acqd, nv, t2, fmap, ti, acq, tr, ro, with_sets)
    got = K3.simulate_acquisition_3d_ge(*args, phase=c["phase"], seed=5, reference=c["ref"], ctx=gpu_ctx)
    want, _ = O.simulate_acquisition_3d_ge(*args, phase=c["phase"], seed=5, reference=c["ref"])
    for e, (mag, ph) in enumerate(got):
        z = mag.astype(np.float64) * np.exp(1j * ph.astype(np.float64))
        assert rel_l2(z, want[e].T.ravel()) <= 1e-5, (name, e)
