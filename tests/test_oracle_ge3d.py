"""Pins of the oracle's 3D gradient-echo restatement (CPU), from the reference's own tests
(kspace3d.rs:2500-2660): each echo equals a per-slice reference built from the 2D forward with
gradient-echo formation, a z-DFT with the partition weights and the 2D reconstruction (class and
voxel modes, 1 and 3 coils); weights varying across partitions blur through-plane; and the GE
line table against the product's."""
from __future__ import annotations

import math

import numpy as np
import pytest

from cases3d import blobs
from mrsim_acq_b200 import kspace3d as K3
from mrsim_acq_b200.api import Acquisition, EchoFormation, LineTiming, PhaseModel, SliceInput, T2
from oracle import oracle as O

TAU = 2.0 * math.pi


def varying_fmap(snx, sny, nz):
    v = np.arange(snx * sny * nz)
    x, y, z = v % snx, (v // snx) % sny, v // (snx * sny)
    fx, fy = x / snx - 0.5, y / sny - 0.5
    return (25.0 * fx - 10.0 * fy + 15.0 * np.exp(-(fx * fx + fy * fy) / 0.02) + 2.0 * z).astype(np.float32)


def ge_train3(kz_segments, tes):
    return K3.ExcitationTrain(kz_segments, K3.KzOrder.Linear, 60.0, list(tes), 2.0)


def ge_acq(n_coils):
    return Acquisition(echo=EchoFormation.Gradient, n_coils=n_coils, signal_scale=100.0, t_inhom=45.0)


def ge_volume(images, nz, kys, w):
    ncomp = len(images)
    weights = np.array([w(p, sy, c) for p in range(nz) for sy in range(kys) for c in range(ncomp)])
    return K3.GeVolume(list(images), weights)


def ge_reference(img, t2, ti, fmap, acq, te, ro, dims, o, w):
    """kspace3d.rs `ge_reference`, restated over the oracle's 2D forward and reconstruction."""
    nx, ny, nz = dims
    snx, sny = nx * o, ny * o
    nplane = snx * sny
    epi = ny // ro.ky_segments
    t = np.zeros(ny)
    pol = np.zeros(ny, np.int8)
    for ky in range(ny):
        j = ky // ro.ky_segments
        a = j if ro.reverse_phase else epi - 1 - j
        t[ky] = (a - (epi - 1) / 2.0) * ro.t_line_ms
        pol[ky] = -1 if a % 2 == 1 else 1
    timing = LineTiming(t.copy(), te + t, t.copy(), pol)
    a = acq.replace(t_echo=te, do_relaxation=True, noise_variance=0.0, n_spikes=0)
    nc = max(acq.n_coils, 1)
    zs = nz // 2
    zk = np.array([[np.exp(1j * TAU * (p - zs) * (z - zs) / nz) for z in range(nz)] for p in range(nz)])
    coil_parts = []
    for q in range(nc):
        k2 = []
        for z in range(nz):
            inp = SliceInput(compartments=[img[z * nplane:(z + 1) * nplane]], t2=[T2.uniform(t2)],
                             t_inhom=[T2.uniform(ti)], fmap=fmap[z * nplane:(z + 1) * nplane], sim=(snx, sny),
                             acq_matrix=(nx, ny), phase0=np.zeros(nplane), z=z, nz=nz)
            k2.append(O.build_coil_kspace(inp, a, q, nc, timing=timing).ravel())
        k2 = np.array(k2)
        kp = zk @ k2 * np.array([w(p) for p in range(nz)])[:, None]
        coil_parts.append((zk.conj().T @ kp) / nz)
    out = np.zeros((nz, ny * nx), np.complex128)
    for z in range(nz):
        out[z] = O.reconstruct_coils(np.array([cp[z].reshape(ny, nx) for cp in coil_parts]), acq).ravel()
    return out.ravel()


def test_ge_lines_match_the_reference_layout():
    t = K3.ge3d_lines(ge_train3(2, [12.0]), K3.Ge3dReadout(2, 0.4), 12, 6)
    assert (t.n_shots, t.n_exc) == (4, 3)
    assert list(t.shot[:4]) == [0, 2, 0, 2] and list(t.excitation[::12]) == [0, 0, 1, 1, 2, 2]
    with pytest.raises(Exception, match="2D readout"):
        K3.ge3d_lines(ge_train3(1, [12.0]), K3.Ge3dReadout(1, 0.4), 12, 1)


@pytest.mark.parametrize("n_coils", [1, 3])
@pytest.mark.parametrize("mode", ["class", "voxel"])
def test_ge3d_matches_the_reference_forward(n_coils, mode):
    nx = ny = 16
    nz, o = 4, 2
    snx, sny = nx * o, ny * o
    nvox = snx * sny * nz
    img = blobs(snx, sny, nz, 1, 1)[0]
    fmap = varying_fmap(snx, sny, nz)
    ro = K3.Ge3dReadout(1, 0.4)
    tes = [12.0, 30.0]
    t2 = [T2.uniform(80.0)] if mode == "class" else [T2.of_map(np.full(nvox, 80.0, np.float32))]
    acq = ge_acq(n_coils)
    got, _ = O.simulate_acquisition_3d_ge([snx, sny, nz], [nx, ny, nz], 1, t2, fmap, [T2.uniform(45.0)], acq,
                                          ge_train3(1, tes), ro, lambda g: ge_volume([img], nz, 1, lambda *_: 0.7),
                                          phase=PhaseModel.none(), seed=5)
    for e, te in enumerate(tes):
        want = ge_reference(img, 80.0, 45.0, fmap, acq, te, ro, (nx, ny, nz), o, lambda p: 0.7)
        assert np.abs(got[e, 0] - want).max() <= 1e-9 * np.abs(want).max()


def test_ge3d_weights_across_partitions_blur_through_plane():
    nx = ny = 12
    nz, o = 6, 2
    snx, sny = nx * o, ny * o
    img = blobs(snx, sny, nz, 1, 1)[0]
    fmap = varying_fmap(snx, sny, nz)
    ro = K3.Ge3dReadout(1, 0.4)
    acq = ge_acq(2)
    w = lambda p: 1.0 + 0.5 * math.cos(p * 1.3)
    got, _ = O.simulate_acquisition_3d_ge([snx, sny, nz], [nx, ny, nz], 1, [T2.uniform(80.0)], fmap, [T2.uniform(45.0)],
                                          acq, ge_train3(2, [12.0]), ro,
                                          lambda g: ge_volume([img], nz, 1, lambda p, sy, c: w(p)),
                                          phase=PhaseModel.none(), seed=5)
    want = ge_reference(img, 80.0, 45.0, fmap, acq, 12.0, ro, (nx, ny, nz), o, w)
    pk = np.abs(want).max()
    assert np.abs(got[0, 0] - want).max() <= 1e-9 * pk
    flat = ge_reference(img, 80.0, 45.0, fmap, acq, 12.0, ro, (nx, ny, nz), o, lambda p: 1.0)
    assert np.abs(flat - want).max() > 0.01 * pk
