"""Pins of the oracle's stack-of-spirals restatement (CPU), from the reference's own tests
(kspace3d.rs:1957-2260, readout.rs `kz_sampling_patterns`): the spiral tables, 3D-is-the-2D-spiral
with relaxation off, class and voxel modes agreeing, partial Fourier zero-filling, and coil rings
along z combining to the single-ring image."""
from __future__ import annotations

import math

import numpy as np
import pytest

from cases3d import blobs, train
from mrsim_acq_b200 import kspace3d as K3
from mrsim_acq_b200.api import Acquisition, KspaceWindow, PhaseModel, SliceInput, T2
from oracle import oracle as O

TAU = 2.0 * math.pi


def spiral_fmap(snx, sny, nz):
    v = np.arange(snx * sny * nz)
    x, y, z = v % snx, (v // snx) % sny, v // (snx * sny)
    return (-15.0 + 30.0 * x / snx + 5.0 * z - 3.0 * y / sny).astype(np.float32)


def spiral_ro(pf=1.0, accel=1):
    return K3.SpiralReadout(2, 4.0, 0.01, 1.2, K3.KzSampling(pf, accel))


def kz_train(nz, kz, b=180.0):
    """kspace3d.rs `kz_train`: one kz segment, centric, etl = the partitions `kz` reads."""
    lo = nz - min(nz, int(round(nz * kz.partial_fourier)))
    c = nz // 2
    n = sum(1 for p in range(nz) if p >= lo and (p - c) % kz.accel == 0)
    return K3.EchoTrain(etl=n, esp_ms=12.0, refocusing_deg=b, kz_order=K3.KzOrder.Centric, kz_segments=1)


def test_spiral_tables_match_the_reference_numbers():
    kz = K3.KzSampling(0.75, 2)
    tr = K3.EchoTrain(etl=13, esp_ms=10.0, refocusing_deg=180.0, kz_order=K3.KzOrder.Centric, kz_segments=1)
    ro = K3.SpiralReadout(2, 4.0, 0.001, 1.2, kz)
    a, b = K3.spiral_lines(tr, ro, 64, 64, 36), O.spiral_lines(tr, ro, 64, 36)
    assert (a.band_start, a.e_c, a.n_shots) == (b["band_start"], b["e_c"], b["n_shots"]) == (9, 1, 2)
    assert [p - 18 for p in range(36) if a.acquired[p]] == [2 * m for m in range(-4, 9)]
    assert (a.echo == b["echo"]).all() and (a.acquired == b["acquired"]).all()
    assert tuple(a.echo[[18, 20, 16, 34, 19, 0]]) == (1, 2, 3, 13, 0, 0)
    lin = K3.EchoTrain(etl=13, esp_ms=10.0, refocusing_deg=180.0, kz_order=K3.KzOrder.Linear, kz_segments=1)
    assert K3.spiral_lines(lin, ro, 64, 64, 36).e_c == 5
    assert int(K3.spiral_lines(K3.EchoTrain(etl=23, esp_ms=10.0, refocusing_deg=180.0), K3.SpiralReadout(
        2, 4.0, 0.001, 1.2, K3.KzSampling(0.625, 1)), 64, 64, 36).acquired.sum()) == 23
    with pytest.raises(Exception, match=r"\(0.5, 1\]"):
        K3.spiral_lines(tr, K3.SpiralReadout(2, 4.0, 0.001, 1.2, K3.KzSampling(0.5, 1)), 64, 64, 36)
    with pytest.raises(Exception, match="13 partitions read"):
        K3.spiral_lines(K3.EchoTrain(etl=6, esp_ms=10.0, refocusing_deg=180.0, kz_segments=2), ro, 64, 64, 36)


def test_spiral_3d_is_the_2d_spiral():
    n, nz, o, ncomp = 16, 4, 2, 2
    s = n * o
    images = blobs(s, s, nz, 1, ncomp)
    fmap = spiral_fmap(s, s, nz)
    t2 = [T2.uniform(80.0)] * ncomp
    acq = Acquisition(do_relaxation=False, do_distortions=True, n_coils=2, signal_scale=100.0)
    vols, _, _ = O.simulate_acquisition_3d_spiral([s, s, nz], [n, n, nz], 1, images, t2, None, fmap, None, acq,
                                                  train(nz, 1, esp_ms=12.0), spiral_ro(), phase=PhaseModel.none(), seed=3)
    tab = O.spiral_lines(train(nz, 1, esp_ms=12.0), spiral_ro(), n, nz)
    k, tau = tab["k"], tab["tau_ms"]
    taus = tau[np.arange(len(k)) % len(tau)]
    nplane = s * s
    want = np.zeros(n * n * nz, np.complex128)
    data = []
    for z in range(nz):
        coils = []
        for q in range(2):
            acc = np.zeros(len(k), np.complex128)
            for im in images:
                inp = SliceInput(compartments=[im[z * nplane:(z + 1) * nplane]], t2=[T2.uniform(80.0)],
                                 fmap=fmap[z * nplane:(z + 1) * nplane], sim=(s, s), acq_matrix=(n, n),
                                 phase0=np.zeros(nplane), z=z, nz=nz)
                acc += O.spiral_kspace_exact(inp, acq, q, 2, k, taus)
            coils.append(acc)
        data.append(coils)
    imgs, _, _, _ = O.spiral_recon(k, n, np.array(data), "rings", ring=2, zsens=np.ones((nz, 2)))
    want = imgs.reshape(nz, n * n).ravel()
    got = vols[0]
    pk = np.abs(want).max()
    assert np.abs(got - want).max() <= 1e-9 * pk


def test_spiral_class_and_voxel_modes_agree():
    n, nz, o, ncomp = 16, 4, 2, 2
    s = n * o
    nvox = s * s * nz
    images = blobs(s, s, nz, 1, ncomp)
    fmap = spiral_fmap(s, s, nz)
    acq = Acquisition(do_relaxation=True, do_distortions=True, signal_scale=100.0, t_inhom=50.0)
    tr = train(nz, 2, esp_ms=12.0, b=130.0)
    full = lambda v: T2.of_map(np.full(nvox, v, np.float32))
    a, _, _ = O.simulate_acquisition_3d_spiral([s, s, nz], [n, n, nz], 1, images, [T2.uniform(80.0), T2.uniform(120.0)],
                                               [T2.uniform(1300.0), T2.uniform(1600.0)], fmap, None, acq, tr,
                                               spiral_ro(), seed=3)
    b, _, _ = O.simulate_acquisition_3d_spiral([s, s, nz], [n, n, nz], 1, images, [full(80.0), full(120.0)],
                                               [full(1300.0), full(1600.0)], fmap, [full(50.0), full(50.0)], acq, tr,
                                               spiral_ro(), seed=3)
    pk = np.abs(a).max()
    assert np.abs(a - b).max() <= 1e-6 * pk


def test_kz_partial_fourier_zero_fills():
    n, nz, o, ncomp = 16, 8, 2, 2
    s = n * o
    images = blobs(s, s, nz, 1, ncomp)
    fmap = spiral_fmap(s, s, nz)
    t2 = [T2.uniform(80.0)] * ncomp
    acq = Acquisition(do_relaxation=False, do_distortions=True, signal_scale=100.0)

    def run(kz):
        return O.simulate_acquisition_3d_spiral([s, s, nz], [n, n, nz], 1, images, t2, None, fmap, None, acq,
                                                kz_train(nz, kz), spiral_ro(kz.partial_fourier, kz.accel),
                                                phase=PhaseModel.none(), seed=3)[0][0]

    full = run(K3.KzSampling(1.0, 1)).reshape(nz, n * n)
    pf = run(K3.KzSampling(0.75, 1)).reshape(nz, n * n)
    lo = 2
    zs = nz // 2
    zk = np.array([[np.exp(1j * TAU * (p - zs) * (z - zs) / nz) for z in range(nz)] for p in range(nz)])
    kp = zk @ full  # [p][i]
    kp[:lo] = 0
    want = (zk.conj().T @ kp) / nz
    pk = np.abs(want).max()
    assert np.abs(pf - want).max() <= 1e-9 * pk
    assert np.abs(pf - full).max() > 1e-3 * pk


def test_coil_rings_combine_to_the_single_ring_image():
    n, nz, o, ncomp = 16, 6, 2, 2
    s = n * o
    images = blobs(s, s, nz, 1, ncomp)
    fmap = spiral_fmap(s, s, nz)
    t2 = [T2.uniform(80.0), T2.uniform(110.0)]
    tr = train(nz, 1, esp_ms=12.0)

    def run(n_coils, rows):
        acq = Acquisition(do_relaxation=False, do_distortions=True, n_coils=n_coils, signal_scale=100.0)
        return O.simulate_acquisition_3d_spiral([s, s, nz], [n, n, nz], 1, images, t2, None, fmap, None, acq, tr,
                                                spiral_ro(), phase=PhaseModel.none(), seed=3,
                                                kz_opts=K3.KzOptions(coil_rows=rows))[0][0]

    one, three = run(2, 1), run(6, 3)
    pk = np.abs(one).max()
    assert np.abs(one - three).max() <= 1e-9 * pk


def test_spiral_shot_images_double_exactly_their_samples():
    """`spiral_shots_select_exactly_their_samples` (kspace3d.rs:2103-2150), the shot-set part: with
    3 interleaves x 2 kz segments, a set with doubled images for shot 4 (interleaf 2, kz segment
    0) doubles exactly its own samples."""
    n, nz, o, ncomp = 16, 4, 2, 2
    s = n * o
    images = blobs(s, s, nz, 1, ncomp)
    fmap = spiral_fmap(s, s, nz)
    t2 = [T2.uniform(80.0), T2.uniform(110.0)]
    acq = Acquisition(do_relaxation=True, do_distortions=True, signal_scale=100.0)
    tr = train(nz, 2, esp_ms=12.0, b=180.0)
    ro = K3.SpiralReadout(3, 4.0, 0.01, 1.2, K3.KzSampling(1.0, 1))
    args = ([s, s, nz], [n, n, nz], 1, images, t2, None, fmap, None, acq, tr, ro)
    tab = O.spiral_lines(tr, ro, n, nz)
    assert tab["n_shots"] == 6
    base = O.spiral_samples_3d(*args, phase=PhaseModel.none())[0]
    doubled = [2.0 * im for im in images]
    moved = O.spiral_samples_3d(*args, phase=PhaseModel.none(), shot_images=[[K3.ShotSet([4], doubled)]])[0]
    nsamp = base.shape[1]
    ns = nsamp // 3
    shot = (np.arange(nsamp)[None, :] // ns) * 2 + tab["kz_segment"][:, None]
    f = np.where(shot == 4, 2.0, 1.0)
    assert np.array_equal(moved, f * base)
    assert np.count_nonzero(shot == 4) == ns * nz // 2
