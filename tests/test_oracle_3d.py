"""Pins of the oracle's 3D GRASE restatement (CPU): the reference's own reduction test
`with_nothing_to_distinguish_partitions_3d_is_2d` and `ghost_polarity_follows_the_acquisition_index`
(kspace3d.rs:1613-1708), the GRASE line tables and kz order against the product's host tables, and
the oracle's EPG against the product's (readout.rs / epg.rs tests)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from cases3d import TAU, blobs, grase, train
from mrsim_acq_b200 import kspace3d as K3
from mrsim_acq_b200 import spiral as S
from mrsim_acq_b200.api import Acquisition, LineTiming, PartialFourierMode, PhaseModel, SliceInput, T2
from oracle import oracle as O


def test_kz_order_and_grase_tables_match_the_product():
    for nz in (1, 2, 5, 6, 7, 36):
        for order in (K3.KzOrder.Centric, K3.KzOrder.Linear):
            assert (K3.kz_order(nz, order) == O.kz_order(nz, int(order))).all()
    assert list(K3.kz_order(7, K3.KzOrder.Centric)) == [3, 4, 2, 5, 1, 6, 0]
    for nz, kzs, kys, order, rev in [(6, 2, 2, K3.KzOrder.Centric, False), (8, 1, 4, K3.KzOrder.Linear, True),
                                     (4, 4, 1, K3.KzOrder.Centric, False)]:
        tr, ro = train(nz, kzs, order), grase(kys, 0.5, rev)
        a, b = K3.grase_lines(tr, ro, 16, nz), O.grase_lines(tr, ro, 16, nz)
        for k in ("shot", "echo", "t_ms", "trf_ms", "polarity"):
            assert (getattr(a, k) == b[k]).all(), k
        assert (a.e_c, a.n_shots) == (b["e_c"], b["n_shots"]) == (a.e_c, kys * kzs)


def test_grase_table_refusals():
    with pytest.raises(Exception, match="ky segments"):
        K3.grase_lines(train(4, 1), grase(3), 16, 4)
    with pytest.raises(Exception, match="kz segments"):
        K3.grase_lines(train(4, 3), grase(1), 16, 4)
    with pytest.raises(Exception, match="echo train length"):
        K3.grase_lines(K3.EchoTrain(etl=3, esp_ms=20.0, refocusing_deg=180.0), grase(1), 16, 4)


@pytest.mark.parametrize("b,t1,t2", [(150.0, 1000.0, 80.0), (111.0, 830.0, 70.0), (180.0, math.inf, 100.0)])
def test_oracle_epg_matches_the_product(b, t1, t2):
    assert np.array_equal(O.epg_cpmg(12, 13.4, b, t1, t2), S.epg_cpmg(12, 13.4, b, t1, t2))


@pytest.mark.parametrize("n_coils,accel", [(1, 1), (3, 2)])
def test_with_nothing_to_distinguish_partitions_3d_is_2d(n_coils, accel):
    nx = ny = 16
    nz, o, nv, ncomp = 6, 2, 2, 2
    snx, sny = nx * o, ny * o
    images = blobs(snx, sny, nz, nv, ncomp)
    fmap = np.zeros(snx * sny * nz, np.float32)
    t2 = [T2.uniform(80.0)] * ncomp
    acq = Acquisition(do_relaxation=False, n_coils=n_coils, accel=accel, acs_lines=6, signal_scale=100.0)
    two = O.acquire_volumes_complex([snx, sny, nz], [nx, ny, nz], nv, images, t2, fmap, acq, 9, 9,
                                    phase=PhaseModel.none())
    z2 = two["re"].astype(np.float64) + 1j * two["im"].astype(np.float64)
    pk = np.abs(z2).max()
    for kys in (1, 2, 4):
        for kzs in (1, 2):
            for order in (K3.KzOrder.Centric, K3.KzOrder.Linear):
                vols, mag, ph = O.simulate_acquisition_3d([snx, sny, nz], [nx, ny, nz], nv, images, t2, None, fmap,
                                                          None, acq, train(nz, kzs, order), grase(kys),
                                                          phase=PhaseModel.none(), seed=9)
                z3 = vols.T.ravel()  # [g][vox] -> vox * nv + g
                assert np.abs(z3 - z2).max() <= 1e-5 * pk, (kys, kzs, order)


@pytest.mark.parametrize("reverse_phase", [False, True])
def test_ghost_polarity_follows_the_acquisition_index(reverse_phase):
    nx, ny, nz, o = 12, 16, 4, 2
    snx, sny = nx * o, ny * o
    images = blobs(snx, sny, nz, 1, 1)
    fmap = np.zeros(snx * sny * nz, np.float32)
    t2 = [T2.uniform(80.0)]
    acq = Acquisition(do_relaxation=False, ghost_offset=0.05, reverse_phase=reverse_phase)
    tr, ro = train(nz, 1), grase(2, 0.5, reverse_phase)
    got = O.kspace_3d_observed([snx, sny, nz], [nx, ny, nz], 1, images, t2, None, fmap, None, acq, tr, ro,
                               phase=PhaseModel.none())[0]
    epi = ny // 2
    t = np.zeros(ny)
    pol = np.zeros(ny, np.int8)
    for ky in range(ny):
        j = ky // 2
        a = j if reverse_phase else epi - 1 - j
        t[ky] = (a - (epi - 1) / 2.0) * 0.5
        pol[ky] = 1 if a % 2 == 0 else -1

    def direct(polarity):
        lt = LineTiming(t.copy(), t.copy(), t.copy(), polarity)
        nplane = snx * sny
        k2 = []
        for z in range(nz):
            pl = images[0][z * nplane:(z + 1) * nplane]
            inp = SliceInput(compartments=[pl], t2=[T2.uniform(80.0)], fmap=fmap[z * nplane:(z + 1) * nplane],
                             sim=(snx, sny), acq_matrix=(nx, ny), phase0=np.zeros(nplane), z=z, nz=nz)
            k2.append(O.build_coil_kspace(inp, acq, 0, 1, timing=lt).ravel())
        zs = nz // 2
        out = np.zeros((nz, ny * nx), np.complex128)
        for p in range(nz):
            for z in range(nz):
                th = TAU * (p - zs) * (z - zs) / nz
                out[p] += k2[z] * complex(math.cos(th), math.sin(th))
        return out.reshape(nz, ny, nx)

    want = direct(pol)
    wrong = direct(np.array([-1 if k % 2 == 1 else 1 for k in range(ny)], np.int8))
    pk = np.abs(want).max()
    assert np.abs(got - want).max() <= 1e-10 * pk
    assert np.abs(got - wrong).max() > 1e-3 * pk


def test_refusals_name_the_input():
    nx = ny = 8
    nz, o = 2, 1
    images = blobs(nx, ny, nz, 1, 1)
    fmap = np.zeros(nx * ny * nz, np.float32)
    with pytest.raises(RuntimeError, match="needs T1"):
        O.simulate_acquisition_3d([nx, ny, nz], [nx, ny, nz], 1, images, [T2.uniform(80.0)], None, fmap, None,
                                  Acquisition(), train(nz, 1, b=150.0), grase(1))


def test_shot_images_double_exactly_their_lines():
    """`shots_and_their_weights` (kspace3d.rs:1844-1901), the per-shot-images part: doubled images
    for shot 1 of a two-segment GRASE train double exactly its lines (odd ky) at the observation
    point and leave the others unchanged."""
    nx = ny = 16
    nz = 4
    nvox = nx * ny * nz
    vox = np.arange(nvox)
    x, y = vox % nx, (vox // nx) % ny
    img = np.where((x >= 5) & (x < 11) & (y >= 6) & (y < 10), 1.0 + 0.1 * x, 0.0).astype(np.float32)
    fmap = np.zeros(nvox, np.float32)
    acq = Acquisition(do_relaxation=False)
    args = ([nx, ny, nz], [nx, ny, nz], 1, [img], [T2.uniform(80.0)], None, fmap, None, acq, train(nz, 1, b=180.0),
            grase(2))
    full = O.kspace_3d_observed(*args, phase=PhaseModel.none())[0]
    moved = O.kspace_3d_observed(*args, phase=PhaseModel.none(),
                                 shot_images=[[K3.ShotSet([1], [2.0 * img])]])[0]
    odd = (np.arange(ny) % 2 == 1)[None, :, None]
    assert np.all(np.abs(moved - 2.0 * full)[np.broadcast_to(odd, full.shape)] <= 1e-12)
    assert np.array_equal(moved[np.broadcast_to(~odd, full.shape)], full[np.broadcast_to(~odd, full.shape)])


def test_shot_images_refusals():
    nx = ny = 8
    nz = 4
    nvox = nx * ny * nz
    img = np.ones(nvox, np.float32)
    args = ([nx, ny, nz], [nx, ny, nz], 1, [img], [T2.uniform(80.0)], None, np.zeros(nvox, np.float32), None,
            Acquisition(do_relaxation=False), train(nz, 1, b=180.0), grase(2))
    with pytest.raises(RuntimeError, match="a shot index beyond the train's 2"):
        O.kspace_3d_observed(*args, shot_images=[[K3.ShotSet([2], [img])]])
