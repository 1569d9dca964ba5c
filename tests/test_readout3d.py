"""Host tables and timing checks of the 3D trains through the C ABI (no GPU), with the reference's
worked numbers (readout.rs tests `every_line_is_read_once_with_ky_only_within_echo_timing`,
`worked_numbers_for_the_acceptance_cases`, `spiral_asl001_numbers`, `ge3d_line_tables`,
`ge3d_timing`; kspace3d.rs `spiral_class_and_voxel_modes_agree` for the segmentation)."""
from __future__ import annotations

import numpy as np
import pytest

from mrsim_acq_b200 import kspace3d as K3
from mrsim_acq_b200.abi import MrsimError
from mrsim_acq_b200.api import Acquisition, T2


def train(nz, kzs, order, esp, b=180.0, etl=None):
    return K3.EchoTrain(etl=etl if etl is not None else nz // kzs, esp_ms=esp, refocusing_deg=b, kz_order=order,
                        kz_segments=kzs, refocusing_time_ms=2.0)


@pytest.mark.parametrize("kys", [1, 2, 4])
@pytest.mark.parametrize("kzs", [1, 2])
@pytest.mark.parametrize("order", [K3.KzOrder.Centric, K3.KzOrder.Linear])
@pytest.mark.parametrize("rev", [False, True])
def test_every_grase_line_is_read_once(kys, kzs, order, rev):
    ny, nz = 16, 8
    t = K3.grase_lines(train(nz, kzs, order, 20.0), K3.GraseReadout(kys, 0.5, rev), ny, nz)
    assert t.n_shots == kys * kzs
    for p in range(nz):
        for ky in range(ny):
            i = p * ny + ky
            assert abs(t.trf_ms[i] - (t.echo[i] * 20.0 + t.t_ms[i])) < 1e-12
            assert t.shot[i] == (ky % kys) * kzs + (t.shot[i] % kzs)
            assert t.t_ms[i] == t.t_ms[ky]
    seg0 = [ky for ky in range(ny) if ky % kys == 0]
    by_time = sorted(seg0, key=lambda ky: t.t_ms[ky])
    for a, b in zip(by_time, by_time[1:]):
        assert t.polarity[a] == -t.polarity[b] and abs(t.t_ms[b] - t.t_ms[a] - 0.5) < 1e-12
    assert by_time[0] == (0 if rev else ny - kys)


def test_grase_worked_numbers():
    ro = K3.GraseReadout(2, 1.0)
    esp = K3.esp_from_echo_time(11.92, 1, ro, 20)
    assert abs(esp - 12.42) < 1e-12
    tr = train(30, 1, K3.KzOrder.Centric, esp, etl=30)
    K3.check_grase_timing(tr, ro, 20, 30, 3000.0, 3500.0)
    esp64 = K3.esp_from_echo_time(11.92, 1, ro, 64)
    with pytest.raises(MrsimError) as e:
        K3.check_grase_timing(train(30, 1, K3.KzOrder.Centric, esp64, etl=30), ro, 64, 30, 3000.0, 3500.0)
    assert "echo spacing must be at least" in str(e.value) and "ky segments" in str(e.value)
    ro5 = K3.GraseReadout(4, 0.2048)
    esp5 = K3.esp_from_echo_time(13.28, 1, ro5, 64)
    assert abs(esp5 - 13.3824) < 1e-12
    tr5 = train(30, 1, K3.KzOrder.Centric, esp5, b=130.0, etl=30)
    K3.check_grase_timing(tr5, ro5, 64, 30, 3800.0, 4950.0)
    with pytest.raises(MrsimError, match="after"):
        K3.check_grase_timing(tr5, ro5, 64, 30, 4600.0, 4950.0)
    tiny = K3.EchoTrain(etl=1, esp_ms=1.9, refocusing_deg=130.0, kz_segments=1, refocusing_time_ms=2.0)
    with pytest.raises(MrsimError):
        K3.check_grase_timing(tiny, K3.GraseReadout(1, 0.0001), 1, 1, 0.0, 1000.0)
    with pytest.raises(MrsimError, match="69"):
        K3.grase_lines(train(4, 1, K3.KzOrder.Centric, 20.0), K3.GraseReadout(4, 0.2), 69, 4)


def test_spiral_asl001_timing():
    ro = K3.SpiralReadout(8, 4.0, 0.004, 1.2)
    tr = K3.EchoTrain(etl=20, esp_ms=0.0, refocusing_deg=111.0, kz_order=K3.KzOrder.Centric, kz_segments=1,
                      refocusing_time_ms=2.0)
    tab = K3.spiral_lines(tr, ro, 64, 64, 20)
    assert tab.samples_per_interleaf == 1000 and (tab.e_c, tab.n_shots) == (1, 8)
    esp = K3.spiral_esp_from_echo_time(10.528, tab.e_c)
    assert abs(esp - 10.528) < 1e-12
    tr = K3.EchoTrain(etl=20, esp_ms=esp, refocusing_deg=111.0, kz_order=K3.KzOrder.Centric, kz_segments=1,
                      refocusing_time_ms=2.0)
    end = K3.check_spiral_timing(tr, ro, 64, 64, 20, 3475.0, 4886.0)
    assert abs(end - 3689.56) < 1e-9
    with pytest.raises(MrsimError, match="next refocusing pulse"):
        K3.check_spiral_timing(tr, K3.SpiralReadout(4, 8.0, 0.004, 1.2), 64, 64, 20, 3475.0, 4886.0)
    with pytest.raises(MrsimError, match="after"):
        K3.check_spiral_timing(tr, ro, 64, 64, 20, 4700.0, 4886.0)
    two = K3.spiral_lines(K3.EchoTrain(etl=10, esp_ms=esp, refocusing_deg=111.0, kz_segments=2), ro, 64, 64, 20)
    assert two.n_shots == 16


def ge_train(kzs, order, tes, spacing=40.0):
    return K3.ExcitationTrain(kzs, order, spacing, list(tes), 2.0)


@pytest.mark.parametrize("order", [K3.KzOrder.Centric, K3.KzOrder.Linear])
@pytest.mark.parametrize("kzs", [1, 2, 8])
def test_ge3d_line_tables(order, kzs):
    ro = K3.Ge3dReadout(2, 0.5)
    ny, nz = 16, 8
    t = K3.ge3d_lines(ge_train(kzs, order, [12.0]), ro, ny, nz)
    assert (t.n_shots, t.n_exc) == (2 * kzs, nz // kzs)
    ordr = list(K3.kz_order(nz, order))
    for p in range(nz):
        pos = ordr.index(p)
        for ky in range(ny):
            i = p * ny + ky
            assert (t.shot[i], t.excitation[i]) == ((ky % 2) * kzs + pos % kzs, pos // kzs)
    assert t.e_c == ordr.index(nz // 2) // kzs


def test_ge3d_line_table_refusals():
    ro = K3.Ge3dReadout(2, 0.5)
    with pytest.raises(MrsimError, match="kz segments"):
        K3.ge3d_lines(ge_train(3, K3.KzOrder.Linear, [12.0]), ro, 16, 8)
    with pytest.raises(MrsimError, match="2D"):
        K3.ge3d_lines(ge_train(1, K3.KzOrder.Linear, [12.0]), ro, 16, 1)
    with pytest.raises(MrsimError, match="ky segments"):
        K3.ge3d_lines(ge_train(1, K3.KzOrder.Linear, [12.0]), K3.Ge3dReadout(3, 0.5), 16, 8)


def test_ge3d_timing():
    ro = K3.Ge3dReadout(2, 0.5)
    chk = lambda tes, spacing, tr: K3.check_ge3d_timing(ge_train(2, K3.KzOrder.Linear, tes, spacing), ro, 16, 8,
                                                        1000.0, tr)
    chk([12.0, 22.0], 40.0, 2000.0)
    with pytest.raises(MrsimError, match="excitation pulse"):
        chk([2.5], 40.0, 2000.0)
    chk([3.0], 40.0, 2000.0)
    with pytest.raises(MrsimError, match="overlap"):
        chk([12.0, 15.5], 40.0, 2000.0)
    chk([12.0, 16.0], 40.0, 2000.0)
    with pytest.raises(MrsimError, match="next excitation pulse"):
        chk([12.0, 32.0], 34.9, 2000.0)
    chk([12.0, 32.0], 35.0, 2000.0)
    with pytest.raises(MrsimError, match="repetition"):
        chk([12.0], 40.0, 1133.9)
    chk([12.0], 40.0, 1134.0)
    with pytest.raises(MrsimError):
        chk([], 40.0, 2000.0)
    one = ge_train(8, K3.KzOrder.Linear, [12.0], 10.0)
    K3.check_ge3d_timing(one, ro, 16, 8, 1000.0, 2000.0)
    with pytest.raises(MrsimError, match="repetition"):
        K3.check_ge3d_timing(one, ro, 16, 8, 1000.0, 1013.9)


def test_spiral_segmentation_is_certified_per_slice():
    n, nz, o = 16, 4, 2
    s = n * o
    nvox = s * s * nz
    v = np.arange(nvox)
    x, y, z = v % s, (v // s) % s, v // (s * s)
    fmap = (-15.0 + 30.0 * x / s + 5.0 * z - 3.0 * y / s).astype(np.float32)
    full = lambda val: T2.of_map(np.full(nvox, val, np.float32))
    acq = Acquisition(do_relaxation=True, do_distortions=True, signal_scale=100.0, t_inhom=50.0)
    tr = K3.EchoTrain(etl=2, esp_ms=12.0, refocusing_deg=130.0, kz_segments=2)
    ro = K3.SpiralReadout(2, 4.0, 0.01, 1.2)
    segs = K3.spiral_segmentation([s, s, nz], [n, n, nz], [full(80.0), full(120.0)], [full(1300.0), full(1600.0)],
                                  fmap, [full(50.0), full(50.0)], acq, tr, ro)
    assert len(segs) == nz and all(g["voxel"] and g["bound"] < 1e-7 and g["l"] <= 64 for g in segs)
    segs = K3.spiral_segmentation([s, s, nz], [n, n, nz], [T2.uniform(80.0)], [T2.uniform(1300.0)], fmap, None, acq,
                                  tr, ro)
    assert [g["z"] for g in segs] == list(range(nz)) and not any(g["voxel"] for g in segs)
    wide = np.full(nvox, 0.0, np.float32)
    wide[0] = 2e6
    with pytest.raises(MrsimError, match="slice 0"):
        K3.spiral_segmentation([s, s, nz], [n, n, nz], [T2.uniform(80.0)], [T2.uniform(1300.0)], wide, None, acq, tr,
                               ro)
