"""The series writer (host code, CPU): NIfTI-1 files read back by an independent reader of the
published format, the reference's header tests (`four_d_header_carries_the_time_step_only_when_
asked`, io.rs tests), its `hires_grid` tests (FOV kept, identity at o = 1, corners coincide), the
qform quaternion reproducing the affine, and the BIDS sidecars' text."""
import gzip
import json
import math
import struct

import numpy as np
import pytest

from mrsim_acq_b200 import io as mio

HDR = "<i10s18sihcc8h3f4h8f3fhcc2f2f2i80s24s2h3f3f4f4f4f16s4s"


def read_nifti(path):
    raw = open(path, "rb").read()
    if str(path).endswith(".gz"):
        raw = gzip.decompress(raw)
    f = struct.unpack(HDR, raw[:348])
    h = {"sizeof_hdr": f[0], "dim": f[7:15], "datatype": f[19], "bitpix": f[20], "pixdim": f[22:30],
         "vox_offset": f[30], "xyzt_units": f[35][0], "qform_code": f[44], "sform_code": f[45],
         "quatern": f[46:49], "qoffset": f[49:52], "srow": [f[52:56], f[56:60], f[60:64]], "magic": f[65]}
    ndim = h["dim"][0]
    shape = h["dim"][1:1 + ndim]
    data = np.frombuffer(raw[int(h["vox_offset"]):], "<f4")
    assert data.size == int(np.prod(shape))
    return h, data


def quatern_to_mat44(b, c, d, qx, qy, qz, dx, dy, dz, qfac):
    """The NIfTI-1 standard's quaternion to matrix (io.rs `quatern_to_mat44`)."""
    a = 1.0 - (b * b + c * c + d * d)
    if a < 1e-7:
        n = math.sqrt(b * b + c * c + d * d)
        b, c, d, a = b / n, c / n, d / n, 0.0
    else:
        a = math.sqrt(a)
    dz = dz * qfac
    return np.array([[(a * a + b * b - c * c - d * d) * dx, 2 * (b * c - a * d) * dy, 2 * (b * d + a * c) * dz, qx],
                     [2 * (b * c + a * d) * dx, (a * a + c * c - b * b - d * d) * dy, 2 * (c * d - a * b) * dz, qy],
                     [2 * (b * d - a * c) * dx, 2 * (c * d + a * b) * dy, (a * a + d * d - c * c - b * b) * dz, qz],
                     [0, 0, 0, 1.0]])


def test_four_d_header_carries_the_time_step_only_when_asked(tmp_path):
    g = np.array([[2.0, 0, 0, 1.0], [0, 2.0, 0, 2.0], [0, 0, 3.0, 3.0], [0, 0, 0, 1]])
    data = np.full(3 * 2 * 2 * 4, 0.5, np.float32)
    mio.write_4d(tmp_path / "timed.nii.gz", [3, 2, 2], 4, data, g, tr_s=4.25)
    h, _ = read_nifti(tmp_path / "timed.nii.gz")
    assert list(h["pixdim"][1:5]) == [2.0, 2.0, 3.0, 4.25] and h["xyzt_units"] == 10
    mio.write_4d(tmp_path / "plain.nii.gz", [3, 2, 2], 4, data, g)
    h, _ = read_nifti(tmp_path / "plain.nii.gz")
    assert list(h["pixdim"][1:5]) == [2.0, 2.0, 3.0, 0.0] and h["xyzt_units"] == 2


def _oblique(left_handed=False):
    rx, ry, rz = (math.radians(v) for v in (4.0, -3.0, 7.0))
    X = np.array([[1, 0, 0], [0, math.cos(rx), -math.sin(rx)], [0, math.sin(rx), math.cos(rx)]])
    Y = np.array([[math.cos(ry), 0, math.sin(ry)], [0, 1, 0], [-math.sin(ry), 0, math.cos(ry)]])
    Z = np.array([[math.cos(rz), -math.sin(rz), 0], [math.sin(rz), math.cos(rz), 0], [0, 0, 1]])
    m = np.eye(4)
    m[:3, :3] = (Z @ Y @ X) * np.array([1.5, 1.75, -3.0 if left_handed else 3.0])[None, :]
    m[:3, 3] = [-12.0, 8.5, -20.0]
    return m


@pytest.mark.parametrize("left", [False, True])
def test_affine_data_and_quaternion_round_trip(tmp_path, left):
    v2w = _oblique(left)
    dims, nt = [5, 4, 3], 6
    rng = np.random.default_rng(1)
    data = rng.random(5 * 4 * 3 * nt).astype(np.float32)  # volume innermost
    mio.write_4d(tmp_path / "a.nii", dims, nt, data, v2w)
    h, back = read_nifti(tmp_path / "a.nii")
    assert h["sizeof_hdr"] == 348 and h["magic"] == b"n+1\x00" and h["datatype"] == 16 and h["bitpix"] == 32
    assert h["dim"][:5] == (4, 5, 4, 3, nt) and h["qform_code"] == 1 and h["sform_code"] == 1
    assert np.array_equal(back.reshape(nt, -1).T.ravel(), data)  # NIfTI stores x fastest, t slowest
    assert np.array_equal(np.array(h["srow"], np.float32), v2w[:3].astype(np.float32))
    q = quatern_to_mat44(*h["quatern"], *h["qoffset"], *h["pixdim"][1:4], h["pixdim"][0])
    assert np.abs(q - v2w).max() < 1e-5
    assert h["pixdim"][0] == (-1.0 if left else 1.0)


def test_three_d_header(tmp_path):
    mio.write_3d(tmp_path / "v.nii.gz", [4, 3, 2], np.arange(24, dtype=np.float32), np.eye(4))
    h, back = read_nifti(tmp_path / "v.nii.gz")
    assert h["dim"][:4] == (3, 4, 3, 2) and np.array_equal(back, np.arange(24, dtype=np.float32))


def test_hires_affine_preserves_the_fov():
    g = np.array([[1.7, 0, 0, -10.0], [0, 1.7, 0, -12.0], [0, 0, 1.7, 3.0], [0, 0, 0, 1]])
    h, dims = mio.hires_grid(g, [8, 8, 2], 4)
    assert dims == [32, 32, 2]
    for ax in range(2):
        assert abs(8 * g[ax, ax] - dims[ax] * h[ax, ax]) < 1e-9
    assert h[2, 2] == g[2, 2]


def test_hires_grid_is_identity_at_o_equals_one():
    g = np.array([[2.0, 0, 0, 1.0], [0, 2.0, 0, 2.0], [0, 0, 3.0, 4.0], [0, 0, 0, 1]])
    h, dims = mio.hires_grid(g, [5, 7, 3], 1)
    assert dims == [5, 7, 3] and np.abs(h - g).max() < 1e-12


def test_hires_corners_coincide_with_the_nominal_grid():
    g = np.array([[1.7, 0, 0, -5.0], [0, 1.7, 0, -7.0], [0, 0, 1.7, 0.5], [0, 0, 0, 1]])
    for o in (2, 3, 4, 8):
        h, _ = mio.hires_grid(g, [6, 9, 2], o)
        for r in range(3):
            nom = g[r, 3] - 0.5 * g[r, 0] - 0.5 * g[r, 1]
            hi = h[r, 3] - 0.5 * h[r, 0] - 0.5 * h[r, 1]
            assert abs(nom - hi) < 1e-9


def _sidecar_text(info, dims, part):
    """The reference's sidecar format (io.rs:206-226), restated."""
    ped = info.phase_encoding_direction
    pe_axis = {"i": 0, "k": 2}.get(ped[:1], 1)
    ees = info.total_readout_time / max(dims[pe_axis] - 1, 1)
    pf = info.partial_fourier
    pf_s = str(int(pf)) if pf == int(pf) else repr(pf)
    b0 = f',\n  "B0FieldSource": "{info.b0_field_source}"' if info.b0_field_source else ""
    common = (f'  "Manufacturer": "{info.manufacturer}",\n  "PhaseEncodingDirection": "{ped}",\n  '
              f'"TotalReadoutTime": {info.total_readout_time:.6f},\n  "EffectiveEchoSpacing": {ees:.8f},\n  '
              f'"EchoTime": {info.echo_time:.4f},\n  "PartialFourier": {pf_s},\n  '
              f'"ParallelReductionFactorInPlane": {info.accel},\n  "MultibandAccelerationFactor": {info.mb}{b0}')
    if part == "mag":
        return "{\n" + common + ',\n  "ImageComparison": "magnitude"\n}\n'
    return "{\n" + common + ',\n  "ImageComparison": "phase",\n  "Units": "rad"\n}\n'


@pytest.mark.parametrize("pf,b0", [(0.75, None), (1.0, "fmap0")])
def test_complex_pair_and_sidecars(tmp_path, pf, b0):
    info = mio.SidecarInfo("aslscan", "j-", 0.0315, 0.03, pf, 2, 3, repetition_time_s=2.5, b0_field_source=b0)
    dims, nv = [4, 5, 3], 2
    rng = np.random.default_rng(2)
    mag = rng.random(60 * nv).astype(np.float32)
    ph = (rng.random(60 * nv).astype(np.float32) - 0.5) * 6.0
    pre = str(tmp_path / "sub-01_dir-AP")
    mio.write_complex_4d(pre, "dwi", dims, nv, mag, ph, np.diag([2.0, 2.0, 2.5, 1.0]), info)
    for part, arr in (("mag", mag), ("phase", ph)):
        h, back = read_nifti(f"{pre}_part-{part}_dwi.nii.gz")
        assert np.array_equal(back.reshape(nv, -1).T.ravel(), arr) and h["pixdim"][4] == 2.5
        text = open(f"{pre}_part-{part}_dwi.json").read()
        assert text == _sidecar_text(info, dims, part)
        json.loads(text)
