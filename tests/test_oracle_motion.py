"""The motion oracle (FP64 restatement of motion.rs / mat.rs) against the reference's own motion
tests, on the CPU: the trilinear edge rule, a translation moving a bright voxel, multiband dropout
(b0 exempt, the multiband partner dropping with its shot), the slab variant agreeing with the
whole volume where no jump crosses the slab edge, and the dropout laws' values."""
import math

import numpy as np

from oracle import oracle as O

ID = np.eye(4)


def rotation_zyx_deg(rx, ry, rz):
    rx, ry, rz = (a * (math.pi / 180.0) for a in (rx, ry, rz))
    X = np.array([[1, 0, 0], [0, math.cos(rx), -math.sin(rx)], [0, math.sin(rx), math.cos(rx)]])
    Y = np.array([[math.cos(ry), 0, math.sin(ry)], [0, 1, 0], [-math.sin(ry), 0, math.cos(ry)]])
    Z = np.array([[math.cos(rz), -math.sin(rz), 0], [math.sin(rz), math.cos(rz), 0], [0, 0, 1]])
    return Z @ (Y @ X)


def oblique_v2w():
    """motion.rs tests `oblique_v2w`: an oblique, anisotropic grid."""
    r = rotation_zyx_deg(4.0, -3.0, 7.0)
    s = [1.5, 1.75, 3.0]
    m = np.eye(4)
    m[:3, :3] = r * np.array(s)[None, :]
    m[:3, 3] = [-12.0, 8.5, -20.0]
    return m


def smooth(dims, phase):
    """motion.rs tests `smooth`."""
    nx, ny, nz = dims
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    a, b, c = x / nx, y / ny, z / nz
    return (1.0 + np.sin(3.0 * a + phase) * np.cos(2.0 * b) + 0.5 * np.sin(4.0 * c)).astype(np.float32).ravel()


def test_trilinear_extends_edge_voxels_half_a_voxel_and_zeroes_beyond():
    dims = [2, 3, 4]
    vol = (1.0 + np.arange(24)).astype(np.float32)
    at = lambda x, y, z: float(vol[x + 2 * (y + 3 * z)])  # noqa: E731
    for dz in (1e-13, 1e-3, 0.25, 0.5):
        assert O.motion_trilinear(vol, dims, [1.0, 2.0, -dz]) == at(1, 2, 0)
        assert O.motion_trilinear(vol, dims, [0.0, 1.0, 3.0 + dz]) == at(0, 1, 3)
    mid = O.motion_trilinear(vol, dims, [-0.3, 1.5, 3.4])
    assert abs(mid - (at(0, 1, 3) + at(0, 2, 3)) / 2.0) < 1e-6
    for p in ([-0.51, 1, 1], [1.51, 1, 1], [0, -0.51, 1], [0, 2.51, 1], [0, 1, -0.51], [0, 1, 3.51]):
        assert O.motion_trilinear(vol, dims, p) == 0.0


def test_apply_motion_translation_shifts_the_head():
    n = 9
    img = np.zeros(n ** 3, np.float32)
    at = lambda x, y, z: x + n * (y + n * z)  # noqa: E731
    img[at(4, 4, 4)] = 1.0
    O.apply_motion([img], [n, n, n], 1, ID, [[0, 0, 0, 2.0, 0, 0]])
    assert img[at(6, 4, 4)] > 0.8 and img[at(4, 4, 4)] < 0.2


def test_multiband_dropout_darkens_dwi_shot_not_b0():
    nx = ny = nz = 4
    ng = 2
    img = np.ones(nx * ny * nz * ng, np.float32)
    gt = O.apply_multiband_motion([img], [nx, ny, nz], ng, ID, 2, False, 1, [0.0, 1000.0], 50.0, 0.0,
                                  [(1, 0, 1.0, (0, 0, 0), (0, 0, 0))])
    at = lambda x, y, z, g: (x + nx * (y + ny * z)) * ng + g  # noqa: E731
    assert img[at(1, 1, 0, 1)] < 0.01 and img[at(1, 1, 2, 1)] < 0.01
    assert abs(img[at(1, 1, 1, 1)] - 1.0) < 0.01 and abs(img[at(1, 1, 0, 0)] - 1.0) < 1e-6
    assert len(gt) == 1 and gt[0][:2] == (1, 0)


def test_multiband_slab_matches_the_full_volume_where_no_jump_crosses_the_edge():
    nx, ny, nz, ng = 4, 3, 6, 2
    mk = lambda: (1.0 + (np.arange(nx * ny * nz * ng) % 13)).astype(np.float32)  # noqa: E731
    # slice_schedule(6, 2, interleaved): groups 0, 2, 1 -> shots {0,3}, {2,5}, {1,4}; slice 4 is in shot 2
    events = [(1, 2, 0.8, (0, 0, 0), (0, 0, 0))]
    full = mk()
    gt_full = O.apply_multiband_motion([full], [nx, ny, nz], ng, ID, 2, True, 1, [0.0, 2000.0], 50.0, 0.0, events)
    orig = mk()
    r = slice(nx * ny * 4 * ng, nx * ny * 6 * ng)
    slab = orig[r].copy()
    gt_slab = O.apply_multiband_motion([slab], [nx, ny, 2], ng, ID, 2, True, 1, [0.0, 2000.0], 50.0, 0.0, events,
                                       slice_z=[4, 5], nz_full=nz)
    assert np.array_equal(slab, full[r]) and not np.array_equal(slab, orig[r])
    assert gt_full == gt_slab and len(gt_full) == 1


def test_dropout_laws():
    def att(kind, drive, floor, mx, g, sev):
        img = np.ones(2 * 2 * 2 * 8, np.float32)
        gt = O.apply_multiband_motion([img], [2, 2, 2], 8, ID, 1, False, kind, drive, floor, mx,
                                      [(g, 0, sev, (0, 0, 0), (0, 0, 0))])
        return gt[0][2]
    assert att(1, [5.0, 1000.0, 2000.0], 50.0, 0.0, 0, 0.5) == 1.0
    assert att(1, [5.0, 1000.0, 2000.0], 50.0, 0.0, 2, 0.5) == 0.5
    assert att(1, [5.0, 1000.0, 2000.0], 50.0, 0.0, 1, 0.5) == 0.75
    assert att(1, [5.0, 1000.0, 2000.0], 50.0, 0.0, 7, 0.5) == 1.0
    assert att(0, [], 0.0, 0.0, 3, 0.5) == 0.5
    want = np.float32(1.0) - np.float32(0.5) * np.float32(1005.0 / 1000.0)
    assert np.float32(att(2, [0.0, 1005.0, 30.0], 50.0, 1000.0, 1, 0.5)) == want
    assert att(2, [1000.0], 50.0, 0.0, 0, 0.9) == 1.0


def test_identity_copies_and_a_small_pose_moves_little():
    dims = [9, 9, 9]
    v = smooth(dims, 0.3)
    out = O.resample_by_pose(v, dims, oblique_v2w(), [0.0, 0.0, 0.0, 0.0, 0.0, 0.0])
    assert np.array_equal(out, v)  # the identity copies
    moved = O.resample_by_pose(v, dims, oblique_v2w(), [1.5, -2.0, 3.0, 0.4, -0.3, 0.2])
    # a small motion: most of the field moves a fraction of a voxel; edge voxels leave the grid
    assert not np.array_equal(moved, v)
    assert np.linalg.norm(moved - v) / np.linalg.norm(v) < 0.3
