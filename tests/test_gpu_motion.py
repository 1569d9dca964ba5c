"""Device motion resampling against the FP64 motion oracle, bit for bit (both evaluate the
reference's FP64 operation order; the device uses no contracted multiply-adds): one volume by a
pose on an oblique grid, a series by per-volume poses, multiband shot motion with dropout on the
whole volume and on a slab, and the operator's in-place motion feeding its forward."""
import numpy as np
import pytest

from mrsim_acq_b200 import api
from mrsim_acq_b200 import motion as M
from oracle import oracle as O
from tests import cases
from tests.test_oracle_motion import oblique_v2w, smooth

pytestmark = pytest.mark.gpu


def _poses(n, seed):
    rng = np.random.default_rng(seed)
    out = [M.Pose(tuple(rng.uniform(-2, 2, 3)), tuple(rng.uniform(-2, 2, 3))) for _ in range(n)]
    out[0] = M.IDENTITY
    return out


def test_resample_by_pose_is_the_oracle_bit_for_bit(gpu_ctx):
    dims = [23, 17, 11]
    v = smooth(dims, 0.4)
    for pose in _poses(5, 1):
        got = M.resample_by_pose(v, dims, oblique_v2w(), pose, ctx=gpu_ctx)
        want = O.resample_by_pose(v, dims, oblique_v2w(), pose.as_array())
        assert np.array_equal(got, want), pose


def test_apply_motion_is_the_oracle_bit_for_bit(gpu_ctx):
    dims, nv = [20, 16, 6], 5
    rng = np.random.default_rng(2)
    imgs = [rng.random(20 * 16 * 6 * nv).astype(np.float32) for _ in range(3)]
    poses = _poses(nv, 3)
    want = [a.copy() for a in imgs]
    O.apply_motion(want, dims, nv, oblique_v2w(), np.stack([p.as_array() for p in poses]))
    M.apply_motion(imgs, dims, nv, oblique_v2w(), poses, ctx=gpu_ctx)
    for a, b in zip(imgs, want):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("slab", [False, True])
def test_multiband_motion_is_the_oracle_bit_for_bit(gpu_ctx, slab):
    nx, ny, nz, nv = 12, 10, 8, 4
    rng = np.random.default_rng(4)
    events = [M.MotionEvent(1, 0, 0.6, (0.5, -0.3, 0.2), (1.0, 0.0, -0.5)),
              M.MotionEvent(1, 2, 0.3, (0.0, 0.4, 0.0), (0.0, 0.7, 0.0)),
              M.MotionEvent(3, 1, 0.9)]
    law = M.DropoutLaw("scaled", [0.0, 1000.0, 500.0, 2000.0], floor=50.0)
    v2w = oblique_v2w()
    if slab:
        z0, z1 = 3, 7
        dims = [nx, ny, z1 - z0]
        kw = dict(slice_z=list(range(z0, z1)), nz_full=nz)
    else:
        dims = [nx, ny, nz]
        kw = {}
    imgs = [rng.random(nx * ny * dims[2] * nv).astype(np.float32) for _ in range(2)]
    want = [a.copy() for a in imgs]
    gt_o = O.apply_multiband_motion(want, dims, nv, v2w, 2, True, 1, law.drive, law.floor, 0.0,
                                    [(e.volume, e.shot, e.severity, e.jump_mm, e.jump_deg) for e in events], **kw)
    gt = M.apply_multiband_motion(imgs, dims, nv, v2w, 2, True, law, events, ctx=gpu_ctx, **kw)
    for a, b in zip(imgs, want):
        assert np.array_equal(a, b)
    assert [(d.volume, d.shot, d.attenuation) for d in gt] == gt_o
    assert all(len(d.slices) == 2 for d in gt)


def test_operator_motion_feeds_the_forward(gpu_ctx):
    """The operator's device images moved in place equal the oracle's moved images: its forward
    matches the oracle forward of the oracle-moved series (rel-L2 <= 1e-5)."""
    s = cases.series_case(nx=16, ny=16, nz=3, o=2, nv=3, ncomp=2)
    acq = api.Acquisition(n_coils=4, accel=2, partial_fourier=0.75, pf_mode=api.PartialFourierMode.Scanner,
                          t_line=0.5, t_echo=30.0)
    kw = dict(t_inhom=s["t_inhom"], phase=api.PhaseModel.hbcd_like(), seed=42)
    v2w = np.diag([1.7, 1.7, 3.0, 1.0])
    poses = _poses(3, 9)
    op = api.EpiOperator(s["sim_dims"], s["acq_dims"], 3, s["t2"], s["fmap"], acq, images=s["images"],
                         echo_times_ms=[30.0], grads=0, ctx=gpu_ctx, **kw)
    M.operator_apply_motion(op, v2w, poses)
    out = op.apply_host(None)
    op.close()
    moved = [np.array(a, np.float32) for a in s["images"]]
    O.apply_motion(moved, s["sim_dims"], 3, v2w, np.stack([p.as_array() for p in poses]))
    want = O.series_forward(s["sim_dims"], s["acq_dims"], 3, moved, s["t2"], s["fmap"], acq, echo_times_ms=[30.0], **kw)
    e = np.linalg.norm(out["kspace"] - want) / np.linalg.norm(want)
    assert e <= 1e-5, e
