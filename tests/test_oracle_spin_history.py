"""The spin-history oracle pinned by the reference's own tests (spin_history.rs:455-737): the
static head, in-plane motion, the through-plane jump's double excitation and skip (analytic
ratios), the slow drift, weights and T1 = 0, and the piece operations (split, coalesce, merges
that keep the edges a cut needs, merging at the later time).  CPU only."""
import math

import numpy as np
import pytest

from oracle import oracle
from mrsim_acq_b200.spin_history import Constant, Inversion, Recovery, Replay, Saturation, Slabs, Source

TR, T1, T_SIG, DT = 4.6, 1.33, 3.6, 0.04
IDENTITY = np.eye(4)


def pose_matrix(rot_deg=(0.0, 0.0, 0.0), trans_mm=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0)):
    """`Pose::to_matrix` (motion.rs:55-68): R = Rz Ry Rx about `center`, then the translation."""
    rx, ry, rz = (math.radians(a) for a in rot_deg)
    X = np.array([[1, 0, 0], [0, math.cos(rx), -math.sin(rx)], [0, math.sin(rx), math.cos(rx)]])
    Y = np.array([[math.cos(ry), 0, math.sin(ry)], [0, 1, 0], [-math.sin(ry), 0, math.cos(ry)]])
    Z = np.array([[math.cos(rz), -math.sin(rz), 0], [math.sin(rz), math.cos(rz), 0], [0, 0, 1]])
    R = Z @ (Y @ X)
    c = np.asarray(center, float)
    m = np.eye(4)
    m[:3, :3] = R
    m[:3, 3] = c - R @ c + np.asarray(trans_mm, float)
    return m


def setup(n, nz, shift):
    """A uniform source of nz 1 mm planes, n x n in-plane, and 5 mm slabs (slice k covers planes
    5k..5k+4 when shift is 0)."""
    nv = n * n * nz
    s = np.eye(4)
    s[2, 2] = 5.0
    s[2, 3] = 2.0 + shift
    src = Source((n, n, nz), np.eye(4), np.full(nv, T1, np.float32), np.ones(nv, np.float32),
                 np.zeros(nv, np.uint8), 1)
    return src, Slabs((n, n, nz // 5), s)


def shot_t(v, s):
    return v * TR + T_SIG + DT * s


def run(n, nz, shift, nvol, presat, pose, history=None):
    """nvol volumes of sequential single-slice shots, shot s of volume v at pose(v, s) (a
    (rot, trans) pair or None); per volume and slice the summed (num, den), and the merges."""
    history = history or oracle.SpinHistory
    src, slabs = setup(n, nz, shift)
    ns = slabs.dims[2]
    pulses = [Saturation(v * TR) for v in range(nvol)] if presat else []
    h = history(src, slabs, pulses)
    center = (n / 2.0, n / 2.0, nz / 2.0)
    mat = lambda p: IDENTITY if p is None else pose_matrix(p[0], p[1], center)
    h.prime([(shot_t(0, s) - TR, [s]) for s in range(ns)], mat(pose(0, 0)))
    out = []
    for v in range(nvol):
        vol = []
        for s in range(ns):
            t_read = T_SIG + DT * s
            ref = Recovery(t_read) if presat else Recovery(TR)
            terms = h.excite(shot_t(v, s), mat(pose(v, s)), [s], ref)
            vol.append((float(terms[0].num[0].astype(np.float64).sum()),
                        float(terms[0].den[0].astype(np.float64).sum())))
        out.append(vol)
    return out, h.merges()


def ratio(x):
    return (x[1] + x[0]) / x[1]


def check_static(history=None):
    for presat, shift in [(False, 0.0), (True, 0.0), (False, 0.3), (True, 1.7)]:
        out, merges = run(4, 20, shift, 3, presat, lambda v, s: None, history)
        assert merges == 0
        for v, vol in enumerate(out):
            for s, x in enumerate(vol):
                if shift != 0.0 and s in (0, len(vol) - 1):
                    continue
                assert x[1] > 0.0 and abs(x[0]) <= 1e-6 * x[1], (presat, shift, v, s, x)


def check_jump(history=None):
    e_tr = 1.0 - math.exp(-TR / T1)
    up = ((0.0, 0.0, 0.0), (0.0, 0.0, 0.5))
    down = ((0.0, 0.0, 0.0), (0.0, 0.0, -0.5))
    jump = lambda p: (lambda v, s: p if v == 1 and s >= 2 else None)
    out, merges = run(4, 20, 0.0, 3, False, jump(up), history)
    assert merges == 0
    want = 1.0 - 0.1 * (1.0 - (1.0 - math.exp(-DT / T1)) / e_tr)
    assert abs(ratio(out[1][2]) - want) < 1e-5
    assert abs(want - 0.9031) < 1e-4
    for s in (0, 1):
        assert abs(out[1][s][0]) <= 1e-6 * out[1][s][1]
    r3 = ratio(out[1][3])
    want3 = 1.0 + 0.1 * ((1.0 - math.exp(-(TR + DT) / T1)) / e_tr - 1.0)
    assert abs(r3 - want3) < 1e-6
    out_p, _ = run(4, 20, 0.0, 3, True, jump(up), history)
    ref_p = 1.0 - math.exp(-(T_SIG + 2.0 * DT) / T1)
    want_p = 1.0 - 0.1 * (1.0 - (1.0 - math.exp(-DT / T1)) / ref_p)
    assert abs(ratio(out_p[1][2]) - want_p) < 1e-5
    out, _ = run(4, 20, 0.0, 3, False, jump(down), history)
    want = 1.0 + 0.1 * ((1.0 - math.exp(-2.0 * TR / T1)) / e_tr - 1.0)
    assert abs(ratio(out[2][2]) - want) < 1e-5
    out_p, _ = run(4, 20, 0.0, 3, True, jump(down), history)
    assert abs(out_p[2][2][0]) <= 1e-6 * out_p[2][2][1]


def check_weights_and_t1_zero(history=None):
    history = history or oracle.SpinHistory
    src, slabs = setup(2, 10, 0.0)
    t1 = src.t1.copy()
    w = src.weight.copy()
    t1[2 * 4] = 0.0
    w[1 + 2 * 4] = 3.0
    h = history(Source(src.dims, src.v2w, t1, w, src.cls, 1), slabs)
    ref = Constant(0.5, 0.0)
    a = h.excite(1.0, IDENTITY, [0], ref)
    cell = lambda x, y: x + 2 * y
    assert abs(a[0].den[0][cell(0, 0)] - 0.5 * 4.0 * 0.2) < 1e-6
    assert abs(a[0].num[0][cell(0, 0)] - 0.5 * 4.0 * 0.2) < 1e-6
    assert abs(a[0].den[0][cell(1, 0)] - 0.5 * (4.0 + 3.0) * 0.2) < 1e-6
    assert abs(a[0].num[0][cell(1, 0)] - 0.5 * (4.0 + 3.0) * 0.2) < 1e-6
    doubled = np.full(40, 2.0, np.float32)
    b = h.excite(1.0, IDENTITY, [1], ref, doubled)
    c2 = h.excite(1.0, IDENTITY, [1], ref)
    assert abs(b[0].den[0][cell(1, 1)] - 2.0 * c2[0].den[0][cell(1, 1)]) < 1e-6
    # the same reference as a callable, evaluated per distinct T1 on the host
    h2 = history(Source(src.dims, src.v2w, t1, w, src.cls, 1), slabs)
    a2 = h2.excite(1.0, IDENTITY, [0], lambda t1: 0.5 if t1 > 0 else 0.0)
    assert np.array_equal(a2[0].num, a[0].num) and np.array_equal(a2[0].den, a[0].den)


def check_full_voxel(history=None):
    history = history or oracle.SpinHistory
    src_m = np.eye(4)
    src_m[2, 2] = 2.0
    s = np.eye(4)
    s[2, 3] = -1.0
    src = Source((1, 1, 1), src_m, np.ones(1, np.float32), np.ones(1, np.float32), np.zeros(1, np.uint8), 1)
    h = history(src, Slabs((1, 1, 3), s))
    one = Constant(1.0, 1.0)
    for i in range(8):
        m = pose_matrix(trans_mm=(0.0, 0.0, -0.5 - 0.02 * i))
        h.excite(float(i), m, [0, 1, 2], one)
    terms = h.excite(8.0, IDENTITY, [1], one)
    assert abs(terms[0].den[0][0] - 1.0) < 1e-6
    assert h.merges() > 0


def test_a_static_head_needs_no_correction():
    check_static()


def test_in_plane_motion_needs_no_correction():
    p = ((0.0, 0.0, 3.0), (1.7, -0.6, 0.0))
    out, _ = run(6, 20, 0.0, 3, False, lambda v, s: p if v == 1 and s >= 2 else None)
    for vol in out:
        for x in vol:
            assert abs(x[0]) <= 1e-6 * x[1], x


def test_a_through_plane_jump_double_excites_and_skips():
    check_jump()


def test_a_slow_drift_changes_smoothly():
    pose = lambda v, s: ((0.0, 0.0, 0.0), (0.0, 0.0, 0.3 * shot_t(v, s) / TR))
    out, merges = run(4, 20, 0.0, 10, False, pose)
    assert merges == 0
    for s in range(1, 3):
        for v in range(2, len(out)):
            a, b = ratio(out[v - 1][s]), ratio(out[v][s])
            assert abs(a - b) < 1e-4 and abs(b - 1.0) < 2e-3, (s, v, a, b)


def test_weights_and_t1_zero():
    check_weights_and_t1_zero()


def test_pieces_split_coalesce_and_merge_when_full():
    p = oracle.Pieces()
    assert p.split(0.25) and p.split(0.75) and p.n == 3
    assert p.split(0.25) and p.n == 3, "an existing edge is not split again"
    p.c.mz[1] = 0.0
    p.c.t[1] = 5.0
    p.coalesce()
    assert p.n == 3
    p.c.mz[1] = 1.0
    p.c.t[1] = -math.inf
    p.coalesce()
    assert p.n == 1
    for i in range(1, 8):
        assert p.split(np.float32(i / 8.0))
        p.c.mz[i] = float(i)
    assert not p.split(0.99), "full"
    p.merge_closest(1.0)
    assert p.n == 7


def test_a_cut_keeps_its_existing_edges():
    p = oracle.Pieces()
    for i in range(1, 8):
        assert p.split(i / 8.0)
    for i in range(8):
        p.c.mz[i] = 0.0 if i < 2 else float(np.float32(0.1 * i))
        p.c.t[i] = 1.0 if i < 2 else float(i)
    merges = p.cut(0.125, 0.6875, 1.0)
    assert merges == 1
    assert p.has_edge(0.125) and p.has_edge(0.6875)
    assert p.n == 8


def test_merging_propagates_both_pieces_to_the_later_time():
    p = oracle.Pieces()
    assert p.split(0.5)
    for i in range(8):
        p.c.mz[i] = 0.0
    p.c.t[0] = 0.0
    p.c.t[1] = 4.6
    p.merge_closest(1.33)
    assert p.n == 1 and p.c.t[0] == 4.6
    want = 0.5 * (1.0 - math.exp(-4.6 / 1.33))
    assert abs(p.c.mz[0] - want) < 1e-6 and abs(want - 0.484264) < 1e-6
    q = oracle.Pieces()
    assert q.split(0.5)
    for i in range(8):
        q.c.mz[i] = 0.0
    q.c.t[0] = 0.0
    q.c.t[1] = 4.6
    q.merge_closest(1.33, [Saturation(4.0)])
    want = 0.5 * (1.0 - math.exp(-0.6 / 1.33))
    assert abs(q.c.mz[0] - want) < 1e-6


def test_a_full_voxel_keeps_the_edges_its_excitation_needs():
    check_full_voxel()


def test_replay_through_pulses():
    t1 = 1.2
    m = oracle.spin_replay(0.0, 0.0, 1.0, t1)
    assert abs(m - (1.0 - math.exp(-1.0 / t1))) < 1e-15
    m_inv = oracle.spin_replay(0.0, 0.0, 1.0, t1, [Inversion(0.5, 1.0)])
    a = 1.0 - math.exp(-0.5 / t1)
    want = 1.0 - (1.0 + a) * math.exp(-0.5 / t1)
    assert abs(m_inv - want) < 1e-15
    assert oracle.spin_replay(0.3, 0.0, 1.0, t1, [Saturation(1.0)]) == 0.0
    assert oracle.spin_replay(0.3, -math.inf, 1.0, t1) == 1.0
    assert oracle.spin_replay(0.3, 0.0, 1.0, 0.0) == 0.0


def test_replay_reference_matches_the_static_closed_form():
    """A static head with presaturation: the Replay reference (Mz from 0 at the previous shot
    through the saturation) is the closed form, and the terms vanish."""
    src, slabs = setup(4, 20, 0.0)
    pulses = [Saturation(v * TR) for v in range(3)]
    h = oracle.SpinHistory(src, slabs, pulses)
    h.prime([(shot_t(0, s) - TR, [s]) for s in range(4)], IDENTITY)
    for v in range(3):
        for s in range(4):
            terms = h.excite(shot_t(v, s), IDENTITY, [s], Replay(0.0, shot_t(v, s) - TR))
            num, den = terms[0].num.astype(np.float64).sum(), terms[0].den.astype(np.float64).sum()
            assert abs(num) <= 1e-6 * den


def test_invalid_inputs_are_refused():
    src, slabs = setup(2, 10, 0.0)
    bad = Source(src.dims, src.v2w, src.t1, src.weight, np.full(40, 3, np.uint8), 2)
    with pytest.raises(RuntimeError, match="class 3 of voxel 0 is not below 2"):
        oracle.SpinHistory(bad, slabs)
    h = oracle.SpinHistory(src, slabs)
    with pytest.raises(RuntimeError, match="slice 7 is outside the 2 slabs"):
        h.excite(1.0, IDENTITY, [7], Constant(1.0))
