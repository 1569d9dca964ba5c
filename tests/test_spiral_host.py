"""Host plans of the stack-of-spirals path, through the C ABI (no GPU): the spiral trajectory
(reference readout.rs tests `spiral_speed_bound_holds_on_the_continuous_trajectory`,
`spiral_sampling_bound_rejects_undersampled_designs`, `spiral_asl001_numbers`), the certified time
segmentation (tseg.rs tests) and the CPMG echo amplitudes (epg.rs tests)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from mrsim_acq_b200 import spiral as S
from mrsim_acq_b200.abi import MrsimError

TAU = 2.0 * math.pi


# ---- spiral trajectory -------------------------------------------------------------------------
def _u(tr, tau):
    t, tc = tr.readout_ms, tr.tau_c_ms
    return np.where(tau < tc, tau / math.sqrt(tc * t), np.sqrt(tau / t))


def _speed(tr, tau):
    t, tc = tr.readout_ms, tr.tau_c_ms
    du = np.where(tau < tc, 1.0 / math.sqrt(tc * t), 0.5 / np.sqrt(tau * t))
    w = TAU * tr.n_turns * _u(tr, tau)
    return tr.k_max * du * np.sqrt(1.0 + w * w)


def _at(tr, s, tau):
    u = _u(tr, tau)
    th = TAU * (tr.n_turns * u + s / tr.interleaves)
    return np.stack([tr.k_max * u * np.cos(th), tr.k_max * u * np.sin(th)], -1)


@pytest.mark.parametrize("nx,n,t,frac,c", [(64, 8, 4.0, 0.8, 1.2), (64, 8, 4.0, 0.8, 1.0), (32, 1, 10.0, 0.5, 1.0),
                                           (32, 4, 2.0, 0.95, 1.5), (128, 16, 6.0, 0.3, 1.2)])
def test_spiral_speed_bound(nx, n, t, frac, c):
    dmax = t / (TAU * (c * nx / (2.0 * n)) * (nx / 2.0))
    dwell = frac * dmax
    try:
        tr = S.spiral_trajectory(nx, nx, n, t, dwell, c)
    except MrsimError as e:
        assert "too short" in str(e)
        return
    tau = t * np.arange(1, 200_001) / 200_000
    vmax = max(float(_speed(tr, tau).max()), float(_speed(tr, np.array([tr.tau_c_ms * (1 - 1e-12)]))[0]))
    assert vmax * dwell <= 1.0 + 1e-12
    assert vmax * dwell >= 1.0 - 1e-6
    # the samples are the continuous trajectory at (j + 1/2) dwell; within one cycle/FOV per step
    assert np.allclose(tr.tau_ms, (np.arange(len(tr.tau_ms)) + 0.5) * dwell, rtol=0, atol=1e-15)
    for s in range(n):
        il = tr.k[s]
        np.testing.assert_allclose(il, _at(tr, s, tr.tau_ms), rtol=0, atol=1e-12)
        step = np.hypot(*np.diff(il, axis=0).T)
        assert step.max() <= 1.0 + 1e-12
    last = tr.k[0, -1]
    assert math.hypot(*last) <= tr.k_max


def test_spiral_sampling_bound_rejects_undersampled_designs():
    with pytest.raises(MrsimError, match="dwell time must be below"):
        S.spiral_trajectory(64, 64, 1, 3.2, 0.1, 1.0)
    dmax = 4.0 / (TAU * 1.2 * 4.0 * 32.0)
    with pytest.raises(MrsimError, match="dwell time must be below"):
        S.spiral_trajectory(64, 64, 8, 4.0, 1.01 * dmax, 1.2)
    with pytest.raises(MrsimError, match="too short"):
        S.spiral_trajectory(64, 64, 8, 4.0, 0.9999 * dmax, 1.2)
    with pytest.raises(MrsimError, match="square"):
        S.spiral_trajectory(64, 48, 8, 4.0, 0.004, 1.2)
    with pytest.raises(MrsimError):
        S.spiral_trajectory(64, 64, 0, 4.0, 0.004, 1.2)
    with pytest.raises(MrsimError, match="at least 1"):
        S.spiral_trajectory(64, 64, 8, 4.0, 0.004, 0.9)
    with pytest.raises(MrsimError):
        S.spiral_trajectory(64, 64, 8, 4.0, 0.0, 1.2)


def test_spiral_asl001_numbers():
    tr = S.spiral_trajectory(64, 64, 8, 4.0, 0.004, 1.2)
    assert len(tr.tau_ms) == 1000
    want = 1.0 / (4.0 * (1.0 / (32.0 * 0.004) ** 2 - 4.0 * math.pi ** 2 * 4.8 * 4.8 / 16.0))
    assert abs(tr.tau_c_ms - want) < 1e-15
    assert abs(S.spiral_tau_c(64, 8, 4.0, 0.004, 1.2) - want) < 1e-15


# ---- time segmentation ---------------------------------------------------------------------------
def _actual(p, tau, d, w):
    e = np.exp((-d + 1j * w) * tau)
    segs = np.exp((-d + 1j * w) * p.tau_l)
    return float(np.abs(e - p.b @ segs).max())


RECTS = [((0.0, 0.0), (-25.0, 25.0)), ((0.0, 0.0), (-100.0, 150.0)), ((0.01, 0.07), (-25.0, 25.0)),
         ((0.1, 1.1), (0.0, 0.0)), ((0.1, 1.1), (-50.0, 50.0)), ((0.0, 0.0), (10.0, 10.0))]


@pytest.mark.parametrize("d,f", RECTS)
def test_tseg_bound_holds_between_grid_points(d, f):
    t = 4.0
    tau = (np.arange(200) + 0.5) * t / 200
    p = S.tseg_plan(tau, t, S.RateRect(d, f))
    assert p.bound < 1e-7 and p.l <= 64
    worst = 0.0
    for a in range(24):
        for c in range(38):
            dd = d[0] + (d[1] - d[0]) * a / 23.0
            ff = f[0] + (f[1] - f[0]) * c / 37.0
            worst = max(worst, _actual(p, tau, dd, TAU * ff / 1000.0))
    assert worst <= p.bound, (worst, p.bound)
    # b_sum is the largest coefficient sum
    assert abs(np.abs(p.b).sum(1).max() - p.b_sum) <= 1e-12 * p.b_sum


def test_tseg_wide_rectangle_is_refused():
    tau = (np.arange(50) + 0.5) * 0.4
    with pytest.raises(MrsimError) as e:
        S.tseg_plan(tau, 20.0, S.RateRect((0.0, 0.0), (-2000.0, 2000.0)))
    assert "64 segments" in str(e.value) and "-2000" in str(e.value)
    with pytest.raises(MrsimError, match="not a fieldmap"):
        S.tseg_plan(tau, 20.0, S.RateRect((0.0, 0.0), (1e12, 1e12)))


def _split(a):
    c = 134217729.0 * a  # Veltkamp: 2^27 + 1
    hi = c - (c - a)
    return hi, a - hi


def _prod_err(a, b, p):
    """a*b - p exactly for p = fl(a*b) (Dekker's two-product; the fused multiply-add's value)."""
    ah, al = _split(a)
    bh, bl = _split(b)
    return ((ah * bh - p) + ah * bl + al * bh) + al * bl


def _cis_dd(w, t):
    """exp(i w t) with the phase reduced in double-double (tseg.rs `cis_dd`)."""
    tau_lo = 2.4492935982947064e-16
    p = w * t
    e = _prod_err(w, t, p)
    k = float(round(p / TAU))
    kh = k * TAU
    ke = _prod_err(k, TAU, kh)
    r = ((p - kh) - ke) - k * tau_lo + e
    return complex(math.cos(r), math.sin(r))


@pytest.mark.parametrize("f", [(1e4, 1e4), (950.0, 1050.0), (-25.0, 25.0)])
def test_tseg_bound_against_double_double(f):
    tau = np.array([0.002, 0.006, 1.234, 3.998])
    p = S.tseg_plan(tau, 4.0, S.RateRect((0.0, 0.0), f))
    worst = 0.0
    for c in range(41):
        w = TAU * (f[0] + (f[1] - f[0]) * c / 40.0) / 1000.0
        for j, t in enumerate(tau):
            e = _cis_dd(w, t) - sum(p.b[j, i] * _cis_dd(w, tl) for i, tl in enumerate(p.tau_l))
            worst = max(worst, abs(e))
    assert worst <= p.bound


@pytest.mark.parametrize("tau,t", [([0.0], 0.0), ([0.5], 1.0), ([], 4.0), ([0.0, 0.0, 0.0], 0.0)])
def test_tseg_degenerate_sample_sets(tau, t):
    # one sample, none, or a readout of zero length (every node at 0: the truncated least squares
    # drops the repeated columns) still give a certified plan of the right shape
    p = S.tseg_plan(np.asarray(tau, np.float64), t, S.RateRect((0.0, 0.02), (-30.0, 30.0)))
    assert p.bound < 1e-7 and p.l >= 2
    assert p.b.shape == (len(tau), p.l)
    for j, tj in enumerate(tau):
        for d in (0.0, 0.01, 0.02):
            for f in (-30.0, 0.0, 30.0):
                z = -d + 1j * TAU * f / 1000.0
                assert abs(np.exp(z * tj) - p.b[j] @ np.exp(z * p.tau_l)) <= p.bound


def test_tseg_segment_count_rule():
    # L starts at ceil(T (f1 - f0)) + 2 (T in s) and only doubles
    tau = (np.arange(2048) + 0.5) * 0.004
    p = S.tseg_plan(tau, 8.192, S.RateRect((0.0, 0.0), (-80.0, 80.0)))
    l0 = math.ceil(8.192e-3 * 160.0) + 2
    assert p.l in [l0 * (1 << i) for i in range(6)]
    assert np.allclose(p.tau_l, np.linspace(0.0, 8.192, p.l), rtol=0, atol=1e-12)


# ---- EPG -------------------------------------------------------------------------------------------
def _isochromats(n_echoes, esp, b_deg, t1, t2, n_iso):
    dec = lambda dt, t: 1.0 if math.isinf(t) else math.exp(-dt / t)
    e1, e2 = dec(esp / 2, t1), dec(esp / 2, t2)
    th = TAU * np.arange(n_iso) / n_iso
    # after the 90 about x: (0, -1, 0)
    m = np.zeros((n_iso, 3))
    m[:, 1] = -1.0
    b = math.radians(b_deg)
    out = []

    def rz(m, a):
        return np.stack([m[:, 0] * np.cos(a) - m[:, 1] * np.sin(a), m[:, 0] * np.sin(a) + m[:, 1] * np.cos(a), m[:, 2]], 1)

    def ry(m, a):
        return np.stack([m[:, 0] * math.cos(a) + m[:, 2] * math.sin(a), m[:, 1],
                         -m[:, 0] * math.sin(a) + m[:, 2] * math.cos(a)], 1)

    def relax(m):
        return np.stack([m[:, 0] * e2, m[:, 1] * e2, m[:, 2] * e1 + 1.0 - e1], 1)

    for _ in range(n_echoes):
        m = relax(rz(ry(rz(relax(m), th), b), th))
        out.append(math.hypot(m[:, 0].mean(), m[:, 1].mean()))
    return np.array(out)


@pytest.mark.parametrize("t1,t2", [(1330.0, 80.0), (830.0, 70.0), (3000.0, 2000.0), (math.inf, 100.0)])
def test_epg_perfect_refocusing_is_t2_decay(t1, t2):
    la = S.epg_cpmg(30, 12.0, 180.0, t1, t2)
    want = -(np.arange(1, 31)) * 12.0 / t2
    assert np.all(np.abs(np.expm1(la - want)) <= 1e-12)


def test_epg_no_decay():
    assert np.all(S.epg_cpmg(10, 12.0, 180.0, math.inf, math.inf) == 0.0)


@pytest.mark.parametrize("t1,t2", [(1330.0, 80.0), (830.0, 70.0), (3000.0, 2000.0), (1650.0, 165.0)])
@pytest.mark.parametrize("b", [130.0, 111.0, 160.0])
def test_epg_reduced_refocusing_matches_isochromats(t1, t2, b):
    la = S.epg_cpmg(30, 13.4, b, t1, t2)
    iso = _isochromats(30, 13.4, b, t1, t2, 2001)
    assert np.abs(np.exp(la) - iso).max() <= 1e-9
    assert math.exp(la[0]) < 0.99 * math.exp(-13.4 / t2)


def test_epg_extreme_relaxation_is_finite():
    la = S.epg_cpmg(20, 10.0, 130.0, 1000.0, 1e-3)
    assert not np.isnan(la).any() and (la <= 0).all()
    la = S.epg_cpmg(20, 10.0, 180.0, 1e-3, 1e-3)
    assert not np.isnan(la).any()


def test_nufft_width_rule():
    assert S.nufft_kernel_width(1e-12) == 13
    assert S.nufft_kernel_width(1e-13) == 14
    assert S.nufft_kernel_width(1e-1) == 2
    assert S.nufft_kernel_width(1e-30) == 16
