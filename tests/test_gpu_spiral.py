"""Device NUFFT pair and spiral forwards against the FP64 oracle and the literal sums.

Mirrors the reference's tests: `two_d_pair_matches_the_direct_sums` and
`two_d_integer_points_reduce_to_the_dft` (nufft.rs:370-445), `exact_spiral_forward_*` and
`segmented_forward_matches_the_exact_sum` (spiral.rs:215-330).  The device computes in FP32:
tolerances are rel-L2 <= 1e-5 against FP64 and a max error of a few 1e-6 of the peak (the
reference's FP64 bars are 1e-10 of the total and 1e-6 of the peak)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from cases import Rng
from mrsim_acq_b200 import spiral as S
from mrsim_acq_b200.abi import MrsimError
from mrsim_acq_b200.api import Acquisition, EchoFormation, SliceInput, T2
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TAU = 2.0 * math.pi


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# ---- the 2D NUFFT pair -----------------------------------------------------------------------------
PAIR_GEOMS = [([16, 16], [-8, -8], [16, 16]), ([24, 20], [-6, -10], [12, 20]), ([9, 12], [-4, -6], [9, 12])]


def _pair_inputs():
    rng = Rng(77)
    out = []
    for n, lo, mo in PAIR_GEOMS:
        np_ = 300
        u = np.array([[(rng.unit() - 0.5) * n[0], (rng.unit() - 0.5) * n[1]] for _ in range(np_)])
        w = np.array([complex(rng.unit() - 0.5, rng.unit() - 0.5) for _ in range(np_)])
        c = np.array([complex(rng.unit() - 0.5, rng.unit() - 0.5) for _ in range(mo[0] * mo[1])])
        out.append((n, lo, mo, u, w, c))
    return out


@pytest.mark.parametrize("case", range(3))
@pytest.mark.parametrize("sign", [1, -1])
def test_pair_matches_direct_sums(gpu_ctx, case, sign):
    n, lo, mo, u, w, c = _pair_inputs()[case]
    nu = S.Nufft2(n, lo, mo, 1e-12, ctx=gpu_ctx)
    got1 = nu.type1(u, w, sign).ravel()
    want1 = O.nufft2_direct(1, n, lo, mo, u, w, sign)
    total = np.abs(w).sum()
    assert np.abs(got1 - want1).max() <= 2e-6 * total
    assert rel_l2(got1, want1) <= 1e-5
    got2 = nu.type2(c, u, sign)
    want2 = O.nufft2_direct(2, n, lo, mo, u, c, sign)
    total = np.abs(c).sum()
    assert np.abs(got2 - want2).max() <= 2e-6 * total
    assert rel_l2(got2, want2) <= 1e-5


@pytest.mark.parametrize("case", range(3))
def test_pair_adjoint_identity(gpu_ctx, case):
    n, lo, mo, u, w, c = _pair_inputs()[case]
    nu = S.Nufft2(n, lo, mo, 1e-12, ctx=gpu_ctx)
    rng = Rng(5)
    y = np.array([complex(rng.unit() - 0.5, rng.unit() - 0.5) for _ in range(len(u))])
    a = nu.type2(c, u, 1).astype(np.complex128)
    b = nu.type1(u, y, -1).ravel().astype(np.complex128)
    lhs, rhs = np.vdot(y, a), np.vdot(b, c)
    scale = np.abs(a).sum() * np.abs(y).sum()
    assert abs(lhs - rhs) <= 1e-6 * scale


def test_integer_points_reduce_to_the_dft(gpu_ctx):
    n = [8, 6]
    u = np.array([[a - 4.0, b - 3.0] for b in range(6) for a in range(8)])
    w = np.array([math.sin(i * 0.37) for i in range(48)], dtype=np.complex128)
    got = S.Nufft2(n, [-4, -3], [8, 6], 1e-12, ctx=gpu_ctx).type1(u, w, 1).ravel()
    want = O.nufft2_direct(1, n, [-4, -3], [8, 6], u, w, 1)
    assert np.abs(got - want).max() <= 1e-6 * np.abs(w).sum()
    assert rel_l2(got, want) <= 1e-5


@pytest.mark.parametrize("tol", [1e-3, 1e-6])
def test_width_rule_follows_the_reference_gridding(gpu_ctx, tol):
    # at a loose tolerance the gridding error dominates: the device must reproduce the reference
    # algorithm's own error (kernel width, beta, deapodization), not merely the direct sum
    n, lo, mo, u, w, c = _pair_inputs()[1]
    nu = S.Nufft2(n, lo, mo, tol, ctx=gpu_ctx)
    for sign in (1, -1):
        got = nu.type2(c, u, sign)
        ref = O.nufft2(2, n, lo, mo, tol, u, c, sign)
        direct = O.nufft2_direct(2, n, lo, mo, u, c, sign)
        # the gridding error itself is far above the FP32 arithmetic's: a fixed bound against the
        # FP64 gridding shows the device reproduces it
        assert rel_l2(ref, direct) > 100 * 2e-6 or tol < 1e-3
        assert rel_l2(got, ref) <= 2e-6
        got1 = nu.type1(u, w, sign).ravel()
        ref1 = O.nufft2(1, n, lo, mo, tol, u, w, sign)
        assert rel_l2(got1, ref1) <= 2e-6


def test_type1_spreading_is_deterministic(gpu_ctx):
    """Type 1 spreads without atomics (every fine cell sums its points in point order): the same
    input gives the same bits, also with thousands of points crowding a few cells, where the order
    of floating-point additions would otherwise vary from run to run; and the result still follows
    the FP64 gridding."""
    rng = np.random.default_rng(3)
    n, lo, mo = [32, 32], [-16, -16], [32, 32]
    u = np.concatenate([rng.normal(0.0, 0.4, (6000, 2)), rng.uniform(-16, 16, (2000, 2))])
    w = rng.normal(size=8000) + 1j * rng.normal(size=8000)
    nu = S.Nufft2(n, lo, mo, 1e-6, ctx=gpu_ctx)
    a = nu.type1(u, w, -1)
    for _ in range(3):
        assert np.array_equal(nu.type1(u, w, -1), a)
    assert rel_l2(a.ravel(), O.nufft2(1, n, lo, mo, 1e-6, u, w, -1)) <= 2e-6
    pos = rng.normal(0.0, 0.7, 5000)
    wts = [rng.normal(size=5000) + 1j * rng.normal(size=5000) for _ in range(2)]
    f = S.Nufft1(64, -20, 41, 1e-12, ctx=gpu_ctx)
    b = f.run(pos, wts)
    assert np.array_equal(f.run(pos, wts), b)


def test_pair_errors(gpu_ctx):
    with pytest.raises(MrsimError, match="inside the coarse Nyquist band"):
        S.Nufft2([16, 16], [-9, -8], [16, 16], 1e-12, ctx=gpu_ctx).type2(np.zeros(256), np.zeros((3, 2)), 1)
    with pytest.raises(MrsimError, match="sign"):
        S.Nufft2([16, 16], [-8, -8], [16, 16], 1e-12, ctx=gpu_ctx).type2(np.zeros(256), np.zeros((3, 2)), 2)


def test_pair_empty_points(gpu_ctx):
    nu = S.Nufft2([16, 16], [-8, -8], [16, 16], 1e-12, ctx=gpu_ctx)
    assert nu.type2(np.ones(256), np.zeros((0, 2)), 1).shape == (0,)
    assert np.all(nu.type1(np.zeros((0, 2)), np.zeros(0), 1) == 0)


# ---- spiral forwards -----------------------------------------------------------------------------
def smooth_maps(n, o):
    """spiral.rs `smooth_maps`: Gaussian blobs, a 50 Hz fieldmap, T2, T2', ln A and object phase."""
    s = n * o
    x, y = np.meshgrid(np.arange(s), np.arange(s))
    u, v = (x + 0.5) / s, (y + 0.5) / s
    g = lambda cx, cy, w: np.exp(-((u - cx) ** 2 + (v - cy) ** 2) / (2 * w * w))
    img = (g(0.4, 0.45, 0.08) + 0.6 * g(0.62, 0.6, 0.06)).astype(np.float32).ravel()
    fmap = (-20.0 + 50.0 * u * v).astype(np.float32).ravel()
    t2 = (40.0 + 80.0 * v).astype(np.float32).ravel()
    tp = (30.0 + 60.0 * (1.0 - u)).astype(np.float32).ravel()
    ph = (0.7 * u - 1.1 * v * v).ravel()
    la = (-0.1 - 0.3 * u).ravel()
    return img, fmap, t2, tp, ph, la


def _acq(**kw):
    base = dict(do_relaxation=True, do_distortions=True, noise_variance=0.0, n_spikes=0, n_coils=2, signal_scale=3.0)
    base.update(kw)
    return Acquisition(**base)


def test_exact_at_cartesian_frequencies_is_the_cartesian_forward(gpu_ctx):
    for o in (1, 2):
        nx = ny = 12
        snx, sny = nx * o, ny * o
        img = np.zeros(snx * sny, np.float32)
        img[(3 * o + 1) + snx * (8 * o)] = 1.0
        img[(9 * o) + snx * (2 * o + o // 2)] = 0.37
        phase0 = 0.3 + 0.01 * np.arange(snx * sny)
        inp = SliceInput(compartments=[img], t2=[T2.uniform(math.inf)], fmap=np.zeros(snx * sny, np.float32),
                         sim=(snx, sny), acq_matrix=(nx, ny), phase0=phase0)
        acq = Acquisition(do_relaxation=False, noise_variance=0.0, n_spikes=0, signal_scale=2.5, n_coils=2)
        ks = np.array([[kx - nx // 2, ky - ny // 2] for ky in range(ny) for kx in range(nx)], dtype=np.float64)
        taus = np.zeros(nx * ny)
        for q in range(2):
            cart = O.build_coil_kspace(inp, acq, q, 2).ravel()
            sp = S.spiral_kspace_exact(inp, acq, q, 2, ks, taus, ctx=gpu_ctx)
            peak = np.abs(cart).max()
            assert np.abs(sp - cart).max() <= 2e-6 * peak


def test_exact_decay_and_off_resonance(gpu_ctx):
    nx = 8
    img = np.zeros(nx * nx, np.float32)
    img[3 + nx * 5] = 1.0
    inp = SliceInput(compartments=[img], t2=[T2.of_map(np.full(nx * nx, 80.0, np.float32))],
                     t_inhom=[T2.of_map(np.full(nx * nx, 50.0, np.float32))],
                     fmap=np.full(nx * nx, 40.0, np.float32), sim=(nx, nx), acq_matrix=(nx, nx),
                     phase0=np.full(nx * nx, 0.4))
    la = np.full(nx * nx, -0.2)
    acq = Acquisition(do_relaxation=True, do_distortions=True, noise_variance=0.0, n_spikes=0)
    tau = 3.0
    k = S.spiral_kspace_exact(inp, acq, 0, 1, np.zeros((1, 2)), np.array([tau]), la, ctx=gpu_ctx)[0]
    amp = acq.signal_scale * O.lib().oracle_coil_sensitivity(0, 1, 3.0, 5.0, nx, nx) / (nx * nx)
    mag = amp * math.exp(-0.2 - tau / 80.0 - tau / 50.0)
    ph = 0.4 + TAU * 40.0 * tau / 1000.0
    want = mag * complex(math.cos(ph), math.sin(ph))
    assert abs(k - want) <= 1e-6 * abs(want)
    off = acq.replace(do_relaxation=False, do_distortions=False)
    k0 = S.spiral_kspace_exact(inp, off, 0, 1, np.zeros((1, 2)), np.array([tau]), la, ctx=gpu_ctx)[0]
    assert abs(k0 - amp * complex(math.cos(0.4), math.sin(0.4))) <= 1e-6 * amp


def _spiral_case(n=32, o=2, interleaves=4, dwell=0.008):
    tr = S.spiral_trajectory(n, n, interleaves, 4.0, dwell, 1.2)
    ns = len(tr.tau_ms)
    k = tr.k.reshape(-1, 2)
    tau_idx = np.arange(len(k)) % ns
    return tr, k, tau_idx, tr.tau_ms[tau_idx]


@pytest.mark.parametrize("mode", ["maps", "multi", "plain"])
def test_exact_matches_the_oracle(gpu_ctx, mode):
    n, o = 32, 2
    s = n * o
    tr, k, tau_idx, taus = _spiral_case(n, o)
    img, fmap, t2m, tpm, ph, la = smooth_maps(n, o)
    if mode == "maps":
        inp = SliceInput(compartments=[img], t2=[T2.of_map(t2m)], t_inhom=[T2.of_map(tpm)], fmap=fmap, sim=(s, s),
                         acq_matrix=(n, n), phase0=ph)
        acq, lam = _acq(), la
    elif mode == "multi":
        comps = [img, (0.5 * img[::-1]).copy(), np.where(img > 0.3, 0.2, 0.0).astype(np.float32)]
        inp = SliceInput(compartments=comps, t2=[T2.uniform(80.0), T2.of_map(t2m), T2.uniform(30.0)],
                         t_inhom=[T2.uniform(40.0), T2.uniform(60.0), T2.of_map(tpm)], fmap=fmap, sim=(s, s),
                         acq_matrix=(n, n), phase0=ph)
        acq, lam = _acq(signal_scale=1.5), la
    else:
        inp = SliceInput(compartments=[img], t2=[T2.uniform(80.0)], fmap=fmap, sim=(s, s), acq_matrix=(n, n))
        acq, lam = _acq(do_relaxation=False, do_distortions=False, n_coils=1), None
    for q in range(max(acq.n_coils, 1)):
        got = S.spiral_kspace_exact(inp, acq, q, max(acq.n_coils, 1), k, taus, lam, ctx=gpu_ctx)
        want = O.spiral_kspace_exact(inp, acq, q, max(acq.n_coils, 1), k, taus, lam)
        assert rel_l2(got, want) <= 1e-5
        assert np.abs(got - want).max() <= 5e-6 * np.abs(want).max()


def test_exact_refuses_gradient_echo_and_eddy(gpu_ctx):
    img = np.ones(64, np.float32)
    inp = SliceInput(compartments=[img], t2=[T2.uniform(80.0)], fmap=np.zeros(64, np.float32), sim=(8, 8),
                     acq_matrix=(8, 8))
    with pytest.raises(MrsimError, match="spin-echo train"):
        S.spiral_kspace_exact(inp, Acquisition(echo=EchoFormation.Gradient), 0, 1, np.zeros((1, 2)), np.zeros(1),
                              ctx=gpu_ctx)


def test_segmented_matches_the_exact_sum(gpu_ctx):
    # spiral.rs `segmented_forward_matches_the_exact_sum`: voxel mode and class mode, two coils
    n, o = 32, 2
    s = n * o
    tr, k, tau_idx, taus = _spiral_case(n, o)
    img, fmap, t2m, tpm, ph, la = smooth_maps(n, o)
    acq = _acq()
    inp = SliceInput(compartments=[img], t2=[T2.of_map(t2m)], t_inhom=[T2.of_map(tpm)], fmap=fmap, sim=(s, s),
                     acq_matrix=(n, n), phase0=ph)
    d = 1.0 / t2m.astype(np.float64) + 1.0 / tpm.astype(np.float64)
    rect = S.RateRect((d.min(), d.max()), (float(fmap.min()), float(fmap.max())))
    plan = S.tseg_plan(tr.tau_ms, 4.0, rect)
    for q in range(2):
        got, info = S.spiral_segmented_forward(inp, acq, q, 2, k, tau_idx, tr.tau_ms, 4.0, rect, la, True,
                                               ctx=gpu_ctx)
        assert info["l"] == plan.l and info["bound"] < 1e-7
        exact = O.spiral_kspace_exact(inp, acq, q, 2, k, taus, la)
        peak = np.abs(exact).max()
        assert np.abs(got - exact).max() <= 5e-6 * peak
        assert rel_l2(got, exact) <= 1e-5
        seg = O.spiral_segmented(inp, acq, q, 2, k, tau_idx, plan.tau_l, plan.b, la, True)
        assert np.abs(seg - exact).max() <= 1e-6 * peak  # the certified FP64 segmentation
        assert rel_l2(got, seg) <= 1e-5
    # class: uniform relaxation as a per-sample weight outside the sum
    inp = SliceInput(compartments=[img], t2=[T2.uniform(70.0)], t_inhom=[T2.uniform(45.0)], fmap=fmap, sim=(s, s),
                     acq_matrix=(n, n), phase0=ph)
    rect_c = S.RateRect((0.0, 0.0), rect.f)
    for q in range(2):
        got, _ = S.spiral_segmented_forward(inp, acq, q, 2, k, tau_idx, tr.tau_ms, 4.0, rect_c, None, False,
                                            ctx=gpu_ctx)
        got = got * np.exp(-taus / 70.0 - taus / 45.0)
        exact = O.spiral_kspace_exact(inp, acq, q, 2, k, taus, None)
        peak = np.abs(exact).max()
        assert np.abs(got - exact).max() <= 5e-6 * peak
        assert rel_l2(got, exact) <= 1e-5


def test_segmented_refuses_several_compartments(gpu_ctx):
    img = np.ones(64, np.float32)
    inp = SliceInput(compartments=[img, img], t2=[T2.uniform(80.0)] * 2, fmap=np.zeros(64, np.float32), sim=(8, 8),
                     acq_matrix=(8, 8))
    with pytest.raises(MrsimError, match="one compartment"):
        S.spiral_segmented_forward(inp, Acquisition(), 0, 1, np.zeros((1, 2)), np.zeros(1, np.int64), np.zeros(1), 1.0,
                                   S.RateRect((0.0, 0.0), (0.0, 0.0)), ctx=gpu_ctx)


# ---- the 1D type-1 NUFFT (`Nufft1`, the `kspace` y-stage's transform) -------------------------------
def _direct1(n, k_lo, n_out, pos, w):
    k = (k_lo + np.arange(n_out))[:, None]
    return (np.exp(1j * TAU * k * pos[None, :] / n) * w[None, :]).sum(1)


def test_nufft1_matches_the_direct_sum(gpu_ctx):
    # nufft.rs `matches_the_direct_sum`: the reference's Rng(42) draws, two weight vectors, the
    # FP64 bar 10 tol x total
    rng = Rng(42)
    for n, k_lo, n_out, tol in [(48, -12, 24, 1e-12), (140, -35, 70, 1e-12), (16, -8, 16, 1e-12), (64, -16, 32, 1e-8)]:
        nsrc = 3 * n
        pos = np.array([(rng.unit() - 0.5) * 3.0 * n for _ in range(nsrc)])
        re = np.array([rng.unit() - 0.5 for _ in range(nsrc)])
        im = np.array([rng.unit() - 0.5 for _ in range(nsrc)])
        re2 = np.array([rng.unit() for _ in range(nsrc)])
        w = [re + 1j * im, re2 + 0j]
        got = S.Nufft1(n, k_lo, n_out, tol, ctx=gpu_ctx).run(pos, w)
        for q in range(2):
            want = _direct1(n, k_lo, n_out, pos, w[q])
            total = np.abs(w[q]).sum()
            assert np.abs(got[q] - want).max() <= 10.0 * tol * total, (n, q)


def test_nufft1_integer_positions_reduce_to_the_dft(gpu_ctx):
    n = 32
    pos = np.arange(n, dtype=np.float64)
    w = np.sin(pos * 0.3) + 0j
    got = S.Nufft1(n, -16, 32, 1e-12, ctx=gpu_ctx).run(pos, [w])[0]
    assert np.abs(got - _direct1(n, -16, 32, pos, w)).max() < 1e-10


def test_nufft1_refuses_a_band_outside_nyquist(gpu_ctx):
    with pytest.raises(MrsimError, match="coarse Nyquist band"):
        S.Nufft1(16, -9, 16, 1e-12, ctx=gpu_ctx).run(np.zeros(3), [np.zeros(3, complex)])
