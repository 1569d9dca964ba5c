"""The device spiral reconstruction (FP64) against the FP64 oracle, which restates the reference's
`SpiralRecon` with its own NUFFT-pair normal operator, and the reference's own accuracy tests
(grid_recon.rs:344-636): band-limited and uniform objects, linearity, single modes, rings, and
the segmented-forward pipeline.  The device applies the normal operator as a Toeplitz
convolution: the same operator to the NUFFT tolerance, so parity is to ~1e-9."""
from __future__ import annotations

import math

import numpy as np
import pytest

from mrsim_acq_b200 import spiral as S
from mrsim_acq_b200.abi import MrsimError
from mrsim_acq_b200.api import Acquisition, KspaceWindow, SliceInput, T2
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TAU = 2.0 * math.pi


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def uniform(seed):
    """grid_recon.rs `uniform`: a deterministic uniform stream on (-1/2, 1/2)."""
    s = seed

    def g():
        nonlocal s
        s = (s * 6364136223846793005 + 1442695040888963407) & ((1 << 64) - 1)
        return (s >> 11) / float(1 << 53) - 0.5

    return g


def design(n, il, dw):
    tr = S.spiral_trajectory(n, n, il, 4.0, dw, 1.2)
    k = tr.k.reshape(-1, 2)
    taus = tr.tau_ms[np.arange(len(k)) % len(tr.tau_ms)]
    return tr, k, taus


def band_limited(n, sigma, kb, cx, cy):
    h = n // 2
    ks = [(kx, ky, math.exp(-2.0 * math.pi ** 2 * sigma * sigma * (kx * kx + ky * ky) / (n * n)))
          for ky in range(-h, h) for kx in range(-h, h) if kx * kx + ky * ky <= kb * kb]
    x, y = np.meshgrid(np.arange(n, dtype=np.float64), np.arange(n, dtype=np.float64))
    obj = np.zeros((n, n))
    for kx, ky, c in ks:
        obj += c * np.cos(TAU * (kx * (x - cx) + ky * (y - cy)) / n)
    obj /= np.abs(obj).max()
    return obj.astype(np.float32).ravel()


def plain():
    return Acquisition(do_relaxation=False, do_distortions=False, noise_variance=0.0, n_spikes=0, n_coils=1,
                       signal_scale=1.0)


def exact_data(obj, n, k, taus, o=1, fmap=None, acq=None):
    s = n * o
    inp = SliceInput(compartments=[obj], t2=[T2.uniform(math.inf)],
                     fmap=np.zeros(s * s, np.float32) if fmap is None else fmap, sim=(s, s), acq_matrix=(n, n),
                     phase0=np.zeros(s * s))
    return O.spiral_kspace_exact(inp, acq or plain(), 0, 1, k, taus), inp


# ---- parity with the oracle --------------------------------------------------------------------------
@pytest.mark.parametrize("window", [KspaceWindow.none(), KspaceWindow.hann()])
def test_matches_the_oracle_32(gpu_ctx, window):
    tr, k, taus = design(32, 4, 0.008)
    g = uniform(99)
    d = np.array([[complex(g(), g()) for _ in range(len(k))] for _ in range(2)])
    rec = S.SpiralRecon(k, 32, window, ctx=gpu_ctx)
    want, lam, its, w = O.spiral_recon(k, 32, d, "image", (window.kind, window.a, window.b))
    assert abs(rec.lambda_hi - lam) <= 1e-9 * lam
    assert rel_l2(rec.weights(), w) <= 1e-12
    got = rec.image(d)
    assert rel_l2(got, want) <= 1e-8
    gw, _, _, _ = O.spiral_recon(k, 32, d[:1], "gridding", iterations=0)
    assert rel_l2(rec.gridding(d[:1]), gw) <= 1e-10


def test_matches_the_oracle_odd_grid(gpu_ctx):
    # 33 x 33: odd band (the bin of +16 is +16) and the direct-DFT lines of non-power-of-two sizes
    tr, k, taus = design(33, 4, 0.007)
    g = uniform(7)
    d = np.array([complex(g(), g()) for _ in range(len(k))])
    rec = S.SpiralRecon(k, 33, iterations=40, ctx=gpu_ctx)
    want, lam, _, _ = O.spiral_recon(k, 33, d[None], "image", iterations=40)
    assert abs(rec.lambda_hi - lam) <= 1e-9 * lam
    assert rel_l2(rec.image(d), want[0]) <= 1e-8


def test_rings_match_the_oracle(gpu_ctx):
    tr, k, taus = design(16, 2, 0.01)
    g = uniform(3)
    nc, ring, parts = 4, 2, 2
    d = np.array([[[complex(g(), g()) for _ in range(len(k))] for _ in range(nc)] for _ in range(parts)])
    zs = np.array([[1.0, 0.9, 0.6, 0.45], [0.3, 1.0, 0.8, 0.2]])
    rec = S.SpiralRecon(k, 16, KspaceWindow.tukey(0.4), ctx=gpu_ctx)
    want, _, _, _ = O.spiral_recon(k, 16, d, "rings", (1, 0.4, 0.0), ring=ring, zsens=zs)
    got = rec.reconstruct_rings(d, ring, zs)
    assert rel_l2(got, want) <= 1e-8
    # `reconstruct`: rings of the coil count, unit z factors
    one = rec.reconstruct(d[0, :2], Acquisition(n_coils=2))
    want1, _, _, _ = O.spiral_recon(k, 16, d[:1, :2], "rings", (1, 0.4, 0.0), ring=2, zsens=np.ones((1, 2)))
    assert rel_l2(one, want1[0]) <= 1e-8


# ---- the reference's accuracy tests ---------------------------------------------------------------
@pytest.mark.parametrize("n,il,dw,sigma,kb", [(32, 4, 0.008, 3.0, 10.0), (64, 8, 0.004, 6.0, 20.0)])
def test_reconstructs_band_limited_and_uniform_objects(gpu_ctx, n, il, dw, sigma, kb):
    tr, k, taus = design(n, il, dw)
    rec = S.SpiralRecon(k, n, ctx=gpu_ctx)
    h = n / 2
    objs = [band_limited(n, sigma, kb, cx, cy) for cx, cy in [(h, h), (0.0, h), (0.0, 0.0)]]
    data = np.array([exact_data(o, n, k, taus)[0] for o in objs])
    imgs = rec.reconstruct_rings(data[:, None, :], 1, np.ones((3, 1)))
    for o, img in zip(objs, imgs):
        err = np.abs(img.ravel() - o.astype(np.float64)).max()
        assert err <= 1e-2, err
    d, _ = exact_data(np.ones(n * n, np.float32), n, k, taus)
    c = (n // 2) * (n + 1)
    gr = rec.gridding(d).ravel()
    assert abs(gr[c].real - 1.0) < 1e-9 and abs(gr[c].imag) < 1e-9
    img = rec.reconstruct(d[None], plain()).ravel()
    assert abs(img[c] - 1.0) <= 1e-3


def test_reconstruction_is_linear(gpu_ctx):
    n = 32
    tr, k, taus = design(n, 4, 0.008)
    rec = S.SpiralRecon(k, n, KspaceWindow.hann(), ctx=gpu_ctx)
    g = uniform(99)
    d1 = np.array([complex(g(), g()) for _ in range(len(k))])
    d2 = np.array([complex(g(), g()) for _ in range(len(k))])
    a, b, ab = rec.image(np.stack([d1, d2, d1 + d2]))
    peak = np.abs(ab).max()
    assert np.abs(ab - a - b).max() <= 1e-12 * peak


def _worst_single_mode(rec, n, k, ks):
    h = n // 2
    worst = 0.0
    x0, y0 = np.meshgrid(np.arange(n), np.arange(n))
    xs = []
    for kx, ky in ks:
        a = TAU * (kx * x0 + ky * y0) / n
        for v in (np.cos(a), np.sin(a)):
            if np.abs(v).max() < 1e-12:
                continue
            xs.append(v.ravel())
    xs = np.array(xs, dtype=np.complex128)
    data = np.array([O.nufft2(2, [n, n], [-h, -h], [n, n], 1e-12, k, x, 1) / (n * n) for x in xs])
    imgs = rec.image(data).reshape(len(xs), -1)
    for img, x in zip(imgs, xs):
        worst = max(worst, float(np.abs(img - x).max()))
    return worst


def _half_disc(kb):
    return [(kx, ky) for ky in range(kb + 1) for kx in range(-kb, kb + 1)
            if kx * kx + ky * ky <= kb * kb and not (ky == 0 and kx < 0)]


def test_every_single_mode_of_the_declared_domain(gpu_ctx):
    tr, k, _ = design(16, 2, 0.01)
    rec = S.SpiralRecon(k, 16, ctx=gpu_ctx)
    assert _worst_single_mode(rec, 16, k, _half_disc(5)) <= 1e-2
    tr, k, _ = design(32, 4, 0.008)
    rec = S.SpiralRecon(k, 32, ctx=gpu_ctx)
    assert _worst_single_mode(rec, 32, k, [(5, 0), (7, 7), (-7, 7), (6, 8), (10, 0), (0, 10)]) <= 1e-2


def test_uniform_off_resonance_pipeline(gpu_ctx):
    # the device segmented forward (FP32) through the device reconstruction against the
    # reconstruction of FP64 exact-sum samples (the reference's bar is 1e-6 of peak in FP64)
    n, o = 32, 2
    s = n * o
    tr, k, taus = design(n, 4, 0.008)
    idx = np.arange(len(k)) % len(tr.tau_ms)
    i = np.arange(s * s)
    obj = np.exp(-(((i % s) - 27.0) ** 2 + ((i // s) - 33.0) ** 2) / 60.0).astype(np.float32)
    fmap = np.full(s * s, 30.0, np.float32)
    acq = plain().replace(do_distortions=True)
    b, inp = exact_data(obj, n, k, taus, o=o, fmap=fmap, acq=acq)
    a, _ = S.spiral_segmented_forward(inp, acq, 0, 1, k, idx, tr.tau_ms, 4.0, S.RateRect((0.0, 0.0), (30.0, 30.0)),
                                      None, False, ctx=gpu_ctx)
    rec = S.SpiralRecon(k, n, ctx=gpu_ctx)
    ia, ib = rec.image(np.stack([a.astype(np.complex128), b]))
    peak = np.abs(ib).max()
    assert np.abs(ia - ib).max() <= 1e-5 * peak


def test_parameter_errors(gpu_ctx):
    tr, k, _ = design(16, 2, 0.01)
    with pytest.raises(MrsimError, match="interval ratio"):
        S.SpiralRecon(k, 16, kappa=1.0, ctx=gpu_ctx)
    rec = S.SpiralRecon(k, 16, iterations=5, ctx=gpu_ctx)
    with pytest.raises(MrsimError, match="rings of 3"):
        rec.reconstruct_rings(np.zeros((4, len(k))), 3, np.ones(4))
