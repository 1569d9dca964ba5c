"""The certified time segmentation with its fits' per-sample work on the device (FP64).

`tseg::plan` (tseg.rs:230-289) builds, for each candidate L and rate-grid size m, a truncated
least-squares fit whose cost grows with the sample times; the device planner runs that part on
the GPU and keeps the Jacobi factorisation and the search over L and m on the host.  Checked
here: the same L, m and node times as the host planner, b_sum and the bound within 1e-5
relative (CUDA's exp / sin / cos may round differently from the host's in the last bit, and the
truncated problem carries that to ~1e-6), and the reference's own certificate test (the bound
holds between grid points) on the device plan's coefficients."""
import time

import numpy as np
import pytest

from mrsim_acq_b200 import spiral as S

pytestmark = pytest.mark.gpu
TAU = 2.0 * np.pi

SPIRAL = (np.arange(2048) + 0.5) * 0.004  # 2048 samples at 4 us, 8.192 ms
CASES = [  # (sample times, readout ms, d, f)
    (SPIRAL, 8.192, (0.0, 0.0), (-80.0, 80.0)),
    (SPIRAL, 8.192, (0.0, 1.0 / 30.0), (-80.0, 80.0)),
    (SPIRAL, 8.192, (0.01, 0.02), (-30.0, 50.0)),
    ((np.arange(200) + 0.5) * 0.02, 4.0, (0.1, 1.1), (-50.0, 50.0)),
    (np.arange(24) * 0.5, 11.5, (0.0, 0.02), (-40.0, 40.0)),  # an EPI echo's line times
    (SPIRAL, 8.192, (0.0, 0.05), (-200.0, 200.0)),  # a wide rectangle: L = 24, a 29 x 29 rate grid
    # a long decay range: L = 48, a 44 x 44 rate grid, so 4 sample times per block, and 37 samples
    # leave a partial last block
    ((np.arange(37) + 0.5) * (8.192 / 37), 8.192, (0.0, 5.0), (-10.0, 10.0)),
]


def _actual(b, tau_l, tau, d, w):
    e = np.exp((-d + 1j * w) * tau)
    segs = np.exp((-d + 1j * w) * tau_l)
    return float(np.abs(e - b @ segs).max())


@pytest.mark.parametrize("case", range(len(CASES)))
def test_device_plan_matches_the_host_plan(case, gpu_ctx):
    tau, t, d, f = CASES[case]
    t0 = time.perf_counter()
    h = S.tseg_plan(tau, t, S.RateRect(d, f))
    t1 = time.perf_counter()
    g = S.tseg_plan(tau, t, S.RateRect(d, f), ctx=gpu_ctx)
    t2 = time.perf_counter()
    print(f"L {g.l} m {g.m}: host {t1 - t0:.3f} s, device {t2 - t1:.3f} s; b_sum {g.b_sum:.6f} vs {h.b_sum:.6f}, "
          f"bound {g.bound:.3e} vs {h.bound:.3e}, max |db| {np.abs(g.b - h.b).max():.1e}")
    assert (g.l, g.m) == (h.l, h.m)
    assert np.array_equal(g.tau_l, h.tau_l)
    assert g.b.shape == h.b.shape
    assert abs(g.b_sum - h.b_sum) <= 1e-5 * h.b_sum
    assert abs(g.bound - h.bound) <= 1e-5 * h.bound
    assert g.grid_err <= 2.0 * h.grid_err + 1e-15
    # b_sum is the largest coefficient sum of the device's own b
    assert abs(np.abs(g.b).sum(1).max() - g.b_sum) <= 1e-12 * g.b_sum
    # the coefficients agree where the rate grid sees them: the interpolants match to far below the bound
    for dd in (d[0], d[1]):
        for ff in (f[0], 0.5 * (f[0] + f[1]), f[1]):
            z = -dd + 1j * TAU * ff / 1000.0
            segs = np.exp(z * g.tau_l)
            assert np.abs(g.b @ segs - h.b @ segs).max() <= 1e-3 * h.bound + 1e-14


@pytest.mark.parametrize("case", [1, 3, 6])
def test_device_plan_bound_holds_between_grid_points(case, gpu_ctx):
    tau, t, d, f = CASES[case]
    p = S.tseg_plan(tau, t, S.RateRect(d, f), ctx=gpu_ctx)
    assert p.bound < 1e-7
    sub = tau[:: max(1, len(tau) // 256)]
    bs = p.b[:: max(1, len(tau) // 256)]
    worst = 0.0
    for a in range(12):
        for c in range(25):
            dd = d[0] + (d[1] - d[0]) * a / 11.0
            ff = f[0] + (f[1] - f[0]) * c / 24.0
            worst = max(worst, _actual(bs, p.tau_l, sub, dd, TAU * ff / 1000.0))
    assert worst <= p.bound, (worst, p.bound)


def test_device_plan_refusals_match_the_host(gpu_ctx):
    from mrsim_acq_b200.abi import MrsimError
    tau = (np.arange(50) + 0.5) * 0.4
    with pytest.raises(MrsimError) as e:
        S.tseg_plan(tau, 20.0, S.RateRect((0.0, 0.0), (-2000.0, 2000.0)), ctx=gpu_ctx)
    assert "64 segments" in str(e.value)
    with pytest.raises(MrsimError, match="not a fieldmap"):
        S.tseg_plan(tau, 20.0, S.RateRect((0.0, 0.0), (1e12, 1e12)), ctx=gpu_ctx)
    p = S.tseg_plan(np.zeros(0), 4.0, S.RateRect((0.0, 0.0), (-10.0, 10.0)), ctx=gpu_ctx)
    assert p.b.shape == (0, p.l) and p.b_sum == 0.0
