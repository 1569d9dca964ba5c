"""The device spin history against the FP64 oracle (spin_history.rs restated): the reference's
own scenarios through the device class, and seeded series with rotations, several classes,
untracked voxels, inversion and saturation pulses, multi-slice shots, per-shot weights, every
kind of reference and batches of shots.  The terms are FP64 sums rounded once to f32 in the
reference's order; the device's `exp` may differ from glibc's in the last bit, so an element
may differ by an f32 rounding: tolerance 2e-6 of the shot's largest denominator."""
import math

import numpy as np
import pytest

from oracle import oracle
from mrsim_acq_b200.spin_history import (Constant, Inversion, Recovery, Replay, Saturation, Shot, Slabs, Source,
                                         SpinHistory)
from tests.test_oracle_spin_history import (IDENTITY, check_full_voxel, check_jump, check_static,
                                            check_weights_and_t1_zero, pose_matrix)

pytestmark = pytest.mark.gpu

TOL = 2e-6


def test_reference_scenarios_on_the_device():
    check_static(SpinHistory)
    check_jump(SpinHistory)
    check_weights_and_t1_zero(SpinHistory)
    check_full_voxel(SpinHistory)


def compare(dev_terms, ora_terms, stats):
    assert (dev_terms is None) == (ora_terms is None)
    if dev_terms is None:
        return
    assert [t.slice for t in dev_terms] == [t.slice for t in ora_terms]
    for d, o in zip(dev_terms, ora_terms):
        scale = max(float(np.abs(o.den).max()), 1e-30)
        for a, b in ((d.num, o.num), (d.den, o.den)):
            err = np.abs(a.astype(np.float64) - b.astype(np.float64))
            assert err.max() <= TOL * scale, (err.max(), scale)
            stats[0] += int(np.count_nonzero(a == b))
            stats[1] += a.size


def random_series(seed, n_classes=3, rot=4.0, jitter=1.2):
    rng = np.random.default_rng(seed)
    nx, ny, nz = 14, 12, 30
    nv = nx * ny * nz
    src_m = np.diag([1.1, 1.2, 1.0, 1.0])
    src_m[:3, 3] = (-0.3, 0.2, 0.1)
    cls = rng.integers(0, n_classes, nv).astype(np.uint8)
    cls[rng.random(nv) < 0.25] = 255
    t1 = rng.uniform(0.3, 2.5, nv).astype(np.float32)
    t1[rng.random(nv) < 0.03] = 0.0
    w = rng.uniform(0.5, 1.5, nv).astype(np.float32)
    slab = np.diag([1.6, 1.5, 3.0, 1.0])
    slab[:3, 3] = (0.1, -0.2, 1.3)
    src = Source((nx, ny, nz), src_m, t1, w, cls, n_classes)
    slabs = Slabs((9, 9, 10), slab)
    pulses = [Inversion(0.7 + 3.0 * v, 0.97) for v in range(6)] + [Saturation(3.0 * v) for v in range(6)]
    center = (nx * 1.1 / 2, ny * 1.2 / 2, nz / 2)
    shots = []
    for v in range(5):
        for g in range(5):
            t = 3.0 * v + 1.0 + 0.2 * g
            pose = (tuple(rng.normal(0, rot / 3, 3)), tuple(rng.normal(0, jitter, 3)))
            m = pose_matrix(pose[0], pose[1], center)
            slices = [g, g + 5] if g % 2 == 0 else [g]
            kind = (v * 5 + g) % 5
            if kind == 0:
                ref = Recovery(3.0)
            elif kind == 1:
                ref = Constant(0.4, 0.1)
            elif kind == 2:
                ref = Replay(0.0, t - 3.0)
            elif kind == 3:
                ref = lambda t1: 1.0 - math.exp(-2.5 / t1) if t1 > 0 else 0.0
            else:
                ref = Recovery(1.5, 0.2)
            weight = rng.uniform(0.0, 2.0, nv).astype(np.float32) if (v + g) % 7 == 3 else None
            shots.append(Shot(t, m, slices, ref, weight))
    prime = [(0.5 + 0.2 * g - 3.0, [g, g + 5]) for g in range(5)]
    return src, slabs, pulses, prime, shots


@pytest.mark.parametrize("seed", [1, 2])
def test_random_series_shot_by_shot(seed):
    src, slabs, pulses, prime, shots = random_series(seed)
    dev = SpinHistory(src, slabs, pulses)
    ora = oracle.SpinHistory(src, slabs, pulses)
    assert dev.n_tracked == ora.n_tracked
    dev.prime(prime, IDENTITY)
    ora.prime(prime, IDENTITY)
    stats = [0, 0]
    for s in shots:
        compare(dev.excite_many([s])[0], ora.excite_many([s])[0], stats)
    assert dev.merges() == ora.merges()
    print(f"bit-identical terms: {stats[0]} of {stats[1]}")
    assert stats[0] >= 0.99 * stats[1]


def test_batches_equal_shot_by_shot():
    """The whole series as one batch (one step launch, one gather) is the shot-by-shot history."""
    src, slabs, pulses, prime, shots = random_series(3)
    one = SpinHistory(src, slabs, pulses)
    many = SpinHistory(src, slabs, pulses)
    one.prime(prime, IDENTITY)
    many.prime(prime, IDENTITY)
    mixed = list(shots)
    mixed.insert(3, Shot(shots[3].t - 0.01, shots[3].transform, [1], None))  # an unread shot inside a batch
    seq = [one.excite_many([s])[0] for s in mixed]
    batch = many.excite_many(mixed)
    assert batch[3] is None and seq[3] is None
    for a, b in zip(seq, batch):
        for x, y in zip(a or [], b or []):
            assert np.array_equal(x.num, y.num) and np.array_equal(x.den, y.den)
    assert one.merges() == many.merges()


def test_merges_under_jitter_match_the_oracle():
    """Thin slabs and through-plane jitter of a few slabs fill the voxels: merges happen on both
    sides, equally often, with the same terms."""
    rng = np.random.default_rng(7)
    nv = 6 * 6 * 8
    src_m = np.diag([1.0, 1.0, 4.0, 1.0])
    src = Source((6, 6, 8), src_m, rng.uniform(0.5, 2.0, nv).astype(np.float32), np.ones(nv, np.float32),
                 np.zeros(nv, np.uint8), 1)
    slab = np.diag([1.0, 1.0, 0.7, 1.0])
    slabs = Slabs((6, 6, 40), slab)
    dev = SpinHistory(src, slabs, [Saturation(5.0)])
    ora = oracle.SpinHistory(src, slabs, [Saturation(5.0)])
    stats = [0, 0]
    for i in range(40):
        m = pose_matrix((0.0, 0.0, 0.0), (0.0, 0.0, float(rng.uniform(-1.5, 1.5))), (3.0, 3.0, 16.0))
        sl = list(range(i % 3, 40, 3))
        s = Shot(0.3 * i, m, sl, Recovery(0.9))
        compare(dev.excite_many([s])[0], ora.excite_many([s])[0], stats)
    assert ora.merges() > 0
    assert dev.merges() == ora.merges()


def test_device_entry_and_invalid_inputs():
    import torch
    src, slabs, pulses, prime, shots = random_series(4)
    dev = SpinHistory(src, slabs, pulses)
    host = SpinHistory(src, slabs, pulses)
    n = dev.terms_size(shots[:4])
    out = torch.zeros(n, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    dev.excite_device(shots[:4], out.data_ptr())
    dev.ctx.synchronize()
    ref = host.excite_many(shots[:4])
    flat = np.concatenate([np.stack([t.num, t.den]).ravel() for terms in ref for t in terms])
    assert np.array_equal(out.cpu().numpy(), flat)
    from mrsim_acq_b200.abi import MrsimError
    with pytest.raises(MrsimError, match="slice 10 is outside the 10 slabs"):
        dev.excite(1.0, IDENTITY, [10], Constant(1.0))
    bad = Source(src.dims, src.v2w, src.t1, src.weight, np.full(src.cls.size, 5, np.uint8), 3)
    with pytest.raises(MrsimError, match="class 5 of voxel 0 is not below 3"):
        SpinHistory(bad, slabs)


def test_coarse_cells_and_rotation_take_the_unstaged_gather():
    """Slab cells of 4 x 4 mm over 1 mm source voxels: a 16 x 8 tile's preimage box holds more
    voxels than a block stages, so the gather walks global memory; tiles at the grid's ragged edge
    (18 x 10 cells); the same terms as the oracle.  Prepared shots give the same terms as lists."""
    rng = np.random.default_rng(11)
    nx, ny, nz = 72, 40, 18
    nv = nx * ny * nz
    cls = np.where(rng.random(nv) < 0.7, 0, 255).astype(np.uint8)
    src = Source((nx, ny, nz), np.eye(4), rng.uniform(0.5, 2.0, nv).astype(np.float32),
                 rng.uniform(0.5, 1.5, nv).astype(np.float32), cls, 1)
    slab = np.diag([4.0, 4.0, 3.0, 1.0])
    slab[:3, 3] = (0.5, 0.5, 1.0)
    slabs = Slabs((18, 10, 6), slab)
    shots = []
    for i in range(6):
        m = pose_matrix((float(rng.normal(0, 8)), float(rng.normal(0, 8)), 20.0), tuple(rng.normal(0, 1.0, 3)),
                        (36.0, 20.0, 9.0))
        shots.append(Shot(0.5 * i, m, [i % 6, (i + 3) % 6], Recovery(1.0)))
    dev = SpinHistory(src, slabs)
    ora = oracle.SpinHistory(src, slabs)
    stats = [0, 0]
    prepared = dev.prepare(shots[:3])
    for a, b in zip(dev.excite_many(prepared), ora.excite_many(shots[:3])):
        compare(a, b, stats)
    for s in shots[3:]:
        compare(dev.excite_many([s])[0], ora.excite_many([s])[0], stats)
    assert dev.merges() == ora.merges()
    assert stats[0] >= 0.99 * stats[1]
