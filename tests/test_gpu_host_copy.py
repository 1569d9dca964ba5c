"""Large host copies through the page-locked staging slots.

A series big enough that its image arrays and its magnitude / phase outputs (8.65 MB each: one
whole 8 MiB slot and a remainder) take the staged path must give, bit for bit, what the same call
gives with page-locked arrays (the direct copies), and echoes that share one set of image arrays
(one upload) must give what echoes with separate copies of them give."""
import ctypes as C

import numpy as np
import pytest
import torch

from mrsim_acq_b200 import abi, api
from mrsim_acq_b200.abi import check, lib
from mrsim_acq_b200.api import Acquisition, AcquisitionInput, PhaseModel
from tests import cases

pytestmark = pytest.mark.gpu
SLOT = 8 << 20


def _pinned(n):
    return torch.empty(n, dtype=torch.float32, pin_memory=True).numpy()


def _pinned_copy(a):
    h = _pinned(a.size)
    h[...] = np.ravel(a)
    return h


def _echoes(ai, per_echo, acq, echoes, ctx, alloc):
    """`simulate_acquisition_echoes` into output arrays from `alloc` (pageable or page-locked)."""
    keep = api._Keep()
    ci = api.acquisition_input_c(ai, keep, with_images=False)
    ne = len(echoes)
    ipe = (C.POINTER(abi.c_f32p) * ne)()
    for e, imgs in enumerate(per_echo):
        ipe[e] = keep.ptrs([np.ravel(a) for a in imgs])
    nx, ny, nz = ai.acq_dims
    n = nx * ny * nz * ai.n_volumes
    mags = [alloc(n) for _ in range(ne)]
    phs = [alloc(n) for _ in range(ne)]
    mp = (abi.c_f32p * ne)(*[m.ctypes.data_as(abi.c_f32p) for m in mags])
    pp = (abi.c_f32p * ne)(*[p.ctypes.data_as(abi.c_f32p) for p in phs])
    check(lib().mrsim_simulate_acquisition_echoes(ctx.handle, C.byref(ci), ipe, C.byref(acq.to_c()),
                                                  keep.f64(echoes), ne, None, None, mp, pp))
    return mags + phs


def test_staged_copies_match_direct_copies_and_shared_uploads(gpu_ctx):
    s = cases.series_case(nx=128, ny=128, nz=4, o=1, nv=33, ncomp=2)
    acq = Acquisition(n_coils=4, t_line=0.25, t_echo=40.0, signal_scale=100.0, noise_variance=1e-3)
    ai = AcquisitionInput(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"],
                          t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=3)
    nbytes = s["images"][0].nbytes
    assert nbytes > SLOT and nbytes % SLOT, "the case must take the staged path with a partial last slot"
    echoes = [40.0, 60.0]
    pageable = lambda n: np.zeros(n, np.float32)  # noqa: E731
    staged = _echoes(ai, [s["images"]] * 2, acq, echoes, gpu_ctx, pageable)
    assert staged[0].nbytes > SLOT and staged[0].nbytes % SLOT
    direct = _echoes(ai, [[_pinned_copy(im) for im in s["images"]]] * 2, acq, echoes, gpu_ctx, _pinned)
    separate = _echoes(ai, [[im.copy() for im in s["images"]] for _ in echoes], acq, echoes, gpu_ctx, pageable)
    assert np.abs(staged[0]).max() > 0
    for a, b, c in zip(staged, direct, separate):
        assert np.array_equal(a, b), "staged and direct copies differ"
        assert np.array_equal(a, c), "a shared upload and separate uploads differ"
