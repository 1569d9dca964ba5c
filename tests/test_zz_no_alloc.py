"""The forward entry point that allocates no device memory (`mrsim_build_coil_kspaces_noalloc`).

It exists for callers that may not call cudaMalloc while they run — a host whose device memory is
all in its own pool or arena, or a pipeline that pre-allocates everything at start-up so that no
call can stall or fail on an allocation.  Its intermediates live in static device arrays that
every call shares, so this test checks two calls in a row on different slices, each against the
FP64 oracle's `build_coil_kspace` (per coil, noise and spikes off) and against the allocating
entry point (`mrsim_build_coil_kspaces`), at the relative-L2 tolerance the other GPU tests use.
It also checks the refusals: a slice above the static limits, and host memory passed where the
entry wants device pointers.  The test owns the device buffers it passes (torch tensors).
This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from mrsim_acq_b200 import abi, api
from oracle import oracle
from tests import cases

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _noalloc(inp, acq):
    import torch
    snx, sny = inp.sim
    nx, ny = inp.acq_matrix
    nc = max(acq.n_coils, 1)
    dev = torch.device("cuda", 0)
    comps = torch.from_numpy(np.stack([np.ravel(c) for c in inp.compartments]).astype(np.float32)).to(dev)
    fmap = torch.from_numpy(np.ravel(inp.fmap).astype(np.float32)).to(dev)
    ph = torch.from_numpy(np.ravel(inp.phase0).astype(np.float64)).to(dev) if inp.phase0 is not None else None
    out = torch.zeros(nc * ny * nx * 2, dtype=torch.float32, device=dev)
    keep = api._Keep()
    s = api.slice_input_c(inp, keep)  # host struct; now point its data at the device buffers
    plane = snx * sny
    ptrs = (abi.c_f32p * len(inp.compartments))()
    for c in range(len(inp.compartments)):
        ptrs[c] = C.cast(comps.data_ptr() + 4 * c * plane, abi.c_f32p)
    s.compartments = ptrs
    s.fmap = C.cast(fmap.data_ptr(), abi.c_f32p)
    s.phase0 = C.cast(ph.data_ptr(), abi.c_f64p) if ph is not None else None
    torch.cuda.synchronize()
    abi.check(abi.lib().mrsim_build_coil_kspaces_noalloc(C.byref(s), C.byref(acq.to_c()), None,
                                                         C.cast(out.data_ptr(), abi.c_f32p)))
    got = out.cpu().numpy().view(np.complex64).reshape(nc, ny, nx)
    del keep
    return got


def _check(inp, acq):
    acq = acq.replace(noise_variance=0.0, n_spikes=0)
    got = _noalloc(inp, acq)
    nc = max(acq.n_coils, 1)
    want = np.stack([oracle.build_coil_kspace(inp, acq, q, nc) for q in range(nc)])
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err <= TOL, f"against the FP64 oracle: {err:.2e}"
    other = api.build_coil_kspaces(inp, acq)
    err2 = np.linalg.norm(got - other) / np.linalg.norm(other)
    assert err2 <= TOL, f"against the allocating entry: {err2:.2e}"


def test_noalloc_matches_the_oracle_on_two_calls_in_a_row():
    golden = cases.golden_cases()
    # a 4-coil GRAPPA-sampled 17x70 slice, then an eddy 16x40 slice: the second call must not see
    # the first call's contents of the shared static arrays
    _check(golden[8][1], golden[8][2])
    _check(golden[17][1], golden[17][2])


def _struct_on_device(inp, keep, dev_comps, dev_fmap, plane=0):
    """The slice struct with its plane pointers on device buffers (contiguous planes `plane`
    floats apart; never read: the call refuses before any copy or launch)."""
    s = api.slice_input_c(inp, keep)
    ptrs = (abi.c_f32p * len(inp.compartments))()
    for c in range(len(inp.compartments)):
        ptrs[c] = C.cast(dev_comps.data_ptr() + 4 * c * plane, abi.c_f32p)
    s.compartments = ptrs
    keep.append(ptrs)
    s.fmap = C.cast(dev_fmap.data_ptr(), abi.c_f32p)
    s.phase0 = None
    return s


def test_noalloc_rejects_a_slice_above_its_limits():
    import torch
    inp, acq = cases.golden_cases()[1][1:]
    big = api.SliceInput(compartments=[np.zeros(1, np.float32)], t2=[api.T2.uniform(80.0)],
                         fmap=np.zeros(1, np.float32), sim=(1024, 1024), acq_matrix=(512, 512))
    keep = api._Keep()
    small = torch.zeros(16, dtype=torch.float32, device="cuda")
    s = _struct_on_device(big, keep, small, small)
    out = torch.zeros(2, dtype=torch.float32, device="cuda")
    rc = abi.lib().mrsim_build_coil_kspaces_noalloc(C.byref(s), C.byref(acq.to_c()), None,
                                                    C.cast(out.data_ptr(), abi.c_f32p))
    assert rc == 1
    assert "static limit" in abi.lib().mrsim_last_error().decode()


def test_noalloc_rejects_host_pointers():
    import torch
    inp, acq = cases.golden_cases()[1][1:]
    keep = api._Keep()
    s = api.slice_input_c(inp, keep)  # every data pointer is host memory
    out = torch.zeros(2, dtype=torch.float32, device="cuda")
    rc = abi.lib().mrsim_build_coil_kspaces_noalloc(C.byref(s), C.byref(acq.to_c()), None,
                                                    C.cast(out.data_ptr(), abi.c_f32p))
    assert rc == 1
    assert "device memory" in abi.lib().mrsim_last_error().decode()
    # a host output buffer is refused too, with device inputs
    snx, sny = inp.sim
    dev = torch.zeros(len(inp.compartments) * snx * sny, dtype=torch.float32, device="cuda")
    s2 = _struct_on_device(inp, keep, dev, dev, plane=snx * sny)
    host_out = np.zeros(2, np.float32)
    rc = abi.lib().mrsim_build_coil_kspaces_noalloc(C.byref(s2), C.byref(acq.to_c()), None,
                                                    host_out.ctypes.data_as(abi.c_f32p))
    assert rc == 1
    assert "kspace" in abi.lib().mrsim_last_error().decode()
