"""GPU parity of the whole per-slice pipeline and the series drivers against the reference's
golden record (f32, bit-exact in the reference; here relative L2 <= 1e-5, FP32 arithmetic) and
against the FP64 oracle for every option the record does not exercise."""
import pathlib

import numpy as np
import pytest

from mrsim_acq_b200 import api
from mrsim_acq_b200.abi import MrsimError
from mrsim_acq_b200.api import Acquisition, AcquisitionInput, AcquisitionOptions, PartialFourierMode, PhaseModel, T2
from oracle import oracle
from tests import cases

pytestmark = pytest.mark.gpu
TOL = 1e-5
GOLD = pathlib.Path(__file__).resolve().parent / "golden" / "p4_baseline" / "default"
GOLD_KSPACE = GOLD.parent / "kspace"


def rel_l2(a, b):
    n = np.linalg.norm(np.ravel(b))
    return np.linalg.norm(np.ravel(a) - np.ravel(b)) / (n if n > 0 else 1.0)


@pytest.mark.parametrize("idx", range(39))
def test_golden_slices_match_the_reference_record(idx, gpu_ctx):
    name, inp, acq = cases.golden_cases()[idx]
    got = api.simulate_slice(inp, acq, ctx=gpu_ctx)
    want = np.fromfile(GOLD / f"{name}.bin", dtype="<f4").view(np.complex64).reshape(got.shape)
    assert rel_l2(got, want) <= TOL, f"{name}: rel-L2 {rel_l2(got, want):.2e}"


@pytest.mark.parametrize("idx", range(39))
def test_golden_slices_match_the_kspace_build_record(idx, gpu_ctx):
    """The reference's `kspace` build record (NUFFT y-stage, FFT x-stage and inverse)."""
    name, inp, acq = cases.golden_cases()[idx]
    got = api.simulate_slice(inp, acq, ctx=gpu_ctx)
    want = np.fromfile(GOLD_KSPACE / f"{name}.bin", dtype="<f4").view(np.complex64).reshape(got.shape)
    assert rel_l2(got, want) <= TOL, f"{name}: rel-L2 {rel_l2(got, want):.2e}"


@pytest.mark.parametrize("idx", range(2))
def test_golden_series_match_the_kspace_build_record(idx, gpu_ctx):
    name, inp, acq = cases.golden_series_inputs()[idx]
    mag, ph = api.simulate_acquisition_oversampled(inp, acq, ctx=gpu_ctx)
    raw = np.fromfile(GOLD_KSPACE / f"{name}.bin", dtype="<f4")
    gm, gp = raw[: raw.size // 2], raw[raw.size // 2:]
    assert rel_l2(mag * np.exp(1j * ph), gm * np.exp(1j * gp)) <= TOL


@pytest.mark.parametrize("idx", range(2))
def test_golden_series_match_the_reference_record(idx, gpu_ctx):
    name, inp, acq = cases.golden_series_inputs()[idx]
    mag, ph = api.simulate_acquisition_oversampled(inp, acq, ctx=gpu_ctx)
    raw = np.fromfile(GOLD / f"{name}.bin", dtype="<f4")
    gm, gp = raw[: raw.size // 2], raw[raw.size // 2:]
    assert rel_l2(mag, gm) <= TOL, rel_l2(mag, gm)
    assert rel_l2(mag * np.exp(1j * ph), gm * np.exp(1j * gp)) <= TOL


def test_slice_captures_match_the_oracle(gpu_ctx):
    name, inp, acq = cases.golden_cases()[10]  # "everything" 17x70 o2: GRAPPA, PF, ghost, eddy
    got = api.simulate_slice_full(inp, acq, ctx=gpu_ctx)
    want = oracle.simulate_slice_full(inp, acq)
    for key in ("combined", "acquired", "reconstructed", "coil_images"):
        assert rel_l2(got[key], want[key]) <= TOL, (key, rel_l2(got[key], want[key]))
    assert np.allclose(got["sensitivities"], want["sensitivities"], rtol=1e-6)
    assert np.array_equal(got["mask"], api.sampling_mask(*inp.acq_matrix, acq))


def _series(nv=3, nz=3, maps=False):
    s = cases.series_case(nx=16, ny=16, nz=nz, o=2, nv=nv, ncomp=2, maps=maps)
    inp = AcquisitionInput(sim_dims=s["sim_dims"], acq_dims=s["acq_dims"], n_volumes=nv, images=s["images"],
                           t2=s["t2"], fmap=s["fmap"], t_inhom=s["t_inhom"],
                           eddy_drive=[(0.4, -0.3, 0.6) if g % 2 else None for g in range(nv)],
                           prep_drive=[(1000.0, (0.6, 0.8, 0.0)) if g != 1 else None for g in range(nv)],
                           phase=PhaseModel.hbcd_like(), seed=11,
                           noise_sigma=np.full(16 * 16 * nz, 0.3, np.float32))
    acq = Acquisition(n_coils=4, accel=2, acs_lines=8, partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner,
                      t_line=0.5, t_echo=40.0, ghost_offset=0.02, eddy_strength=0.5, eddy_quad=0.05,
                      eddy_phase=0.01, noise_variance=1.0, n_spikes=1, spike_amplitude=0.2,
                      window=api.KspaceWindow.hann())
    return inp, acq


def _oracle_series(inp, acq, opts=None, exc=None, rec=None):
    o = {}
    if opts is not None:
        o = dict(slice_z=opts.slice_z, nz_full=opts.nz_full, kspace_slices=opts.kspace_slices,
                 acquired=opts.acquired, reconstructed=opts.reconstructed, coil_images=opts.coil_images,
                 t_echo_per_volume=opts.t_echo_per_volume, grappa_calibration=opts.grappa_calibration)
    return oracle.acquire_volumes_complex(inp.sim_dims, inp.acq_dims, inp.n_volumes, inp.images, inp.t2, inp.fmap, acq,
                                          inp.seed if exc is None else exc, inp.seed if rec is None else rec,
                                          options=o, t_inhom=inp.t_inhom, eddy_drive=inp.eddy_drive,
                                          prep_drive=inp.prep_drive, phase=inp.phase, noise_sigma=inp.noise_sigma)


def test_series_with_every_option_matches_the_oracle(gpu_ctx):
    inp, acq = _series(maps=True)
    opts = AcquisitionOptions(kspace_slices=[2, 0], acquired=True, reconstructed=True, coil_images=True,
                              t_echo_per_volume=[40.0, 45.0, 40.0])
    got = api.simulate_acquisition_complex(inp, acq, opts, ctx=gpu_ctx)
    want = _oracle_series(inp, acq, opts)
    z = got["re"] + 1j * got["im"]
    w = want["re"] + 1j * want["im"]
    assert rel_l2(z, w) <= TOL, rel_l2(z, w)
    for key in ("acquired", "reconstructed", "coil_images", "combined"):
        gw = want[key].view(np.complex64).reshape(got[key].shape)
        assert rel_l2(got[key], gw) <= TOL, (key, rel_l2(got[key], gw))
    assert np.array_equal(got["mask"], want["mask"].reshape(16, 16).astype(bool))


def test_a_slab_reproduces_its_slices_of_the_full_series(gpu_ctx):
    """kspace.rs:4353: slice_z/nz_full make a slab see the full run's seeds and z terms."""
    inp, acq = _series(nv=2, nz=4)
    full = api.simulate_acquisition_complex(inp, acq, ctx=gpu_ctx)
    nx, ny, nz = inp.acq_dims
    snx, sny, _ = inp.sim_dims
    keep = [1, 3]
    imgs = [a.reshape(nz, sny * snx * inp.n_volumes)[keep].reshape(-1) for a in inp.images]
    slab = AcquisitionInput(sim_dims=(snx, sny, 2), acq_dims=(nx, ny, 2), n_volumes=2, images=imgs, t2=inp.t2,
                            fmap=inp.fmap.reshape(nz, -1)[keep].reshape(-1), t_inhom=inp.t_inhom,
                            eddy_drive=inp.eddy_drive, prep_drive=inp.prep_drive, phase=inp.phase, seed=inp.seed,
                            noise_sigma=inp.noise_sigma.reshape(nz, -1)[keep].reshape(-1))
    acq_nograppa = acq.replace(accel=1)  # GRAPPA fits on the slab's own slices; compare without it
    full = api.simulate_acquisition_complex(inp, acq_nograppa, ctx=gpu_ctx)
    part = api.simulate_acquisition_complex(slab, acq_nograppa, AcquisitionOptions(slice_z=keep, nz_full=nz),
                                            ctx=gpu_ctx)
    fz = (full["re"] + 1j * full["im"]).reshape(nz, ny * nx, 2)[keep]
    pz = (part["re"] + 1j * part["im"]).reshape(2, ny * nx, 2)
    assert rel_l2(pz, fz) <= TOL


def test_echoes_match_the_oracle_with_salted_receiver_seeds(gpu_ctx):
    inp, acq = _series(nv=2, nz=2)
    tes = [30.0, 50.0]
    imgs = [inp.images, [0.8 * a for a in inp.images]]
    got = api.simulate_acquisition_echoes(inp, imgs, acq, tes, ctx=gpu_ctx)
    for e, te in enumerate(tes):
        salt = int(oracle.lib().oracle_echo_salt(e))
        inp_e = AcquisitionInput(**{**inp.__dict__, "images": imgs[e]})
        w = _oracle_series(inp_e, acq.replace(t_echo=te), exc=inp.seed, rec=inp.seed ^ salt)
        wz = w["re"] + 1j * w["im"]
        mag, ph = got[e]
        assert rel_l2(mag * np.exp(1j * ph), wz) <= TOL, e


def test_explicit_grappa_calibration_matches_the_oracle(gpu_ctx):
    inp, acq = _series(nv=2, nz=2)
    snx, sny, nz = inp.sim_dims
    cal = [a.reshape(-1, inp.n_volumes)[:, 1].copy() * 1.1 for a in inp.images]
    opts = AcquisitionOptions(grappa_calibration=(cal, 99))
    got = api.simulate_acquisition_complex(inp, acq, opts, ctx=gpu_ctx)
    want = _oracle_series(inp, acq, opts)
    assert rel_l2(got["re"] + 1j * got["im"], want["re"] + 1j * want["im"]) <= TOL


def test_progress_counts_every_volume(gpu_ctx):
    inp, acq = _series(nv=3, nz=1)
    seen = []
    api.simulate_acquisition_complex(inp, acq, AcquisitionOptions(progress=lambda d, t: seen.append((d, t))),
                                     ctx=gpu_ctx)
    assert seen == [(1, 3), (2, 3), (3, 3)]


def test_invalid_inputs_fail_with_the_reference_messages(gpu_ctx):
    inp, acq = _series(nv=1, nz=1)
    with pytest.raises(MrsimError, match="trf = .* ms <= 0 on an acquired line"):
        api.simulate_acquisition_complex(inp, acq.replace(t_echo=1.0), ctx=gpu_ctx)
    bad = AcquisitionInput(**{**inp.__dict__, "t2": [T2.of_map(np.zeros(32 * 32, np.float32)), inp.t2[1]]})
    with pytest.raises(MrsimError, match="T2 map for compartment 0: T2 map value 0 at index 0 is not strictly positive"):
        api.simulate_acquisition_complex(bad, acq, ctx=gpu_ctx)
    with pytest.raises(MrsimError, match="echo times must increase strictly"):
        api.simulate_acquisition_echoes(inp, [inp.images, inp.images], acq, [40.0, 30.0], ctx=gpu_ctx)
    with pytest.raises(MrsimError, match="slice_z entries must be below nz_full 1"):
        api.simulate_acquisition_complex(inp, acq, AcquisitionOptions(slice_z=[3], nz_full=1), ctx=gpu_ctx)


@pytest.mark.parametrize("maps", [False, True])
def test_series_with_eight_ring_coils_matches_the_oracle(maps, gpu_ctx):
    """Eight ring coils put the series on the coil-class forward (class rows through the x-stage);
    GRAPPA, noise, spikes, recon and the coil combine downstream of it against the oracle."""
    inp, acq = _series(nv=2, nz=2, maps=maps)
    acq = acq.replace(n_coils=8)
    opts = AcquisitionOptions(kspace_slices=[1], acquired=True, reconstructed=True, coil_images=True)
    got = api.simulate_acquisition_complex(inp, acq, opts, ctx=gpu_ctx)
    want = _oracle_series(inp, acq, opts)
    z = got["re"] + 1j * got["im"]
    w = want["re"] + 1j * want["im"]
    assert rel_l2(z, w) <= TOL, rel_l2(z, w)
    for key in ("acquired", "reconstructed", "coil_images", "combined"):
        gw = want[key].view(np.complex64).reshape(got[key].shape)
        assert rel_l2(got[key], gw) <= TOL, (key, rel_l2(got[key], gw))


def test_magnitude_and_phase_split_on_the_device(gpu_ctx):
    """`simulate_acquisition_oversampled` returns magnitude and phase from the device output pass
    (kspace.rs:1839-1846): the magnitude is sqrt(re^2 + im^2) in f32 bit for bit, the phase
    atan2(im, re) within 2 f32 ulp of the host's."""
    name, inp, acq = cases.golden_series_inputs()[0]
    out = api.simulate_acquisition_complex(inp, acq, ctx=gpu_ctx)
    mag, ph = api.simulate_acquisition_oversampled(inp, acq, ctx=gpu_ctx)
    re, im = out["re"].astype(np.float32), out["im"].astype(np.float32)
    want = np.sqrt(re * re + im * im, dtype=np.float32)
    assert np.array_equal(mag, want)
    wph = np.arctan2(im, re).astype(np.float32)
    ulp = np.abs(ph.view(np.int32).astype(np.int64) - wph.view(np.int32).astype(np.int64))
    assert ulp.max() <= 2, ulp.max()
