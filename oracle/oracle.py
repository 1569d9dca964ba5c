"""TEST INFRASTRUCTURE ONLY — ctypes binding of the FP64 oracle (liboracle, mrsim_oracle.cpp).

The oracle is a CPU restatement of the reference crate's 2D EPI k-space path, pinned bit for bit
to the reference's golden record.  Only the tests, `__graft_entry__.smoke()` and `bench.py`'s
CPU-baseline / reference arm load it, as the checker and the timed CPU baseline; the product
library (mrsim_acq_b200) never imports, links or calls it.
"""
from __future__ import annotations

import ctypes as C
import pathlib
import subprocess
from typing import Optional, Sequence

import numpy as np

from mrsim_acq_b200 import abi
from mrsim_acq_b200.api import Acquisition, PhaseModel, SliceInput, T2, _Keep, slice_input_c

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "libmrsim_oracle.so"
_lib = None


def build() -> pathlib.Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        P = C.POINTER
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_golden_name.restype = C.c_char_p
        L.oracle_golden_output.restype = C.c_int64
        L.oracle_golden_output.argtypes = [C.c_int, P(C.c_uint32), C.c_int64]
        L.oracle_set_kspace_build.argtypes = [C.c_int]
        L.oracle_kspace_build.restype = C.c_int
        L.oracle_build_coil_kspace.argtypes = [P(abi.SliceInput_), P(abi.Acquisition_), C.c_int64, C.c_int64,
                                               abi.c_f64p, abi.c_f64p, abi.c_f64p, P(C.c_int8), abi.c_f64p, abi.c_f64p]
        L.oracle_reference_coil_kspace.argtypes = [P(abi.SliceInput_), P(abi.Acquisition_), C.c_int64, C.c_int64,
                                                   abi.c_f64p]
        L.oracle_simulate_slice.argtypes = [P(abi.SliceInput_), P(abi.Acquisition_), abi.c_f32p]
        L.oracle_simulate_slice_full.argtypes = [P(abi.SliceInput_), P(abi.Acquisition_)] + [abi.c_f64p] * 5
        L.oracle_series_forward.argtypes = [P(abi.AcquisitionInput_), P(abi.Acquisition_), abi.c_f64p, C.c_int64,
                                            P(C.c_int64), C.c_int64, C.c_int, abi.c_f64p]
        L.oracle_series_adjoint.argtypes = [P(abi.AcquisitionInput_), P(abi.Acquisition_), abi.c_f64p, C.c_int64,
                                            P(C.c_int64), C.c_int64, C.c_int, abi.c_f64p, abi.c_f64p, abi.c_f64p,
                                            abi.c_f64p]
        L.oracle_acquire_volumes_complex.argtypes = [P(abi.AcquisitionInput_), P(abi.Acquisition_),
                                                     P(abi.AcquisitionOptions_), C.c_uint64, C.c_uint64, C.c_int,
                                                     P(abi.AcquisitionOutput_)]
        L.oracle_sampling_mask.argtypes = [C.c_int64, C.c_int64, P(abi.Acquisition_), P(C.c_uint8)]
        L.oracle_pf_skipped_lines.restype = C.c_int64
        L.oracle_pf_skipped_lines.argtypes = [C.c_int64, P(abi.Acquisition_)]
        L.oracle_line_timing.argtypes = [P(abi.Acquisition_), C.c_int64, C.c_int64, abi.c_f64p, abi.c_f64p,
                                         abi.c_f64p, P(C.c_int8)]
        L.oracle_epi_order.argtypes = [P(abi.Acquisition_), C.c_int64, C.c_int64, P(C.c_int64)]
        L.oracle_validate_acquisition_timing.argtypes = [P(abi.Acquisition_), C.c_int64, C.c_int64]
        L.oracle_inverse_2d.argtypes = [abi.c_f64p, C.c_int64, C.c_int64, abi.c_f64p]
        L.oracle_rng_next.restype = C.c_uint64
        L.oracle_rng_next.argtypes = [C.c_uint64, C.c_int64, P(C.c_uint64)]
        L.oracle_echo_salt.restype = C.c_uint64
        L.oracle_echo_salt.argtypes = [C.c_uint64]
        L.oracle_coil_sensitivity.restype = C.c_double
        L.oracle_coil_sensitivity.argtypes = [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int64, C.c_int64]
        i64p = P(C.c_int64)
        L.oracle_nufft2.argtypes = [C.c_int32, i64p, i64p, i64p, C.c_double, abi.c_f64p, C.c_int64, abi.c_f64p,
                                    C.c_int32, abi.c_f64p]
        L.oracle_nufft2_direct.argtypes = [C.c_int32, i64p, i64p, i64p, abi.c_f64p, C.c_int64, abi.c_f64p,
                                           C.c_int32, abi.c_f64p]
        L.oracle_spiral_kspace_exact.argtypes = [P(abi.SliceInput_), P(abi.Acquisition_), C.c_int64, C.c_int64,
                                                 abi.c_f64p, abi.c_f64p, C.c_int64, abi.c_f64p, abi.c_f64p]
        L.oracle_spiral_segmented.argtypes = [P(abi.SliceInput_), P(abi.Acquisition_), C.c_int64, C.c_int64,
                                              abi.c_f64p, i64p, C.c_int64, abi.c_f64p, C.c_int64, abi.c_f64p,
                                              abi.c_f64p, C.c_int32, abi.c_f64p]
        L.oracle_spiral_recon.argtypes = [abi.c_f64p, C.c_int64, C.c_int64, C.c_int32, C.c_double, C.c_double,
                                          C.c_int64, C.c_double, C.c_int32, C.c_int32, abi.c_f64p, C.c_int64,
                                          C.c_int64, C.c_int64, abi.c_f64p, abi.c_f64p, abi.c_f64p, i64p,
                                          abi.c_f64p]
        A3 = P(abi.Acquisition3dInput_)
        L.oracle_kz_order.argtypes = [C.c_int64, C.c_int32, i64p]
        L.oracle_epg_cpmg.argtypes = [C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double, abi.c_f64p]
        L.oracle_grase_lines.argtypes = [P(abi.EchoTrain_), P(abi.GraseReadout_), C.c_int64, C.c_int64, i64p, i64p,
                                         abi.c_f64p, abi.c_f64p, P(C.c_int8), i64p, i64p]
        L.oracle_kspace_3d_observed.argtypes = [A3, P(abi.Acquisition_), P(abi.EchoTrain_), P(abi.GraseReadout_),
                                                C.c_int64, abi.c_f64p]
        L.oracle_simulate_acquisition_3d.argtypes = [A3, P(abi.Acquisition_), P(abi.EchoTrain_), P(abi.GraseReadout_),
                                                     C.c_uint64, C.c_int32, abi.c_f64p, abi.c_f32p, abi.c_f32p]
        L.oracle_simulate_acquisition_3d_ge.argtypes = [P(abi.AcquisitionGeInput_), P(abi.Acquisition_),
                                                        P(abi.ExcitationTrain_), P(abi.Ge3dReadout_), C.c_uint64,
                                                        C.c_int32, abi.c_f64p, P(abi.c_f32p), P(abi.c_f32p)]
        L.oracle_reconstruct_coils.argtypes = [abi.c_f64p, C.c_int64, C.c_int64, C.c_int64, P(abi.Acquisition_),
                                               abi.c_f64p]
        KO = P(abi.KzOptions_)
        L.oracle_spiral_lines.argtypes = [P(abi.EchoTrain_), P(abi.SpiralReadout_), C.c_int64, C.c_int64,
                                          P(C.c_uint8), i64p, i64p, i64p, i64p, i64p, abi.c_f64p, abi.c_f64p]
        L.oracle_spiral_samples_3d.argtypes = [A3, P(abi.Acquisition_), P(abi.EchoTrain_), P(abi.SpiralReadout_), KO,
                                               C.c_int64, abi.c_f64p]
        L.oracle_simulate_acquisition_3d_spiral.argtypes = [A3, P(abi.Acquisition_), P(abi.EchoTrain_),
                                                            P(abi.SpiralReadout_), KO, C.c_uint64, C.c_int32,
                                                            abi.c_f64p, abi.c_f32p, abi.c_f32p]
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        raise RuntimeError(lib().oracle_last_error().decode())


# ---- golden record -----------------------------------------------------------------------------
def set_kspace_build(on: bool) -> None:
    """Every later oracle call follows the reference's `kspace` build (NUFFT y-stage, FFT x-stage
    and inverse; on) or its default build (off)."""
    lib().oracle_set_kspace_build(1 if on else 0)


class kspace_build:
    """`with oracle.kspace_build(): ...` runs the block under the reference's `kspace` build."""

    def __enter__(self):
        set_kspace_build(True)

    def __exit__(self, *exc):
        set_kspace_build(False)


def golden_outputs(kspace: bool = False) -> list[tuple[str, np.ndarray]]:
    """The reference's golden record regenerated by the oracle: (name, uint32 bit patterns), of
    the default build or (kspace=True) of the `kspace` build."""
    L = lib()
    out = []
    set_kspace_build(kspace)
    try:
        for i in range(L.oracle_golden_count()):
            name = L.oracle_golden_name(i).decode()
            n = L.oracle_golden_output(i, None, 0)
            buf = np.zeros(n, np.uint32)
            L.oracle_golden_output(i, buf.ctypes.data_as(C.POINTER(C.c_uint32)), n)
            out.append((name, buf))
    finally:
        set_kspace_build(False)
    return out


# ---- tables --------------------------------------------------------------------------------------
def sampling_mask(nx, ny, acq: Acquisition) -> np.ndarray:
    m = np.zeros(nx * ny, np.uint8)
    _check(lib().oracle_sampling_mask(nx, ny, C.byref(acq.to_c()), m.ctypes.data_as(C.POINTER(C.c_uint8))))
    return m.reshape(ny, nx).astype(bool)


def line_timing(acq: Acquisition, nx, ny):
    t, trf, tread = (np.zeros(ny) for _ in range(3))
    pol = np.zeros(ny, np.int8)
    _check(lib().oracle_line_timing(C.byref(acq.to_c()), nx, ny, t.ctypes.data_as(abi.c_f64p),
                                    trf.ctypes.data_as(abi.c_f64p), tread.ctypes.data_as(abi.c_f64p),
                                    pol.ctypes.data_as(C.POINTER(C.c_int8))))
    return t, trf, tread, pol


# ---- per slice ---------------------------------------------------------------------------------
def build_coil_kspace(inp: SliceInput, acq: Acquisition, coil: int, ncoils: int, timing=None,
                      log_amp=None) -> np.ndarray:
    keep = _Keep()
    s = slice_input_c(inp, keep)
    nx, ny = inp.acq_matrix
    out = np.zeros(nx * ny * 2)
    t = [None] * 4
    if timing is not None:
        t = [keep.f64(timing.t_ms), keep.f64(timing.trf_ms), keep.f64(timing.tread_ms)]
        pol = np.ascontiguousarray(timing.polarity, np.int8)
        keep.append(pol)
        t.append(pol.ctypes.data_as(C.POINTER(C.c_int8)))
    la = keep.f64(np.ravel(log_amp)) if log_amp is not None else None
    _check(lib().oracle_build_coil_kspace(C.byref(s), C.byref(acq.to_c()), coil, ncoils, t[0], t[1], t[2], t[3], la,
                                          out.ctypes.data_as(abi.c_f64p)))
    return out.view(np.complex128).reshape(ny, nx)


def reference_coil_kspace(inp: SliceInput, acq: Acquisition, coil: int, ncoils: int) -> np.ndarray:
    keep = _Keep()
    s = slice_input_c(inp, keep)
    nx, ny = inp.acq_matrix
    out = np.zeros(nx * ny * 2)
    _check(lib().oracle_reference_coil_kspace(C.byref(s), C.byref(acq.to_c()), coil, ncoils,
                                              out.ctypes.data_as(abi.c_f64p)))
    return out.view(np.complex128).reshape(ny, nx)


def simulate_slice(inp: SliceInput, acq: Acquisition) -> np.ndarray:
    keep = _Keep()
    s = slice_input_c(inp, keep)
    nx, ny = inp.acq_matrix
    out = np.zeros(nx * ny * 2, np.float32)
    _check(lib().oracle_simulate_slice(C.byref(s), C.byref(acq.to_c()), out.ctypes.data_as(abi.c_f32p)))
    return out.view(np.complex64).reshape(ny, nx)


def simulate_slice_full(inp: SliceInput, acq: Acquisition, capture=True) -> dict:
    keep = _Keep()
    s = slice_input_c(inp, keep)
    nx, ny = inp.acq_matrix
    nc = max(acq.n_coils, 1)
    comb = np.zeros(nx * ny * 2)
    bufs = {k: np.zeros(nc * nx * ny * 2) for k in ("acquired", "reconstructed", "coil_images")} if capture else {}
    sens = np.zeros(nc * nx * ny)

    def p(a):
        return a.ctypes.data_as(abi.c_f64p) if a is not None else None

    _check(lib().oracle_simulate_slice_full(C.byref(s), C.byref(acq.to_c()), p(comb), p(bufs.get("acquired")),
                                            p(bufs.get("reconstructed")), p(bufs.get("coil_images")), p(sens)))
    out = {"combined": comb.view(np.complex128).reshape(ny, nx), "sensitivities": sens.reshape(nc, ny, nx)}
    for k, v in bufs.items():
        out[k] = v.view(np.complex128).reshape(nc, ny, nx)
    return out


# ---- series --------------------------------------------------------------------------------------
def _series_input(keep: _Keep, sim_dims, acq_dims, n_volumes, images, t2, fmap, t_inhom=None, eddy_drive=None,
                  prep_drive=None, phase: Optional[PhaseModel] = None, seed=0, noise_sigma=None):
    inp = abi.AcquisitionInput_()
    for i in range(3):
        inp.sim_dims[i] = sim_dims[i]
        inp.acq_dims[i] = acq_dims[i]
    inp.n_volumes = n_volumes
    inp.ncomp = len(t2)
    inp.images = keep.ptrs([np.ravel(a) for a in images])
    inp.t2 = keep.t2s(t2)
    inp.t_inhom = keep.t2s(t_inhom) if t_inhom is not None else None
    inp.fmap = keep.f32(np.ravel(fmap))
    if eddy_drive is not None:
        flags = np.array([d is not None for d in eddy_drive], np.int32)
        vals = np.array([d if d is not None else (0.0, 0.0, 0.0) for d in eddy_drive], np.float64)
        keep += [flags, vals]
        inp.eddy_drive_set = flags.ctypes.data_as(C.POINTER(C.c_int32))
        inp.eddy_drive = vals.ctypes.data_as(abi.c_f64p)
    if prep_drive is not None:
        flags = np.array([d is not None for d in prep_drive], np.int32)
        vals = np.array([(d[0], *d[1]) if d is not None else (0, 0, 0, 0) for d in prep_drive], np.float64)
        keep += [flags, vals]
        inp.prep_drive_set = flags.ctypes.data_as(C.POINTER(C.c_int32))
        inp.prep_drive = vals.ctypes.data_as(abi.c_f64p)
    ph = (phase or PhaseModel.none()).to_c()
    keep.append(ph)
    inp.phase = C.pointer(ph)
    inp.seed = int(seed)
    if noise_sigma is not None:
        inp.noise_sigma = keep.f32(np.ravel(noise_sigma))
    return inp


def series_forward(sim_dims, acq_dims, n_volumes, images, t2, fmap, acq: Acquisition, echo_times_ms=None,
                   threads=1, slice_z=None, nz_full=0, **kw) -> np.ndarray:
    keep = _Keep()
    inp = _series_input(keep, sim_dims, acq_dims, n_volumes, images, t2, fmap, **kw)
    ne = len(echo_times_ms) if echo_times_ms is not None else 1
    tes = keep.f64(echo_times_ms) if echo_times_ms is not None else None
    nx, ny, nz = acq_dims
    nc = max(acq.n_coils, 1)
    out = np.zeros(n_volumes * nz * nc * ne * ny * nx * 2)
    sz = None
    if slice_z is not None:
        a = np.ascontiguousarray(slice_z, np.int64)
        keep.append(a)
        sz = a.ctypes.data_as(C.POINTER(C.c_int64))
    _check(lib().oracle_series_forward(C.byref(inp), C.byref(acq.to_c()), tes, ne, sz, nz_full, threads,
                                       out.ctypes.data_as(abi.c_f64p)))
    return out.view(np.complex128).reshape(n_volumes, nz, nc, ne, ny, nx)


def series_adjoint(sim_dims, acq_dims, n_volumes, images, t2, fmap, acq: Acquisition, kspace, echo_times_ms=None,
                   threads=1, slice_z=None, nz_full=0, **kw) -> dict:
    keep = _Keep()
    inp = _series_input(keep, sim_dims, acq_dims, n_volumes, images, t2, fmap, **kw)
    ne = len(echo_times_ms) if echo_times_ms is not None else 1
    tes = keep.f64(echo_times_ms) if echo_times_ms is not None else None
    snx, sny, nz = sim_dims
    nc = len(t2)
    k = np.ascontiguousarray(kspace, np.complex128)
    cg = np.zeros(n_volumes * nz * nc * sny * snx * 2)
    fg = np.zeros(n_volumes * nz * sny * snx)
    rg = np.zeros(n_volumes * nz * nc * sny * snx)
    sz = None
    if slice_z is not None:
        a = np.ascontiguousarray(slice_z, np.int64)
        keep.append(a)
        sz = a.ctypes.data_as(C.POINTER(C.c_int64))
    _check(lib().oracle_series_adjoint(C.byref(inp), C.byref(acq.to_c()), tes, ne, sz, nz_full, threads,
                                       k.ctypes.data_as(abi.c_f64p), cg.ctypes.data_as(abi.c_f64p),
                                       fg.ctypes.data_as(abi.c_f64p), rg.ctypes.data_as(abi.c_f64p)))
    return {"comp_grad": cg.view(np.complex128).reshape(n_volumes, nz, nc, sny, snx),
            "fmap_grad": fg.reshape(n_volumes, nz, sny, snx), "r2_grad": rg.reshape(n_volumes, nz, nc, sny, snx)}


def acquire_volumes_complex(sim_dims, acq_dims, n_volumes, images, t2, fmap, acq: Acquisition, excitation_seed,
                            receiver_seed, threads=1, options: Optional[dict] = None, **kw) -> dict:
    keep = _Keep()
    inp = _series_input(keep, sim_dims, acq_dims, n_volumes, images, t2, fmap, seed=receiver_seed, **kw)
    o = abi.AcquisitionOptions_()
    options = options or {}
    nx, ny, nz = acq_dims
    if options.get("t_echo_per_volume") is not None:
        o.t_echo_per_volume = keep.f64(options["t_echo_per_volume"])
    if options.get("slice_z") is not None:
        a = np.ascontiguousarray(options["slice_z"], np.int64)
        keep.append(a)
        o.slice_z = a.ctypes.data_as(C.POINTER(C.c_int64))
    o.nz_full = int(options.get("nz_full", 0))
    caps = options.get("kspace_slices")
    nsl = 0
    if caps is not None:
        a = np.ascontiguousarray(caps, np.int64)
        keep.append(a)
        o.kspace_slices = a.ctypes.data_as(C.POINTER(C.c_int64))
        o.n_kspace_slices = nsl = len(caps)
        o.capture_acquired = int(options.get("acquired", False))
        o.capture_reconstructed = int(options.get("reconstructed", False))
        o.capture_coil_images = int(options.get("coil_images", False))
    if options.get("grappa_calibration") is not None:
        cal_images, cal_seed = options["grappa_calibration"]
        o.has_grappa_calibration = 1
        o.grappa_calibration_images = keep.ptrs([np.ravel(a) for a in cal_images])
        o.grappa_calibration_seed = int(cal_seed)
    nvox = nx * ny * nz
    nc = max(acq.n_coils, 1)
    re = np.zeros(nvox * n_volumes, np.float32)
    im = np.zeros(nvox * n_volumes, np.float32)
    out = abi.AcquisitionOutput_()
    out.re = re.ctypes.data_as(abi.c_f32p)
    out.im = im.ctypes.data_as(abi.c_f32p)
    cap = {}
    if nsl:
        for key in ("acquired", "reconstructed", "coil_images"):
            if options.get(key):
                cap[key] = np.zeros(n_volumes * nsl * nc * nx * ny * 2, np.float32)
                setattr(out, key, cap[key].ctypes.data_as(abi.c_f32p))
        cap["combined"] = np.zeros(n_volumes * nsl * nx * ny * 2, np.float32)
        out.combined = cap["combined"].ctypes.data_as(abi.c_f32p)
        cap["mask"] = np.zeros(nx * ny, np.uint8)
        out.mask = cap["mask"].ctypes.data_as(C.POINTER(C.c_uint8))
        cap["sensitivities"] = np.zeros(nc * nx * ny, np.float32)
        out.sensitivities = cap["sensitivities"].ctypes.data_as(abi.c_f32p)
    _check(lib().oracle_acquire_volumes_complex(C.byref(inp), C.byref(acq.to_c()), C.byref(o), excitation_seed,
                                                receiver_seed, threads, C.byref(out)))
    res = {"re": re, "im": im}
    res.update(cap)
    return res


# ---- stack-of-spirals path -----------------------------------------------------------------------
def _i64(v):
    a = np.ascontiguousarray(v, dtype=np.int64)
    return a, a.ctypes.data_as(C.POINTER(C.c_int64))


def nufft2(type_: int, n, m_lo, m_out, tol: float, u: np.ndarray, data: np.ndarray, sign: int) -> np.ndarray:
    """`Nufft2::type1` / `type2` (nufft.rs:225-292) in FP64 (gridding with a direct fine-grid DFT)."""
    (na, npp), (la, lp), (ma, mp) = _i64(n), _i64(m_lo), _i64(m_out)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 2)
    d = np.ascontiguousarray(np.asarray(data, dtype=np.complex128).ravel())
    out = np.zeros(int(ma[0] * ma[1]) if type_ == 1 else len(u), np.complex128)
    _check(lib().oracle_nufft2(type_, npp, lp, mp, tol, u.ctypes.data_as(abi.c_f64p), len(u),
                               d.view(np.float64).ctypes.data_as(abi.c_f64p), sign,
                               out.view(np.float64).ctypes.data_as(abi.c_f64p)))
    return out


def nufft2_direct(type_: int, n, m_lo, m_out, u: np.ndarray, data: np.ndarray, sign: int) -> np.ndarray:
    """The literal sums of the 2D NUFFT pair (FP64)."""
    (na, npp), (la, lp), (ma, mp) = _i64(n), _i64(m_lo), _i64(m_out)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 2)
    d = np.ascontiguousarray(np.asarray(data, dtype=np.complex128).ravel())
    out = np.zeros(int(ma[0] * ma[1]) if type_ == 1 else len(u), np.complex128)
    _check(lib().oracle_nufft2_direct(type_, npp, lp, mp, u.ctypes.data_as(abi.c_f64p), len(u),
                                      d.view(np.float64).ctypes.data_as(abi.c_f64p), sign,
                                      out.view(np.float64).ctypes.data_as(abi.c_f64p)))
    return out


def spiral_kspace_exact(inp: SliceInput, acq: Acquisition, coil: int, ncoils: int, k, tau, log_amp=None) -> np.ndarray:
    """`spiral_kspace_exact` (spiral.rs:107-137), FP64."""
    keep = _Keep()
    s = slice_input_c(inp, keep)
    k = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 2)
    tau = np.ascontiguousarray(tau, dtype=np.float64)
    la = keep.f64(np.ravel(log_amp)) if log_amp is not None else None
    out = np.zeros(len(k), np.complex128)
    _check(lib().oracle_spiral_kspace_exact(C.byref(s), C.byref(acq.to_c()), coil, ncoils,
                                            k.ctypes.data_as(abi.c_f64p), tau.ctypes.data_as(abi.c_f64p), len(k), la,
                                            out.view(np.float64).ctypes.data_as(abi.c_f64p)))
    return out


def spiral_segmented(inp: SliceInput, acq: Acquisition, coil: int, ncoils: int, k, tau_idx, tau_l, b,
                     log_amp=None, decay_inside=True) -> np.ndarray:
    """`SegmentedForward::apply` (spiral.rs:174-201) for the plan (tau_l, b), type-2 transforms as
    exact sums, FP64."""
    keep = _Keep()
    s = slice_input_c(inp, keep)
    k = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 2)
    ti, tip = _i64(tau_idx)
    tl = np.ascontiguousarray(tau_l, dtype=np.float64)
    bb = np.ascontiguousarray(np.asarray(b, dtype=np.complex128))
    la = keep.f64(np.ravel(log_amp)) if log_amp is not None else None
    out = np.zeros(len(k), np.complex128)
    _check(lib().oracle_spiral_segmented(C.byref(s), C.byref(acq.to_c()), coil, ncoils, k.ctypes.data_as(abi.c_f64p),
                                         tip, len(k), tl.ctypes.data_as(abi.c_f64p), len(tl),
                                         bb.view(np.float64).ctypes.data_as(abi.c_f64p), la, int(bool(decay_inside)),
                                         out.view(np.float64).ctypes.data_as(abi.c_f64p)))
    return out


def spiral_recon(k, n: int, data, mode: str = "image", window=(0, 0.0, 0.0), iterations: int = 80,
                 kappa: float = 100.0, band: bool = True, ring: int = 1, zsens=None):
    """`SpiralRecon` (grid_recon.rs:54-325) in FP64 with the reference's NUFFT-pair normal operator.
    mode "image" / "gridding": data [batch, npts]; "rings": data [partition, coil, npts], zsens
    [partition, coil].  Returns (images [batch, n, n], lambda_hi, power iterations, weights)."""
    k = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 2)
    npts = len(k)
    d = np.ascontiguousarray(np.asarray(data, dtype=np.complex128))
    m = {"rings": 0, "image": 1, "gridding": 2}[mode]
    if m == 0:
        d = d.reshape(-1, d.shape[-2], npts)
        batch, ncoils = d.shape[0], d.shape[1]
        zs = np.ascontiguousarray(np.asarray(zsens, dtype=np.float64).reshape(batch, ncoils))
        zp = zs.ctypes.data_as(abi.c_f64p)
    else:
        d = d.reshape(-1, npts)
        batch, ncoils, zp = d.shape[0], 1, None
    out = np.zeros(batch * n * n, np.complex128)
    lam = C.c_double()
    its = C.c_int64()
    w = np.zeros(npts)
    _check(lib().oracle_spiral_recon(k.ctypes.data_as(abi.c_f64p), npts, n, int(window[0]), float(window[1]),
                                     float(window[2]), iterations, kappa, int(band), m,
                                     d.view(np.float64).ctypes.data_as(abi.c_f64p), batch, ncoils, ring, zp,
                                     out.view(np.float64).ctypes.data_as(abi.c_f64p), C.byref(lam), C.byref(its),
                                     w.ctypes.data_as(abi.c_f64p)))
    return out.reshape(batch, n, n), lam.value, its.value, w


# ---- the 3D GRASE echo train -------------------------------------------------------------------------
def kz_order(nz: int, order: int) -> np.ndarray:
    out = np.zeros(nz, np.int64)
    _check(lib().oracle_kz_order(nz, int(order), out.ctypes.data_as(C.POINTER(C.c_int64))))
    return out


def epg_cpmg(n: int, esp: float, b: float, t1: float, t2: float) -> np.ndarray:
    out = np.zeros(n)
    _check(lib().oracle_epg_cpmg(n, esp, b, t1, t2, out.ctypes.data_as(abi.c_f64p)))
    return out


def grase_lines(train, ro, ny: int, nz: int) -> dict:
    n = ny * nz
    shot, echo = np.zeros(n, np.int64), np.zeros(n, np.int64)
    t, trf, pol = np.zeros(n), np.zeros(n), np.zeros(n, np.int8)
    e_c, n_shots = C.c_int64(), C.c_int64()
    P = C.POINTER(C.c_int64)
    _check(lib().oracle_grase_lines(C.byref(train.to_c()), C.byref(ro.to_c()), ny, nz, shot.ctypes.data_as(P),
                                    echo.ctypes.data_as(P), t.ctypes.data_as(abi.c_f64p), trf.ctypes.data_as(abi.c_f64p),
                                    pol.ctypes.data_as(C.POINTER(C.c_int8)), C.byref(e_c), C.byref(n_shots)))
    return {"shot": shot, "echo": echo, "t_ms": t, "trf_ms": trf, "polarity": pol, "e_c": e_c.value,
            "n_shots": n_shots.value}


def kspace_3d_observed(sim_dims, acq_dims, n_volumes, images, t2, t1, fmap, t_inhom, acq: Acquisition, train, ro,
                       line_weights=None, phase=None, g: int = 0, shot_images=None) -> np.ndarray:
    """`kspace_3d_observed` (kspace3d.rs:439-456), FP64: complex128 [coil, p, ky, kx]."""
    from mrsim_acq_b200.kspace3d import acquisition_3d_input_c
    keep = _Keep()
    s = acquisition_3d_input_c(sim_dims, acq_dims, n_volumes, images, t2, t1, fmap, t_inhom, phase, line_weights,
                               None, keep, shot_images)
    nx, ny, nz = acq_dims
    nc = max(acq.n_coils, 1)
    out = np.zeros(nc * nz * ny * nx, np.complex128)
    _check(lib().oracle_kspace_3d_observed(C.byref(s), C.byref(acq.to_c()), C.byref(train.to_c()), C.byref(ro.to_c()),
                                           g, out.view(np.float64).ctypes.data_as(abi.c_f64p)))
    return out.reshape(nc, nz, ny, nx)


def simulate_acquisition_3d(sim_dims, acq_dims, n_volumes, images, t2, t1, fmap, t_inhom, acq: Acquisition, train, ro,
                            line_weights=None, phase=None, seed: int = 0, grappa_calibration=None, threads: int = 0,
                            shot_images=None):
    """`simulate_acquisition_3d` (kspace3d.rs:549-589), FP64: (complex volumes [g, vox], mag, phase)."""
    import os
    from mrsim_acq_b200.kspace3d import acquisition_3d_input_c
    keep = _Keep()
    s = acquisition_3d_input_c(sim_dims, acq_dims, n_volumes, images, t2, t1, fmap, t_inhom, phase, line_weights,
                               grappa_calibration, keep, shot_images)
    nvox = int(np.prod(acq_dims))
    vols = np.zeros(n_volumes * nvox, np.complex128)
    mag, ph = np.zeros(nvox * n_volumes, np.float32), np.zeros(nvox * n_volumes, np.float32)
    _check(lib().oracle_simulate_acquisition_3d(C.byref(s), C.byref(acq.to_c()), C.byref(train.to_c()),
                                                C.byref(ro.to_c()), int(seed) & 0xFFFFFFFFFFFFFFFF,
                                                threads or (os.cpu_count() or 1),
                                                vols.view(np.float64).ctypes.data_as(abi.c_f64p),
                                                mag.ctypes.data_as(abi.c_f32p), ph.ctypes.data_as(abi.c_f32p)))
    return vols.reshape(n_volumes, nvox), mag, ph


# ---- the stack of spirals ------------------------------------------------------------------------------
def spiral_lines(train, ro, n: int, nz: int) -> dict:
    acq = np.zeros(nz, np.uint8)
    echo, seg = np.zeros(nz, np.int64), np.zeros(nz, np.int64)
    vals = [C.c_int64() for _ in range(3)]
    from mrsim_acq_b200.spiral import spiral_trajectory
    tr = spiral_trajectory(n, n, ro.interleaves, ro.readout_ms, ro.dwell_ms, ro.radial_oversampling)
    k = np.zeros(tr.k.size)
    tau = np.zeros(len(tr.tau_ms))
    P = C.POINTER(C.c_int64)
    _check(lib().oracle_spiral_lines(C.byref(train.to_c()), C.byref(ro.to_c()), n, nz,
                                     acq.ctypes.data_as(C.POINTER(C.c_uint8)), echo.ctypes.data_as(P),
                                     seg.ctypes.data_as(P), *[C.byref(v) for v in vals], k.ctypes.data_as(abi.c_f64p),
                                     tau.ctypes.data_as(abi.c_f64p)))
    return {"acquired": acq.astype(bool), "echo": echo, "kz_segment": seg, "band_start": vals[0].value,
            "e_c": vals[1].value, "n_shots": vals[2].value, "k": k.reshape(-1, 2), "tau_ms": tau}


def _kz_c(kz_opts, keep):
    return C.byref(kz_opts.to_c(keep)) if kz_opts is not None else None


def spiral_samples_3d(sim_dims, acq_dims, n_volumes, images, t2, t1, fmap, t_inhom, acq: Acquisition, train, ro,
                      line_weights=None, phase=None, g: int = 0, kz_opts=None, shot_images=None) -> np.ndarray:
    """`SpiralPlan::samples_all` with the exact in-plane sum, FP64: complex128 [coil, partition, sample]."""
    from mrsim_acq_b200.kspace3d import acquisition_3d_input_c
    keep = _Keep()
    s = acquisition_3d_input_c(sim_dims, acq_dims, n_volumes, images, t2, t1, fmap, t_inhom, phase, line_weights,
                               None, keep, shot_images)
    nz = acq_dims[2]
    tab = spiral_lines(train, ro, acq_dims[0], nz)
    nsamp = len(tab["k"])
    nc = max(acq.n_coils, 1)
    out = np.zeros(nc * nz * nsamp, np.complex128)
    _check(lib().oracle_spiral_samples_3d(C.byref(s), C.byref(acq.to_c()), C.byref(train.to_c()), C.byref(ro.to_c()),
                                          _kz_c(kz_opts, keep), g, out.view(np.float64).ctypes.data_as(abi.c_f64p)))
    return out.reshape(nc, nz, nsamp)


def simulate_acquisition_3d_spiral(sim_dims, acq_dims, n_volumes, images, t2, t1, fmap, t_inhom, acq: Acquisition,
                                   train, ro, line_weights=None, phase=None, seed: int = 0, kz_opts=None,
                                   threads: int = 0, shot_images=None):
    """`spiral_volumes` (kspace3d.rs:1472-1569), FP64: (complex volumes [g, vox], mag, phase)."""
    import os
    from mrsim_acq_b200.kspace3d import acquisition_3d_input_c
    keep = _Keep()
    s = acquisition_3d_input_c(sim_dims, acq_dims, n_volumes, images, t2, t1, fmap, t_inhom, phase, line_weights,
                               None, keep, shot_images)
    nvox = int(np.prod(acq_dims))
    vols = np.zeros(n_volumes * nvox, np.complex128)
    mag, ph = np.zeros(nvox * n_volumes, np.float32), np.zeros(nvox * n_volumes, np.float32)
    _check(lib().oracle_simulate_acquisition_3d_spiral(C.byref(s), C.byref(acq.to_c()), C.byref(train.to_c()),
                                                       C.byref(ro.to_c()), _kz_c(kz_opts, keep),
                                                       int(seed) & 0xFFFFFFFFFFFFFFFF, threads or (os.cpu_count() or 1),
                                                       vols.view(np.float64).ctypes.data_as(abi.c_f64p),
                                                       mag.ctypes.data_as(abi.c_f32p), ph.ctypes.data_as(abi.c_f32p)))
    return vols.reshape(n_volumes, nvox), mag, ph


# ---- the 3D gradient-echo train ----------------------------------------------------------------------
def simulate_acquisition_3d_ge(sim_dims, acq_dims, n_volumes, t2, fmap, t_inhom, acq: Acquisition, train, ro, volume,
                               phase=None, seed: int = 0, reference=None, threads: int = 0):
    """`simulate_acquisition_3d_ge` (kspace3d.rs:732-856), FP64: complex volumes [e, g, vox] and per
    echo (mag, phase) f32."""
    import os
    from mrsim_acq_b200.kspace3d import _GeVolumes, ge_input_c
    keep = _Keep()
    vols = _GeVolumes(volume, len(t2))
    s = ge_input_c(sim_dims, acq_dims, n_volumes, t2, fmap, t_inhom, phase, vols, reference, keep)
    nvox = int(np.prod(acq_dims))
    ne = len(train.echo_times_ms)
    out = np.zeros(ne * n_volumes * nvox, np.complex128)
    mags = [np.zeros(nvox * n_volumes, np.float32) for _ in range(ne)]
    phs = [np.zeros(nvox * n_volumes, np.float32) for _ in range(ne)]
    mp = (abi.c_f32p * ne)(*[m.ctypes.data_as(abi.c_f32p) for m in mags])
    pp = (abi.c_f32p * ne)(*[p.ctypes.data_as(abi.c_f32p) for p in phs])
    _check(lib().oracle_simulate_acquisition_3d_ge(C.byref(s), C.byref(acq.to_c()), C.byref(train.to_c(keep)),
                                                   C.byref(ro.to_c()), int(seed) & 0xFFFFFFFFFFFFFFFF,
                                                   threads or (os.cpu_count() or 1),
                                                   out.view(np.float64).ctypes.data_as(abi.c_f64p), mp, pp))
    return out.reshape(ne, n_volumes, nvox), list(zip(mags, phs))


def reconstruct_coils(coils: np.ndarray, acq: Acquisition) -> np.ndarray:
    """`reconstruct_coils` (kspace.rs:1291-1298) without GRAPPA, FP64: coils [nc, ny, nx] -> [ny, nx]."""
    k = np.ascontiguousarray(coils, dtype=np.complex128)
    nc, ny, nx = k.shape
    out = np.zeros(ny * nx, np.complex128)
    _check(lib().oracle_reconstruct_coils(k.view(np.float64).ctypes.data_as(abi.c_f64p), nc, nx, ny,
                                          C.byref(acq.to_c()), out.view(np.float64).ctypes.data_as(abi.c_f64p)))
    return out.reshape(ny, nx)


# ---- image motion (motion.rs) -----------------------------------------------------------------------
def _motion_lib():
    L = lib()
    if not getattr(L, "_motion_typed", False):
        P = C.POINTER
        i64p = P(C.c_int64)
        L.oracle_motion_trilinear.argtypes = [abi.c_f32p, i64p, abi.c_f64p, abi.c_f32p]
        L.oracle_resample_by_pose.argtypes = [abi.c_f32p, i64p, abi.c_f64p, abi.c_f64p, abi.c_f32p]
        L.oracle_apply_motion.argtypes = [P(abi.c_f32p), C.c_int64, i64p, C.c_int64, abi.c_f64p, abi.c_f64p]
        L.oracle_apply_multiband_motion.argtypes = [P(abi.c_f32p), C.c_int64, i64p, C.c_int64, abi.c_f64p, C.c_int64,
                                                    C.c_int32, C.c_int32, abi.c_f64p, C.c_int64, C.c_double, C.c_double,
                                                    i64p, i64p, abi.c_f32p, abi.c_f64p, abi.c_f64p, C.c_int64, i64p,
                                                    C.c_int64, i64p, i64p, abi.c_f32p, i64p]
        L._motion_typed = True
    return L


def _i64(a):
    a = np.ascontiguousarray(a, np.int64)
    return a, a.ctypes.data_as(C.POINTER(C.c_int64))


def motion_trilinear(vol, dims, p) -> float:
    v = np.ascontiguousarray(vol, np.float32)
    d, dp = _i64(dims)
    pp = np.ascontiguousarray(p, np.float64)
    out = np.zeros(1, np.float32)
    _motion_lib().oracle_motion_trilinear(v.ctypes.data_as(abi.c_f32p), dp, pp.ctypes.data_as(abi.c_f64p),
                                          out.ctypes.data_as(abi.c_f32p))
    return float(out[0])


def resample_by_pose(src, dims, v2w, pose) -> np.ndarray:
    s = np.ascontiguousarray(src, np.float32).ravel()
    out = np.zeros_like(s)
    d, dp = _i64(dims)
    m = np.ascontiguousarray(v2w, np.float64).reshape(16)
    p = np.ascontiguousarray(pose, np.float64).reshape(6)
    _motion_lib().oracle_resample_by_pose(s.ctypes.data_as(abi.c_f32p), dp, m.ctypes.data_as(abi.c_f64p),
                                          p.ctypes.data_as(abi.c_f64p), out.ctypes.data_as(abi.c_f32p))
    return out


def apply_motion(images, dims, n_volumes, v2w, poses) -> None:
    """In place; poses is n_volumes x 6 (rot_deg, trans_mm)."""
    ptrs = (abi.c_f32p * len(images))(*[a.ctypes.data_as(abi.c_f32p) for a in images])
    d, dp = _i64(dims)
    m = np.ascontiguousarray(v2w, np.float64).reshape(16)
    p = np.ascontiguousarray(poses, np.float64).reshape(-1)
    _motion_lib().oracle_apply_motion(ptrs, len(images), dp, n_volumes, m.ctypes.data_as(abi.c_f64p),
                                      p.ctypes.data_as(abi.c_f64p))


def apply_multiband_motion(images, dims, n_volumes, v2w, mb, interleaved, law_kind, drive, floor, max_, events,
                           slice_z=None, nz_full=0):
    """In place; events are (volume, shot, severity, jump_mm[3], jump_deg[3]); returns the dropped
    shots as (volume, shot, attenuation)."""
    ptrs = (abi.c_f32p * len(images))(*[a.ctypes.data_as(abi.c_f32p) for a in images])
    d, dp = _i64(dims)
    m = np.ascontiguousarray(v2w, np.float64).reshape(16)
    dr = np.ascontiguousarray(drive, np.float64)
    n = len(events)
    vol, vp = _i64([e[0] for e in events] or [0])
    shot, sp = _i64([e[1] for e in events] or [0])
    sev = np.ascontiguousarray([e[2] for e in events] or [0], np.float32)
    jm = np.ascontiguousarray([e[3] for e in events] or [(0, 0, 0)], np.float64)
    jd = np.ascontiguousarray([e[4] for e in events] or [(0, 0, 0)], np.float64)
    sz, szp = _i64(slice_z) if slice_z is not None else (None, None)
    ov, ovp = _i64(np.zeros(max(n, 1)))
    osh, oshp = _i64(np.zeros(max(n, 1)))
    oa = np.zeros(max(n, 1), np.float32)
    nd, ndp = _i64([0])
    _motion_lib().oracle_apply_multiband_motion(ptrs, len(images), dp, n_volumes, m.ctypes.data_as(abi.c_f64p), mb,
                                                int(interleaved), law_kind, dr.ctypes.data_as(abi.c_f64p), dr.size,
                                                floor, max_, vp, sp, sev.ctypes.data_as(abi.c_f32p),
                                                jm.ctypes.data_as(abi.c_f64p), jd.ctypes.data_as(abi.c_f64p), n, szp,
                                                nz_full, ovp, oshp, oa.ctypes.data_as(abi.c_f32p), ndp)
    return [(int(ov[i]), int(osh[i]), float(oa[i])) for i in range(int(nd[0]))]


# ---- spin history (spin_history.rs) -----------------------------------------------------------
class OraclePieces(C.Structure):
    """One voxel's pieces (`Pieces`, spin_history.rs:87-92), for the reference's piece tests."""
    _fields_ = [("n", C.c_int32), ("pad", C.c_int32), ("start", C.c_float * 8), ("mz", C.c_float * 8),
                ("t", C.c_double * 8)]


def _spin_lib():
    L = lib()
    if not getattr(L, "_spin_typed", False):
        P = C.POINTER
        pp = P(OraclePieces)
        pul = P(abi.Pulse_)
        L.oracle_pieces_relaxed.argtypes = [pp]
        L.oracle_pieces_split.argtypes = [pp, C.c_float]
        L.oracle_pieces_has_edge.argtypes = [pp, C.c_float]
        L.oracle_pieces_coalesce.argtypes = [pp]
        L.oracle_pieces_cut.restype = C.c_uint64
        L.oracle_pieces_cut.argtypes = [pp, C.c_float, C.c_float, C.c_double, pul, C.c_int64]
        L.oracle_pieces_merge_closest.argtypes = [pp, C.c_double, pul, C.c_int64, abi.c_f32p, C.c_int32]
        L.oracle_spin_replay.restype = C.c_double
        L.oracle_spin_replay.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, pul, C.c_int64]
        L.oracle_spin_new.restype = C.c_void_p
        L.oracle_spin_new.argtypes = [P(C.c_int64), abi.c_f64p, abi.c_f32p, abi.c_f32p, P(C.c_uint8), C.c_int64,
                                      P(C.c_int64), abi.c_f64p, pul, C.c_int64, C.c_char_p, C.c_int64]
        L.oracle_spin_step.argtypes = [C.c_void_p, P(abi.SpinShot_), abi.c_f32p, C.c_char_p, C.c_int64]
        L.oracle_spin_merges.restype = C.c_uint64
        L.oracle_spin_merges.argtypes = [C.c_void_p]
        L.oracle_spin_n_tracked.restype = C.c_int64
        L.oracle_spin_n_tracked.argtypes = [C.c_void_p]
        L.oracle_spin_free.argtypes = [C.c_void_p]
        L._spin_typed = True
    return L


class Pieces:
    """The reference's `Pieces` operations on one voxel (f32 edges and Mz, f64 times)."""

    def __init__(self):
        self.c = OraclePieces()
        _spin_lib().oracle_pieces_relaxed(C.byref(self.c))

    n = property(lambda self: self.c.n)

    def split(self, u: float) -> bool:
        return bool(_spin_lib().oracle_pieces_split(C.byref(self.c), u))

    def has_edge(self, u: float) -> bool:
        return bool(_spin_lib().oracle_pieces_has_edge(C.byref(self.c), u))

    def coalesce(self) -> None:
        _spin_lib().oracle_pieces_coalesce(C.byref(self.c))

    def cut(self, u0: float, u1: float, t1: float, pulses=()) -> int:
        from mrsim_acq_b200.spin_history import pulses_c
        arr, n = pulses_c(list(pulses))
        return int(_spin_lib().oracle_pieces_cut(C.byref(self.c), u0, u1, t1, arr, n))

    def merge_closest(self, t1: float, pulses=(), protect=()) -> None:
        from mrsim_acq_b200.spin_history import pulses_c
        arr, n = pulses_c(list(pulses))
        pr = np.ascontiguousarray(list(protect) or [0.0], np.float32)
        _spin_lib().oracle_pieces_merge_closest(C.byref(self.c), t1, arr, n, pr.ctypes.data_as(abi.c_f32p),
                                                len(protect))


def spin_replay(mz: float, t_from: float, t_to: float, t1: float, pulses=()) -> float:
    from mrsim_acq_b200.spin_history import pulses_c
    arr, n = pulses_c(list(pulses))
    return float(_spin_lib().oracle_spin_replay(mz, t_from, t_to, t1, arr, n))


class SpinHistory:
    """The FP64 restatement of `SpinHistory` with the library's Python interface (`prime`,
    `excite`, `excite_many`, `merges`, `n_tracked`)."""

    def __init__(self, source, slabs, pulses=()):
        from mrsim_acq_b200.spin_history import NO_CLASS, _RefValues, pulses_c
        L = _spin_lib()
        dims = np.ascontiguousarray(source.dims, np.int64)
        t1 = np.ascontiguousarray(source.t1, np.float32).ravel()
        w = np.ascontiguousarray(source.weight, np.float32).ravel()
        cls = np.ascontiguousarray(source.cls, np.uint8).ravel()
        sdims = np.ascontiguousarray(slabs.dims, np.int64)
        v2w = np.ascontiguousarray(source.v2w, np.float64).reshape(16)
        sv2w = np.ascontiguousarray(slabs.v2w, np.float64).reshape(16)
        parr, npul = pulses_c(list(pulses))
        err = C.create_string_buffer(512)
        P = C.POINTER(C.c_int64)
        self._h = None
        h = L.oracle_spin_new(dims.ctypes.data_as(P), v2w.ctypes.data_as(abi.c_f64p), t1.ctypes.data_as(abi.c_f32p),
                              w.ctypes.data_as(abi.c_f32p), cls.ctypes.data_as(C.POINTER(C.c_uint8)),
                              int(source.n_classes), sdims.ctypes.data_as(P), sv2w.ctypes.data_as(abi.c_f64p), parr,
                              npul, err, 512)
        if not h:
            raise RuntimeError(err.value.decode())
        self._h = h
        self.n_classes = int(source.n_classes)
        self.cells = int(sdims[0] * sdims[1])
        self._ref_values = _RefValues(t1[cls != NO_CLASS].astype(np.float64))

    @property
    def n_tracked(self) -> int:
        return int(_spin_lib().oracle_spin_n_tracked(self._h))

    def excite_many(self, shots) -> list:
        from mrsim_acq_b200.spin_history import shots_c, unpack_terms
        L = _spin_lib()
        keep: list = []
        arr = shots_c(shots, self._ref_values, keep)
        outs = []
        err = C.create_string_buffer(512)
        for i, s in enumerate(shots):
            n = 0 if s.mz_ref is None else len(s.slices) * 2 * self.n_classes * self.cells
            buf = np.zeros(max(n, 1), np.float32)
            if L.oracle_spin_step(self._h, C.byref(arr[i]), buf.ctypes.data_as(abi.c_f32p), err, 512) != 0:
                raise RuntimeError(err.value.decode())
            outs.append(buf[:n])
        flat = np.concatenate(outs) if outs else np.zeros(0, np.float32)
        return unpack_terms(shots, flat, self.n_classes, self.cells)

    def excite(self, t, transform, slices, mz_ref, weight=None) -> list:
        from mrsim_acq_b200.spin_history import Shot
        return self.excite_many([Shot(t, transform, slices, mz_ref, weight)])[0]

    def prime(self, shots, transform) -> None:
        from mrsim_acq_b200.spin_history import Shot
        self.excite_many([Shot(t, transform, sl, None) for t, sl in shots])

    def merges(self) -> int:
        return int(_spin_lib().oracle_spin_merges(self._h))

    def __del__(self):
        try:
            if self._h:
                _spin_lib().oracle_spin_free(self._h)
                self._h = None
        except Exception:
            pass
