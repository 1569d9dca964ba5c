"""Python mirror of the reference's k-space API (Rust `mrsim_acq::kspace`), over the C ABI.

Names, fields, defaults and error behaviour follow the reference crate: `Acquisition` and its
`Default` (kspace.rs:166-267), `T2Slice`/`T2Volume` (kspace.rs:380-393), `SliceInput`
(kspace.rs:458-496), `PhaseModel` (phase.rs:130-205), `sampling_mask` (kspace.rs:546),
`LineTiming::for_acquisition` (kspace.rs:310), `validate_acquisition_timing` (kspace.rs:411).
Failures raise `MrsimError` carrying the reference's panic message.  Every compute call runs the
CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import enum
import threading
from typing import Optional, Sequence

import numpy as np

from . import abi
from .abi import check, lib


class PartialFourierMode(enum.IntEnum):  # kspace.rs:85-106
    FiberfoxCompatible = 0
    Contiguous = 1
    Scanner = 2


class EchoFormation(enum.IntEnum):  # kspace.rs:207-212
    Spin = 0
    Gradient = 1


@dataclasses.dataclass(frozen=True)
class KspaceWindow:  # kspace.rs:126-161
    kind: int = 0
    a: float = 0.0
    b: float = 0.0

    @staticmethod
    def none():
        return KspaceWindow(0)

    @staticmethod
    def tukey(alpha: float):
        return KspaceWindow(1, alpha)

    @staticmethod
    def hann():
        return KspaceWindow(2)

    @staticmethod
    def fermi(radius: float, width: float):
        return KspaceWindow(3, radius, width)


@dataclasses.dataclass
class Acquisition:
    """`Acquisition` with the reference's `Default` (kspace.rs:239-267)."""

    t_line: float = 1.0
    t_echo: float = 90.0
    t_inhom: float = 50.0
    signal_scale: float = 100.0
    reverse_phase: bool = False
    do_distortions: bool = True
    do_relaxation: bool = True
    noise_variance: float = 0.0
    partial_fourier: float = 1.0
    pf_mode: PartialFourierMode = PartialFourierMode.FiberfoxCompatible
    ghost_offset: float = 0.0
    eddy_strength: float = 0.0
    eddy_quad: float = 0.0
    eddy_phase: float = 0.0
    eddy_tau: float = 70.0
    n_spikes: int = 0
    spike_amplitude: float = 1.0
    window: KspaceWindow = KspaceWindow()
    n_coils: int = 1
    accel: int = 1
    acs_lines: int = 24
    seed: int = 0
    echo: EchoFormation = EchoFormation.Spin

    def replace(self, **kw) -> "Acquisition":
        return dataclasses.replace(self, **kw)

    def to_c(self) -> abi.Acquisition_:
        a = abi.Acquisition_()
        a.t_line, a.t_echo, a.t_inhom, a.signal_scale = self.t_line, self.t_echo, self.t_inhom, self.signal_scale
        a.reverse_phase, a.do_distortions, a.do_relaxation = (int(self.reverse_phase), int(self.do_distortions),
                                                              int(self.do_relaxation))
        a.pf_mode = int(self.pf_mode)
        a.noise_variance, a.partial_fourier, a.ghost_offset = self.noise_variance, self.partial_fourier, self.ghost_offset
        a.eddy_strength, a.eddy_quad, a.eddy_phase, a.eddy_tau = (self.eddy_strength, self.eddy_quad,
                                                                  self.eddy_phase, self.eddy_tau)
        a.n_spikes, a.spike_amplitude = int(self.n_spikes), self.spike_amplitude
        a.window_kind, a.window_a, a.window_b = self.window.kind, self.window.a, self.window.b
        a.echo = int(self.echo)
        a.n_coils, a.accel, a.acs_lines, a.seed = int(self.n_coils), int(self.accel), int(self.acs_lines), int(self.seed)
        return a


@dataclasses.dataclass(frozen=True)
class T2:
    """`T2Slice` / `T2Volume`: a uniform value (ms) or a map."""

    value: float = 0.0
    map: Optional[np.ndarray] = None

    @staticmethod
    def uniform(v: float) -> "T2":
        return T2(float(v), None)

    @staticmethod
    def of_map(m) -> "T2":
        return T2(0.0, np.ascontiguousarray(m, dtype=np.float32))


@dataclasses.dataclass
class PhaseModel:
    """`PhaseModel` (phase.rs:130): global + background polynomial + optional prep phase."""

    global_: float = 0.0
    background: Sequence[float] = (0.0,) * 10
    prep: Optional[tuple] = None  # (c_q, sigma_dx, sigma_rot)

    @staticmethod
    def hbcd_like() -> "PhaseModel":  # phase.rs:187
        return PhaseModel(0.0, (0.0, 0.13, 0.10, 0.02, 0, 0, 0, 0, 0, 0), (0.0425, 1.0, 2.0e-3))

    @staticmethod
    def none() -> "PhaseModel":  # phase.rs:197
        return PhaseModel(0.0, (0.0,) * 10, (0.0, 0.0, 0.0))

    def to_c(self) -> abi.PhaseModel_:
        p = abi.PhaseModel_()
        p.global_ = self.global_
        for i, v in enumerate(self.background):
            p.background[i] = float(v)
        if self.prep is not None:
            p.has_prep = 1
            p.c_q, p.sigma_dx, p.sigma_rot = self.prep
        return p


@dataclasses.dataclass
class SliceInput:
    """`SliceInput` (kspace.rs:458-496).  Planes are on the sim grid, layout x + snx*y."""

    compartments: Sequence[np.ndarray]
    t2: Sequence[T2]
    fmap: np.ndarray
    sim: tuple
    acq_matrix: tuple
    t_inhom: Optional[Sequence[T2]] = None
    phase0: Optional[np.ndarray] = None
    z: int = 0
    nz: int = 1
    eddy_drive: Optional[Sequence[float]] = None
    prep_drive: Optional[tuple] = None
    slice_seed: int = 0


class _Keep(list):
    """Holds numpy buffers alive while a C structure points at them."""

    def f32(self, a) -> C.POINTER(C.c_float):
        a = np.ascontiguousarray(a, dtype=np.float32)
        self.append(a)
        return a.ctypes.data_as(abi.c_f32p)

    def f64(self, a) -> C.POINTER(C.c_double):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.append(a)
        return a.ctypes.data_as(abi.c_f64p)

    def t2s(self, vals: Sequence[T2]):
        arr = (abi.T2_ * max(1, len(vals)))()
        for i, t in enumerate(vals):
            if t.map is not None:
                arr[i].map = self.f32(t.map)
                arr[i].is_map = 1
            else:
                arr[i].value = float(t.value)
        self.append(arr)
        return arr

    def ptrs(self, arrays):
        ps = (abi.c_f32p * max(1, len(arrays)))()
        for i, a in enumerate(arrays):
            ps[i] = self.f32(a)
        self.append(ps)
        return ps


def slice_input_c(inp: SliceInput, keep: _Keep) -> abi.SliceInput_:
    s = abi.SliceInput_()
    s.compartments = keep.ptrs([np.ravel(c) for c in inp.compartments])
    s.ncomp = len(inp.compartments)
    s.t2 = keep.t2s(inp.t2)
    s.t_inhom = keep.t2s(inp.t_inhom) if inp.t_inhom is not None else None
    s.fmap = keep.f32(np.ravel(inp.fmap))
    s.phase0 = keep.f64(np.ravel(inp.phase0)) if inp.phase0 is not None else None
    s.sim[0], s.sim[1] = inp.sim
    s.acq_matrix[0], s.acq_matrix[1] = inp.acq_matrix
    s.z, s.nz = inp.z, inp.nz
    if inp.eddy_drive is not None:
        s.has_eddy_drive = 1
        for i in range(3):
            s.eddy_drive[i] = float(inp.eddy_drive[i])
    if inp.prep_drive is not None:
        s.has_prep_drive = 1
        s.prep_magnitude = float(inp.prep_drive[0])
        for i in range(3):
            s.prep_direction[i] = float(inp.prep_drive[1][i])
    s.slice_seed = int(inp.slice_seed) & 0xFFFFFFFFFFFFFFFF
    return s


@dataclasses.dataclass
class AcquisitionInput:
    """`AcquisitionInput` (kspace.rs:1720-1740).  Images: one array per compartment on the sim grid,
    layout (x + snx*(y + sny*z))*n_volumes + g."""

    sim_dims: tuple
    acq_dims: tuple
    n_volumes: int
    images: Sequence[np.ndarray]
    t2: Sequence[T2]
    fmap: np.ndarray
    t_inhom: Optional[Sequence[T2]] = None
    eddy_drive: Optional[Sequence] = None
    prep_drive: Optional[Sequence] = None
    phase: PhaseModel = dataclasses.field(default_factory=PhaseModel.none)
    seed: int = 0
    noise_sigma: Optional[np.ndarray] = None


@dataclasses.dataclass
class AcquisitionOptions:
    """`AcquisitionOptions` (kspace.rs:1744-1762) with `SliceCapture` flags (kspace.rs:1184)."""

    slice_z: Optional[Sequence[int]] = None
    nz_full: int = 0
    kspace_slices: Optional[Sequence[int]] = None
    acquired: bool = False
    reconstructed: bool = False
    coil_images: bool = False
    t_echo_per_volume: Optional[Sequence[float]] = None
    progress: Optional[object] = None
    grappa_calibration: Optional[tuple] = None  # (images per compartment, seed)


def acquisition_input_c(inp: AcquisitionInput, keep: _Keep, with_images: bool = True) -> abi.AcquisitionInput_:
    c = abi.AcquisitionInput_()
    for i in range(3):
        c.sim_dims[i] = inp.sim_dims[i]
        c.acq_dims[i] = inp.acq_dims[i]
    c.n_volumes = inp.n_volumes
    c.ncomp = len(inp.t2)
    if with_images and inp.images is not None:
        c.images = keep.ptrs([np.ravel(a) for a in inp.images])
    c.t2 = keep.t2s(inp.t2)
    c.t_inhom = keep.t2s(inp.t_inhom) if inp.t_inhom is not None else None
    c.fmap = keep.f32(np.ravel(inp.fmap))
    if inp.eddy_drive is not None:
        flags = np.array([d is not None for d in inp.eddy_drive], np.int32)
        vals = np.array([d if d is not None else (0.0, 0.0, 0.0) for d in inp.eddy_drive], np.float64)
        keep += [flags, vals]
        c.eddy_drive_set = flags.ctypes.data_as(C.POINTER(C.c_int32))
        c.eddy_drive = vals.ctypes.data_as(abi.c_f64p)
    if inp.prep_drive is not None:
        flags = np.array([d is not None for d in inp.prep_drive], np.int32)
        vals = np.array([(d[0], *d[1]) if d is not None else (0, 0, 0, 0) for d in inp.prep_drive], np.float64)
        keep += [flags, vals]
        c.prep_drive_set = flags.ctypes.data_as(C.POINTER(C.c_int32))
        c.prep_drive = vals.ctypes.data_as(abi.c_f64p)
    ph = (inp.phase or PhaseModel.none()).to_c()
    keep.append(ph)
    c.phase = C.pointer(ph)
    c.seed = int(inp.seed) & 0xFFFFFFFFFFFFFFFF
    if inp.noise_sigma is not None:
        c.noise_sigma = keep.f32(np.ravel(inp.noise_sigma))
    return c


def acquisition_options_c(o: Optional[AcquisitionOptions], keep: _Keep) -> abi.AcquisitionOptions_:
    c = abi.AcquisitionOptions_()
    if o is None:
        return c
    if o.slice_z is not None:
        a = np.ascontiguousarray(o.slice_z, np.int64)
        keep.append(a)
        c.slice_z = a.ctypes.data_as(C.POINTER(C.c_int64))
    c.nz_full = int(o.nz_full)
    if o.kspace_slices is not None:
        a = np.ascontiguousarray(o.kspace_slices, np.int64)
        keep.append(a)
        c.kspace_slices = a.ctypes.data_as(C.POINTER(C.c_int64))
        c.n_kspace_slices = len(o.kspace_slices)
        c.capture_acquired, c.capture_reconstructed, c.capture_coil_images = (int(o.acquired), int(o.reconstructed),
                                                                              int(o.coil_images))
    if o.t_echo_per_volume is not None:
        c.t_echo_per_volume = keep.f64(o.t_echo_per_volume)
    if o.progress is not None:
        cb = abi.PROGRESS_FN(lambda done, total, user: o.progress(done, total))
        keep.append(cb)
        c.progress = cb
    if o.grappa_calibration is not None:
        imgs, seed = o.grappa_calibration
        c.has_grappa_calibration = 1
        c.grappa_calibration_images = keep.ptrs([np.ravel(a) for a in imgs])
        c.grappa_calibration_seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return c


# ---- host tables -------------------------------------------------------------------------------
def sampling_mask(nx: int, ny: int, acq: Acquisition) -> np.ndarray:
    """`sampling_mask` (kspace.rs:546): bool mask, layout kx + nx*ky (returned as [ny, nx])."""
    m = np.zeros(nx * ny, np.uint8)
    check(lib().mrsim_sampling_mask(nx, ny, C.byref(acq.to_c()), m.ctypes.data_as(C.POINTER(C.c_uint8))))
    return m.reshape(ny, nx).astype(bool)


def pf_skipped_lines(ny: int, acq: Acquisition) -> int:
    return int(lib().mrsim_pf_skipped_lines(ny, C.byref(acq.to_c())))


@dataclasses.dataclass
class LineTiming:
    """`LineTiming` (kspace.rs:292-325)."""

    t_ms: np.ndarray
    trf_ms: np.ndarray
    tread_ms: np.ndarray
    polarity: np.ndarray

    @staticmethod
    def for_acquisition(acq: Acquisition, nx: int, ny: int) -> "LineTiming":
        t, trf, tread = (np.zeros(ny) for _ in range(3))
        pol = np.zeros(ny, np.int8)
        check(lib().mrsim_line_timing(C.byref(acq.to_c()), nx, ny, t.ctypes.data_as(abi.c_f64p),
                                      trf.ctypes.data_as(abi.c_f64p), tread.ctypes.data_as(abi.c_f64p),
                                      pol.ctypes.data_as(C.POINTER(C.c_int8))))
        return LineTiming(t, trf, tread, pol)


def validate_acquisition_timing(acq: Acquisition, nx: int, ny: int) -> None:
    check(lib().mrsim_validate_acquisition_timing(C.byref(acq.to_c()), nx, ny))


def epi_order(nx: int, ny: int, acq: Acquisition) -> np.ndarray:
    o = np.zeros(ny, np.int64)
    check(lib().mrsim_epi_order(C.byref(acq.to_c()), nx, ny, o.ctypes.data_as(C.POINTER(C.c_int64))))
    return o


# ---- device context ----------------------------------------------------------------------------
class Context:
    """One CUDA stream + workspace on one device (`mrsim_context`)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().mrsim_context_create(device, C.byref(h)))
        self.handle = h
        self.device = device

    @property
    def stream(self) -> int:
        return lib().mrsim_context_stream(self.handle) or 0

    def synchronize(self):
        check(lib().mrsim_context_synchronize(self.handle))

    def probe_fp32_tflops(self) -> float:
        v = C.c_double()
        check(lib().mrsim_probe_fp32_tflops(self.handle, C.byref(v)))
        return v.value

    def close(self):
        if self.handle:
            lib().mrsim_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default = threading.local()


def default_context(device: int = 0) -> Context:
    ctxs = getattr(_default, "ctxs", None)
    if ctxs is None:
        ctxs = _default.ctxs = {}
    if device not in ctxs:
        ctxs[device] = Context(device)
    return ctxs[device]


# ---- per-slice forward -------------------------------------------------------------------------
def build_coil_kspaces(inp: SliceInput, acq: Acquisition, timing: Optional[LineTiming] = None,
                       log_amp: Optional[np.ndarray] = None, ctx: Optional[Context] = None) -> np.ndarray:
    """Every coil's acquired k-space of one slice (`build_coil_kspace_timed`, kspace.rs:607-1042),
    spikes and noise included: complex128 array [n_coils, ny, nx] (FP32 arithmetic)."""
    ctx = ctx or default_context()
    keep = _Keep()
    s = slice_input_c(inp, keep)
    nx, ny = inp.acq_matrix
    nc = max(int(acq.n_coils), 1)
    out = np.zeros(nc * nx * ny * 2)
    t = [None] * 4
    if timing is not None:
        t = [keep.f64(timing.t_ms), keep.f64(timing.trf_ms), keep.f64(timing.tread_ms)]
        pol = np.ascontiguousarray(timing.polarity, dtype=np.int8)
        keep.append(pol)
        t.append(pol.ctypes.data_as(C.POINTER(C.c_int8)))
    la = keep.f64(np.ravel(log_amp)) if log_amp is not None else None
    check(lib().mrsim_build_coil_kspaces(ctx.handle, C.byref(s), C.byref(acq.to_c()), t[0], t[1], t[2], t[3], la,
                                         out.ctypes.data_as(abi.c_f64p)))
    return out.view(np.complex128).reshape(nc, ny, nx)


def simulate_slice_kspace(inp: SliceInput, acq: Acquisition, ctx: Optional[Context] = None) -> np.ndarray:
    """`simulate_slice_kspace` (kspace.rs:1144): coil 0's acquired k-space [ny, nx]."""
    return build_coil_kspaces(inp, acq, ctx=ctx)[0]


def simulate_slice(inp: SliceInput, acq: Acquisition, ctx: Optional[Context] = None) -> np.ndarray:
    """`simulate_slice` (kspace.rs:1229): the Roemer-combined image [ny, nx] complex64 (f32 pairs)."""
    ctx = ctx or default_context()
    keep = _Keep()
    s = slice_input_c(inp, keep)
    nx, ny = inp.acq_matrix
    out = np.zeros(nx * ny * 2, np.float32)
    check(lib().mrsim_simulate_slice(ctx.handle, C.byref(s), C.byref(acq.to_c()), out.ctypes.data_as(abi.c_f32p)))
    return out.view(np.complex64).reshape(ny, nx)


def simulate_slice_full(inp: SliceInput, acq: Acquisition, capture: bool = True,
                        ctx: Optional[Context] = None) -> dict:
    """`simulate_slice_full` (kspace.rs:1241) with every `SliceCapture` intermediate."""
    ctx = ctx or default_context()
    keep = _Keep()
    s = slice_input_c(inp, keep)
    nx, ny = inp.acq_matrix
    nc = max(int(acq.n_coils), 1)
    comb = np.zeros(nx * ny * 2, np.float32)
    bufs = {k: np.zeros(nc * nx * ny * 2, np.float32) for k in ("acquired", "reconstructed", "coil_images")} \
        if capture else {}
    sens = np.zeros(nc * nx * ny, np.float32)
    mask = np.zeros(nx * ny, np.uint8)

    def p(a):
        return a.ctypes.data_as(abi.c_f32p) if a is not None else None

    check(lib().mrsim_simulate_slice_full(ctx.handle, C.byref(s), C.byref(acq.to_c()), p(comb),
                                          p(bufs.get("acquired")), p(bufs.get("reconstructed")),
                                          p(bufs.get("coil_images")), p(sens),
                                          mask.ctypes.data_as(C.POINTER(C.c_uint8))))
    out = {"combined": comb.view(np.complex64).reshape(ny, nx), "sensitivities": sens.reshape(nc, ny, nx),
           "mask": mask.reshape(ny, nx).astype(bool)}
    for k, v in bufs.items():
        out[k] = v.view(np.complex64).reshape(nc, ny, nx)
    return out


def simulate_acquisition_complex(inp: AcquisitionInput, acq: Acquisition,
                                 opts: Optional[AcquisitionOptions] = None, ctx: Optional[Context] = None) -> dict:
    """`simulate_acquisition_complex` (kspace.rs:1803): re and im in the layout vox*n_volumes + g,
    plus the k-space capture of `opts.kspace_slices` ([vol, slice, coil, ky, kx] complex64)."""
    ctx = ctx or default_context()
    keep = _Keep()
    ci = acquisition_input_c(inp, keep)
    co = acquisition_options_c(opts, keep)
    nx, ny, nz = inp.acq_dims
    nv = inp.n_volumes
    nc = max(int(acq.n_coils), 1)
    n = nx * ny * nz * nv
    re, im = np.zeros(n, np.float32), np.zeros(n, np.float32)
    o = abi.AcquisitionOutput_()
    o.re, o.im = re.ctypes.data_as(abi.c_f32p), im.ctypes.data_as(abi.c_f32p)
    res = {"re": re, "im": im}
    nsl = len(opts.kspace_slices) if opts is not None and opts.kspace_slices is not None else 0
    if nsl:
        for key in ("acquired", "reconstructed", "coil_images"):
            if getattr(opts, key):
                res[key] = np.zeros((nv, nsl, nc, ny, nx), np.complex64)
                setattr(o, key, C.cast(res[key].ctypes.data, abi.c_f32p))
        res["combined"] = np.zeros((nv, nsl, ny, nx), np.complex64)
        o.combined = C.cast(res["combined"].ctypes.data, abi.c_f32p)
        res["mask"] = np.zeros((ny, nx), np.uint8)
        o.mask = res["mask"].ctypes.data_as(C.POINTER(C.c_uint8))
        res["sensitivities"] = np.zeros((nc, ny, nx), np.float32)
        o.sensitivities = res["sensitivities"].ctypes.data_as(abi.c_f32p)
    check(lib().mrsim_simulate_acquisition_complex(ctx.handle, C.byref(ci), C.byref(acq.to_c()),
                                                   C.byref(co) if opts is not None else None, C.byref(o)))
    if "mask" in res:
        res["mask"] = res["mask"].astype(bool)
    return res


def simulate_acquisition_oversampled(inp: AcquisitionInput, acq: Acquisition, ctx: Optional[Context] = None):
    """`simulate_acquisition_oversampled` (kspace.rs:1687): (magnitude, phase), f32."""
    ctx = ctx or default_context()
    keep = _Keep()
    ci = acquisition_input_c(inp, keep)
    nx, ny, nz = inp.acq_dims
    n = nx * ny * nz * inp.n_volumes
    mag, ph = np.zeros(n, np.float32), np.zeros(n, np.float32)
    check(lib().mrsim_simulate_acquisition_oversampled(ctx.handle, C.byref(ci), C.byref(acq.to_c()),
                                                       mag.ctypes.data_as(abi.c_f32p), ph.ctypes.data_as(abi.c_f32p)))
    return mag, ph


def simulate_acquisition_echoes(inp: AcquisitionInput, images_per_echo: Sequence[Sequence[np.ndarray]],
                                acq: Acquisition, echo_times_ms: Sequence[float],
                                grappa_calibration: Optional[Sequence[tuple]] = None, ctx: Optional[Context] = None):
    """`simulate_acquisition_echoes` (kspace.rs:2152): [(magnitude, phase)] per echo."""
    ctx = ctx or default_context()
    keep = _Keep()
    ci = acquisition_input_c(inp, keep, with_images=False)
    ne = len(echo_times_ms)
    ipe = (C.POINTER(abi.c_f32p) * max(ne, 1))()
    for e, imgs in enumerate(images_per_echo):
        ipe[e] = keep.ptrs([np.ravel(a) for a in imgs])
    cal, seeds = None, None
    if grappa_calibration is not None:
        cal = (C.POINTER(abi.c_f32p) * ne)()
        sd = np.zeros(ne, np.uint64)
        for e, (imgs, seed) in enumerate(grappa_calibration):
            cal[e] = keep.ptrs([np.ravel(a) for a in imgs])
            sd[e] = seed
        keep += [cal, sd]
        seeds = sd.ctypes.data_as(C.POINTER(C.c_uint64))
    nx, ny, nz = inp.acq_dims
    n = nx * ny * nz * inp.n_volumes
    mags = [np.zeros(n, np.float32) for _ in range(ne)]
    phs = [np.zeros(n, np.float32) for _ in range(ne)]
    mp = (abi.c_f32p * max(ne, 1))(*[m.ctypes.data_as(abi.c_f32p) for m in mags])
    pp = (abi.c_f32p * max(ne, 1))(*[p.ctypes.data_as(abi.c_f32p) for p in phs])
    check(lib().mrsim_simulate_acquisition_echoes(ctx.handle, C.byref(ci), ipe, C.byref(acq.to_c()),
                                                  keep.f64(echo_times_ms), ne, cal, seeds, mp, pp))
    return list(zip(mags, phs))


# ---- the series forward/adjoint operator ----------------------------------------------------------
def _operator_input(keep, sim_dims, acq_dims, n_volumes, t2, fmap, images=None, t_inhom=None, eddy_drive=None,
                    prep_drive=None, phase=None, seed=0) -> abi.AcquisitionInput_:
    inp = abi.AcquisitionInput_()
    for i in range(3):
        inp.sim_dims[i] = sim_dims[i]
        inp.acq_dims[i] = acq_dims[i]
    inp.n_volumes = n_volumes
    inp.ncomp = len(t2)
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
    if images is not None:
        inp.images = keep.ptrs([np.ravel(a) for a in images])
    keep.append(inp)
    return inp


class EpiBatch:
    """Several series of different geometries as one plan (`mrsim_epi_batch`): each stage of a
    forward or adjoint is one launch over every unit of every series.  `series` holds dicts with
    sim_dims, acq_dims, n_volumes, t2, fmap, images and optionally t_inhom, eddy_drive,
    prep_drive, phase, seed."""

    def __init__(self, series: Sequence[dict], acq: Acquisition, echo_times_ms: Optional[Sequence[float]] = None,
                 grads: int = 0, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        keep = _Keep()
        ins = [_operator_input(keep, s["sim_dims"], s["acq_dims"], s["n_volumes"], s["t2"], s["fmap"],
                               s.get("images"), s.get("t_inhom"), s.get("eddy_drive"), s.get("prep_drive"),
                               s.get("phase"), s.get("seed", 0)) for s in series]
        arr = (C.POINTER(abi.AcquisitionInput_) * len(ins))(*[C.pointer(i) for i in ins])
        tes = keep.f64(np.asarray(echo_times_ms, np.float64)) if echo_times_ms is not None else None
        ne = len(echo_times_ms) if echo_times_ms is not None else 0
        h = C.c_void_p()
        check(lib().mrsim_epi_batch_create(self.ctx.handle, len(ins), arr, C.byref(acq.to_c()), tes, ne, int(grads),
                                           C.byref(h)))
        self.handle = h
        self.series = [dict(s) for s in series]
        self.n_coils = max(int(acq.n_coils), 1)
        self.n_echoes = max(ne, 1)

    @property
    def samples(self) -> int:
        return int(lib().mrsim_epi_batch_samples(self.handle))

    def forward(self):
        check(lib().mrsim_epi_batch_forward(self.handle))

    def adjoint(self):
        check(lib().mrsim_epi_batch_adjoint(self.handle))

    def download(self, i: int) -> dict:
        s = self.series[i]
        snx, sny, nz = s["sim_dims"]
        nx, ny, _ = s["acq_dims"]
        nv, nc = s["n_volumes"], len(s["t2"])
        k = np.zeros((nv, nz, self.n_coils, self.n_echoes, ny, nx), np.complex64)
        g = np.zeros((nv, nz, nc, sny, snx), np.complex64)
        check(lib().mrsim_epi_batch_download(self.handle, i, C.cast(k.ctypes.data, abi.c_f32p),
                                             C.cast(g.ctypes.data, abi.c_f32p)))
        return {"kspace": k, "comp_grad": g}

    def close(self):
        if getattr(self, "handle", None):
            lib().mrsim_epi_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class EpiOperator:
    """The batched forward/adjoint operator of a 2D EPI series (`mrsim_epi_operator`)."""

    def __init__(self, sim_dims, acq_dims, n_volumes: int, t2: Sequence[T2], fmap: np.ndarray, acq: Acquisition,
                 images: Optional[Sequence[np.ndarray]] = None, echo_times_ms: Optional[Sequence[float]] = None,
                 t_inhom: Optional[Sequence[T2]] = None, eddy_drive=None, prep_drive=None,
                 phase: Optional[PhaseModel] = None, seed: int = 0, grads: int = 3,
                 slice_z=None, nz_full: int = 0, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        keep = _Keep()
        inp = _operator_input(keep, sim_dims, acq_dims, n_volumes, t2, fmap, images, t_inhom, eddy_drive, prep_drive,
                              phase, seed)
        tes = keep.f64(np.asarray(echo_times_ms, np.float64)) if echo_times_ms is not None else None
        ne = len(echo_times_ms) if echo_times_ms is not None else 0
        sz = None
        if slice_z is not None:
            a = np.ascontiguousarray(slice_z, dtype=np.int64)
            keep.append(a)
            sz = a.ctypes.data_as(C.POINTER(C.c_int64))
        h = C.c_void_p()
        check(lib().mrsim_epi_operator_create(self.ctx.handle, C.byref(inp), C.byref(acq.to_c()), tes, ne, sz,
                                              int(nz_full), int(grads), C.byref(h)))
        self.handle = h
        self.sim_dims, self.acq_dims, self.n_volumes, self.ncomp = tuple(sim_dims), tuple(acq_dims), n_volumes, len(t2)
        self.n_coils = max(int(acq.n_coils), 1)
        self.n_echoes = max(ne, 1)
        self.grads = grads

    @property
    def samples(self) -> int:
        return int(lib().mrsim_epi_operator_samples(self.handle))

    def buffers(self) -> dict:
        ps = [abi.c_f32p() for _ in range(5)]
        check(lib().mrsim_epi_operator_buffers(self.handle, *[C.byref(p) for p in ps]))
        names = ("images", "kspace", "comp_grad", "fmap_grad", "r2_grad")
        return {n: (C.cast(p, C.c_void_p).value or 0) for n, p in zip(names, ps)}

    def upload_images(self, images: Sequence[np.ndarray]):
        keep = _Keep()
        check(lib().mrsim_epi_operator_upload_images(self.handle, keep.ptrs([np.ravel(a) for a in images])))

    def set_fieldmap(self, fmap: np.ndarray):
        """Replace the fieldmap (Hz, [z][sny][snx] or flat, float32) for the forwards and adjoints
        after this call."""
        snx, sny, nz = self.sim_dims
        f = np.ascontiguousarray(fmap, np.float32).ravel()
        if f.size != snx * sny * nz:
            raise ValueError(f"fieldmap has {f.size} values, the operator {snx * sny * nz}")
        check(lib().mrsim_epi_operator_set_fieldmap(self.handle, C.cast(f.ctypes.data, abi.c_f32p)))

    def forward(self):
        check(lib().mrsim_epi_operator_forward(self.handle))

    def adjoint(self):
        check(lib().mrsim_epi_operator_adjoint(self.handle))

    STAGES = ("statics", "forward_ystage", "forward_xstage", "adjoint_xstage", "adjoint_ystage")

    def stage(self, i: int):
        check(lib().mrsim_epi_operator_stage(self.handle, int(i)))

    def shapes(self) -> dict:
        snx, sny, nz = self.sim_dims
        nx, ny, _ = self.acq_dims
        nv, nc, q, ne = self.n_volumes, self.ncomp, self.n_coils, self.n_echoes
        return {"images": (nv, nz, nc, sny, snx), "kspace": (nv, nz, q, ne, ny, nx),
                "comp_grad": (nv, nz, nc, sny, snx), "fmap_grad": (nv, nz, sny, snx), "r2_grad": (nv, nz, nc, sny, snx)}

    def apply_host(self, images: Optional[Sequence[np.ndarray]], out: Optional[dict] = None) -> dict:
        """Synchronous host-buffer pass: forward, then the adjoint of that k-space.  `out` may hold
        preallocated (e.g. pinned) arrays; complex outputs are complex64."""
        shp = self.shapes()
        if out is None:
            out = {"kspace": np.zeros(shp["kspace"], np.complex64), "comp_grad": np.zeros(shp["comp_grad"], np.complex64),
                   "fmap_grad": np.zeros(shp["fmap_grad"], np.float32) if self.grads & 1 else None,
                   "r2_grad": np.zeros(shp["r2_grad"], np.float32) if self.grads & 2 else None}
        keep = _Keep()
        imgs = keep.ptrs([np.ravel(a) for a in images]) if images is not None else None

        def p(a):
            return None if a is None else C.cast(a.ctypes.data, abi.c_f32p)

        check(lib().mrsim_epi_operator_apply_host(self.handle, imgs, p(out["kspace"]), p(out["comp_grad"]),
                                                  p(out.get("fmap_grad")), p(out.get("r2_grad"))))
        return out

    def acquired_rows(self) -> tuple:
        """(first, step, count): the acquired k-space rows of every echo (count 0: irregular)."""
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().mrsim_epi_operator_acquired_rows(self.handle, C.byref(a), C.byref(b), C.byref(c)))
        return int(a.value), int(b.value), int(c.value)

    def apply_host_compact(self, images: Optional[Sequence[np.ndarray]], out: Optional[dict] = None) -> dict:
        """`apply_host` with the k-space as [g][z][coil][echo][acquired row][kx] (the acquired rows
        only); gradients set to None in `out` are not computed into the host."""
        shp = self.shapes()
        nv, nz, q, ne, ny, nx = shp["kspace"]
        _, _, rows = self.acquired_rows()
        if out is None:
            out = {"kspace": np.zeros((nv, nz, q, ne, rows, nx), np.complex64),
                   "comp_grad": np.zeros(shp["comp_grad"], np.complex64),
                   "fmap_grad": np.zeros(shp["fmap_grad"], np.float32) if self.grads & 1 else None,
                   "r2_grad": np.zeros(shp["r2_grad"], np.float32) if self.grads & 2 else None}
        keep = _Keep()
        imgs = keep.ptrs([np.ravel(a) for a in images]) if images is not None else None

        def p(a):
            return None if a is None else C.cast(a.ctypes.data, abi.c_f32p)

        check(lib().mrsim_epi_operator_apply_host_compact(self.handle, imgs, p(out["kspace"]), p(out.get("comp_grad")),
                                                          p(out.get("fmap_grad")), p(out.get("r2_grad"))))
        return out

    def host_bytes_for(self, kspace=True, comp_grad=True, fmap_grad=True, r2_grad=True) -> tuple:
        """(upload, download) bytes of a host-buffer call with the given outputs."""
        up, down = C.c_int64(), C.c_int64()
        m = (1 if kspace else 0) | (2 if comp_grad else 0) | (4 if fmap_grad else 0) | (8 if r2_grad else 0)
        check(lib().mrsim_epi_operator_host_bytes_for(self.handle, m, C.byref(up), C.byref(down)))
        return int(up.value), int(down.value)

    def host_bytes(self) -> tuple:
        """(upload, download) bytes one `apply_host` call moves over the host link with every
        output requested (acquired k-space rows only when they form a uniform stride)."""
        up, down = C.c_int64(), C.c_int64()
        check(lib().mrsim_epi_operator_host_bytes(self.handle, C.byref(up), C.byref(down)))
        return int(up.value), int(down.value)

    def adjoint_host(self, kspace: np.ndarray) -> dict:
        """Synchronous adjoint / VJP of a host k-space (complex64, the k-space buffer's shape)."""
        shp = self.shapes()
        k = np.ascontiguousarray(kspace, np.complex64)
        if k.shape != shp["kspace"]:
            raise ValueError(f"k-space shape {k.shape} != {shp['kspace']}")
        out = {"comp_grad": np.zeros(shp["comp_grad"], np.complex64),
               "fmap_grad": np.zeros(shp["fmap_grad"], np.float32) if self.grads & 1 else None,
               "r2_grad": np.zeros(shp["r2_grad"], np.float32) if self.grads & 2 else None}

        def p(a):
            return None if a is None else C.cast(a.ctypes.data, abi.c_f32p)

        check(lib().mrsim_epi_operator_adjoint_host(self.handle, p(k), p(out["comp_grad"]), p(out["fmap_grad"]),
                                                    p(out["r2_grad"])))
        return out

    SEGMENTED = {"exact": 0, "f16": 1, "bf16": 2}

    def set_segmented(self, precision: str = "f16"):
        """Select the y-stages: "exact" (per-line phasors, FP32), or the time-segmented tensor-core
        contractions in split "f16" or split "bf16" (`mrsim_epi_operator_set_segmented`)."""
        check(lib().mrsim_epi_operator_set_segmented(self.handle, self.SEGMENTED[precision]))

    def segmentation(self) -> dict:
        """The segmentation in use: per-group segment counts and certified bounds, and the tensor
        FLOP of one forward and one adjoint pass (empty lists on the exact path)."""
        n = C.c_int32()
        ls = (C.c_int32 * 64)()
        bs = (C.c_double * 64)()
        ff, fa = C.c_double(), C.c_double()
        check(lib().mrsim_epi_operator_segmentation(self.handle, C.byref(n), ls, bs, 64, C.byref(ff), C.byref(fa)))
        k = min(int(n.value), 64)
        return {"L": [int(ls[i]) for i in range(k)], "bound": [float(bs[i]) for i in range(k)],
                "flops_forward": float(ff.value), "flops_adjoint": float(fa.value)}

    def tune(self, cache_path: Optional[str] = None, segmented: bool = False) -> dict:
        """The autotuner (`mrsim_epi_operator_tune`): keeps the fastest plan for this shape and
        returns {"choice": ..., "ms": timed forward + adjoint of the timed units, 0 if cached}."""
        buf = C.create_string_buffer(256)
        ms = C.c_double()
        check(lib().mrsim_epi_operator_tune(self.handle, str(cache_path).encode() if cache_path else None,
                                            1 if segmented else 0, buf, 256, C.byref(ms)))
        return {"choice": buf.value.decode(), "ms": float(ms.value)}

    def segmented_status(self) -> int:
        code = C.c_int32()
        check(lib().mrsim_epi_operator_segmented_status(self.handle, C.byref(code)))
        return int(code.value)

    def close(self):
        if getattr(self, "handle", None):
            lib().mrsim_epi_operator_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
