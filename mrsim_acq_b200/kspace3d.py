"""Python mirror of the reference's 3D echo-train acquisition (`kspace3d.rs`, `readout.rs:75-700`)
over the C ABI: `EchoTrain`, `KzOrder`, `Readout3d::Grase` / `Readout3d::Spiral`, `KzSampling`,
`KzOptions`, `LineWeights`, `kz_order`, `grase_lines`, `spiral_lines`, `simulate_acquisition_3d`
(GRASE or stack of spirals), `kspace_3d_observed` and `spiral_samples_3d`; and the 3D
gradient-echo train: `ExcitationTrain`, `Ge3dReadout`, `GeVolume`, `ge3d_lines`,
`simulate_acquisition_3d_ge`.  The acquisition runs on
the device (no CPU path)."""
from __future__ import annotations

import ctypes as C
import dataclasses
import enum
from typing import Optional, Sequence

import numpy as np

from . import abi
from .abi import check, lib
from .api import Acquisition, Context, PhaseModel, T2, _Keep, default_context


class KzOrder(enum.IntEnum):  # readout.rs:75-80
    Centric = 0
    Linear = 1


@dataclasses.dataclass
class EchoTrain:
    """`EchoTrain` (readout.rs:82-95)."""

    etl: int
    esp_ms: float
    refocusing_deg: float
    kz_order: KzOrder = KzOrder.Centric
    kz_segments: int = 1
    refocusing_time_ms: float = 2.0

    def to_c(self) -> abi.EchoTrain_:
        return abi.EchoTrain_(int(self.etl), float(self.esp_ms), float(self.refocusing_deg), int(self.kz_order), 0,
                              int(self.kz_segments), float(self.refocusing_time_ms))


@dataclasses.dataclass
class GraseReadout:
    """`Readout3d::Grase` (readout.rs:103-106)."""

    ky_segments: int
    t_line_ms: float
    reverse_phase: bool = False

    def to_c(self) -> abi.GraseReadout_:
        return abi.GraseReadout_(int(self.ky_segments), float(self.t_line_ms), int(bool(self.reverse_phase)), 0)


@dataclasses.dataclass
class KzSampling:
    """`KzSampling` (readout.rs:107-160)."""

    partial_fourier: float = 1.0
    accel: int = 1

    def to_c(self) -> abi.KzSampling_:
        return abi.KzSampling_(float(self.partial_fourier), int(self.accel))


@dataclasses.dataclass
class SpiralReadout:
    """`Readout3d::Spiral` (readout.rs:103-106)."""

    interleaves: int
    readout_ms: float
    dwell_ms: float
    radial_oversampling: float = 1.2
    kz: KzSampling = dataclasses.field(default_factory=KzSampling)

    def to_c(self) -> abi.SpiralReadout_:
        return abi.SpiralReadout_(int(self.interleaves), float(self.readout_ms), float(self.dwell_ms),
                                  float(self.radial_oversampling), self.kz.to_c())


@dataclasses.dataclass
class KzOptions:
    """`KzOptions` (kspace3d.rs:1173-1178): calibration_images one sim volume per compartment."""

    coil_rows: int = 1
    calibration_images: Optional[Sequence[np.ndarray]] = None
    calibration_seed: int = 0
    pocs: bool = False

    def to_c(self, keep: _Keep) -> abi.KzOptions_:
        o = abi.KzOptions_()
        o.coil_rows = int(self.coil_rows)
        if self.calibration_images is not None:
            o.calibration_images = keep.ptrs([np.ravel(a) for a in self.calibration_images])
        o.calibration_seed = int(self.calibration_seed) & 0xFFFFFFFFFFFFFFFF
        o.pocs = int(bool(self.pocs))
        keep.append(o)
        return o


@dataclasses.dataclass
class SpiralTable:
    """`Spiral3dTable` (readout.rs:622-651), per partition."""

    acquired: np.ndarray
    echo: np.ndarray
    kz_segment: np.ndarray
    band_start: int
    e_c: int
    n_shots: int
    samples_per_interleaf: int


def spiral_lines(train: EchoTrain, ro: SpiralReadout, nx: int, ny: int, nz: int) -> SpiralTable:
    acq = np.zeros(nz, np.uint8)
    echo, seg = np.zeros(nz, np.int64), np.zeros(nz, np.int64)
    vals = [C.c_int64() for _ in range(4)]
    P = C.POINTER(C.c_int64)
    check(lib().mrsim_spiral_lines(C.byref(train.to_c()), C.byref(ro.to_c()), nx, ny, nz,
                                   acq.ctypes.data_as(C.POINTER(C.c_uint8)), echo.ctypes.data_as(P),
                                   seg.ctypes.data_as(P), *[C.byref(v) for v in vals]))
    return SpiralTable(acq.astype(bool), echo, seg, *[v.value for v in vals])


@dataclasses.dataclass
class LineWeights:
    """`LineWeights` (kspace3d.rs:46-60): w[(g * n_shots + s) * n_compartments + c]."""

    n_shots: int
    n_compartments: int
    w: np.ndarray


@dataclasses.dataclass
class GraseTable:
    """`Grase3dTable` (readout.rs:236-280): per line p * ny + ky."""

    shot: np.ndarray
    echo: np.ndarray
    t_ms: np.ndarray
    trf_ms: np.ndarray
    polarity: np.ndarray
    e_c: int
    n_shots: int


def kz_order(nz: int, order: KzOrder) -> np.ndarray:
    out = np.zeros(nz, np.int64)
    check(lib().mrsim_kz_order(nz, int(order), out.ctypes.data_as(C.POINTER(C.c_int64))))
    return out


def grase_lines(train: EchoTrain, ro: GraseReadout, ny: int, nz: int) -> GraseTable:
    n = ny * nz
    shot, echo = np.zeros(n, np.int64), np.zeros(n, np.int64)
    t, trf, pol = np.zeros(n), np.zeros(n), np.zeros(n, np.int8)
    e_c, n_shots = C.c_int64(), C.c_int64()
    P = C.POINTER(C.c_int64)
    check(lib().mrsim_grase_lines(C.byref(train.to_c()), C.byref(ro.to_c()), ny, nz, shot.ctypes.data_as(P),
                                  echo.ctypes.data_as(P), t.ctypes.data_as(abi.c_f64p), trf.ctypes.data_as(abi.c_f64p),
                                  pol.ctypes.data_as(C.POINTER(C.c_int8)), C.byref(e_c), C.byref(n_shots)))
    return GraseTable(shot, echo, t, trf, pol, e_c.value, n_shots.value)


@dataclasses.dataclass
class ShotSet:
    """`ShotSet` (kspace3d.rs:59-65): the images one set of shots of one volume saw (per-shot
    motion), one simulation-grid volume (x + snx*(y + sny*z)) per compartment.  Every line (spiral:
    interleave) of a shot in `shots` is computed from these images; a shot in several sets takes
    the first."""

    shots: Sequence[int]
    images: Sequence[Optional[np.ndarray]]


def shot_sets_c(sets: Sequence[ShotSet], keep: _Keep):
    """A C array of `mrsim_shot_set` (None images stay NULL)."""
    arr = (abi.ShotSet_ * max(1, len(sets)))()
    for i, st in enumerate(sets):
        sh = np.ascontiguousarray(st.shots, np.int64)
        keep.append(sh)
        ps = (abi.c_f32p * max(1, len(st.images)))()
        for c, im in enumerate(st.images):
            ps[c] = keep.f32(np.ravel(im)) if im is not None and np.size(im) > 0 else None
        keep.append(ps)
        arr[i] = abi.ShotSet_(sh.ctypes.data_as(C.POINTER(C.c_int64)), sh.size, ps)
    keep.append(arr)
    return arr


def acquisition_3d_input_c(sim_dims, acq_dims, n_volumes, images, t2: Sequence[T2], t1: Optional[Sequence[T2]], fmap,
                           t_inhom: Optional[Sequence[T2]], phase: Optional[PhaseModel],
                           line_weights: Optional[LineWeights], grappa_calibration, keep: _Keep,
                           shot_images: Optional[Sequence[Sequence[ShotSet]]] = None):
    s = abi.Acquisition3dInput_()
    for i in range(3):
        s.sim_dims[i] = int(sim_dims[i])
        s.acq_dims[i] = int(acq_dims[i])
    s.n_volumes = int(n_volumes)
    s.ncomp = len(images)
    s.images = keep.ptrs([np.ravel(a) for a in images])
    s.t2 = keep.t2s(t2)
    s.t1 = keep.t2s(t1) if t1 is not None else None
    s.fmap = keep.f32(np.ravel(fmap))
    s.t_inhom = keep.t2s(t_inhom) if t_inhom is not None else None
    if phase is not None:
        pm = phase.to_c()
        keep.append(pm)
        s.phase = C.pointer(pm)
    if line_weights is not None:
        s.line_weights = keep.f64(np.ravel(line_weights.w))
    if grappa_calibration is not None:
        cal_images, cal_seed = grappa_calibration
        s.has_grappa_calibration = 1
        s.grappa_calibration_images = keep.ptrs([np.ravel(a) for a in cal_images])
        s.grappa_calibration_seed = int(cal_seed) & 0xFFFFFFFFFFFFFFFF
    if shot_images is not None:
        if len(shot_images) != n_volumes:
            raise ValueError("shot images per volume")
        lists = (C.POINTER(abi.ShotSet_) * max(1, n_volumes))()
        counts = np.zeros(max(1, n_volumes), np.int64)
        for g, sets in enumerate(shot_images):
            if sets:
                lists[g] = C.cast(shot_sets_c(sets, keep), C.POINTER(abi.ShotSet_))
                counts[g] = len(sets)
        keep.append(lists)
        keep.append(counts)
        s.shot_sets = lists
        s.n_shot_sets = counts.ctypes.data_as(C.POINTER(C.c_int64))
    return s


def simulate_acquisition_3d(sim_dims, acq_dims, n_volumes: int, images, t2: Sequence[T2], t1: Optional[Sequence[T2]],
                            fmap, t_inhom: Optional[Sequence[T2]], acq: Acquisition, train: EchoTrain,
                            readout, line_weights: Optional[LineWeights] = None,
                            phase: Optional[PhaseModel] = None, seed: int = 0, grappa_calibration=None,
                            kz_opts: Optional[KzOptions] = None, ctx: Optional[Context] = None,
                            shot_images: Optional[Sequence[Sequence[ShotSet]]] = None):
    """`simulate_acquisition_3d` / `_kz` (kspace3d.rs:549-589), GRASE or stack of spirals:
    (magnitude, phase) f32 at vox * nv + g.  `shot_images`: per volume its ShotSets, or None."""
    ctx = ctx or default_context()
    keep = _Keep()
    s = acquisition_3d_input_c(sim_dims, acq_dims, n_volumes, images, t2, t1, fmap, t_inhom, phase, line_weights,
                               grappa_calibration, keep, shot_images)
    n = int(np.prod(acq_dims)) * n_volumes
    mag, ph = np.zeros(n, np.float32), np.zeros(n, np.float32)
    if isinstance(readout, SpiralReadout):
        ko = C.byref(kz_opts.to_c(keep)) if kz_opts is not None else None
        check(lib().mrsim_simulate_acquisition_3d_spiral(ctx.handle, C.byref(s), C.byref(acq.to_c()),
                                                         C.byref(train.to_c()), C.byref(readout.to_c()), ko,
                                                         int(seed) & 0xFFFFFFFFFFFFFFFF,
                                                         mag.ctypes.data_as(abi.c_f32p), ph.ctypes.data_as(abi.c_f32p)))
        return mag, ph
    if kz_opts is not None:
        raise ValueError("coil rings along z and kz undersampling are the stack of spirals', not GRASE's")
    check(lib().mrsim_simulate_acquisition_3d(ctx.handle, C.byref(s), C.byref(acq.to_c()), C.byref(train.to_c()),
                                              C.byref(readout.to_c()), int(seed) & 0xFFFFFFFFFFFFFFFF,
                                              mag.ctypes.data_as(abi.c_f32p), ph.ctypes.data_as(abi.c_f32p)))
    return mag, ph


def spiral_samples_3d(sim_dims, acq_dims, n_volumes: int, images, t2: Sequence[T2], t1: Optional[Sequence[T2]], fmap,
                      t_inhom: Optional[Sequence[T2]], acq: Acquisition, train: EchoTrain, readout: SpiralReadout,
                      line_weights: Optional[LineWeights] = None, phase: Optional[PhaseModel] = None, g: int = 0,
                      kz_opts: Optional[KzOptions] = None, ctx: Optional[Context] = None,
                      shot_images: Optional[Sequence[Sequence[ShotSet]]] = None) -> np.ndarray:
    """`SpiralPlan::samples_all` (kspace3d.rs:1047-1060): complex64 [coil, partition, sample] before noise."""
    ctx = ctx or default_context()
    keep = _Keep()
    s = acquisition_3d_input_c(sim_dims, acq_dims, n_volumes, images, t2, t1, fmap, t_inhom, phase, line_weights,
                               None, keep, shot_images)
    nz = acq_dims[2]
    tab = spiral_lines(train, readout, acq_dims[0], acq_dims[1], nz)
    nsamp = tab.samples_per_interleaf * readout.interleaves
    nc = max(int(acq.n_coils), 1)
    out = np.zeros(nc * nz * nsamp, np.complex64)
    ko = C.byref(kz_opts.to_c(keep)) if kz_opts is not None else None
    check(lib().mrsim_spiral_samples_3d(ctx.handle, C.byref(s), C.byref(acq.to_c()), C.byref(train.to_c()),
                                        C.byref(readout.to_c()), ko, g,
                                        out.view(np.float32).ctypes.data_as(abi.c_f32p)))
    return out.reshape(nc, nz, nsamp)


def kspace_3d_observed(sim_dims, acq_dims, n_volumes: int, images, t2: Sequence[T2], t1: Optional[Sequence[T2]], fmap,
                       t_inhom: Optional[Sequence[T2]], acq: Acquisition, train: EchoTrain, readout: GraseReadout,
                       line_weights: Optional[LineWeights] = None, phase: Optional[PhaseModel] = None, g: int = 0,
                       ctx: Optional[Context] = None,
                       shot_images: Optional[Sequence[Sequence[ShotSet]]] = None) -> np.ndarray:
    """`kspace_3d_observed` (kspace3d.rs:439-456): complex64 [coil, p, ky, kx] of volume g."""
    ctx = ctx or default_context()
    keep = _Keep()
    s = acquisition_3d_input_c(sim_dims, acq_dims, n_volumes, images, t2, t1, fmap, t_inhom, phase, line_weights,
                               None, keep, shot_images)
    nx, ny, nz = acq_dims
    nc = max(int(acq.n_coils), 1)
    out = np.zeros(nc * nz * ny * nx, np.complex64)
    check(lib().mrsim_kspace_3d_observed(ctx.handle, C.byref(s), C.byref(acq.to_c()), C.byref(train.to_c()),
                                         C.byref(readout.to_c()), g, out.view(np.float32).ctypes.data_as(abi.c_f32p)))
    return out.reshape(nc, nz, ny, nx)


# ---- the 3D gradient-echo train ------------------------------------------------------------------------
@dataclasses.dataclass
class ExcitationTrain:
    """`ExcitationTrain` (readout.rs:362-369)."""

    kz_segments: int
    kz_order: KzOrder
    exc_spacing_ms: float
    echo_times_ms: Sequence[float]
    excitation_time_ms: float = 2.0

    def to_c(self, keep: _Keep) -> abi.ExcitationTrain_:
        t = abi.ExcitationTrain_()
        t.kz_segments = int(self.kz_segments)
        t.kz_order = int(self.kz_order)
        t.exc_spacing_ms = float(self.exc_spacing_ms)
        t.echo_times_ms = keep.f64(np.asarray(self.echo_times_ms, dtype=np.float64))
        t.n_echoes = len(self.echo_times_ms)
        t.excitation_time_ms = float(self.excitation_time_ms)
        keep.append(t)
        return t


@dataclasses.dataclass
class Ge3dReadout:
    """`Ge3dReadout` (readout.rs:374-379)."""

    ky_segments: int
    t_line_ms: float
    reverse_phase: bool = False

    def to_c(self) -> abi.Ge3dReadout_:
        return abi.Ge3dReadout_(int(self.ky_segments), float(self.t_line_ms), int(bool(self.reverse_phase)), 0)


@dataclasses.dataclass
class GeVolume:
    """`GeVolume` (kspace3d.rs:592-603): per compartment one sim volume (None = unused), the
    excitation weights w[(p * ky_segments + sy) * ncomp + c] and the per-shot images."""

    images: Sequence[Optional[np.ndarray]]
    weights: np.ndarray
    shot_images: Optional[Sequence[ShotSet]] = None


@dataclasses.dataclass
class GeTable:
    """`Ge3dTable` (readout.rs:393-407)."""

    shot: np.ndarray
    excitation: np.ndarray
    t_ms: np.ndarray
    polarity: np.ndarray
    n_shots: int
    n_exc: int
    e_c: int


def ge3d_lines(train: ExcitationTrain, ro: Ge3dReadout, ny: int, nz: int) -> GeTable:
    keep = _Keep()
    n = ny * nz
    shot, exc = np.zeros(n, np.int64), np.zeros(n, np.int64)
    t, pol = np.zeros(n), np.zeros(n, np.int8)
    vals = [C.c_int64() for _ in range(3)]
    P = C.POINTER(C.c_int64)
    check(lib().mrsim_ge3d_lines(C.byref(train.to_c(keep)), C.byref(ro.to_c()), ny, nz, shot.ctypes.data_as(P),
                                 exc.ctypes.data_as(P), t.ctypes.data_as(abi.c_f64p),
                                 pol.ctypes.data_as(C.POINTER(C.c_int8)), *[C.byref(v) for v in vals]))
    return GeTable(shot, exc, t, pol, *[v.value for v in vals])


class _GeVolumes:
    """The `volume` callback over a Python callable, keeping each volume's buffers alive."""

    def __init__(self, volume, ncomp):
        self.volume, self.ncomp, self.keep = volume, ncomp, None
        self.error = None
        self.fn = abi.GE_VOLUME_FN(self._call)

    @staticmethod
    def fill(v: GeVolume, ncomp: int, keep: _Keep) -> abi.GeVolume_:
        out = abi.GeVolume_()
        ps = (abi.c_f32p * max(1, ncomp))()
        for c in range(ncomp):
            im = v.images[c]
            ps[c] = keep.f32(np.ravel(im)) if im is not None and np.size(im) > 0 else None
        keep.append(ps)
        out.images = ps
        out.weights = keep.f64(np.ravel(v.weights))
        if v.shot_images:
            out.shot_sets = C.cast(shot_sets_c(v.shot_images, keep), C.POINTER(abi.ShotSet_))
            out.n_shot_sets = len(v.shot_images)
        return out

    def _call(self, g, user, out):
        try:
            self.keep = _Keep()
            out[0] = self.fill(self.volume(int(g)), self.ncomp, self.keep)
            return 0
        except Exception as e:  # the library turns a non-zero return into an error
            self.error = e
            return 1


def ge_input_c(sim_dims, acq_dims, n_volumes, t2: Sequence[T2], fmap, t_inhom: Optional[Sequence[T2]],
               phase: Optional[PhaseModel], vols: _GeVolumes, reference: Optional[GeVolume], keep: _Keep):
    s = abi.AcquisitionGeInput_()
    for i in range(3):
        s.sim_dims[i] = int(sim_dims[i])
        s.acq_dims[i] = int(acq_dims[i])
    s.n_volumes = int(n_volumes)
    s.ncomp = len(t2)
    s.t2 = keep.t2s(t2)
    s.fmap = keep.f32(np.ravel(fmap))
    s.t_inhom = keep.t2s(t_inhom) if t_inhom is not None else None
    if phase is not None:
        pm = phase.to_c()
        keep.append(pm)
        s.phase = C.pointer(pm)
    s.volume = vols.fn
    if reference is not None:
        r = _GeVolumes.fill(reference, len(t2), keep)
        keep.append(r)
        s.reference = C.pointer(r)
    return s


def simulate_acquisition_3d_ge(sim_dims, acq_dims, n_volumes: int, t2: Sequence[T2], fmap,
                               t_inhom: Optional[Sequence[T2]], acq: Acquisition, train: ExcitationTrain,
                               readout: Ge3dReadout, volume, phase: Optional[PhaseModel] = None, seed: int = 0,
                               reference: Optional[GeVolume] = None, ctx: Optional[Context] = None):
    """`simulate_acquisition_3d_ge` (kspace3d.rs:837-856): per echo (magnitude, phase) f32 at vox * nv + g.
    `volume(g)` returns the GeVolume of volume g, called once per volume on this thread."""
    ctx = ctx or default_context()
    keep = _Keep()
    vols = _GeVolumes(volume, len(t2))
    s = ge_input_c(sim_dims, acq_dims, n_volumes, t2, fmap, t_inhom, phase, vols, reference, keep)
    n = int(np.prod(acq_dims)) * n_volumes
    ne = len(train.echo_times_ms)
    mags = [np.zeros(n, np.float32) for _ in range(ne)]
    phs = [np.zeros(n, np.float32) for _ in range(ne)]
    mp = (abi.c_f32p * ne)(*[m.ctypes.data_as(abi.c_f32p) for m in mags])
    pp = (abi.c_f32p * ne)(*[p.ctypes.data_as(abi.c_f32p) for p in phs])
    status = lib().mrsim_simulate_acquisition_3d_ge(ctx.handle, C.byref(s), C.byref(acq.to_c()),
                                                    C.byref(train.to_c(keep)), C.byref(readout.to_c()),
                                                    int(seed) & 0xFFFFFFFFFFFFFFFF, mp, pp)
    if vols.error is not None:
        raise vols.error
    check(status)
    return list(zip(mags, phs))


# ---- timing checks of the trains (readout.rs:286-288, 326-354, 460-500, 702-730) -------------------
def esp_from_echo_time(te_ms: float, e_c: int, ro: GraseReadout, ny: int) -> float:
    return float(lib().mrsim_esp_from_echo_time(te_ms, e_c, C.byref(ro.to_c()), ny))


def spiral_esp_from_echo_time(te_ms: float, e_c: int) -> float:
    return float(lib().mrsim_spiral_esp_from_echo_time(te_ms, e_c))


def check_grase_timing(train: EchoTrain, ro: GraseReadout, ny: int, nz: int, t_exc_ms: float, tr_ms: float) -> None:
    check(lib().mrsim_check_grase_timing(C.byref(train.to_c()), C.byref(ro.to_c()), ny, nz, t_exc_ms, tr_ms))


def check_ge3d_timing(train: ExcitationTrain, ro: Ge3dReadout, ny: int, nz: int, t_exc_ms: float, tr_ms: float) -> None:
    keep = _Keep()
    check(lib().mrsim_check_ge3d_timing(C.byref(train.to_c(keep)), C.byref(ro.to_c()), ny, nz, t_exc_ms, tr_ms))


def check_spiral_timing(train: EchoTrain, ro: SpiralReadout, nx: int, ny: int, nz: int, t_exc_ms: float,
                        tr_ms: float) -> float:
    end = C.c_double()
    check(lib().mrsim_check_spiral_timing(C.byref(train.to_c()), C.byref(ro.to_c()), nx, ny, nz, t_exc_ms, tr_ms,
                                          C.byref(end)))
    return end.value


def spiral_segmentation(sim_dims, acq_dims, t2: Sequence[T2], t1: Optional[Sequence[T2]], fmap,
                        t_inhom: Optional[Sequence[T2]], acq: Acquisition, train: EchoTrain, readout: SpiralReadout):
    """`spiral_segmentation` (kspace3d.rs:1441-1470): a list of dicts (z, voxel, l, m, b_sum, bound)."""
    keep = _Keep()
    s = acquisition_3d_input_c(sim_dims, acq_dims, 0, [np.zeros(1, np.float32)] * len(t2), t2, t1, fmap, t_inhom,
                               None, None, None, keep)
    n = C.c_int64()
    check(lib().mrsim_spiral_segmentation(C.byref(s), C.byref(acq.to_c()), C.byref(train.to_c()),
                                          C.byref(readout.to_c()), 0, None, C.byref(n)))
    rows = (abi.SpiralSegmentationRow_ * max(1, n.value))()
    check(lib().mrsim_spiral_segmentation(C.byref(s), C.byref(acq.to_c()), C.byref(train.to_c()),
                                          C.byref(readout.to_c()), n.value, rows, C.byref(n)))
    return [dict(z=r.z, voxel=bool(r.voxel), l=r.l, m=r.m, b_sum=r.b_sum, bound=r.bound) for r in rows[:n.value]]
