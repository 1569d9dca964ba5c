"""Spin history of slice-selective excitations under head motion (reference `spin_history.rs`), on
the device.

Mirrors the reference's names: `Source` (spin_history.rs:42-50), `Slabs` (:53-57), `Pulse`
(`Inversion`, `Saturation`, :63-69), `SliceTerms` (:80-85), `SpinHistory` with `prime` (:303),
`excite` (:311) and `merges` (:296), and `NO_CLASS` / `MAX_PIECES` (:34-37).  Source arrays use
the reference's layout `x + nx*(y + ny*z)`; `v2w` matrices are 4x4 voxel-to-world affines and a
shot's `transform` is the world-space head transform (p' = m p), as `Pose.to_matrix` makes it.

The reference's `mz_ref` is a closure of T1.  Here it is either a callable (evaluated once per
distinct T1 of the tracked voxels on the host, then looked up per voxel on the device) or one of
the closed forms the device evaluates itself: `Recovery(tau, a)` = 1 - (1 - a) e^{-tau/T1},
`Constant(a, b)` = a where T1 > 0 else b, `Replay(mz, t_from)` = the static head's Mz at the shot
from `mz` just after `t_from` through the series' pulses.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Callable, Optional, Sequence, Union

import numpy as np

from . import abi
from .abi import check, lib
from .api import Context, default_context

NO_CLASS = 255
MAX_PIECES = 8


@dataclasses.dataclass
class Source:
    """The tissue in the head frame: per voxel T1 (s), weight and class (`NO_CLASS`: untracked)."""

    dims: Sequence[int]
    v2w: np.ndarray
    t1: np.ndarray
    weight: np.ndarray
    cls: np.ndarray
    n_classes: int


@dataclasses.dataclass
class Slabs:
    """The slice stack in the scanner frame: the grid whose z index is the slice."""

    dims: Sequence[int]
    v2w: np.ndarray


@dataclasses.dataclass(frozen=True)
class Inversion:
    t: float
    epsilon: float = 1.0


@dataclasses.dataclass(frozen=True)
class Saturation:
    t: float


@dataclasses.dataclass(frozen=True)
class Recovery:
    """mz_ref = 1 - (1 - a) e^{-tau / T1}: recovery from `a` over `tau` seconds."""

    tau: float
    a: float = 0.0


@dataclasses.dataclass(frozen=True)
class Constant:
    """mz_ref = a where T1 > 0, else b."""

    a: float
    b: float = 0.0


@dataclasses.dataclass(frozen=True)
class Replay:
    """mz_ref = Mz at the shot's time from `mz` just after `t_from`, through the series' pulses."""

    mz: float
    t_from: float


MzRef = Union[Recovery, Constant, Replay, Callable[[float], float], None]


@dataclasses.dataclass
class SliceTerms:
    """One excited slice's terms, `[class][x + nx*y]` on the slab grid."""

    slice: int
    num: np.ndarray
    den: np.ndarray


@dataclasses.dataclass
class Shot:
    """One excitation: time (s), head transform, slab indices, reference (None: read no terms, as
    `prime` does) and an optional per-source-voxel weight for this shot only."""

    t: float
    transform: np.ndarray
    slices: Sequence[int]
    mz_ref: MzRef = None
    weight: Optional[np.ndarray] = None


def pulses_c(pulses) -> tuple:
    arr = (abi.Pulse_ * max(len(pulses), 1))()
    for i, p in enumerate(pulses):
        if isinstance(p, Inversion):
            arr[i] = abi.Pulse_(0, float(p.t), float(p.epsilon))
        elif isinstance(p, Saturation):
            arr[i] = abi.Pulse_(1, float(p.t), 0.0)
        else:
            raise TypeError(f"not a pulse: {p!r}")
    return arr, len(pulses)


class _RefValues:
    """Per-tracked-voxel values of a callable reference (one call per distinct T1)."""

    def __init__(self, tracked_t1: np.ndarray):
        self.uniq, self.inv = np.unique(tracked_t1, return_inverse=True)

    def __call__(self, f) -> np.ndarray:
        vals = np.array([float(f(float(t))) for t in self.uniq], np.float64)
        return np.ascontiguousarray(vals[self.inv])


def shots_c(shots: Sequence[Shot], ref_values: _RefValues, keep: list):
    """The C array of `mrsim_spin_shot` (arrays it points to are kept alive in `keep`)."""
    arr = (abi.SpinShot_ * max(len(shots), 1))()
    for i, s in enumerate(shots):
        sl = np.ascontiguousarray(s.slices, np.int64)
        keep.append(sl)
        m = np.ascontiguousarray(s.transform, np.float64).reshape(16)
        r = abi.MzReference_(0, 0.0, 0.0, None)
        ref = s.mz_ref
        if ref is None:
            pass
        elif isinstance(ref, Recovery):
            r = abi.MzReference_(1, float(ref.a), float(ref.tau), None)
        elif isinstance(ref, Constant):
            r = abi.MzReference_(2, float(ref.a), float(ref.b), None)
        elif isinstance(ref, Replay):
            r = abi.MzReference_(3, float(ref.mz), float(ref.t_from), None)
        elif callable(ref):
            v = ref_values(ref)
            keep.append(v)
            r = abi.MzReference_(4, 0.0, 0.0, v.ctypes.data_as(abi.c_f64p))
        else:
            raise TypeError(f"not a reference magnetisation: {ref!r}")
        w = None
        if s.weight is not None:
            wa = np.ascontiguousarray(s.weight, np.float32).ravel()
            keep.append(wa)
            w = wa.ctypes.data_as(abi.c_f32p)
        arr[i] = abi.SpinShot_(float(s.t), (C.c_double * 16)(*m.tolist()),
                               sl.ctypes.data_as(C.POINTER(C.c_int64)), sl.size, r, w)
    return arr


def unpack_terms(shots: Sequence[Shot], flat: np.ndarray, n_classes: int, cells: int) -> list:
    """The packed terms ([slice in shot][num, den][class][cell] per reading shot) as SliceTerms."""
    out, o = [], 0
    for s in shots:
        if s.mz_ref is None:
            out.append(None)
            continue
        terms = []
        for z in s.slices:
            blk = flat[o:o + 2 * n_classes * cells].reshape(2, n_classes, cells)
            terms.append(SliceTerms(int(z), blk[0].copy(), blk[1].copy()))
            o += 2 * n_classes * cells
        out.append(terms)
    return out


class PreparedShots:
    """Shots marshalled once into the C shot array (`SpinHistory.prepare`), for callers that run
    the same shot list again or want the marshalling out of a timed loop."""

    def __init__(self, shots: Sequence[Shot], ref_values: "_RefValues"):
        self.shots = list(shots)
        self.keep: list = []
        self.arr = shots_c(self.shots, ref_values, self.keep)

    def __len__(self):
        return len(self.shots)


class SpinHistory:
    """`SpinHistory` (spin_history.rs:171-422) with its state resident on the device."""

    def __init__(self, source: Source, slabs: Slabs, pulses: Sequence = (), ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        dims = np.ascontiguousarray(source.dims, np.int64)
        nv = int(np.prod(dims))
        t1 = np.ascontiguousarray(source.t1, np.float32).ravel()
        w = np.ascontiguousarray(source.weight, np.float32).ravel()
        cls = np.ascontiguousarray(source.cls, np.uint8).ravel()
        if t1.size != nv or w.size != nv or cls.size != nv:
            raise ValueError("one value per source voxel")
        sdims = np.ascontiguousarray(slabs.dims, np.int64)
        v2w = np.ascontiguousarray(source.v2w, np.float64).reshape(16)
        sv2w = np.ascontiguousarray(slabs.v2w, np.float64).reshape(16)
        parr, npul = pulses_c(list(pulses))
        h = C.c_void_p()
        check(lib().mrsim_spin_history_create(self.ctx.handle, dims.ctypes.data_as(C.POINTER(C.c_int64)),
                                              v2w.ctypes.data_as(abi.c_f64p), t1.ctypes.data_as(abi.c_f32p),
                                              w.ctypes.data_as(abi.c_f32p),
                                              cls.ctypes.data_as(C.POINTER(C.c_uint8)), int(source.n_classes),
                                              sdims.ctypes.data_as(C.POINTER(C.c_int64)),
                                              sv2w.ctypes.data_as(abi.c_f64p), parr, npul, C.byref(h)))
        self._h = h
        self.n_classes = int(source.n_classes)
        self.cells = int(sdims[0] * sdims[1])
        self._ref_values = _RefValues(t1[cls != NO_CLASS].astype(np.float64))

    @property
    def handle(self):
        return self._h

    @property
    def n_tracked(self) -> int:
        n = C.c_int64()
        check(lib().mrsim_spin_history_n_tracked(self._h, C.byref(n)))
        return n.value

    def prime(self, shots: Sequence[tuple], transform) -> None:
        """The fictitious volume before the series: each (time, slices) excites at `transform`."""
        times = np.ascontiguousarray([s[0] for s in shots] or [0.0], np.float64)
        offs = np.zeros(len(shots) + 1, np.int64)
        flat = []
        for i, s in enumerate(shots):
            flat.extend(int(z) for z in s[1])
            offs[i + 1] = len(flat)
        sl = np.ascontiguousarray(flat or [0], np.int64)
        m = np.ascontiguousarray(transform, np.float64).reshape(16)
        P = C.POINTER(C.c_int64)
        check(lib().mrsim_spin_history_prime(self._h, times.ctypes.data_as(abi.c_f64p), sl.ctypes.data_as(P),
                                             offs.ctypes.data_as(P), len(shots), m.ctypes.data_as(abi.c_f64p)))

    def prepare(self, shots: Sequence[Shot]) -> PreparedShots:
        """The shots marshalled for `excite_many` / `excite_device` (callable references are
        evaluated here, once)."""
        return PreparedShots(shots, self._ref_values)

    def _arr(self, shots):
        if isinstance(shots, PreparedShots):
            return shots.arr, shots.shots
        keep: list = []
        arr = shots_c(shots, self._ref_values, keep)
        self._keep = keep
        return arr, shots

    def terms_size(self, shots) -> int:
        arr, _ = self._arr(shots)
        n = C.c_int64()
        check(lib().mrsim_spin_history_terms_size(self._h, arr, len(shots), C.byref(n)))
        return n.value

    def excite_many(self, shots) -> list:
        """The shots (a list of Shot or PreparedShots) in order, in one batch on the device; per
        shot its SliceTerms (None for a shot with no reference)."""
        arr, shots = self._arr(shots)
        n = C.c_int64()
        check(lib().mrsim_spin_history_terms_size(self._h, arr, len(shots), C.byref(n)))
        flat = np.zeros(max(n.value, 1), np.float32)
        check(lib().mrsim_spin_history_excite(self._h, arr, len(shots), flat.ctypes.data_as(abi.c_f32p)))
        return unpack_terms(shots, flat, self.n_classes, self.cells)

    def excite_device(self, shots, out_ptr: int) -> None:
        """The shots (a list of Shot or PreparedShots) in order with the packed terms written to
        device memory at `out_ptr` (queued on the context's stream)."""
        arr, shots = self._arr(shots)
        check(lib().mrsim_spin_history_excite_device(self._h, arr, len(shots), C.c_void_p(out_ptr)))

    def excite(self, t: float, transform, slices: Sequence[int], mz_ref: MzRef,
               weight: Optional[np.ndarray] = None) -> list:
        """One shot: the terms of each of `slices` against `mz_ref(T1)`, then the excitation."""
        if mz_ref is None:
            raise ValueError("excite reads terms: give a reference magnetisation")
        return self.excite_many([Shot(t, transform, slices, mz_ref, weight)])[0]

    def merges(self) -> int:
        m = C.c_uint64()
        check(lib().mrsim_spin_history_merges(self._h, C.byref(m)))
        return m.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().mrsim_spin_history_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
