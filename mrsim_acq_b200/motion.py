"""Rigid image motion before the k-space forward (reference `motion.rs`), on the device.

Mirrors the reference's names: `Pose` (motion.rs:43-91), `resample_by_pose` (motion.rs:430),
`apply_motion` (motion.rs:466), `slice_schedule` (motion.rs:486), `DropoutLaw` (motion.rs:625),
`MotionEvent` / `DroppedShot` (motion.rs:608-624) and `apply_multiband_motion(_slab)`
(motion.rs:666-772).  Images use the reference's series layout, one array per compartment with
`vox * n_volumes + g`; `v2w` is the grid's 4x4 voxel-to-world affine."""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional, Sequence

import numpy as np

from . import abi
from .abi import check, lib
from .api import Context, default_context


@dataclasses.dataclass(frozen=True)
class Pose:
    """A rigid pose: rotation in degrees about x, y, z (R = Rz Ry Rx) and translation in mm."""

    rot_deg: tuple = (0.0, 0.0, 0.0)
    trans_mm: tuple = (0.0, 0.0, 0.0)

    def as_array(self) -> np.ndarray:
        return np.array(list(self.rot_deg) + list(self.trans_mm), np.float64)

    def to_matrix(self, center) -> np.ndarray:
        """The world-space 4x4 transform of the pose about `center` (`Pose::to_matrix`
        motion.rs:55-68): R = Rz Ry Rx, translation c - R c + t, so `center` maps to center + t."""
        rx, ry, rz = (np.deg2rad(a) for a in self.rot_deg)
        X = np.array([[1.0, 0.0, 0.0], [0.0, np.cos(rx), -np.sin(rx)], [0.0, np.sin(rx), np.cos(rx)]])
        Y = np.array([[np.cos(ry), 0.0, np.sin(ry)], [0.0, 1.0, 0.0], [-np.sin(ry), 0.0, np.cos(ry)]])
        Z = np.array([[np.cos(rz), -np.sin(rz), 0.0], [np.sin(rz), np.cos(rz), 0.0], [0.0, 0.0, 1.0]])
        R = Z @ (Y @ X)
        c = np.asarray(center, np.float64)
        m = np.eye(4)
        m[:3, :3] = R
        m[:3, 3] = c - R @ c + np.asarray(self.trans_mm, np.float64)
        return m


IDENTITY = Pose()


@dataclasses.dataclass
class DropoutLaw:
    """`DropoutLaw`: kind "uniform" (1 - severity), "scaled" (1 - severity drive/max(drive),
    drive < floor exempt) or "scaled_to" (the same with the given max)."""

    kind: str = "uniform"
    drive: Sequence[float] = ()
    floor: float = 0.0
    max: float = 0.0

    def to_c(self, keep: list) -> abi.DropoutLaw_:
        d = np.ascontiguousarray(self.drive, np.float64)
        keep.append(d)
        kinds = {"uniform": 0, "scaled": 1, "scaled_to": 2}
        return abi.DropoutLaw_(kinds[self.kind], d.ctypes.data_as(abi.c_f64p) if d.size else None, d.size,
                               float(self.floor), float(self.max))


@dataclasses.dataclass
class MotionEvent:
    volume: int
    shot: int
    severity: float
    jump_mm: tuple = (0.0, 0.0, 0.0)
    jump_deg: tuple = (0.0, 0.0, 0.0)


@dataclasses.dataclass
class DroppedShot:
    volume: int
    shot: int
    slices: list
    attenuation: float


def _v2w(v2w) -> np.ndarray:
    a = np.ascontiguousarray(v2w, np.float64).reshape(16)
    return a


def resample_by_pose(src: np.ndarray, dims, v2w, pose: Pose, ctx: Optional[Context] = None) -> np.ndarray:
    ctx = ctx or default_context()
    s = np.ascontiguousarray(src, np.float32).ravel()
    out = np.zeros_like(s)
    d = np.ascontiguousarray(dims, np.int64)
    m, p = _v2w(v2w), pose.as_array()
    check(lib().mrsim_resample_by_pose(ctx.handle, s.ctypes.data_as(abi.c_f32p), d.ctypes.data_as(C.POINTER(C.c_int64)),
                                       m.ctypes.data_as(abi.c_f64p), p.ctypes.data_as(abi.c_f64p),
                                       out.ctypes.data_as(abi.c_f32p)))
    return out


def _ptrs(images):
    arr = (abi.c_f32p * len(images))()
    for i, a in enumerate(images):
        if a.dtype != np.float32 or not a.flags.c_contiguous:
            raise ValueError("images must be C-contiguous float32 arrays (moved in place)")
        arr[i] = a.ctypes.data_as(abi.c_f32p)
    return arr


def apply_motion(images: Sequence[np.ndarray], dims, n_volumes: int, v2w, poses: Sequence[Pose],
                 ctx: Optional[Context] = None) -> None:
    """Moves every volume g of every compartment by poses[g], in place."""
    ctx = ctx or default_context()
    d = np.ascontiguousarray(dims, np.int64)
    ps = np.concatenate([(poses[g] if g < len(poses) else IDENTITY).as_array() for g in range(n_volumes)])
    m = _v2w(v2w)
    check(lib().mrsim_apply_motion(ctx.handle, _ptrs(images), len(images), d.ctypes.data_as(C.POINTER(C.c_int64)),
                                   n_volumes, m.ctypes.data_as(abi.c_f64p), ps.ctypes.data_as(abi.c_f64p)))


def apply_multiband_motion(images: Sequence[np.ndarray], dims, n_volumes: int, v2w, mb: int, interleaved: bool,
                           law: DropoutLaw, events: Sequence[MotionEvent], slice_z=None, nz_full: int = 0,
                           ctx: Optional[Context] = None) -> list:
    """`apply_multiband_motion_slab` in place; returns the dropped shots."""
    ctx = ctx or default_context()
    keep = []
    d = np.ascontiguousarray(dims, np.int64)
    m = _v2w(v2w)
    ev = (abi.MotionEvent_ * max(len(events), 1))()
    for i, e in enumerate(events):
        ev[i] = abi.MotionEvent_(e.volume, e.shot, e.severity, (C.c_double * 3)(*e.jump_mm),
                                 (C.c_double * 3)(*e.jump_deg))
    sz = None
    if slice_z is not None:
        a = np.ascontiguousarray(slice_z, np.int64)
        keep.append(a)
        sz = a.ctypes.data_as(C.POINTER(C.c_int64))
    cap = max(len(events), 1)
    dropped = (abi.DroppedShot_ * cap)()
    n = C.c_int64()
    lw = law.to_c(keep)
    check(lib().mrsim_apply_multiband_motion(ctx.handle, _ptrs(images), len(images),
                                             d.ctypes.data_as(C.POINTER(C.c_int64)), n_volumes,
                                             m.ctypes.data_as(abi.c_f64p), mb, int(interleaved), C.byref(lw), ev,
                                             len(events), sz, nz_full, dropped, cap, C.byref(n)))
    return [DroppedShot(int(dropped[i].volume), int(dropped[i].shot),
                        [int(dropped[i].slices[k]) for k in range(dropped[i].n_slices)], float(dropped[i].attenuation))
            for i in range(n.value)]


def operator_apply_motion(op, v2w, poses: Sequence[Pose]) -> None:
    """`apply_motion` on an `EpiOperator`'s device images (its slab of slices), in place."""
    ps = np.concatenate([(poses[g] if g < len(poses) else IDENTITY).as_array() for g in range(op.n_volumes)])
    m = _v2w(v2w)
    check(lib().mrsim_epi_operator_apply_motion(op.handle, m.ctypes.data_as(abi.c_f64p), ps.ctypes.data_as(abi.c_f64p)))
