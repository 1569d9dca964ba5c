"""Writing the series (reference `io.rs`): NIfTI-1 volumes with the grid's voxel-to-world affine,
the BIDS part-mag / part-phase pair with sidecars, and the simulation grid (`hires_grid`).
Host code: no device needed."""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional

import numpy as np

from . import abi
from .abi import check, lib


def _i64(a):
    a = np.ascontiguousarray(a, np.int64)
    return a, a.ctypes.data_as(C.POINTER(C.c_int64))


def _v2w(v2w):
    return np.ascontiguousarray(v2w, np.float64).reshape(16)


def write_4d(path: str, dims, nt: int, data: np.ndarray, v2w, tr_s: Optional[float] = None) -> None:
    """`write_4d_timed` io.rs:135-146: data in (x + nx (y + ny z)) nt + t order."""
    d, dp = _i64(dims)
    x = np.ascontiguousarray(data, np.float32).ravel()
    m = _v2w(v2w)
    check(lib().mrsim_write_nifti_4d(str(path).encode(), dp, nt, x.ctypes.data_as(abi.c_f32p),
                                     m.ctypes.data_as(abi.c_f64p), float(tr_s) if tr_s else 0.0))


def write_3d(path: str, dims, data: np.ndarray, v2w) -> None:
    """`write_3d` io.rs:149-156."""
    d, dp = _i64(dims)
    x = np.ascontiguousarray(data, np.float32).ravel()
    m = _v2w(v2w)
    check(lib().mrsim_write_nifti_3d(str(path).encode(), dp, x.ctypes.data_as(abi.c_f32p), m.ctypes.data_as(abi.c_f64p)))


def hires_grid(v2w, dims, o: int):
    """`hires_grid` io.rs:104-124: (v2w 4x4, dims) of the grid refined in-plane by o."""
    d, dp = _i64(dims)
    m = _v2w(v2w)
    out = np.zeros(16)
    od, odp = _i64([0, 0, 0])
    check(lib().mrsim_hires_grid(m.ctypes.data_as(abi.c_f64p), dp, int(o), out.ctypes.data_as(abi.c_f64p), odp))
    return out.reshape(4, 4), [int(v) for v in od]


@dataclasses.dataclass
class SidecarInfo:
    """`SidecarInfo` io.rs:162-184."""

    manufacturer: str
    phase_encoding_direction: str
    total_readout_time: float
    echo_time: float
    partial_fourier: float
    accel: int
    mb: int
    repetition_time_s: Optional[float] = None
    b0_field_source: Optional[str] = None

    def to_c(self) -> abi.SidecarInfo_:
        return abi.SidecarInfo_(self.manufacturer.encode(), self.phase_encoding_direction.encode(),
                                self.total_readout_time, self.echo_time, self.partial_fourier, self.accel, self.mb,
                                int(self.repetition_time_s is not None), self.repetition_time_s or 0.0,
                                self.b0_field_source.encode() if self.b0_field_source is not None else None)


def write_complex_4d(out_prefix: str, suffix: str, dims, n_volumes: int, mag: np.ndarray, phase: np.ndarray, v2w,
                     info: SidecarInfo) -> None:
    """`write_complex_4d` io.rs:186-228."""
    d, dp = _i64(dims)
    a = np.ascontiguousarray(mag, np.float32).ravel()
    p = np.ascontiguousarray(phase, np.float32).ravel()
    m = _v2w(v2w)
    ci = info.to_c()
    check(lib().mrsim_write_complex_4d(str(out_prefix).encode(), suffix.encode(), dp, n_volumes,
                                       a.ctypes.data_as(abi.c_f32p), p.ctypes.data_as(abi.c_f32p),
                                       m.ctypes.data_as(abi.c_f64p), C.byref(ci)))
