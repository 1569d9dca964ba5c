"""Python mirror of the reference's stack-of-spirals pieces, over the C ABI.

`spiral_tau_c` / `spiral_trajectory` (readout.rs:564-620), `tseg.plan` (tseg.rs:230-289),
`epg_cpmg` (epg.rs:101-125), the 2D NUFFT pair `Nufft2` (nufft.rs:125-299), the spiral
forwards `spiral_kspace_exact` / `SegmentedForward` (spiral.rs:83-201) and the reconstruction
`SpiralRecon` (grid_recon.rs:54-325).  Host plans run in the
library's C++; the NUFFT pair and the forwards run on the device (no CPU path).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional, Sequence

import numpy as np

from . import abi
from .abi import check, lib
from .api import Acquisition, Context, KspaceWindow, SliceInput, _Keep, default_context, slice_input_c


def spiral_tau_c(nx: int, interleaves: int, readout_ms: float, dwell_ms: float, radial_oversampling: float) -> float:
    out = C.c_double()
    check(lib().mrsim_spiral_tau_c(nx, interleaves, readout_ms, dwell_ms, radial_oversampling, C.byref(out)))
    return out.value


@dataclasses.dataclass
class SpiralTrajectory:
    """`SpiralTrajectory` (readout.rs:463-560): k [interleaf, sample, 2] in cycles/FOV."""

    interleaves: int
    radial_oversampling: float
    readout_ms: float
    dwell_ms: float
    k_max: float
    n_turns: float
    tau_c_ms: float
    tau_ms: np.ndarray
    k: np.ndarray


def spiral_trajectory(nx: int, ny: int, interleaves: int, readout_ms: float, dwell_ms: float,
                      radial_oversampling: float) -> SpiralTrajectory:
    info = abi.SpiralInfo_()
    check(lib().mrsim_spiral_trajectory(nx, ny, interleaves, readout_ms, dwell_ms, radial_oversampling, 0, None, None,
                                        C.byref(info)))
    n = int(info.samples)
    k = np.zeros((interleaves, n, 2))
    tau = np.zeros(n)
    check(lib().mrsim_spiral_trajectory(nx, ny, interleaves, readout_ms, dwell_ms, radial_oversampling, n,
                                        k.ctypes.data_as(abi.c_f64p), tau.ctypes.data_as(abi.c_f64p), C.byref(info)))
    return SpiralTrajectory(interleaves, radial_oversampling, readout_ms, dwell_ms, info.k_max, info.n_turns,
                            info.tau_c_ms, tau, k)


@dataclasses.dataclass
class RateRect:
    """`RateRect` (tseg.rs:52-57): decay d (1/ms) and off-resonance f (Hz) intervals."""

    d: tuple
    f: tuple


@dataclasses.dataclass
class TsegPlan:
    """`TsegPlan` (tseg.rs:60-75): b [sample, segment] complex."""

    l: int
    m: int
    tau_l: np.ndarray
    b: np.ndarray
    b_sum: float
    grid_err: float
    bound: float


def _pair(v) -> np.ndarray:
    return np.ascontiguousarray([float(v[0]), float(v[1])], dtype=np.float64)


_TSEG_L_MAX = 64  # the planner refuses past 64 segments


def tseg_plan(tau: np.ndarray, t_ms: float, rect: RateRect, ctx: Optional[Context] = None) -> TsegPlan:
    """`tseg::plan`.  With `ctx` the fits' per-sample work runs on that context's device in FP64
    (the planner the device forwards use: the same L and m, b_sum and bound to ~1e-6); without it
    the whole plan runs on the host."""
    tau = np.ascontiguousarray(tau, dtype=np.float64)
    d, f = _pair(rect.d), _pair(rect.f)
    info = abi.TsegInfo_()
    tp = tau.ctypes.data_as(abi.c_f64p)
    if ctx is not None:
        tau_l = np.zeros(_TSEG_L_MAX)
        b = np.zeros(len(tau) * _TSEG_L_MAX * 2)
        check(lib().mrsim_tseg_plan_device(ctx.handle, tp, len(tau), t_ms, d.ctypes.data_as(abi.c_f64p),
                                           f.ctypes.data_as(abi.c_f64p), _TSEG_L_MAX, tau_l.ctypes.data_as(abi.c_f64p),
                                           b.ctypes.data_as(abi.c_f64p), C.byref(info)))
        L = int(info.l)
        return TsegPlan(L, int(info.m), tau_l[:L].copy(), b[:len(tau) * L * 2].view(np.complex128).reshape(len(tau), L),
                        info.b_sum, info.grid_err, info.bound)
    check(lib().mrsim_tseg_plan(tp, len(tau), t_ms, d.ctypes.data_as(abi.c_f64p), f.ctypes.data_as(abi.c_f64p), 0,
                                None, None, C.byref(info)))
    L = int(info.l)
    tau_l = np.zeros(L)
    b = np.zeros(len(tau) * L * 2)
    check(lib().mrsim_tseg_plan(tp, len(tau), t_ms, d.ctypes.data_as(abi.c_f64p), f.ctypes.data_as(abi.c_f64p), L,
                                tau_l.ctypes.data_as(abi.c_f64p), b.ctypes.data_as(abi.c_f64p), C.byref(info)))
    return TsegPlan(L, int(info.m), tau_l, b.view(np.complex128).reshape(len(tau), L), info.b_sum, info.grid_err,
                    info.bound)


def epg_cpmg(n_echoes: int, esp_ms: float, refocusing_deg: float, t1_ms: float, t2_ms: float) -> np.ndarray:
    out = np.zeros(max(n_echoes, 0))
    check(lib().mrsim_epg_cpmg(n_echoes, esp_ms, refocusing_deg, t1_ms, t2_ms, out.ctypes.data_as(abi.c_f64p)))
    return out


def nufft_kernel_width(tol: float) -> int:
    return int(lib().mrsim_nufft_kernel_width(tol))


class Nufft1:
    """`Nufft1` (nufft.rs:25-112) on the device, FP64: period n, outputs at k_lo .. k_lo + n_out."""

    def __init__(self, n: int, k_lo: int, n_out: int, tol: float, ctx: Optional[Context] = None):
        self.n, self.k_lo, self.n_out, self.tol = int(n), int(k_lo), int(n_out), float(tol)
        self.ctx = ctx or default_context()

    def kernel_width(self) -> int:
        return nufft_kernel_width(self.tol)

    def run(self, pos: np.ndarray, weights: Sequence[np.ndarray]) -> np.ndarray:
        """`run`: weights = complex vectors sharing `pos`; returns complex128 [len(weights), n_out]."""
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.complex128).reshape(-1, len(pos)))
        out = np.zeros((len(w), self.n_out), np.complex128)
        check(lib().mrsim_nufft1(self.ctx.handle, self.n, self.k_lo, self.n_out, self.tol,
                                 pos.ctypes.data_as(abi.c_f64p), len(pos), w.view(np.float64).ctypes.data_as(abi.c_f64p),
                                 len(w), out.view(np.float64).ctypes.data_as(abi.c_f64p)))
        return out


class Nufft2:
    """`Nufft2` (nufft.rs:125-299): periods n, modes m_lo .. m_lo + m_out per axis.  Modes are
    complex arrays [m_out1, m_out0] (layout (m0 - m_lo0) + m_out0 (m1 - m_lo1)); points u [npts, 2]."""

    def __init__(self, n: Sequence[int], m_lo: Sequence[int], m_out: Sequence[int], tol: float,
                 ctx: Optional[Context] = None):
        self.n = np.ascontiguousarray(n, dtype=np.int64)
        self.m_lo = np.ascontiguousarray(m_lo, dtype=np.int64)
        self.m_out = np.ascontiguousarray(m_out, dtype=np.int64)
        self.tol = float(tol)
        self.ctx = ctx or default_context()

    def kernel_width(self) -> int:
        return nufft_kernel_width(self.tol)

    def _geom(self):
        P = C.POINTER(C.c_int64)
        return self.n.ctypes.data_as(P), self.m_lo.ctypes.data_as(P), self.m_out.ctypes.data_as(P)

    def type1(self, u: np.ndarray, wts: np.ndarray, sign: int) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 2)
        w = np.ascontiguousarray(np.asarray(wts, dtype=np.complex64).ravel())
        out = np.zeros(int(self.m_out[0] * self.m_out[1]), np.complex64)
        check(lib().mrsim_nufft2_type1(self.ctx.handle, *self._geom(), self.tol, u.ctypes.data_as(abi.c_f64p), len(u),
                                       w.view(np.float32).ctypes.data_as(abi.c_f32p), int(sign),
                                       out.view(np.float32).ctypes.data_as(abi.c_f32p)))
        return out.reshape(int(self.m_out[1]), int(self.m_out[0]))

    def type2(self, c: np.ndarray, u: np.ndarray, sign: int) -> np.ndarray:
        u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 2)
        c = np.ascontiguousarray(np.asarray(c, dtype=np.complex64).ravel())
        if c.size != int(self.m_out[0] * self.m_out[1]):
            raise ValueError("mode array does not match m_out")
        out = np.zeros(len(u), np.complex64)
        check(lib().mrsim_nufft2_type2(self.ctx.handle, *self._geom(), self.tol,
                                       c.view(np.float32).ctypes.data_as(abi.c_f32p), u.ctypes.data_as(abi.c_f64p),
                                       len(u), int(sign), out.view(np.float32).ctypes.data_as(abi.c_f32p)))
        return out


def spiral_kspace_exact(inp: SliceInput, acq: Acquisition, coil: int, ncoils: int, k: np.ndarray, tau_ms: np.ndarray,
                        log_amp: Optional[np.ndarray] = None, ctx: Optional[Context] = None) -> np.ndarray:
    """`spiral_kspace_exact` (spiral.rs:107-137) on the device: complex64 [npts]."""
    ctx = ctx or default_context()
    keep = _Keep()
    s = slice_input_c(inp, keep)
    k = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 2)
    tau = np.ascontiguousarray(tau_ms, dtype=np.float64)
    if len(tau) != len(k):
        raise ValueError("one time per sample")
    la = keep.f64(np.ravel(log_amp)) if log_amp is not None else None
    out = np.zeros(len(k), np.complex64)
    check(lib().mrsim_spiral_kspace_exact(ctx.handle, C.byref(s), C.byref(acq.to_c()), coil, ncoils,
                                          k.ctypes.data_as(abi.c_f64p), tau.ctypes.data_as(abi.c_f64p), len(k), la,
                                          out.view(np.float32).ctypes.data_as(abi.c_f32p)))
    return out


def spiral_segmented_forward(inp: SliceInput, acq: Acquisition, coil: int, ncoils: int, k: np.ndarray,
                             tau_idx: np.ndarray, tau_ms: np.ndarray, t_ms: float, rect: RateRect,
                             log_amp: Optional[np.ndarray] = None, decay_inside: bool = True,
                             ctx: Optional[Context] = None):
    """`SegmentedForward::new(...).apply(segment_inputs(...))` (spiral.rs:83-201) on the device.
    Returns (complex64 [npts], info dict of the plan)."""
    ctx = ctx or default_context()
    keep = _Keep()
    s = slice_input_c(inp, keep)
    k = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 2)
    ti = np.ascontiguousarray(tau_idx, dtype=np.int64)
    tau = np.ascontiguousarray(tau_ms, dtype=np.float64)
    d, f = _pair(rect.d), _pair(rect.f)
    la = keep.f64(np.ravel(log_amp)) if log_amp is not None else None
    out = np.zeros(len(k), np.complex64)
    info = abi.TsegInfo_()
    check(lib().mrsim_spiral_segmented_forward(ctx.handle, C.byref(s), C.byref(acq.to_c()), coil, ncoils,
                                               k.ctypes.data_as(abi.c_f64p), ti.ctypes.data_as(C.POINTER(C.c_int64)),
                                               len(k), tau.ctypes.data_as(abi.c_f64p), len(tau), t_ms,
                                               d.ctypes.data_as(abi.c_f64p), f.ctypes.data_as(abi.c_f64p), la,
                                               int(bool(decay_inside)),
                                               out.view(np.float32).ctypes.data_as(abi.c_f32p), C.byref(info)))
    return out, {"l": int(info.l), "m": int(info.m), "bound": info.bound, "b_sum": info.b_sum,
                 "grid_err": info.grid_err}


# ---- the reconstruction ----------------------------------------------------------------------------
LS_ITERATIONS = 80
LS_KAPPA = 100.0


def _c128(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128))


class SpiralRecon:
    """`SpiralRecon` (grid_recon.rs:54-325) on the device, FP64.  Images are complex128 [n, n]
    (layout x + n y)."""

    def __init__(self, k: np.ndarray, n: int, window: Optional[KspaceWindow] = None,
                 iterations: int = LS_ITERATIONS, kappa: float = LS_KAPPA, band_limited: bool = True,
                 ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.k = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 2)
        self.n = int(n)
        window = window or KspaceWindow.none()
        h = C.c_void_p()
        check(lib().mrsim_spiral_recon_create(self.ctx.handle, self.k.ctypes.data_as(abi.c_f64p), len(self.k), self.n,
                                              int(window.kind), float(window.a), float(window.b), int(iterations),
                                              float(kappa), int(bool(band_limited)), C.byref(h)))
        self.handle = h

    @classmethod
    def new(cls, k, n, window=None, ctx=None) -> "SpiralRecon":
        return cls(k, n, window, ctx=ctx)

    @property
    def npts(self) -> int:
        return len(self.k)

    def _info(self):
        lam, its = C.c_double(), C.c_int64()
        w = np.zeros(self.npts)
        check(lib().mrsim_spiral_recon_info(self.handle, C.byref(lam), C.byref(its), w.ctypes.data_as(abi.c_f64p)))
        return lam.value, its.value, w

    @property
    def lambda_hi(self) -> float:
        return self._info()[0]

    @property
    def power_iterations(self) -> int:
        return self._info()[1]

    def weights(self) -> np.ndarray:
        return self._info()[2]

    def _run(self, fn, d, batch_shape):
        d = _c128(d)
        batch = d.size // self.npts
        if d.size != batch * self.npts or batch == 0:
            raise ValueError("one value per sample")
        out = np.zeros(batch * self.n * self.n, np.complex128)
        check(fn(self.handle, d.view(np.float64).ctypes.data_as(abi.c_f64p), batch,
                 out.view(np.float64).ctypes.data_as(abi.c_f64p)))
        return out.reshape(batch_shape + (self.n, self.n))

    def gridding(self, d) -> np.ndarray:
        d = _c128(d)
        return self._run(lib().mrsim_spiral_recon_gridding, d, d.shape[:-1])

    def image(self, d) -> np.ndarray:
        d = _c128(d)
        return self._run(lib().mrsim_spiral_recon_image, d, d.shape[:-1])

    def reconstruct_rings(self, coil_samples, ring: int, zsens) -> np.ndarray:
        """coil_samples [(partition,) coil, npts]; zsens [(partition,) coil] -> [(partition,) n, n]."""
        cs = _c128(coil_samples)
        single = cs.ndim == 2
        if single:
            cs = cs[None]
        zs = np.ascontiguousarray(np.asarray(zsens, dtype=np.float64).reshape(cs.shape[0], cs.shape[1]))
        out = np.zeros(cs.shape[0] * self.n * self.n, np.complex128)
        check(lib().mrsim_spiral_recon_rings(self.handle, cs.view(np.float64).ctypes.data_as(abi.c_f64p), cs.shape[0],
                                             cs.shape[1], int(ring), zs.ctypes.data_as(abi.c_f64p),
                                             out.view(np.float64).ctypes.data_as(abi.c_f64p)))
        out = out.reshape(cs.shape[0], self.n, self.n)
        return out[0] if single else out

    def reconstruct(self, coil_samples, acq: Acquisition) -> np.ndarray:
        nc = max(int(acq.n_coils), 1)
        cs = _c128(coil_samples)
        if cs.shape[-2] != nc:
            raise ValueError("one sample set per coil")
        return self.reconstruct_rings(cs, nc, np.ones(cs.shape[:-1]))

    def close(self):
        if getattr(self, "handle", None):
            lib().mrsim_spiral_recon_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
