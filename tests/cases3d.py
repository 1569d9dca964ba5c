"""Seeded inputs of the 3D echo-train tests: the reference's `blobs` phantom (kspace3d.rs tests),
echo trains and readouts."""
from __future__ import annotations

import math

import numpy as np

from mrsim_acq_b200.kspace3d import EchoTrain, GraseReadout, KzOrder

TAU = 2.0 * math.pi


def blobs(snx, sny, nz, nv, ncomp):
    """kspace3d.rs `blobs`: a smooth blob per compartment, varying across volumes and slices, in the
    entry points' vox * n_volumes + g layout."""
    nvox = snx * sny * nz
    vox = np.arange(nvox)
    x, y, z = vox % snx, (vox // snx) % sny, vox // (snx * sny)
    fx, fy, fz = x / snx, y / sny, z / nz
    out = []
    for c in range(ncomp):
        b = np.exp(-((fx - 0.5 - 0.05 * c) ** 2 + (fy - 0.45) ** 2) / 0.04) * (1.0 + 0.5 * np.sin(TAU * fz))
        v = np.zeros(nvox * nv, np.float32)
        for g in range(nv):
            v[g::nv] = ((1.0 + 0.1 * g) * b).astype(np.float32)
        out.append(v)
    return out


def train(nz, kz_segments, order=KzOrder.Centric, esp_ms=20.0, b=180.0):
    return EchoTrain(etl=nz // kz_segments, esp_ms=esp_ms, refocusing_deg=b, kz_order=order, kz_segments=kz_segments,
                     refocusing_time_ms=2.0)


def grase(ky_segments, t_line_ms=0.5, reverse_phase=False):
    return GraseReadout(ky_segments=ky_segments, t_line_ms=t_line_ms, reverse_phase=reverse_phase)
