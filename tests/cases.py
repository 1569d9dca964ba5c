"""Seeded inputs shared by the tests: the reference's golden-record cases (tests/golden_baseline.rs
of the reference crate) regenerated in numpy with the reference's SplitMix64 stream, and small
series for the operator tests."""
from __future__ import annotations

import math

import numpy as np

from mrsim_acq_b200.api import Acquisition, EchoFormation, PartialFourierMode, SliceInput, T2

TAU = 2.0 * math.pi
M64 = (1 << 64) - 1


class Rng:
    """`Rng` (kspace.rs:59-77): SplitMix64 + Box-Muller, in Python integers."""

    def __init__(self, seed):
        self.s = seed & M64

    def next_u64(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & M64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)

    def unit(self):
        return ((self.next_u64() >> 11) + 0.5) / float(1 << 53)


GEOMETRIES = [(17, 70, 2), (16, 40, 1), (8, 9, 3)]


def golden_geometry_inputs(rng, nx, ny, o):
    """The per-geometry inputs of golden_baseline.rs:33-50 (consumes `rng` in the same order)."""
    snx, sny = nx * o, ny * o
    n = snx * sny
    i = np.arange(n)
    x = (i % snx) / snx
    y = (i // snx) / sny
    comps = []
    for c in range(3):
        blob = np.exp(-(((x - 0.5) * (x - 0.5) + (y - 0.45) * (y - 0.45)) / (0.03 * (c + 1))))
        u = np.array([rng.unit() for _ in range(n)])
        comps.append((blob + 0.05 * u).astype(np.float32))
    u = np.array([rng.unit() for _ in range(n)])
    fmap = (300.0 * (np.sin(3.0 * x) * np.cos(2.0 * y + 1.0)) + 20.0 * u).astype(np.float32)
    phase0 = np.array([TAU * rng.unit() for _ in range(n)])
    t2map = (60.0 + 80.0 * ((i % snx) / snx)).astype(np.float32)
    timap = (30.0 + 40.0 * ((i // snx) / sny)).astype(np.float32)
    return comps, fmap, phase0, t2map, timap


def golden_cases():
    """(name, SliceInput, Acquisition) for the 39 per-slice golden cases, in record order."""
    full = Acquisition(do_distortions=True, do_relaxation=True, signal_scale=100.0)
    rng = Rng(0xC0FFEE)
    out = []
    for nx, ny, o in GEOMETRIES:
        comps, fmap, phase0, t2map, timap = golden_geometry_inputs(rng, nx, ny, o)
        uniform = [T2.uniform(70.0), T2.uniform(100.0), T2.uniform(2000.0)]
        mapped = [T2.of_map(t2map), T2.uniform(100.0), T2.of_map(t2map)]
        ti_mapped = [T2.of_map(timap), T2.uniform(45.0), T2.of_map(timap)]
        cases = [
            ("clean", full.replace(do_distortions=False, do_relaxation=False), None, False),
            ("distortion+relaxation", full, None, False),
            ("reverse", full.replace(reverse_phase=True), None, False),
            ("ghost", full.replace(ghost_offset=0.015), None, False),
            ("eddy-poly", full.replace(eddy_strength=3.0, eddy_quad=0.4, eddy_tau=70.0), (0.3, -0.8, 0.5), False),
            ("eddy-phase", full.replace(eddy_phase=0.2), (0.6, 0.6, 0.5), False),
            ("pf-fiberfox", full.replace(partial_fourier=0.75), None, False),
            ("pf-contiguous-reverse", full.replace(partial_fourier=0.75, pf_mode=PartialFourierMode.Contiguous,
                                                   reverse_phase=True), None, False),
            ("grappa-coils", full.replace(accel=2, acs_lines=6, n_coils=4), None, False),
            ("grappa3", full.replace(accel=3, acs_lines=8, n_coils=4), None, False),
            ("everything", full.replace(ghost_offset=0.02, eddy_strength=2.0, eddy_quad=0.3, eddy_phase=0.1,
                                        partial_fourier=0.8, accel=2, acs_lines=8, n_coils=3), (0.5, 0.5, 0.7), False),
            ("maps", full, None, True),
            ("maps-coils-noise", full.replace(n_coils=3, noise_variance=4.0), None, True),
        ]
        for name, acq, eddy, maps in cases:
            inp = SliceInput(compartments=comps, t2=mapped if maps else uniform, fmap=fmap, sim=(nx * o, ny * o),
                             acq_matrix=(nx, ny), t_inhom=ti_mapped if maps else None, phase0=phase0, z=3, nz=9,
                             eddy_drive=eddy, slice_seed=7)
            out.append((f"slice-{nx}x{ny}o{o}-{name}", inp, acq))
    return out


def literal_sum_cases():
    """The 17 cases x 3 geometries of `restructured_forward_matches_the_literal_sum`
    (kspace.rs:3362-3433): (name, SliceInput, Acquisition, coil, ncoils)."""
    full = Acquisition(do_distortions=True, do_relaxation=True, signal_scale=100.0)
    rng = Rng(0xC0FFEE)
    out = []
    for nx, ny, o in GEOMETRIES:
        comps, fmap, phase0, _, _ = golden_geometry_inputs(rng, nx, ny, o)
        t2 = [T2.uniform(70.0), T2.uniform(100.0), T2.uniform(2000.0)]
        G = EchoFormation.Gradient
        cases = [
            ("clean", full.replace(do_distortions=False, do_relaxation=False), None, 0, 1),
            ("distortion+relaxation", full, None, 0, 1),
            ("reverse", full.replace(reverse_phase=True), None, 0, 1),
            ("ghost", full.replace(ghost_offset=0.015), None, 0, 1),
            ("eddy-poly", full.replace(eddy_strength=3.0, eddy_quad=0.4, eddy_tau=70.0), (0.3, -0.8, 0.5), 0, 1),
            ("eddy-phase", full.replace(eddy_phase=0.2), (0.6, 0.6, 0.5), 0, 1),
            ("pf-fiberfox", full.replace(partial_fourier=0.75), None, 0, 1),
            ("pf-scanner-eddy", full.replace(partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner,
                                             eddy_strength=3.0, eddy_quad=0.4, eddy_phase=0.1), (0.3, -0.8, 0.5), 0, 1),
            ("pf-scanner-reverse-grappa", full.replace(partial_fourier=0.8, pf_mode=PartialFourierMode.Scanner,
                                                       reverse_phase=True, eddy_strength=2.0, accel=2, acs_lines=8,
                                                       n_coils=3), (0.5, 0.5, 0.7), 1, 3),
            ("pf-contiguous-reverse", full.replace(partial_fourier=0.75, pf_mode=PartialFourierMode.Contiguous,
                                                   reverse_phase=True), None, 0, 1),
            ("grappa-coils", full.replace(accel=2, acs_lines=6, n_coils=4), None, 2, 4),
            ("grappa3", full.replace(accel=3, acs_lines=8, n_coils=4), None, 1, 4),
            ("everything", full.replace(ghost_offset=0.02, eddy_strength=2.0, eddy_quad=0.3, eddy_phase=0.1,
                                        partial_fourier=0.8, accel=2, acs_lines=8, n_coils=3), (0.5, 0.5, 0.7), 0, 3),
            ("ge-clean", full.replace(echo=G, do_distortions=False, do_relaxation=False), None, 0, 1),
            ("ge-distortion+relaxation", full.replace(echo=G), None, 0, 1),
            ("ge-everything", full.replace(echo=G, ghost_offset=0.02, eddy_strength=2.0, eddy_quad=0.3, eddy_phase=0.1,
                                           partial_fourier=0.8, accel=2, acs_lines=8, n_coils=3, reverse_phase=True),
             (0.5, 0.5, 0.7), 0, 3),
        ]
        for name, acq, eddy, coil, ncoils in cases:
            inp = SliceInput(compartments=comps, t2=t2, fmap=fmap, sim=(nx * o, ny * o), acq_matrix=(nx, ny),
                             phase0=phase0, z=3, nz=9, eddy_drive=eddy, slice_seed=0)
            out.append((f"{nx}x{ny}o{o}-{name}", inp, acq, coil, ncoils))
    return out


def box_hires(snx, sny, x0, x1, y0, y1):
    """`box_hires` (kspace.rs:498-516)."""
    v = np.zeros(snx * sny, np.float32)
    for y in range(sny):
        fy = min(max(min(y + 1.0, y1) - max(float(y), y0), 0.0), 1.0)
        if fy <= 0.0:
            continue
        for x in range(snx):
            fx = min(max(min(x + 1.0, x1) - max(float(x), x0), 0.0), 1.0)
            v[x + snx * y] = np.float32(fx * fy)
    return v


def series_case(nx=16, ny=16, nz=2, o=2, nv=2, ncomp=3, seed=5, maps=False):
    """A small seeded series: blob images, a smooth fieldmap, uniform or mapped T2."""
    snx, sny = nx * o, ny * o
    nsim = snx * sny * nz
    rng = np.random.default_rng(seed)
    vox = np.arange(nsim)
    x = (vox % snx) / snx
    y = ((vox // snx) % sny) / sny
    z = vox // (snx * sny)
    imgs = []
    for c in range(ncomp):
        base = np.exp(-(((x - 0.5) ** 2 + (y - 0.48) ** 2) / (0.04 * (c + 1)))) * (1.0 + 0.05 * z)
        per_vol = [base * (1.0 + 0.02 * g) + 0.02 * rng.random(nsim) for g in range(nv)]
        arr = np.stack(per_vol, axis=1).astype(np.float32)  # vox*nv + g
        imgs.append(arr.ravel())
    fmap = (60.0 * np.sin(2.0 * np.pi * x) * np.cos(np.pi * y) + 5.0 * z).astype(np.float32)
    t2 = [T2.uniform(80.0), T2.uniform(250.0), T2.uniform(30.0)][:ncomp]
    ti = [T2.uniform(40.0), T2.uniform(60.0), T2.uniform(20.0)][:ncomp]
    if maps:
        t2 = [T2.of_map((60.0 + 40.0 * x).astype(np.float32))] + t2[1:]
    return dict(sim_dims=(snx, sny, nz), acq_dims=(nx, ny, nz), n_volumes=nv, images=imgs, t2=t2, t_inhom=ti,
                fmap=fmap)


def golden_series_inputs():
    """The series cases of golden_baseline.rs:90-124: (name, AcquisitionInput, Acquisition)."""
    from mrsim_acq_b200.api import AcquisitionInput, PhaseModel
    nx, ny, nz, o, nv = 16, 16, 3, 2, 4
    snx, sny = nx * o, ny * o
    nsim = snx * sny * nz
    rng = Rng(0xBA5E)
    images = []
    for c in range(2):
        i = np.arange(nsim * nv)
        v = i // nsim
        vox = i % nsim
        x = (vox % snx) / snx
        y = ((vox // snx) % sny) / sny
        blob = np.exp(-(((x - 0.5) * (x - 0.5) + (y - 0.5) * (y - 0.5)) / 0.05))
        u = np.array([rng.unit() for _ in range(nsim * nv)])
        by_volume = ((1.0 + 0.1 * c + 0.01 * v) * blob + 0.02 * u).astype(np.float32)
        images.append(np.ascontiguousarray(by_volume.reshape(nv, nsim).T).reshape(-1))  # vox*nv + g
    idx = np.arange(nsim)
    fmap = (40.0 * ((idx % snx) / snx - 0.5)).astype(np.float32)
    t2map = (50.0 + (idx % 7) * 10.0).astype(np.float32)
    acq = Acquisition(n_coils=3, accel=2, acs_lines=6, noise_variance=2.0, signal_scale=100.0, t_echo=30.0, t_line=0.5)
    out = []
    for name, t2 in (("series-uniform", [T2.uniform(80.0), T2.uniform(160.0)]),
                     ("series-mapped", [T2.of_map(t2map), T2.uniform(160.0)])):
        inp = AcquisitionInput(sim_dims=(snx, sny, nz), acq_dims=(nx, ny, nz), n_volumes=nv, images=images, t2=t2,
                               fmap=fmap, phase=PhaseModel.hbcd_like(), seed=42)
        out.append((name, inp, acq))
    return out
