"""Benchmark of the exact-DFT k-space forward + adjoint on B200 (one JSON line on rank 0).

Workload: the batched 2D EPI series — scan 64x64 on a 128x128 sim grid, 30 slices, 40 volumes
with seeded rigid motion, 3 compartments (T2 80/250/30 ms, T2' 40/60/20 ms), 8 ring coils,
GRAPPA R=2 sampling, partial Fourier 6/8 (Scanner), ghost 0.05, echoes TE 15/35/55 ms.
Synthetic seeded data of that shape (no dataset exists for it).  A step is one forward over
every (volume, slice, echo, coil) plus one adjoint/VJP (complex images, fieldmap and R2
gradients) of the k-space it produced.  Metric: acquired k-space samples per second.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the reference's CPU algorithm (the FP64 C++ restatement in oracle/, the
reference crate being Rust and unbuildable here) on the host cores, on a bounded sample of the
same workload.  Under torchrun each rank runs its own copy of the series (weak scaling, no
collective on the data path); rank 0 prints the max-over-ranks timing.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "exact-DFT k-space samples/s (fwd+adjoint)"
WORKLOAD = dict(name="epi-series-64x64-sim128-z30-v40-c3-q8-r2-pf0.75-te3", nx=64, ny=64, o=2, nz=30, nv=40,
                ncomp=3, n_coils=8, echoes=(15.0, 35.0, 55.0))


def make_acquisition():
    from mrsim_acq_b200.api import Acquisition, KspaceWindow, PartialFourierMode
    return Acquisition(n_coils=WORKLOAD["n_coils"], accel=2, acs_lines=24, partial_fourier=0.75,
                       pf_mode=PartialFourierMode.Scanner, t_line=0.5, t_echo=30.0, ghost_offset=0.05,
                       window=KspaceWindow.hann(), signal_scale=100.0)


def make_inputs(seed=1, z0=0, z1=None):
    """Seeded synthetic series: a 10-ellipse phantom split into 3 compartments, a per-volume
    rigid motion (rotation <= 2 deg, translation <= 2 mm at 3.4 mm voxels) evaluated analytically,
    and a fieldmap of 3 Gaussian blobs (+-60 Hz, sigma 8-20 px).  Layouts are the reference's.
    Slices [z0, z1) only (a rank's slab): the same values as those slices of the whole series."""
    from mrsim_acq_b200.api import T2
    W = WORKLOAD
    nx, ny, o, nz_full, nv, nc = W["nx"], W["ny"], W["o"], W["nz"], W["nv"], W["ncomp"]
    z1 = nz_full if z1 is None else z1
    nz = z1 - z0
    snx, sny = nx * o, ny * o
    rng = np.random.default_rng(seed)
    ell = []
    for k in range(10):
        ell.append(dict(cx=rng.uniform(0.3, 0.7), cy=rng.uniform(0.3, 0.7), a=rng.uniform(0.05, 0.25),
                        b=rng.uniform(0.05, 0.25), th=rng.uniform(0, np.pi), mag=rng.uniform(0.2, 1.0), comp=k % nc))
    ys, xs = np.meshgrid((np.arange(sny) + 0.5) / sny, (np.arange(snx) + 0.5) / snx, indexing="ij")
    images = np.zeros((nc, nz, sny, snx, nv), np.float32)
    vox_mm = 3.4
    for g in range(nv):
        rot = np.deg2rad(rng.uniform(-2, 2))
        tx, ty = rng.uniform(-2, 2, 2) / (vox_mm * nx)
        cr, sr = np.cos(rot), np.sin(rot)
        X = cr * (xs - 0.5) - sr * (ys - 0.5) + 0.5 - tx
        Y = sr * (xs - 0.5) + cr * (ys - 0.5) + 0.5 - ty
        for z in range(nz):
            zf = (z0 + z - nz_full / 2) / nz_full
            for e in ell:
                scale = math.sqrt(max(0.0, 1.0 - (zf / 0.6) ** 2))
                if scale <= 0:
                    continue
                c, s = np.cos(e["th"]), np.sin(e["th"])
                u = (c * (X - e["cx"]) + s * (Y - e["cy"])) / (e["a"] * scale)
                v = (-s * (X - e["cx"]) + c * (Y - e["cy"])) / (e["b"] * scale)
                images[e["comp"], z, :, :, g] += np.float32(e["mag"]) * (u * u + v * v <= 1.0)
    imgs = [np.ascontiguousarray(images[c]).reshape(-1) for c in range(nc)]  # vox*nv + g
    fmap = np.zeros((nz, sny, snx), np.float32)
    zz = np.arange(z0, z1)[:, None, None]
    for _ in range(3):
        amp, sig = rng.uniform(-60, 60), rng.uniform(8, 20) * o
        cx, cy, cz = rng.uniform(0.3, 0.7) * snx, rng.uniform(0.3, 0.7) * sny, rng.uniform(0.2, 0.8) * nz_full
        fmap += (amp * np.exp(-(((xs * snx - cx) ** 2 + (ys * sny - cy) ** 2) / (2 * sig * sig)
                                + (zz - cz) ** 2 / (2 * (nz_full / 3) ** 2)))).astype(np.float32)
    t2 = [T2.uniform(80.0), T2.uniform(250.0), T2.uniform(30.0)]
    ti = [T2.uniform(40.0), T2.uniform(60.0), T2.uniform(20.0)]
    return dict(sim_dims=(snx, sny, nz), acq_dims=(nx, ny, nz), n_volumes=nv, images=imgs, t2=t2, t_inhom=ti,
                fmap=fmap.reshape(-1))


class Clocks:
    """nvidia-smi clock and throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None
        # the samples go to a temporary file unless MRSIM_CLOCKS_DIR names a folder to keep them in
        keep = os.environ.get("MRSIM_CLOCKS_DIR")
        folder = keep if keep else tempfile.mkdtemp(prefix="mrsim_clocks_")
        self.path = os.path.join(folder, f"clocks_rank{device}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        self.p.wait()
        self.f.close()
        rows = [r.split(", ") for r in open(self.path).read().strip().splitlines() if r.strip()]
        sm = [float(r[1]) for r in rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows if len(r) > 8 for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# DRAM bytes per unit (one slice of one volume) of the two y-stage kernels, from one ncu capture of
# this workload at 24 volumes (720 units): dram__bytes.sum.per_second x gpu__time_duration.sum of
# yadjoint_q_kernel<6,4,3,0,1,1> (946.1 MB) and ystage_q_kernel<8,6,3,0> (463.5 MB).
# Traffic grows with the units processed (each unit reads and writes its own planes).
NCU_DRAM_BYTES_PER_UNIT = {"adjoint_ystage": 946.1e6 / 720, "forward_ystage": 463.5e6 / 720}


def algorithmic_flops(op_units, n_lines, snx, sny, nx, ncoils, ncomp):
    """Per launch over all units: the canonical per-(slice, volume, echo) work of the exact DFT,
    y-stage 4*Q*C*snx*sny*ny_acq and x-stage 8*Q*snx*nx*ny_acq, summed over echoes (n_lines is
    every echo's acquired lines of one unit)."""
    y = 4.0 * ncoils * ncomp * snx * sny * n_lines * op_units
    x = 8.0 * ncoils * snx * nx * n_lines * op_units
    return y, x


def max_over_ranks(v, world, device="cuda"):
    """The maximum of a per-rank scalar over every rank of the job (the value itself on one rank):
    step times are reported as the slowest rank's."""
    if world <= 1:
        return float(v)
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


STAGES = ["statics", "forward_ystage", "forward_xstage", "adjoint_xstage", "adjoint_ystage"]


def time_stages(op, stream, ctx, steps, warmup):
    """Device time of `steps` forward + adjoint passes (the five stages in order, CUDA events on the
    context stream): (total ms, per-stage mean ms)."""
    import torch

    def step(evs=None):
        for i in range(5):
            if evs is not None:
                evs[i].record(stream)
            op.stage(i)
        if evs is not None:
            evs[5].record(stream)

    for _ in range(warmup):
        step()
    ctx.synchronize()
    t_begin = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(6)] for _ in range(steps)]
    t_begin.record(stream)
    for k in range(steps):
        step(evs[k])
    t_end.record(stream)
    t_end.synchronize()
    ctx.synchronize()
    stage_ms = np.array([[evs[k][i].elapsed_time(evs[k][i + 1]) for i in range(5)] for k in range(steps)])
    return t_begin.elapsed_time(t_end), stage_ms.mean(axis=0)


def segmented_comparison(args, inp, acq, ctx, stream, samples):
    """The time-segmented tensor-core pair against the exact pair with the same outputs (k-space
    and the complex-image adjoint, grads = 0), on the same workload: samples/s, the ratio, the
    segmentation, and the forward contraction's tensor-pipe roofline."""
    from mrsim_acq_b200.api import EpiOperator, PhaseModel
    pk, pk_kind = peaks()
    tensor_peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))

    def make():
        return EpiOperator(inp["sim_dims"], inp["acq_dims"], inp["n_volumes"], inp["t2"], inp["fmap"], acq,
                           images=inp["images"], echo_times_ms=WORKLOAD["echoes"], t_inhom=inp["t_inhom"],
                           phase=PhaseModel.hbcd_like(), seed=42, grads=0, ctx=ctx)

    out = {}
    op = make()
    tot, st = time_stages(op, stream, ctx, args.steps, args.warmup)
    op.close()
    exact_ms = tot / args.steps
    out["exact_same_outputs"] = {"value": samples / (exact_ms * 1e-3), "ms_per_step": exact_ms,
                                 "stage_ms": dict(zip(STAGES, [round(float(v), 4) for v in st]))}
    for prec in ("f16", "bf16"):
        op = make()
        op.set_segmented(prec)
        info = op.segmentation()
        tot, st = time_stages(op, stream, ctx, args.steps, args.warmup)
        status = op.segmented_status()
        op.close()
        ms = tot / args.steps
        ach_f = info["flops_forward"] / (st[1] * 1e-3) / 1e12
        ach_a = info["flops_adjoint"] / (st[4] * 1e-3) / 1e12
        out[prec] = {"value": samples / (ms * 1e-3), "ms_per_step": ms, "ratio_to_exact": exact_ms / ms,
                     "status": status, "L": info["L"], "max_bound": max(info["bound"]) if info["bound"] else None,
                     "tensor_flop_per_pass": {"forward": info["flops_forward"], "adjoint": info["flops_adjoint"]},
                     "stage_ms": dict(zip(STAGES, [round(float(v), 4) for v in st])),
                     "roofline": {"bound": "tensor", "kernel": "ts_forward_kernel", "achieved": ach_f,
                                  "peak": tensor_peak, "unit": "TFLOP/s", "frac": ach_f / tensor_peak,
                                  "adjoint_achieved": ach_a, "adjoint_frac": ach_a / tensor_peak,
                                  "peak_source": f"bf16_tflops_sustained ({pk_kind})",
                                  "flop_count": "2 M N K per MMA, the three split products (hi*hi, lo*hi, hi*lo)"}}
    out["note"] = ("the same k-space and complex-image adjoint from both paths; ratio_to_exact > 1 means the "
                   "segmented pair is faster")
    return out


def scale_measurements(args, ctx, stream):
    """The larger configurations on one GPU, beside the headline workload: the precision-at-scale
    geometry (scan 128x128 on 256x256, 32 ring coils, 3 compartments, 60 slices x 20 volumes, all
    128 lines; the exact pair with the complex-image adjoint, device-timed) and one volume of the
    stack of spirals (64x64x48 on a 128x128 grid, 16 coils in 2 rings, 32 interleaves x 2048
    samples at 4 us, kz partial Fourier 6/8 and R = 2, +-80 Hz; the host-buffer call, transfers
    included); the precision-at-scale mixed batch (64/96/128 with 17/23/31 slices, one plan) and
    its GRASE train (64x64x32, 4 shots, 150-degree refocusing)."""
    from mrsim_acq_b200.api import T2, Acquisition, EpiOperator, PhaseModel
    out = {}
    nx, o, nz, nv, nc = 128, 2, 60, 20, 3
    snx = nx * o
    ys, xs = np.meshgrid((np.arange(snx) + 0.5) / snx, (np.arange(snx) + 0.5) / snx, indexing="ij")
    blob = np.exp(-((xs - 0.5) ** 2 + (ys - 0.48) ** 2) / 0.05).astype(np.float32)
    zs = 1.0 + 0.3 * np.sin(np.arange(nz) / 7.0)
    imgs = []
    for c in range(nc):
        vol = (blob[None, :, :] * (0.6 + 0.2 * c) * zs[:, None, None].astype(np.float32)).reshape(-1)
        imgs.append(np.repeat(vol, nv) * np.float32(1.0))  # vox * nv + g: volumes alike
    fmap = np.tile((60.0 * (blob - 0.5)).astype(np.float32).reshape(-1), nz)
    acq = Acquisition(n_coils=32, t_line=0.5, t_echo=40.0, ghost_offset=0.05, signal_scale=100.0)
    op = EpiOperator((snx, snx, nz), (nx, nx, nz), nv, [T2.uniform(80.0), T2.uniform(250.0), T2.uniform(30.0)],
                     fmap, acq, images=imgs, echo_times_ms=[40.0],
                     t_inhom=[T2.uniform(40.0), T2.uniform(60.0), T2.uniform(20.0)], phase=PhaseModel.hbcd_like(),
                     seed=42, grads=0, ctx=ctx)
    steps = 3
    tot, st = time_stages(op, stream, ctx, steps, 1)
    smp = op.samples
    op.close()
    out["precision_at_scale"] = {"config": "scan 128x128 on 256x256, 32 ring coils, 3 compartments, "
                                           "60 slices x 20 volumes, 128 lines, TE 40 ms",
                                 "samples_per_step": smp, "ms_per_step": tot / steps,
                                 "value": smp / (tot / steps * 1e-3), "unit": "samples/s",
                                 "stage_ms": dict(zip(STAGES, [round(float(v), 3) for v in st])),
                                 "note": "exact pair (per-coil kernels: a ring of 32 takes no coil-class path); "
                                         "the segmented path refuses this shape (more than 16 line groups)"}
    out["stack_of_spirals"] = spiral_measurement(ctx)
    out["mixed_batch"] = mixed_batch_measurement(ctx, stream)
    out["grase"] = grase_measurement(ctx)
    # the plain single-shot case on the device (launch-bound: one unit)
    c1, acq1 = c1_inputs()
    op = EpiOperator(c1["sim_dims"], c1["acq_dims"], 1, c1["t2"], c1["fmap"], acq1, images=c1["images"],
                     t_inhom=c1["t_inhom"], phase=PhaseModel.none(), seed=42, grads=0, ctx=ctx)
    tot, st = time_stages(op, stream, ctx, 20, 3)
    smp1 = op.samples
    op.close()
    out["plain_single_shot"] = {"config": "scan 64x64 on 128x128, 1 slice, 1 coil, 1 compartment, TE 30 ms",
                                "samples_per_step": smp1, "ms_per_step": tot / 20,
                                "value": smp1 / (tot / 20 * 1e-3), "unit": "samples/s",
                                "note": "one unit: five launches of a few microseconds each"}
    return out


def pipeline_measurement(ctx, inp, acq, cpu=True):
    """The whole reference pipeline of the benchmark series through its reference-compatible entry
    point (`simulate_acquisition_echoes`, kspace.rs:2152): per echo the exact forward, the receiver
    noise, GRAPPA R = 2 fitted on the echo's first volume, the Hann window, the inverse DFT and the
    Roemer combine, host buffers in and magnitude / phase out, by wall clock; beside it the FP64
    oracle's pipeline (`acquire_volumes_complex`) on one volume of one echo on the host cores."""
    from mrsim_acq_b200 import api
    from mrsim_acq_b200.api import AcquisitionInput, PhaseModel
    W = WORKLOAD
    a = acq.replace(noise_variance=1.56)  # image SNR about 40 at the phantom's mean magnitude
    ai = AcquisitionInput(inp["sim_dims"], inp["acq_dims"], inp["n_volumes"], inp["images"], inp["t2"], inp["fmap"],
                          t_inhom=inp["t_inhom"], phase=PhaseModel.hbcd_like(), seed=9)
    echoes = list(W["echoes"])
    per_echo = [inp["images"]] * len(echoes)
    api.simulate_acquisition_echoes(ai, per_echo, a, echoes, ctx=ctx)  # warm
    runs = []
    for _ in range(3):
        t0 = time.perf_counter()
        api.simulate_acquisition_echoes(ai, per_echo, a, echoes, ctx=ctx)
        runs.append(time.perf_counter() - t0)
    dt = float(np.median(runs))
    nx, ny, nz = inp["acq_dims"]
    nv = inp["n_volumes"]
    voxels = nx * ny * nz * nv * len(echoes)
    res = {"config": f"the benchmark series ({nv} volumes x {nz} slices x {len(echoes)} echoes, {W['n_coils']} coils, "
                     "3 compartments) with noise variance 1.56, GRAPPA R=2 from each echo's first volume, Hann "
                     "window, Roemer combine",
           "seconds_per_series": dt, "seconds_per_series_runs": [round(r, 4) for r in runs],
           "value": voxels / dt, "unit": "reconstructed voxels/s",
           "timing": "mrsim_simulate_acquisition_echoes with host buffers (pageable numpy arrays) by wall clock, the "
                     "median of 3 calls after a warm-up call (inputs up, magnitude and phase down)"}
    if cpu:
        import os
        from oracle import oracle
        snx, sny, _ = inp["sim_dims"]
        one = [im[0::nv].copy() for im in inp["images"]]
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        oracle.acquire_volumes_complex(inp["sim_dims"], inp["acq_dims"], 1, one, inp["t2"], inp["fmap"],
                                       a.replace(t_echo=echoes[0]), 9, 9, threads=threads, t_inhom=inp["t_inhom"],
                                       phase=PhaseModel.hbcd_like())
        ct = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": nx * ny * nz / ct, "unit": "reconstructed voxels/s", "cores": threads,
                               "kind": "port", "sample": f"1 volume x {nz} slices x 1 echo, FP64 oracle pipeline "
                                                         f"(GRAPPA fitted on that volume), {ct:.2f} s"}
        # the reference's `kspace` build on the same sample: NUFFT y-stage, FFT x-stage and inverse
        with oracle.kspace_build():
            t0 = time.perf_counter()
            oracle.acquire_volumes_complex(inp["sim_dims"], inp["acq_dims"], 1, one, inp["t2"], inp["fmap"],
                                           a.replace(t_echo=echoes[0]), 9, 9, threads=threads,
                                           t_inhom=inp["t_inhom"], phase=PhaseModel.hbcd_like())
            kt = time.perf_counter() - t0
        res["cpu_baseline_kspace_build"] = {"value": nx * ny * nz / kt, "unit": "reconstructed voxels/s",
                                            "cores": threads, "kind": "port",
                                            "sample": f"the same sample under the reference's `kspace` build "
                                                      f"(NUFFT y-stage, FFT x-stage and inverse), {kt:.2f} s"}
    return res


def spiral_measurement(ctx, reps=2):
    """One volume of the stack of spirals (64x64x48 on a 128x128 grid, 16 coils in 2 rings, 32
    interleaves x 2048 samples at 4 us, kz partial Fourier 6/8 and R = 2, +-80 Hz): the forward
    alone (`spiral_samples_3d`) and the whole acquisition with its reconstruction
    (`simulate_acquisition_3d`: forward, noise, kz GRAPPA fill, POCS, gridding + CG per partition),
    host-buffer calls by wall clock, host<->device copies included."""
    from mrsim_acq_b200 import kspace3d as K3
    from mrsim_acq_b200.api import T2, Acquisition
    o, n, nzs = 2, 64, 48
    sg = n * o
    kz = K3.KzSampling(0.75, 2)
    lo = nzs - min(nzs, int(round(nzs * kz.partial_fourier)))
    etl = sum(1 for p in range(nzs) if p >= lo and (p - nzs // 2) % kz.accel == 0)
    train = K3.EchoTrain(etl=etl, esp_ms=12.0, refocusing_deg=180.0, kz_order=K3.KzOrder.Centric, kz_segments=1)
    ro = K3.SpiralReadout(32, 8.192, 0.004, 1.2, kz)
    vox = np.arange(sg * sg * nzs)
    x, y, z = (vox % sg) / sg, ((vox // sg) % sg) / sg, (vox // (sg * sg)) / nzs
    img = (np.exp(-((x - 0.5) ** 2 + (y - 0.47) ** 2) / 0.04) * (1.0 + 0.3 * np.sin(6.3 * z))).astype(np.float32)
    fm = (80.0 * np.exp(-((x - 0.4) ** 2 + (y - 0.4) ** 2) / 0.02) - 80.0 * np.exp(-((x - 0.65) ** 2 + (y - 0.6) ** 2)
                                                                                     / 0.015)).astype(np.float32)
    acq3 = Acquisition(do_relaxation=True, do_distortions=True, n_coils=16, signal_scale=100.0, noise_variance=1e-4)
    args3 = ((sg, sg, nzs), (n, n, nzs), 1, [img], [T2.uniform(80.0)], [T2.uniform(1300.0)], fm, None, acq3, train, ro)
    kzo = K3.KzOptions(coil_rows=2, calibration_images=[img], calibration_seed=3, pocs=True)
    K3.spiral_samples_3d(*args3, kz_opts=kzo, ctx=ctx)  # warm
    t0 = time.perf_counter()
    for _ in range(reps):
        smp3 = K3.spiral_samples_3d(*args3, kz_opts=kzo, ctx=ctx)
    dt = (time.perf_counter() - t0) / reps
    acquired = int(np.count_nonzero(np.abs(smp3).reshape(16, nzs, -1).sum(axis=2)[0]))
    n_samp = 16 * acquired * smp3.shape[2]
    K3.simulate_acquisition_3d(*args3, seed=5, kz_opts=kzo, ctx=ctx)  # warm
    t0 = time.perf_counter()
    for _ in range(reps):
        K3.simulate_acquisition_3d(*args3, seed=5, kz_opts=kzo, ctx=ctx)
    dt_full = (time.perf_counter() - t0) / reps
    return {"config": "64x64x48 on 128x128, 16 coils in 2 rings, 32 x 2048 samples at 4 us, kz PF 6/8 R=2, +-80 Hz, "
                      "1 compartment, certified segmentation",
            "acquired_partitions": acquired, "samples_per_volume": n_samp,
            "seconds_per_volume": dt, "value": n_samp / dt, "unit": "samples/s",
            "acquisition_with_reconstruction_seconds_per_volume": dt_full,
            "acquisition_with_reconstruction_samples_per_s": n_samp / dt_full,
            "timing": "host-buffer calls (mrsim_spiral_samples_3d; mrsim_simulate_acquisition_3d_spiral with noise, "
                      "kz GRAPPA fill, POCS and the per-partition gridding + CG reconstruction) by wall clock, "
                      "host<->device copies included"}


def mixed_batch_measurement(ctx, stream, steps=3):
    """The precision-at-scale configuration's mixed batch: scans of 64, 96 and 128 on 2x grids with
    uneven slice counts 17, 23 and 31 (one volume each), 32 ring coils, 3 compartments, all lines,
    TE 40 ms, as one plan (`mrsim_epi_batch`: each stage one launch over every unit of every
    geometry); forward + complex-image adjoint, CUDA events on the context stream."""
    import torch
    from mrsim_acq_b200.api import T2, Acquisition, EpiBatch, PhaseModel
    acq = Acquisition(n_coils=32, t_line=0.5, t_echo=40.0, ghost_offset=0.05, signal_scale=100.0)
    series = []
    for n, nz in ((64, 17), (96, 23), (128, 31)):
        snx = 2 * n
        ys, xs = np.meshgrid((np.arange(snx) + 0.5) / snx, (np.arange(snx) + 0.5) / snx, indexing="ij")
        blob = np.exp(-((xs - 0.5) ** 2 + (ys - 0.48) ** 2) / 0.05).astype(np.float32)
        zs = (1.0 + 0.3 * np.sin(np.arange(nz) / 7.0)).astype(np.float32)
        imgs = [(blob[None] * np.float32(0.6 + 0.2 * c) * zs[:, None, None]).reshape(-1) for c in range(3)]
        fmap = np.tile((60.0 * (blob - 0.5)).astype(np.float32).reshape(-1), nz)
        series.append(dict(sim_dims=(snx, snx, nz), acq_dims=(n, n, nz), n_volumes=1, images=imgs, fmap=fmap,
                           t2=[T2.uniform(80.0), T2.uniform(250.0), T2.uniform(30.0)],
                           t_inhom=[T2.uniform(40.0), T2.uniform(60.0), T2.uniform(20.0)],
                           phase=PhaseModel.hbcd_like(), seed=42))
    b = EpiBatch(series, acq, echo_times_ms=[40.0], grads=0, ctx=ctx)
    b.forward()
    b.adjoint()
    ctx.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(steps):
        b.forward()
        b.adjoint()
    t1.record(stream)
    t1.synchronize()
    ctx.synchronize()
    ms = t0.elapsed_time(t1) / steps
    smp = b.samples
    b.close()
    return {"config": "scans 64/96/128 on 2x grids, 17/23/31 slices, 1 volume each, 32 ring coils, 3 compartments, "
                      "64/96/128 lines, TE 40 ms, one plan", "units": 17 + 23 + 31, "samples_per_step": smp,
            "ms_per_step": ms, "value": smp / (ms * 1e-3), "unit": "samples/s",
            "timing": "forward + complex-image adjoint, CUDA events on the context stream, mean of 3 after a warm-up"}


def grase_measurement(ctx):
    """The precision-at-scale configuration's GRASE train: 64x64x32 on a 128x128 grid, 4 shots (4 ky
    segments, one kz segment), echo spacing 20 ms, 150-degree refocusing (CPMG amplitudes from T1
    and T2), 32 ring coils, 3 compartments, one volume: the host-buffer call
    `simulate_acquisition_3d` (forward, noise, per-partition reconstruction), wall clock."""
    from mrsim_acq_b200 import kspace3d as K3
    from mrsim_acq_b200.api import T2, Acquisition, PhaseModel
    n, o, nz = 64, 2, 32
    sg = n * o
    vox = np.arange(sg * sg * nz)
    x, y, z = (vox % sg) / sg, ((vox // sg) % sg) / sg, (vox // (sg * sg)) / nz
    imgs = [(np.exp(-((x - 0.5 - 0.05 * c) ** 2 + (y - 0.47) ** 2) / 0.04) * (1.0 + 0.3 * np.sin(6.3 * z))
             ).astype(np.float32) for c in range(3)]
    fm = (40.0 * np.exp(-((x - 0.4) ** 2 + (y - 0.4) ** 2) / 0.02)).astype(np.float32)
    acq = Acquisition(do_relaxation=True, do_distortions=True, n_coils=32, signal_scale=100.0, noise_variance=1e-4)
    tr = K3.EchoTrain(etl=nz, esp_ms=20.0, refocusing_deg=150.0, kz_order=K3.KzOrder.Centric, kz_segments=1,
                      refocusing_time_ms=2.0)
    ro = K3.GraseReadout(ky_segments=4, t_line_ms=0.5, reverse_phase=False)
    args = ((sg, sg, nz), (n, n, nz), 1, imgs, [T2.uniform(80.0), T2.uniform(250.0), T2.uniform(30.0)],
            [T2.uniform(1330.0), T2.uniform(4000.0), T2.uniform(900.0)], fm, None, acq, tr, ro)
    K3.simulate_acquisition_3d(*args, phase=PhaseModel.none(), seed=5, ctx=ctx)  # warm
    runs = []
    for _ in range(3):
        t0 = time.perf_counter()
        K3.simulate_acquisition_3d(*args, phase=PhaseModel.none(), seed=5, ctx=ctx)
        runs.append(time.perf_counter() - t0)
    dt = float(np.median(runs))
    smp = 32 * nz * n * n
    return {"config": "GRASE 64x64x32 on 128x128, 4 shots, ESP 20 ms, 150-degree refocusing with T1, 32 ring coils, "
                      "3 compartments, 1 volume", "samples_per_volume": smp, "seconds_per_volume": dt,
            "seconds_per_volume_runs": [round(r, 4) for r in runs], "value": smp / dt, "unit": "samples/s",
            "timing": "mrsim_simulate_acquisition_3d with host buffers by wall clock (forward, noise, reconstruction), "
                      "median of 3 after a warm-up"}


def spin_history_series():
    """The spin-history workload at the reference's motivating size: a 197x233x100 source of 1 mm
    voxels (T1 1.33 s, every third voxel tracked), slabs of 128x136 cells x 20 slices of 5 mm, 40
    volumes of 20 sequential single-slice shots (TR 4.6 s, 40 ms apart) under a slow drift of
    0.5 mm through-plane with a (0.5, 0, 0.3) degree tilt, referenced to the 4.6 s saturation
    recovery."""
    from mrsim_acq_b200.motion import Pose
    from mrsim_acq_b200.spin_history import Recovery, Shot, Slabs, Source
    nx, ny, nz = 197, 233, 100
    nvox = nx * ny * nz
    cls = np.where(np.arange(nvox) % 3 == 0, 0, 255).astype(np.uint8)
    src = Source((nx, ny, nz), np.eye(4), np.full(nvox, 1.33, np.float32), np.ones(nvox, np.float32), cls, 1)
    s = np.eye(4)
    s[0, 0], s[1, 1], s[2, 2], s[2, 3] = 197.0 / 128.0, 233.0 / 136.0, 5.0, 2.0
    slabs = Slabs((128, 136, 20), s)
    center = (98.0, 116.0, 50.0)

    def volume(v):
        return [Shot(v * 4.6 + 3.6 + 0.04 * k,
                     Pose((0.5, 0.0, 0.3), (0.0, 0.0, 0.5 * (v + k / 20.0) / 40.0)).to_matrix(center), [k],
                     Recovery(4.6)) for k in range(20)]
    return src, slabs, volume


def spin_history_measurement(ctx, stream, cpu=True, n_vol=40):
    """The spin history (one batch of 20 shots per volume) on the device: the first volume untimed
    (kernels loaded, the history's buffers grown), then CUDA events on the context stream around
    the remaining volumes; beside it the FP64 oracle on one host thread over the same series (the
    CPU baseline) and the device's agreement with it over every volume."""
    import torch
    from mrsim_acq_b200.spin_history import SpinHistory
    src, slabs, volume = spin_history_series()
    vols = [volume(v) for v in range(n_vol)]
    t0 = time.perf_counter()
    h = SpinHistory(src, slabs, ctx=ctx)
    build_s = time.perf_counter() - t0
    per = h.terms_size(vols[0])
    out = torch.zeros(per * n_vol, dtype=torch.float32, device="cuda")
    prepared = [h.prepare(v) for v in vols]  # the shot arrays a C caller would hold
    torch.cuda.synchronize()
    h.excite_device(prepared[0], out.data_ptr())
    ctx.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(stream)
    for v in range(1, n_vol):
        h.excite_device(prepared[v], out.data_ptr() + 4 * per * v)
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - w0
    dev_ms = e0.elapsed_time(e1)
    timed = 20 * (n_vol - 1)
    merges = h.merges()
    res = {"config": f"source 197x233x100 (1 in 3 tracked), slabs 128x136x20, {n_vol} volumes x 20 single-slice "
                     "shots, drift 0.5 mm + tilt, reference 1 - e^{-4.6/T1}",
           "excitations_timed": timed, "tracked_voxels": h.n_tracked, "device_ms": dev_ms, "wall_ms": wall * 1e3,
           "value": timed / (dev_ms * 1e-3), "unit": "excitations/s", "merges": merges,
           "build_s": build_s, "launches": 2 * (n_vol - 1),
           "timing": "CUDA events on the context stream around the batch calls of volumes 1.. (one per volume; volume 0 "
                     "untimed as the warm-up) through the C ABI (the "
                     "library's host table preparation between launches included; the shot arrays marshalled "
                     "beforehand, as a C caller holds them)"}
    if cpu:
        from oracle import oracle
        n_cpu = n_vol
        t0 = time.perf_counter()
        o = oracle.SpinHistory(src, slabs)
        o_build = time.perf_counter() - t0
        t0 = time.perf_counter()
        ora = [o.excite_many(vols[v]) for v in range(n_cpu)]
        cpu_s = time.perf_counter() - t0
        dev = out[:per * n_cpu].cpu().numpy()
        flat = np.concatenate([np.stack([t.num, t.den]).ravel() for vol in ora for terms in vol for t in terms])
        scale = float(np.abs(flat).max())
        res["cpu_baseline"] = {"value": 20 * n_cpu / cpu_s, "unit": "excitations/s", "cores": 1, "kind": "port",
                               "sample": f"the same {n_cpu} volumes ({20 * n_cpu} excitations), FP64 oracle, "
                                         f"{cpu_s:.2f} s (+ {o_build:.2f} s to build)"}
        res["merges_oracle"] = o.merges()
        res["parity"] = {"bit_identical": int(np.count_nonzero(dev == flat)), "elements": int(flat.size),
                                       "max_abs_err_over_max": float(np.abs(dev.astype(np.float64) - flat).max()
                                                                     / max(scale, 1e-30))}
    h.close()
    return res


def run_ours(args, rank, world, local_rank):
    import torch
    from mrsim_acq_b200 import api
    torch.cuda.set_device(local_rank)
    ctx = api.Context(local_rank)
    acq = make_acquisition()
    # one series, sharded by slice ranges across the ranks (the slab semantics: global slice
    # indices, nz_full): every rank builds and computes only its slab
    from mrsim_acq_b200 import shard
    z0, z1 = shard.slice_ranges(WORKLOAD["nz"], world)[rank]
    inp = make_inputs(seed=1, z0=z0, z1=z1)
    from mrsim_acq_b200.api import EpiOperator, PhaseModel
    op = EpiOperator(inp["sim_dims"], inp["acq_dims"], inp["n_volumes"], inp["t2"], inp["fmap"], acq,
                     images=inp["images"], echo_times_ms=WORKLOAD["echoes"], t_inhom=inp["t_inhom"],
                     phase=PhaseModel.hbcd_like(), seed=42, grads=3, ctx=ctx, slice_z=list(range(z0, z1)),
                     nz_full=WORKLOAD["nz"])
    samples = op.samples
    total_samples = int(shard.allreduce_scalar(samples, "sum")) if world > 1 else samples
    # the autotuner picks the plan for this shape (cached per shape in a temporary file)
    tuned = op.tune(os.path.join(tempfile.gettempdir(), f"mrsim_tune_rank{rank}.txt"))
    stream = torch.cuda.ExternalStream(ctx.stream)
    snx, sny, nz = inp["sim_dims"]
    nx, ny, _ = inp["acq_dims"]
    units = inp["n_volumes"] * nz
    n_lines = samples // (units * acq.n_coils * nx)
    fy, fx = algorithmic_flops(units, n_lines, snx, sny, nx, acq.n_coils, WORKLOAD["ncomp"])

    def step(evs=None):
        for i in range(5):
            if evs is not None:
                evs[i].record(stream)
            op.stage(i)
        if evs is not None:
            evs[5].record(stream)

    for _ in range(args.warmup):
        step()
    ctx.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = Clocks(local_rank)
    clocks.start()
    ctx.synchronize()
    torch.cuda.synchronize()
    t_begin = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(6)] for _ in range(args.steps)]
    t_begin.record(stream)
    for k in range(args.steps):
        step(evs[k])
    t_end.record(stream)
    t_end.synchronize()
    ctx.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    total_ms = t_begin.elapsed_time(t_end)
    stage_ms = np.array([[evs[k][i].elapsed_time(evs[k][i + 1]) for i in range(5)] for k in range(args.steps)])
    stage_avg = stage_ms.mean(axis=0)
    ms_step = max_over_ranks(total_ms, world) / args.steps

    # end to end through the host-buffer C ABI call (pinned host memory)
    shp = op.shapes()
    pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()  # noqa: E731
    host_imgs = []
    for a in inp["images"]:
        h = pin(a.shape, torch.float32)
        h[...] = a
        host_imgs.append(h)
    out = {"kspace": pin(shp["kspace"] + (2,), torch.float32).view(np.complex64)[..., 0],
           "comp_grad": pin(shp["comp_grad"] + (2,), torch.float32).view(np.complex64)[..., 0],
           "fmap_grad": pin(shp["fmap_grad"], torch.float32), "r2_grad": pin(shp["r2_grad"], torch.float32)}
    e2e_steps = 0 if args.no_e2e else max(2, min(args.steps, 5))
    for _ in range(2 if e2e_steps else 0):
        op.apply_host(host_imgs, out)
    if world > 1:
        torch.distributed.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        op.apply_host(host_imgs, out)
    e1.record(stream)
    e1.synchronize()
    e2e_zf_ms = max_over_ranks(e0.elapsed_time(e1) / max(e2e_steps, 1), world)
    # the same outputs with the k-space in the compact layout (acquired rows only: no zero fill)
    first, step_rows, count = op.acquired_rows()
    kc = pin(shp["kspace"][:4] + (count, shp["kspace"][5], 2), torch.float32).view(np.complex64)[..., 0]
    out_c = dict(out, kspace=kc)
    for _ in range(2 if e2e_steps else 0):
        op.apply_host_compact(host_imgs, out_c)
    if world > 1:
        torch.distributed.barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        op.apply_host_compact(host_imgs, out_c)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / max(e2e_steps, 1), world)
    # bytes that cross the host link per call (the library skips k-space rows the sampling never
    # acquires and zero-fills them on the host)
    h2d, d2h = op.host_bytes()
    if world > 1:  # every rank's slab crosses its own host link
        h2d, d2h = int(shard.allreduce_scalar(h2d)), int(shard.allreduce_scalar(d2h))

    fp32 = ctx.probe_fp32_tflops()
    pk, pk_kind = peaks()
    # dominant kernel: the larger of the forward / adjoint y-stages
    dom = 1 if stage_avg[1] >= stage_avg[4] else 4
    dom_name = ["statics", "forward_ystage", "forward_xstage", "adjoint_xstage", "adjoint_ystage"][dom]
    achieved = fy / (stage_avg[dom] * 1e-3) / 1e12
    traffic = NCU_DRAM_BYTES_PER_UNIT[dom_name] * units
    res = {
        "metric": METRIC, "value": total_samples / (ms_step * 1e-3), "unit": "samples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD["name"], "sim_grid": [snx, sny], "acq_matrix": [nx, ny], "slices": nz,
                   "volumes": inp["n_volumes"], "echoes": list(WORKLOAD["echoes"]), "compartments": WORKLOAD["ncomp"],
                   "coils": acq.n_coils, "accel": acq.accel, "partial_fourier": acq.partial_fourier,
                   "samples_per_step": total_samples,
                   "parallelism": f"slices x{world} (one series sharded by slice ranges, no data-path collective)",
                   "autotune": tuned["choice"],
                   "l2": "inputs (236 MB images) larger than L2; no flush"},
        "e2e": {"value": total_samples / (e2e_ms * 1e-3) if e2e_steps else None, "unit": "samples/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "call": "mrsim_epi_operator_apply_host_compact (host images in; the acquired k-space rows and "
                        "the complex-image, fieldmap and R2 gradients out)"
                        + ("" if e2e_steps else "; not run (--no-e2e)"),
                "zero_filled_layout": {"value": total_samples / (e2e_zf_ms * 1e-3) if e2e_steps else None,
                                       "call": "mrsim_epi_operator_apply_host (the reference's zero-filled "
                                               "k-space layout: the same bytes cross the link, the host also "
                                               "zero-fills the rows never acquired)"}},
        "roofline": {"bound": "fp32", "kernel": dom_name,
                     "achieved": achieved, "peak": fp32, "unit": "TFLOP/s", "frac": achieved / fp32,
                     "peak_source": "measured live: register FMA loop on this GPU (no FP32 entry in MEASURED_PEAKS.json)",
                     "algorithmic_flops_per_launch": fy, "traffic": traffic,
                     "traffic_source": "ncu DRAM bytes per unit (24-volume capture) x units of this launch",
                     "stage_ms": dict(zip(["statics", "forward_ystage", "forward_xstage", "adjoint_xstage",
                                           "adjoint_ystage"], [round(float(v), 4) for v in stage_avg]))},
        "gpu_launches": 5 * args.steps,  # this rank's kernels in the timed region
        "clocks": clk,
    }
    if not args.no_scale and world == 1:
        res["scale"] = scale_measurements(args, ctx, stream)
        res["pipeline"] = pipeline_measurement(ctx, inp, acq, cpu=not args.no_cpu_baseline)
        res["spin_history"] = spin_history_measurement(ctx, stream, cpu=not args.no_cpu_baseline)
        res["gpu_launches_spin_history"] = res["spin_history"]["launches"]
    if not args.no_segmented and world == 1:
        res["segmented"] = segmented_comparison(args, inp, acq, ctx, stream, samples)
        res["gpu_launches"] += 3 * 6 * args.steps  # three more operators, up to 6 launches a step
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res["cpu_baseline"] = cpu_baseline(acq, inp, sample_volumes=args.cpu_volumes, sample_slices=args.cpu_slices)
        res["cpu_baseline"].update(cpu_baseline_extra(acq, inp))
    return res, op, ctx


def cpu_baseline(acq, inp, sample_volumes=1, sample_slices=8, threads=None):
    """The oracle (FP64 restatement of the reference's rotor forward, plus its FP64 transpose) on
    the host cores, forward + adjoint over a bounded sample of the same workload."""
    from oracle import oracle
    threads = threads or os.cpu_count() or 1
    snx, sny, nz = inp["sim_dims"]
    nx, ny, _ = inp["acq_dims"]
    nv = inp["n_volumes"]
    # the sample: `sample_volumes` volumes x `sample_slices` slices, every echo and coil
    vol = np.stack([a.reshape(nz, sny, snx, nv)[:sample_slices, :, :, :sample_volumes] for a in inp["images"]])
    imgs = [np.ascontiguousarray(vol[c]).reshape(-1) for c in range(vol.shape[0])]
    fmap = inp["fmap"].reshape(nz, sny, snx)[:sample_slices].reshape(-1)
    sim = (snx, sny, sample_slices)
    acqd = (nx, ny, sample_slices)
    from mrsim_acq_b200.api import PhaseModel
    kw = dict(t_inhom=inp["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42, nz_full=nz)
    t0 = time.perf_counter()
    k = oracle.series_forward(sim, acqd, sample_volumes, imgs, inp["t2"], fmap, acq, echo_times_ms=WORKLOAD["echoes"],
                              threads=threads, **kw)
    oracle.series_adjoint(sim, acqd, sample_volumes, imgs, inp["t2"], fmap, acq, k, echo_times_ms=WORKLOAD["echoes"],
                          threads=threads, **kw)
    dt = time.perf_counter() - t0
    rows = int(oracle.sampling_mask(nx, ny, acq)[:, 0].sum())
    samples = sample_volumes * sample_slices * acq.n_coils * len(WORKLOAD["echoes"]) * rows * nx
    return {"value": samples / dt, "unit": "samples/s", "cores": threads, "kind": "port",
            "sample": f"{sample_volumes} volume x {sample_slices} slices x {len(WORKLOAD['echoes'])} echoes x "
                      f"{acq.n_coils} coils ({samples} samples), forward + adjoint, FP64, {dt:.2f} s"}


def c1_inputs():
    """The plain single-shot case: scan 64x64 on 128x128, one slice, one coil, one compartment; a
    seeded 10-ellipse phantom (magnitudes U(0.2, 1), zero phase), T2 80 / T2' 40 ms, spin echo at
    TE 30 ms, 0.5 ms lines, ky order; a fieldmap of 3 Gaussian blobs (U(-60, 60) Hz, sigma
    U(8, 20) px)."""
    from mrsim_acq_b200.api import T2, Acquisition
    n, o = 64, 2
    s = n * o
    rng = np.random.default_rng(1)
    ys, xs = np.meshgrid((np.arange(s) + 0.5) / s, (np.arange(s) + 0.5) / s, indexing="ij")
    img = np.zeros((s, s), np.float32)
    for _ in range(10):
        cx, cy, a, b, th, mag = (rng.uniform(0.3, 0.7), rng.uniform(0.3, 0.7), rng.uniform(0.05, 0.25),
                                 rng.uniform(0.05, 0.25), rng.uniform(0, np.pi), rng.uniform(0.2, 1.0))
        c, sn = np.cos(th), np.sin(th)
        u = (c * (xs - cx) + sn * (ys - cy)) / a
        v = (-sn * (xs - cx) + c * (ys - cy)) / b
        img += np.float32(mag) * (u * u + v * v <= 1.0)
    rng2 = np.random.default_rng(2)
    fmap = np.zeros((s, s), np.float32)
    for _ in range(3):
        amp, sig = rng2.uniform(-60, 60), rng2.uniform(8, 20) * o
        cx, cy = rng2.uniform(0.3, 0.7) * s, rng2.uniform(0.3, 0.7) * s
        fmap += (amp * np.exp(-((xs * s - cx) ** 2 + (ys * s - cy) ** 2) / (2 * sig * sig))).astype(np.float32)
    acq = Acquisition(t_line=0.5, t_echo=30.0, t_inhom=40.0)
    return dict(sim_dims=(s, s, 1), acq_dims=(n, n, 1), n_volumes=1, images=[img.reshape(-1)], t2=[T2.uniform(80.0)],
                t_inhom=[T2.uniform(40.0)], fmap=fmap.reshape(-1)), acq


def cpu_baseline_extra(acq, inp):
    """The exact FP64 port on one host thread (a small sample of the benchmark series), and the
    plain single-shot case (forward + adjoint) on one thread."""
    from oracle import oracle
    from mrsim_acq_b200.api import PhaseModel
    one = cpu_baseline(acq, inp, sample_volumes=1, sample_slices=4, threads=1)
    c1, acq1 = c1_inputs()
    kw = dict(t_inhom=c1["t_inhom"], phase=PhaseModel.none(), seed=42)
    t0 = time.perf_counter()
    reps = 5
    for _ in range(reps):
        k = oracle.series_forward(c1["sim_dims"], c1["acq_dims"], 1, c1["images"], c1["t2"], c1["fmap"], acq1,
                                  threads=1, **kw)
        oracle.series_adjoint(c1["sim_dims"], c1["acq_dims"], 1, c1["images"], c1["t2"], c1["fmap"], acq1, k,
                              threads=1, **kw)
    dt = (time.perf_counter() - t0) / reps
    return {"single_thread": {"value": one["value"], "unit": "samples/s", "cores": 1, "sample": one["sample"]},
            "plain_single_shot": {"value": 4096 / dt, "unit": "samples/s", "cores": 1,
                                  "sample": f"scan 64x64 on 128x128, 1 slice, 1 coil, 1 compartment, forward + "
                                            f"adjoint, FP64, {dt * 1e3:.1f} ms"}}


def run_reference(args):
    acq = make_acquisition()
    inp = make_inputs(seed=1)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_baseline(acq, inp, sample_volumes=1, sample_slices=1, threads=threads)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_baseline(acq, inp, sample_volumes=1, sample_slices=args.ref_slices, threads=threads))
    wall = time.perf_counter() - t0
    v = float(np.median([r["value"] for r in vals]))
    cb = dict(vals[0])
    cb["value"] = v
    return {"metric": METRIC, "value": v, "unit": "samples/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD["name"], "note": "each step is a bounded sample of the series "
                       "(1 volume x %d slices, every echo and coil) on the host cores" % args.ref_slices},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-slices", type=int, default=30)
    ap.add_argument("--cpu-volumes", type=int, default=3)
    ap.add_argument("--ref-slices", type=int, default=30)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass (profiling runs)")
    ap.add_argument("--no-segmented", action="store_true", help="skip the time-segmented comparison")
    ap.add_argument("--no-scale", action="store_true", help="skip the larger-configuration measurements")
    ap.add_argument("--volumes", type=int, default=0, help="override the volume count (smaller profiling case)")
    ap.add_argument("--spin-history-only", action="store_true",
                    help="run only the spin-history workload and print its line (profiling)")
    ap.add_argument("--spin-volumes", type=int, default=40, help="volumes of the spin-history series")
    ap.add_argument("--spiral-only", action="store_true",
                    help="run only the stack-of-spirals volume and print its line (profiling)")
    ap.add_argument("--c5-only", action="store_true",
                    help="run only the mixed-geometry batch and the GRASE train and print their line (profiling)")
    ap.add_argument("--pipeline-only", action="store_true",
                    help="run only the whole-pipeline series (with --volumes: a smaller one) and print its line "
                         "(profiling)")
    args = ap.parse_args()
    if args.volumes > 0:
        WORKLOAD["nv"] = args.volumes
        WORKLOAD["name"] = WORKLOAD["name"].replace("-v40-", f"-v{args.volumes}-")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if args.spiral_only:
        from mrsim_acq_b200 import api
        print(json.dumps(spiral_measurement(api.Context(local_rank), reps=1)), flush=True)
        return
    if args.c5_only:
        import torch
        from mrsim_acq_b200 import api
        ctx = api.Context(local_rank)
        stream = torch.cuda.ExternalStream(ctx.stream)
        print(json.dumps({"mixed_batch": mixed_batch_measurement(ctx, stream), "grase": grase_measurement(ctx)}),
              flush=True)
        return
    if args.pipeline_only:
        from mrsim_acq_b200 import api
        print(json.dumps(pipeline_measurement(api.Context(local_rank), make_inputs(seed=1), make_acquisition(),
                                              cpu=not args.no_cpu_baseline)), flush=True)
        return
    if args.spin_history_only:
        import torch
        from mrsim_acq_b200 import api
        ctx = api.Context(local_rank)
        stream = torch.cuda.ExternalStream(ctx.stream)
        print(json.dumps(spin_history_measurement(ctx, stream, cpu=not args.no_cpu_baseline,
                                                  n_vol=args.spin_volumes)), flush=True)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res, op, ctx = run_ours(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(res), flush=True)
    op.close()
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
