"""One series sharded across two ranks by slice ranges (gloo, CPU): each rank computes its slab
through the slab semantics (`slice_z`, `nz_full`), rank 0 assembles the slabs, and the result is
bit for bit the single-rank result; a fieldmap descent step on slabs (loss summed and gradient
maximum taken over ranks) equals the unsharded step.  The per-rank compute here is the FP64
oracle, the stand-in for each rank's GPU operator on a CPU-only host: the host logic under test
(ranges, slab inputs, gather, scalar reductions) is the same for both."""
from __future__ import annotations

import os
import socket
import sys

import numpy as np
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _series(nz=5, nv=2):
    from mrsim_acq_b200.api import Acquisition, PartialFourierMode, PhaseModel
    from tests import cases
    s = cases.series_case(nx=16, ny=16, nz=nz, o=2, nv=nv, ncomp=2)
    acq = Acquisition(n_coils=4, accel=2, partial_fourier=0.75, pf_mode=PartialFourierMode.Scanner, t_line=0.5,
                      t_echo=30.0, ghost_offset=0.03, eddy_phase=0.1)
    kw = dict(t_inhom=s["t_inhom"], phase=PhaseModel.hbcd_like(), seed=42,
              eddy_drive=[(0.5, -0.4, 0.7)] * nv, prep_drive=[(1000.0, (0.6, 0.8, 0.0))] * nv)
    return s, acq, [20.0, 40.0], kw


def _init(rank, world, port):
    sys.path.insert(0, ROOT)
    torch.distributed.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                         world_size=world)


def _assemble_main(rank, world, port, out):
    _init(rank, world, port)
    try:
        from mrsim_acq_b200 import shard
        from oracle import oracle
        s, acq, tes, kw = _series()
        nz = s["sim_dims"][2]
        ranges = shard.slice_ranges(nz, world)
        z0, z1 = ranges[rank]
        sl = shard.slab_inputs(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["fmap"], z0, z1)
        k = oracle.series_forward(sl["sim_dims"], sl["acq_dims"], sl["n_volumes"], sl["images"], s["t2"], sl["fmap"],
                                  acq, echo_times_ms=tes, slice_z=sl["slice_z"], nz_full=sl["nz_full"], **kw)
        adj = oracle.series_adjoint(sl["sim_dims"], sl["acq_dims"], sl["n_volumes"], sl["images"], s["t2"], sl["fmap"],
                                    acq, k, echo_times_ms=tes, slice_z=sl["slice_z"], nz_full=sl["nz_full"], **kw)
        full = {name: shard.gather_slabs(a, 1, ranges, rank, world)
                for name, a in (("kspace", k), ("comp_grad", adj["comp_grad"]), ("fmap_grad", adj["fmap_grad"]))}
        if rank == 0:
            want_k = oracle.series_forward(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"],
                                           acq, echo_times_ms=tes, **kw)
            want = oracle.series_adjoint(s["sim_dims"], s["acq_dims"], s["n_volumes"], s["images"], s["t2"], s["fmap"],
                                         acq, want_k, echo_times_ms=tes, **kw)
            out["kspace"] = bool(np.array_equal(full["kspace"], want_k))
            out["comp_grad"] = bool(np.array_equal(full["comp_grad"], want["comp_grad"]))
            out["fmap_grad"] = bool(np.array_equal(full["fmap_grad"], want["fmap_grad"]))
            out["ranges"] = ranges
    finally:
        torch.distributed.destroy_process_group()


def _loss_grad_fn(s, acq, tes, kw, sobs, sl=None):
    from oracle import oracle

    def lg(f):
        if sl is None:
            k = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], f, acq, echo_times_ms=tes,
                                      **kw)
            r = k - sobs
            g = oracle.series_adjoint(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], f, acq, r,
                                      echo_times_ms=tes, **kw)["fmap_grad"]
        else:
            k = oracle.series_forward(sl["sim_dims"], sl["acq_dims"], 1, sl["images"], s["t2"], f, acq,
                                      echo_times_ms=tes, slice_z=sl["slice_z"], nz_full=sl["nz_full"], **kw)
            r = k - sobs
            g = oracle.series_adjoint(sl["sim_dims"], sl["acq_dims"], 1, sl["images"], s["t2"], f, acq, r,
                                      echo_times_ms=tes, slice_z=sl["slice_z"], nz_full=sl["nz_full"], **kw)["fmap_grad"]
        return float(np.sum(np.abs(r) ** 2)), g.reshape(-1)
    return lg


def _descent_main(rank, world, port, out):
    _init(rank, world, port)
    try:
        from mrsim_acq_b200 import shard
        from oracle import oracle
        s, acq, tes, kw = _series(nv=1)
        snx, sny, nz = s["sim_dims"]
        truth = (s["fmap"] + 4.0 * np.cos(np.arange(s["fmap"].size) / 37.0)).astype(np.float32)
        sobs = oracle.series_forward(s["sim_dims"], s["acq_dims"], 1, s["images"], s["t2"], truth, acq,
                                     echo_times_ms=tes, **kw)
        ranges = shard.slice_ranges(nz, world)
        z0, z1 = ranges[rank]
        sl = shard.slab_inputs(s["sim_dims"], s["acq_dims"], 1, s["images"], s["fmap"], z0, z1)
        lg = _loss_grad_fn(s, acq, tes, kw, sobs[:, z0:z1], sl)
        f = sl["fmap"].copy()
        L, g = lg(f)
        L = shard.allreduce_scalar(L, "sum")
        alpha = 1.0
        steps = []
        for _ in range(3):
            f, L, g, alpha, ok = shard.descent_step(f, lg, alpha, L, g)
            steps.append((L, alpha, ok))
        fs = shard.gather_slabs(f.reshape(1, z1 - z0, sny * snx), 1, ranges, rank, world)
        if rank == 0:
            lg1 = _loss_grad_fn(s, acq, tes, kw, sobs)
            f1 = s["fmap"].copy()
            L1, g1 = lg1(f1)
            a1 = 1.0
            ref = []
            for _ in range(3):
                f1, L1, g1, a1, ok = shard.descent_step(f1, lg1, a1, L1, g1, reduce=False)
                ref.append((L1, a1, ok))
            out["fieldmap_equal"] = bool(np.array_equal(fs.reshape(-1), f1))
            out["accepts"] = [st[2] for st in steps] == [r[2] for r in ref]
            out["loss_rel"] = max(abs(a[0] - b[0]) / b[0] for a, b in zip(steps, ref))
            out["any_accepted"] = any(r[2] for r in ref)
    finally:
        torch.distributed.destroy_process_group()


def test_slice_ranges():
    sys.path.insert(0, ROOT)
    from mrsim_acq_b200 import shard
    assert shard.slice_ranges(30, 8) == [(0, 4), (4, 8), (8, 12), (12, 16), (16, 20), (20, 24), (24, 27), (27, 30)]
    assert shard.slice_ranges(2, 3) == [(0, 1), (1, 2), (2, 2)]
    assert shard.slice_ranges(16, 1) == [(0, 16)]


def _spawn(fn):
    world, port = 2, _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.start_processes(fn, args=(world, port, out), nprocs=world, start_method="spawn")
        return dict(out)


def test_two_ranks_assemble_the_single_rank_series_bit_for_bit():
    out = _spawn(_assemble_main)
    assert out["ranges"] == [(0, 3), (3, 5)]
    assert out["kspace"] and out["comp_grad"] and out["fmap_grad"], out


def test_sharded_fieldmap_descent_equals_the_unsharded_steps():
    out = _spawn(_descent_main)
    assert out["any_accepted"] and out["accepts"], out
    assert out["fieldmap_equal"], out
    assert out["loss_rel"] <= 1e-12, out


def test_bench_slab_inputs_are_the_series_slices():
    """bench.py builds a rank's slab directly: the same values as those slices of the whole series."""
    sys.path.insert(0, ROOT)
    import bench
    saved = dict(bench.WORKLOAD)
    try:
        bench.WORKLOAD["nv"] = 2
        full = bench.make_inputs(seed=1)
        part = bench.make_inputs(seed=1, z0=7, z1=12)
    finally:
        bench.WORKLOAD.clear()
        bench.WORKLOAD.update(saved)
    snx, sny, nz = full["sim_dims"]
    assert part["sim_dims"] == (snx, sny, 5)
    for a, b in zip(full["images"], part["images"]):
        assert np.array_equal(a.reshape(nz, -1)[7:12].ravel(), b)
    assert np.array_equal(full["fmap"].reshape(nz, -1)[7:12].ravel(), part["fmap"])
