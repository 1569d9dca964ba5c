"""One EPI series sharded across ranks (one process per GPU): each rank takes a range of slices of
every volume, through the reference's slab semantics (`AcquisitionOptions::slice_z / nz_full`,
kspace.rs:1745-1750: a slab of slices keeps each slice's global index, so its phase model,
timing and seeds are those of the full series).  A rank uploads only its slab's images and
fieldmap, computes its units, and writes its own output slab; `gather_slabs` assembles the
slabs on rank 0 over torch.distributed (NCCL on GPUs, gloo on CPU).  A fieldmap fit all-reduces
only scalars (the loss, the gradient's largest magnitude): the fieldmap gradient of a slice
depends on that slice alone.

The reference parallelises over volumes with rayon (kspace.rs:2064-2070); slices are the unit
here because the slab semantics carry every per-slice input (global slice index, fieldmap and
maps slab) while volumes share nothing but their images."""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import numpy as np


def slice_ranges(nz: int, world: int) -> list[tuple[int, int]]:
    """Contiguous slice ranges, one per rank, sizes differing by at most one (ranks past nz get
    empty ranges)."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    base, extra = divmod(nz, world)
    out, z = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((z, z + n))
        z += n
    return out


def slab_inputs(sim_dims, acq_dims, n_volumes: int, images: Sequence[np.ndarray], fmap: np.ndarray,
                z0: int, z1: int, t2=None, t_inhom=None) -> dict:
    """The inputs of slices [z0, z1) in the operator's creation layouts: images per compartment
    `vox * n_volumes + g` (vox = x + snx (y + sny z)), fieldmap `[z][y][x]`, voxel maps of T2 /
    T2' likewise; plus `slice_z` (global indices) and `nz_full`."""
    from mrsim_acq_b200.api import T2
    snx, sny, nz = sim_dims
    plane = snx * sny
    imgs = [np.ascontiguousarray(np.asarray(a).reshape(nz, plane * n_volumes)[z0:z1]).reshape(-1) for a in images]
    f = np.ascontiguousarray(np.asarray(fmap).reshape(nz, plane)[z0:z1]).reshape(-1)

    def maps(v):
        if v is None:
            return None
        return [T2.of_map(np.ascontiguousarray(np.asarray(m.map).reshape(nz, plane)[z0:z1]).reshape(-1))
                if m.is_map else m for m in v]

    return dict(sim_dims=(snx, sny, z1 - z0), acq_dims=(acq_dims[0], acq_dims[1], z1 - z0), n_volumes=n_volumes,
                images=imgs, fmap=f, t2=maps(t2), t_inhom=maps(t_inhom), slice_z=list(range(z0, z1)), nz_full=nz)


def _dist():
    import torch.distributed as dist
    return dist


def _device_for_backend():
    import torch
    dist = _dist()
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def gather_slabs(local: Optional[np.ndarray], z_axis: int, ranges: Sequence[tuple[int, int]], rank: int,
                 world: int) -> Optional[np.ndarray]:
    """Every rank passes its output slab (slices along `z_axis`, any other axes equal across
    ranks); rank 0 returns the assembled array in slice order, the others None.  Slabs travel as
    raw bytes padded to the largest slab (one all_gather), so the assembled array is bit for bit
    the slabs' contents."""
    if world == 1:
        return local
    import torch
    dist = _dist()
    dev = _device_for_backend()
    sizes = [z1 - z0 for z0, z1 in ranges]
    # the shape of one slice along z_axis, from the slab (every rank with slices has the same)
    shape = list(local.shape)
    per_slice = int(np.prod(shape)) // max(shape[z_axis], 1) if shape[z_axis] else 0
    # the other axes, to carry the shape to ranks with empty slabs
    meta = torch.tensor([per_slice, local.dtype.itemsize] + shape[:z_axis] + shape[z_axis + 1:], dtype=torch.int64,
                        device=dev)
    metas = [torch.zeros_like(meta) for _ in range(world)]
    dist.all_gather(metas, meta)
    ref = max(range(world), key=lambda r: int(metas[r][0]))
    per_slice, itemsize = int(metas[ref][0]), int(metas[ref][1])
    others = [int(v) for v in metas[ref][2:]]
    nbytes_max = max(sizes) * per_slice * itemsize
    # move z to the front so a slab is one contiguous block per rank
    moved = np.ascontiguousarray(np.moveaxis(local, z_axis, 0)).view(np.uint8).reshape(-1)
    buf = torch.zeros(nbytes_max, dtype=torch.uint8, device=dev)
    if moved.size:
        buf[: moved.size] = torch.from_numpy(moved).to(dev)
    bufs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf)
    if rank != 0:
        return None
    parts = []
    for r, n in enumerate(sizes):
        if n == 0:
            continue
        raw = bufs[r][: n * per_slice * itemsize].cpu().numpy()
        zfirst = raw.view(local.dtype).reshape([n] + others)
        parts.append(zfirst)
    full = np.concatenate(parts, axis=0)
    return np.moveaxis(full, 0, z_axis)


def allreduce_scalar(v: float, op: str = "sum", reduce: bool = True) -> float:
    """A float64 scalar reduced over every rank (sum or max); the value itself without a
    process group (or with `reduce` false)."""
    dist = _dist()
    if not reduce or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(v)
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX)
    return float(t.item())


def descent_step(f: np.ndarray, loss_grad: Callable[[np.ndarray], tuple], alpha: float, loss: float,
                 grad: np.ndarray, reduce: bool = True) -> tuple:
    """One step of the fieldmap descent on a rank's slab (the fit of the differentiation
    workload): move by at most `alpha` Hz along -grad (scaled by the largest |grad| over every
    rank), accept on a lower total loss (summed over ranks), else halve alpha.  `loss_grad(f)`
    returns this rank's (partial loss, fieldmap gradient).  Returns (f, loss, grad, alpha,
    accepted); the same on every rank, whatever the slab split.  `reduce` false: a single-rank fit
    of the whole series."""
    gmax = allreduce_scalar(float(np.abs(grad).max()) if grad.size else 0.0, "max", reduce)
    fn = (f - (alpha / gmax) * grad).astype(np.float32) if gmax > 0 else f
    ln, gn = loss_grad(fn)
    ln = allreduce_scalar(ln, "sum", reduce)
    if ln < loss:
        return fn, ln, gn, alpha * 1.3, True
    return f, loss, grad, alpha * 0.5, False
