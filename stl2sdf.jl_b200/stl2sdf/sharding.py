"""Multi-GPU split of the hot path: one process per GPU, no exchange during compute.

Every grid node is independent, so one grid is cut into z-slabs (whole x-y layers, z being the
slowest index, so each slab is one contiguous block of the x-fastest field) and a batch of meshes
is dealt out by longest-processing-time (LPT) order on the estimated work ngp * log2(nel).  Each
rank holds the whole mesh (it builds its own LBVH from the host arrays), computes its part through
the C ABI, and rank 0 gathers the parts with ``torch.distributed`` (NCCL on GPUs, gloo on CPU).
The reference is single-process (``Threads.@threads`` over nodes, RaycastingSignDetection.jl:354,
dfOnTriangularMesh.jl:58); this module is the distributed counterpart of that loop.
"""

from __future__ import annotations

import math

import numpy as np


def zslab_bounds(nz_layers: int, world: int, rank: int):
    """(k0, k1) inclusive z layers of `rank` when `nz_layers` layers are split over `world`
    ranks as evenly as possible (the first nz_layers % world ranks get one more), or None when the
    rank gets no layer."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(int(nz_layers), world)
    size = base + (1 if rank < extra else 0)
    if size == 0:
        return None
    k0 = rank * base + min(rank, extra)
    return k0, k0 + size - 1


def lpt_assign(works, world: int):
    """Longest-processing-time assignment: item indices per rank, heaviest items first, each to
    the least-loaded rank (ties to the lower rank).  Deterministic, so every rank computes the
    same plan without communication."""
    loads = [0.0] * world
    plan = [[] for _ in range(world)]
    for i in sorted(range(len(works)), key=lambda k: (-float(works[k]), k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        plan[r].append(i)
        loads[r] += float(works[i])
    return plan


def mesh_work(ngp: int, nel: int) -> float:
    return float(ngp) * math.log2(max(2, int(nel)))


def gather_zslabs(part: np.ndarray, N, group=None, device=None):
    """Concatenation along z of every rank's slab (as split by zslab_bounds) on rank 0; None on
    the other ranks.  `device` is the torch device of the collective buffers (a CUDA device for
    NCCL, None / 'cpu' for gloo)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    layer = int((N[0] + 1) * (N[1] + 1))
    sizes = []
    for r in range(world):
        b = zslab_bounds(int(N[2]) + 1, world, r)
        sizes.append(0 if b is None else (b[1] - b[0] + 1) * layer)
    if part.shape[0] != sizes[rank]:
        raise ValueError(f"rank {rank} slab has {part.shape[0]} values, expected {sizes[rank]}")
    cap = max(sizes)
    buf = torch.zeros(cap, dtype=torch.float64, device=device)
    if sizes[rank]:
        buf[: sizes[rank]] = torch.from_numpy(np.ascontiguousarray(part, np.float64)).to(buf.device)
    outs = [torch.empty_like(buf) for _ in range(world)] if rank == 0 else None
    dist.gather(buf, outs, dst=0, group=group)
    if rank != 0:
        return None
    return np.concatenate([outs[r][: sizes[r]].cpu().numpy() for r in range(world)])


def local_device(device=None) -> int:
    """CUDA ordinal of this rank's GPU: the index of `device` (a torch device, an int or a 'cuda:k'
    string) when given, else LOCAL_RANK from the launcher's environment, else 0."""
    import os

    if device is None:
        return int(os.environ.get("LOCAL_RANK", "0"))
    if isinstance(device, int):
        return device
    if isinstance(device, str):
        return int(device.split(":", 1)[1]) if ":" in device else 0
    idx = getattr(device, "index", None)
    return int(idx) if idx is not None else 0


def sdf_zslab(X, IEN, origin, h, N, compute=None, group=None, device=None, **vote):
    """The whole sdf field of grid (origin, h, N) computed as z-slabs, one per rank, gathered on
    rank 0 (returned there; None elsewhere).  compute(k0, k1) -> slab values; the default builds a
    context on this rank's GPU -- `device` when given, else the LOCAL_RANK torchrun sets (one process
    per GPU), else GPU 0 -- and calls sdfgpu_sdf_slab."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    b = zslab_bounds(int(N[2]) + 1, world, rank)
    if compute is None:
        from . import _native

        ctx = _native.Context(local_device(device))
        ctx.set_mesh(X, IEN)

        def compute(k0, k1):
            return ctx.sdf_slab(origin, h, N, k0, k1, **vote)

    part = compute(*b) if b is not None else np.empty(0)
    return gather_zslabs(part, N, group=group, device=device)
