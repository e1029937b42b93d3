"""Multi-GPU plumbing: one process per GPU, no collective on the data path.

Every (frame, voxel) output of the beamformer is independent and the only
reduction (compounding over transmits) stays inside one GPU, so work splits
into independent units:

* ensembles: each rank beamforms its own acquisitions (weak scaling);
* frames of one ensemble: rank r takes a contiguous frame range and writes
  its slice of the output (:func:`frame_shard`);
* depth slabs of one volume (:func:`zslab_shard`), for volumes too large
  for one device.

The collectives here are bookkeeping only: the slowest rank's time
(:func:`max_over_ranks`) and an optional gather of frame slices to one rank
(:func:`gather_frames`).  They run on whatever backend the process group has
(NCCL between GPUs, gloo on the host).
"""
from __future__ import annotations


def frame_shard(n_frame: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [begin, end) frame range of a rank: sizes differ by at most
    one and every frame belongs to exactly one rank."""
    if world < 1 or not 0 <= rank < world or n_frame < 0:
        raise ValueError("need 0 <= rank < world and n_frame >= 0")
    q, r = divmod(n_frame, world)
    begin = rank * q + min(rank, r)
    return begin, begin + q + (1 if rank < r else 0)


def zslab_shard(n_z: int, rank: int, world: int, align: int = 16) -> tuple[int, int]:
    """Contiguous [z0, z1) depth range of a rank, cut at multiples of
    ``align`` (the fused kernel's tile depth) except at the end."""
    if align < 1:
        raise ValueError("align >= 1")
    blocks = -(-n_z // align)
    b0, b1 = frame_shard(blocks, rank, world)
    return min(b0 * align, n_z), min(b1 * align, n_z)


def max_over_ranks(value: float, device=None) -> float:
    """Largest value over the ranks of the default process group (the time a
    multi-GPU step takes is the slowest rank's); the value itself without a
    process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_frames(local, n_frame: int, dst: int = 0):
    """Collects each rank's frame slice (``local`` = output rows of
    frame_shard(n_frame, rank, world)) into the full [n_frame, ...] tensor on
    rank ``dst`` (None elsewhere).  Slices are padded to the longest so one
    all-gather of equal shapes carries them."""
    import torch
    import torch.distributed as dist
    if local.is_complex():   # carried as (re, im) pairs: not every backend moves complex tensors
        full = gather_frames(torch.view_as_real(local), n_frame, dst)
        return None if full is None else torch.view_as_complex(full)
    world, rank = dist.get_world_size(), dist.get_rank()
    longest = -(-n_frame // world)
    b, e = frame_shard(n_frame, rank, world)
    if local.shape[0] != e - b:
        raise ValueError(f"rank {rank} holds {local.shape[0]} frames, its shard is {e - b}")
    pad = torch.zeros((longest,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: e - b] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    if rank != dst:
        return None
    out = torch.empty((n_frame,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    for r, p in enumerate(parts):
        rb, re_ = frame_shard(n_frame, r, world)
        out[rb:re_] = p[: re_ - rb]
    return out
