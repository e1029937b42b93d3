"""Multi-GPU plumbing: one process per GPU, no collective on the data path.

Every (frame, voxel) output of the beamformer is independent and the only
reduction (compounding over transmits) stays inside one GPU, so work splits
into independent units:

* ensembles: each rank beamforms its own acquisitions (weak scaling);
* frames of one ensemble: rank r takes a contiguous frame range and writes
  its slice of the output (:func:`frame_shard`);
* depth slabs of one volume (:func:`zslab_shard`), for volumes too large
  for one device;
* :func:`bf_rca_sharded` runs ``bf_rca`` on one acquisition split either way
  and gathers the volume on one rank.

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


def gather_axis(local, n_total: int, shard, axis: int = 0, dst: int = 0):
    """Collects each rank's slice along ``axis`` (rank r holds indices
    ``shard(n_total, r, world)``) into the full tensor on rank ``dst`` (None
    elsewhere).  Slices are padded to the longest so that one all-gather of
    equal shapes carries them; complex tensors travel as (re, im) pairs."""
    import torch
    import torch.distributed as dist
    if local.is_complex():   # not every backend moves complex tensors
        full = gather_axis(torch.view_as_real(local), n_total, shard, axis % local.dim(), dst)
        return None if full is None else torch.view_as_complex(full)
    world, rank = dist.get_world_size(), dist.get_rank()
    axis = axis % local.dim()
    spans = [shard(n_total, r, world) for r in range(world)]
    longest = max(e - b for b, e in spans)
    b, e = spans[rank]
    if local.shape[axis] != e - b:
        raise ValueError(f"rank {rank} holds {local.shape[axis]} entries along axis {axis}, its shard is {e - b}")
    shape = list(local.shape)
    shape[axis] = longest
    pad = torch.zeros(shape, dtype=local.dtype, device=local.device)
    pad.narrow(axis, 0, e - b).copy_(local)
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    if rank != dst:
        return None
    shape[axis] = n_total
    out = torch.empty(shape, dtype=local.dtype, device=local.device)
    for (rb, re_), part in zip(spans, parts):
        out.narrow(axis, rb, re_ - rb).copy_(part.narrow(axis, 0, re_ - rb))
    return out


def gather_frames(local, n_frame: int, dst: int = 0):
    """Collects each rank's frame slice (``local`` = output rows of
    frame_shard(n_frame, rank, world)) into the full [n_frame, ...] tensor on
    rank ``dst`` (None elsewhere)."""
    return gather_axis(local, n_frame, frame_shard, 0, dst)


def _n_transmits(Transmit: dict) -> int:
    import numpy as np
    for k in ("thetaX", "virtualSourceX", "thetaY", "virtualSourceY"):
        if k in Transmit:
            return int(np.asarray(Transmit[k]).size)
    raise ValueError("Transmit needs thetaX/thetaY or virtualSourceX/Y/Z")


def _to_group_tensor(x):
    """An output as a tensor the process group's backend can move."""
    import numpy as np
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(x)) if not isinstance(x, torch.Tensor) else x
    if dist.get_backend() == "nccl" and not t.is_cuda:
        t = t.cuda()
    if dist.get_backend() != "nccl" and t.is_cuda:
        t = t.cpu()
    return t.contiguous()


def bf_rca_sharded(data, Geometry: dict, Transmit: dict, Param: dict, Options=None, *, split: str = "frames",
                   dst: int = 0, align: int = 16, beamform=None):
    """``bf_rca`` of one acquisition split over the ranks of the default
    process group, gathered on rank ``dst``.

    split = "frames": rank r beamforms frames frame_shard(n_frame, r, world) of
    the acquisition -- the axis the reference wrapper itself cuts the
    acquisition along (bfVirtualSourceGeneric_RCA.m:587-594) -- and the frame
    slices are gathered along the last axis.  split = "zslab": rank r
    beamforms depth rows zslab_shard(Nz, r, world, align) of the grid for
    every frame, gathered along the first axis.  Every (voxel, frame) output
    is computed by exactly one rank and the compounding over transmits stays
    on that rank, so the gather is the only collective.

    ``data`` is the whole acquisition in the reference layout [Ns, channels,
    1, events] (events: transmit fastest, then frames) on every rank.
    ``beamform`` is the per-rank call, ``bf_rca`` by default.  Returns
    (dataBf, mask) on rank ``dst`` as torch tensors (None, None elsewhere)."""
    import numpy as np
    import torch.distributed as dist
    if beamform is None:
        from .beamformer import bf_rca as beamform
    world, rank = dist.get_world_size(), dist.get_rank()
    O = dict(Options or {})
    if split == "frames":
        n_tx = _n_transmits(Transmit)
        n_event = int(data.shape[-1])
        if n_event % n_tx:
            raise ValueError(f"{n_event} events are not a whole number of frames of {n_tx} transmits")
        n_frame = n_event // n_tx
        if n_frame < world:
            raise ValueError(f"{n_frame} frames cannot be split over {world} ranks")
        b, e = frame_shard(n_frame, rank, world)
        db, mk = beamform(data[..., b * n_tx:e * n_tx], Geometry, Transmit, Param, O)
        full = gather_axis(_to_group_tensor(db), n_frame, frame_shard, axis=-1, dst=dst)
        mask = _to_group_tensor(mk) if rank == dst else None   # frame-independent: the same on every rank
        return full, mask
    if split == "zslab":
        nz = int(np.shape(Geometry["gridBfX"])[0])
        if nz < world:
            raise ValueError(f"{nz} depth rows cannot be split over {world} ranks")
        shard = lambda n, r, w: zslab_shard(n, r, w, align)   # noqa: E731
        z0, z1 = shard(nz, rank, world)
        G = dict(Geometry)
        for k in ("gridBfX", "gridBfY", "gridBfZ"):
            G[k] = np.asarray(Geometry[k])[z0:z1]
        if z1 > z0:
            db, mk = beamform(data, G, Transmit, Param, O)
            db, mk = _to_group_tensor(db), _to_group_tensor(mk)
        else:   # an empty slab (more ranks than aligned slabs): contributes nothing
            G1 = dict(G)
            for k in ("gridBfX", "gridBfY", "gridBfZ"):
                G1[k] = np.asarray(Geometry[k])[:1]
            db1, mk1 = beamform(data, G1, Transmit, Param, O)
            db, mk = _to_group_tensor(db1)[:0], _to_group_tensor(mk1)[:0]
        return (gather_axis(db, nz, shard, axis=0, dst=dst), gather_axis(mk, nz, shard, axis=0, dst=dst))
    raise ValueError(f"split must be 'frames' or 'zslab', not {split!r}")
