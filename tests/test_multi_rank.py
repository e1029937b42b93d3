"""Host side of the multi-GPU path, run as world-size-2 process groups on the
CPU (gloo): frame and depth-slab sharding cover every unit once, the step
time is the slowest rank's, frame slices gather back in order, and only
rank 0 reports."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from simu_rca_ab_b200.multi import frame_shard, gather_frames, max_over_ranks, zslab_shard


@pytest.mark.parametrize("n", [0, 1, 7, 8, 200, 203])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_frame_shards_cover_each_frame_once(n, world):
    seen = []
    sizes = []
    for r in range(world):
        b, e = frame_shard(n, r, world)
        seen.extend(range(b, e))
        sizes.append(e - b)
    assert seen == list(range(n))
    assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("nz,world,align", [(160, 8, 16), (384, 3, 16), (100, 4, 8), (5, 2, 16)])
def test_zslabs_are_aligned_and_cover_the_volume(nz, world, align):
    zs = [zslab_shard(nz, r, world, align) for r in range(world)]
    assert zs[0][0] == 0 and zs[-1][1] == nz
    for (a0, a1), (b0, b1) in zip(zs, zs[1:]):
        assert a1 == b0 and a0 <= a1
    for z0, _ in zs:
        assert z0 % align == 0 or z0 == nz


def test_bad_shard_arguments_raise():
    with pytest.raises(ValueError):
        frame_shard(10, 2, 2)
    with pytest.raises(ValueError):
        zslab_shard(10, 0, 1, align=0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n_frame, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # a rank "beamforms" its frame slice: frame f of the full output is f + 1j*f
        b, e = frame_shard(n_frame, rank, world)
        local = torch.stack([torch.full((3, 5), complex(f, -f), dtype=torch.complex64) for f in range(b, e)]) \
            if e > b else torch.zeros((0, 3, 5), dtype=torch.complex64)
        full = gather_frames(local, n_frame, dst=0)
        slow = max_over_ranks(10.0 * (rank + 1))
        if rank == 0:
            ref = torch.stack([torch.full((3, 5), complex(f, -f), dtype=torch.complex64) for f in range(n_frame)])
            q.put(("rank0", bool(torch.equal(full, ref)), slow))
        else:
            q.put(("other", full is None, slow))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_frame", [7, 200])
def test_two_ranks_gather_frames_and_take_the_slowest_time(n_frame):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n_frame, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    by = {r[0]: r for r in res}
    assert by["rank0"][1] is True            # rank 0 holds every frame, in order
    assert by["other"][1] is True            # the others hold nothing
    assert by["rank0"][2] == by["other"][2] == 20.0   # max over ranks


def test_max_over_ranks_without_a_group_is_the_value():
    assert max_over_ranks(3.5) == 3.5
