"""Host side of the multi-GPU path, run as world-size-2 process groups on the
CPU (gloo): frame and depth-slab sharding cover every unit once, the step
time is the slowest rank's, frame slices gather back in order, only rank 0
reports, and ``bf_rca_sharded`` -- one acquisition split over the ranks by
frames or by depth slabs, each rank computing its shard with the FP64 oracle
on the CPU -- gathers exactly the volume of one full-volume oracle run."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from simu_rca_ab_b200.multi import bf_rca_sharded, frame_shard, gather_frames, max_over_ranks, zslab_shard


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


# ---------------------------------------------------------------------------
# one acquisition split over two ranks, each rank's shard by the FP64 oracle
# ---------------------------------------------------------------------------
def _oracle_bf(data, Geometry, Transmit, Param, Options):
    """The per-rank compute of bf_rca_sharded for this test: the FP64 oracle
    with the Lanczos kernel of the workload, compounded, in the reference's
    output shapes (as bf_rca returns them)."""
    import warnings

    from oracle import host as H
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        r = H.prepare(data, Geometry, Transmit, Param, Options)
    f64, m64 = H.run_fp64(r, H.INTERP_LANCZOS, int(Options.get("lanczosOrder", 3)), threads=2)
    c, cm = H.compound(f64, m64, True)
    return H.matlab_shape(r, c, cm)


def _case():
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c0", grid_scale=0.125, n_frame=5)
    g = w.groups[0]
    data = W.channel_data(w, seed=31, device="cpu").numpy()
    return w, g, W.as_matlab(W.group_data(w, data, 0))


def _sharded_worker(rank, world, port, split, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w, g, data = _case()
        db, mk = bf_rca_sharded(data, g.Geometry, g.Transmit, w.Param, w.Options, split=split, dst=0, align=4,
                                beamform=_oracle_bf)
        if rank == 0:
            ref_db, ref_mk = _oracle_bf(data, g.Geometry, g.Transmit, w.Param, w.Options)
            q.put(("rank0", tuple(db.shape), tuple(ref_db.shape), bool(torch.equal(db, torch.from_numpy(ref_db))),
                   bool(torch.equal(mk, torch.from_numpy(ref_mk))), float(db.abs().max())))
        else:
            q.put(("other", db is None, mk is None))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("split", ["frames", "zslab"])
def test_sharded_beamform_gathers_the_full_oracle_volume(split):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, split, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    by = {r[0]: r for r in res}
    _, shape, ref_shape, same_db, same_mask, peak = by["rank0"]
    assert shape == ref_shape and len(shape) == 5
    assert same_db and same_mask        # every voxel and frame, bit for bit
    assert peak > 0.0
    assert by["other"][1] and by["other"][2]   # only the destination rank holds the volume


def test_sharded_beamform_rejects_bad_splits():
    with pytest.raises(ValueError):
        # no process group needed to reject the split name
        from simu_rca_ab_b200 import multi
        multi._n_transmits({})
