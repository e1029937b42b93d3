"""The serving loop (rcabf_server_*): continuous batching on one device.

* every request of a mixed burst (three probe/grid/transmit sets, 1-6
  frames, FP32 and FP16 storage) gives exactly the bits it gives alone;
* requests that share a kernel variant are fused into one launch;
* admission: a request larger than the whole HBM budget is refused, a full
  queue answers BUSY, a wait that runs out answers TIMEOUT;
* requests accumulating into one output apply in arrival order.
"""
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _geom(eng, w, gi=0):
    from simu_rca_ab_b200.params import normalize
    g = w.groups[gi]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return eng.geometry(normalize(np.zeros(1, np.complex64), g.Geometry, g.Transmit, w.Param, w.Options))


def _request(eng, w, gi, seed, storage, dev):
    """(geometry, iq, n_sample, n_frame, iq_dtype, storage code) of one request."""
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    data = W.channel_data(w, seed=seed, device=dev)
    iq = W.group_data(w, data, gi).contiguous()
    if storage == "float16":
        iq = iq.to(torch.complex32)
    code = {"float32": L.STORE_F32, "float16": L.STORE_F16}[storage]
    return _geom(eng, w, gi), iq, w.n_sample, w.n_frame, L.IQ_C32 if storage == "float16" else L.IQ_C64, code


def _alone(eng, req):
    import torch
    g, iq, ns, nf, iqd, code = req
    out = torch.empty((nf, 1, g.n_pix), dtype=torch.complex64, device=iq.device)
    mask = torch.empty((1, g.n_pix), dtype=torch.float32, device=iq.device)
    eng.run(g, eng.make_args(g, iq, iq_dtype=iqd, n_sample=ns, n_frame=nf, out=out, mask=mask, compound=True,
                             storage=code))
    torch.cuda.synchronize()
    return out, mask


def test_mixed_burst_gives_the_bits_of_each_request_alone(cuda):
    import torch
    from simu_rca_ab_b200 import beamformer as B
    from simu_rca_ab_b200 import workloads as W
    from simu_rca_ab_b200.server import Server
    eng = B.default_engine()
    rng = np.random.default_rng(0)
    shapes = [("c0", 0.25, 0), ("c0", 0.5, 0), ("c1", 0.25, 1)]
    reqs = []
    for k in range(12):
        name, scale, gi = shapes[k % 3]
        w = W.get(name, grid_scale=scale, n_frame=int(rng.integers(1, 7)))
        storage = "float16" if k % 2 else "float32"
        reqs.append(_request(eng, w, gi, seed=100 + k, storage=storage, dev=cuda))
    refs = [_alone(eng, r) for r in reqs]
    with Server(eng, 2 << 30, n_streams=3, max_batch=8) as srv:
        outs, tickets = [], []
        for g, iq, ns, nf, iqd, code in reqs:
            out = torch.full((nf, 1, g.n_pix), float("nan"), dtype=torch.complex64, device=cuda)
            mask = torch.full((1, g.n_pix), float("nan"), dtype=torch.float32, device=cuda)
            tickets.append(srv.submit_beamform(g, iq, out, iq_dtype=iqd, n_sample=ns, n_frame=nf, mask=mask,
                                               storage=code))
            outs.append((out, mask))
        for t in tickets:
            assert srv.wait(t, 120.0) == 0
        st = srv.stats()
    torch.cuda.synchronize()
    for (o, m), (ro, rm) in zip(outs, refs):
        assert torch.equal(o, ro)
        assert torch.equal(m, rm)
    assert st.completed == len(reqs) and st.rejected == 0
    assert 1 <= st.launches <= len(reqs)
    assert 0 < st.p50_ms <= st.p99_ms <= st.max_ms
    assert st.units_done > 0 and st.arena_peak_bytes > 0
    print(f"mixed burst: {st.launches} launches for {len(reqs)} requests, p50 {st.p50_ms:.2f} ms, "
          f"p99 {st.p99_ms:.2f} ms")


def test_batching_window_fuses_requests_and_wait_times_out(cuda):
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import beamformer as B
    from simu_rca_ab_b200 import workloads as W
    from simu_rca_ab_b200.server import Server
    eng = B.default_engine()
    w = W.get("c0", grid_scale=0.5, n_frame=2)
    reqs = [_request(eng, w, 0, seed=200 + k, storage="float32", dev=cuda) for k in range(3)]
    refs = [_alone(eng, r)[0] for r in reqs]
    with Server(eng, 1 << 30, n_streams=2, max_batch=8, batch_window_us=300_000) as srv:
        outs, tickets = [], []
        for g, iq, ns, nf, iqd, code in reqs:
            out = torch.empty((nf, 1, g.n_pix), dtype=torch.complex64, device=cuda)
            tickets.append(srv.submit_beamform(g, iq, out, iq_dtype=iqd, n_sample=ns, n_frame=nf, storage=code))
            outs.append(out)
        # the window holds the requests for 0.3 s: an immediate wait runs out
        with pytest.raises(L.RcabfError) as ex:
            srv.wait(tickets[0], 0.0)
        assert ex.value.status == L.ERR_TIMEOUT
        assert srv.poll(tickets[1]) is None
        for t in tickets:
            assert srv.wait(t, 60.0) == 0
        st = srv.stats()
    assert st.launches == 1          # one persistent launch for the three requests
    for o, r in zip(outs, refs):
        assert torch.equal(o, r)


def test_admission_budget_and_full_queue(cuda):
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import beamformer as B
    from simu_rca_ab_b200 import workloads as W
    from simu_rca_ab_b200.server import Server
    eng = B.default_engine()
    small = _request(eng, W.get("c0", grid_scale=0.25, n_frame=1), 0, seed=300, storage="float32", dev=cuda)
    big = _request(eng, W.get("c0", grid_scale=0.25, n_frame=8), 0, seed=301, storage="float32", dev=cuda)

    def args(req, out):
        g, iq, ns, nf, iqd, code = req
        return eng.make_args(g, iq, iq_dtype=iqd, n_sample=ns, n_frame=nf, out=out, mask=None, compound=True,
                             storage=code)

    g = small[0]
    need_small = eng.workspace_bytes(g, args(small, torch.empty((1, 1, g.n_pix), dtype=torch.complex64,
                                                                 device=cuda)))
    out_big = torch.empty((8, 1, g.n_pix), dtype=torch.complex64, device=cuda)
    need_big = eng.workspace_bytes(g, args(big, out_big))
    assert need_big > need_small
    budget = (need_small + need_big) // 2
    with Server(eng, budget, n_streams=1, max_queue=2, batch_window_us=300_000) as srv:
        with pytest.raises(L.RcabfError) as ex:
            srv.submit(g, args(big, out_big))
        assert ex.value.status == L.ERR_OOM_ADMISSION
        outs = [torch.empty((1, 1, g.n_pix), dtype=torch.complex64, device=cuda) for _ in range(3)]
        t0 = srv.submit(g, args(small, outs[0]), keep=(outs[0],))
        t1 = srv.submit(g, args(small, outs[1]), keep=(outs[1],))
        with pytest.raises(L.RcabfError) as ex:   # the window still holds the first two
            srv.submit(g, args(small, outs[2]))
        assert ex.value.status == L.ERR_BUSY
        assert srv.wait(t0, 60.0) == 0 and srv.wait(t1, 60.0) == 0
        st = srv.stats()
    ref = _alone(eng, small)[0]
    assert torch.equal(outs[0], ref) and torch.equal(outs[1], ref)
    assert st.rejected == 2 and st.completed == 2


def test_accumulating_requests_apply_in_arrival_order(cuda):
    import torch
    from simu_rca_ab_b200 import beamformer as B
    from simu_rca_ab_b200 import workloads as W
    from simu_rca_ab_b200.server import Server
    eng = B.default_engine()
    w = W.get("c1", grid_scale=0.25, n_frame=2)
    from simu_rca_ab_b200 import _lib as L
    data = W.channel_data(w, seed=400, device=cuda)
    geoms = [_geom(eng, w, gi) for gi in range(len(w.groups))]
    iqs = [W.group_data(w, data, gi).contiguous() for gi in range(len(w.groups))]
    ref = torch.empty((w.n_frame, 1, geoms[0].n_pix), dtype=torch.complex64, device=cuda)
    for gi, g in enumerate(geoms):    # the two transmit groups summed in order, one call each
        eng.run(g, eng.make_args(g, iqs[gi], iq_dtype=L.IQ_C64, n_sample=w.n_sample, n_frame=w.n_frame, out=ref,
                                 mask=None, compound=True, accumulate=gi > 0))
    torch.cuda.synchronize()
    out = torch.full_like(ref, float("nan"))
    with Server(eng, 1 << 30, n_streams=4) as srv:
        ts = [srv.submit_beamform(g, iqs[gi], out, iq_dtype=L.IQ_C64, n_sample=w.n_sample, n_frame=w.n_frame,
                                  accumulate=gi > 0) for gi, g in enumerate(geoms)]
        for t in ts:
            assert srv.wait(t, 60.0) == 0
    assert torch.equal(out, ref)
