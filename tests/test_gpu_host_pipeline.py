"""rcabf_beamform_host: channel data and output in host memory, frames in
chunks whose copies overlap the beamforming.  Its output must be the bits
rcabf_beamform gives on device copies of the same buffers, whatever the
chunking (whole frame blocks or not), with accumulation, per-transmit
output and the mask (computed once, with the first chunk)."""
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(cuda):
    import torch
    from simu_rca_ab_b200 import beamformer as B
    from simu_rca_ab_b200 import workloads as W
    from simu_rca_ab_b200.params import normalize
    w = W.get("c2", n_frame=40, grid_scale=0.5)
    data = W.channel_data(w, seed=9, device="cuda")
    eng = B.Engine("cuda")
    g0 = w.groups[0]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        geom = eng.geometry(normalize(np.zeros(1, np.complex64), g0.Geometry, g0.Transmit, w.Param, w.Options))
    yield w, data.to(torch.complex32).contiguous(), eng, geom
    eng.close()


def _device(setup, compound=True, prior=None):
    import torch
    from simu_rca_ab_b200 import _lib as L
    w, iq, eng, geom = setup
    T = 1 if compound else geom.n_tx
    out = prior.cuda().clone() if prior is not None else torch.empty((w.n_frame, T, geom.n_pix),
                                                                     dtype=torch.complex64, device="cuda")
    mask = torch.zeros((T, geom.n_pix), dtype=torch.float32, device="cuda")
    a = eng.make_args(geom, iq, iq_dtype=L.IQ_C32, n_sample=w.n_sample, n_frame=w.n_frame, out=out, mask=mask,
                      compound=compound, storage=L.STORE_F16, accumulate=prior is not None)
    eng.run(geom, a)
    torch.cuda.synchronize()
    return out.cpu(), mask.cpu()


def _host(setup, chunk, compound=True, prior=None):
    import torch
    from simu_rca_ab_b200 import _lib as L
    w, iq, eng, geom = setup
    T = 1 if compound else geom.n_tx
    iq_h = iq.cpu().pin_memory()
    out_h = torch.empty((w.n_frame, T, geom.n_pix), dtype=torch.complex64).pin_memory()
    if prior is not None:
        out_h.copy_(prior)
    mask = torch.zeros((T, geom.n_pix), dtype=torch.float32, device="cuda")
    a = eng.make_args(geom, iq_h, iq_dtype=L.IQ_C32, n_sample=w.n_sample, n_frame=w.n_frame, out=out_h, mask=mask,
                      compound=compound, storage=L.STORE_F16, accumulate=prior is not None, host=True)
    eng.run_host(geom, a, frames_per_chunk=chunk)
    torch.cuda.synchronize()
    return out_h.clone(), mask.cpu()


@pytest.mark.parametrize("chunk", [0, 16, 24, 7, 40])
def test_host_pipeline_gives_the_device_call_bits(setup, chunk):
    import torch
    ref, ref_mask = _device(setup)
    got, mask = _host(setup, chunk)
    assert torch.equal(got, ref) and torch.equal(mask, ref_mask)


def test_host_pipeline_per_transmit_and_accumulate(setup):
    import torch
    w, iq, eng, geom = setup
    g = torch.Generator().manual_seed(3)
    prior = torch.randn((w.n_frame, geom.n_tx, geom.n_pix), dtype=torch.complex64, generator=g)
    ref, ref_mask = _device(setup, compound=False, prior=prior)
    got, mask = _host(setup, 16, compound=False, prior=prior)
    assert torch.equal(got, ref) and torch.equal(mask, ref_mask)


def test_host_pipeline_refusals(setup):
    import ctypes as C
    import torch
    from simu_rca_ab_b200 import _lib as L
    w, iq, eng, geom = setup
    iq_h = iq.cpu().pin_memory()
    out_h = torch.empty((w.n_frame * geom.n_ele, geom.n_tx, geom.n_pix), dtype=torch.complex64).pin_memory()
    a = eng.make_args(geom, iq_h, iq_dtype=L.IQ_C32, n_sample=w.n_sample, n_frame=w.n_frame, out=out_h, mask=None,
                      compound=False, storage=L.STORE_F16, per_channel=True, host=True)
    n = C.c_size_t()
    assert L.lib().rcabf_beamform_host_workspace_size(C.c_void_p(geom.ptr), C.byref(a), 0, C.byref(n)) == 102
    a = eng.make_args(geom, iq_h, iq_dtype=L.IQ_C32, n_sample=w.n_sample, n_frame=w.n_frame, out=out_h, mask=None,
                      compound=True, storage=L.STORE_F16, host=True)
    ws = torch.empty(1024, dtype=torch.uint8, device="cuda")
    a.workspace, a.workspace_bytes = ws.data_ptr(), ws.numel()
    assert L.lib().rcabf_beamform_host(C.c_void_p(geom.ptr), C.byref(a), 0, None) == 103
