"""rcabf_beamform_noalloc: the fused path with its workspace in a static device
array (no allocation per call), through the C ABI, against rcabf_beamform.

The entry point serves callers that may not call cudaMalloc (acquisition
loops that must not stall on an allocation, hosts that own the device memory
pool); these tests check that it gives the bits of the allocating entry point
on two calls in a row (a stale workspace would show on the second) and that
it rejects what it cannot hold.

The file name sorts last so that the static region is exercised both in a
fresh process (run alone) and after every other test of the suite.
"""
import ctypes as C
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOALLOC_MAX = 64 << 20   # RCABF_NOALLOC_WORKSPACE_BYTES


def _geometry(w):
    from simu_rca_ab_b200 import beamformer as B
    from simu_rca_ab_b200.params import normalize
    eng = B.default_engine()
    g0 = w.groups[0]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        geom = eng.geometry(normalize(np.zeros(1, np.complex64), g0.Geometry, g0.Transmit, w.Param, w.Options))
    return eng, geom


def _args(eng, geom, w, iq, out, mask, code):
    from simu_rca_ab_b200 import _lib as L
    return eng.make_args(geom, iq, iq_dtype=L.IQ_C32 if code == L.STORE_F16 else L.IQ_C64,
                         n_sample=w.n_sample, n_frame=w.n_frame, out=out, mask=mask, compound=True,
                         storage=code, kernel=L.KERNEL_FUSED)


def _noalloc(geom, a):
    import torch
    from simu_rca_ab_b200 import _lib as L
    a.workspace = None
    a.workspace_bytes = 0
    st = torch.cuda.current_stream().cuda_stream
    return L.lib().rcabf_beamform_noalloc(C.c_void_p(geom.ptr), C.byref(a), C.c_void_p(st))


@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_noalloc_matches_beamform_on_two_calls_in_a_row(cuda, storage):
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c0", n_frame=4)
    eng, geom = _geometry(w)
    code = {"float32": L.STORE_F32, "float16": L.STORE_F16}[storage]
    dt = torch.complex32 if storage == "float16" else torch.complex64
    # two different acquisitions, so a stale workspace would show
    iqs = [W.channel_data(w, seed=s, device=cuda).contiguous().to(dt) for s in (21, 22)]
    probe = _args(eng, geom, w, iqs[0], torch.empty((w.n_frame, 1, geom.n_pix), dtype=torch.complex64,
                                                    device=cuda), None, code)
    assert eng.plan(geom, probe)["kernel"].startswith("fused")
    assert 0 < eng.workspace_bytes(geom, probe) <= NOALLOC_MAX
    for iq in iqs:
        out_ref = torch.empty((w.n_frame, 1, geom.n_pix), dtype=torch.complex64, device=cuda)
        mask_ref = torch.empty((1, geom.n_pix), dtype=torch.float32, device=cuda)
        eng.run(geom, _args(eng, geom, w, iq, out_ref, mask_ref, code))
        out = torch.full_like(out_ref, float("nan"))
        mask = torch.full_like(mask_ref, float("nan"))
        L.check(_noalloc(geom, _args(eng, geom, w, iq, out, mask, code)), "rcabf_beamform_noalloc")
        torch.cuda.synchronize()
        assert torch.equal(out, out_ref)
        assert torch.equal(mask, mask_ref)
        assert float(out_ref.abs().max()) > 0.0
    n = C.c_int64()
    L.check(L.lib().rcabf_take_error_count(C.byref(n)))
    assert n.value == 0


def test_noalloc_call_leaves_device_free_memory_unchanged(cuda):
    """After the first call on the device (which looks up the static array
    and, with lazy module loading, loads the module that holds it), further
    calls change nothing in the device's free memory: they allocate nothing."""
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c0", n_frame=4)
    eng, geom = _geometry(w)
    iq = W.channel_data(w, seed=23, device=cuda).contiguous().to(torch.complex32)
    out = torch.empty((w.n_frame, 1, geom.n_pix), dtype=torch.complex64, device=cuda)
    mask = torch.empty((1, geom.n_pix), dtype=torch.float32, device=cuda)
    args = [_args(eng, geom, w, iq, out, mask, L.STORE_F16) for _ in range(4)]
    L.check(_noalloc(geom, args[0]), "rcabf_beamform_noalloc (set-up call)")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for a in args[1:]:
        L.check(_noalloc(geom, a), "rcabf_beamform_noalloc")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes across noalloc calls"
    assert float(out.abs().max()) > 0.0


def test_noalloc_rejects_plans_larger_than_the_static_workspace(cuda):
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c0", n_frame=24)
    eng, geom = _geometry(w)
    iq = torch.zeros((w.n_frame, geom.n_tx, geom.n_ele, w.n_sample), dtype=torch.complex64, device=cuda)
    out = torch.zeros((w.n_frame, 1, geom.n_pix), dtype=torch.complex64, device=cuda)
    a = _args(eng, geom, w, iq, out, None, L.STORE_F32)
    assert eng.workspace_bytes(geom, a) > NOALLOC_MAX
    st = _noalloc(geom, a)
    torch.cuda.synchronize()
    assert st == 103   # RCABF_ERR_WORKSPACE_TOO_SMALL
    assert "static workspace" in L.lib().rcabf_last_error().decode()
    assert float(out.abs().max()) == 0.0


def test_noalloc_rejects_the_plain_kernel(cuda):
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c0", n_frame=1)
    eng, geom = _geometry(w)
    iq = torch.zeros((1, geom.n_tx, geom.n_ele, w.n_sample), dtype=torch.complex64, device=cuda)
    out = torch.zeros((1, 1, geom.n_pix), dtype=torch.complex64, device=cuda)
    a = _args(eng, geom, w, iq, out, None, L.STORE_F32)
    a.kernel = L.KERNEL_PLAIN
    assert _noalloc(geom, a) == 102   # RCABF_ERR_UNSUPPORTED
