"""The tensor-core kernel (fused_tc_kernel.cuh, tcgen05.mma) through the C ABI:
against the FP64 oracle (-60 dB RMS), against the voxel-blocked SIMT kernel on
the same FP16 slabs, over both weight precisions (hi + remainder FP16 terms,
single FP16), the interpolation kernels, frame blocks, partial tiles at the
grid edges, accumulation into the output, and the cases it declines."""
import ctypes as C
import warnings

import numpy as np
import pytest

from oracle import host as H

pytestmark = pytest.mark.gpu

DB_TOL = -60.0


def _errcount():
    from simu_rca_ab_b200 import _lib as L
    n = C.c_int64()
    L.check(L.lib().rcabf_take_error_count(C.byref(n)))
    return n.value


def _setup(w, seed):
    import torch
    from simu_rca_ab_b200 import beamformer as B
    from simu_rca_ab_b200 import workloads as W
    from simu_rca_ab_b200.params import normalize
    g0 = w.groups[0]
    data = W.channel_data(w, seed=seed, device="cuda")
    eng = B.default_engine()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        geom = eng.geometry(normalize(np.zeros(1, np.complex64), g0.Geometry, g0.Transmit, w.Param, w.Options))
    return data, eng, geom, data.contiguous().to(torch.complex32)


def _run(w, eng, geom, iq, kernel, compound=True, accumulate=False, out=None, storage=None):
    import torch
    from simu_rca_ab_b200 import _lib as L
    if out is None:
        out = torch.empty((w.n_frame, 1 if compound else geom.n_tx, geom.n_pix), dtype=torch.complex64,
                          device="cuda")
    a = eng.make_args(geom, iq, iq_dtype=L.IQ_C32 if iq.dtype == torch.complex32 else L.IQ_C64,
                      n_sample=w.n_sample, n_frame=w.n_frame, out=out, mask=None, compound=compound,
                      storage=L.STORE_F16 if storage is None else storage, kernel=kernel, accumulate=accumulate)
    plan = eng.plan(geom, a)
    eng.run(geom, a)
    torch.cuda.synchronize()
    return out, plan


def _fp64(w, data, pix):
    from simu_rca_ab_b200 import workloads as W
    g0 = w.groups[0]
    dn = data.cpu().numpy()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        r = H.prepare(W.as_matlab(dn), g0.Geometry, g0.Transmit, w.Param, {"flagMaskTransmit": False})
    code = {"quadratic": H.INTERP_QUAD3, "ref6": H.INTERP_REF6}.get(w.Options.get("interpolation"), H.INTERP_LANCZOS)
    f64, m64 = H.run_fp64(r, code, w.lanczos_a, data=dn, pix=pix)
    return H.compound(f64, m64, True)[0][:, 0]


@pytest.fixture(scope="module")
def c2_40(cuda):
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c2", n_frame=40)
    return (w,) + _setup(w, 5)


@pytest.mark.parametrize("kname", ["tc", "tc16"])
def test_tensor_core_kernel_vs_fp64_and_simt_on_the_ensemble_geometry(c2_40, kname):
    from simu_rca_ab_b200 import _lib as L
    w, data, eng, geom, iq = c2_40
    kern = {"tc": L.KERNEL_FUSED_TC, "tc16": L.KERNEL_FUSED_TC_FP16W}[kname]
    out, plan = _run(w, eng, geom, iq, kern)
    assert plan["kernel"].startswith("fused_tensor_core"), plan
    assert _errcount() == 0
    ref_simt, plan_s = _run(w, eng, geom, iq, L.KERNEL_FUSED_TMEM)
    assert plan_s["kernel"] == "fused_voxel_blocked_tmem"
    o = out[:, 0].cpu().numpy()
    pix = np.sort(np.random.default_rng(17).choice(geom.n_pix, 1024, replace=False))
    rms, peak = H.error_db(o[:, pix], _fp64(w, data, pix))
    rel = H.rel_rms(o, ref_simt[:, 0].cpu().numpy())
    print(f"{kname} (c2 geometry, 40 frames, plan {plan}): {rms:.1f} dB RMS, {peak:.1f} dB peak vs FP64; "
          f"rel RMS vs the SIMT kernel {rel:.2e}")
    assert rms <= DB_TOL
    # both round the samples alike; the hi + remainder weights (~22 bits) and
    # the tensor cores' FP32 accumulation differ from the SIMT kernel's FP32
    # arithmetic by ~5e-5 (-86 dB), single FP16 weights by ~2e-4 (-74 dB)
    assert rel < (2e-4 if kname == "tc" else 1e-3)
    assert np.isfinite(o).all()


@pytest.mark.parametrize("kname,n_frame", [("tc", 100), ("tc16", 100), ("tc", 33), ("tc", 300), ("tc", 200),
                                           ("tc16", 232)])
def test_frame_blocks_and_padding(cuda, kname, n_frame):
    """One block of 104 frames for 100 frames (either weight precision), a
    block padded from 33 to 40 frames, two blocks of 152 frames for 300, and
    the widest blocks (200 frames with hi + remainder weights, 232 with single
    FP16 weights: accumulators wider than one MMA's 256 columns) give every
    frame the SIMT kernel's value."""
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c2", n_frame=n_frame)
    data, eng, geom, iq = _setup(w, 8)
    kern = {"tc": L.KERNEL_FUSED_TC, "tc16": L.KERNEL_FUSED_TC_FP16W}[kname]
    out, plan = _run(w, eng, geom, iq, kern)
    ref, _ = _run(w, eng, geom, iq, L.KERNEL_FUSED_TMEM)
    print(kname, n_frame, plan)
    assert plan["frames_per_block"] == {100: 104, 33: 40, 300: 152, 200: 200, 232: 232}[n_frame]
    assert _errcount() == 0
    rel = H.rel_rms(out.cpu().numpy(), ref.cpu().numpy())
    assert rel < (2e-4 if kname == "tc" else 1e-3), rel
    # every frame carries signal (no frame of a block left out)
    per_frame = out[:, 0].abs().amax(dim=1).cpu().numpy()
    assert (per_frame > 0).all()


@pytest.mark.parametrize("interp,a", [("quadratic", 0), ("ref6", 0), ("lanczos", 2), ("lanczos", 3)])
def test_interpolation_kernels_and_partial_tiles(cuda, interp, a):
    """Every interpolation kernel, on the 64 x 64 x 128 grid of the 64+64
    probe cut to 60 x 60 lateral voxels (partial tiles along both lateral
    axes), against the FP64 oracle."""
    import numpy as np
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c0", n_frame=32)
    g0 = w.groups[0]
    for k in ("gridBfX", "gridBfY", "gridBfZ"):
        g0.Geometry[k] = np.ascontiguousarray(np.asarray(g0.Geometry[k])[:, :60, :60])
    w.grid_shape = (w.grid_shape[0], 60, 60)
    w.Options = {**w.Options, "interpolation": interp, "lanczosOrder": max(a, 2)}
    if a:
        w.lanczos_a = a
    data, eng, geom, iq = _setup(w, 9)
    out, plan = _run(w, eng, geom, iq, L.KERNEL_FUSED_TC)
    assert plan["kernel"] == "fused_tensor_core", plan
    assert _errcount() == 0
    o = out[:, 0].cpu().numpy()
    pix = np.sort(np.random.default_rng(19).choice(geom.n_pix, 1024, replace=False))
    rms, _ = H.error_db(o[:, pix], _fp64(w, data, pix))
    print(f"tensor-core {interp}{a or ''} on a 60x60x128 grid (plan {plan}): {rms:.1f} dB vs FP64")
    assert rms <= DB_TOL


def test_accumulate_adds_into_the_output(c2_40):
    import torch
    from simu_rca_ab_b200 import _lib as L
    w, data, eng, geom, iq = c2_40
    once, _ = _run(w, eng, geom, iq, L.KERNEL_FUSED_TC)
    twice, _ = _run(w, eng, geom, iq, L.KERNEL_FUSED_TC)
    _run(w, eng, geom, iq, L.KERNEL_FUSED_TC, accumulate=True, out=twice)
    assert torch.equal(twice, 2 * once)


def test_declined_cases(c2_40):
    """Per-transmit output and FP32 storage are not tensor-core work: the call
    is refused (RCABF_ERR_UNSUPPORTED)."""
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    w, data, eng, geom, iq = c2_40
    with pytest.raises(Exception):
        _run(w, eng, geom, iq, L.KERNEL_FUSED_TC, compound=False)
    with pytest.raises(Exception):
        _run(w, eng, geom, data.contiguous(), L.KERNEL_FUSED_TC, storage=L.STORE_F32)
    # by name it also takes fewer than 32 frames (one block padded to 32);
    # the planner's own choice leaves those to the SIMT kernels
    w8 = W.get("c2", n_frame=8)
    out8, plan8 = _run(w8, eng, geom, iq[:8].contiguous(), L.KERNEL_FUSED_TC)
    assert plan8["kernel"] == "fused_tensor_core" and plan8["frames_per_block"] == 32
    ref8, plan_auto = _run(w8, eng, geom, iq[:8].contiguous(), L.KERNEL_AUTO)
    assert not plan_auto["kernel"].startswith("fused_tensor_core")
    assert H.rel_rms(out8.cpu().numpy(), ref8.cpu().numpy()) < 2e-4
    assert _errcount() == 0


def test_bf16_slabs_on_the_tensor_cores(c2_40):
    """BF16 slabs (the Doppler ensemble's other storage): BF16 x BF16 MMAs
    with hi + remainder BF16 weights (~16 bits).  Against the SIMT kernel on
    the same BF16 slabs, and against the FP64 oracle at BF16's storage floor
    (-45 dB, as the SIMT BF16 tests); single-term weights are refused for
    BF16 (8 bits would not do)."""
    from simu_rca_ab_b200 import _lib as L
    w, data, eng, geom, iq = c2_40
    x = data.contiguous()
    out, plan = _run(w, eng, geom, x, L.KERNEL_AUTO, storage=L.STORE_BF16)
    assert plan["kernel"] == "fused_tensor_core", plan
    assert _errcount() == 0
    ref, plan_s = _run(w, eng, geom, x, L.KERNEL_FUSED_TMEM, storage=L.STORE_BF16)
    assert plan_s["kernel"] == "fused_voxel_blocked_tmem"
    o = out[:, 0].cpu().numpy()
    rel = H.rel_rms(o, ref[:, 0].cpu().numpy())
    pix = np.sort(np.random.default_rng(23).choice(geom.n_pix, 1024, replace=False))
    rms, _ = H.error_db(o[:, pix], _fp64(w, data, pix))
    print(f"BF16 slabs, tensor cores: {rms:.1f} dB vs FP64; rel RMS vs the SIMT kernel {rel:.2e}")
    assert rel < 2e-4
    assert rms <= -45.0
    with pytest.raises(Exception):
        _run(w, eng, geom, x, L.KERNEL_FUSED_TC_FP16W, storage=L.STORE_BF16)
