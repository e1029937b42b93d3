"""Parity of the CUDA path (through the C ABI) with the oracle.

* REF_COMPAT tables + the reference's interpolation kernels: against the
  reference kernel source compiled for sm_100a without fast math or FMA
  contraction (oracle/_ref/librca_ref_gpu_strict.so), tolerance 1e-4
  relative RMS (expected: identical bits).
* EXACT tables: against the FP64 oracle, tolerance -60 dB RMS for FP32 and
  FP16 storage.  BF16 storage cannot reach -60 dB: rounding the channel data
  to an 8-bit mantissa alone costs about -57 dB.  For it the bar is that the
  kernel adds nothing to that rounding: -60 dB against the FP64 oracle run on
  the BF16-rounded data, and the total within 1 dB of that storage floor.
* Internal consistency: fused vs plain kernel, frame-block sizes, batch vs
  single launches, per-transmit vs compounded, both receive orientations,
  point-list grids, the transmit-cone mask, real (interleaved RF) input.
"""
import warnings

import numpy as np
import pytest

from oracle import host as H
from tests.golden.make_golden import CASES, case, load

pytestmark = pytest.mark.gpu

REF_TOL = 1e-4          # relative RMS, REF_COMPAT vs reference kernel
DB_FP32 = -60.0         # dB RMS vs FP64 oracle
DB_FP16 = -60.0
DB_BF16 = None          # BF16: measured against its storage floor, see _check_bf16


def _bf16_rounded(a):
    """The channel data as BF16 storage holds it (round to nearest even)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a).astype(np.complex64))
    r = torch.view_as_real(t).to(torch.bfloat16).to(torch.float32)
    return torch.view_as_complex(r.contiguous()).numpy()


def _check_bf16(out, ref, ref_rounded, label):
    """BF16 storage: the kernel's error against the FP64 oracle of the
    BF16-rounded data must be below -60 dB (the kernel adds nothing to the
    storage rounding), and its total error within 1 dB of the storage floor
    (the FP64 oracle of the rounded data against that of the original)."""
    floor, _ = H.error_db(ref_rounded, ref)
    own, _ = H.error_db(out, ref_rounded)
    total, peak = H.error_db(out, ref)
    print(f"{label} bfloat16: {total:.1f} dB RMS ({peak:.1f} dB peak) vs FP64; BF16 storage floor {floor:.1f} dB; "
          f"kernel vs FP64 of the rounded data {own:.1f} dB")
    assert own <= -60.0
    assert total <= floor + 1.0


@pytest.fixture(scope="module")
def bf(cuda):
    from simu_rca_ab_b200 import beamformer as B
    return B


def run(bf, data, G, T, P, O, **opts):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return bf.bf_rca(data, G, T, P, {**O, **opts})


def _errcount():
    import ctypes as C
    from simu_rca_ab_b200 import _lib as L
    n = C.c_int64()
    L.check(L.lib().rcabf_take_error_count(C.byref(n)))
    return n.value


# --------------------------------------------------------------------------
# REF_COMPAT vs the reference kernel on the GPU
# --------------------------------------------------------------------------
@pytest.mark.skipif(not H.have_ref_gpu("strict"), reason="oracle/_ref GPU build missing")
@pytest.mark.parametrize("kernel", ["fused", "plain"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_ref_compat_matches_reference_kernel(bf, name, kernel):
    data, G, T, P, O, outs = load(name)
    r = H.prepare(data, G, T, P, O)
    o2, m2 = H.run_ref_gpu(r, "strict")
    c2, mc2 = H.compound(o2, m2, True)
    db_ref, mk_ref = H.matlab_shape(r, c2, mc2)
    db, mk = run(bf, data, G, T, P, O, tableMode="ref_compat", kernel=kernel)
    assert db.shape == db_ref.shape and mk.shape == mk_ref.shape
    err = H.rel_rms(db, db_ref)
    print(f"{name} {kernel}: rel RMS vs reference GPU kernel {err:.3e}, "
          f"identical bits {np.array_equal(db, db_ref)}, vs golden O1 {H.rel_rms(db, outs['dataBf']):.3e}")
    assert err <= REF_TOL
    assert np.allclose(mk, mk_ref, rtol=1e-6, atol=1e-6)
    assert _errcount() == 0


@pytest.mark.skipif(not H.have_ref_gpu("strict"), reason="oracle/_ref GPU build missing")
def test_ref_compat_per_transmit_output(bf):
    data, G, T, P, O, _ = load("ref6_rx_x")
    r = H.prepare(data, G, T, P, {**O, "flagCompounding": False})
    o2, m2 = H.run_ref_gpu(r, "strict")
    db_ref, mk_ref = H.matlab_shape(r, o2, m2)
    db, mk = run(bf, data, G, T, P, O, tableMode="ref_compat", flagCompounding=False)
    assert db.shape == db_ref.shape
    assert H.rel_rms(db, db_ref) <= REF_TOL
    assert np.allclose(mk, mk_ref, rtol=1e-6, atol=1e-6)


@pytest.mark.skipif(not H.have_ref_gpu("fast"), reason="oracle/_ref GPU build missing")
def test_report_reference_fast_math_build(bf):
    """The reference as its wrapper compiles it (-use_fast_math): reported,
    bounded loosely (fast-math trig on ~1e3 rad arguments)."""
    data, G, T, P, O, _ = load("ref6_rx_x")
    r = H.prepare(data, G, T, P, O)
    o_fast, m_fast = H.run_ref_gpu(r, "fast")
    o_str, _ = H.run_ref_gpu(r, "strict")
    db, _ = run(bf, data, G, T, P, O, tableMode="ref_compat", flagCompounding=False)
    db_fast, _ = H.matlab_shape(r, o_fast, m_fast)
    e = H.rel_rms(db, db_fast)
    print(f"REF_COMPAT vs reference -use_fast_math build: {e:.3e}; "
          f"reference fast vs strict: {H.rel_rms(o_fast, o_str):.3e}")
    assert e < 0.2


# --------------------------------------------------------------------------
# EXACT tables vs the FP64 oracle (physical synthetic data)
# --------------------------------------------------------------------------
@pytest.fixture(scope="module")
def c0_small(cuda):
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c0", grid_scale=0.25, n_frame=3)
    data = W.channel_data(w, seed=3, device="cuda").cpu().numpy()
    g = w.groups[0]
    return w, W.as_matlab(W.group_data(w, data, 0)), g.Geometry, g.Transmit, w.Param, w.Options


INTERPS = [("quadratic", 0, H.INTERP_QUAD3), ("ref6", 0, H.INTERP_REF6), ("lanczos", 2, H.INTERP_LANCZOS),
           ("lanczos", 3, H.INTERP_LANCZOS), ("lanczos", 4, H.INTERP_LANCZOS)]


@pytest.mark.parametrize("interp,a,code", INTERPS)
@pytest.mark.parametrize("storage,tol", [("float32", DB_FP32), ("float16", DB_FP16), ("bfloat16", DB_BF16)])
def test_exact_vs_fp64_oracle(bf, c0_small, interp, a, code, storage, tol):
    w, data, G, T, P, O = c0_small
    r = H.prepare(data, G, T, P, O)
    f64, m64 = H.run_fp64(r, code, a, data=np.asarray(data).transpose(3, 2, 1, 0).reshape(
        r.n_frame, r.n_tx, r.n_ch, r.n_sample))
    c64, cm64 = H.compound(f64, m64, True)
    ref, mref = H.matlab_shape(r, c64, cm64)
    db, mk = run(bf, data, G, T, P, O, interpolation=interp, lanczosOrder=max(a, 2), storage=storage)
    assert np.allclose(mk, mref, rtol=1e-5, atol=1e-4)
    if storage == "bfloat16":
        dr = _bf16_rounded(np.asarray(data).transpose(3, 2, 1, 0).reshape(r.n_frame, r.n_tx, r.n_ch, r.n_sample))
        f64r, m64r = H.run_fp64(r, code, a, data=dr)
        refr, _ = H.matlab_shape(r, *H.compound(f64r, m64r, True))
        _check_bf16(db, ref, refr, f"EXACT {interp}{a or ''}")
        return
    rms, peak = H.error_db(db, ref)
    print(f"EXACT {interp}{a or ''} {storage}: {rms:.1f} dB RMS, {peak:.1f} dB peak vs FP64")
    assert rms <= tol


def test_exact_receive_y_points_and_mask(bf):
    for kw in (dict(receive_x=False, mask_tx=False), dict(receive_x=True, mask_tx=False, points=True),
               dict(receive_x=False, mask_tx=True)):
        data, G, T, P, O = case(7, lanczos=False, ns=128, **kw)
        r = H.prepare(data, G, T, P, O)
        f64, m64 = H.run_fp64(r, H.INTERP_QUAD3)
        c, cm = H.compound(f64, m64, True)
        ref, mref = H.matlab_shape(r, c, cm)
        db, mk = run(bf, data, G, T, P, O)
        rms, _ = H.error_db(db, ref)
        print(kw, f"{rms:.1f} dB")
        assert rms <= DB_FP32
        # the cone test compares angles computed in FP64 on both sides
        assert np.allclose(mk, mref, rtol=1e-5, atol=1e-4)


@pytest.mark.parametrize("storage", ["float32", "float16", "bfloat16"])
def test_fused_equals_plain_and_frame_blocks(bf, c0_small, storage):
    """Frame blocking does not change any frame's arithmetic: every fused
    variant gives identical bits.  The plain kernel evaluates the window
    directly instead of through the polyphase table: within 1e-4 (-80 dB)."""
    w, data, G, T, P, O = c0_small
    outs = {}
    for kern in ("fused", "fused_noblock"):
        for fb in (1, 2, 4, 8, 16, 24, 32, 40):
            outs[(kern, fb)], _ = run(bf, data, G, T, P, O, kernel=kern, framesPerBlock=fb, storage=storage)
    plain, _ = run(bf, data, G, T, P, O, kernel="plain", storage=storage)
    # one voxel per thread: table weights, identical bits for every frame block
    for fb in (2, 4, 8, 16, 24, 32, 40):
        assert np.array_equal(outs[("fused_noblock", fb)], outs[("fused_noblock", 1)]), fb
    # voxel-blocked kernel (frame blocks 2, 4, 8, 16): polynomial weights
    for fb in (4, 8, 16):
        assert np.array_equal(outs[("fused", fb)], outs[("fused", 2)]), fb
    assert H.rel_rms(outs[("fused", 8)], outs[("fused_noblock", 8)]) < 1e-4
    if storage == "float32":
        assert H.rel_rms(outs[("fused", 8)], plain) < 1e-4, H.rel_rms(outs[("fused", 8)], plain)
        assert H.rel_rms(outs[("fused_noblock", 8)], plain) < 1e-4
    assert _errcount() == 0


def test_real_rf_input_and_torch_io(bf):
    import torch
    data, G, T, P, O, outs = load("ref6_real_rf")
    db_np, _ = run(bf, data, G, T, P, O, tableMode="ref_compat")
    db_t, mk_t = run(bf, torch.from_numpy(data).cuda(), G, T, P, O, tableMode="ref_compat")
    assert isinstance(db_t, torch.Tensor) and db_t.is_cuda
    assert np.array_equal(db_t.cpu().numpy(), db_np)
    assert H.rel_rms(db_np, outs["dataBf"]) < 0.1


def test_complex32_input_matches_fp16_storage(bf, c0_small):
    import torch
    w, data, G, T, P, O = c0_small
    a, _ = run(bf, data, G, T, P, O, storage="float16")
    t = torch.from_numpy(np.ascontiguousarray(data)).cuda().to(torch.complex32)
    b, _ = run(bf, t, G, T, P, O)
    assert H.rel_rms(b.cpu().numpy(), a) < 1e-6


def test_batch_launch_equals_single_launches(bf, c0_small):
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200.params import normalize
    w, data, G, T, P, O = c0_small
    eng = bf.default_engine()
    acqs = [normalize(data, G, T, P, {**O, "lanczosOrder": a}) for a in (4, 4)]
    acqs[1].fnumber = 2.0
    geoms = [eng.geometry(a) for a in acqs]
    iq = torch.from_numpy(np.ascontiguousarray(np.asarray(data).transpose(3, 2, 1, 0))).cuda()
    iq = iq.reshape(w.n_frame, w.n_tx, w.n_ele, w.n_sample)          # [frame][tx][element][sample]
    singles = [eng.beamform(g, iq, frames_per_block=4)[0].clone() for g in geoms]
    outs, args, wss = [], [], []
    for g in geoms:
        o = torch.empty_like(singles[0])
        a = eng.make_args(g, iq, iq_dtype=L.IQ_C64, n_sample=w.n_sample, n_frame=w.n_frame, out=o,
                          mask=None, compound=True, frames_per_block=4)
        wss.append(torch.empty(eng.workspace_bytes(g, a), dtype=torch.uint8, device="cuda"))
        outs.append(o)
        args.append(a)
    eng.run_batch(geoms, args, wss)
    torch.cuda.synchronize()
    for s, o in zip(singles, outs):
        assert torch.equal(s, o)


def test_bf_iq_rca_pmig_style(bf):
    import torch
    rng = np.random.default_rng(5)
    raw = (rng.normal(size=(128, 32, 6)) + 1j * rng.normal(size=(128, 32, 6))).astype(np.complex64)
    pmig = {"c": 1540, "fc": 7.8e6, "fsIQ": 15.6e6, "pitch": 0.3e-3, "theta": np.deg2rad([-3, 0, 3]),
            "t0": -2e-6, "dx": 0.3e-3, "dz": 0.1e-3, "Nx": 16, "Nz": 24, "Zmin": 3e-3, "fnum": 1.0, "order": 8}
    iq = bf.BfIQRCA(raw, pmig)
    assert iq.shape == (24, 16, 2)
    assert np.isfinite(iq).all() and np.abs(iq).max() > 0


# --------------------------------------------------------------------------
# Full Doppler-ensemble geometry (96 x 96 x 160 voxels, 128 elements,
# 11 transmits), 8 frames: the voxel-blocked kernel against the FP64 oracle
# on random voxels, and against the one-voxel-per-thread kernel.
# --------------------------------------------------------------------------
@pytest.fixture(scope="module")
def c2_small(cuda):
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c2", n_frame=8)
    data = W.channel_data(w, seed=5, device="cuda")
    return w, data


def _beamform_dev(bf, w, data, storage, kernel):
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200.params import normalize
    eng = bf.default_engine()
    g0 = w.groups[0]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        geom = eng.geometry(normalize(np.zeros(1, np.complex64), g0.Geometry, g0.Transmit, w.Param, w.Options))
    code = {"float32": L.STORE_F32, "float16": L.STORE_F16, "bfloat16": L.STORE_BF16}[storage]
    iq = data.contiguous() if storage != "float16" else data.contiguous().to(torch.complex32)
    out = torch.empty((w.n_frame, 1, geom.n_pix), dtype=torch.complex64, device="cuda")
    a = eng.make_args(geom, iq, iq_dtype=L.IQ_C32 if storage == "float16" else L.IQ_C64, n_sample=w.n_sample,
                      n_frame=w.n_frame, out=out, mask=None, compound=True, storage=code,
                      kernel={"fused": L.KERNEL_FUSED, "fused_noblock": L.KERNEL_FUSED_NOBLOCK}[kernel])
    plan = eng.plan(geom, a)
    eng.run(geom, a)
    torch.cuda.synchronize()
    return out[:, 0].cpu().numpy(), plan


@pytest.mark.parametrize("storage,tol", [("float32", DB_FP32), ("float16", DB_FP16), ("bfloat16", DB_BF16)])
def test_voxel_blocked_kernel_vs_fp64_on_c2_geometry(bf, c2_small, storage, tol):
    from simu_rca_ab_b200 import workloads as W
    w, data = c2_small
    out, plan = _beamform_dev(bf, w, data, storage, "fused")
    assert plan["kernel"].startswith("fused_voxel_blocked"), plan
    rng = np.random.default_rng(7)
    pix = np.sort(rng.choice(out.shape[1], 1024, replace=False))
    dn = data.cpu().numpy()
    g0 = w.groups[0]
    r = H.prepare(W.as_matlab(dn), g0.Geometry, g0.Transmit, w.Param, {"flagMaskTransmit": False})
    f64, m64 = H.run_fp64(r, H.INTERP_LANCZOS, 4, data=dn, pix=pix)
    c64, _ = H.compound(f64, m64, True)
    if storage == "bfloat16":
        f64r, m64r = H.run_fp64(r, H.INTERP_LANCZOS, 4, data=_bf16_rounded(dn), pix=pix)
        _check_bf16(out[:, pix], c64[:, 0], H.compound(f64r, m64r, True)[0][:, 0], "voxel-blocked, c2 geometry,")
    else:
        rms, peak = H.error_db(out[:, pix], c64[:, 0])
        print(f"voxel-blocked {storage} on c2 geometry: {rms:.1f} dB RMS, {peak:.1f} dB peak; plan {plan}")
        assert rms <= tol
    if storage == "float32":
        ref, plan2 = _beamform_dev(bf, w, data, storage, "fused_noblock")
        assert plan2["kernel"] == "fused"
        assert H.rel_rms(out, ref) < 1e-4
    assert _errcount() == 0


def test_cuda_graph_capture_replays_the_same_bits(bf, c2_small):
    """The whole beamform call (ingest, window ranges, fused kernel, mask)
    captured once in a CUDA graph and replayed gives the eager call's bits."""
    import ctypes as C
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200.params import normalize
    w, data = c2_small
    eng = bf.default_engine()
    g0 = w.groups[0]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        geom = eng.geometry(normalize(np.zeros(1, np.complex64), g0.Geometry, g0.Transmit, w.Param, w.Options))
    iq = data.contiguous().to(torch.complex32)
    out = torch.empty((w.n_frame, 1, geom.n_pix), dtype=torch.complex64, device="cuda")
    mask = torch.empty((1, geom.n_pix), dtype=torch.float32, device="cuda")
    a = eng.make_args(geom, iq, iq_dtype=L.IQ_C32, n_sample=w.n_sample, n_frame=w.n_frame, out=out, mask=mask,
                      compound=True, storage=L.STORE_F16)
    ws = torch.empty(max(256, eng.workspace_bytes(geom, a)), dtype=torch.uint8, device="cuda")
    eng.run(geom, a, workspace=ws)
    torch.cuda.synchronize()
    ref, ref_mask = out.clone(), mask.clone()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        eng.run(geom, a, workspace=ws)
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        eng.run(geom, a, workspace=ws)
    out.zero_()
    mask.zero_()
    for _ in range(2):
        g.replay()
    torch.cuda.synchronize()
    assert torch.equal(out, ref) and torch.equal(mask, ref_mask)
    n = C.c_int64()
    L.check(L.lib().rcabf_take_error_count(C.byref(n)))
    assert n.value == 0


def test_autotune_keeps_the_fastest_choice_and_the_result(bf, c2_small):
    """rcabf_autotune times tile shapes / frame blocks / kernel families on
    the C2 geometry and later plans use its choice; the tuned result agrees
    with the planner's own within the cross-kernel tolerance."""
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200.params import normalize
    w, data = c2_small
    eng = bf.Engine("cuda")          # a geometry of its own: the tuned choice stays here
    g0 = w.groups[0]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        geom = eng.geometry(normalize(np.zeros(1, np.complex64), g0.Geometry, g0.Transmit, w.Param, w.Options))
    iq = data.contiguous().to(torch.complex32)

    def call():
        out = torch.empty((w.n_frame, 1, geom.n_pix), dtype=torch.complex64, device="cuda")
        a = eng.make_args(geom, iq, iq_dtype=L.IQ_C32, n_sample=w.n_sample, n_frame=w.n_frame, out=out,
                          mask=None, compound=True, storage=L.STORE_F16)
        return out, a

    before, a = call()
    plan0 = eng.plan(geom, a)
    eng.run(geom, a)
    torch.cuda.synchronize()
    scratch, a2 = call()
    res = eng.autotune(geom, a2, iters=1)
    assert res["candidates"] >= 2 and res["best_ms"] <= res["default_ms"] + 1e-6
    after, a3 = call()
    plan1 = eng.plan(geom, a3)
    assert plan1["frames_per_block"] == res["frames_per_block"]
    assert plan1["tile"] == [res["tile_u"], res["tile_v"], res["tile_z"]]
    if res["tensor_core"]:
        assert plan1["kernel"] == "fused_tensor_core"
    else:
        assert plan1["kernel"] == {0: "fused", 1: "fused_voxel_blocked", 2: "fused_voxel_blocked_tmem"}[
            res["voxel_blocked"]]
    eng.run(geom, a3)
    torch.cuda.synchronize()
    assert H.rel_rms(after.cpu().numpy(), before.cpu().numpy()) < 1e-4
    if plan1["kernel"] == plan0["kernel"]:
        if plan1["tile"] == plan0["tile"]:
            assert torch.equal(after, before)   # the frame block changes no arithmetic
        else:
            # the tile sets the transmit order of the sums (voxel-blocked
            # kernel): FP32 rounding only
            assert H.rel_rms(after.cpu().numpy(), before.cpu().numpy()) < 1e-5
    print("autotune", res, "default plan", plan0)
    eng.close()
