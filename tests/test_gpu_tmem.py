"""The voxel-blocked kernel with its accumulators in tensor memory (TMEM,
sm_100a) against the same kernel with register accumulators.

Both variants evaluate the same FMA chains in the same order per voxel and
frame, so their outputs are expected to be identical bits: compounded and
per-transmit output, FP32 / FP16 / BF16 storage, frame counts that leave a
frame block partly empty, both receive orientations (two geometries), the
accumulate-into-out mode, frame blocks of 2 to 16.  The TMEM variant also
meets the FP64 oracle on the C2 geometry at the voxel-blocked kernel's own
tolerance; geometries without voxel blocking are refused when it is asked
for by name.
"""
import warnings

import numpy as np
import pytest

from oracle import host as H

pytestmark = pytest.mark.gpu

DB_FP16 = -60.0   # dB RMS vs the FP64 oracle (FP16 storage)


@pytest.fixture(scope="module")
def eng(cuda):
    from simu_rca_ab_b200 import beamformer as B
    e = B.Engine("cuda")
    yield e
    e.close()


def _errcount():
    import ctypes as C
    from simu_rca_ab_b200 import _lib as L
    n = C.c_int64()
    L.check(L.lib().rcabf_take_error_count(C.byref(n)))
    return n.value


def _geom(eng, w, gi):
    from simu_rca_ab_b200.params import normalize
    g = w.groups[gi]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return eng.geometry(normalize(np.zeros(1, np.complex64), g.Geometry, g.Transmit, w.Param, w.Options))


def _run(eng, w, data, gi, *, storage, kernel, compound=True, fb=0, out=None, accumulate=False):
    """Beamforms group gi; returns (out [frame][1 or tx][pix] on the device, plan)."""
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    geom = _geom(eng, w, gi)
    d = W.group_data(w, data, gi).contiguous()
    code = {"float32": L.STORE_F32, "float16": L.STORE_F16, "bfloat16": L.STORE_BF16}[storage]
    iq = d.to(torch.complex32) if storage == "float16" else d
    n_t = 1 if compound else w.groups[gi].n_tx
    if out is None:
        out = torch.empty((w.n_frame, n_t, geom.n_pix), dtype=torch.complex64, device="cuda")
    a = eng.make_args(geom, iq, iq_dtype=L.IQ_C32 if storage == "float16" else L.IQ_C64, n_sample=w.n_sample,
                      n_frame=w.n_frame, out=out, mask=None, compound=compound, storage=code,
                      kernel=kernel, frames_per_block=fb, accumulate=accumulate)
    plan = eng.plan(geom, a)
    eng.run(geom, a)
    torch.cuda.synchronize()
    return out, plan


def _pair(eng, w, data, gi, **kw):
    from simu_rca_ab_b200 import _lib as L
    t, pt = _run(eng, w, data, gi, kernel=L.KERNEL_FUSED_TMEM, **kw)
    r, pr = _run(eng, w, data, gi, kernel=L.KERNEL_FUSED_REGS, **kw)
    assert pt["kernel"] == "fused_voxel_blocked_tmem", pt
    assert pr["kernel"] == "fused_voxel_blocked", pr
    assert pt["frames_per_block"] == pr["frames_per_block"]
    return t, r, pt


@pytest.fixture(scope="module")
def c2_11(cuda):
    """C2 geometry, 11 frames: the full grid (window <= 64 rows, row shift 1)
    and the grid at half resolution (114-row windows, row shift 2; FP16 /
    BF16 register staging holds them only at 8-frame blocks)."""
    from simu_rca_ab_b200 import workloads as W
    out = {}
    for name, scale in (("full", 1.0), ("half", 0.5)):
        w = W.get("c2", n_frame=11, grid_scale=scale)
        out[name] = (w, W.channel_data(w, seed=11, device="cuda"))
    return out


@pytest.fixture(scope="module")
def c1_small(cuda):
    """C1 (two receive orientations, +-10 degree steering), 4 frames; the full
    grid, whose 0.2 mm voxels keep a block's delay spread within 2 rows."""
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c1", n_frame=4)
    return w, W.channel_data(w, seed=3, device="cuda")


@pytest.mark.parametrize("storage", ["float32", "float16", "bfloat16"])
@pytest.mark.parametrize("grid,fb", [("full", 16), ("full", 8), ("half", 8), ("full", 4), ("half", 2)])
@pytest.mark.parametrize("compound", [True, False])
def test_tmem_accumulators_give_the_register_kernels_bits(eng, c2_11, storage, grid, fb, compound):
    import torch
    w, data = c2_11[grid]
    t, r, plan = _pair(eng, w, data, 0, storage=storage, fb=fb, compound=compound)
    same = torch.equal(t, r)
    err = H.rel_rms(t.cpu().numpy(), r.cpu().numpy())
    print(f"c2 (11 frames, {grid} grid) {storage} fb {fb} compound {compound}: identical {same}, "
          f"rel RMS {err:.2e}; plan {plan}")
    assert same
    assert _errcount() == 0


@pytest.mark.parametrize("gi", [0, 1])
def test_tmem_both_receive_orientations(eng, c1_small, gi):
    import torch
    w, data = c1_small
    t, r, plan = _pair(eng, w, data, gi, storage="float32", compound=True)
    print(f"c1 group {gi}: plan {plan}")
    assert torch.equal(t, r)
    assert _errcount() == 0


def test_tmem_accumulate_into_out(eng, c2_11):
    import torch
    from simu_rca_ab_b200 import _lib as L
    w, data = c2_11["full"]
    base, _ = _run(eng, w, data, 0, storage="float16", kernel=L.KERNEL_FUSED_TMEM, fb=16)
    g = torch.Generator(device="cuda").manual_seed(1)
    prior = torch.randn(base.shape, dtype=torch.complex64, device="cuda", generator=g)
    out = prior.clone()
    _run(eng, w, data, 0, storage="float16", kernel=L.KERNEL_FUSED_TMEM, fb=16, out=out, accumulate=True)
    assert torch.equal(out, prior + base)
    assert _errcount() == 0


def test_tmem_vs_fp64_on_c2_geometry(eng, cuda):
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c2", n_frame=8)
    data = W.channel_data(w, seed=5, device="cuda")
    out, plan = _run(eng, w, data, 0, storage="float16", kernel=L.KERNEL_FUSED_TMEM)
    assert plan["kernel"] == "fused_voxel_blocked_tmem" and plan["frames_per_block"] == 16, plan
    out = out[:, 0].cpu().numpy()
    rng = np.random.default_rng(7)
    pix = np.sort(rng.choice(out.shape[1], 1024, replace=False))
    dn = data.cpu().numpy()
    g0 = w.groups[0]
    r = H.prepare(W.as_matlab(dn), g0.Geometry, g0.Transmit, w.Param, {"flagMaskTransmit": False})
    f64, m64 = H.run_fp64(r, H.INTERP_LANCZOS, 4, data=dn, pix=pix)
    c64, _ = H.compound(f64, m64, True)
    rms, peak = H.error_db(out[:, pix], c64[:, 0])
    print(f"TMEM accumulators, FP16 storage, c2 geometry: {rms:.1f} dB RMS, {peak:.1f} dB peak; plan {plan}")
    assert rms <= DB_FP16
    assert _errcount() == 0


def test_tmem_refuses_reference_tables(eng, c2_11):
    from simu_rca_ab_b200 import _lib as L
    w, data = c2_11["full"]
    # the reference-compatible tables have no voxel-blocked kernel
    w2 = type(w)(**{**w.__dict__, "Options": {**w.Options, "tableMode": "ref_compat", "interpolation": "ref6"}})
    with pytest.raises(L.RcabfError) as e:
        _run(eng, w2, data, 0, storage="float32", kernel=L.KERNEL_FUSED_TMEM)
    assert e.value.status == L.ERR_UNSUPPORTED
    assert _errcount() == 0
