"""Parity at the sizes the beamformer is measured on, through the drop-in
``bf_rca`` call (C ABI underneath).

* c0 in full (64+64 probe, 16 plane waves, [512 x 64 x 16 x 1], grid
  64 x 64 x 128, seeded scatterers): reference-compatible tables with the
  reference's quadratic and 6-tap kernels, compounded and per transmit,
  against the reference kernel source compiled for sm_100a without fast math
  (oracle/_ref/librca_ref_gpu_strict.so; frames chunked as
  bfVirtualSourceGeneric_RCA.m:587-594 chunks them) at 1e-4 relative RMS;
  exact tables with Lanczos a = 3 against the FP64 oracle at -60 dB.
* c1 on 2 frames: the row-transmit / column-receive and column-transmit /
  row-receive halves beamformed separately and added, as
  MATLAB/script_All.m:371-382 adds them, FP32 and FP16 storage, against the
  FP64 oracle on random voxels.
* c4 (256+256 probe, f-number 1.0, FP16 storage, 4 frames): the whole
  256 x 256 x 384 volume beamformed, checked against the FP64 oracle on
  voxels drawn from its central 64 x 64 x 96 sub-volume.
* ``BfIQRCA(Raw, pmig)`` (the Python/beamformer/beamformer.py call style,
  pmig keys of beamformer.py:45-111) against ``bf_rca`` on the same
  acquisition, and against the FP64 oracle.
"""
import warnings

import numpy as np
import pytest

from oracle import host as H

pytestmark = pytest.mark.gpu

REF_TOL = 1e-4
DB_TOL = -60.0


@pytest.fixture(scope="module")
def bf(cuda):
    from simu_rca_ab_b200 import beamformer as B
    return B


def _quiet(fn, *a, **k):
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        return fn(*a, **k)


def _flat(db):
    """[Nz, Nx, Ny, T, F] (MATLAB order) -> [F][T][pixel] with the pixel index
    column-major over the grid, as the oracle indexes it."""
    a = db.cpu().numpy() if hasattr(db, "cpu") else np.asarray(db)
    nz, nx, ny, T, F = a.shape
    return a.reshape(nz * nx * ny, T, F, order="F").transpose(2, 1, 0)


def _fp64_group(w, dn_group, g, pix):
    """FP64 oracle (Lanczos a of the workload) of one receive orientation,
    compounded, on the pixel subset: [F][pix]."""
    from simu_rca_ab_b200 import workloads as W
    r = _quiet(H.prepare, W.as_matlab(dn_group), g.Geometry, g.Transmit, w.Param, {"flagMaskTransmit": False})
    f64, m64 = H.run_fp64(r, H.INTERP_LANCZOS, w.lanczos_a, data=dn_group, pix=pix)
    c64, _ = H.compound(f64, m64, True)
    return c64[:, 0]


# --------------------------------------------------------------------------
# c0 in full
# --------------------------------------------------------------------------
@pytest.fixture(scope="module")
def c0_full(cuda):
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c0")
    data = W.channel_data(w, seed=0, device="cuda").cpu().numpy()
    g = w.groups[0]
    return w, W.as_matlab(W.group_data(w, data, 0)), g


@pytest.mark.skipif(not H.have_ref_gpu("strict"), reason="oracle/_ref GPU build missing")
@pytest.mark.parametrize("interp,compound,mask_tx", [("quadratic", True, False), ("quadratic", False, True),
                                                     ("ref6", True, True), ("ref6", False, False)])
def test_c0_ref_compat_matches_reference_kernel(bf, c0_full, interp, compound, mask_tx):
    w, data, g = c0_full
    O = {"flagCompounding": compound, "flagMaskTransmit": mask_tx,
         "flagInterpolationLanczos": interp == "ref6"}
    r = _quiet(H.prepare, data, g.Geometry, g.Transmit, w.Param, O)
    o2, m2 = H.run_ref_gpu(r, "strict")
    c2, mc2 = H.compound(o2, m2, compound)
    db_ref, mk_ref = H.matlab_shape(r, c2, mc2)
    db, mk = _quiet(bf.bf_rca, data, g.Geometry, g.Transmit, w.Param, {**O, "tableMode": "ref_compat"})
    assert db.shape == db_ref.shape == (128, 64, 64, 1 if compound else 16, 1)
    err = H.rel_rms(db, db_ref)
    print(f"c0 REF_COMPAT {interp} compound={compound} mask={mask_tx}: rel RMS {err:.3e} vs the reference "
          f"kernel (sm_100a strict), identical bits {np.array_equal(db, db_ref)}")
    assert err <= REF_TOL
    assert np.allclose(mk, mk_ref, rtol=1e-6, atol=1e-6)


def test_c0_exact_lanczos3_vs_fp64(bf, c0_full):
    from simu_rca_ab_b200 import workloads as W
    w, data, g = c0_full
    db, _ = _quiet(bf.bf_rca, data, g.Geometry, g.Transmit, w.Param, w.Options)
    pix = np.sort(np.random.default_rng(11).choice(w.n_pix, 8192, replace=False))
    dn = np.asarray(data).transpose(3, 2, 1, 0).reshape(w.n_frame, g.n_tx, w.n_ele, w.n_sample)
    ref = _fp64_group(w, dn, g, pix)
    rms, peak = H.error_db(_flat(db)[:, 0, pix], ref)
    print(f"c0 EXACT Lanczos-3 FP32 storage: {rms:.1f} dB RMS, {peak:.1f} dB peak vs FP64 (8192 voxels)")
    assert rms <= DB_TOL


# --------------------------------------------------------------------------
# c1: both receive orientations added, 2 frames
# --------------------------------------------------------------------------
@pytest.fixture(scope="module")
def c1_two_frames(cuda):
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c1", n_frame=2)
    return w, W.channel_data(w, seed=1, device="cuda")


@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_c1_both_orientations_vs_fp64(bf, c1_two_frames, storage):
    import torch
    from simu_rca_ab_b200 import workloads as W
    w, data = c1_two_frames
    total = None
    for gi, g in enumerate(w.groups):
        d = W.group_data(w, data, gi).contiguous()
        if storage == "float16":
            d = d.to(torch.complex32)
        db, _ = _quiet(bf.bf_rca, W.as_matlab(d), g.Geometry, g.Transmit, w.Param, {**w.Options, "storage": storage})
        total = db if total is None else total + db           # script_All.m:382
    out = _flat(total)[:, 0]
    pix = np.sort(np.random.default_rng(12).choice(w.n_pix, 2048, replace=False))
    dn = data.cpu().numpy()
    ref = sum(_fp64_group(w, np.ascontiguousarray(W.group_data(w, dn, gi)), g, pix) for gi, g in enumerate(w.groups))
    rms, peak = H.error_db(out[:, pix], ref)
    print(f"c1 (2 frames, both orientations) {storage}: {rms:.1f} dB RMS, {peak:.1f} dB peak vs FP64 (2048 voxels)")
    assert rms <= DB_TOL


# --------------------------------------------------------------------------
# c4: FP16, whole volume beamformed, central 64 x 64 x 96 sub-volume checked
# --------------------------------------------------------------------------
def test_c4_fp16_subvolume_vs_fp64(bf, cuda):
    import torch
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c4")
    data = W.channel_data(w, seed=4, device="cuda")
    nz, nx, ny = w.grid_shape
    total = None
    for gi, g in enumerate(w.groups):
        d = W.group_data(w, data, gi).contiguous().to(torch.complex32)
        db, _ = _quiet(bf.bf_rca, W.as_matlab(d), g.Geometry, g.Transmit, w.Param, {**w.Options, "storage": "float16"})
        total = db if total is None else total + db
        del d
    assert tuple(total.shape) == (nz, nx, ny, 1, w.n_frame)
    iz, ix, iy = np.meshgrid(np.arange(nz // 2 - 48, nz // 2 + 48), np.arange(nx // 2 - 32, nx // 2 + 32),
                             np.arange(ny // 2 - 32, ny // 2 + 32), indexing="ij")
    sub = (iz + nz * (ix + nx * iy)).ravel()
    assert sub.size == 64 * 64 * 96
    pix = np.sort(np.random.default_rng(13).choice(sub, 2048, replace=False))
    flat = total.permute(4, 3, 2, 1, 0).reshape(w.n_frame, -1)     # [F][pixel], pixel column-major
    out = flat[:, torch.from_numpy(pix).to(flat.device)].cpu().numpy()
    del total, flat
    dn = data.cpu().numpy()
    del data
    ref = sum(_fp64_group(w, np.ascontiguousarray(W.group_data(w, dn, gi)), g, pix) for gi, g in enumerate(w.groups))
    rms, peak = H.error_db(out, ref)
    print(f"c4 FP16 (4 frames, both orientations): {rms:.1f} dB RMS, {peak:.1f} dB peak vs FP64 "
          f"(2048 voxels of the central 64x64x96 sub-volume)")
    assert rms <= DB_TOL


# --------------------------------------------------------------------------
# BfIQRCA(Raw, pmig) against bf_rca
# --------------------------------------------------------------------------
def test_bf_iq_rca_pmig_matches_bf_rca_and_fp64(bf, cuda):
    from simu_rca_ab_b200 import workloads as W
    w = W.get("c0", grid_scale=0.25, n_frame=3)
    g = w.groups[0]
    data = W.channel_data(w, seed=14, device="cuda").cpu().numpy()     # [F][T][E][S]
    F, T, E, S = data.shape
    raw = data.transpose(3, 2, 1, 0).reshape((S, E, T * F), order="F")   # events: transmit fastest
    nz, nx, ny = w.grid_shape
    x = np.asarray(g.Geometry["gridBfX"])[0, :, 0]
    y = np.asarray(g.Geometry["gridBfY"])[0, 0, :]
    z = np.asarray(g.Geometry["gridBfZ"])[:, 0, 0]
    P = w.Param
    pmig = {"c": P["speedOfSound"], "fc": P["demodulationFrequency"], "fsIQ": P["samplingFrequency"],
            "pitch": 0.3e-3, "theta": np.asarray(g.Transmit["thetaY"]), "t0": P["startTime"],
            "dx": x[1] - x[0], "dy": y[1] - y[0], "dz": z[1] - z[0], "Nx": nx, "Ny": ny, "Nz": nz,
            "Xmin": x[0], "Ymin": y[0], "Zmin": z[0], "fnum": P["fnumber"], "order": 2 * w.lanczos_a}
    iq = bf.BfIQRCA(raw, pmig)
    assert iq.shape == (nz, nx, ny, F)
    # the same acquisition through the structs; the pmig grid is rebuilt from
    # Xmin + i dx, so it agrees with the workload's grid to FP64 rounding
    db, _ = _quiet(bf.bf_rca, W.as_matlab(data), g.Geometry, g.Transmit, P, w.Options)
    e = H.rel_rms(iq, db[:, :, :, 0, :])
    print(f"BfIQRCA vs bf_rca: rel RMS {e:.2e}, identical bits {np.array_equal(iq, db[:, :, :, 0, :])}")
    assert e < 1e-6
    # interleaved real input (I, Q along the samples, beamformer.py:118-120)
    inter = np.empty((2 * S, E, T * F), np.float32)
    inter[0::2], inter[1::2] = raw.real, raw.imag
    assert H.rel_rms(bf.BfIQRCA(inter, pmig), iq) < 1e-6
    pix = np.sort(np.random.default_rng(15).choice(w.n_pix, 2048, replace=False))
    ref = _fp64_group(w, data, g, pix)
    rms, _ = H.error_db(iq.reshape(-1, F, order="F").T[:, pix], ref)
    print(f"BfIQRCA vs FP64: {rms:.1f} dB RMS")
    assert rms <= DB_TOL


def test_per_transmit_output_past_2_31_elements(cuda):
    """Per-transmit output (no compounding) of 140 frames of the Doppler
    ensemble geometry: 140 x 11 x 1.47M = 2.27e9 output elements (18 GB),
    past the 2^31 that limits the reference's int indexing and frame chunks
    (bfVirtualSourceGeneric_RCA.m:587-594).  The last 4 frames, whose
    outputs sit past element 2^31, equal the same 4 frames beamformed alone."""
    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import beamformer as B
    from simu_rca_ab_b200 import workloads as W
    from simu_rca_ab_b200.params import normalize
    w = W.get("c2", n_frame=140)
    g0 = w.groups[0]
    data = W.channel_data(w, seed=21, device="cuda").to(torch.complex32)
    eng = B.default_engine()
    geom = _quiet(eng.geometry, normalize(np.zeros(1, np.complex64), g0.Geometry, g0.Transmit, w.Param, w.Options))
    n_tx, n_pix = geom.n_tx, geom.n_pix
    assert 140 * n_tx * n_pix > 2 ** 31

    def run(iq, n_frame):
        out = torch.empty((n_frame, n_tx, n_pix), dtype=torch.complex64, device="cuda")
        a = eng.make_args(geom, iq, iq_dtype=L.IQ_C32, n_sample=w.n_sample, n_frame=n_frame, out=out, mask=None,
                          compound=False, storage=L.STORE_F16)
        eng.run(geom, a)
        torch.cuda.synchronize()
        return out

    big = run(data.contiguous(), 140)
    tail = big[136:].cpu().numpy()
    first = big[0, 0].abs().amax().item()
    del big
    torch.cuda.empty_cache()
    alone = run(data[136:].contiguous(), 4).cpu().numpy()
    rel = H.rel_rms(tail, alone)
    print(f"per-transmit output of 140 frames (2.27e9 elements): last 4 frames vs alone rel {rel:.2e}")
    assert first > 0 and np.isfinite(tail).all() and np.abs(tail).max() > 0
    assert rel < 1e-6
