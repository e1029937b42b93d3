"""The reference's aberration-law and no-sum beamformer variants on the GPU.

* ``Param.AbLawRx`` per element (Hyp1_save/..._ab_1.cu:306-311) or per
  (transmit, element) (Hyp2/..._ab_2.cu:306-311), and one output per receive
  element (NoSum/..._Nosum.cu, NoSum_ab/..._Nosum_ab.cu, through
  ``bf_rca_nosum``): REF_COMPAT tables against the same reference kernels
  compiled for sm_100a without fast math (identical bits expected, 1e-4
  relative RMS allowed), and against their committed host outputs;
* EXACT tables against the FP64 oracle with the same options (-60 dB).
"""
import warnings

import numpy as np
import pytest

from oracle import host as H
from tests.golden.make_golden import VARIANT_CASES, load

pytestmark = pytest.mark.gpu

REF_TOL = 1e-4
DB_EXACT = -60.0


@pytest.fixture(scope="module")
def bf(cuda):
    from simu_rca_ab_b200 import beamformer as B
    return B


def _param_law(ab):
    """The fixture's law ([element] or [tx][element], seconds) as the
    reference wrappers take Param.AbLawRx: a MATLAB [element x tx] matrix
    whose column-major order is the kernel's [tx][element] index."""
    return None if ab is None else (ab if np.ndim(ab) == 1 else np.asarray(ab).T)


def _nosum_shape(r, out):
    """[element][frame][tx][pix] -> the no-sum wrapper's [Nz, Nx, Ny, tx, frame, element]."""
    s1, s2, s3 = r.grid_shape
    E, F, T, _ = out.shape
    return out.reshape(E, F, T, s3, s2, s1).transpose(5, 4, 3, 2, 1, 0)


def _run(bf, name, table_mode):
    data, G, T, P, O, outs = load(name)
    kernel = str(outs["kernel"])
    ab = outs.get("ab_law")
    P2 = dict(P)
    if ab is not None:
        P2["AbLawRx"] = _param_law(ab)
    opts = {**O, "flagCompounding": False, "tableMode": table_mode}
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        if kernel.startswith("nosum"):
            db, mk = bf.bf_rca_nosum(data, G, T, P2, opts)
        else:
            db, mk = bf.bf_rca(data, G, T, P2, opts)
    r = H.prepare(data, G, T, P, {**O, "flagCompounding": False})
    return db, mk, r, kernel, ab, outs


@pytest.mark.parametrize("name", sorted(VARIANT_CASES))
def test_ref_compat_variants_match_the_reference_kernels(bf, name):
    db, mk, r, kernel, ab, outs = _run(bf, name, "ref_compat")
    per_ch = kernel.startswith("nosum")
    shape = _nosum_shape if per_ch else (lambda r_, o: H.matlab_shape(r_, o, outs["mask_tx"])[0])
    golden = shape(r, outs["out"])
    assert db.shape == golden.shape
    e_gold = H.rel_rms(db, golden)
    if H.have_ref_gpu("strict", kernel):
        o2, m2 = H.run_ref_gpu(r, "strict", kernel=kernel, ab_law=ab)
        ref = shape(r, o2)
        e = H.rel_rms(db, ref)
        print(f"{name}: rel RMS vs reference {kernel} kernel (sm_100a strict) {e:.3e}, "
              f"identical bits {np.array_equal(db, ref)}; vs its host build {e_gold:.3e}")
        assert e <= REF_TOL
        assert np.allclose(mk, H.matlab_shape(r, o2[0] if per_ch else o2, m2)[1], rtol=1e-6, atol=1e-6)
    assert e_gold < 0.1


@pytest.mark.parametrize("name", sorted(VARIANT_CASES))
def test_exact_variants_match_the_fp64_oracle(bf, name):
    db, mk, r, kernel, ab, outs = _run(bf, name, "exact")
    per_ch = kernel.startswith("nosum")
    interp = H.INTERP_REF6 if r.lanczos else H.INTERP_QUAD3
    f64, _ = H.run_fp64(r, interp, 3, per_channel=per_ch, ab_law=ab,
                        ab_per_tx=ab is not None and np.ndim(ab) == 2)
    ref = _nosum_shape(r, f64) if per_ch else H.matlab_shape(r, f64, outs["mask_tx"])[0]
    rms, peak = H.error_db(db, ref)
    print(f"{name} EXACT: {rms:.1f} dB RMS, {peak:.1f} dB peak vs FP64")
    assert rms <= DB_EXACT


def test_per_channel_terms_sum_to_the_beamformed_volume(bf):
    """Summing the no-sum output over elements gives the summed beamformer
    (per transmit), within FP32 summation-order differences."""
    data, G, T, P, O, outs = load("ref6_rx_x")
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        per, _ = bf.bf_rca_nosum(data, G, T, P, {**O, "tableMode": "exact"})
        summed, _ = bf.bf_rca(data, G, T, P, {**O, "flagCompounding": False, "tableMode": "exact",
                                                "kernel": "plain"})
    assert H.rel_rms(per.sum(axis=-1), summed) < 1e-5


@pytest.mark.parametrize("table_mode", ["ref_compat", "exact"])
@pytest.mark.parametrize("name", ["nosumab_ref6_rx_y", "nosum_quad3_rx_x_mask"])
def test_per_channel_all_frames_launch_gives_the_per_frame_kernels_bits(bf, name, table_mode):
    """The per-channel output of every frame from one launch (pc_das_kernel,
    the planner's choice) against the one-launch-per-frame kernel (by name):
    identical bits on ten frames (the fixture's events repeated at five
    scales), with an aberration law and with the cone mask, in both table
    modes."""
    data, G, T, P, O, outs = load(name)
    ab = outs.get("ab_law")
    P2 = dict(P)
    if ab is not None:
        P2["AbLawRx"] = _param_law(ab)
    d5 = np.concatenate([data * (1.0 + 0.25 * f) for f in range(5)], axis=-1)   # events axis
    opts = {**O, "flagCompounding": False, "tableMode": table_mode}
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        one, m1 = bf.bf_rca_nosum(d5, G, T, P2, opts)
        per, m2 = bf.bf_rca_nosum(d5, G, T, P2, {**opts, "kernel": "plain"})
        single, _ = bf.bf_rca_nosum(data, G, T, P2, opts)
    assert one.shape == per.shape and one.shape[-2] == 5 * single.shape[-2]
    assert np.array_equal(one, per)
    assert np.array_equal(m1, m2)
    assert np.abs(one).max() > 0
