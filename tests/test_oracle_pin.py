"""Pins the oracle before it is trusted.

* The C restatement of the reference arithmetic (oracle/rca_oracle.c,
  FP32 mode) reproduces the committed golden outputs of the reference kernel
  source (tests/golden, made by O1) bit for bit.
* The same, live against O1 on fresh seeded cases (when oracle/_ref is built).
* The FP64 oracle in C agrees with the independent NumPy FP64 restatement.
* The FP64 oracle agrees with the reference kernel where FP32 is not lossy
  (virtual sources close to the array: no cancellation in the transmit delay).
"""
import numpy as np
import pytest

from oracle import fp64 as F64
from oracle import host as H
from tests.golden.make_golden import CASES, VARIANT_CASES, case, load


@pytest.mark.parametrize("name", sorted(CASES))
def test_c_restatement_matches_golden_bitwise(name):
    data, G, T, P, O, outs = load(name)
    r = H.prepare(data, G, T, P, O)
    per_tx, mask_tx = H.run_c32(r)
    assert np.array_equal(per_tx.astype(np.complex64).view(np.float32), outs["per_tx"].view(np.float32))
    assert np.array_equal(mask_tx, outs["mask_tx"])
    comp, mc = H.compound(per_tx.astype(np.complex64), mask_tx, True)
    db, mk = H.matlab_shape(r, comp, mc)
    assert db.shape == outs["dataBf"].shape and mk.shape == outs["mask"].shape
    assert np.array_equal(db, outs["dataBf"]) and np.array_equal(mk, outs["mask"])


@pytest.mark.skipif(not H.have_ref_cpu(), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed,rx,lan,mask", [(11, True, True, True), (12, False, False, True),
                                              (13, True, False, False)])
def test_c_restatement_matches_reference_source_live(seed, rx, lan, mask):
    data, G, T, P, O = case(seed, rx, lan, mask, ns=128, grid=(20, 10, 8))
    r = H.prepare(data, G, T, P, O)
    o1, m1 = H.run_ref_cpu(r)
    c1, cm = H.run_c32(r)
    assert np.array_equal(o1.view(np.float32), c1.view(np.float32))
    assert np.array_equal(m1, cm)


@pytest.mark.parametrize("interp,a", [(H.INTERP_QUAD3, 0), (H.INTERP_REF6, 0), (H.INTERP_LANCZOS, 2),
                                      (H.INTERP_LANCZOS, 3), (H.INTERP_LANCZOS, 4)])
def test_fp64_c_matches_numpy(interp, a):
    data, G, T, P, O = case(21, True, False, False, ns=128)
    r = H.prepare(data, G, T, P, O)
    c64, cm = H.run_fp64(r, interp, a)
    n64, nm = F64.das_fp64(r, interp, a)
    assert H.rel_rms(c64, n64) < 1e-13
    assert np.allclose(cm, nm, rtol=1e-13, atol=1e-12)


@pytest.mark.skipif(not H.have_ref_cpu(), reason="oracle/_ref not built")
@pytest.mark.parametrize("lan", [False, True])
def test_fp64_oracle_matches_reference_without_cancellation(lan):
    # Virtual sources 5 mm behind the array: the transmit delay keeps full
    # FP32 precision, so the reference and the FP64 model must agree closely.
    data, G, T, P, O = case(31, True, lan, False, ns=128)
    T = {"virtualSourceX": np.zeros(4), "virtualSourceY": np.linspace(-1e-3, 1e-3, 4),
         "virtualSourceZ": np.full(4, -5e-3), "flagReceiveX": True}
    r = H.prepare(data, G, T, P, O)
    o1, _ = H.run_ref_cpu(r)
    f1, _ = H.run_fp64(r, H.INTERP_REF6 if lan else H.INTERP_QUAD3)
    rms, _ = H.error_db(o1, f1)
    assert rms < -75, rms


def test_reference_fp32_transmit_delay_error_is_visible():
    # With a 10 m virtual source the reference's FP32 transmit delay cancels
    # catastrophically; its output then sits about -33 dB from the FP64 model.
    data, G, T, P, O = case(41, True, False, False, ns=128)
    r = H.prepare(data, G, T, P, O)
    c1, _ = H.run_c32(r)
    f1, _ = H.run_fp64(r, H.INTERP_QUAD3)
    rms, _ = H.error_db(c1, f1)
    assert -45 < rms < -20, rms


REF_VARIANTS = [("ab1", False, False), ("ab2", False, True), ("nosum", True, None), ("nosumab", True, False)]


@pytest.mark.parametrize("kernel,per_channel,ab_per_tx", REF_VARIANTS)
@pytest.mark.parametrize("rx,lan,mask", [(True, True, False), (False, False, True)])
def test_c_restatement_matches_reference_variants(kernel, per_channel, ab_per_tx, rx, lan, mask):
    """The aberration-law kernels (Hyp1_save/..._ab_1.cu, Hyp2/..._ab_2.cu)
    and the per-channel kernels (NoSum/..._Nosum.cu, NoSum_ab/..._Nosum_ab.cu),
    compiled from their own sources, against the C restatement with the
    corresponding option: identical bits."""
    if not H.have_ref_cpu(kernel):
        pytest.skip("oracle/_ref variant build missing")
    data, G, T, P, O = case(61, rx, lan, mask, ns=128)
    r = H.prepare(data, G, T, P, O)
    rng = np.random.default_rng(62)
    ab = None
    if ab_per_tx is not None:
        ab = rng.uniform(-40e-9, 40e-9, (r.n_tx, r.n_ch) if ab_per_tx else r.n_ch)
    o1, m1 = H.run_ref_cpu(r, kernel=kernel, ab_law=ab)
    c1, cm = H.run_c32(r, per_channel=per_channel, ab_law=ab, ab_per_tx=bool(ab_per_tx))
    assert o1.shape == c1.shape
    assert np.array_equal(o1.astype(np.complex64).view(np.float32), c1.astype(np.complex64).view(np.float32))
    assert np.array_equal(m1, cm)
    assert np.abs(o1).max() > 0


@pytest.mark.parametrize("name", sorted(VARIANT_CASES))
def test_c_restatement_matches_variant_golden_bitwise(name):
    """Committed outputs of the reference's aberration-law / per-channel
    kernels (made by O1, tests/golden/make_golden.py) against the C
    restatement: identical bits, no reference tree needed."""
    data, G, T, P, O, outs = load(name)
    kernel = str(outs["kernel"])
    r = H.prepare(data, G, T, P, O)
    ab = outs.get("ab_law")
    c1, cm = H.run_c32(r, per_channel=kernel.startswith("nosum"), ab_law=ab,
                       ab_per_tx=ab is not None and np.ndim(ab) == 2)
    assert np.array_equal(c1.astype(np.complex64).view(np.float32), outs["out"].view(np.float32))
    assert np.array_equal(cm, outs["mask_tx"])
