"""SVD clutter filter (SVDClutterFilter.m) against its FP64 restatement.

CPU: the component selection of every filter type follows the reference's
round(w * nT) and 1-based inclusive ranges.  GPU: on a seeded ensemble with
strong low-rank tissue, a weaker blood subspace and noise, the filtered
ensemble matches the FP64 oracle within 1e-4 relative RMS (-80 dB) for
low / high / band / stop filters, with and without noise weights, in the
beamformer's layout and in MATLAB's.
"""
import numpy as np
import pytest

from oracle import clutter as OC


@pytest.mark.parametrize("n", [8, 64, 200, 201])
@pytest.mark.parametrize("w,kind", [((0.1,), "low"), ((0.13,), "high"), ((0.1, 0.9), "band"),
                                    ((0.05, 0.95), "stop"), ((0.0, 1.0), "band"), ((0.5,), "low"),
                                    ((0.0078125, 0.5), "band")])
def test_component_selection_follows_the_reference(n, w, kind):
    from simu_rca_ab_b200.clutter import keep_components
    assert np.array_equal(keep_components(n, w, kind), OC.keep_matlab(n, w, kind))


def test_bad_cutoffs_raise():
    from simu_rca_ab_b200.clutter import keep_components
    with pytest.raises(ValueError):
        keep_components(10, (1.2,), "low")
    with pytest.raises(ValueError):
        keep_components(10, (0.2,), "band")


def _ensemble(n_pix=6000, n_t=64, seed=0):
    """[pix][t] complex: rank-4 tissue (+60 dB), rank-10 blood (+20 dB), noise."""
    rng = np.random.default_rng(seed)
    t = np.arange(n_t)
    tissue = sum(rng.normal(size=n_pix)[:, None] * 1000.0 / (k + 1) *
                 np.exp(2j * np.pi * (0.002 * k) * t)[None, :] for k in range(4))
    blood = sum(rng.normal(size=n_pix)[:, None] * 10.0 / (k + 1) *
                np.exp(2j * np.pi * (0.05 + 0.03 * k) * t + 1j * rng.uniform(0, 6.28))[None, :] for k in range(10))
    noise = (rng.normal(size=(n_pix, n_t)) + 1j * rng.normal(size=(n_pix, n_t))) * 0.5
    return (tissue + blood + noise).astype(np.complex64)


CASES = [((4 / 64,), "low"), ((5 / 64,), "high"), ((5 / 64, 14 / 64), "band"), ((4 / 64, 15 / 64), "stop")]


@pytest.mark.gpu
@pytest.mark.parametrize("w,kind", CASES)
@pytest.mark.parametrize("weighted", [False, True])
def test_filter_matches_fp64_oracle(cuda, w, kind, weighted):
    import torch
    from simu_rca_ab_b200.clutter import svd_clutter_filter
    c = _ensemble()
    nz, nx, ny = 15, 20, 20                                       # 6000 pixels
    iq = np.asfortranarray(c.reshape(nz, nx, ny, 64, order="F"))  # MATLAB [Nz, Nx, Ny, nT]
    mask = None
    if weighted:
        mask = np.asfortranarray(np.random.default_rng(1).uniform(0.5, 2.0, (nz, nx, ny)))
    keep = OC.keep_matlab(64, w, kind)
    ref, ev_ref = OC.svd_filter_fp64(iq.reshape(-1, 64, order="F"),
                                     None if mask is None else mask.reshape(-1, order="F"), keep)
    out, ev = svd_clutter_filter(iq, mask, w, kind)
    assert out.shape == iq.shape
    got = np.asarray(out).reshape(-1, 64, order="F")
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    print(f"{kind} {w} weighted={weighted}: rel RMS {err:.2e}")
    assert err < 1e-4
    assert np.allclose(ev, ev_ref, rtol=1e-4, atol=1e-5 * ev_ref[0])
    # the beamformer's own layout: [frame][pixel] on the device, time axis 0
    x = torch.from_numpy(np.ascontiguousarray(c.T)).cuda()
    out2, _ = svd_clutter_filter(x, None if mask is None else torch.from_numpy(
        np.ascontiguousarray(mask.reshape(-1, order="F"))).cuda(), w, kind, time_axis=0, order="C")
    assert torch.allclose(out2.cpu(), torch.from_numpy(np.ascontiguousarray(got.T)), rtol=0, atol=1e-3 *
                          float(np.abs(ref).max()))


@pytest.mark.gpu
def test_filter_on_the_beamformed_c2_ensemble_removes_tissue(cuda):
    """Beamformer -> clutter filter on a reduced C2 ensemble: a high-pass
    filter removes the static tissue subspace, so the filtered energy is far
    below the unfiltered one and its top eigen-components carry almost all
    of the ensemble's energy."""
    import warnings

    import torch
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import beamformer as B
    from simu_rca_ab_b200 import workloads as W
    from simu_rca_ab_b200.clutter import svd_clutter_filter
    from simu_rca_ab_b200.params import normalize
    w = W.get("c2", n_frame=32, grid_scale=0.5)
    data = W.channel_data(w, seed=9, device="cuda")
    eng = B.default_engine()
    g0 = w.groups[0]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        geom = eng.geometry(normalize(np.zeros(1, np.complex64), g0.Geometry, g0.Transmit, w.Param, w.Options))
    out = torch.empty((w.n_frame, 1, geom.n_pix), dtype=torch.complex64, device="cuda")
    eng.run(geom, eng.make_args(geom, data.contiguous(), iq_dtype=L.IQ_C64, n_sample=w.n_sample,
                                n_frame=w.n_frame, out=out, mask=None, compound=True))
    x = out[:, 0]
    xf, ev = svd_clutter_filter(x, None, (3 / 32,), "high", time_axis=0, order="C")
    e_in = float((x.abs() ** 2).sum())
    e_out = float((xf.abs() ** 2).sum())
    print(f"C2 ensemble (32 frames): filtered / unfiltered energy {e_out / e_in:.3e}, top eigenvalues {ev[:4]}")
    assert e_out < 0.2 * e_in
    assert float(ev[:2].sum()) > 0.5 * float(ev.sum())
