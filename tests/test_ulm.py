"""ULM super-localisation (Python/superloc/superloc.py) on the GPU against
the oracle's FP64 restatement (oracle/ulm.py).

Parity is unpinned: the reference needs ArrayFire, which is not installed,
so the oracle is pinned by known answers instead -- the convolution by a
direct sum, the parabola fit by Gaussian spots at known sub-pixel positions
(log of a Gaussian is a parabola: the fit is exact), the whole filter by
finding moving spots where they were put, the binning by hand-worked edge
cases of the reference's int16 rules.  The GPU stages then match the oracle:
maps within FP32 rounding, candidate masks and density maps exactly, fitted
positions within 1e-3 pixel.
"""
import numpy as np
import pytest

from oracle import ulm as O


def _rng(seed):
    return np.random.default_rng(seed)


def _psf(kz=9, kx=7, f=0.25):
    z = np.arange(kz) - (kz - 1) / 2
    x = np.arange(kx) - (kx - 1) / 2
    env = np.exp(-(z[:, None] ** 2) / 6.0 - (x[None, :] ** 2) / 4.0)
    return (env * np.exp(2j * np.pi * f * z)[:, None]).astype(np.complex64)


def spots(nz=48, nx=48, nt=12, n=6, seed=0, noise=0.02, sigma=1.4):
    """Frames of complex Gaussian spots moving by <= 0.3 pixel per frame,
    with their true (z, x) per frame, plus complex noise."""
    rng = _rng(seed)
    # on a jittered grid, at least ~10 pixels apart whatever they move
    gz = np.linspace(12, nz - 12, 3)
    gx = np.linspace(12, nx - 12, (n + 2) // 3)
    cells = np.array([(a, b) for a in gz for b in gx])[:n]
    z0 = cells[:, 0] + rng.uniform(-1.5, 1.5, n)
    x0 = cells[:, 1] + rng.uniform(-1.5, 1.5, n)
    vz, vx = rng.uniform(-0.3, 0.3, n), rng.uniform(-0.3, 0.3, n)
    amp = rng.uniform(1.0, 2.0, n) * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    zz, xx = np.meshgrid(np.arange(nz), np.arange(nx), indexing="ij")
    iq = np.zeros((nz, nx, nt), np.complex128)
    truth = np.zeros((nt, n, 2))
    for t in range(nt):
        for k in range(n):
            zc, xc = z0[k] + vz[k] * t, x0[k] + vx[k] * t
            truth[t, k] = (zc, xc)
            iq[:, :, t] += amp[k] * np.exp(-((zz - zc) ** 2 + (xx - xc) ** 2) / (2 * sigma ** 2))
    iq += noise * (rng.standard_normal(iq.shape) + 1j * rng.standard_normal(iq.shape))
    return iq.astype(np.complex64), truth


# ---------------------------------------------------------------- oracle pins
@pytest.mark.parametrize("kz,kx", [(5, 5), (4, 6), (7, 3)])
def test_oracle_convolution_is_arrayfire_same_mode(kz, kx):
    rng = _rng(1)
    sig = rng.standard_normal((9, 8, 2)) + 1j * rng.standard_normal((9, 8, 2))
    ker = rng.standard_normal((kz, kx)) + 1j * rng.standard_normal((kz, kx))
    out = O._conv_same_2d(sig, ker)
    ref = np.zeros_like(out)
    for t in range(2):
        for z in range(9):
            for x in range(8):
                for a in range(kz):
                    for b in range(kx):
                        zi, xi = z + kz // 2 - a, x + kx // 2 - b
                        if 0 <= zi < 9 and 0 <= xi < 8:
                            ref[z, x, t] += sig[zi, xi, t] * ker[a, b]
    assert np.allclose(out, ref, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("dz,dx", [(0.0, 0.0), (0.31, -0.42), (-0.49, 0.17)])
def test_oracle_parabola_fit_recovers_a_gaussian_spot(dz, dx):
    """log of a Gaussian spot is a parabola, so the Hann-weighted fit returns
    its sub-pixel centre exactly (square map: x, z as the reference reads them)."""
    n, nt, sigma = 21, 3, 1.7
    zz, xx = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    m = np.exp(-((zz - 10 - dz) ** 2 + (xx - 10 - dx) ** 2) / (2 * sigma ** 2))
    amap = np.repeat(m[:, :, None], nt, 2)
    pos = O.super_loc_filter(amap.astype(complex), amap.astype(complex), fit=1)
    # the static spot is found once per ensemble frame, at its centre
    assert pos.shape[1] == nt - 1
    assert np.allclose(pos[2], 10 + dz, atol=1e-9) and np.allclose(pos[0], 10 + dx, atol=1e-9)
    assert np.all(pos[1] == 0)


def test_oracle_filter_finds_moving_spots():
    iq, truth = spots()
    corr = O.psf_corr_map_2d(iq, _psf(7, 7, 0.0).real.astype(complex))
    pos = O.super_loc_filter(corr, iq, fit=0)
    found = 0
    for t in range(iq.shape[2] - 1):
        sel = pos[4] == t
        for k in range(truth.shape[1]):
            z, x = truth[t, k]
            d = np.hypot(pos[2, sel] - z, pos[0, sel] - x)
            found += bool(d.size and d.min() < 0.75)
    # every spot of every frame localised within 0.75 pixel (the lag-1
    # ensemble averages two frames the spot moved between)
    assert found == (iq.shape[2] - 1) * truth.shape[1]


def test_oracle_bins_follow_the_reference_int16_rules():
    bins = np.arange(10) * 0.5                   # 10 bins of 0.5 from 0
    v = np.array([-3.0, 0.2, 0.5, 4.74, 4.75, 5.0, 7.0, 1e6, np.nan])
    # (v - 0) / 0.5 -> int16: -6, 0, 1, 9, 9, 10, 14, wrap(2e6), NaN->0
    i = O._bins(v, bins)
    wrap = np.int32(2_000_000).astype(np.int16)   # 2e6 mod 2^16, signed
    exp_wrap = 0 if wrap <= 0 else (wrap if wrap < 10 else 9)
    assert list(i[:7]) == [0, 0, 1, 9, 9, 0, 9]  # 10 (the bin count) -> 0, > count -> last
    assert i[7] == exp_wrap and i[8] == 0


def test_oracle_density_and_velocity_maps():
    rng = _rng(2)
    pos = np.zeros((5, 200))
    pos[0], pos[1], pos[2] = rng.uniform(0, 4, 200), rng.uniform(0, 2, 200), rng.uniform(0, 3, 200)
    pos[4] = rng.integers(0, 4, 200)
    vel = rng.standard_normal((3, 200))
    xb, yb, zb, tb = np.arange(8) * 0.5, np.arange(4) * 0.5, np.arange(6) * 0.5, np.arange(4)
    dens = O.density_mapping_nd(pos, xb, yb, zb)
    assert dens.shape == (6, 8, 4) and dens.sum() == 200
    d2, vm = O.velocity_mapping_nd(pos, vel, xb, [0.0], zb)     # one y bin: maps squeeze to (z, x)
    assert d2.sum() == 200 and vm.shape[:2] == (6, 8)
    dt = O.density_mapping_ndt(pos, xb, yb, zb, tb)
    assert dt.shape == (6, 8, 4, 4) and dt.sum() == 200
    d3, vt = O.velocity_mapping_ndt(pos, vel, xb, yb, zb, tb)
    assert vt.shape == (6, 8, 4, 4, 3) and np.array_equal(d3, dt)


# ----------------------------------------------------------------- GPU parity
@pytest.mark.gpu
@pytest.mark.parametrize("kz,kx,shape", [(9, 7, (48, 48, 6)), (8, 6, (40, 56, 5)), (33, 33, (70, 64, 3))])
def test_psf_corr_map_matches_oracle(cuda, kz, kx, shape):
    from simu_rca_ab_b200 import ulm as U
    rng = _rng(3)
    iq = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    psf = _psf(kz, kx)
    got = U.PsfCorrMap2D(iq, psf)
    ref = O.psf_corr_map_2d(iq, psf)
    assert got.shape == ref.shape and got.dtype == np.complex64
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    print(f"PsfCorrMap2D {shape} psf {kz}x{kx}: rel RMS {err:.2e}")
    assert err < 1e-5


@pytest.mark.gpu
def test_regional_max_is_exact(cuda):
    from simu_rca_ab_b200 import ulm as U
    rng = _rng(4)
    m = rng.standard_normal((33, 41, 4)).astype(np.float32)
    m[5:8, 5:8, 0] = 10.0                                    # a plateau: every pixel of it is a maximum
    got = U.ImRegionalMax(m, 3)
    assert np.array_equal(got, O.regional_max(m, 3))
    assert got[5:8, 5:8, 0].all()


def _stages(iq, psf, fit):
    """The GPU's maps, detections and positions, stage by stage."""
    import torch
    from simu_rca_ab_b200 import ulm as U
    corr = U.PsfCorrMap2D(torch.from_numpy(iq).cuda(), psf)
    cm, _ = U._to_dev(corr, torch.complex64)
    em, _ = U._to_dev(torch.from_numpy(iq).cuda(), torch.complex64)
    Cm, Em = U._ensemble(cm, 5), U._ensemble(em, 5)
    lin, val = U._detect(Cm, Em, 3, fit)
    pos = U.SuperLocFilter(corr, torch.from_numpy(iq).cuda(), fit=fit)
    f = lambda t: t.permute(2, 1, 0).cpu().numpy().astype(np.float64)
    return corr.cpu().numpy(), f(Cm), f(Em), lin.cpu().numpy(), val.cpu().numpy(), pos.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("fit", [0, 1])
@pytest.mark.parametrize("nz,nx", [(48, 48), (40, 52)])
def test_super_loc_filter_stages_match_oracle(cuda, fit, nz, nx):
    iq, _ = spots(nz=nz, nx=nx, nt=10, seed=5 + fit)
    psf = _psf(7, 7, 0.0).real.astype(np.complex64)
    corr, C64, E64, lin, val, pos = _stages(iq, psf, fit)
    # ensemble maps: GPU (FP32) vs oracle on the GPU's correlation map
    Cref, Eref = O.ensemble_map(corr), O.ensemble_map(iq)
    assert np.linalg.norm(C64 - Cref) / np.linalg.norm(Cref) < 1e-5
    assert np.linalg.norm(E64 - Eref) / np.linalg.norm(Eref) < 1e-5
    # candidate mask and order: exact, given the GPU's own maps
    bw = O.detection_mask(C64, E64, 5, fit)
    ref_lin = np.flatnonzero(bw.reshape(-1, order="F"))
    src = (C64 if fit == 0 else E64).reshape(-1, order="F")
    ref_lin = ref_lin[np.argsort(-np.abs(src[ref_lin]), kind="stable")]
    assert np.array_equal(lin, ref_lin)
    assert np.array_equal(val, np.abs(src[ref_lin]).astype(np.float32))
    # positions: the oracle's fit on the same map and candidates.  The
    # offset -m1 / (2 m2) amplifies FP32 rounding of the moments (~1e-5) by
    # (1 + 2 |offset|) / (2 |m2|): 1e-3 pixel where the log-map is curved (the
    # spots), the propagated bound (x10) where it is nearly flat (noise).
    ref, mx, mz = O.gauss_fit(lin, val.astype(np.float64), C64 if fit == 0 else E64, moments=True)
    assert ref.shape == pos.shape
    assert np.array_equal(np.isfinite(ref), np.isfinite(pos))
    n_loose = 0
    for row, m in ((0, mx), (2, mz)):      # x, z in pixels
        ok = np.isfinite(ref[row])
        sub = -0.5 * m[1, ok] / m[2, ok]
        bound = 1e-3 + 5e-5 * (1 + 2 * np.abs(sub)) / np.abs(m[2, ok])
        assert np.all(np.abs(pos[row, ok] - ref[row, ok]) <= bound)
        n_loose += int(np.sum(bound > 2e-3))
    assert np.array_equal(pos[1], ref[1]) and np.array_equal(pos[4], ref[4]) and np.array_equal(pos[3], val)
    # the whole oracle pipeline (FP64 maps) finds the same candidates but
    # for near-ties of FP32 rounding
    full = O.super_loc_filter(corr, iq, fit=fit)
    assert abs(full.shape[1] - pos.shape[1]) <= max(2, pos.shape[1] // 100)
    print(f"SuperLocFilter fit {fit} {nz}x{nx}: {pos.shape[1]} detections (oracle {full.shape[1]}), "
          f"{n_loose} coordinates of nearly flat fits checked against the propagated bound")


@pytest.mark.gpu
def test_density_and_velocity_maps_match_oracle(cuda):
    from simu_rca_ab_b200 import ulm as U
    rng = _rng(6)
    n = 5000
    pos = np.zeros((5, n))
    pos[0], pos[1], pos[2] = rng.uniform(-1, 5, n), rng.uniform(-0.5, 2.5, n), rng.uniform(-1, 4, n)
    pos[4] = rng.integers(0, 5, n)
    pos[0, :4] = [4.0, 3.5, np.nan, 1e7]                       # bin-count, last, NaN and wrapped edges
    vel = rng.standard_normal((3, n))
    xb, yb, zb, tb = np.arange(8) * 0.5, np.arange(4) * 0.5, np.arange(6) * 0.5, np.arange(4)
    assert np.array_equal(U.DensityMappingND(pos, xb, yb, zb), O.density_mapping_nd(pos, xb, yb, zb))
    assert np.array_equal(U.DensityMappingNDt(pos, xb, yb, zb, tb), O.density_mapping_ndt(pos, xb, yb, zb, tb))
    d, v = U.VelocityMappingND(pos, vel, xb, [0.0], zb)
    dr, vr = O.velocity_mapping_nd(pos, vel, xb, [0.0], zb)
    assert np.array_equal(d, dr) and np.allclose(v, vr, rtol=1e-12, atol=1e-12)
    d, v = U.VelocityMappingNDt(pos, vel, xb, yb, zb, tb)
    dr, vr = O.velocity_mapping_ndt(pos, vel, xb, yb, zb, tb)
    assert np.array_equal(d, dr) and np.allclose(v, vr, rtol=1e-12, atol=1e-12)
