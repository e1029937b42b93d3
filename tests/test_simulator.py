"""The frequency-domain simulator (SimUS_CUDARCA) against the reference's own
field kernels.

CPU: the product's host set-up and the oracle's independent restatement of
SimUS_CUDARCA.m:81-246 agree; the reference kernels compiled for the host
(O1) run.  GPU: the element field (rcabf_sim_element_field), combined with
the transmit delay / apodisation / pulse / impulse responses as the product
combines them, reproduces the reference kernels TXfield and RXfield compiled
for sm_100a (O2, no fast math) and for the host (O1) within 1e-4 relative
RMS, with a flat and with a focused elevation aperture; the whole simulation
(frames, events, the fields evaluated inside the transmit and receive sums,
the inverse transforms as direct sums, sub-sampling: rcabf_sim_tx_field,
rcabf_sim_rx_spectrum, rcabf_sim_rf) reproduces the reference pipeline run
with the O1 kernels within 1e-4.
"""
import numpy as np
import pytest

from oracle import simulator as OS


def sim_case(seed=0, n_ele=12, n_sub=3, n_scat=15, n_tx=2, n_frame=2, focus=20e-3, moving=True, baffle=1):
    """Seeded RCA set-up: transmit rows (strips along x) and receive columns
    (strips along y) of n_ele elements, n_sub sub-elements along each strip."""
    rng = np.random.default_rng(seed)
    pitch, f0, c = 0.3e-3, 7.8e6, 1540.0
    pos = (np.arange(n_ele) - (n_ele - 1) / 2) * pitch
    strip = (np.arange(n_sub) - (n_sub - 1) / 2) * (n_ele * pitch / n_sub)
    tx = np.zeros((n_ele, 5, n_sub))
    rx = np.zeros((n_ele, 5, n_sub))
    for q in range(n_sub):
        tx[:, 0, q], tx[:, 1, q] = strip[q], pos          # rows: at y = pos, spread along x
        rx[:, 0, q], rx[:, 1, q] = pos, strip[q]          # columns: at x = pos, spread along y
    t = np.arange(0, 2 / f0, 1 / 250e6)
    ir = np.sin(2 * np.pi * f0 * t) * np.hanning(t.size)
    trans = lambda p: {"frequency": f0, "impulseResponse": ir, "lensCorrection": 0.1e-6, "ElementPos": p,
                       "ElementHeight": 2e-3, "ElementWidth": 0.27e-3, "ElementElevationFocus": focus,
                       "baffle": baffle}
    n_event = n_tx * n_frame
    base = np.stack([rng.uniform(-1.5e-3, 1.5e-3, n_scat), rng.uniform(-1.5e-3, 1.5e-3, n_scat),
                     rng.uniform(3e-3, 6e-3, n_scat), rng.rayleigh(1.0, n_scat)], 1)
    scat = np.repeat(base[:, :, None], n_event, 2)
    if moving:       # events of a frame see different positions
        scat[:, :3, :] += rng.normal(0, 20e-6, (n_scat, 3, n_event))
    th = np.deg2rad(np.linspace(-5, 5, n_tx))
    TXSI = [{"pulseShape": np.sin(2 * np.pi * f0 * t), "Delay": pos * np.sin(a) / c - (pos * np.sin(a) / c).min(),
             "Apod": np.hanning(n_ele + 2)[1:-1]} for a in th]
    RXSI = [{"samplingFrequency": 4 * f0, "demodFrequency": f0, "startTime": 2e-6, "numelSample": 256,
             "sampleMode": "NS200BW", "InputFilter": np.array([1.0]), "Apod": np.ones(n_ele)} for _ in th]
    Media = {"speedOfSound": c, "attenuation": 0.5, "scattererPos": scat}
    return Media, trans(tx), trans(rx), TXSI, RXSI


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def test_raw_length_is_the_interleave_of_the_two_subsampled_rows():
    """Raw's fast-time length: RF(1:sub:end) and RF(2:sub:end) interleaved,
    each cut to the shorter (SimUS_CUDARCA.m:385-386)."""
    from simu_rca_ab_b200.simulator import _out_samples
    for sub in (2, 4, 8):
        for numel in range(1, 40):
            rf = np.arange(numel)
            assert _out_samples(numel, sub) == 2 * min(rf[0::sub].size, rf[1::sub].size), (numel, sub)


def test_host_setups_agree():
    from simu_rca_ab_b200.simulator import sim_plan
    case = sim_case()
    a, b = sim_plan(*case), OS.plan(*case)
    for key in ("n_tx", "n_event", "sub", "n_fast", "n_freq", "numel"):
        assert a[key] == b[key], key
    for key in ("k", "pulse", "ir_tx", "ir_rx", "ipf", "delay", "apod", "rx_apod", "pos_tx", "pos_rx", "scat"):
        assert np.allclose(a[key], b[key], rtol=1e-12, atol=1e-15), key


@pytest.mark.skipif(not OS.have_sim_cpu(), reason="oracle/_ref simulator build missing")
def test_reference_host_pipeline_runs():
    p = OS.plan(*sim_case(n_frame=1))
    raw, rf = OS.simulate(p)
    assert raw.shape == (256, 12, 2) and np.isfinite(raw).all() and np.abs(raw).max() > 0


def _ours_tx_rx(p, j):
    """The product's transmit field [s][f] and receive field [s][e][f] of
    transmit event j of the first frame, composed as sim_us_rca composes them."""
    import torch
    from simu_rca_ab_b200 import simulator as S
    dev = torch.device("cuda")
    k = torch.from_numpy(p["k"].astype(np.complex64)).cuda()
    w = torch.from_numpy(np.real(p["k"]).astype(np.float32) * np.float32(p["c"])).cuda()
    r = torch.from_numpy(np.ascontiguousarray(p["scat"][:, :3, j].T, dtype=np.float32)).cuda()
    st = torch.cuda.current_stream().cuda_stream
    e_tx = S._element_field(dev, r, torch.from_numpy(S._ele_layout(p["pos_tx"])).cuda(), k, p["tx"], p["c"], st)
    e_rx = S._element_field(dev, r, torch.from_numpy(S._ele_layout(p["pos_rx"])).cuda(), k, p["rx"], p["c"], st)
    d = torch.from_numpy(p["delay"][:, j].astype(np.float32)).cuda()
    a = torch.from_numpy(p["apod"][:, j].astype(np.float32)).cuda()
    wt = a[None] * torch.polar(torch.ones_like(d)[None].expand(k.shape[0], -1), w[:, None] * d[None])   # [f, e]
    fac = torch.from_numpy((np.conj(p["pulse"]) * np.conj(p["ir_tx"])).astype(np.complex64)).cuda()
    tx = torch.einsum("fse,fe->sf", e_tx, wt) * fac[None]
    rx = e_rx.permute(1, 2, 0) * torch.from_numpy(p["ir_rx"].astype(np.complex64)).cuda()[None, None]
    return tx.cpu().numpy(), rx.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("focus,baffle", [(20e-3, 1), (100.0, 0)])
def test_element_field_reproduces_the_reference_kernels(cuda, focus, baffle):
    p = OS.plan(*sim_case(focus=focus, baffle=baffle))
    n_sub = p["pos_tx"].shape[2]
    ev = list(range(p["n_tx"]))
    for variant in ("strict",):
        if not OS.have_sim_gpu(variant):
            pytest.skip("oracle/_ref simulator GPU build missing")
    ref_tx = OS.txfield_gpu("strict", p["scat"][:, :3, ev], p["pos_tx"], p["k"], p["pulse"], p["ir_tx"],
                            p["delay"], p["apod"], p["tx"], p["c"], n_sub)          # [tx][s][f]
    for j in ev:
        tx, rx = _ours_tx_rx(p, j)
        ref_rx = OS.rxfield_gpu("strict", p["scat"][:, :3, j], p["pos_rx"], p["k"], p["ir_rx"], p["rx"], p["c"], n_sub)
        e_tx, e_rx = _rel(tx, ref_tx[j]), _rel(rx, ref_rx)
        msg = f"focus {focus}: TX {e_tx:.2e}, RX {e_rx:.2e} rel RMS vs the reference kernels (sm_100a strict)"
        if OS.have_sim_cpu():
            o1_tx = OS.txfield_cpu(p["scat"][:, :3, ev], p["pos_tx"], p["k"], p["pulse"], p["ir_tx"], p["delay"],
                                   p["apod"], p["tx"], p["c"], n_sub)
            msg += f"; vs host build {_rel(tx, o1_tx[j]):.2e}; O1 vs O2 {_rel(o1_tx[j], ref_tx[j]):.2e}"
        print(msg)
        assert e_tx < 1e-4 and e_rx < 1e-4


@pytest.mark.gpu
@pytest.mark.skipif(not OS.have_sim_cpu(), reason="oracle/_ref simulator build missing")
@pytest.mark.parametrize("moving,n_tx", [(True, 2), (False, 2), (False, 18)])
def test_simulation_matches_the_reference_pipeline(cuda, moving, n_tx):
    """Moving scatterers (one group per event), static ones (the frame's
    events as one group) and 18 transmits (groups of 16 and 2)."""
    from simu_rca_ab_b200.simulator import sim_us_rca
    case = sim_case(moving=moving, n_tx=n_tx)
    raw, rf = sim_us_rca(*case, return_rf=True)
    raw_ref, rf_ref = OS.simulate(OS.plan(*case))
    assert raw.shape == raw_ref.shape
    e = _rel(raw, raw_ref)
    print(f"simulation (moving={moving}, {n_tx} tx): Raw {e:.2e} rel RMS vs the reference pipeline (O1 kernels)")
    assert e < 1e-4
    assert _rel(rf, rf_ref) < 1e-4
