"""Frequency-domain ultrasound simulator on the GPU: drop-in for
``SimUS_CUDARCA(Media, TransTX, TransRX, TXSI, RXSI, Options)``
(MATLAB/lib/simulator/SimUS_CUDARCA.m), the producer of the RCA channel data
the beamformer consumes.

For each frame (nTX consecutive events) and each transmit event:

  TX(f, s)     = conj(P(f)) conj(IRtx(f)) sum_e E_tx(f, s, e) a_e exp(i w (d_e - t_rx)) * bsc(s)
  S(f, e')     = IPFilt(f) IRrx(f) a'_e' sum_s E_rx(f, s, e') TX(f, s)
  RF(:, e')   += real(ifft(conj(S(:, e')), nFastTime))

with E the element field (librcabf ``rcabf_sim_element_field``: Green's
function, directivities, lens phase), d / a the transmit delays and
apodisation, a' the receive apodisation, P / IR / IPFilt the spectra of the
pulse, impulse responses and input filter (SimUS_CUDARCA.m:111-246, 254-322).
The element field is evaluated once per event (once per frame when all its
events share scatterer positions); the sums over elements and scatterers are
batched complex GEMMs over frequency (cuBLAS), the inverse transforms cuFFT.
The output Raw interleaves RF(1:sub:end) and RF(2:sub:end) as the reference
does (SimUS_CUDARCA.m:338-339), the quadrature-sampled layout the
beamformer's real-input path reads.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib as L

SIM_FS = 250e6      # sampling rate of pulse shapes and impulse responses (SimUS_CUDARCA.m:101)
SUB = {"NS200BW": 2, "BS100BW": 4, "BS50BW": 8}


def _arr(x, dtype=np.float64):
    return np.asarray(x, dtype=dtype)


def sim_plan(Media, TransTX, TransRX, TXSI, RXSI):
    """The host-side quantities of SimUS_CUDARCA.m:81-200 (float64 numpy)."""
    TXSI = TXSI if isinstance(TXSI, (list, tuple)) else [TXSI]
    RXSI = RXSI if isinstance(RXSI, (list, tuple)) else [RXSI]
    pos_tx = _arr(TransTX["ElementPos"])
    if pos_tx.ndim == 2:
        pos_tx = pos_tx[:, :, None]
    if TransRX:
        pos_rx = _arr(TransRX["ElementPos"])
        if pos_rx.ndim == 2:
            pos_rx = pos_rx[:, :, None]
    else:
        pos_rx, TransRX = pos_tx, TransTX
    n_sub_tx = pos_tx.shape[2]
    n_sub_rx = n_sub_tx          # the reference takes the transmit array's count for both (SimUS_CUDARCA.m:93)
    scat = _arr(Media["scattererPos"])
    if scat.ndim == 2:
        scat = scat[:, :, None]
    n_tx = len(TXSI)
    n_event = scat.shape[2]
    if n_event % n_tx:
        raise ValueError("scattererPos needs a whole number of frames of nTX events")
    r0, x0 = RXSI[0], TXSI[0]
    out_fs = float(r0["samplingFrequency"])
    pulse_dur = np.size(x0["pulseShape"]) / SIM_FS
    rx_start = float(r0["startTime"]) - 1.0 / float(TransTX["frequency"])
    max_delay = max(float(np.max(_arr(t["Delay"]))) for t in TXSI)
    sub = SUB.get(r0.get("sampleMode", "NS200BW"))
    if sub is None:
        raise ValueError(f"sampling mode {r0.get('sampleMode')} not implemented")
    t_max = float(r0["numelSample"]) / out_fs + pulse_dur + max_delay + rx_start
    n_fast = int(128 * math.ceil(t_max * out_fs / 128))
    n_freq = n_fast // 2
    freq = np.linspace(0, out_fs / 2, n_freq).astype(np.float32).astype(np.float64)
    c = float(Media["speedOfSound"])
    k = 2 * np.pi * freq / c
    k = k + 1j * (float(Media.get("attenuation", 0.0)) / 8.7 * k * c / (2 * np.pi * 1e4))
    n2 = int(math.ceil(n_fast * SIM_FS / out_fs))
    spec = lambda x, n: np.fft.fft(np.ravel(_arr(x)), n)[:n_freq]
    pulse = spec(x0["pulseShape"], n2)
    ir_tx = spec(TransTX["impulseResponse"], n2)
    ir_rx = spec(TransRX["impulseResponse"], n2)
    ipf = np.fft.fft(np.ravel(_arr(r0["InputFilter"])), n_fast)[:n_freq]
    delay = np.stack([np.ravel(_arr(t["Delay"])) for t in TXSI], 1)   # [n_ele_tx, n_tx]
    apod = np.stack([np.ravel(_arr(t["Apod"])) for t in TXSI], 1)
    rx_apod = np.stack([np.ravel(_arr(r.get("Apod", np.ones(pos_rx.shape[0])))) for r in
                        (RXSI if len(RXSI) == n_tx else RXSI * n_tx)], 1)  # [n_ele_rx, n_tx]
    return dict(pos_tx=pos_tx, pos_rx=pos_rx[:, :, :n_sub_rx], scat=scat, n_tx=n_tx, n_event=n_event, sub=sub,
                n_fast=n_fast, n_freq=n_freq, k=k, c=c, pulse=pulse, ir_tx=ir_tx, ir_rx=ir_rx, ipf=ipf,
                delay=delay - rx_start, apod=apod, rx_apod=rx_apod, numel=int(math.ceil(float(r0["numelSample"]))),
                tx=TransTX, rx=TransRX)


def _ele_layout(pos):
    """[n_ele, 5, n_sub] (x, y, z, az, el) -> float32 [n_sub][5][n_ele]."""
    return np.ascontiguousarray(np.transpose(pos, (2, 1, 0)), dtype=np.float32)


def _element_field(dev, r_scat, ele, k, trans, c, stream):
    """E [n_f][n_scat][n_ele] complex64 (device) through rcabf_sim_element_field."""
    n_f, n_scat = k.shape[0], r_scat.shape[1]
    n_sub, _, n_ele = ele.shape
    out = torch.empty((n_f, n_scat, n_ele), dtype=torch.complex64, device=dev)
    st = L.lib().rcabf_sim_element_field(
        C.c_void_p(out.data_ptr()), C.c_void_p(r_scat.data_ptr()), C.c_void_p(ele.data_ptr()),
        C.c_void_p(k.data_ptr()), float(np.ravel(trans["ElementWidth"])[0]),
        float(np.ravel(trans["ElementHeight"])[0]), float(np.ravel(trans["ElementElevationFocus"])[0]),
        int(np.ravel(trans["baffle"])[0]), float(trans["lensCorrection"]), float(c), n_scat, n_ele, n_f, n_sub,
        C.c_void_p(stream))
    L.check(st, "rcabf_sim_element_field")
    return out


def sim_us_rca(Media, TransTX, TransRX, TXSI, RXSI, Options=None, *, device=None, return_rf: bool = False):
    """Simulated raw channel data [fast time (I/Q interleaved), element, event]
    (float32 numpy, SimUS_CUDARCA.m's Raw); ``return_rf`` also returns the RF
    before sub-sampling."""
    if not torch.cuda.is_available():
        raise RuntimeError("the simulator runs on a CUDA device; no CPU path exists")
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else torch.device(device).index or 0)
    p = sim_plan(Media, TransTX, TransRX, TXSI, RXSI)
    n_tx, n_f, n_fast = p["n_tx"], p["n_freq"], p["n_fast"]
    cplx = lambda a: torch.from_numpy(np.asarray(a, np.complex64)).to(dev)
    k = cplx(p["k"])
    w = torch.from_numpy(np.real(p["k"]).astype(np.float32) * np.float32(p["c"])).to(dev)     # angular frequency
    tx_fac = (cplx(p["pulse"]).conj() * cplx(p["ir_tx"]).conj())                               # [f]
    rx_fac = cplx(p["ipf"]) * cplx(p["ir_rx"])                                                  # [f]
    delay = torch.from_numpy(p["delay"].astype(np.float32)).to(dev)                           # [e, tx]
    apod = torch.from_numpy(p["apod"].astype(np.float32)).to(dev)
    # transmit weights W[f][e][tx] = apod exp(i w (delay - t_rx))
    wtx = apod[None] * torch.polar(torch.ones_like(delay)[None].expand(n_f, -1, -1),
                                   w[:, None, None] * delay[None])
    rx_apod = torch.from_numpy(p["rx_apod"].astype(np.float32)).to(dev)                       # [e', tx]
    ele_tx = torch.from_numpy(_ele_layout(p["pos_tx"])).to(dev)
    ele_rx = torch.from_numpy(_ele_layout(p["pos_rx"])).to(dev)
    n_ele_rx = p["pos_rx"].shape[0]
    scat = p["scat"]
    n_event = p["n_event"]
    rf = torch.zeros((n_event, n_ele_rx, n_fast), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for frame in range(n_event // n_tx):
            ev = list(range(frame * n_tx, (frame + 1) * n_tx))
            pos = scat[:, :3, ev]                     # [s, 3, tx]
            bsc = torch.from_numpy(scat[:, 3, ev].astype(np.float32)).to(dev)   # [s, tx]
            same = all(np.array_equal(pos[:, :, 0], pos[:, :, j]) for j in range(1, n_tx))
            groups = [list(range(n_tx))] if same else [[j] for j in range(n_tx)]
            for grp in groups:
                r = torch.from_numpy(np.ascontiguousarray(pos[:, :, grp[0]].T, dtype=np.float32)).to(dev)
                e_tx = _element_field(dev, r, ele_tx, k, p["tx"], p["c"], stream)      # [f, s, e]
                e_rx = _element_field(dev, r, ele_rx, k, p["rx"], p["c"], stream)      # [f, s, e']
                idx = torch.as_tensor(grp, device=dev)
                txf = torch.bmm(e_tx, wtx[:, :, idx])                                 # [f, s, g]
                txf = txf * tx_fac[:, None, None] * bsc[None, :, idx]
                spec = torch.bmm(e_rx.transpose(1, 2), txf)                           # [f, e', g]
                spec = spec * rx_fac[:, None, None] * rx_apod[None, :, idx]
                sig = torch.fft.ifft(spec.conj(), n=n_fast, dim=0).real              # [t, e', g]
                rf[[ev[j] for j in grp]] += sig.permute(2, 1, 0)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    n = p["numel"]
    rf = rf[:, :, :n] if n_fast >= n else torch.nn.functional.pad(rf, (0, n - n_fast))
    sub = p["sub"]
    a = rf[:, :, 0::sub]
    b = rf[:, :, 1::sub]
    m = min(a.shape[2], b.shape[2])
    raw = torch.stack([a[:, :, :m], b[:, :, :m]], dim=3).reshape(n_event, n_ele_rx, 2 * m)
    raw_np = raw.permute(2, 1, 0).cpu().numpy()          # [fast time, element, event]
    if return_rf:
        return raw_np, rf.permute(2, 1, 0).cpu().numpy()
    return raw_np
