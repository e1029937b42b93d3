"""Frequency-domain ultrasound simulator on the GPU: drop-in for
``SimUS_CUDARCA(Media, TransTX, TransRX, TXSI, RXSI, Options)``
(MATLAB/lib/simulator/SimUS_CUDARCA.m), the producer of the RCA channel data
the beamformer consumes.

For each frame (nTX consecutive events) and each transmit event:

  TX(f, s)     = conj(P(f)) conj(IRtx(f)) sum_e E_tx(f, s, e) a_e exp(i w (d_e - t_rx)) * bsc(s)
  S(f, e')     = IPFilt(f) IRrx(f) a'_e' sum_s E_rx(f, s, e') TX(f, s)
  RF(:, e')   += real(ifft(conj(S(:, e')), nFastTime))

with E the element field (Green's function, directivities, lens phase), d /
a the transmit delays and apodisation, a' the receive apodisation, P / IR /
IPFilt the spectra of the pulse, impulse responses and input filter
(SimUS_CUDARCA.m:111-246, 254-322).  Three librcabf kernels per group of
events that share scatterer positions (a whole frame when the scatterers do
not move between its events, else one event), up to 16 transmits at a time:
``rcabf_sim_tx_field`` (TX, the element field evaluated in the sum over
elements), ``rcabf_sim_rx_spectrum`` (S, the receive field evaluated in the
sum over scatterers) and ``rcabf_sim_rf`` (the inverse transform as a direct
sum over the frequencies, evaluated only at the samples the output keeps).
The output Raw interleaves RF(1:sub:end) and RF(2:sub:end) as the reference
does (SimUS_CUDARCA.m:385-386), the quadrature-sampled layout the
beamformer's real-input path reads.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib as L

SIM_FS = 250e6      # sampling rate of pulse shapes and impulse responses (SimUS_CUDARCA.m:101)
SIM_GMAX = 16       # transmits one rcabf_sim_tx_field / rcabf_sim_rx_spectrum call takes
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


def _props(trans):
    """(width, height, elevation focus, baffle, lens correction) of an array,
    in the argument order of rcabf_sim_tx_field / rcabf_sim_rx_spectrum."""
    return (float(np.ravel(trans["ElementWidth"])[0]), float(np.ravel(trans["ElementHeight"])[0]),
            float(np.ravel(trans["ElementElevationFocus"])[0]), int(np.ravel(trans["baffle"])[0]),
            float(trans["lensCorrection"]))


def _out_samples(numel: int, sub: int) -> int:
    """Length of Raw along fast time: the interleave of RF(1:sub:end) and
    RF(2:sub:end), each cut to the shorter of the two."""
    return 2 * min(-(-numel // sub), -(-(numel - 1) // sub))


def sim_us_rca(Media, TransTX, TransRX, TXSI, RXSI, Options=None, *, device=None, return_rf: bool = False):
    """Simulated raw channel data [fast time (I/Q interleaved), element, event]
    (float32 numpy, SimUS_CUDARCA.m's Raw); ``return_rf`` also returns the RF
    before sub-sampling."""
    if not torch.cuda.is_available():
        raise RuntimeError("the simulator runs on a CUDA device; no CPU path exists")
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else torch.device(device).index or 0)
    p = sim_plan(Media, TransTX, TransRX, TXSI, RXSI)
    n_tx, n_f, n_fast = p["n_tx"], p["n_freq"], p["n_fast"]
    cplx = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.complex64)).to(dev)
    flt = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    k = cplx(p["k"])
    tx_fac = cplx(np.conj(p["pulse"]) * np.conj(p["ir_tx"]))                                  # [f]
    rx_fac = cplx(p["ipf"] * p["ir_rx"])                                                      # [f]
    delay = p["delay"].astype(np.float32)                                                     # [e, tx]
    apod = p["apod"].astype(np.float32)
    rx_apod = p["rx_apod"].astype(np.float32)                                                 # [e', tx]
    ele_tx = torch.from_numpy(_ele_layout(p["pos_tx"])).to(dev)
    ele_rx = torch.from_numpy(_ele_layout(p["pos_rx"])).to(dev)
    n_ele_rx = p["pos_rx"].shape[0]
    n_ele_tx, n_sub_tx, n_sub_rx = p["pos_tx"].shape[0], p["pos_tx"].shape[2], p["pos_rx"].shape[2]
    twiddle = cplx(np.exp(2j * np.pi * np.arange(n_fast) / n_fast))
    scat = p["scat"]
    n_event = p["n_event"]
    numel, sub = p["numel"], p["sub"]
    n_out = _out_samples(numel, sub)
    raw = torch.empty((n_event, n_ele_rx, n_out), dtype=torch.float32, device=dev)
    rf = torch.empty((n_event, n_ele_rx, numel), dtype=torch.float32, device=dev) if return_rf else None
    stream = torch.cuda.current_stream(dev).cuda_stream
    lib = L.lib()
    ptx, prx = _props(p["tx"]), _props(p["rx"])
    c = float(p["c"])
    for frame in range(n_event // n_tx):
        ev = list(range(frame * n_tx, (frame + 1) * n_tx))
        pos = scat[:, :3, ev]                     # [s, 3, tx]
        n_scat = pos.shape[0]
        same = all(np.array_equal(pos[:, :, 0], pos[:, :, j]) for j in range(1, n_tx))
        groups = [list(range(n_tx))] if same else [[j] for j in range(n_tx)]
        groups = [g[i:i + SIM_GMAX] for g in groups for i in range(0, len(g), SIM_GMAX)]
        for grp in groups:
            G = len(grp)
            r = flt(pos[:, :, grp[0]].T)                                      # [3][s]
            bsc = flt(scat[:, 3, [ev[j] for j in grp]].T)                    # [g][s]
            d = flt(delay[:, grp].T)                                          # [g][e]
            a = flt(apod[:, grp].T)
            ra = flt(rx_apod[:, grp].T)                                       # [g][e']
            txf = torch.empty((n_f, n_scat, G), dtype=torch.complex64, device=dev)
            L.check(lib.rcabf_sim_tx_field(
                C.c_void_p(txf.data_ptr()), C.c_void_p(r.data_ptr()), C.c_void_p(bsc.data_ptr()),
                C.c_void_p(ele_tx.data_ptr()), C.c_void_p(k.data_ptr()), C.c_void_p(tx_fac.data_ptr()),
                C.c_void_p(d.data_ptr()), C.c_void_p(a.data_ptr()), G, *ptx, c, n_scat, n_ele_tx, n_f, n_sub_tx,
                C.c_void_p(stream)), "rcabf_sim_tx_field")
            spec = torch.empty((n_f, n_ele_rx, G), dtype=torch.complex64, device=dev)
            L.check(lib.rcabf_sim_rx_spectrum(
                C.c_void_p(spec.data_ptr()), C.c_void_p(txf.data_ptr()), C.c_void_p(r.data_ptr()),
                C.c_void_p(ele_rx.data_ptr()), C.c_void_p(k.data_ptr()), C.c_void_p(rx_fac.data_ptr()),
                C.c_void_p(ra.data_ptr()), G, *prx, c, n_scat, n_ele_rx, n_f, n_sub_rx, C.c_void_p(stream)),
                "rcabf_sim_rx_spectrum")
            evs = [ev[j] for j in grp]
            e0, e1 = evs[0], evs[-1] + 1
            contiguous = evs == list(range(e0, e1))
            for buf, sb, n in ((raw, sub, n_out), (rf, 0, numel)):
                if buf is None or n == 0:
                    continue
                dst = buf[e0:e1] if contiguous else torch.empty((G, n_ele_rx, n), dtype=torch.float32, device=dev)
                L.check(lib.rcabf_sim_rf(C.c_void_p(dst.data_ptr()), C.c_void_p(spec.data_ptr()),
                                         C.c_void_p(twiddle.data_ptr()), n_f, n_ele_rx, G, n_fast, sb, n,
                                         C.c_void_p(stream)), "rcabf_sim_rf")
                if not contiguous:
                    buf[evs] = dst
    raw_np = raw.permute(2, 1, 0).cpu().numpy()          # [fast time, element, event]
    if return_rf:
        return raw_np, rf.permute(2, 1, 0).cpu().numpy()
    return raw_np
