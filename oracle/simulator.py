"""TEST INFRASTRUCTURE ONLY: the reference simulator run here, the checker of
simu_rca_ab_b200.simulator.

The reference's own field kernels TXfield / RXfield
(MATLAB/lib/simulator/SimUS_CUDARCA.cu:209-379), compiled from their source
for the host (oracle/_ref/libsim_ref_cpu.so, "O1") or for sm_100a
(libsim_ref_gpu_{strict,fast}.so, "O2"), driven by a numpy restatement of
the wrapper's host code (SimUS_CUDARCA.m:81-340): the same per-frame loop,
per-transmit receive fields, sums, inverse transforms and sub-sampling.
plan() restates the wrapper's host set-up (SimUS_CUDARCA.m:81-246):
sample counts, single-precision frequency grid and complex wavenumbers,
spectra of the pulse, impulse responses and input filter, delay and
apodisation laws.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_SIM_CPU = HERE / "_ref" / "libsim_ref_cpu.so"
LIB_SIM_GPU = {v: HERE / "_ref" / f"libsim_ref_gpu_{v}.so" for v in ("strict", "fast")}
_libs = {}


def _load(path):
    if path not in _libs:
        if not path.exists():
            raise FileNotFoundError(f"{path} missing (make -C oracle)")
        _libs[path] = C.CDLL(str(path))
    return _libs[path]


def have_sim_cpu():
    return LIB_SIM_CPU.exists()


def have_sim_gpu(v="strict"):
    return LIB_SIM_GPU[v].exists()


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _c(a):
    return np.ascontiguousarray(a, dtype=np.complex64)


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _scalars(trans, c):
    return [C.c_float(float(np.ravel(trans["ElementWidth"])[0])), C.c_float(float(np.ravel(trans["ElementHeight"])[0])),
            C.c_float(float(np.ravel(trans["ElementElevationFocus"])[0])), C.c_float(float(np.ravel(trans["baffle"])[0])),
            C.c_float(float(trans["lensCorrection"])), C.c_float(float(c))]


def txfield_cpu(r_scat, r_ele, k, pulse, ir, delay, apod, trans, c, n_sub):
    """O1 TXfield: r_scat [s, 3, tx] (MATLAB layout), r_ele [e, 5, sub];
    returns TX [tx][s][f] complex64 (the kernel's memory order)."""
    L = _load(LIB_SIM_CPU)
    n_s, _, n_tx = r_scat.shape
    n_e = r_ele.shape[0]
    n_f = k.shape[0]
    rs = _f(np.transpose(r_scat, (2, 1, 0)))     # memory: s fastest, then component, then tx
    re_ = _f(np.transpose(r_ele, (2, 1, 0)))
    out = np.zeros((n_tx, n_s, n_f), np.complex64)
    args = [_ptr(out), _ptr(rs), _ptr(re_), _ptr(_c(k)), _ptr(_c(pulse)), _ptr(_c(ir)),
            _ptr(_f(delay.T)), _ptr(_f(apod.T))] + _scalars(trans, c)
    args += [C.c_int(n_s), C.c_int(n_e), C.c_int(n_f), C.c_int(n_tx), C.c_int(n_sub), C.c_int(0)]
    L.sim_ref_cpu_txfield.restype = C.c_int
    assert L.sim_ref_cpu_txfield(*args) == 0
    return out


def rxfield_cpu(r_scat, r_ele, k, ir, trans, c, n_sub):
    """O1 RXfield: r_scat [s, 3]; returns RX [s][e][f] complex64."""
    L = _load(LIB_SIM_CPU)
    n_s = r_scat.shape[0]
    n_e = r_ele.shape[0]
    n_f = k.shape[0]
    rs = _f(r_scat.T)
    re_ = _f(np.transpose(r_ele, (2, 1, 0)))
    out = np.zeros((n_s, n_e, n_f), np.complex64)
    args = [_ptr(out), _ptr(rs), _ptr(re_), _ptr(_c(k)), _ptr(_c(ir))] + _scalars(trans, c)
    args += [C.c_int(n_s), C.c_int(n_e), C.c_int(n_f), C.c_int(n_sub), C.c_int(0)]
    L.sim_ref_cpu_rxfield.restype = C.c_int
    assert L.sim_ref_cpu_rxfield(*args) == 0
    return out


def txfield_gpu(variant, r_scat, r_ele, k, pulse, ir, delay, apod, trans, c, n_sub):
    """O2 TXfield on the GPU (torch for device memory); same layout as txfield_cpu."""
    import torch
    L = _load(LIB_SIM_GPU[variant])
    n_s, _, n_tx = r_scat.shape
    n_e = r_ele.shape[0]
    n_f = k.shape[0]
    t = lambda a: torch.from_numpy(a).cuda()
    rs = t(_f(np.transpose(r_scat, (2, 1, 0))))
    re_ = t(_f(np.transpose(r_ele, (2, 1, 0))))
    tensors = [t(_c(k)), t(_c(pulse)), t(_c(ir)), t(_f(delay.T)), t(_f(apod.T))]
    out = torch.zeros((n_tx, n_s, n_f), dtype=torch.complex64, device="cuda")
    p = lambda x: C.c_void_p(x.data_ptr())
    args = [p(out), p(rs), p(re_)] + [p(x) for x in tensors] + _scalars(trans, c)
    args += [C.c_int(n_s), C.c_int(n_e), C.c_int(n_f), C.c_int(n_tx), C.c_int(n_sub),
             C.c_void_p(torch.cuda.current_stream().cuda_stream)]
    L.sim_ref_gpu_txfield.restype = C.c_int
    assert L.sim_ref_gpu_txfield(*args) == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def rxfield_gpu(variant, r_scat, r_ele, k, ir, trans, c, n_sub):
    import torch
    L = _load(LIB_SIM_GPU[variant])
    n_s = r_scat.shape[0]
    n_e = r_ele.shape[0]
    n_f = k.shape[0]
    t = lambda a: torch.from_numpy(a).cuda()
    rs, re_, kk, irr = t(_f(r_scat.T)), t(_f(np.transpose(r_ele, (2, 1, 0)))), t(_c(k)), t(_c(ir))
    out = torch.zeros((n_s, n_e, n_f), dtype=torch.complex64, device="cuda")
    p = lambda x: C.c_void_p(x.data_ptr())
    args = [p(out), p(rs), p(re_), p(kk), p(irr)] + _scalars(trans, c)
    args += [C.c_int(n_s), C.c_int(n_e), C.c_int(n_f), C.c_int(n_sub),
             C.c_void_p(torch.cuda.current_stream().cuda_stream)]
    L.sim_ref_gpu_rxfield.restype = C.c_int
    assert L.sim_ref_gpu_rxfield(*args) == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def plan(Media, TransTX, TransRX, TXSI, RXSI) -> dict:
    """SimUS_CUDARCA.m:81-246 in numpy (structs as dicts, TXSI / RXSI as lists)."""
    import math
    fs_sim = 250e6                                         # :101
    ptx = np.asarray(TransTX["ElementPos"], float)
    ptx = ptx[:, :, None] if ptx.ndim == 2 else ptx
    prx = np.asarray(TransRX["ElementPos"], float) if TransRX else ptx
    prx = prx[:, :, None] if prx.ndim == 2 else prx
    trx = TransRX if TransRX else TransTX
    n_sub = ptx.shape[2]                                   # :88, :93 (the transmit count for both)
    sc = np.asarray(Media["scattererPos"], float)
    sc = sc[:, :, None] if sc.ndim == 2 else sc
    n_tx = len(TXSI)
    out_fs = float(RXSI[0]["samplingFrequency"])
    t_start = float(RXSI[0]["startTime"]) - 1.0 / float(TransTX["frequency"])          # :106
    d_max = max(float(np.max(t["Delay"])) for t in TXSI)                               # :108-111
    sub = {"NS200BW": 2, "BS100BW": 4, "BS50BW": 8}[RXSI[0].get("sampleMode", "NS200BW")]   # :114-131
    t_max = (float(RXSI[0]["numelSample"]) / out_fs + np.size(TXSI[0]["pulseShape"]) / fs_sim + d_max + t_start)
    n_fast = 128 * math.ceil(t_max * out_fs / 128)                                      # :136
    n_f = n_fast // 2
    f = np.linspace(0, out_fs / 2, n_f).astype(np.float32)                              # :138
    c = float(Media["speedOfSound"])
    kr = (2 * np.pi * f.astype(np.float64) / c)
    k = kr + 1j * (float(Media.get("attenuation", 0.0)) / 8.7 * kr * c / (2 * np.pi * 1e4))   # :141-143
    n2 = math.ceil(n_fast * fs_sim / out_fs)                                            # :160-162
    fft1 = lambda x, n: np.fft.fft(np.ravel(np.asarray(x, float)), n)[:n_f]
    rxsi = RXSI if len(RXSI) == n_tx else list(RXSI) * n_tx
    return dict(pos_tx=ptx, pos_rx=prx[:, :, :n_sub], scat=sc, n_tx=n_tx, n_event=sc.shape[2], sub=sub,
                n_fast=n_fast, n_freq=n_f, k=k, c=c, pulse=fft1(TXSI[0]["pulseShape"], n2),
                ir_tx=fft1(TransTX["impulseResponse"], n2), ir_rx=fft1(trx["impulseResponse"], n2),
                ipf=np.fft.fft(np.ravel(np.asarray(RXSI[0]["InputFilter"], float)), n_fast)[:n_f],
                delay=np.stack([np.ravel(t["Delay"]) for t in TXSI], 1) - t_start,
                apod=np.stack([np.ravel(t["Apod"]) for t in TXSI], 1),
                rx_apod=np.stack([np.ravel(r.get("Apod", np.ones(prx.shape[0]))) for r in rxsi], 1),
                numel=math.ceil(float(RXSI[0]["numelSample"])), tx=TransTX, rx=trx)


def simulate(plan) -> tuple[np.ndarray, np.ndarray]:
    """SimUS_CUDARCA.m:254-340 with the O1 field kernels: (Raw, RF), Raw
    [fast time, element, event] and RF [fast time, element, event]."""
    p = plan
    n_tx, n_f, n_fast = p["n_tx"], p["n_freq"], p["n_fast"]
    scat = p["scat"]
    n_event = p["n_event"]
    n_ele_rx = p["pos_rx"].shape[0]
    n_sub = p["pos_tx"].shape[2]
    rf = np.zeros((n_fast, n_ele_rx, n_event))
    for frame in range(n_event // n_tx):
        ev = list(range(frame * n_tx, (frame + 1) * n_tx))
        r_scat = scat[:, :3, ev]
        bsc = scat[:, 3, ev]                                    # [s, tx]
        tx = txfield_cpu(r_scat, p["pos_tx"], p["k"], p["pulse"], p["ir_tx"], p["delay"], p["apod"], p["tx"],
                         p["c"], n_sub)                          # [tx][s][f]
        tx = tx * bsc.T[:, :, None].astype(np.float32)
        tx[np.isnan(tx)] = 0
        for j in range(n_tx):
            rx = rxfield_cpu(r_scat[:, :, j], p["pos_rx"], p["k"], p["ir_rx"], p["rx"], p["c"], n_sub)  # [s][e][f]
            rx = rx * p["rx_apod"][:, j].astype(np.float32)[None, :, None]
            spec = np.einsum("sf,sef->fe", tx[j].astype(np.complex128), rx.astype(np.complex128)) * p["ipf"][:, None]
            sig = np.real(np.fft.ifft(np.conj(spec), n_fast, axis=0))
            rf[:, :, ev[j]] += sig
    n = p["numel"]
    rf = rf[:n] if n_fast >= n else np.concatenate([rf, np.zeros((n - n_fast, n_ele_rx, n_event))], 0)
    sub = p["sub"]
    a, b = rf[0::sub], rf[1::sub]
    m = min(a.shape[0], b.shape[0])
    raw = np.empty((2 * m, n_ele_rx, n_event))
    raw[0::2], raw[1::2] = a[:m], b[:m]
    return raw, rf
