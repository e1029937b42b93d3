"""TEST INFRASTRUCTURE ONLY -- NumPy float64 restatement of the RCA
delay-and-sum model (MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.cu
lines 255-383 with exact arithmetic), vectorised over (pixel, element) per
transmit and frame.  It cross-checks the C oracle's FP64 mode
(oracle/rca_oracle.c:oracle_rca_fp64) on small cases.
"""
from __future__ import annotations

import numpy as np

from .host import INTERP_LANCZOS, INTERP_QUAD3, INTERP_REF6, RefArgs


def _sinc(x):
    return np.sinc(x)  # sin(pi x) / (pi x), 1 at 0


def weights(interp: int, a: int, d: np.ndarray):
    """(lo, [weights per tap]) for fractional offsets d in [0, 1)."""
    if interp == INTERP_QUAD3:                               # RCA.cu:355-357
        return 1, [d * (d - 1) / 2, -(d - 1) * (d + 1), d * (d + 1) / 2]
    if interp == INTERP_REF6:                                # RCA.cu:331-336
        return 2, [_sinc(d - (j - 2)) * _sinc((d - (j - 2)) / 2) for j in range(6)]
    ws = []
    for j in range(2 * a):                                   # Lanczos-a
        x = d - (j - (a - 1))
        ws.append(np.where(np.abs(x) < a, _sinc(x) * _sinc(x / a), 0.0))
    return a - 1, ws


def das_fp64(r: RefArgs, interp: int, a: int = 0, data=None):
    """Per-transmit output [frame][tx][pix] complex128 and mask [tx][pix]."""
    d = r.d64
    gx, gy, gz = d["gx"], d["gy"], d["gz"]
    ex, ey, ez = d["ex"], d["ey"], d["ez"]
    fs, fd, c, t0, F = d["fs"], d["fd"], d["c"], d["t0"], d["fnumber"]
    if data is None:
        iq = r.data[..., 0::2].astype(np.float64) + 1j * r.data[..., 1::2].astype(np.float64)
    else:
        iq = np.asarray(data).astype(np.complex128)
    nf, nt, nc, ns = iq.shape
    out = np.zeros((nf, nt, gx.size), np.complex128)
    mask = np.zeros((nt, gx.size))
    if r.mask_transmit:
        raise NotImplementedError("transmit cone not restated here; use oracle.host.run_fp64")
    lat_p = gx if r.receive_x else gy
    lat_e = ex if r.receive_x else ey
    ap = np.abs(lat_p[:, None] - lat_e[None, :])             # [P, E]
    apf = gz[:, None] / F
    valid = ap < apf
    apod = np.where(valid, 0.5 * (1 + np.cos(np.pi * ap / np.where(valid, apf, 1.0))), 0.0)
    drx = np.sqrt(ap ** 2 + (gz[:, None] - ez[None, :]) ** 2) / c
    for t in range(nt):
        if r.receive_x:
            dtx = (np.sqrt((gy - d["vsy"][t]) ** 2 + (gz - d["vsz"][t]) ** 2) - d["md"][t]) / c
        else:
            dtx = (np.sqrt((gx - d["vsx"][t]) ** 2 + (gz - d["vsz"][t]) ** 2) - d["md"][t]) / c
        mask[t] = apod.sum(1)
        idx = (dtx[:, None] + drx + t0) * fs
        fl = np.floor(idx)
        lo, ws = weights(interp, a, idx - fl)
        hi = len(ws) - 1 - lo
        ok = valid & (fl >= lo) & (fl < ns - 1 - hi)
        n0 = np.where(ok, fl, lo).astype(np.int64)
        rot = apod * np.exp(1j * (2 * np.pi * idx * fd / fs - 4 * np.pi * fd * gz[:, None] / c))
        rot = np.where(ok, rot, 0.0)
        e_idx = np.arange(nc)[None, :]
        for f in range(nf):
            s = np.zeros(idx.shape, np.complex128)
            for j, w in enumerate(ws):
                s += w * iq[f, t][e_idx, n0 - lo + j]
            out[f, t] = (s * rot).sum(1)
    return out, mask
