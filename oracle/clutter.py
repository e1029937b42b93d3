"""TEST INFRASTRUCTURE ONLY: FP64 numpy restatement of the reference's SVD
clutter filter, the checker of simu_rca_ab_b200.clutter.

Follows MATLAB/lib/clutterFilter/SVDClutterFilter.m:1-45:
  IQf = IQ ./ sqrt(Mask)                       (:23, Mask = ones by default, :16-17)
  C   = reshape(IQf, [], nT)                   (:24, Casorati: pixels x time)
  [V, S] = svd(C' * C)                         (:25-26, in double)
  Ncut = round(w * nT)                         (:12)
  keep = 1:Ncut(1) ('low'), Ncut(1):end ('high'), [1:Ncut(1), Ncut(2):end]
         ('stop'), Ncut(1):Ncut(2) (otherwise, 'band')   (:28-45, 1-based)
  IQf = (C * V(:, keep)) * V(:, keep)'         (reshaped back, still weighted)
The Python version (Python/clutterfilter/SVDClutterFilter.py:10-23) keeps the
0-based half-open columns int(w0*nT):int(w1*nT) of a band instead.
Parity is unpinned: the reference runs in MATLAB (or ArrayFire), neither of
which exists here; this restatement is checked for self-consistency only.
"""
from __future__ import annotations

import numpy as np


def keep_matlab(n: int, w, kind: str = "band") -> np.ndarray:
    """Boolean mask over the n singular components (descending order) that
    SVDClutterFilter.m keeps for normalized cutoffs w and filter type."""
    w = np.atleast_1d(np.asarray(w, dtype=np.float64))
    if w.min() < 0 or w.max() > 1:
        raise ValueError("w must be is the normalized cutoff frequency [0 1]")
    ncut = np.floor(w * n + 0.5).astype(int)    # MATLAB round (half away from zero; w, n >= 0)
    idx = np.arange(1, n + 1)
    if kind == "low":
        k = idx <= ncut[0]
    elif kind == "high":
        k = idx >= ncut[0]
    elif kind == "stop":
        k = (idx <= ncut[0]) | (idx >= ncut[1])
    else:
        k = (idx >= ncut[0]) & (idx <= ncut[1])
    return k


def keep_python(n: int, wcut) -> np.ndarray:
    """Columns int(w0 n):int(w1 n) (0-based, half-open), SVDClutterFilter.py:14-20."""
    w = np.asarray(wcut, dtype=np.float64)
    k = np.zeros(n, bool)
    k[int(w[0] * n):int(w[1] * n)] = True
    return k


def svd_filter_fp64(iq: np.ndarray, mask=None, keep=None):
    """iq [..., nT] complex (time last, any pixel layout); returns
    (filtered [..., nT] complex128, eigenvalues descending)."""
    x = np.asarray(iq, dtype=np.complex128)
    shp = x.shape
    c = x.reshape(-1, shp[-1])
    if mask is not None:
        c = c / np.sqrt(np.asarray(mask, dtype=np.float64).reshape(-1))[:, None]
    g = c.conj().T @ c
    ev, vec = np.linalg.eigh(g)
    order = np.argsort(ev)[::-1]
    ev, vec = ev[order], vec[:, order]
    v = vec[:, keep]
    out = (c @ v) @ v.conj().T
    return out.reshape(shp), ev
