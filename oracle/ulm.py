"""Test infrastructure: FP64 numpy restatement of the reference's ULM
super-localisation (Python/superloc/superloc.py), the checker for the GPU
path in simu_rca_ab_b200/ulm.py.  Only tests/, the smoke check and the CPU
baseline of bench.py use it; the product never calls it.

Parity unpinned: the reference runs on ArrayFire (arrayfire-python), which
is not installed here, so these functions restate its documented semantics
and are checked by known-answer cases, not against the reference's output.
The ArrayFire behaviours relied on:

* ``af.from_ndarray`` / ``to_ndarray`` keep numpy's logical indices.
* ``af.convolve3(signal, kernel)`` (CONV_MODE.DEFAULT): true convolution,
  zero outside the signal, output the size of the signal, kernel element
  ``K // 2`` (per dimension) on the output sample:
  ``out[i] = sum_f signal[i + K // 2 - f] * kernel[f]``; a 2-D kernel on a
  3-D signal convolves every slice along the third dimension.
* ``af.dilate(I, ones(3, 3))``: 3 x 3 maximum per slice; the maps dilated
  here are non-negative (or boolean), so the border value does not change
  the result.
* ``af.where`` lists linear indices in column-major order (dimension 0
  fastest); ``af.sort_index(..., is_ascending=False)`` orders by value,
  taken here as stable (ties keep the ``where`` order).
* ``af.inverse`` of the 3 x 3 fit matrices and the fit sums in float32; this
  restatement uses float64 (tests compare within a tolerance).
"""
from __future__ import annotations

import warnings

import numpy as np


def _conv_same_2d(sig: np.ndarray, ker: np.ndarray) -> np.ndarray:
    """ArrayFire convolve3 (DEFAULT mode) of every [:, :, t] slice with a
    2-D kernel: out[z, x] = sum_{a, b} sig[z + KZ//2 - a, x + KX//2 - b] * ker[a, b]."""
    nz, nx = sig.shape[:2]
    kz, kx = ker.shape
    out = np.zeros(sig.shape, dtype=np.result_type(sig.dtype, ker.dtype))
    for a in range(kz):
        dz = kz // 2 - a
        for b in range(kx):
            dx = kx // 2 - b
            z0, z1 = max(0, -dz), min(nz, nz - dz)
            x0, x1 = max(0, -dx), min(nx, nx - dx)
            if z0 >= z1 or x0 >= x1:
                continue
            out[z0:z1, x0:x1] += sig[z0 + dz:z1 + dz, x0 + dx:x1 + dx] * ker[a, b]
    return out


def _conv_same_t(sig: np.ndarray, ker: np.ndarray) -> np.ndarray:
    """ArrayFire convolve3 with a 1 x 1 x K kernel (along dimension 2)."""
    nt = sig.shape[2]
    k = ker.size
    out = np.zeros(sig.shape, dtype=np.result_type(sig.dtype, ker.dtype))
    for f in range(k):
        d = k // 2 - f
        t0, t1 = max(0, -d), min(nt, nt - d)
        if t0 < t1:
            out[:, :, t0:t1] += sig[:, :, t0 + d:t1 + d] * ker[f]
    return out


def psf_corr_map_2d(IQ: np.ndarray, psf: np.ndarray) -> np.ndarray:
    """PsfCorrMap2D (superloc.py:12-48): the PSF correlation map of every
    frame, normalised by the local energy under the PSF footprint and by the
    PSF norm.  (The batched form gives the same maps.)"""
    IQ = np.asarray(IQ, np.complex128)
    psf = np.asarray(psf, np.complex128)
    norm_psf = np.sqrt(np.sum(np.abs(psf) ** 2))
    mask = np.ones(psf.shape)
    with np.errstate(divide="ignore", invalid="ignore"):
        norm_iq = np.sqrt(_conv_same_2d(np.abs(IQ) ** 2, mask))
        return _conv_same_2d(IQ, np.conj(psf)) / norm_iq / norm_psf


def regional_max(I: np.ndarray, siz: int = 3) -> np.ndarray:
    """ImRegionalMax (superloc.py:51-53): dilate(I, ones(siz, siz)) == I, per slice."""
    I = np.asarray(I)
    r = siz // 2
    nz, nx = I.shape[:2]
    pad = np.full((nz + 2 * r, nx + 2 * r) + I.shape[2:], -np.inf)
    pad[r:r + nz, r:r + nx] = I
    dil = np.full(I.shape, -np.inf)
    for a in range(siz):
        for b in range(siz):
            dil = np.maximum(dil, pad[a:a + nz, b:b + nx])
    return dil == I


def _dilate_bool(B: np.ndarray) -> np.ndarray:
    nz, nx = B.shape[:2]
    pad = np.zeros((nz + 2, nx + 2) + B.shape[2:], bool)
    pad[1:1 + nz, 1:1 + nx] = B
    out = np.zeros(B.shape, bool)
    for a in range(3):
        for b in range(3):
            out |= pad[a:a + nz, b:b + nx]
    return out


def init_gaussian_fit(siz_filter: int = 5):
    """InitGaussianFit (superloc.py:56-100): the Hann-weighted moment
    matrices of the 1-D parabola fits and their inverses."""
    edge = siz_filter // 2 + 1
    roi = np.linspace(-edge, edge, 2 * edge + 1)
    roix, roiz = np.meshgrid(roi, roi)
    h = np.hanning(2 * edge + 1)
    hann = h[:, None] * h[None, :]
    ata_x = np.array([[np.sum(hann * roix ** (i + j)) for j in range(3)] for i in range(3)])
    ata_z = np.array([[np.sum(hann * roiz ** (i + j)) for j in range(3)] for i in range(3)])
    return roi, hann, roix, roiz, np.linalg.inv(ata_x), np.linalg.inv(ata_z)


def ensemble_map(M: np.ndarray, siz_ens: int = 5) -> np.ndarray:
    """sqrt|Hann-smoothed lag-1 product| along time (superloc.py:114-120)."""
    M = np.asarray(M, np.complex128)
    ker = np.hanning(siz_ens)
    ker = ker / np.sum(ker)
    P = M[:, :, :-1] * np.conj(M[:, :, 1:])
    return np.sqrt(np.abs(_conv_same_t(P, ker)))


def detection_mask(C: np.ndarray, E: np.ndarray, siz_filter: int = 5, fit: int = 0) -> np.ndarray:
    """The candidate mask of SuperLocFilter (superloc.py:124-136)."""
    edge = siz_filter // 2 + 1
    roi = np.zeros(C.shape, bool)
    roi[edge:C.shape[0] - edge, edge:C.shape[1] - edge, :] = True
    if fit == 0:
        bw = regional_max(C, 3) & _dilate_bool(regional_max(E, 3))
    else:
        bw = regional_max(E, 3)
    return bw & roi


def super_loc_filter(CorrMap: np.ndarray, IQmap: np.ndarray, siz_filter: int = 5, siz_ens: int = 5,
                     fit: int = 0) -> np.ndarray:
    """SuperLocFilter (superloc.py:103-213): PosLoc [5, N] = (x + sub-x, 0,
    z + sub-z, value, frame) of every candidate, by decreasing value."""
    nz, nx, _ = np.shape(CorrMap)
    edge = siz_filter // 2 + 1
    C = ensemble_map(CorrMap, siz_ens)
    E = ensemble_map(IQmap, siz_ens)
    bw = detection_mask(C, E, siz_filter, fit)
    lin = np.flatnonzero(bw.reshape(-1, order="F"))              # af.where: column-major
    src = C if fit == 0 else E
    val = np.abs(src.reshape(-1, order="F")[lin])
    order = np.argsort(-val, kind="stable")
    return gauss_fit(lin[order], val[order], src, siz_filter)


def gauss_fit(lin: np.ndarray, val: np.ndarray, amap: np.ndarray, siz_filter: int = 5, moments: bool = False):
    """The sub-pixel fit of SuperLocFilter (superloc.py:140-213) for the
    candidates `lin` (column-major linear indices into the fitted ensemble
    map `amap`, (Nz, Nx, Nt - 1)) with values `val`: PosLoc [5, N] (and,
    with ``moments``, the fitted parabola coefficients mx, mz [3, N])."""
    nz, nx = amap.shape[:2]
    n0, n1 = nz, nx
    edge = siz_filter // 2 + 1
    flat = np.asarray(amap).reshape(-1, order="F")
    lin = np.asarray(lin, np.int64)
    # the reference indexes meshgrid(ix, iz, it) flattened in Fortran order
    # with the column-major mask index (superloc.py:140-168)
    ix = (lin % (n0 * n1)) // n1
    iz = lin % n1
    it = lin // (n0 * n1)
    roi, hann, roix, roiz, ata_xm, ata_zm = init_gaussian_fit(siz_filter)
    atx = np.zeros((3, lin.size))
    atz = np.zeros((3, lin.size))
    for ixr in range(roi.size):
        for izr in range(roi.size):
            idx = (iz - edge + izr) + (ix - edge + ixr) * nz + it * nz * nx
            # inside the map for square maps; for non-square ones the
            # reference's index mapping can leave it (its result is then
            # undefined): NaN, as the GPU path
            ok = (idx >= 0) & (idx < flat.size)
            with np.errstate(divide="ignore"):
                lg = np.where(ok, np.log(np.abs(flat[np.where(ok, idx, 0)])), np.nan)
            w = hann[izr, ixr]
            atx[0] += lg * w
            atx[1] += lg * w * roix[izr, ixr]
            atx[2] += lg * w * roix[izr, ixr] ** 2
            atz[0] += lg * w
            atz[1] += lg * w * roiz[izr, ixr]
            atz[2] += lg * w * roiz[izr, ixr] ** 2
    mx = ata_xm @ atx
    mz = ata_zm @ atz
    with np.errstate(divide="ignore", invalid="ignore"):
        subx = -0.5 * mx[1] / mx[2]
        subz = -0.5 * mz[1] / mz[2]
    pos = np.zeros((5, lin.size))
    pos[0] = ix + subx
    pos[2] = iz + subz
    pos[3] = val
    pos[4] = it
    return (pos, mx, mz) if moments else pos


def _bins(v, bins):
    """The reference's bin index: int16 truncation, negatives to 0, past the
    last bin to the last bin, exactly the bin count to 0 (superloc.py:232-245)."""
    n = len(bins)
    with warnings.catch_warnings(), np.errstate(all="ignore"):
        warnings.simplefilter("ignore", RuntimeWarning)
        d = np.mean(np.diff(bins))                 # NaN for a single bin, as there
        i = ((np.asarray(v) - min(bins)) / d).astype(np.int16)
    i = (i > 0) * i
    return ((n - i) > 0) * i + ((n - i) < 0) * (n - 1)


def density_mapping_nd(pos, xbins=(0, 1), ybins=(0, 1), zbins=(0, 1)):
    """DensityMappingND (superloc.py:216-251)."""
    pos = np.asarray(pos)
    pos = pos.reshape(pos.shape[0], -1, order="F")
    ix, iy, iz = _bins(pos[0], xbins), _bins(pos[1], ybins), _bins(pos[2], zbins)
    dens = np.zeros((len(zbins), len(xbins), len(ybins)))
    np.add.at(dens, (iz, ix, iy), 1)
    return np.squeeze(dens)


def velocity_mapping_nd(pos, vel, xbins=(0, 1), ybins=(0, 1), zbins=(0, 1)):
    """VelocityMappingND (superloc.py:255-301): density and mean velocity."""
    pos = np.asarray(pos)
    vel = np.asarray(vel)
    pos = pos.reshape(pos.shape[0], -1, order="F")
    vel = vel.reshape(vel.shape[0], -1, order="F")
    ix, iy, iz = _bins(pos[0], xbins), _bins(pos[1], ybins), _bins(pos[2], zbins)
    dens = np.zeros((len(zbins), len(xbins), len(ybins)))
    velm = np.zeros((3, len(zbins), len(xbins), len(ybins)))
    np.add.at(dens, (iz, ix, iy), 1)
    for c in range(3):
        np.add.at(velm[c], (iz, ix, iy), vel[c])
    velm = velm.transpose((1, 2, 0, 3))
    with np.errstate(divide="ignore", invalid="ignore"):
        velm = np.squeeze(velm) / dens
    velm[np.isnan(velm)] = 0
    return np.squeeze(dens), velm


def density_mapping_ndt(pos, xbins=(0, 1), ybins=(0, 1), zbins=(0, 1), tbins=(0, 1)):
    """DensityMappingNDt (superloc.py:305-343): density per time bin (pos row 4)."""
    pos = np.asarray(pos)
    pos = pos.reshape(pos.shape[0], -1, order="F")
    ix, iy, iz = _bins(pos[0], xbins), _bins(pos[1], ybins), _bins(pos[2], zbins)
    it = _bins(pos[4], tbins)
    dens = np.zeros((len(zbins), len(xbins), len(ybins), len(tbins)))
    np.add.at(dens, (iz, ix, iy, it), 1)
    return np.squeeze(dens)


def velocity_mapping_ndt(pos, vel, xbins=(0, 1), ybins=(0, 1), zbins=(0, 1), tbins=(0, 1)):
    """VelocityMappingNDt (superloc.py:346-402)."""
    pos = np.asarray(pos)
    vel = np.asarray(vel)
    pos = pos.reshape(pos.shape[0], -1, order="F")
    vel = vel.reshape(vel.shape[0], -1, order="F")
    ix, iy, iz = _bins(pos[0], xbins), _bins(pos[1], ybins), _bins(pos[2], zbins)
    it = _bins(pos[4], tbins)
    shape = (len(zbins), len(xbins), len(ybins), len(tbins))
    dens = np.zeros(shape)
    velm = np.zeros((3,) + shape)
    np.add.at(dens, (iz, ix, iy, it), 1)
    for c in range(3):
        np.add.at(velm[c], (iz, ix, iy, it), vel[c])
    with np.errstate(divide="ignore", invalid="ignore"):
        for c in range(3):
            velm[c] = velm[c] / dens
    velm = np.squeeze(velm.transpose((1, 2, 3, 4, 0)))
    velm[np.isnan(velm)] = 0
    return np.squeeze(dens), velm
