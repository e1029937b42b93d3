"""ULM super-localisation on the GPU: drop-in for Python/superloc/superloc.py
(PsfCorrMap2D, ImRegionalMax, InitGaussianFit, SuperLocFilter,
DensityMappingND, VelocityMappingND, DensityMappingNDt, VelocityMappingNDt),
same names, arguments and results, with ArrayFire replaced by librcabf's
kernels (``rcabf_ulm_*``, csrc/ulm_kernels.cu).

Maps are (Nz, Nx, Nt) arrays as in the reference: numpy arrays in, numpy
arrays out; CUDA torch tensors in, CUDA torch tensors out (no host copy).
On the device a map is stored z fastest, then x, then frame -- the
column-major layout of the reference's ArrayFire arrays, so linear indices
(the detection order) mean the same on both sides.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _need_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("ULM runs on a CUDA device; no CPU path exists")


def _to_dev(a, dtype) -> tuple[torch.Tensor, bool]:
    """(Nz, Nx, Nt) array -> device tensor [Nt][Nx][Nz] of `dtype`; returns
    it and whether the input was numpy."""
    if isinstance(a, torch.Tensor):
        t = a if a.is_cuda else a.cuda()
        return t.to(dtype).permute(2, 1, 0).contiguous(), False
    arr = np.asarray(a)
    if arr.ndim == 2:
        arr = arr[:, :, None]
    t = torch.from_numpy(np.ascontiguousarray(arr.transpose(2, 1, 0)))
    return t.to(dtype).cuda(), True


def _from_dev(t: torch.Tensor, numpy_out: bool):
    """Device [Nt][Nx][Nz] -> (Nz, Nx, Nt)."""
    v = t.permute(2, 1, 0)
    return v.cpu().numpy() if numpy_out else v


def PsfCorrMap2D(IQ, psf, batchsize=0):
    """The PSF correlation map of every frame (superloc.py:12-48):
    conv(IQ, conj(psf)) / sqrt(conv(|IQ|^2, ones)) / ||psf||, ArrayFire's
    same-size convolution.  ``batchsize`` only split the reference's work;
    the result does not depend on it (it must still divide Nt, as there)."""
    _need_cuda()
    nt_in = np.shape(IQ)[2] if np.ndim(IQ) == 3 else 1
    if batchsize and nt_in % int(batchsize):
        raise ValueError("IQ must be decomposable into batches of batchsize frames")
    iq, numpy_out = _to_dev(IQ, torch.complex64)
    p = np.asarray(psf.cpu() if isinstance(psf, torch.Tensor) else psf).astype(np.complex64)
    if p.ndim != 2:
        raise ValueError("psf must be a 2-D kernel")
    norm = float(np.sqrt(np.sum(np.abs(p.astype(np.complex128)) ** 2)))
    psf_dev = torch.from_numpy(np.ascontiguousarray(p.T)).cuda()      # column-major kz x kx
    nt, nx, nz = iq.shape
    out = torch.empty_like(iq)
    L.check(L.lib().rcabf_ulm_psf_corr(C.c_void_p(out.data_ptr()), C.c_void_p(iq.data_ptr()),
                                       C.c_void_p(psf_dev.data_ptr()), norm, nz, nx, nt, p.shape[0], p.shape[1],
                                       _stream()), "rcabf_ulm_psf_corr")
    res = _from_dev(out, numpy_out)
    return res[:, :, 0] if (numpy_out and np.ndim(IQ) == 2) else res


def ImRegionalMax(I, SizKern=3):
    """dilate(I, ones(3, 3)) == I per frame (superloc.py:51-53)."""
    _need_cuda()
    if SizKern != 3:
        raise ValueError("ImRegionalMax: only the 3 x 3 neighbourhood the reference uses is implemented")
    m, numpy_out = _to_dev(I, torch.float32)
    nt, nx, nz = m.shape
    bw = torch.empty(m.shape, dtype=torch.uint8, device=m.device)
    L.check(L.lib().rcabf_ulm_regional_max(C.c_void_p(bw.data_ptr()), C.c_void_p(m.data_ptr()), nz, nx, nt,
                                           _stream()), "rcabf_ulm_regional_max")
    out = _from_dev(bw.bool(), numpy_out)
    return out[:, :, 0] if (numpy_out and np.ndim(I) == 2) else out


def InitGaussianFit(SizFilter=5):
    """(roi, Hann, Hannx, Hannx2, Hannz, Hannz2, AtAxm, AtAzm) of the
    Hann-weighted parabola fits (superloc.py:56-100), float32 numpy."""
    edge = int(SizFilter / 2) + 1
    roi = np.linspace(-edge, edge, 2 * edge + 1)
    roix, roiz = np.meshgrid(roi, roi)
    h = np.hanning(2 * edge + 1)
    hann = h[:, None] * h[None, :]
    hx, hz = hann * roix, hann * roiz
    ata_x = np.array([[np.sum(hann * roix ** (i + j)) for j in range(3)] for i in range(3)])
    ata_z = np.array([[np.sum(hann * roiz ** (i + j)) for j in range(3)] for i in range(3)])
    f = lambda a: np.asarray(a, np.float32)
    return (f(roi), f(hann), f(hx), f(hx * roix), f(hz), f(hz * roiz), f(np.linalg.inv(ata_x)),
            f(np.linalg.inv(ata_z)))


def _ensemble(m: torch.Tensor, siz_ens: int) -> torch.Tensor:
    nt, nx, nz = m.shape
    k = np.hanning(siz_ens)
    k = torch.from_numpy((k / np.sum(k)).astype(np.float32)).cuda()
    out = torch.empty((nt - 1, nx, nz), dtype=torch.float32, device=m.device)
    L.check(L.lib().rcabf_ulm_ensemble(C.c_void_p(out.data_ptr()), C.c_void_p(m.data_ptr()),
                                       C.c_void_p(k.data_ptr()), siz_ens, nz, nx, nt, _stream()),
            "rcabf_ulm_ensemble")
    return out


def _detect(Cm: torch.Tensor, Em: torch.Tensor, edge: int, fit: int):
    """Candidates in the reference's order: by decreasing value, ties in
    column-major (af.where) order."""
    nt1, nx, nz = Em.shape
    n = nt1 * nx * nz
    count = torch.zeros(1, dtype=torch.int64, device=Em.device)
    cap = n // 4 + 1024
    while True:
        lin = torch.empty(cap, dtype=torch.int64, device=Em.device)
        val = torch.empty(cap, dtype=torch.float32, device=Em.device)
        L.check(L.lib().rcabf_ulm_detect(C.c_void_p(lin.data_ptr()), C.c_void_p(val.data_ptr()),
                                         C.c_void_p(count.data_ptr()), C.c_void_p(Cm.data_ptr()),
                                         C.c_void_p(Em.data_ptr()), nz, nx, nt1, edge, fit, cap, _stream()),
                "rcabf_ulm_detect")
        k = int(count.item())
        if k <= cap:
            break
        cap = k
    lin, val = lin[:k], val[:k]
    lin, o = torch.sort(lin)                       # column-major order first
    val = val[o]
    val, o = torch.sort(val, descending=True, stable=True)
    return lin[o], val


def SuperLocFilter(CorrMap, IQmap, SizFilter=5, SizEns=5, fit=0):
    """PosLoc [5, N] (superloc.py:103-213): x + sub-x, 0, z + sub-z, value,
    frame of every candidate, by decreasing value."""
    _need_cuda()
    if fit not in (0, 1):
        raise ValueError("fit must be 0 (correlation map) or 1 (envelope)")
    cm, numpy_out = _to_dev(CorrMap, torch.complex64)
    em, _ = _to_dev(IQmap, torch.complex64)
    if cm.shape != em.shape:
        raise ValueError("CorrMap and IQmap must have the same shape")
    nt, nx, nz = cm.shape
    edge = int(SizFilter / 2) + 1
    Cm = _ensemble(cm, SizEns)
    Em = _ensemble(em, SizEns)
    lin, val = _detect(Cm, Em, edge, fit)
    roi, hann, _, _, _, _, axi, azi = InitGaussianFit(SizFilter)
    # hann[izr + w ixr] = Hann[izr, ixr]
    consts = np.concatenate([hann.T.reshape(-1), roi, axi.reshape(-1), azi.reshape(-1)]).astype(np.float32)
    consts = torch.from_numpy(consts).cuda()
    n = lin.numel()
    pos = torch.empty((5, n), dtype=torch.float32, device=cm.device)
    L.check(L.lib().rcabf_ulm_gauss_fit(C.c_void_p(pos.data_ptr()), C.c_void_p(lin.data_ptr()),
                                        C.c_void_p(val.data_ptr()), n,
                                        C.c_void_p((Cm if fit == 0 else Em).data_ptr()), nz, nx, nt - 1, edge,
                                        C.c_void_p(consts.data_ptr()), _stream()), "rcabf_ulm_gauss_fit")
    return pos.cpu().numpy() if numpy_out else pos


def _bins(bins_list, pos_rows, vel_rows=0) -> L.UlmBins:
    b = L.UlmBins()
    b.struct_size = C.sizeof(L.UlmBins)
    b.pos_rows, b.vel_rows = pos_rows, vel_rows
    for k, bins in enumerate(bins_list):
        bins = np.asarray(bins, np.float64)
        b.min[k] = float(np.min(bins))
        b.step[k] = float(np.mean(np.diff(bins))) if bins.size > 1 else float("nan")   # NaN, as np.mean of none
        b.n[k] = bins.size
    return b


def _histogram(pos, vel, bins_list, use_t):
    """Device histograms [nz][nx][ny][nt] (and [3][...]) of the positions."""
    _need_cuda()
    is_t = isinstance(pos, torch.Tensor)
    p = pos.detach().cpu().numpy() if is_t else np.asarray(pos)
    p = p.reshape(p.shape[0], -1, order="F")
    rows = p.shape[0]
    pd = torch.from_numpy(np.ascontiguousarray(p.T, dtype=np.float64)).cuda()        # [n][rows]
    n = pd.shape[0]
    vd, vrows = None, 0
    if vel is not None:
        v = vel.detach().cpu().numpy() if isinstance(vel, torch.Tensor) else np.asarray(vel)
        v = v.reshape(v.shape[0], -1, order="F")
        vrows = v.shape[0]
        vd = torch.from_numpy(np.ascontiguousarray(v.T, dtype=np.float64)).cuda()
    b = _bins(bins_list, rows, vrows)
    nx_, ny_, nz_ = b.n[0], b.n[1], b.n[2]
    nt_ = b.n[3] if use_t else 1
    dens = torch.zeros((nz_, nx_, ny_, nt_), dtype=torch.float64, device="cuda")
    velm = torch.zeros((3, nz_, nx_, ny_, nt_), dtype=torch.float64, device="cuda") if vel is not None else None
    L.check(L.lib().rcabf_ulm_density(C.c_void_p(dens.data_ptr()),
                                      C.c_void_p(velm.data_ptr()) if velm is not None else None,
                                      C.c_void_p(pd.data_ptr()), n,
                                      C.c_void_p(vd.data_ptr()) if vd is not None else None, C.byref(b),
                                      1 if use_t else 0, _stream()), "rcabf_ulm_density")
    d = dens.cpu().numpy()
    vm = velm.cpu().numpy() if velm is not None else None
    if not use_t:
        d = d[..., 0]
        vm = vm[..., 0] if vm is not None else None
    return d, vm


def DensityMappingND(pos, xbins=[0, 1], ybins=[0, 1], zbins=[0, 1]):
    """Localisation count per (z, x, y) bin (superloc.py:216-251)."""
    d, _ = _histogram(pos, None, (xbins, ybins, zbins), False)
    return np.squeeze(d)


def VelocityMappingND(pos, vel, xbins=[0, 1], ybins=[0, 1], zbins=[0, 1]):
    """(DensMap, mean velocity map) (superloc.py:255-301); the map's layout
    follows the reference's transposes and squeezes."""
    d, vm = _histogram(pos, vel, (xbins, ybins, zbins), False)
    vm = vm.transpose((1, 2, 0, 3))
    with np.errstate(divide="ignore", invalid="ignore"):
        vm = np.squeeze(vm) / d
    vm[np.isnan(vm)] = 0
    return np.squeeze(d), vm


def DensityMappingNDt(pos, xbins=[0, 1], ybins=[0, 1], zbins=[0, 1], tbins=[0, 1]):
    """Localisation count per (z, x, y, t) bin (superloc.py:305-343)."""
    d, _ = _histogram(pos, None, (xbins, ybins, zbins, tbins), True)
    return np.squeeze(d)


def VelocityMappingNDt(pos, vel, xbins=[0, 1], ybins=[0, 1], zbins=[0, 1], tbins=[0, 1]):
    """(DensMap, mean velocity map) per time bin (superloc.py:346-402)."""
    d, vm = _histogram(pos, vel, (xbins, ybins, zbins, tbins), True)
    with np.errstate(divide="ignore", invalid="ignore"):
        for c in range(3):
            vm[c] = vm[c] / d
    vm = np.squeeze(vm.transpose((1, 2, 3, 4, 0)))
    vm[np.isnan(vm)] = 0
    return np.squeeze(d), vm
