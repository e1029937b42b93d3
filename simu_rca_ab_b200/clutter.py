"""SVD clutter filter of a beamformed ensemble, on the GPU.

Drop-in for ``SVDClutterFilter(IQ, Mask, w, type)``
(MATLAB/lib/clutterFilter/SVDClutterFilter.m:1-45), the consumer of the
Doppler ensemble the beamformer produces:

1. weight each pixel by 1/sqrt(Mask) (the noise weight; ones by default);
2. Casorati Gram matrix G = C^H C of the [pixels x time] matrix C;
3. eigen-decomposition of G (Hermitian, nT x nT), components in descending
   order of eigenvalue (the singular values of the reference's svd(G));
4. keep the components the filter type selects from round(w * nT) and
   project: C_f = C V V^H.

Step 2 is the dense contraction (nT x nT x pixels; 2.4e11 real
multiply-adds for the C2 ensemble of 1.47M voxels x 200 frames).  The
reference forms it in double (the eigen-components the filter separates span
60 dB and more); here it runs on the int8 tensor cores
(``rcabf_casorati_gram``, casorati_gram.cu): every FP32 value is cut into
four 7-bit integer slices under a power-of-two scale per (frame part, chunk
of pixels), the slice products accumulate exactly in int32, and levels and
chunks combine in FP64 -- about 1e-10 of max|G| from an FP64 Gram.
``gram="fp64"`` forms it instead as a cuBLAS ZGEMM in FP64 (the comparator).
Step 3 runs in FP64 on the device (cuSOLVER through torch.linalg.eigh) on
the nT x nT matrix; step 4, the projection, is a CGEMM in FP32 with TF32 off
(its error is relative to the input magnitude, ~1e-7).

The beamformer's output [frame][pixel] is already the Casorati matrix's
transpose in memory (pixel fastest, as MATLAB's reshape(IQ, [], nT)), so no
copy is made.
"""
from __future__ import annotations

import numpy as np
import torch


def keep_components(n: int, w, kind: str = "band") -> np.ndarray:
    """Components (descending eigenvalue order) SVDClutterFilter.m keeps:
    Ncut = round(w * n); 'low' 1:Ncut(1), 'high' Ncut(1):end, 'stop'
    [1:Ncut(1), Ncut(2):end], otherwise ('band') Ncut(1):Ncut(2), 1-based
    and inclusive (SVDClutterFilter.m:12, 28-45)."""
    w = np.atleast_1d(np.asarray(w, dtype=np.float64))
    if w.min() < 0 or w.max() > 1:
        raise ValueError("w must be is the normalized cutoff frequency [0 1]")
    if kind in ("band", "stop") and w.size < 2:
        raise ValueError(f"a {kind} filter needs two cutoffs")
    ncut = np.floor(w * n + 0.5).astype(int)
    idx = np.arange(1, n + 1)
    if kind == "low":
        return idx <= ncut[0]
    if kind == "high":
        return idx >= ncut[0]
    if kind == "stop":
        return (idx <= ncut[0]) | (idx >= ncut[1])
    return (idx >= ncut[0]) & (idx <= ncut[1])


def gram_plan(n_frame: int, n_pix: int, chunk_voxels: int = 0) -> dict:
    """Tile plan of the tensor-core Gram (rcabf_gram_plan) as a dict."""
    import ctypes as C

    from . import _lib as L
    p = L.GramPlan()
    p.struct_size = C.sizeof(L.GramPlan)
    L.check(L.lib().rcabf_casorati_gram_plan(int(n_frame), int(n_pix), int(chunk_voxels), C.byref(p)),
            "rcabf_casorati_gram_plan")
    return {k: getattr(p, k) for k, _ in L.GramPlan._fields_ if k != "struct_size"}


def casorati_gram(x: torch.Tensor, chunk_voxels: int = 0, workspace: torch.Tensor | None = None) -> torch.Tensor:
    """G = conj(x) x^T (complex128, nT x nT) of a [frame][pixel] complex64
    CUDA tensor on the int8 tensor cores: the IQf' * IQf of
    SVDClutterFilter.m:25 with IQf = x^T.  Rows may be strided (pixels
    contiguous).  Raises if librcabf is missing (no other path)."""
    from . import _lib as L
    if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.complex64 and x.ndim == 2):
        raise ValueError("x must be a 2-D complex64 CUDA tensor [frame][pixel]")
    if x.stride(1) != 1:
        x = x.contiguous()
    n_t, n_pix = x.shape
    plan = gram_plan(n_t, n_pix, chunk_voxels)
    nbytes = int(plan["workspace_bytes"])
    if workspace is None or workspace.numel() < nbytes + 256:
        workspace = torch.empty(nbytes + 256, dtype=torch.uint8, device=x.device)
    base = workspace.data_ptr()
    ws = base + ((-base) % 256)
    g = torch.empty((n_t, n_t), dtype=torch.complex128, device=x.device)
    with torch.cuda.device(x.device):
        st = torch.cuda.current_stream(x.device).cuda_stream
        L.check(L.lib().rcabf_casorati_gram(g.data_ptr(), x.data_ptr(), n_t, n_pix, x.stride(0), int(chunk_voxels),
                                            ws, nbytes, st), "rcabf_casorati_gram")
    return g


def _casorati_t(iq: torch.Tensor, time_axis: int) -> torch.Tensor:
    """[time][pixels] view (or copy) of an ensemble."""
    x = iq.movedim(time_axis, 0)
    return x.reshape(x.shape[0], -1)


def svd_clutter_filter(IQ, Mask=None, w=(0.0, 1.0), type: str = "band", *, time_axis: int = -1,
                       order: str = "F", keep: np.ndarray | None = None, gram: str = "tensor_core"):
    """SVD clutter filter of an ensemble; returns (IQf, eig_val).

    IQ: complex tensor (CUDA) or array, time along ``time_axis``.  ``order``
    gives how pixels are laid out when IQ is a MATLAB-shaped array
    [Nz, Nx, Ny, nT] ('F': column-major, as bf_rca returns it; the filter
    itself does not depend on the pixel order).  Mask: per-pixel noise
    weights (same pixel shape), or None.  ``keep`` overrides (w, type) with
    an explicit boolean mask of components.  IQf has IQ's shape and stays
    weighted by 1/sqrt(Mask), as in the reference.  ``gram``: "tensor_core"
    (the int8 slice Gram) or "fp64" (cuBLAS ZGEMM).
    """
    if gram not in ("tensor_core", "fp64"):
        raise ValueError("gram must be 'tensor_core' or 'fp64'")
    if not torch.cuda.is_available():
        raise RuntimeError("the clutter filter runs on a CUDA device; no CPU path exists")
    as_numpy = not isinstance(IQ, torch.Tensor)
    t = torch.as_tensor(IQ) if not as_numpy else torch.from_numpy(np.ascontiguousarray(IQ) if order == "C"
                                                                   else np.asfortranarray(IQ))
    if not t.is_complex():
        raise ValueError("IQ must be complex")
    t = t.to("cuda", torch.complex64)
    shape = t.shape
    ax = time_axis % t.ndim
    # [time][pixel] with pixels in memory order of the non-time axes
    x = t.movedim(ax, 0)
    if order == "F" and t.ndim > 2:
        # column-major pixel order (MATLAB reshape): reverse the pixel axes
        x = x.permute(0, *range(x.ndim - 1, 0, -1))
    x = x.reshape(x.shape[0], -1).contiguous()
    n_t, n_pix = x.shape
    if Mask is not None:
        m = torch.as_tensor(np.asarray(Mask) if not isinstance(Mask, torch.Tensor) else Mask)
        m = m.to("cuda", torch.float32)
        if order == "F" and m.ndim > 1:
            m = m.permute(*range(m.ndim - 1, -1, -1))
        m = m.reshape(-1)
        if m.numel() != n_pix:
            raise ValueError("Mask must have one weight per pixel")
        x = x * torch.rsqrt(m)[None, :]
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        # G[i][j] = sum_p conj(x_i) x_j at FP64 accuracy (the reference forms
        # it in double: tissue clutter sits 40-60 dB above blood, so an FP32
        # Gram would blur the weak eigen-components the filter separates)
        if gram == "tensor_core":
            g = casorati_gram(x)
        else:
            x64 = x.to(torch.complex128)
            g = x64.conj() @ x64.T
            del x64
        ev, vec = torch.linalg.eigh(g)                         # ascending
        ev, vec = ev.flip(0), vec.flip(1)                      # descending, as svd(G)
        k = keep if keep is not None else keep_components(n_t, w, type)
        kt = torch.as_tensor(np.asarray(k, bool), device=x.device)
        v = vec[:, kt].to(torch.complex64)
        proj = v @ v.conj().T                                  # V V^H
        xf = proj.conj() @ x                                   # rows: (C V V^H)^T
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    # back to IQ's layout
    y = xf
    if order == "F" and t.ndim > 2:
        pix_shape = [shape[i] for i in range(len(shape)) if i != ax]
        y = y.reshape([n_t] + pix_shape[::-1]).permute(0, *range(len(pix_shape), 0, -1))
    else:
        y = y.reshape([n_t] + [shape[i] for i in range(len(shape)) if i != ax])
    y = y.movedim(0, ax)
    eig = ev.real
    if as_numpy:
        return y.cpu().numpy(), eig.cpu().numpy()
    return y, eig
