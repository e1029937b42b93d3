"""RCA delay-and-sum I/Q beamformer: Python drop-in over librcabf.

Two call styles:

``bf_rca(data, Geometry, Transmit, Param, Options=None) -> (dataBf, mask)``
    The reference wrapper ``bfVirtualSourceGeneric_RCA(data, Geometry,
    Transmit, Param, Options)`` (MATLAB/lib/beamformer/RCA/
    bfVirtualSourceGeneric_RCA.m:1-724) with MATLAB structs as dicts.  ``data``
    is indexed like the MATLAB array, [samples, x-channels, y-channels,
    events] (events = transmits x frames, transmit fastest); NumPy arrays give
    NumPy results, torch tensors give torch results on the same device.
    ``dataBf`` has shape size(gridBfX) + (1 or nTx, nFrame) and ``mask``
    size(gridBfX) + (1 or nTx,), both in MATLAB (column-major) order.

``BfIQRCA(Raw, pmig) -> IQ``
    The ``Python/beamformer`` call style (beamformer.py:33 ``BfIQFlatLinear``)
    for an RCA probe: a ``pmig`` parameter dict in, a compounded volume out.

Both run on the GPU through the C ABI (include/rcabf.h); there is no CPU
path.  ``Engine`` is the lower-level API: geometry handles kept resident on
the device and device tensors in/out, for batching and serving.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import math
import threading
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .params import Acquisition, RCAError, normalize

try:
    import torch
except ImportError as e:  # pragma: no cover
    raise ImportError("simu_rca_ab_b200 needs PyTorch for device memory and streams") from e


def _stream_ptr(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, torch.cuda.Stream):
        return stream.cuda_stream
    return int(stream)


@dataclass
class GeometryHandle:
    """A geometry built by librcabf and resident on one device."""
    ptr: int
    device: int
    n_pix: int
    n_tx: int
    n_ele: int
    grid_shape: tuple
    acq: Acquisition

    def sources(self):
        """(vs_x, vs_y, vs_z, min_dist) the library derived (RCA.m:527-558)."""
        out = [np.zeros(self.n_tx) for _ in range(4)]
        L.check(L.lib().rcabf_geometry_sources(C.c_void_p(self.ptr), *(L.dptr(a) for a in out)),
                "rcabf_geometry_sources")
        return tuple(out)


def _desc_from_acq(acq: Acquisition):
    """Fills an rcabf_geometry_desc; returns it and the arrays it points to."""
    g = acq.grid
    keep = [acq.ele_x, acq.ele_y, acq.ele_z, g.x, g.y, g.z]
    d = L.GeometryDesc()
    d.struct_size = C.sizeof(L.GeometryDesc)
    d.receive_x = 1 if acq.receive_x else 0
    d.n_ele = acq.n_ele
    d.pos_ele_x, d.pos_ele_y, d.pos_ele_z = (L.dptr(a) for a in keep[:3])
    d.aperture_x, d.aperture_y, d.aperture_z = acq.aperture
    d.grid_kind = g.kind
    d.n_z, d.n_x, d.n_y = g.n_z, g.n_x, g.n_y
    d.grid_x, d.grid_y, d.grid_z = (L.dptr(a) for a in keep[3:6])
    d.stride_z, d.stride_x, d.stride_y = g.stride_z, g.stride_x, g.stride_y
    d.n_tx = acq.n_tx
    d.use_theta = 1 if acq.use_theta else 0
    if acq.use_theta:
        keep += [acq.theta_x, acq.theta_y]
        d.theta_x, d.theta_y = L.dptr(acq.theta_x), L.dptr(acq.theta_y)
    else:
        keep += [acq.vs_x, acq.vs_y, acq.vs_z]
        d.vs_x, d.vs_y, d.vs_z = L.dptr(acq.vs_x), L.dptr(acq.vs_y), L.dptr(acq.vs_z)
    d.fs, d.fd, d.c, d.t0, d.fnumber = acq.fs, acq.fd, acq.c, acq.t0, acq.fnumber
    d.interp, d.lanczos_a, d.table_mode = acq.interp, acq.lanczos_a, acq.table_mode
    d.mask_transmit = 1 if acq.mask_transmit else 0
    if acq.ab_law is not None:
        keep.append(acq.ab_law)
        d.ab_law = L.dptr(acq.ab_law)
        d.ab_per_tx = 1 if acq.ab_per_tx else 0
    return d, keep


def _geom_key(acq: Acquisition, device: int) -> str:
    h = hashlib.sha1()
    g = acq.grid
    for a in (acq.ele_x, acq.ele_y, acq.ele_z, g.x, g.y, g.z, acq.theta_x, acq.theta_y, acq.vs_x,
              acq.vs_y, acq.vs_z, acq.ab_law):
        h.update(b"-" if a is None else np.ascontiguousarray(a).tobytes())
    h.update(repr((device, acq.receive_x, acq.aperture, g.kind, g.shape, g.n_z, g.n_x, g.n_y, g.stride_z,
                   g.stride_x, g.stride_y, acq.use_theta, acq.fs, acq.fd, acq.c, acq.t0, acq.fnumber,
                   acq.interp, acq.lanczos_a, acq.table_mode, acq.mask_transmit, acq.ab_per_tx)).encode())
    return h.hexdigest()


# rcabf_iq_dtype -> (torch dtype of the buffer, buffer elements per I/Q sample)
_IQ_TORCH = {L.IQ_C64: (torch.complex64, 1), L.IQ_C32: (torch.complex32, 1),
             L.IQ_BF16X2: (torch.bfloat16, 2), L.IQ_RF_F32: (torch.float32, 2)}


def _iq_dtype_of(t: "torch.Tensor", layout: str) -> int:
    if t.dtype == torch.complex64:
        return L.IQ_C64
    if t.dtype == torch.complex32:
        return L.IQ_C32
    raise TypeError(f"unsupported channel-data dtype {t.dtype}")


class Engine:
    """Device-resident beamforming engine: geometry cache + workspaces."""

    def __init__(self, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("simu_rca_ab_b200 needs a CUDA device (sm_100a); no CPU path exists")
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else
                                   torch.device(device).index or 0)
        self._geoms: dict[str, GeometryHandle] = {}
        self._ws: dict[int, torch.Tensor] = {}
        self._lock = threading.Lock()
        L.lib()

    # -- geometry ------------------------------------------------------------
    def geometry(self, acq: Acquisition, stream=None) -> GeometryHandle:
        key = _geom_key(acq, self.device.index)
        with self._lock:
            h = self._geoms.get(key)
        if h is not None:
            return h
        d, keep = _desc_from_acq(acq)
        out = C.c_void_p()
        with torch.cuda.device(self.device):
            st = L.lib().rcabf_create_geometry(C.byref(d), C.c_void_p(_stream_ptr(stream)), C.byref(out))
        if st != L.OK:
            raise RCAError(L.lib().rcabf_status_string(st).decode().split(":")[-1],
                           f"geometry rejected by librcabf (status {st})")
        n = [C.c_int64() for _ in range(3)]
        L.lib().rcabf_geometry_info(out, *(C.byref(x) for x in n))
        h = GeometryHandle(out.value, self.device.index, n[0].value, n[1].value, n[2].value,
                           acq.grid.shape, acq)
        with self._lock:
            self._geoms[key] = h
        del keep
        return h

    def close(self):
        with self._lock:
            for h in self._geoms.values():
                L.lib().rcabf_destroy_geometry(C.c_void_p(h.ptr))
            self._geoms.clear()
            self._ws.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- beamforming ---------------------------------------------------------
    def make_args(self, geom: GeometryHandle, iq: "torch.Tensor", *, iq_dtype: int, n_sample: int,
                  n_frame: int, out: "torch.Tensor", mask: "torch.Tensor | None", compound: bool,
                  storage: int = L.STORE_F32, kernel: int = L.KERNEL_AUTO, accumulate: bool = False,
                  frames_per_block: int = 0, per_channel: bool = False, host: bool = False) -> L.BeamformArgs:
        # The C ABI takes raw pointers: check every buffer holds what the
        # sizes claim before handing it over.  host: iq and out in host
        # memory (pinned for overlap) for run_host; the mask stays on the device.
        T = 1 if compound else geom.n_tx
        dt, per_sample = _IQ_TORCH[iq_dtype]
        if iq.dtype != dt:
            raise ValueError(f"channel data dtype {iq.dtype} does not match iq_dtype {iq_dtype} ({dt})")
        need_in = n_frame * geom.n_tx * geom.n_ele * n_sample * per_sample
        if n_frame < 1 or n_sample < 1 or iq.numel() < need_in or not iq.is_contiguous():
            raise ValueError(f"channel data holds {iq.numel()} elements, {need_in} needed "
                             f"({n_frame} frames x {geom.n_tx} tx x {geom.n_ele} elements x {n_sample} samples)")
        if per_channel and compound:
            raise ValueError("per-channel output has no compounding over transmits")
        n_out = n_frame * T * geom.n_pix * (geom.n_ele if per_channel else 1)
        if out.dtype != torch.complex64 or out.numel() < n_out or not out.is_contiguous():
            raise ValueError("out must be a contiguous complex64 tensor of ([element] x) frames x (1 or tx) x pixels")
        if mask is not None and (mask.dtype != torch.float32 or mask.numel() < T * geom.n_pix):
            raise ValueError("mask must be a float32 tensor of (1 or tx) x pixels")
        for t in ((mask,) if mask is not None else ()) + (() if host else (iq, out)):
            if t.device != self.device:
                raise ValueError(f"tensor on {t.device}, engine on {self.device}")
        if host and (iq.device.type != "cpu" or out.device.type != "cpu"):
            raise ValueError("host=True: channel data and output must be host tensors (pinned for overlap)")
        a = L.BeamformArgs()
        a.struct_size = C.sizeof(L.BeamformArgs)
        a.iq_dtype = iq_dtype
        a.iq = iq.data_ptr()
        a.n_sample, a.n_ch, a.n_tx, a.n_frame = n_sample, geom.n_ele, geom.n_tx, n_frame
        a.storage = storage
        a.compound = 1 if compound else 0
        a.out = out.data_ptr()
        a.mask = mask.data_ptr() if mask is not None else None
        a.accumulate = 1 if accumulate else 0
        a.kernel = kernel
        a.frames_per_block = frames_per_block
        a.per_channel = 1 if per_channel else 0
        return a

    def plan(self, geom: GeometryHandle, a: L.BeamformArgs) -> dict:
        """The launch plan librcabf picks for these arguments."""
        import json
        buf = C.create_string_buffer(1024)
        L.check(L.lib().rcabf_describe_plan(C.c_void_p(geom.ptr), C.byref(a), buf, 1024), "rcabf_describe_plan")
        return json.loads(buf.value.decode())

    def autotune(self, geom: GeometryHandle, a: L.BeamformArgs, iters: int = 1, stream=None) -> dict:
        """Times the fused kernel's launch choices on these arguments and keeps
        the fastest for this geometry, frame count and storage (rcabf_autotune):
        later calls plan with it.  Overwrites the arguments' output."""
        r = L.TuneResult()
        r.struct_size = C.sizeof(L.TuneResult)
        with torch.cuda.device(self.device):
            L.check(L.lib().rcabf_autotune(C.c_void_p(geom.ptr), C.byref(a), C.c_void_p(_stream_ptr(stream)),
                                           iters, C.byref(r)), "rcabf_autotune")
        return {f: getattr(r, f) for f, _ in L.TuneResult._fields_ if f not in ("struct_size", "reserved")}

    def workspace_bytes(self, geom: GeometryHandle, a: L.BeamformArgs) -> int:
        n = C.c_size_t()
        L.check(L.lib().rcabf_beamform_workspace_size(C.c_void_p(geom.ptr), C.byref(a), C.byref(n)),
                "rcabf_beamform_workspace_size")
        return n.value

    def _workspace(self, nbytes: int, stream_ptr: int) -> "torch.Tensor":
        ws = self._ws.get(stream_ptr)
        if ws is None or ws.numel() < nbytes:
            ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
            self._ws[stream_ptr] = ws
        return ws

    def run(self, geom: GeometryHandle, a: L.BeamformArgs, stream=None, workspace=None) -> None:
        """Launches one beamform (asynchronous on `stream`)."""
        sp = _stream_ptr(stream)
        need = self.workspace_bytes(geom, a)
        ws = workspace if workspace is not None else self._workspace(need, sp)
        a.workspace = ws.data_ptr() if need else None
        a.workspace_bytes = ws.numel() if need else 0
        with torch.cuda.device(self.device):
            L.check(L.lib().rcabf_beamform(C.c_void_p(geom.ptr), C.byref(a), C.c_void_p(sp)), "rcabf_beamform")

    def run_host(self, geom: GeometryHandle, a: L.BeamformArgs, frames_per_chunk: int = 0, stream=None,
                 workspace=None) -> None:
        """rcabf_beamform_host: channel data and output in host memory (args
        made with host=True), frames in chunks whose copies in and out
        overlap the beamforming of their neighbours.  Asynchronous on
        `stream`: synchronise it before reading the output."""
        sp = _stream_ptr(stream)
        n = C.c_size_t()
        L.check(L.lib().rcabf_beamform_host_workspace_size(C.c_void_p(geom.ptr), C.byref(a), frames_per_chunk,
                                                           C.byref(n)), "rcabf_beamform_host_workspace_size")
        ws = workspace if workspace is not None else self._workspace(n.value, sp)
        a.workspace = ws.data_ptr()
        a.workspace_bytes = ws.numel()
        with torch.cuda.device(self.device):
            L.check(L.lib().rcabf_beamform_host(C.c_void_p(geom.ptr), C.byref(a), frames_per_chunk, C.c_void_p(sp)),
                    "rcabf_beamform_host")

    def run_batch(self, geoms: list, args: list, workspaces: list, stream=None) -> None:
        """One persistent fused launch over several acquisitions."""
        n = len(geoms)
        arr = (L.BeamformArgs * n)()
        for i, (g, a, w) in enumerate(zip(geoms, args, workspaces)):
            a.workspace = w.data_ptr()
            a.workspace_bytes = w.numel()
            arr[i] = a
        gp = (C.c_void_p * n)(*[g.ptr for g in geoms])
        with torch.cuda.device(self.device):
            L.check(L.lib().rcabf_beamform_batch(n, gp, arr, C.c_void_p(_stream_ptr(stream))),
                    "rcabf_beamform_batch")

    def beamform(self, geom: GeometryHandle, iq: "torch.Tensor", *, n_sample: int | None = None,
                 iq_dtype: int | None = None, compound: bool = True, storage: int = L.STORE_F32,
                 kernel: int = L.KERNEL_AUTO, with_mask: bool = True, out=None, mask=None,
                 frames_per_block: int = 0, stream=None):
        """Beamforms device channel data laid out [frame][tx][element][sample].

        Returns (out [frame][1 or tx][pixel] complex64, mask [1 or tx][pixel]).
        """
        if iq_dtype is None:
            iq_dtype = _iq_dtype_of(iq, "iq")
        if n_sample is None:
            n_sample = iq.shape[-1]
        per = geom.n_tx * geom.n_ele * n_sample
        n_frame = iq.numel() // per if iq_dtype != L.IQ_RF_F32 else iq.numel() // (2 * per)
        if n_frame * per * (2 if iq_dtype == L.IQ_RF_F32 else 1) != iq.numel() or n_frame < 1:
            raise ValueError("channel data size is not frames x transmits x elements x samples")
        T = 1 if compound else geom.n_tx
        if out is None:
            out = torch.empty((n_frame, T, geom.n_pix), dtype=torch.complex64, device=self.device)
        if with_mask and mask is None:
            mask = torch.empty((T, geom.n_pix), dtype=torch.float32, device=self.device)
        a = self.make_args(geom, iq, iq_dtype=iq_dtype, n_sample=n_sample, n_frame=n_frame, out=out,
                           mask=mask if with_mask else None, compound=compound, storage=storage,
                           kernel=kernel, frames_per_block=frames_per_block)
        self.run(geom, a, stream=stream)
        return out, mask


_ENGINES: dict[int, Engine] = {}


def default_engine(device=None) -> Engine:
    dev = torch.cuda.current_device() if device is None else torch.device(device).index or 0
    e = _ENGINES.get(dev)
    if e is None:
        e = _ENGINES[dev] = Engine(dev)
    return e


def _prepare_data(data, acq: Acquisition, device):
    """Channel data -> device tensor in [event][channel][sample] memory order.

    ``data`` is indexed [samples, x-channels, y-channels, events]
    (RCA.m:470); channels = x-channels * y-channels (x fastest).  Complex
    data is I/Q; real data is I/Q interleaved along the samples with Q
    negated, IQ(n) = RF(2n) - i RF(2n+1) (RCA.m:475-477).
    """
    is_torch = isinstance(data, torch.Tensor)
    shape = tuple(data.shape)
    if len(shape) > 4:
        shape = shape[:3] + (int(np.prod(shape[3:])),)
    shape = shape + (1,) * (4 - len(shape))
    n_s, cx, cy, ne = shape
    if is_torch:
        t = data.reshape(data.shape[:3] + (-1,)) if data.dim() > 4 else data
        while t.dim() < 4:
            t = t.unsqueeze(-1)
        t = t.permute(3, 2, 1, 0)
        if t.is_complex():
            if t.dtype == torch.complex128:
                t = t.to(torch.complex64)
        else:
            t = t.to(torch.float32)
        t = t.to(device).contiguous()
    else:
        a = np.asarray(data)
        if a.ndim > 4:
            a = a.reshape(a.shape[:3] + (-1,), order="F")
        a = a.reshape(shape, order="F")
        if np.iscomplexobj(a):
            a = a.astype(np.complex64, copy=False)
        else:
            a = a.astype(np.float32, copy=False)
        flat = np.ascontiguousarray(a.transpose(3, 2, 1, 0))
        t = torch.from_numpy(flat).to(device)
    if t.is_complex():
        iq_dtype = L.IQ_C64 if t.dtype == torch.complex64 else L.IQ_C32
        n_sample = n_s
    else:
        if n_s % 2:
            raise RCAError("dataNotNumeric", "real (interleaved I/Q) data needs an even number of samples")
        iq_dtype = L.IQ_RF_F32
        n_sample = n_s // 2
    n_ch = cx * cy
    return t, iq_dtype, n_sample, n_ch, ne


def bf_rca(data, Geometry, Transmit, Param, Options=None, *, engine: Engine | None = None,
           stream=None, return_torch: bool | None = None):
    """Drop-in for ``bfVirtualSourceGeneric_RCA(data, Geometry, Transmit, Param, Options)``.

    Returns ``(dataBf, mask)`` with the reference's shapes (RCA.m:715-722):
    dataBf [*size(gridBfX), 1 or nTx, nFrame] complex64 and
    mask [*size(gridBfX), 1 or nTx] float32.
    """
    acq = normalize(data, Geometry, Transmit, Param, Options)
    eng = engine or default_engine()
    geom = eng.geometry(acq, stream=stream)
    t, iq_dtype, n_sample, n_ch, n_event = _prepare_data(data, acq, eng.device)
    if n_ch != geom.n_ele:
        raise RCAError("posEleInvalid", f"data has {n_ch} channels but {geom.n_ele} element positions")
    if n_event % geom.n_tx:
        raise RCAError("virtualSourcesNotSameLength",
                       f"{n_event} events are not a whole number of frames of {geom.n_tx} transmits")
    n_frame = n_event // geom.n_tx
    T = 1 if acq.compounding else geom.n_tx
    out = torch.empty((n_frame, T, geom.n_pix), dtype=torch.complex64, device=eng.device)
    mask = torch.empty((T, geom.n_pix), dtype=torch.float32, device=eng.device)
    a = eng.make_args(geom, t, iq_dtype=iq_dtype, n_sample=n_sample, n_frame=n_frame, out=out, mask=mask,
                      compound=acq.compounding, storage=acq.storage, kernel=acq.kernel,
                      frames_per_block=acq.frames_per_block)
    eng.run(geom, a, stream=stream)
    s1, s2, s3 = acq.grid.shape
    # [frame][tx][pixel], pixel column-major over the grid -> MATLAB order
    dataBf = out.view(n_frame, T, s3, s2, s1).permute(4, 3, 2, 1, 0)
    maskv = mask.view(T, s3, s2, s1).permute(3, 2, 1, 0)
    as_torch = isinstance(data, torch.Tensor) if return_torch is None else return_torch
    if as_torch:
        return dataBf, maskv
    return dataBf.cpu().numpy(), maskv.cpu().numpy()


def bf_rca_nosum(data, Geometry, Transmit, Param, Options=None, *, engine: Engine | None = None,
                 stream=None, return_torch: bool | None = None):
    """Drop-in for ``bfVirtualSourceGeneric_RCA_Nosum`` and, with
    ``Param.AbLawRx`` per element, ``bfVirtualSourceGeneric_RCA_Nosum_ab``
    (MATLAB/lib/beamformer/NoSum*/…_Nosum*.m): one beamformed value per
    receive element, no compounding.

    Returns ``(dataBf, mask)``: dataBf [*size(gridBfX), nTx, nFrame, nChannel]
    complex64 (Nosum.m:716-718) and mask [*size(gridBfX), nTx] float32.
    """
    acq = normalize(data, Geometry, Transmit, Param, Options)
    eng = engine or default_engine()
    geom = eng.geometry(acq, stream=stream)
    t, iq_dtype, n_sample, n_ch, n_event = _prepare_data(data, acq, eng.device)
    if n_ch != geom.n_ele:
        raise RCAError("posEleInvalid", f"data has {n_ch} channels but {geom.n_ele} element positions")
    if n_event % geom.n_tx:
        raise RCAError("virtualSourcesNotSameLength",
                       f"{n_event} events are not a whole number of frames of {geom.n_tx} transmits")
    n_frame = n_event // geom.n_tx
    T = geom.n_tx
    out = torch.empty((geom.n_ele, n_frame, T, geom.n_pix), dtype=torch.complex64, device=eng.device)
    mask = torch.empty((T, geom.n_pix), dtype=torch.float32, device=eng.device)
    # every frame in one launch (pc_das_kernel); Options.kernel = 'plain'
    # keeps the one-launch-per-frame kernel
    kern = L.KERNEL_PLAIN if acq.kernel == L.KERNEL_PLAIN else L.KERNEL_AUTO
    a = eng.make_args(geom, t, iq_dtype=iq_dtype, n_sample=n_sample, n_frame=n_frame, out=out, mask=mask,
                      compound=False, storage=acq.storage, kernel=kern, per_channel=True)
    eng.run(geom, a, stream=stream)
    s1, s2, s3 = acq.grid.shape
    dataBf = out.view(geom.n_ele, n_frame, T, s3, s2, s1).permute(5, 4, 3, 2, 1, 0)
    maskv = mask.view(T, s3, s2, s1).permute(3, 2, 1, 0)
    as_torch = isinstance(data, torch.Tensor) if return_torch is None else return_torch
    if as_torch:
        return dataBf, maskv
    return dataBf.cpu().numpy(), maskv.cpu().numpy()


def _pmig_acquisition(pmig: dict, n_ch: int, n_sample_iq: int):
    """Maps ``pmig`` keys (beamformer.py:45-111) onto the RCA structs."""
    p = dict(pmig)
    p.setdefault("c", 1540.0)
    p.setdefault("fc", 3e6)
    p.setdefault("lbd", p["c"] / p["fc"])
    p.setdefault("fs", 4 * p["fc"])
    p.setdefault("sub", 2)
    p.setdefault("fsIQ", p["fs"] / p["sub"])
    p.setdefault("pitch", p["lbd"])
    p.setdefault("theta", [0.0])
    p.setdefault("t0", 0.0)
    p.setdefault("dx", p["pitch"])
    p.setdefault("dy", p["dx"])
    p.setdefault("dz", p["lbd"])
    p.setdefault("Nx", n_ch)
    p.setdefault("Ny", 1)
    p.setdefault("Nz", n_ch)
    p.setdefault("Xmin", -(p["Nx"] - 1) * p["dx"] / 2)
    p.setdefault("Ymin", -(p["Ny"] - 1) * p["dy"] / 2)
    p.setdefault("Zmin", 0.0)
    p.setdefault("fnum", 1)
    rx_x = bool(p.get("receiveX", True))
    theta = np.atleast_1d(np.asarray(p["theta"], dtype=np.float64))
    pos = (np.arange(n_ch) - (n_ch - 1) / 2) * p["pitch"]
    zeros = np.zeros(n_ch)
    x = p["Xmin"] + np.arange(p["Nx"]) * p["dx"]
    y = p["Ymin"] + np.arange(p["Ny"]) * p["dy"]
    z = p["Zmin"] + np.arange(p["Nz"]) * p["dz"]
    X, Z, Y = np.meshgrid(x, z, y)          # [Nz, Nx, Ny] as in script_All.m:198
    ap = (n_ch - 1) * p["pitch"]
    G = {"gridBfX": X, "gridBfY": Y, "gridBfZ": Z,
         "posEleX": pos if rx_x else zeros, "posEleY": zeros if rx_x else pos, "posEleZ": zeros,
         "apertureX": ap, "apertureY": ap, "apertureZ": 0.0}
    Tr = {"thetaX": np.zeros_like(theta) if rx_x else theta,
          "thetaY": theta if rx_x else np.zeros_like(theta), "flagReceiveX": rx_x}
    Pa = {"samplingFrequency": p["fsIQ"], "demodulationFrequency": p["fc"], "speedOfSound": p["c"],
          "startTime": p["t0"], "fnumber": p["fnum"]}
    O = {"flagCompounding": True, "flagMaskTransmit": bool(p.get("maskTransmit", False))}
    order = p.get("order")
    if order is None or order <= 3:
        O["interpolation"] = "quadratic"
    elif order in (4, 6, 8):
        O["interpolation"] = "lanczos"
        O["lanczosOrder"] = order // 2
    else:
        raise ValueError(f"pmig['order'] = {order}: supported 3 (quadratic), 4, 6, 8 (Lanczos a = order/2)")
    for k in ("storage", "kernel", "tableMode"):
        if k in p:
            O[k] = p[k]
    return G, Tr, Pa, O, (int(p["Nz"]), int(p["Nx"]), int(p["Ny"]))


def BfIQRCA(Raw, pmig: dict, **kw):
    """RCA beamformer in the ``Python/beamformer`` call style.

    ``Raw`` is [NtIQ, Nchannel, Nevent] (or with extra trailing event axes),
    complex I/Q, or real with I and Q interleaved along the samples as in
    beamformer.py:118-120 (IQ = Raw[0::2] + 1j Raw[1::2]).  Events are
    transmits x frames, transmit fastest.  Extra ``pmig`` keys for the RCA
    probe: ``receiveX`` (receive on the x elements, transmit steered in y;
    default True), ``Ny``/``dy``/``Ymin`` (elevation grid), ``order``
    (3: quadratic; 4/6/8: Lanczos with order/2 lobes).  Returns the
    compounded volume IQ[Nz, Nx, Nframe] (IQ[Nz, Nx, Ny, Nframe] when Ny > 1).
    """
    is_torch = isinstance(Raw, torch.Tensor)
    if not is_torch:
        R = np.asarray(Raw)
        if R.ndim > 3:
            R = R.reshape(R.shape[0], R.shape[1], -1, order="F")
        if not np.iscomplexobj(R):
            R = R[0::2] + 1j * R[1::2]
        R = R.astype(np.complex64)
        nt, nch, nev = R.shape
        data = R.reshape(nt, nch, 1, nev, order="F")
    else:
        R = Raw
        if R.dim() > 3:
            R = R.reshape(R.shape[0], R.shape[1], -1)
        if not R.is_complex():
            R = torch.complex(R[0::2].float(), R[1::2].float())
        nt, nch, nev = R.shape
        data = R.unsqueeze(2)
    G, Tr, Pa, O, (nz, nx, ny) = _pmig_acquisition(pmig, nch, nt)
    import warnings
    from .params import RCAWarning
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RCAWarning)
        dataBf, _ = bf_rca(data, G, Tr, Pa, O, **kw)
    nframe = dataBf.shape[-1]
    if ny == 1:
        return dataBf.reshape(nz, nx, nframe) if not is_torch else dataBf[:, :, 0, 0, :]
    return dataBf[:, :, :, 0, :]
