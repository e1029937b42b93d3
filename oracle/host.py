"""TEST INFRASTRUCTURE ONLY -- the oracle's host side.

Nothing in the product imports this module; tests/, __graft_entry__.smoke()
and bench.py's accuracy and CPU-baseline legs use it as the checker.

``prepare`` restates the host preprocessing of the reference wrapper
MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.m for valid inputs:
  data layout       .m:470-485   (complex -> interleaved; real -> Q negated)
  grid flattening   .m:491-493   (column-major)
  element centring  .m:500-502
  apertures         .m:505-521
  virtual sources   .m:527-547   (r = 10 m)
  min distance      .m:551-558   (element Y paired with source X, as written)
  single casts      .m:459-464, 598-636
  compounding       .m:689-697   (sum over transmits; here sequential in
                                  transmit order, in single precision)
  output reshape    .m:715-722
and runs the same kernel arguments through
  O1  the reference kernel source compiled for the CPU (oracle/_ref/librca_ref_cpu.so)
  O2  the reference kernel source compiled for sm_100a (oracle/_ref/librca_ref_gpu_*.so)
  C32 the plain-C restatement of the reference arithmetic (oracle/_build/liboracle.so)
  F64 the double-precision delay-and-sum oracle (oracle/_build/liboracle.so)
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_ORACLE = HERE / "_build" / "liboracle.so"
LIB_REF_CPU = HERE / "_ref" / "librca_ref_cpu.so"
LIB_REF_GPU = {v: HERE / "_ref" / f"librca_ref_gpu_{v}.so" for v in ("strict", "fast", "default")}
# reference kernel variants (oracle/ref_variant.h): aberration law per element
# (ab1) or per (transmit, element) (ab2), one output per receive element
# (nosum), both (nosumab)
KERNEL_VARIANTS = ("ab1", "ab2", "nosum", "nosumab")
LIB_REF_CPU_VAR = {k: HERE / "_ref" / f"librca_ref_cpu_{k}.so" for k in KERNEL_VARIANTS}
LIB_REF_GPU_VAR = {k: HERE / "_ref" / f"librca_ref_gpu_strict_{k}.so" for k in KERNEL_VARIANTS}
_HAS_AB = {"base": False, "ab1": True, "ab2": True, "nosum": False, "nosumab": True}
_PER_CH = {"base": False, "ab1": False, "ab2": False, "nosum": True, "nosumab": True}

INTERP_QUAD3, INTERP_REF6, INTERP_LANCZOS = 0, 1, 2

_f = C.POINTER(C.c_float)
_d = C.POINTER(C.c_double)


def n_threads() -> int:
    return int(os.environ.get("ORACLE_THREADS", os.cpu_count() or 1))


@dataclass
class RefArgs:
    """The reference kernel's arguments (single precision) plus their
    double-precision sources for the FP64 oracle."""
    data: np.ndarray            # float32 [frame][tx][ch][2*ns] interleaved
    gx: np.ndarray
    gy: np.ndarray
    gz: np.ndarray
    ex: np.ndarray
    ey: np.ndarray
    ez: np.ndarray
    vsx: np.ndarray
    vsy: np.ndarray
    vsz: np.ndarray
    min_dist: np.ndarray
    receive_x: bool
    ap: tuple
    fs: float
    fd: float
    c: float
    t0: float
    fnumber: float
    n_pix: int
    n_ch: int
    n_tx: int
    n_frame: int
    n_sample: int               # I/Q samples per channel
    lanczos: bool
    mask_transmit: bool
    compounding: bool
    grid_shape: tuple
    d64: dict                   # double-precision versions


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).astype(np.float32))


def prepare(data, Geometry: dict, Transmit: dict, Param: dict, Options: dict | None = None) -> RefArgs:
    """RCA.m:459-636 for valid inputs.  ``data`` is indexed like the MATLAB
    array [samples, x-channels, y-channels, events]."""
    O = dict(Options or {})
    a = np.asarray(data)
    shape = a.shape + (1,) * (4 - a.ndim)
    a = a.reshape(shape, order="F")
    ns, cx, cy, ne = shape
    n_ch = cx * cy
    if np.iscomplexobj(a):                                   # .m:481-484
        flat = np.asfortranarray(a.astype(np.complex64)).reshape(-1, order="F")
        inter = np.empty(flat.size * 2, np.float32)
        inter[0::2], inter[1::2] = flat.real, flat.imag
        ns_iq = ns
    else:                                                    # .m:475-477
        inter = np.asfortranarray(a.astype(np.float32)).reshape(-1, order="F").copy()
        inter[1::2] = -inter[1::2]
        ns_iq = ns // 2
    G = Geometry
    gshape = np.shape(G["gridBfX"])
    gshape = tuple(gshape) + (1,) * (3 - len(gshape))
    gx64 = np.asarray(G["gridBfX"], float).reshape(-1, order="F")   # .m:491-493
    gy64 = np.asarray(G["gridBfY"], float).reshape(-1, order="F")
    gz64 = np.asarray(G["gridBfZ"], float).reshape(-1, order="F")
    ex64 = np.asarray(G["posEleX"], float).reshape(-1, order="F")
    ey64 = np.asarray(G["posEleY"], float).reshape(-1, order="F")
    ez64 = np.asarray(G["posEleZ"], float).reshape(-1, order="F")
    ex64, ey64, ez64 = ex64 - ex64.mean(), ey64 - ey64.mean(), ez64 - ez64.mean()   # .m:500-502
    ap = []
    for k, e in (("apertureX", ex64), ("apertureY", ey64), ("apertureZ", ez64)):   # .m:505-521
        ap.append(float(G[k]) if k in G else float(e.max() - e.min()))
    T = Transmit
    if "thetaX" in T:                                        # .m:527-541
        thx = np.asarray(T["thetaX"], float).ravel()
        thy = np.asarray(T["thetaY"], float).ravel()
        vz64 = -10.0 / np.sqrt(1 + np.tan(thx) ** 2 + np.tan(thy) ** 2)
        vx64, vy64 = vz64 * np.tan(thx), vz64 * np.tan(thy)
    else:
        vx64, vy64, vz64 = (np.asarray(T[k], float).ravel() for k in ("virtualSourceX", "virtualSourceY", "virtualSourceZ"))
    md64 = np.array([np.min(np.sqrt((ey64 - vx64[s]) ** 2 + (ex64 - vy64[s]) ** 2 + (ez64 - vz64[s]) ** 2))
                     for s in range(vx64.size)])             # .m:551-558
    n_tx = vx64.size
    n_pix = gx64.size
    n_frame = ne // n_tx                                     # .m:576-578
    P = Param
    c = float(P.get("speedOfSound", 1540.0))
    t0 = float(P.get("startTime", 0.0))
    fnum = float(P.get("fnumber", 1.0))
    data3 = inter.reshape(n_frame, n_tx, n_ch, 2 * ns_iq)
    return RefArgs(
        data=np.ascontiguousarray(data3, dtype=np.float32),
        gx=_f32(gx64), gy=_f32(gy64), gz=_f32(gz64), ex=_f32(ex64), ey=_f32(ey64), ez=_f32(ez64),
        vsx=_f32(vx64), vsy=_f32(vy64), vsz=_f32(vz64), min_dist=_f32(md64),
        receive_x=bool(T.get("flagReceiveX", True)),
        ap=tuple(float(np.float32(v)) for v in ap),
        fs=float(np.float32(P["samplingFrequency"])), fd=float(np.float32(P["demodulationFrequency"])),
        c=float(np.float32(c)), t0=float(np.float32(t0)), fnumber=float(np.float32(fnum)),
        n_pix=n_pix, n_ch=n_ch, n_tx=n_tx, n_frame=n_frame, n_sample=ns_iq,
        lanczos=bool(O.get("flagInterpolationLanczos", False)),
        mask_transmit=bool(O.get("flagMaskTransmit", True)),
        compounding=bool(O.get("flagCompounding", True)),
        grid_shape=gshape,
        d64=dict(gx=gx64, gy=gy64, gz=gz64, ex=ex64, ey=ey64, ez=ez64, vsx=vx64, vsy=vy64, vsz=vz64,
                 md=md64, ap=tuple(ap), fs=float(P["samplingFrequency"]),
                 fd=float(P["demodulationFrequency"]), c=c, t0=t0, fnumber=fnum))


# ---------------------------------------------------------------------------
def _p(a, t=_f):
    return a.ctypes.data_as(t)


_libs = {}


def _load(path: Path):
    if path not in _libs:
        if not path.exists():
            raise FileNotFoundError(f"{path} missing (make -C oracle)")
        _libs[path] = C.CDLL(str(path))
    return _libs[path]


def have_ref_cpu(kernel: str = "base") -> bool:
    return (LIB_REF_CPU if kernel == "base" else LIB_REF_CPU_VAR[kernel]).exists()


def have_ref_gpu(variant="strict", kernel: str = "base") -> bool:
    return (LIB_REF_GPU[variant] if kernel == "base" else LIB_REF_GPU_VAR[kernel]).exists()


def _ab_arg(kernel: str, ab_law):
    """The aberration law as the reference variants take it: float32 seconds,
    [element] (ab1, nosumab) or [transmit][element] (ab2)."""
    if not _HAS_AB[kernel]:
        return None
    if ab_law is None:
        raise ValueError(f"kernel variant {kernel} needs an aberration law")
    return np.ascontiguousarray(ab_law, dtype=np.float32).ravel()


def _kernel_args(r: RefArgs, data_ptr, out_ptr, mask_ptr, ptrs=None):
    ptrs = ptrs or {}
    g = lambda k: ptrs.get(k, _p(getattr(r, k)))
    return [out_ptr, mask_ptr, data_ptr, g("gx"), g("gy"), g("gz"), g("ex"), g("ey"), g("ez"),
            g("vsx"), g("vsy"), g("vsz"), g("min_dist"), C.c_int(int(r.receive_x)),
            C.c_float(r.ap[0]), C.c_float(r.ap[1]), C.c_float(r.ap[2]), C.c_float(r.fs), C.c_float(r.fd),
            C.c_float(r.c), C.c_float(r.t0), C.c_float(r.fnumber)]


def run_ref_cpu(r: RefArgs, threads: int | None = None, kernel: str = "base", ab_law=None):
    """O1: a reference kernel source on the host.  Returns per-transmit
    (dataBf [frame][tx][pix] complex64 -- [channel][frame][tx][pix] for the
    per-channel variants -- and mask [tx][pix])."""
    L = _load(LIB_REF_CPU if kernel == "base" else LIB_REF_CPU_VAR[kernel])
    shape = ((r.n_ch,) if _PER_CH[kernel] else ()) + (r.n_frame, r.n_tx, r.n_pix, 2)
    out = np.zeros(shape, np.float32)
    mask = np.zeros((r.n_tx, r.n_pix), np.float32)
    ab = _ab_arg(kernel, ab_law)
    args = _kernel_args(r, _p(r.data), _p(out), _p(mask))
    args.insert(-1, _p(ab) if ab is not None else None)   # AbLawRx comes before fnumber
    args += [C.c_int(r.n_pix), C.c_int(r.n_ch), C.c_int(r.n_tx), C.c_int(r.n_frame), C.c_int(r.n_sample),
             C.c_int(int(r.lanczos)), C.c_int(int(r.mask_transmit)), C.c_int(threads or n_threads())]
    L.rca_ref_cpu_run.restype = C.c_int
    assert L.rca_ref_cpu_run(*args) == 0
    return out[..., 0] + 1j * out[..., 1], mask


def run_c32(r: RefArgs, threads: int | None = None, per_channel=False, ab_law=None, ab_per_tx=False):
    """C restatement of the reference arithmetic (oracle/rca_oracle.c)."""
    L = _load(LIB_ORACLE)
    shape = (r.n_ch, r.n_frame, r.n_tx, r.n_pix, 2) if per_channel else (r.n_frame, r.n_tx, r.n_pix, 2)
    out = np.zeros(shape, np.float32)
    mask = np.zeros((r.n_tx, r.n_pix), np.float32)
    ab = None if ab_law is None else np.ascontiguousarray(ab_law, dtype=np.float32)
    args = _kernel_args(r, _p(r.data), _p(out), _p(mask))
    args += [C.c_int64(r.n_pix), C.c_int64(r.n_ch), C.c_int64(r.n_tx), C.c_int64(r.n_frame),
             C.c_int64(r.n_sample), C.c_int(int(r.lanczos)), C.c_int(int(r.mask_transmit)),
             C.c_int(int(per_channel)), _p(ab) if ab is not None else None, C.c_int(int(ab_per_tx)),
             C.c_int(threads or n_threads())]
    L.oracle_rca_fp32ref.restype = C.c_int
    assert L.oracle_rca_fp32ref(*args) == 0
    return out[..., 0] + 1j * out[..., 1], mask


def run_fp64(r: RefArgs, interp: int, lanczos_a: int = 0, data=None, threads: int | None = None,
             per_channel=False, ab_law=None, ab_per_tx=False, pix: np.ndarray | None = None):
    """Double-precision oracle on the same geometry.  ``data`` overrides the
    channel data ([frame][tx][ch][sample] complex); ``pix`` restricts the
    evaluation to a subset of pixel indices (returns those columns only)."""
    L = _load(LIB_ORACLE)
    d = r.d64
    if data is None:
        dat = r.data.astype(np.float64)
    else:
        dat = np.ascontiguousarray(np.asarray(data).astype(np.complex128)).view(np.float64)
    gx, gy, gz = d["gx"], d["gy"], d["gz"]
    if pix is not None:
        gx, gy, gz = (np.ascontiguousarray(a[pix]) for a in (gx, gy, gz))
    n_pix = gx.size
    shape = (r.n_ch, r.n_frame, r.n_tx, n_pix, 2) if per_channel else (r.n_frame, r.n_tx, n_pix, 2)
    out = np.zeros(shape, np.float64)
    mask = np.zeros((r.n_tx, n_pix), np.float64)
    dat = np.ascontiguousarray(dat)
    ab = None if ab_law is None else np.ascontiguousarray(ab_law, dtype=np.float64)
    L.oracle_rca_fp64.restype = C.c_int
    st = L.oracle_rca_fp64(
        _p(out, _d), _p(mask, _d), _p(dat, _d), None,
        _p(np.ascontiguousarray(gx), _d), _p(np.ascontiguousarray(gy), _d), _p(np.ascontiguousarray(gz), _d),
        _p(d["ex"], _d), _p(d["ey"], _d), _p(d["ez"], _d),
        _p(d["vsx"], _d), _p(d["vsy"], _d), _p(d["vsz"], _d), _p(d["md"], _d),
        C.c_int(int(r.receive_x)), C.c_double(d["ap"][0]), C.c_double(d["ap"][1]), C.c_double(d["ap"][2]),
        C.c_double(d["fs"]), C.c_double(d["fd"]), C.c_double(d["c"]), C.c_double(d["t0"]),
        C.c_double(d["fnumber"]),
        C.c_int64(n_pix), C.c_int64(r.n_ch), C.c_int64(r.n_tx), C.c_int64(r.n_frame), C.c_int64(r.n_sample),
        C.c_int(interp), C.c_int(lanczos_a), C.c_int(int(r.mask_transmit)), C.c_int(int(per_channel)),
        _p(ab, _d) if ab is not None else None, C.c_int(int(ab_per_tx)), C.c_int(threads or n_threads()))
    assert st == 0, st
    return out[..., 0] + 1j * out[..., 1], mask


def active_units(r: RefArgs, interp: int, lanczos_a: int = 0, threads: int | None = None) -> int:
    """Exact count of (pixel, rx, tx) inside the aperture and the sample window, per frame."""
    L = _load(LIB_ORACLE)
    d = r.d64
    lo, hi = {INTERP_QUAD3: (1, 1), INTERP_REF6: (2, 3)}.get(interp, (lanczos_a - 1, lanczos_a))
    L.oracle_rca_active_units.restype = C.c_int64
    return int(L.oracle_rca_active_units(
        _p(d["gx"], _d), _p(d["gy"], _d), _p(d["gz"], _d), _p(d["ex"], _d), _p(d["ey"], _d), _p(d["ez"], _d),
        _p(d["vsx"], _d), _p(d["vsy"], _d), _p(d["vsz"], _d), _p(d["md"], _d), C.c_int(int(r.receive_x)),
        C.c_double(d["fs"]), C.c_double(d["c"]), C.c_double(d["t0"]), C.c_double(d["fnumber"]),
        C.c_int64(r.n_pix), C.c_int64(r.n_ch), C.c_int64(r.n_tx), C.c_int64(r.n_sample),
        C.c_int(lo), C.c_int(hi), C.c_int(threads or n_threads())))


def run_ref_gpu(r: RefArgs, variant: str = "strict", kernel: str = "base", ab_law=None):
    """O2: a reference kernel source on the GPU (torch for device memory).
    Frames are chunked as the reference wrapper does (RCA.m:587-594).
    Per-channel variants return [channel][frame][tx][pix]."""
    import torch
    if kernel != "base" and variant != "strict":
        raise ValueError("the kernel variants are built strict only")
    L = _load(LIB_REF_GPU[variant] if kernel == "base" else LIB_REF_GPU_VAR[kernel])
    per_ch = _PER_CH[kernel]
    ab = _ab_arg(kernel, ab_law)
    L.rca_ref_gpu_launch.restype = C.c_int
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    tens = {k: t(getattr(r, k)) for k in ("gx", "gy", "gz", "ex", "ey", "ez", "vsx", "vsy", "vsz", "min_dist")}
    dptr = {k: C.cast(C.c_void_p(v.data_ptr()), _f) for k, v in tens.items()}
    max_siz = 2 ** 31 - 1
    n_chunks = int(np.ceil(2 * r.n_pix * r.n_tx * r.n_frame / max_siz))
    bounds = np.round(np.linspace(0, r.n_frame, n_chunks + 1)).astype(int)
    out = np.zeros(((r.n_ch,) if per_ch else ()) + (r.n_frame, r.n_tx, r.n_pix), np.complex64)
    mask = None
    mask_d = torch.zeros((r.n_tx, r.n_pix), dtype=torch.float32, device=dev)
    ab_d = t(ab) if ab is not None else None
    st = torch.cuda.current_stream().cuda_stream
    for k in range(n_chunks):
        f0, f1 = bounds[k], bounds[k + 1]
        dchunk = t(r.data[f0:f1])
        ob = torch.zeros(((r.n_ch,) if per_ch else ()) + (f1 - f0, r.n_tx, r.n_pix, 2), dtype=torch.float32,
                         device=dev)
        args = _kernel_args(r, C.cast(C.c_void_p(dchunk.data_ptr()), _f), C.cast(C.c_void_p(ob.data_ptr()), _f),
                            C.cast(C.c_void_p(mask_d.data_ptr()), _f), dptr)
        args.insert(-1, C.cast(C.c_void_p(ab_d.data_ptr()), _f) if ab_d is not None else None)
        args += [C.c_int(r.n_pix), C.c_int(r.n_ch), C.c_int(r.n_tx), C.c_int(int(f1 - f0)), C.c_int(r.n_sample),
                 C.c_int(int(r.lanczos)), C.c_int(int(r.mask_transmit)), C.c_void_p(st)]
        rc = L.rca_ref_gpu_launch(*args)
        assert rc == 0, rc
        torch.cuda.synchronize()
        o = ob.cpu().numpy()
        if per_ch:
            out[:, f0:f1] = o[..., 0] + 1j * o[..., 1]
        else:
            out[f0:f1] = o[..., 0] + 1j * o[..., 1]
        if mask is None:
            mask = mask_d.cpu().numpy().copy()
    return out, mask


def time_ref_gpu(r: RefArgs, variant: str = "fast", iters: int = 2, warmup: int = 1):
    """Times O2 -- the reference kernel on the GPU -- the way the reference
    wrapper runs it (bfVirtualSourceGeneric_RCA.m:587-594 frame chunks so that
    2*nPix*nTx*nFrame < 2^31, .m:640-650 launch shape, .m:689-697 compounding
    sum over transmits on the device), with the channel data already resident
    on the device.  Returns (ms per run over all of r's frames, chunks)."""
    import torch
    L = _load(LIB_REF_GPU[variant])
    L.rca_ref_gpu_launch.restype = C.c_int
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    tens = {k: t(getattr(r, k)) for k in ("gx", "gy", "gz", "ex", "ey", "ez", "vsx", "vsy", "vsz", "min_dist")}
    dptr = {k: C.cast(C.c_void_p(v.data_ptr()), _f) for k, v in tens.items()}
    n_chunks = int(np.ceil(2 * r.n_pix * r.n_tx * r.n_frame / (2 ** 31 - 1)))
    bounds = np.round(np.linspace(0, r.n_frame, n_chunks + 1)).astype(int)
    fmax = int(np.max(np.diff(bounds)))
    data_d = t(r.data)
    mask_d = torch.zeros((r.n_tx, r.n_pix), dtype=torch.float32, device=dev)
    ob = torch.empty((fmax, r.n_tx, r.n_pix, 2), dtype=torch.float32, device=dev)
    comp = torch.empty((r.n_frame, r.n_pix, 2), dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream()

    def run():
        for k in range(n_chunks):
            f0, f1 = int(bounds[k]), int(bounds[k + 1])
            d = C.cast(C.c_void_p(data_d[f0:f1].data_ptr()), _f)
            args = _kernel_args(r, d, C.cast(C.c_void_p(ob.data_ptr()), _f),
                                C.cast(C.c_void_p(mask_d.data_ptr()), _f), dptr)
            args.insert(-1, None)
            args += [C.c_int(r.n_pix), C.c_int(r.n_ch), C.c_int(r.n_tx), C.c_int(f1 - f0), C.c_int(r.n_sample),
                     C.c_int(int(r.lanczos)), C.c_int(int(r.mask_transmit)), C.c_void_p(st.cuda_stream)]
            assert L.rca_ref_gpu_launch(*args) == 0
            torch.sum(ob[: f1 - f0], dim=1, out=comp[f0:f1])

    for _ in range(warmup):
        run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(iters):
        run()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / iters, n_chunks


def compound(per_tx: np.ndarray, mask_tx: np.ndarray, compounding: bool = True):
    """RCA.m:689-697: sum over transmits (sequential, single precision)."""
    if not compounding:
        return per_tx, mask_tx
    acc = per_tx[:, 0].copy()
    for t in range(1, per_tx.shape[1]):
        acc = (acc + per_tx[:, t]).astype(per_tx.dtype)
    m = mask_tx[0].copy()
    for t in range(1, mask_tx.shape[0]):
        m = (m + mask_tx[t]).astype(mask_tx.dtype)
    return acc[:, None], m[None]


def matlab_shape(r: RefArgs, dataBf: np.ndarray, mask: np.ndarray):
    """RCA.m:715-722: [Nz, Nx, Ny, (tx), frame] column-major."""
    s1, s2, s3 = r.grid_shape
    F, T, P = dataBf.shape
    db = dataBf.reshape(F, T, s3, s2, s1).transpose(4, 3, 2, 1, 0)
    mk = mask.reshape(T, s3, s2, s1).transpose(3, 2, 1, 0)
    return db, mk


def error_db(y: np.ndarray, ref: np.ndarray):
    """(rms_dB, peak_dB) of y against ref."""
    y = np.asarray(y).astype(np.complex128).ravel()
    ref = np.asarray(ref).astype(np.complex128).ravel()
    d = y - ref
    rms = 20 * np.log10(np.linalg.norm(d) / max(np.linalg.norm(ref), 1e-300) + 1e-300)
    peak = 20 * np.log10(np.abs(d).max() / max(np.abs(ref).max(), 1e-300) + 1e-300)
    return float(rms), float(peak)


def rel_rms(y, ref) -> float:
    y = np.asarray(y).astype(np.complex128).ravel()
    ref = np.asarray(ref).astype(np.complex128).ravel()
    return float(np.linalg.norm(y - ref) / max(np.linalg.norm(ref), 1e-300))
