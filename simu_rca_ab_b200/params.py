"""Argument validation and normalisation for the RCA beamformer drop-in.

Mirrors the checks and defaults of the reference wrapper
``MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.m`` (lines 136-455):
the same fields, the same defaults, and the same error identifiers
(``RCAError.identifier`` is ``"bfVirtualSourceGeneric_RCA:<id>"``).  MATLAB
structs become Python dicts; ``islogical`` means a Python/NumPy bool;
``isnumeric`` excludes bools, as in MATLAB.
"""
from __future__ import annotations

import math
import numbers
import warnings
from dataclasses import dataclass, field

import numpy as np

MFILE = "bfVirtualSourceGeneric_RCA"


class RCAError(ValueError):
    """A reference wrapper error: ``identifier`` is the MATLAB error id."""

    def __init__(self, ident: str, message: str):
        self.identifier = f"{MFILE}:{ident}"
        super().__init__(f"{message} [{self.identifier}]")


class RCAWarning(UserWarning):
    """A reference wrapper warning (the MATLAB warning id is in the text)."""


def _warn(ident: str, message: str) -> None:
    warnings.warn(f"{message} [{MFILE}:{ident}]", RCAWarning, stacklevel=4)


def _is_bool(x) -> bool:
    return isinstance(x, (bool, np.bool_))


def _is_numeric_array(x) -> bool:
    try:
        import torch
        if isinstance(x, torch.Tensor):
            return x.dtype != torch.bool
    except ImportError:  # pragma: no cover
        pass
    if _is_bool(x):
        return False
    if isinstance(x, numbers.Number):
        return True
    a = np.asarray(x)
    return a.dtype.kind in "iufc"


def _is_numeric_scalar(x) -> bool:
    if _is_bool(x):
        return False
    if isinstance(x, numbers.Real):
        return True
    a = np.asarray(x)
    return a.dtype.kind in "iuf" and a.size == 1


def _scalar(x) -> float:
    return float(np.asarray(x).reshape(-1)[0])


def _vec(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, order="F"))


@dataclass
class GridSpec:
    """Voxel grid in the library's terms (rcabf_geometry_desc grid fields)."""
    kind: int                    # 0 rectilinear, 1 points
    shape: tuple                 # sizeGridBf: the grid array's own shape, padded to 3
    n_z: int
    n_x: int
    n_y: int
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    stride_z: int = 1
    stride_x: int = 0
    stride_y: int = 0

    @property
    def n_pix(self) -> int:
        return int(np.prod(self.shape))


def grid_spec(gx, gy, gz) -> GridSpec:
    """Classifies the beamforming grid.

    The reference takes three same-size coordinate arrays and flattens them
    column-major (RCA.m:491-493, 573), so pixel p is the Fortran linear index
    into the grid array.  When each coordinate varies along one array axis
    only (a meshgrid, e.g. ``meshgrid(x, z, y)`` giving [Nz, Nx, Ny] as in
    script_All.m:198) the grid is rectilinear and the library keeps separable
    tables; otherwise every pixel is an independent point.
    """
    X, Y, Z = (np.asarray(a, dtype=np.float64) for a in (gx, gy, gz))
    shape = tuple(X.shape) + (1,) * (3 - X.ndim) if X.ndim <= 3 else None
    if shape is None or X.ndim > 3:
        shape = (X.size, 1, 1)
    X3, Y3, Z3 = (a.reshape(shape, order="F") for a in (X, Y, Z))

    def varying_axes(a):
        axes = []
        for k in range(3):
            if shape[k] > 1:
                first = np.take(a, [0], axis=k)
                if not np.array_equal(a, np.broadcast_to(first, a.shape)):
                    axes.append(k)
        return axes

    vx, vy, vz = varying_axes(X3), varying_axes(Y3), varying_axes(Z3)
    rect = len(vx) <= 1 and len(vy) <= 1 and len(vz) <= 1
    if rect:
        used = [v[0] for v in (vx, vy, vz) if v]
        rect = len(set(used)) == len(used)
    if rect:
        free = [k for k in sorted(range(3), key=lambda k: shape[k]) if k not in [v[0] for v in (vx, vy, vz) if v]]
        ax = {}
        for name, v in (("x", vx), ("y", vy), ("z", vz)):
            ax[name] = v[0] if v else free.pop(0)
        rect = sorted(ax.values()) == [0, 1, 2]
    if rect:
        strides = (1, shape[0], shape[0] * shape[1])

        def axis_vec(a3, k):
            idx = [0, 0, 0]
            idx[k] = slice(None)
            return np.ascontiguousarray(a3[tuple(idx)], dtype=np.float64)

        return GridSpec(kind=0, shape=shape,
                        n_z=shape[ax["z"]], n_x=shape[ax["x"]], n_y=shape[ax["y"]],
                        x=axis_vec(X3, ax["x"]), y=axis_vec(Y3, ax["y"]), z=axis_vec(Z3, ax["z"]),
                        stride_z=strides[ax["z"]], stride_x=strides[ax["x"]], stride_y=strides[ax["y"]])
    n = int(np.prod(shape))
    return GridSpec(kind=1, shape=shape, n_z=n, n_x=1, n_y=1,
                    x=_vec(X3), y=_vec(Y3), z=_vec(Z3), stride_z=1, stride_x=0, stride_y=0)


@dataclass
class Acquisition:
    """Normalised Geometry / Transmit / Param / Options."""
    grid: GridSpec
    ele_x: np.ndarray
    ele_y: np.ndarray
    ele_z: np.ndarray
    aperture: tuple               # (x, y, z); NaN = derive from the elements
    use_theta: bool
    theta_x: np.ndarray | None
    theta_y: np.ndarray | None
    vs_x: np.ndarray | None
    vs_y: np.ndarray | None
    vs_z: np.ndarray | None
    receive_x: bool
    fs: float
    fd: float
    c: float
    t0: float
    fnumber: float
    lanczos_flag: bool
    compounding: bool
    mask_transmit: bool
    decrease_factor: int
    interp: int                   # rcabf_interp
    lanczos_a: int
    table_mode: int               # rcabf_table_mode
    storage: int                  # rcabf_storage
    kernel: int                   # rcabf_kernel
    frames_per_block: int
    ab_law: np.ndarray | None = None
    ab_per_tx: bool = False
    extra: dict = field(default_factory=dict)

    @property
    def n_tx(self) -> int:
        return int((self.theta_x if self.use_theta else self.vs_x).size)

    @property
    def n_ele(self) -> int:
        return int(self.ele_x.size)


_STORAGE = {"float32": 0, "single": 0, "fp32": 0, "float16": 1, "half": 1, "fp16": 1,
            "bfloat16": 2, "bf16": 2}
_KERNEL = {"auto": 0, "fused": 1, "plain": 2, "fused_noblock": 3, "fused_tmem": 4, "fused_regs": 5,
           "fused_tc": 6, "fused_tc_fp16w": 7}
_TABLES = {"exact": 0, "ref_compat": 1}


def normalize(data, Geometry, Transmit, Param, Options=None) -> Acquisition:
    """Checks and completes the reference structs (RCA.m:136-455)."""
    # --- data (RCA.m:137-149)
    if not _is_numeric_array(data):
        raise RCAError("dataNotNumeric", "Input data ('data') must be a numeric array!")
    # --- Options (RCA.m:153-197)
    if Options is None or (isinstance(Options, (list, tuple)) and len(Options) == 0):
        Options = {}
    if not isinstance(Options, dict):
        raise RCAError("OptionsNotStruct", "Options ('Options') must be a structure!")
    lanczos = Options.get("flagInterpolationLanczos", False)
    if not _is_bool(lanczos):
        raise RCAError("flagInterpolationLanczosInvalid",
                       "Interpolation method ('Options.flagInterpolationLanczos') is invalid; it must be a "
                       "boolean (true = Lanczos 5-lobes, false = quadratic)!")
    compounding = Options.get("flagCompounding", True)
    if not _is_bool(compounding):
        raise RCAError("flagCompoundingInvalid", "Compounding flag ('Options.flagCompounding') must be a boolean!")
    mask_tx = Options.get("flagMaskTransmit", True)
    if not _is_bool(mask_tx):
        raise RCAError("flagMaskTransmitInvalid", "Transmit mask flag ('Options.flagMaskTransmit') must be a boolean!")
    dec = Options.get("decreaseFactorGPU", 1)
    if not _is_numeric_scalar(dec) or math.floor(_scalar(dec)) != _scalar(dec) or _scalar(dec) < 0:
        raise RCAError("decreaseFactorGPUInvalid", "GPU decrease factor ('Options.decreaseFactorGPU') must be a positive integer!")

    # --- Geometry (RCA.m:200-306)
    G = Geometry if isinstance(Geometry, dict) else {}
    if not all(k in G for k in ("gridBfX", "gridBfY", "gridBfZ")):
        raise RCAError("gridBfMissing", "Beamforming grids ('Geometry.gridBfX', 'Geometry.gridBfY', and "
                                        "'Geometry.gridBfX')are required!")
    gX, gY, gZ = G["gridBfX"], G["gridBfY"], G["gridBfZ"]
    if (not all(_is_numeric_array(a) for a in (gX, gY, gZ))
            or not (np.size(gX) == np.size(gY) == np.size(gZ)) or np.size(gX) < 1):
        raise RCAError("gridBfInvalid", "Beamforming grids ('Geometry.gridBfX', 'Geometry.gridBfY', and "
                                        "'Geometry.gridBfX') must must be 3D numeric meshgrids and have the same size!")
    if not all(k in G for k in ("posEleX", "posEleY", "posEleZ")):
        raise RCAError("posEleMissing", "Element positions ('Geometry.posEleX', 'Geometry.posEleY', and "
                                        "'Geometry.posEleZ')are required!")
    eX, eY, eZ = G["posEleX"], G["posEleY"], G["posEleZ"]
    if (not all(_is_numeric_array(a) for a in (eX, eY, eZ))
            or not (np.size(eX) == np.size(eY) == np.size(eZ)) or np.size(eX) < 1):
        raise RCAError("posEleInvalid", "Pposition of the element ('Geometry.posEleX', 'Geometry.posEleY', and "
                                        "'Geometry.posEleZ') must be numeric arrays and have the same size!")
    aps = []
    for ax in "XYZ":
        key = f"aperture{ax}"
        if key not in G:
            _warn(f"aperture{ax}Default", f"Aperture along the {ax.lower()}-axis ('Param.aperture{ax}') is missing, "
                                          "the position of the elements will be used to estimate it.")
            aps.append(math.nan)
        elif not _is_numeric_scalar(G[key]):
            raise RCAError(f"aperture{ax}Invalid",
                           f"Aperture along the {ax.lower()}-axis ('Geometry.aperture{ax}') must be a single numeric value!")
        else:
            aps.append(_scalar(G[key]))

    # --- Transmit (RCA.m:309-379)
    if not isinstance(Transmit, dict):
        raise RCAError("TransmitNotStruct", "Transmit ('Transmit') must be a structure array!")
    has_theta = any(k in Transmit for k in ("thetaX", "thetaY"))
    has_vs = any(k in Transmit for k in ("virtualSourceX", "virtualSourceY", "virtualSourceZ"))
    theta_x = theta_y = vs_x = vs_y = vs_z = None
    if has_theta == has_vs:
        raise RCAError("ThetaORVirtualSourceRequired",
                       "Origin of the insonification(s) ('thetaX' and 'thetaY' OR 'virtualSourceX', 'virtualSourceY', "
                       "and 'virtualSourceZ') is required and must be unique (use either angle(s) OR virtual source(s))!")
    elif "thetaX" in Transmit and "thetaY" in Transmit:
        use_theta = True
        _warn("thetaToVirtualSource", "Tilt angles ('Transmit.thetaX' and 'Transmit.thetaY') will be converted to "
                                      "virtual source(s)")
        if np.size(Transmit["thetaX"]) != np.size(Transmit["thetaY"]):
            raise RCAError("tiltsNotSameLength", "Tilts ('Param.thetaX' and 'Param.thetaY')  must have the same length!")
        theta_x, theta_y = _vec(Transmit["thetaX"]), _vec(Transmit["thetaY"])
    elif all(k in Transmit for k in ("virtualSourceX", "virtualSourceY", "virtualSourceZ")):
        use_theta = False
        n = {np.size(Transmit[k]) for k in ("virtualSourceX", "virtualSourceY", "virtualSourceZ")}
        if len(n) != 1:
            raise RCAError("virtualSourcesNotSameLength", "Virtual sources ('Param.virtualSourceX', "
                                                          "'Param.virtualSourceY', and 'Param.virtualSourceZ') must have the same length!")
        vs_x, vs_y, vs_z = (_vec(Transmit[k]) for k in ("virtualSourceX", "virtualSourceY", "virtualSourceZ"))
    else:
        raise RCAError("ThetaORVirtualSourceInvalid",
                       "Origin of the insonification(s) ('thetaX' and 'thetaY' OR 'virtualSourceX', 'virtualSourceY', "
                       "and 'virtualSourceZ') is incorrect. Verify that all axes/positions are well defined and that "
                       "you are using either angle(s) OR virtual source(s))!")
    receive_x = Transmit.get("flagReceiveX", True)
    if not _is_bool(receive_x):
        raise RCAError("flagReceiveXInvalid", "Transmit receive channel flag ('Transmit.flagReceiveX') must be a boolean!")

    # --- Param (RCA.m:382-455)
    if not isinstance(Param, dict):
        raise RCAError("ParamNotStruct", "Parameters ('Param') must be a structure array!")
    if "samplingFrequency" not in Param:
        raise RCAError("samplingFrequencyMissing", "Sampling frequency ('Param.samplingFrequency') is required!")
    if not _is_numeric_scalar(Param["samplingFrequency"]):
        raise RCAError("samplingFrequencyInvalid", "Sampling frequency ('Param.samplingFrequency') must be a single numeric value!")
    if "demodulationFrequency" not in Param:
        raise RCAError("demodulationFrequencyMissing", "Demodulation frequency ('Param.demodulationFrequency') is required!")
    if not _is_numeric_scalar(Param["demodulationFrequency"]):
        raise RCAError("demodulationFrequencyInvalid", "Demodulation frequency ('Param.demodulationFrequency') must be a single numeric value!")
    if "speedOfSound" not in Param:
        c = 1540.0
        _warn("speedOfSoundDefault", "Speed of sound ('Param.speedOfSound') is missing, default = 1540 m/s.")
    elif not _is_numeric_scalar(Param["speedOfSound"]):
        raise RCAError("speedOfSoundInvalid", "Speed of sound  ('Param.speedOfSound') must be a single numeric value!")
    else:
        c = _scalar(Param["speedOfSound"])
    if "startTime" not in Param:
        t0 = 0.0
        _warn("startTimeDefault", "Start time ('Param.startTime') is missing, default = 0.")
    elif not _is_numeric_scalar(Param["startTime"]):
        raise RCAError("startTimeInvalid", "Start time ('Param.startTime') must be a single numeric value!")
    else:
        t0 = _scalar(Param["startTime"])
    if "fnumber" not in Param:
        fnumber = 1.0
        _warn("fnumberDefault", "F-number ('Param.fnumber') is missing, default = 1.")
    elif not _is_numeric_scalar(Param["fnumber"]):
        # the reference reports this with the start-time identifier (RCA.m:449-454)
        raise RCAError("startTimeInvalid", "F-number  ('Param.startTime') must be a single numeric value!")
    else:
        fnumber = _scalar(Param["fnumber"])

    # --- extensions of this library (Options fields the reference does not have)
    interp_name = Options.get("interpolation")
    a = int(Options.get("lanczosOrder", 3))
    if interp_name is None:
        interp = 1 if lanczos else 0
    else:
        interp = {"quadratic": 0, "quad3": 0, "ref6": 1, "lanczos5lobes": 1, "lanczos": 2}.get(str(interp_name).lower())
        if interp is None:
            raise RCAError("flagInterpolationLanczosInvalid", f"unknown interpolation {interp_name!r}")
    if interp == 2 and a not in (2, 3, 4):
        raise RCAError("flagInterpolationLanczosInvalid", f"Lanczos order must be 2, 3 or 4 (got {a})")
    tm = _TABLES.get(str(Options.get("tableMode", "exact")).lower())
    st = _STORAGE.get(str(Options.get("storage", "float32")).lower())
    kn = _KERNEL.get(str(Options.get("kernel", "auto")).lower())
    if tm is None or st is None or kn is None:
        raise ValueError("Options.tableMode / storage / kernel: unknown value")
    ab = Options.get("abLawRx", Param.get("AbLawRx"))
    ab_law, ab_per_tx = None, False
    if ab is not None:
        ab_law = np.asarray(ab, dtype=np.float64)
        ab_per_tx = ab_law.ndim == 2 and ab_law.shape[0] > 1 and ab_law.shape[1] > 1
        ab_law = np.ascontiguousarray(ab_law.reshape(-1, order="F"))  # [tx][element] as in ..._ab_2.cu:306

    return Acquisition(
        grid=grid_spec(gX, gY, gZ),
        ele_x=_vec(eX), ele_y=_vec(eY), ele_z=_vec(eZ), aperture=tuple(aps),
        use_theta=use_theta, theta_x=theta_x, theta_y=theta_y, vs_x=vs_x, vs_y=vs_y, vs_z=vs_z,
        receive_x=bool(receive_x), fs=_scalar(Param["samplingFrequency"]),
        fd=_scalar(Param["demodulationFrequency"]), c=c, t0=t0, fnumber=fnumber,
        lanczos_flag=bool(lanczos), compounding=bool(compounding), mask_transmit=bool(mask_tx),
        decrease_factor=int(_scalar(dec)), interp=interp, lanczos_a=a if interp == 2 else 0,
        table_mode=tm, storage=st, kernel=kn, frames_per_block=int(Options.get("framesPerBlock", 0)),
        ab_law=ab_law, ab_per_tx=ab_per_tx)
