"""ctypes binding of librcabf (the C ABI declared in include/rcabf.h).

The shared library is built in-tree (``python -m simu_rca_ab_b200.build``)
and loaded from this package directory.  There is no fallback: if the
library is missing, importing the beamformer raises.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "librcabf.so"

# enums (include/rcabf.h)
INTERP_QUAD3, INTERP_REF6, INTERP_LANCZOS = 0, 1, 2
TABLES_EXACT, TABLES_REF_COMPAT = 0, 1
GRID_RECTILINEAR, GRID_POINTS = 0, 1
IQ_C64, IQ_C32, IQ_BF16X2, IQ_RF_F32 = 0, 1, 2, 3
STORE_F32, STORE_F16, STORE_BF16 = 0, 1, 2
KERNEL_AUTO, KERNEL_FUSED, KERNEL_PLAIN, KERNEL_FUSED_NOBLOCK, KERNEL_FUSED_TMEM, KERNEL_FUSED_REGS = 0, 1, 2, 3, 4, 5
KERNEL_FUSED_TC, KERNEL_FUSED_TC_FP16W = 6, 7

OK = 0
ERR_UNSUPPORTED = 102
ERR_OOM_ADMISSION = 104
ERR_TIMEOUT = 105
ERR_BUSY = 110
ERR_PENDING = 111

_dp = C.POINTER(C.c_double)


class GeometryDesc(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32), ("receive_x", C.c_int32),
        ("n_ele", C.c_int64),
        ("pos_ele_x", _dp), ("pos_ele_y", _dp), ("pos_ele_z", _dp),
        ("aperture_x", C.c_double), ("aperture_y", C.c_double), ("aperture_z", C.c_double),
        ("grid_kind", C.c_int32), ("reserved0", C.c_int32),
        ("n_z", C.c_int64), ("n_x", C.c_int64), ("n_y", C.c_int64),
        ("grid_x", _dp), ("grid_y", _dp), ("grid_z", _dp),
        ("stride_z", C.c_int64), ("stride_x", C.c_int64), ("stride_y", C.c_int64),
        ("n_tx", C.c_int64),
        ("use_theta", C.c_int32), ("reserved1", C.c_int32),
        ("theta_x", _dp), ("theta_y", _dp),
        ("vs_x", _dp), ("vs_y", _dp), ("vs_z", _dp),
        ("fs", C.c_double), ("fd", C.c_double), ("c", C.c_double), ("t0", C.c_double),
        ("fnumber", C.c_double),
        ("interp", C.c_int32), ("lanczos_a", C.c_int32), ("table_mode", C.c_int32),
        ("mask_transmit", C.c_int32),
        ("ab_law", _dp), ("ab_per_tx", C.c_int32), ("reserved2", C.c_int32),
    ]


class BeamformArgs(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32), ("iq_dtype", C.c_int32),
        ("iq", C.c_void_p),
        ("n_sample", C.c_int64), ("n_ch", C.c_int64), ("n_tx", C.c_int64), ("n_frame", C.c_int64),
        ("storage", C.c_int32), ("compound", C.c_int32),
        ("out", C.c_void_p), ("mask", C.c_void_p),
        ("accumulate", C.c_int32), ("kernel", C.c_int32),
        ("workspace", C.c_void_p), ("workspace_bytes", C.c_size_t),
        ("frames_per_block", C.c_int32), ("reserved0", C.c_int32),
        ("stage_events", C.POINTER(C.c_void_p)),
        ("per_channel", C.c_int32), ("reserved1", C.c_int32),
    ]


class TuneResult(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32), ("voxel_blocked", C.c_int32), ("frames_per_block", C.c_int32),
        ("tile_u", C.c_int32), ("tile_v", C.c_int32), ("tile_z", C.c_int32),
        ("window_rows", C.c_int32), ("candidates", C.c_int32),
        ("best_ms", C.c_double), ("default_ms", C.c_double),
        ("tensor_core", C.c_int32), ("reserved", C.c_int32),
    ]


class ServerConfig(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32), ("device", C.c_int32),
        ("hbm_budget_bytes", C.c_size_t),
        ("n_streams", C.c_int32), ("max_queue", C.c_int32),
        ("max_batch", C.c_int32), ("batch_window_us", C.c_int32),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32), ("reserved", C.c_int32),
        ("submitted", C.c_int64), ("completed", C.c_int64), ("rejected", C.c_int64),
        ("launches", C.c_int64), ("in_flight", C.c_int64), ("queued", C.c_int64),
        ("p50_ms", C.c_double), ("p95_ms", C.c_double), ("p99_ms", C.c_double),
        ("mean_ms", C.c_double), ("max_ms", C.c_double),
        ("units_done", C.c_double), ("busy_s", C.c_double), ("span_s", C.c_double),
        ("arena_bytes", C.c_size_t), ("arena_peak_bytes", C.c_size_t),
    ]


class UlmBins(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32), ("pos_rows", C.c_int32), ("vel_rows", C.c_int32), ("reserved", C.c_int32),
        ("min", C.c_double * 4), ("step", C.c_double * 4), ("n", C.c_int64 * 4),
    ]


class GramPlan(C.Structure):
    _fields_ = [
        ("struct_size", C.c_int32), ("chunk_voxels", C.c_int32), ("n_chunks", C.c_int32),
        ("column_block", C.c_int32), ("n_tiles", C.c_int32), ("launches", C.c_int32),
        ("workspace_bytes", C.c_size_t), ("mma_int_ops", C.c_double),
    ]


# Every symbol include/rcabf.h declares, with its ctypes signature.
_SIGS = {
    "rcabf_status_string": (C.c_char_p, [C.c_int]),
    "rcabf_abi_version": (C.c_int, []),
    "rcabf_last_error": (C.c_char_p, []),
    "rcabf_create_geometry": (C.c_int, [C.POINTER(GeometryDesc), C.c_void_p, C.POINTER(C.c_void_p)]),
    "rcabf_destroy_geometry": (C.c_int, [C.c_void_p]),
    "rcabf_geometry_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64)]),
    "rcabf_geometry_sources": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "rcabf_beamform_workspace_size": (C.c_int, [C.c_void_p, C.POINTER(BeamformArgs), C.POINTER(C.c_size_t)]),
    "rcabf_beamform": (C.c_int, [C.c_void_p, C.POINTER(BeamformArgs), C.c_void_p]),
    "rcabf_describe_plan": (C.c_int, [C.c_void_p, C.POINTER(BeamformArgs), C.c_char_p, C.c_size_t]),
    "rcabf_beamform_batch": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), C.POINTER(BeamformArgs), C.c_void_p]),
    "rcabf_beamform_noalloc": (C.c_int, [C.c_void_p, C.POINTER(BeamformArgs), C.c_void_p]),
    "rcabf_beamform_host_workspace_size": (C.c_int, [C.c_void_p, C.POINTER(BeamformArgs), C.c_int32,
                                                     C.POINTER(C.c_size_t)]),
    "rcabf_beamform_host": (C.c_int, [C.c_void_p, C.POINTER(BeamformArgs), C.c_int32, C.c_void_p]),
    "rcabf_autotune": (C.c_int, [C.c_void_p, C.POINTER(BeamformArgs), C.c_void_p, C.c_int,
                                 C.POINTER(TuneResult)]),
    "rcabf_server_create": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]),
    "rcabf_server_submit": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(BeamformArgs), C.POINTER(C.c_uint64)]),
    "rcabf_server_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_int)]),
    "rcabf_server_wait_for": (C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.POINTER(C.c_int)]),
    "rcabf_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    "rcabf_server_destroy": (C.c_int, [C.c_void_p]),
    "rcabf_sim_element_field": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                          C.c_float, C.c_int, C.c_float, C.c_float, C.c_int64, C.c_int64,
                                          C.c_int64, C.c_int64, C.c_void_p]),
    "rcabf_sim_tx_field": (C.c_int, [C.c_void_p] * 8 + [C.c_int64, C.c_float, C.c_float, C.c_float, C.c_int,
                                                        C.c_float, C.c_float, C.c_int64, C.c_int64, C.c_int64,
                                                        C.c_int64, C.c_void_p]),
    "rcabf_sim_rx_spectrum": (C.c_int, [C.c_void_p] * 7 + [C.c_int64, C.c_float, C.c_float, C.c_float, C.c_int,
                                                           C.c_float, C.c_float, C.c_int64, C.c_int64, C.c_int64,
                                                           C.c_int64, C.c_void_p]),
    "rcabf_sim_rf": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                               C.c_int32, C.c_int64, C.c_void_p]),
    "rcabf_ulm_psf_corr": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_int64, C.c_int64,
                                     C.c_int64, C.c_int32, C.c_int32, C.c_void_p]),
    "rcabf_ulm_ensemble": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int64,
                                     C.c_int64, C.c_void_p]),
    "rcabf_ulm_regional_max": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p]),
    "rcabf_ulm_detect": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                   C.c_int64, C.c_int64, C.c_int32, C.c_int32, C.c_int64, C.c_void_p]),
    "rcabf_ulm_gauss_fit": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                      C.c_int64, C.c_int64, C.c_int32, C.c_void_p, C.c_void_p]),
    "rcabf_ulm_density": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                    C.POINTER(UlmBins), C.c_int32, C.c_void_p]),
    "rcabf_take_error_count": (C.c_int, [C.POINTER(C.c_int64)]),
    "rcabf_take_launch_count": (C.c_int, [C.POINTER(C.c_int64)]),
    "rcabf_measure_fp32_peak": (C.c_int, [C.POINTER(C.c_double), C.c_void_p]),
    "rcabf_casorati_gram_plan": (C.c_int, [C.c_int64, C.c_int64, C.c_int32, C.POINTER(GramPlan)]),
    "rcabf_casorati_gram": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int32,
                                      C.c_void_p, C.c_size_t, C.c_void_p]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads librcabf.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"librcabf.so not found at {LIB_PATH}; build it with `python -m simu_rca_ab_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def declared_symbols() -> list[str]:
    return list(_SIGS)


class RcabfError(RuntimeError):
    """A librcabf status code; ``identifier`` is the reference error id."""

    def __init__(self, status: int, where: str = ""):
        self.status = int(status)
        self.identifier = lib().rcabf_status_string(int(status)).decode()
        detail = lib().rcabf_last_error().decode() if self.status == 106 else ""
        super().__init__(f"{self.identifier} (status {self.status}){': ' + where if where else ''}"
                         f"{' -- ' + detail if detail else ''}")


def check(status: int, where: str = "") -> None:
    if status != OK:
        raise RcabfError(status, where)


def dptr(a) -> "C.POINTER(C.c_double)":
    """Pointer to a contiguous float64 numpy array (caller keeps it alive)."""
    return a.ctypes.data_as(_dp)


NAN = math.nan
