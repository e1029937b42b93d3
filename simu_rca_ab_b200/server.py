"""Python side of the librcabf serving loop (rcabf_server_*).

A :class:`Server` owns an HBM arena (the admission budget), a few CUDA
streams and a scheduler thread inside librcabf.  :meth:`Server.submit` queues
one beamforming request and returns at once; requests that arrive while
others run are admitted as streams and arena space free up, and queued
requests that run the same kernel variant are fused into one persistent
launch.  The caller keeps the request's tensors alive until it completes
(the server holds a reference to them until :meth:`wait` or :meth:`poll`
reports it done).
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass

import torch

from . import _lib as L
from .beamformer import Engine, GeometryHandle


@dataclass
class ServerStats:
    submitted: int
    completed: int
    rejected: int
    launches: int
    in_flight: int
    queued: int
    p50_ms: float
    p95_ms: float
    p99_ms: float
    mean_ms: float
    max_ms: float
    units_done: float
    busy_s: float
    span_s: float
    arena_bytes: int
    arena_peak_bytes: int


class Server:
    """Continuous-batching beamforming server on one device."""

    def __init__(self, engine: Engine, hbm_budget_bytes: int, *, n_streams: int = 4, max_queue: int = 1024,
                 max_batch: int = 24, batch_window_us: int = 0):
        self.engine = engine
        cfg = L.ServerConfig()
        cfg.struct_size = C.sizeof(L.ServerConfig)
        cfg.device = engine.device.index
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        cfg.n_streams = n_streams
        cfg.max_queue = max_queue
        cfg.max_batch = max_batch
        cfg.batch_window_us = batch_window_us
        h = C.c_void_p()
        L.check(L.lib().rcabf_server_create(C.byref(cfg), C.byref(h)), "rcabf_server_create")
        self._h = h
        self._keep: dict[int, tuple] = {}
        self._lock = threading.Lock()

    def submit(self, geom: GeometryHandle, args: L.BeamformArgs, keep: tuple = ()) -> int:
        """Queues one request; returns its ticket.  Raises RcabfError with
        status 104 (over the HBM budget) or 110 (queue full) when refused."""
        t = C.c_uint64()
        L.check(L.lib().rcabf_server_submit(self._h, C.c_void_p(geom.ptr), C.byref(args), C.byref(t)),
                "rcabf_server_submit")
        with self._lock:
            self._keep[t.value] = (geom, args) + tuple(keep)
        return t.value

    def submit_beamform(self, geom: GeometryHandle, iq: torch.Tensor, out: torch.Tensor, *, iq_dtype: int,
                        n_sample: int, n_frame: int, mask: torch.Tensor | None = None, compound: bool = True,
                        storage: int = L.STORE_F32, kernel: int = L.KERNEL_AUTO, accumulate: bool = False) -> int:
        a = self.engine.make_args(geom, iq, iq_dtype=iq_dtype, n_sample=n_sample, n_frame=n_frame, out=out,
                                  mask=mask, compound=compound, storage=storage, kernel=kernel,
                                  accumulate=accumulate)
        return self.submit(geom, a, keep=(iq, out, mask))

    def poll(self, ticket: int) -> int | None:
        """None while the request runs, else its status (0 = done)."""
        st = C.c_int()
        r = L.lib().rcabf_server_poll(self._h, C.c_uint64(ticket), C.byref(st))
        if r == L.ERR_PENDING:
            return None
        L.check(r, "rcabf_server_poll")
        self._release(ticket)
        return st.value

    def wait(self, ticket: int, timeout_s: float = 60.0) -> int:
        """Waits for a request; returns its status, raises RcabfError(105) on timeout."""
        st = C.c_int()
        L.check(L.lib().rcabf_server_wait_for(self._h, C.c_uint64(ticket), C.c_double(timeout_s), C.byref(st)),
                "rcabf_server_wait_for")
        self._release(ticket)
        return st.value

    def stats(self) -> ServerStats:
        s = L.ServerStats()
        s.struct_size = C.sizeof(L.ServerStats)
        L.check(L.lib().rcabf_server_get_stats(self._h, C.byref(s)), "rcabf_server_get_stats")
        return ServerStats(**{f: getattr(s, f) for f, _ in L.ServerStats._fields_
                              if f not in ("struct_size", "reserved")})

    def close(self):
        if self._h is not None and self._h.value:
            L.check(L.lib().rcabf_server_destroy(self._h), "rcabf_server_destroy")
        self._h = None
        self._keep.clear()

    def _release(self, ticket: int):
        with self._lock:
            self._keep.pop(ticket, None)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
