#!/usr/bin/env python
"""Benchmark of the RCA delay-and-sum beamformer on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2]
    python bench.py --impl reference ...          # the reference's CPU arm

Metric: nominal voxel.rx.tx per second (voxels x receive elements x
transmits, summed over frames) for the Doppler-ensemble workload c2
(128+128 probe, 11 plane waves, 200 frames of [768 x 128 x 11] I/Q stored
as FP16, 96 x 96 x 160 voxels, Lanczos a = 4, f-number 1.2), seeded
synthetic data.  One step = one full beamform of the acquisition: ingest of
the channel data into the FP16 frame-blocked layout, the window-range
tables, the fused delay-and-sum kernel over all frames and transmits, and
the mask.

value     : device-resident inputs, CUDA events on the launching stream.
e2e       : the same through the C ABI with host (pinned) buffers
            (rcabf_beamform_host): the step's H2D copy of the channel data
            and D2H copy of the volume are inside the timed region, in frame
            chunks overlapped with the beamforming.
roofline  : the fused kernel's FP32 work (active units x (8a + 8) FLOP)
            over its event-timed duration, against the FP32 FMA peak measured
            live on this GPU.
Multi-GPU : each rank beamforms its own ensemble (weak scaling, no
            data-path collective); time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DAS voxel·rx·tx/s (nominal, summed over frames)"
UNIT = "voxel·rx·tx/s"
# plan kernel -> CUDA kernel function
KERNEL_NAMES = {"fused_voxel_blocked": "fused_vb_kernel", "fused_voxel_blocked_tmem": "fused_vb_kernel",
                "fused": "fused_das_kernel", "plain": "plain_das_kernel", "fused_tensor_core": "fused_tc_kernel",
                "fused_tensor_core_fp16w": "fused_tc_kernel"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--frames", type=int, default=None, help="override the workload's frame count (profiling cases)")
    ap.add_argument("--storage", default=None, help="float32 | float16 | bfloat16 (default: workload's)")
    ap.add_argument("--kernel", default="fused", choices=["fused", "plain", "tmem", "regs", "tc", "tc16"],
                    help="fused: the planner's (or autotuner's) choice; tmem / regs: the voxel-blocked kernel "
                         "with tensor-memory / register accumulators; tc / tc16: the tensor-core kernel with "
                         "hi + remainder / single FP16 weights")
    ap.add_argument("--frames-per-block", type=int, default=0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-frame FP32 kernel comparison")
    ap.add_argument("--no-serving", action="store_true", help="skip the c3 serving-mix measurement")
    ap.add_argument("--no-graph", action="store_true", help="skip the CUDA-graph replay of the step")
    ap.add_argument("--no-autotune", action="store_true", help="use the planner's launch choice untimed")
    ap.add_argument("--no-clutter", action="store_true", help="skip the SVD clutter filter of the ensemble")
    ap.add_argument("--no-simulator", action="store_true", help="skip the simulator timing")
    ap.add_argument("--no-ulm", action="store_true", help="skip the ULM super-localisation timing")
    ap.add_argument("--no-per-channel", action="store_true", help="skip the no-sum (per-channel) timing")
    ap.add_argument("--serving-requests", type=int, default=48)
    ap.add_argument("--serving-rates", default="6,60", help="c3 Poisson arrival rates (requests/s), comma-separated")
    ap.add_argument("--no-serving-plain", action="store_true", help="skip serving the stream on the plain kernel")
    ap.add_argument("--plain-frames", type=int, default=10)
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip the reference kernel on the GPU")
    ap.add_argument("--no-tc16", action="store_true",
                    help="skip the tensor-core kernel with single FP16 weights (timed beside the default)")
    ap.add_argument("--ref-gpu-frames", type=int, default=20,
                    help="frames of the workload the reference GPU kernel is timed on")
    ap.add_argument("--cpu-sample-frames", type=int, default=4)
    ap.add_argument("--cpu-sample-z", type=int, default=8)
    return ap.parse_args()


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def cpu_baseline(w, data_np, frames: int, zrows: int, kind_pref="reference"):
    """The reference kernel source on the host cores (oracle/_ref, OpenMP
    over all cores) on a z-slab x frame sample of the workload; rate in
    voxel.rx.tx/s.  Falls back to the C restatement ("port")."""
    import numpy as np

    from oracle import host as H
    from simu_rca_ab_b200 import workloads as W

    kind = "reference" if (kind_pref == "reference" and H.have_ref_cpu()) else "port"
    total_units, total_s = 0, 0.0
    for gi, g in enumerate(w.groups):
        G = dict(g.Geometry)
        for k in ("gridBfX", "gridBfY", "gridBfZ"):
            G[k] = np.asarray(G[k])[:zrows]
        d = W.as_matlab(W.group_data(w, data_np[:frames], gi))
        O = {"flagInterpolationLanczos": True, "flagCompounding": True, "flagMaskTransmit": False}
        r = H.prepare(d, G, g.Transmit, w.Param, O)
        t = time.perf_counter()
        if kind == "reference":
            H.run_ref_cpu(r)
        else:
            H.run_c32(r)
        total_s += time.perf_counter() - t
        total_units += r.n_pix * r.n_ch * r.n_tx * r.n_frame
    cores = os.cpu_count()
    nz, nx, ny = w.grid_shape
    return {"value": total_units / total_s, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": f"{w.name}: z-slab {zrows} of {nz} depth rows x {nx}x{ny} lateral, all "
                      f"{w.n_tx} tx x {w.n_ele} rx, {frames} of {w.n_frame} frames; reference 6-tap "
                      f"'Lanczos 5-lobes' kernel (the reference has no Lanczos-{w.lanczos_a}); "
                      f"{total_units:.3e} units in {total_s:.1f} s on {cores} threads"}


def serving_leg(eng, dev, n_requests: int, rates, seed: int = 3, plain: bool = True):
    """c3: Poisson streams of mixed requests through the serving loop
    (rcabf_server_*), submitted in real time at their arrival times, at each
    arrival rate of ``rates`` (the lowest first); then the lowest-rate stream
    served again through the same loop with every request on the plain
    per-frame kernel (one request per launch, no fusion), for comparison.
    The admission budget is the configuration's 150 GB of HBM when the
    device has it free (with 8 GB kept back), else what is free."""
    import warnings

    import numpy as np
    import torch

    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    from simu_rca_ab_b200.params import normalize
    from simu_rca_ab_b200.server import Server

    geoms, data = {}, {}

    def stream(rate_hz):
        reqs = W.serving_mix(seed, n_requests, rate_hz)
        # geometry tables per probe / transmit set / grid, channel data per
        # probe / transmit set (frames sliced per request): resident before
        # the stream starts
        maxf = {}
        for r in reqs:
            maxf[(r.probe, r.n_tx)] = max(maxf.get((r.probe, r.n_tx), 0), r.n_frame)
        for (probe, ntx), nf in maxf.items():
            if (probe, ntx) not in data or data[(probe, ntx)].shape[0] < nf:
                w = W.c3_workload(probe, ntx, W.C3_GRIDS[0], nf)
                data[(probe, ntx)] = W.channel_data(w, seed=seed + probe + ntx, device=dev)
        items = []
        for r in reqs:
            w = W.c3_workload(r.probe, r.n_tx, r.grid, r.n_frame)
            key = (r.probe, r.n_tx, r.grid)
            if key not in geoms:
                g = w.groups[0]
                with warnings.catch_warnings():
                    warnings.simplefilter("ignore")
                    geoms[key] = eng.geometry(normalize(np.zeros(1, np.complex64), g.Geometry, g.Transmit, w.Param,
                                                        w.Options))
            iq = data[(r.probe, r.n_tx)][: r.n_frame].contiguous()
            if r.storage == "float16":
                iq = iq.to(torch.complex32)
            out = torch.empty((r.n_frame, 1, geoms[key].n_pix), dtype=torch.complex64, device=dev)
            items.append((r, geoms[key], iq, out, w.units()))
        return items

    def args(r, g, iq, out, kernel):
        code = L.STORE_F16 if r.storage == "float16" else L.STORE_F32
        iqd = L.IQ_C32 if r.storage == "float16" else L.IQ_C64
        return eng.make_args(g, iq, iq_dtype=iqd, n_sample=iq.shape[-1], n_frame=iq.shape[0], out=out, mask=None,
                             compound=True, storage=code, kernel=kernel)

    def serve(items, kernel, budget):
        # the first launch of each kernel variant sets its shared-memory limit
        # inside the stream, as it would in a live service.  The arena is one
        # allocation: step down from the budget until the device grants it
        # (the stream's own buffers are allocated by now)
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        while True:
            try:
                srv = Server(eng, budget, n_streams=4, max_queue=4 * n_requests, max_batch=24)
                break
            except L.RcabfError:
                if budget < 16e9:
                    raise
                budget = int(budget * 0.95)
        tickets = []
        t0 = time.perf_counter()
        for r, g, iq, out, _ in items:
            delay = r.arrival_s - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets.append(srv.submit(g, args(r, g, iq, out, kernel), keep=(iq, out)))
        for t in tickets:
            srv.wait(t, 900.0)
        st = srv.stats()
        srv.close()
        torch.cuda.synchronize()
        return {"p50_ms": st.p50_ms, "p95_ms": st.p95_ms, "p99_ms": st.p99_ms, "mean_ms": st.mean_ms,
                "max_ms": st.max_ms, "value": st.units_done / st.span_s if st.span_s > 0 else None, "unit": UNIT,
                "launches": st.launches, "requests": len(items), "busy_s": st.busy_s, "span_s": st.span_s,
                "arena_peak_bytes": st.arena_peak_bytes, "hbm_budget_bytes": budget}

    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info(dev)
    budget = int(min(150e9, free - 8e9))
    res = {"workload": f"c3 serving mix: {n_requests} requests per stream, Poisson arrivals (seed {seed}); probe "
                       "64+64 or 128+128, 1-32 tx, 1-64 frames, grids 32x32x64..128x128x256, FP32/FP16 storage, "
                       "f-number 1.5, Lanczos a=3; channel data and geometry tables resident",
           "hbm_budget_bytes": budget,
           "rates": []}
    items0 = None
    for rate in sorted(rates):
        items = stream(rate)
        if items0 is None:
            items0 = items
        r = serve(items, L.KERNEL_AUTO, budget)
        r["rate_hz"] = rate
        r["units"] = sum(x[4] for x in items)
        r["fused_launches"] = r["launches"] < r["requests"]
        res["rates"].append(r)
    if plain and items0 is not None:
        r = serve(items0, L.KERNEL_PLAIN, budget)
        r["rate_hz"] = min(rates)
        r["how"] = "the lowest-rate stream served through rcabf_server_* with every request on plain_das_kernel"
        res["plain_kernel"] = r
    granted = [r["hbm_budget_bytes"] for r in res["rates"]]
    res["hbm_budget_note"] = (
        "150 GB as configured" if granted and min(granted) >= 150e9 else
        f"150 GB configured, {free / 1e9:.1f} GB free before the streams' buffers; each stream's admission arena "
        f"is one allocation, the largest the device granted once that stream's channel data and outputs were "
        f"resident: {', '.join(f'{b / 1e9:.1f}' for b in granted)} GB (hbm_budget_bytes per stream)")
    return res


def ulm_leg(dev, seed: int = 11, nz: int = 256, nx: int = 256, nt: int = 400, n_bubbles: int = 48):
    """ULM super-localisation (simu_rca_ab_b200.ulm, the reference's
    Python/superloc/superloc.py) on a synthetic 2-D block: nz x nx pixels x
    nt frames of complex Gaussian microbubble spots (sigma 1.5 px, moving up
    to 0.4 px per frame) in -30 dB noise, resident on the device; a 9 x 9
    Gaussian PSF.  Times PsfCorrMap2D + SuperLocFilter (fit 0) on the
    device, and DensityMappingND of the localisations."""
    import numpy as np
    import torch

    from simu_rca_ab_b200 import ulm as U
    g = torch.Generator(device=dev).manual_seed(seed)
    rnd = lambda *s: torch.rand(*s, generator=g, device=dev)
    z0, x0 = 12 + rnd(n_bubbles) * (nz - 24), 12 + rnd(n_bubbles) * (nx - 24)
    vz, vx = (rnd(n_bubbles) - 0.5) * 0.8, (rnd(n_bubbles) - 0.5) * 0.8
    amp = (0.5 + rnd(n_bubbles)) * torch.exp(1j * 2 * np.pi * rnd(n_bubbles))
    zz = torch.arange(nz, device=dev, dtype=torch.float32)[:, None, None]
    xx = torch.arange(nx, device=dev, dtype=torch.float32)[None, :, None]
    tt = torch.arange(nt, device=dev, dtype=torch.float32)[None, None, :]
    iq = torch.zeros((nz, nx, nt), dtype=torch.complex64, device=dev)
    for b in range(n_bubbles):
        zc = (z0[b] + vz[b] * tt).remainder(nz)
        xc = (x0[b] + vx[b] * tt).remainder(nx)
        iq += amp[b] * torch.exp(-((zz - zc) ** 2 + (xx - xc) ** 2) / (2 * 1.5 ** 2))
    iq += 0.03 * torch.complex(torch.randn(iq.shape, generator=g, device=dev),
                               torch.randn(iq.shape, generator=g, device=dev))
    k = np.arange(9) - 4.0
    psf = np.exp(-(k[:, None] ** 2 + k[None, :] ** 2) / (2 * 1.5 ** 2)).astype(np.complex64)

    def run():
        corr = U.PsfCorrMap2D(iq, psf)
        return U.SuperLocFilter(corr, iq, 5, 5, 0)

    run()
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    corr = U.PsfCorrMap2D(iq, psf)
    e1.record()
    pos = U.SuperLocFilter(corr, iq, 5, 5, 0)
    e2.record()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dens = U.DensityMappingND(pos, np.arange(nx * 4) / 4.0, [0.0], np.arange(nz * 4) / 4.0)
    dens_ms = (time.perf_counter() - t0) * 1e3
    corr_ms, loc_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)
    return {"what": f"ULM (superloc.py): PsfCorrMap2D (9x9 PSF) + SuperLocFilter (fit 0) on {nz}x{nx} px x {nt} "
                    f"frames of {n_bubbles} moving microbubbles in -30 dB noise, device-resident; "
                    "DensityMappingND at 4x super-resolution (host arrays in and out)",
            "corr_ms": corr_ms, "superloc_ms": loc_ms, "ms": corr_ms + loc_ms,
            "frames_per_s": nt / ((corr_ms + loc_ms) / 1e3), "localisations": int(pos.shape[1]),
            "density_ms": dens_ms, "density_total": float(dens.sum())}


def simulator_leg(dev, seed: int = 7):
    """The frequency-domain simulator (sim_us_rca) on a 64+64 RCA set-up:
    transmit rows / receive columns of 64 strips (8 sub-elements each),
    16 plane waves, 200 scatterers, 2 frames, 1024 samples at 31.2 MHz."""
    import numpy as np
    import torch

    from simu_rca_ab_b200.simulator import sim_plan, sim_us_rca
    rng = np.random.default_rng(seed)
    n_ele, n_sub, n_tx, n_scat, n_frame = 64, 8, 16, 200, 2
    pitch, f0, c = 0.3e-3, 7.8e6, 1540.0
    pos = (np.arange(n_ele) - (n_ele - 1) / 2) * pitch
    strip = (np.arange(n_sub) - (n_sub - 1) / 2) * (n_ele * pitch / n_sub)
    tx = np.zeros((n_ele, 5, n_sub))
    rx = np.zeros((n_ele, 5, n_sub))
    for q in range(n_sub):
        tx[:, 0, q], tx[:, 1, q] = strip[q], pos
        rx[:, 0, q], rx[:, 1, q] = pos, strip[q]
    t = np.arange(0, 2 / f0, 1 / 250e6)
    ir = np.sin(2 * np.pi * f0 * t) * np.hanning(t.size)
    trans = lambda p: {"frequency": f0, "impulseResponse": ir, "lensCorrection": 0.0, "ElementPos": p,
                       "ElementHeight": 2e-3, "ElementWidth": 0.27e-3, "ElementElevationFocus": 20e-3, "baffle": 1}
    n_event = n_tx * n_frame
    base = np.stack([rng.uniform(-9e-3, 9e-3, n_scat), rng.uniform(-9e-3, 9e-3, n_scat),
                     rng.uniform(5e-3, 25e-3, n_scat), rng.rayleigh(1.0, n_scat)], 1)
    scat = np.repeat(base[:, :, None], n_event, 2)
    th = np.deg2rad(np.linspace(-8, 8, n_tx))
    TXSI = [{"pulseShape": np.sin(2 * np.pi * f0 * t), "Delay": pos * np.sin(a) / c - (pos * np.sin(a) / c).min(),
             "Apod": np.ones(n_ele)} for a in th]
    RXSI = [{"samplingFrequency": 4 * f0, "demodFrequency": f0, "startTime": 0.0, "numelSample": 1024,
             "sampleMode": "NS200BW", "InputFilter": np.array([1.0]), "Apod": np.ones(n_ele)} for _ in th]
    case = ({"speedOfSound": c, "attenuation": 0.5, "scattererPos": scat}, trans(tx), trans(rx), TXSI, RXSI)
    sim_us_rca(*case)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    raw = sim_us_rca(*case)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    p = sim_plan(*case)
    evals = p["n_freq"] * n_scat * n_ele * n_sub * 2 * n_frame   # element-field terms (transmit + receive arrays)
    return {"what": f"sim_us_rca: {n_ele}+{n_ele} RCA strips x {n_sub} sub-elements, {n_tx} plane waves, "
                    f"{n_scat} scatterers, {n_frame} frames, {p['n_freq']} frequencies, Raw {list(raw.shape)}",
            "ms": 1e3 * el, "element_field_terms_per_s": evals / el,
            "note": "scatterers static within a frame: the frame's 16 transmits as one group; per group "
                    "rcabf_sim_tx_field (fields summed over elements), rcabf_sim_rx_spectrum (summed over "
                    "scatterers), rcabf_sim_rf (inverse transform at the kept samples); host set-up included"}


def per_channel_leg(eng, dev, n_frame: int = 100):
    """The no-sum beamformer (bf_rca_nosum, the reference's
    bfVirtualSourceGeneric_RCA_Nosum) as the dataset producer calls it
    (MATLAB/save_simus_sh.m:354-393): one value per receive element on a
    1 x 1 x 17 line of depths, here on the 64+64 probe of the single-volume
    workload with its 16 transmits and n_frame frames of channel data
    resident.  Times every frame in one launch (the planner's choice) against
    one launch per frame (the plain kernel by name); the outputs are compared
    bit for bit."""
    import numpy as np
    import torch

    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import workloads as W
    from simu_rca_ab_b200.params import normalize
    w = W.get("c0", n_frame=n_frame)
    g = w.groups[0]
    G = dict(g.Geometry)
    z = np.linspace(5e-3, 25e-3, 17).reshape(17, 1, 1)
    G.update(gridBfX=np.zeros_like(z), gridBfY=np.zeros_like(z), gridBfZ=z)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        geom = eng.geometry(normalize(np.zeros(1, np.complex64), G, g.Transmit, w.Param, w.Options))
    iq = W.group_data(w, W.channel_data(w, seed=3, device=dev), 0).contiguous()
    outs = {}
    times = {}
    for name, kern in (("all_frames", L.KERNEL_AUTO), ("per_frame", L.KERNEL_PLAIN)):
        out = torch.empty((geom.n_ele, n_frame, geom.n_tx, geom.n_pix), dtype=torch.complex64, device=dev)
        a = eng.make_args(geom, iq, iq_dtype=L.IQ_C64, n_sample=w.n_sample, n_frame=n_frame, out=out, mask=None,
                          compound=False, storage=L.STORE_F32, kernel=kern, per_channel=True)
        for _ in range(2):
            eng.run(geom, a)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 5
        e0.record()
        for _ in range(reps):
            eng.run(geom, a)
        e1.record()
        torch.cuda.synchronize()
        times[name] = e0.elapsed_time(e1) / reps
        outs[name] = out
    return {"what": f"bf_rca_nosum: 64+64 probe, 16 transmits, 64 receive elements, {n_frame} frames, 1x1x17 "
                    f"depths; output [element][frame][tx][pixel]",
            "all_frames_ms": times["all_frames"], "per_frame_launches_ms": times["per_frame"],
            "speedup": times["per_frame"] / times["all_frames"],
            "identical": bool(torch.equal(outs["all_frames"], outs["per_frame"]))}


WORKLOAD_KIND = {"c0": "single volume, 64+64 probe", "c1": "row + column transmits compounded, 128+128 probe",
                 "c2": "Doppler ensemble", "c4": "large volume, 256+256 probe, row + column transmits"}


def tensor_peak():
    """Dense FP16/BF16 tensor peak (TFLOP/s) and where it comes from: the
    pool's measured figure (sustained: the kernel runs inside a long step)
    when MEASURED_PEAKS.json is present, else the pool's earlier burst
    measurement."""
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            d = json.loads(f.read_text())
            for k in ("bf16_tflops_sustained", "bf16_tflops"):
                if d.get(k):
                    return float(d[k]), f"MEASURED_PEAKS.json {k} (of measured)"
        except (ValueError, OSError):
            pass
    return 1590.0, "1.59 PFLOP/s dense bf16 burst, an earlier measurement on this pool (of fallback)"


def int8_peak(dev):
    """Dense int8 tensor throughput (TOP/s) measured live: cuBLASLt int8 GEMM
    (torch._int_mm, 8192^3, 2 N^3 ops), best of 5 after warm-up."""
    import torch
    n = 8192
    a = torch.randint(-64, 64, (n, n), dtype=torch.int8, device=dev)
    b = torch.randint(-64, 64, (n, n), dtype=torch.int8, device=dev).t()
    for _ in range(3):
        torch._int_mm(a, b)
    best = None
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch._int_mm(a, b)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def clutter_leg(x, dev, reps: int = 5):
    """The SVD clutter filter of the beamformed ensemble x ([frame][voxel]):
    its Gram on the int8 tensor cores (rcabf_casorati_gram) against the FP64
    cuBLAS ZGEMM Gram, the whole filter with each, on the device (CUDA events
    on the current stream, median of ``reps`` after a warm-up)."""
    import numpy as np
    import torch
    from simu_rca_ab_b200.clutter import casorati_gram, gram_plan, svd_clutter_filter

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    n_t, n_pix = x.shape
    plan = gram_plan(n_t, n_pix)
    ws = torch.empty(int(plan["workspace_bytes"]) + 256, dtype=torch.uint8, device=dev)
    g_tc = casorati_gram(x, workspace=ws)
    ms_tc = timed(lambda: casorati_gram(x, workspace=ws))
    x64 = x.to(torch.complex128)
    g64 = x64.conj() @ x64.T
    ms_64 = timed(lambda: x.to(torch.complex128).conj() @ x.to(torch.complex128).T)
    del x64
    gerr = float((g_tc - g64).abs().max() / g64.abs().max())
    del g_tc, g64
    peak = int8_peak(dev)
    tops = plan["mma_int_ops"] / (ms_tc * 1e-3) / 1e12
    ms_f_tc = timed(lambda: svd_clutter_filter(x, None, (0.1,), "high", time_axis=0, order="C"))
    ms_f_64 = timed(lambda: svd_clutter_filter(x, None, (0.1,), "high", time_axis=0, order="C", gram="fp64"))
    xf, ev = svd_clutter_filter(x, None, (0.1,), "high", time_axis=0, order="C")
    xr, _ = svd_clutter_filter(x, None, (0.1,), "high", time_axis=0, order="C", gram="fp64")
    frel = float((xf - xr).abs().pow(2).sum().sqrt() / xr.abs().pow(2).sum().sqrt())
    kept = float((xf.abs() ** 2).sum() / (x.abs() ** 2).sum())
    del xf, xr, ws
    return {"what": f"SVDClutterFilter high-pass w=0.1 on the beamformed ensemble ({n_pix} voxels x {n_t} "
                    "frames): Gram on the int8 tensor cores (4 x 7-bit slices, exact int32 sums, FP64 "
                    "levels and chunks), FP64 eigh, FP32 projection (CGEMM)",
            "ms": ms_f_tc, "ms_with_fp64_zgemm_gram": ms_f_64, "energy_kept": kept,
            "filtered_rel_vs_fp64_gram": frel,
            "gram": {"ms": ms_tc, "ms_fp64_zgemm": ms_64, "speedup_vs_fp64_zgemm": ms_64 / ms_tc,
                     "max_err_rel_max_fp64": gerr, "mma_int_ops": plan["mma_int_ops"],
                     "int_tops": tops, "int8_peak_tops": peak,
                     "int8_peak_source": "cuBLASLt int8 GEMM 8192^3 measured live (torch._int_mm)",
                     "tensor_frac": tops / peak, "plan": plan,
                     "note": "ms covers the 4 launches (slicing, MMA, chunk reduction, assembly); "
                             "tensor_frac is the MMA work of the whole call over that time"}}


def ref_gpu_leg(w, data, frames: int, variant: str = "fast"):
    """The reference's own CUDA kernel on this GPU (bfVirtualSourceGeneric_RCA.cu
    compiled from its source; "fast" = -use_fast_math, as the reference
    wrapper builds it at bfVirtualSourceGeneric_RCA.m:796), launched the way
    the wrapper launches it (block 1024, grid [ceil(nPix/1024), nTx,
    nFrameChunk], frames chunked per .m:587-594, compounding sum over
    transmits on the device per .m:689-697), channel data resident on the
    device, on the first ``frames`` frames; rate in voxel.rx.tx/s.  Both of
    the reference's interpolation kernels are timed: its 6-tap "Lanczos
    5-lobes" option and its default quadratic."""
    from oracle import host as H
    from simu_rca_ab_b200 import workloads as W

    if not H.have_ref_gpu(variant):
        return {"unavailable": f"oracle/_ref/librca_ref_gpu_{variant}.so not built"}
    res = {"kernel": f"reference bfVirtualSourceGeneric_RCA.cu, sm_100a, {variant} build"
                     + (" (-use_fast_math, as the reference wrapper compiles it)" if variant == "fast" else ""),
           "frames": frames}
    for name, lz in (("ref6", True), ("quadratic", False)):
        ms, units, chunks = 0.0, 0, 0
        for gi, g in enumerate(w.groups):
            d = W.group_data(w, data[:frames], gi).cpu().numpy()
            r = H.prepare(W.as_matlab(d), g.Geometry, g.Transmit, w.Param,
                          {"flagInterpolationLanczos": lz, "flagCompounding": True, "flagMaskTransmit": False})
            t, nc = H.time_ref_gpu(r, variant)
            ms += t
            chunks += nc
            units += r.n_pix * r.n_ch * r.n_tx * r.n_frame
        res[name] = {"value": units / (ms * 1e-3), "unit": UNIT, "ms": ms, "launches": chunks}
    return res


def run_reference(a, rank):
    """--impl reference: the reference's own kernel source on the host cores."""
    if rank != 0:
        return
    import numpy as np

    from simu_rca_ab_b200 import workloads as W
    w = W.get(a.workload)
    frames = max(1, a.cpu_sample_frames)
    data = W.channel_data(w, seed=0, device="cpu", frames=list(range(frames))).numpy()
    vals = []
    for _ in range(a.warmup):
        cpu_baseline(w, data, 1, 2)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        vals.append(cpu_baseline(w, data, frames, a.cpu_sample_z))
    el = time.perf_counter() - t0
    v = statistics.median(x["value"] for x in vals)
    cb = dict(vals[-1])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * el / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded point scatterers)",
            "config": {"workload": f"{w.name}: bounded sample per step ({cb['sample']})",
                       "interp": "reference 6-tap"},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "gpu_launches": 0}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def main():
    a = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        return run_reference(a, rank)

    import ctypes as C
    import warnings

    import numpy as np
    import torch

    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200 import beamformer as B
    from simu_rca_ab_b200 import workloads as W
    from simu_rca_ab_b200.multi import max_over_ranks
    from simu_rca_ab_b200.params import normalize

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    w = W.get(a.workload, n_frame=a.frames)
    storage = a.storage or w.storage
    st_code = {"float32": L.STORE_F32, "float16": L.STORE_F16, "bfloat16": L.STORE_BF16}[storage]
    kern = {"plain": L.KERNEL_PLAIN, "tmem": L.KERNEL_FUSED_TMEM, "regs": L.KERNEL_FUSED_REGS,
            "tc": L.KERNEL_FUSED_TC, "tc16": L.KERNEL_FUSED_TC_FP16W}.get(a.kernel, L.KERNEL_FUSED)

    data = W.channel_data(w, seed=rank, device=dev)                       # [F][T][E][S] complex64
    in_dtype = torch.complex32 if storage == "float16" else torch.complex64
    iq_code = L.IQ_C32 if in_dtype == torch.complex32 else L.IQ_C64
    eng = B.Engine(dev)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        geoms = [eng.geometry(normalize(np.zeros(1, np.complex64), g.Geometry, g.Transmit, w.Param, w.Options))
                 for g in w.groups]
    iq_dev = [W.group_data(w, data, gi).contiguous().to(in_dtype) for gi in range(len(w.groups))]
    F = w.n_frame
    n_pix = geoms[0].n_pix
    out = torch.empty((F, 1, n_pix), dtype=torch.complex64, device=dev)
    mask = torch.empty((1, n_pix), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in w.groups]
    for ee in evs:
        for e in ee:
            e.record(stream)
    ev_arr = [(C.c_void_p * 5)(*[e.cuda_event for e in ee]) for ee in evs]
    args = []
    for gi, g in enumerate(geoms):
        ar = eng.make_args(g, iq_dev[gi], iq_dtype=iq_code, n_sample=w.n_sample, n_frame=F, out=out, mask=mask,
                           compound=True, storage=st_code, kernel=kern, accumulate=gi > 0,
                           frames_per_block=a.frames_per_block)
        ar.stage_events = C.cast(ev_arr[gi], C.POINTER(C.c_void_p))
        args.append(ar)
    tune = None
    if not a.no_autotune and kern == L.KERNEL_FUSED and a.frames_per_block == 0:
        # launch choice (tile shape, window depth, frame block, kernel family)
        # measured on this workload before the timed region
        tune = [eng.autotune(g, ar, iters=1) for g, ar in zip(geoms, args)]
    ws = [torch.empty(max(256, eng.workspace_bytes(g, ar)), dtype=torch.uint8, device=dev)
          for g, ar in zip(geoms, args)]
    plan = eng.plan(geoms[0], args[0])

    def step():
        for g, ar, wsp in zip(geoms, args, ws):
            eng.run(g, ar, stream=stream, workspace=wsp)

    def barrier():
        if pg:
            pg.barrier()

    peak = C.c_double()
    L.check(L.lib().rcabf_measure_fp32_peak(C.byref(peak), C.c_void_p(stream.cuda_stream)))
    for _ in range(max(3, a.warmup)):
        step()
    torch.cuda.synchronize()
    n0 = C.c_int64()
    L.lib().rcabf_take_launch_count(C.byref(n0))

    # stage events of every timed step (ingest, ranges, fused kernel, mask),
    # recorded by the library on the launching stream
    t_stage = [[[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in w.groups] for _ in range(a.steps)]
    for sk in t_stage:
        for ee in sk:
            for e in ee:
                e.record(stream)
    t_stage_arr = [[C.cast((C.c_void_p * 5)(*[e.cuda_event for e in ee]), C.POINTER(C.c_void_p)) for ee in sk]
                   for sk in t_stage]
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    t_ev = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    t_ev[0].record(stream)
    for k in range(a.steps):
        for gi, ar in enumerate(args):
            ar.stage_events = t_stage_arr[k][gi]
        step()
        t_ev[k + 1].record(stream)
    torch.cuda.synchronize()
    for gi, ar in enumerate(args):   # later calls record into the first event set
        ar.stage_events = C.cast(ev_arr[gi], C.POINTER(C.c_void_p))
    barrier()
    clk = clocks.stop()
    launches = C.c_int64()
    L.lib().rcabf_take_launch_count(C.byref(launches))
    step_ms = [t_ev[k].elapsed_time(t_ev[k + 1]) for k in range(a.steps)]
    total_ms = t_ev[0].elapsed_time(t_ev[-1])
    total_ms = max_over_ranks(total_ms, dev)
    units = w.units()
    value = units * world * a.steps / (total_ms * 1e-3)

    # the same step captured once in a CUDA graph (no stage events inside) and
    # replayed: checked bit-identical to the eager step, then timed
    graph = None
    if not a.no_graph:
        try:
            step()
            torch.cuda.synchronize()
            eager_out = out.clone()
            g_args = []
            for ar in args:
                c = L.BeamformArgs.from_buffer_copy(ar)
                c.stage_events = None
                g_args.append(c)
            side = torch.cuda.Stream(dev)
            side.wait_stream(stream)
            with torch.cuda.stream(side):
                for g, ar, wsp in zip(geoms, g_args, ws):
                    eng.run(g, ar, workspace=wsp)
            stream.wait_stream(side)
            torch.cuda.synchronize()
            L.lib().rcabf_take_launch_count(C.byref(C.c_int64()))
            cg = torch.cuda.CUDAGraph()
            with torch.cuda.graph(cg):
                for g, ar, wsp in zip(geoms, g_args, ws):
                    eng.run(g, ar, workspace=wsp)
            per_step = C.c_int64()
            L.lib().rcabf_take_launch_count(C.byref(per_step))
            out.zero_()
            cg.replay()
            torch.cuda.synchronize()
            same = bool(torch.equal(out, eager_out))
            barrier()
            g0e, g1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            g0e.record(stream)
            for _ in range(a.steps):
                cg.replay()
            g1e.record(stream)
            torch.cuda.synchronize()
            g_ms = g0e.elapsed_time(g1e)
            g_ms = max_over_ranks(g_ms, dev)
            graph = {"ms_per_step": g_ms / a.steps, "value": units * world * a.steps / (g_ms * 1e-3),
                     "kernels_per_step": int(per_step.value), "identical_to_eager": same}
            del cg
        except Exception as ex:   # reported in the line, the eager number stands
            graph = {"error": f"{type(ex).__name__}: {ex}"}

    # the downstream SVD clutter filter on this ensemble: Gram on the int8
    # tensor cores against the FP64 ZGEMM Gram, eigen-decomposition,
    # projection, timed on the device
    clutter = None
    if not a.no_clutter and rank == 0:
        try:
            clutter = clutter_leg(out[:, 0], dev)
        except Exception as ex:
            clutter = {"error": f"{type(ex).__name__}: {ex}"}

    # fused-kernel time per launch: the stage events of the timed steps,
    # averaged over the steps
    def stage_mean(i, j):
        return sum(ee[i].elapsed_time(ee[j]) for sk in t_stage for ee in sk) / a.steps

    fused_ms = stage_mean(2, 3)
    stage_ms = {"ingest": stage_mean(0, 1), "ranges": stage_mean(1, 2), "das": fused_ms, "mask": stage_mean(3, 4),
                "of": f"the {a.steps} timed steps (mean)"}

    # e2e: host pinned buffers through the C ABI (rcabf_beamform_host: the
    # frames go through in chunks, each chunk's copies in and out overlapping
    # the beamforming of its neighbours)
    e2e = None
    if not a.no_e2e:
        # a stream of ensembles through the same call, as an acquisition loop
        # issues them: two slots (pinned host buffers, device workspace,
        # stream) alternate, so that one ensemble's copy out runs under the
        # next one's copy in and beamforming; inside a call the frames also
        # go through in chunks whose copies overlap their neighbours'
        # beamforming.  The latency of one call alone is reported beside it.
        streams = [stream, torch.cuda.Stream(dev)]
        slots = []
        for si in range(2):
            h_in = [t.cpu().pin_memory() for t in iq_dev]
            h_out = torch.empty(out.shape, dtype=out.dtype, pin_memory=True)
            h_mask = torch.empty_like(mask)
            h_args = [eng.make_args(g, h_in[gi], iq_dtype=iq_code, n_sample=w.n_sample, n_frame=F, out=h_out,
                                    mask=h_mask, compound=True, storage=st_code, kernel=kern, accumulate=gi > 0,
                                    frames_per_block=a.frames_per_block, host=True)
                      for gi, g in enumerate(geoms)]
            slots.append((h_in, h_out, h_args))
        out_bytes = out.numel() * out.element_size()
        # later groups add into the output: their chunks are read in as well
        h2d = sum(t.numel() * t.element_size() for t in slots[0][0]) + out_bytes * (len(geoms) - 1)
        d2h = out_bytes * len(geoms)

        def e2e_call(k):
            for g, ar in zip(geoms, slots[k % 2][2]):
                eng.run_host(g, ar, 0, streams[k % 2])

        for k in range(4):
            e2e_call(k)
        torch.cuda.synchronize()
        barrier()
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0.record(stream)
        e2e_call(0)
        l1.record(stream)
        torch.cuda.synchronize()
        lat_ms = l0.elapsed_time(l1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        streams[1].wait_event(e0)
        for k in range(a.steps):
            e2e_call(k)
        stream.wait_stream(streams[1])
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
        e2e_ms = max_over_ranks(e2e_ms, dev)
        same = bool(torch.equal(slots[0][1], slots[1][1]))
        e2e = {"value": units * world * a.steps / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms / a.steps,
               "call": "rcabf_beamform_host (host buffers in and out), two ensembles in flight on two streams",
               "latency_one_call_ms": lat_ms, "slots_identical": same}

    # the plain one-launch-per-frame kernel on FP32 storage, complex64 input
    # (the comparator of the fused path), timed on a sample of the frames
    plain = None
    if not a.no_plain and a.kernel != "plain":
        pf = max(1, min(a.plain_frames, F))
        p_in = [W.group_data(w, data[:pf], gi).contiguous() for gi in range(len(w.groups))]
        p_out = torch.empty((pf, 1, n_pix), dtype=torch.complex64, device=dev)
        p_args = [eng.make_args(g, p_in[gi], iq_dtype=L.IQ_C64, n_sample=w.n_sample, n_frame=pf, out=p_out,
                                mask=None, compound=True, storage=L.STORE_F32, kernel=L.KERNEL_PLAIN,
                                accumulate=gi > 0) for gi, g in enumerate(geoms)]

        def plain_step():
            for g, ar in zip(geoms, p_args):
                eng.run(g, ar, stream=stream)

        plain_step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plain_step()
        e1.record(stream)
        torch.cuda.synchronize()
        p_ms = e0.elapsed_time(e1)
        p_val = units / F * pf / (p_ms * 1e-3)
        plain = {"value": p_val, "unit": UNIT, "frames": pf, "ms": p_ms,
                 "kernel": "plain_das_kernel (one launch per frame, FP32 storage, complex64 input)",
                 "ratio": (value / world) / p_val}
        del p_in, p_out

    # the tensor-core kernel with single FP16 weights (chosen by name only):
    # the same step, timed, and its error against the FP64 oracle below
    tc16, out16 = None, None
    if not a.no_tc16 and plan.get("kernel") == "fused_tensor_core" and rank == 0:
        try:
            out16 = torch.empty_like(out)
            a16 = [eng.make_args(g, iq_dev[gi], iq_dtype=iq_code, n_sample=w.n_sample, n_frame=F, out=out16,
                                 mask=None, compound=True, storage=st_code, kernel=L.KERNEL_FUSED_TC_FP16W,
                                 accumulate=gi > 0) for gi, g in enumerate(geoms)]
            ws16 = [torch.empty(max(256, eng.workspace_bytes(g, ar)), dtype=torch.uint8, device=dev)
                    for g, ar in zip(geoms, a16)]

            def step16():
                for g, ar, wsp in zip(geoms, a16, ws16):
                    eng.run(g, ar, stream=stream, workspace=wsp)

            step16()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(a.steps):
                step16()
            e1.record(stream)
            torch.cuda.synchronize()
            ms16 = e0.elapsed_time(e1) / a.steps
            tc16 = {"kernel": "fused_tc_kernel, single FP16 weights (RCABF_KERNEL_FUSED_TC_FP16W)",
                    "ms_per_step": ms16, "value": units / (ms16 * 1e-3), "unit": UNIT,
                    "plan": eng.plan(geoms[0], a16[0])}
            del ws16
        except Exception as ex:
            tc16 = {"error": f"{type(ex).__name__}: {ex}"}
            out16 = None

    ref_gpu = None
    if not a.no_ref_gpu and rank == 0:
        try:
            ref_gpu = ref_gpu_leg(w, data, max(1, min(a.ref_gpu_frames, F)))
            for k in ("ref6", "quadratic"):
                if k in ref_gpu:
                    ref_gpu[k]["ratio"] = (value / world) / ref_gpu[k]["value"]
        except Exception as ex:
            ref_gpu = {"error": f"{type(ex).__name__}: {ex}"}
        torch.cuda.synchronize()
        torch.cuda.empty_cache()

    serving = None
    if not a.no_serving and rank == 0:
        try:
            serving = serving_leg(eng, dev, a.serving_requests, [float(x) for x in a.serving_rates.split(",")],
                                  plain=not a.no_serving_plain)
        except Exception as ex:   # reported, not hidden: the line says what failed
            serving = {"error": f"{type(ex).__name__}: {ex}"}
        torch.cuda.synchronize()

    sim = None
    if not a.no_simulator and rank == 0:
        try:
            sim = simulator_leg(dev)
        except Exception as ex:
            sim = {"error": f"{type(ex).__name__}: {ex}"}

    per_ch = None
    if not a.no_per_channel and rank == 0:
        try:
            per_ch = per_channel_leg(eng, dev)
        except Exception as ex:
            per_ch = {"error": f"{type(ex).__name__}: {ex}"}

    ulm = None
    if not a.no_ulm and rank == 0:
        try:
            ulm = ulm_leg(dev)
        except Exception as ex:
            ulm = {"error": f"{type(ex).__name__}: {ex}"}

    line = None
    if rank == 0:
        from oracle import host as H
        # active units (inside aperture and sample window), counted exactly by the oracle
        active = 0
        for gi, g in enumerate(w.groups):
            r = H.prepare(np.zeros((w.n_sample, w.n_ele, 1, g.n_tx), np.complex64), g.Geometry, g.Transmit,
                          w.Param, {"flagMaskTransmit": False})
            active += H.active_units(r, H.INTERP_LANCZOS, w.lanczos_a)
        active *= F
        fpu = 8 * w.lanczos_a + 8
        achieved = active * fpu / (fused_ms * 1e-3) / 1e12
        kname = KERNEL_NAMES.get(plan.get("kernel"), plan.get("kernel"))
        traffic = None
        tf = ROOT / "profiles" / f"traffic_{kname}_{w.name}_{storage}.json"
        if tf.exists():
            traffic = json.loads(tf.read_text()).get("dram_bytes_per_launch")
        fp32 = {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": achieved / peak.value,
                "peak_source": "FP32 FMA probe kernel timed live in this run (MEASURED_PEAKS.json has no FP32 figure)",
                "work": f"{active:.4e} active units x {fpu} FLOP ({active / (units):.3f} of nominal)",
                "nominal_achieved": units * fpu / (fused_ms * 1e-3) / 1e12}
        mma = sum(eng.plan(g, ar).get("mma_flops", 0.0) for g, ar in zip(geoms, args))
        if mma > 0:
            # the tensor-core kernel: its dense MMA work (the banded products
            # as issued, counted exactly from the windows) against the tensor
            # peak; the algorithmic FP32 work it stands for is fp32_equivalent
            tpk, tsrc = tensor_peak()
            ach_t = mma / (fused_ms * 1e-3) / 1e12
            roof = {"bound": "tensor", "achieved": ach_t, "peak": tpk, "unit": "TFLOP/s", "frac": ach_t / tpk,
                    "traffic": traffic, "peak_source": tsrc, "kernel": kname, "kernel_ms": fused_ms,
                    "work": f"{mma:.4e} dense MMA FLOPs per step (16-row window chunks x weight matrices x "
                            f"2 x 128 x N x 16, N = 2 x frames per block)",
                    "fp32_equivalent": fp32}
        else:
            roof = dict(fp32)
            roof.update({"traffic": traffic, "kernel": kname, "kernel_ms": fused_ms})
        acc = None
        if not a.no_accuracy:
            rng = np.random.default_rng(123)
            pix = np.sort(rng.choice(n_pix, size=min(2048, n_pix), replace=False))
            frames = sorted(set([0, F // 2, F - 1]))
            ref = 0
            g0 = w.groups[0]
            for gi, g in enumerate(w.groups):
                dg = W.group_data(w, data[frames], gi).cpu().numpy()
                r = H.prepare(W.as_matlab(dg), g.Geometry, g.Transmit, w.Param, {"flagMaskTransmit": False})
                f64, m64 = H.run_fp64(r, H.INTERP_LANCZOS, w.lanczos_a, data=dg, pix=pix)
                c64, _ = H.compound(f64, m64, True)
                ref = ref + c64[:, 0]
            ours = out[frames][:, 0, :].cpu().numpy()[:, pix]
            rms, pk = H.error_db(ours, ref)
            acc = {"rms_db": rms, "peak_db": pk, "vs": "FP64 oracle (complex64 input before storage rounding)",
                   "sample": f"{pix.size} random voxels x frames {frames}"}
            if tc16 is not None and out16 is not None:
                r16, p16 = H.error_db(out16[frames][:, 0, :].cpu().numpy()[:, pix], ref)
                tc16.update({"rms_db": r16, "peak_db": p16})
        cb = None
        if not a.no_cpu_baseline:
            dnp = data[: a.cpu_sample_frames].cpu().numpy()
            cb = cpu_baseline(w, dnp, a.cpu_sample_frames, a.cpu_sample_z)
        lat = sorted(step_ms)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": total_ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded point scatterers, -30 dB noise)",
            "config": {"workload": f"{w.name}: {WORKLOAD_KIND.get(w.name, 'acquisition')}, "
                                   f"[{w.n_sample} x {w.n_ele} x {w.n_tx} x {F}] I/Q, "
                                   f"grid {w.grid_shape[1]}x{w.grid_shape[2]}x{w.grid_shape[0]}, Lanczos a={w.lanczos_a}, "
                                   f"f-number {w.Param['fnumber']}",
                       "storage": storage, "kernel": a.kernel, "l2": "inputs larger than L2 (no flush needed)",
                       "units_per_step": units, "parallelism": f"weak x{world} (independent ensembles)",
                       "plan": plan, "autotune": tune},
            "latency": {"p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
            "stage_ms": stage_ms, "roofline": roof, "cpu_baseline": cb, "e2e": e2e, "plain_kernel": plain, "reference_gpu": ref_gpu,
            "serving": serving, "graph": graph, "clutter_filter": clutter, "simulator": sim, "per_channel": per_ch, "ulm": ulm,
            "tensor_core_fp16_weights": tc16,
            "gpu_launches": int(launches.value), "clocks": clk, "accuracy": acc,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
