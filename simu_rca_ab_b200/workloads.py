"""Benchmark / test workloads and their seeded synthetic channel data.

Five acquisitions (RCA probes, plane-wave transmits, voxel grids) with the
sizes of the configurations this beamformer is measured on:

  c0  64+64 probe, 16 row plane waves -8..8 deg, [512 x 64 x 16 x 1] complex64,
      grid 64 x 64 x 128, f-number 1.5, Lanczos a = 3 (CPU-runnable case)
  c1  128+128 probe, 16 row + 16 column plane waves -10..10 deg (two receive
      orientations, compounded), [1024 x 128 x 32 x 8], grid 128 x 128 x 256,
      f-number 1.2, Lanczos a = 4
  c2  Doppler ensemble: 11 row plane waves -5..5 deg, [768 x 128 x 11 x 200],
      FP16/BF16 storage, grid 96 x 96 x 160, f-number 1.2, Lanczos a = 4
  c3  serving mix: a seeded stream of requests of mixed sizes (serving_mix)
  c4  256+256 probe, 32 row + 32 column plane waves -12..12 deg,
      [2048 x 256 x 64 x 4] FP16, grid 256 x 256 x 384, f-number 1.0, Lanczos a = 4

No public dataset is involved: point scatterers are drawn from
``numpy.random.default_rng(seed)``; each contributes a 2-cycle
Gaussian-enveloped pulse at its exact round-trip delay under the same
virtual-source transmit / element receive model the beamformer inverts,
demodulated at f0, plus circular complex Gaussian noise at -30 dB of the
noiseless signal's RMS.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

C_SOUND = 1540.0


def _deg(a):
    return np.deg2rad(np.asarray(a, dtype=np.float64))


@dataclass
class Group:
    """One receive orientation: the reference wrapper's Geometry/Transmit."""
    Geometry: dict
    Transmit: dict
    tx0: int          # first transmit of this group in the data's transmit axis
    n_tx: int


@dataclass
class Workload:
    name: str
    n_sample: int
    n_frame: int
    n_ele: int
    Param: dict
    Options: dict
    groups: list
    grid_shape: tuple           # (Nz, Nx, Ny)
    lanczos_a: int
    storage: str = "float32"
    scatter: dict = field(default_factory=dict)

    @property
    def n_tx(self) -> int:
        return sum(g.n_tx for g in self.groups)

    @property
    def n_pix(self) -> int:
        return int(np.prod(self.grid_shape))

    def units(self) -> int:
        """Nominal voxel.rx.tx count summed over frames."""
        return self.n_pix * self.n_ele * self.n_tx * self.n_frame

    def flop_per_unit(self) -> int:
        taps = {0: 3, 1: 6}.get(self._interp_code(), 2 * self.lanczos_a)
        return 4 * taps + 8 if taps != 3 else 20

    def _interp_code(self):
        it = str(self.Options.get("interpolation", "lanczos")).lower()
        return {"quadratic": 0, "ref6": 1}.get(it, 2)


def rca_probe(n: int, pitch: float):
    pos = (np.arange(n) - (n - 1) / 2.0) * pitch
    return pos


def make_grid(nx: int, ny: int, nz: int, lat_x: float, lat_y: float, z0: float, z_span: float):
    x = (np.arange(nx) - (nx - 1) / 2.0) * (lat_x / nx)
    y = (np.arange(ny) - (ny - 1) / 2.0) * (lat_y / ny)
    z = z0 + np.arange(nz) * (z_span / nz)
    X, Z, Y = np.meshgrid(x, z, y)  # [Nz, Nx, Ny] (script_All.m:198)
    return X, Y, Z


def _group(n, pitch, receive_x, thetas, X, Y, Z, tx0):
    pos = rca_probe(n, pitch)
    zeros = np.zeros(n)
    ap = (n - 1) * pitch
    G = {"gridBfX": X, "gridBfY": Y, "gridBfZ": Z,
         "posEleX": pos if receive_x else zeros, "posEleY": zeros if receive_x else pos, "posEleZ": zeros,
         "apertureX": ap, "apertureY": ap, "apertureZ": 0.0}
    th = _deg(thetas)
    T = {"thetaX": np.zeros_like(th) if receive_x else th,
         "thetaY": th if receive_x else np.zeros_like(th), "flagReceiveX": bool(receive_x)}
    return Group(G, T, tx0, th.size)


def get(name: str, *, n_frame: int | None = None, grid_scale: float = 1.0) -> Workload:
    """Workload by name; ``n_frame`` / ``grid_scale`` shrink it for tests."""
    name = name.lower()
    if name == "c0":
        n, pitch, f0, fs, ns, nf = 64, 0.3e-3, 7.8e6, 15.6e6, 512, 1
        nx = ny = 64
        nz = 128
        lat, z0, zs = 19e-3, 5e-3, 20e-3
        fnum, a = 1.5, 3
        tx = [(True, np.linspace(-8, 8, 16))]
        scat = {"n": 200, "x": (-9.5e-3, 9.5e-3), "y": (-9.5e-3, 9.5e-3), "z": (5e-3, 25e-3)}
    elif name == "c1":
        n, pitch, f0, fs, ns, nf = 128, 0.2e-3, 7.8e6, 15.6e6, 1024, 8
        nx = ny = 128
        nz = 256
        lat, z0, zs = 25.4e-3, 5e-3, 25e-3
        fnum, a = 1.2, 4
        tx = [(True, np.linspace(-10, 10, 16)), (False, np.linspace(-10, 10, 16))]
        scat = {"n": 1000, "x": (-12.7e-3, 12.7e-3), "y": (-12.7e-3, 12.7e-3), "z": (5e-3, 30e-3),
                "jitter": 5e-6}
    elif name == "c2":
        n, pitch, f0, fs, ns, nf = 128, 0.2e-3, 7.8e6, 15.6e6, 768, 200
        nx = ny = 96
        nz = 160
        lat, z0, zs = 25.4e-3, 5e-3, 25e-3
        fnum, a = 1.2, 4
        tx = [(True, np.linspace(-5, 5, 11))]
        scat = {"n": 2000, "x": (-12.7e-3, 12.7e-3), "y": (-12.7e-3, 12.7e-3), "z": (5e-3, 30e-3),
                "vessel": {"n": 300, "radius": 1e-3, "y": 0.0, "z": 17.5e-3, "vmax": 20e-3, "prf": 5e3}}
    elif name == "c4":
        n, pitch, f0, fs, ns, nf = 256, 0.2e-3, 5e6, 10e6, 2048, 4
        nx = ny = 256
        nz = 384
        lat, z0, zs = 51.2e-3, 5e-3, 40e-3
        fnum, a = 1.0, 4
        tx = [(True, np.linspace(-12, 12, 32)), (False, np.linspace(-12, 12, 32))]
        scat = {"n": 5000, "x": (-25.6e-3, 25.6e-3), "y": (-25.6e-3, 25.6e-3), "z": (5e-3, 45e-3),
                "layer": {"n": 2000, "z": (20e-3, 24e-3), "gain_db": 10.0}}
    else:
        raise KeyError(f"unknown workload {name!r} (c0, c1, c2, c4; c3 is the serving mix)")
    if n_frame is not None:
        nf = n_frame
    if grid_scale != 1.0:
        nx = max(1, int(round(nx * grid_scale)))
        ny = max(1, int(round(ny * grid_scale)))
        nz = max(1, int(round(nz * grid_scale)))
    X, Y, Z = make_grid(nx, ny, nz, lat, lat, z0, zs)
    groups, t0i = [], 0
    for rx, th in tx:
        g = _group(n, pitch, rx, th, X, Y, Z, t0i)
        groups.append(g)
        t0i += g.n_tx
    Param = {"samplingFrequency": fs, "demodulationFrequency": f0, "speedOfSound": C_SOUND,
             "startTime": -(2 * z0 / C_SOUND - 16 / fs), "fnumber": fnum}
    Options = {"flagCompounding": True, "flagMaskTransmit": False, "interpolation": "lanczos",
               "lanczosOrder": a}
    return Workload(name, ns, nf, n, Param, Options, groups, (nz, nx, ny), a,
                    storage="float16" if name in ("c2", "c4") else "float32", scatter=scat)


# ---------------------------------------------------------------------------
# c3: the serving mix
# ---------------------------------------------------------------------------
C3_GRIDS = [(64, 32, 32), (128, 64, 64), (160, 96, 96), (256, 128, 128)]   # (Nz, Nx, Ny)
C3_TX = [1, 2, 4, 8, 16, 32]


def c3_workload(probe: int, n_tx: int, grid: tuple, n_frame: int) -> Workload:
    """One serving-mix acquisition: a 64+64 probe (the c0 physics) or a
    128+128 probe (the c1 physics), n_tx row plane waves received on the
    columns, the given grid over the probe's field of view, f-number 1.5 and
    Lanczos a = 3 for every request, synthesis as c0 (200 scatterers)."""
    if probe == 64:
        pitch, f0, fs, ns, lat, z0, zs, span = 0.3e-3, 7.8e6, 15.6e6, 512, 19e-3, 5e-3, 20e-3, 8.0
    elif probe == 128:
        pitch, f0, fs, ns, lat, z0, zs, span = 0.2e-3, 7.8e6, 15.6e6, 1024, 25.4e-3, 5e-3, 25e-3, 10.0
    else:
        raise ValueError("probe is 64 or 128 elements per side")
    nz, nx, ny = grid
    X, Y, Z = make_grid(nx, ny, nz, lat, lat, z0, zs)
    th = np.linspace(-span, span, n_tx) if n_tx > 1 else np.zeros(1)
    g = _group(probe, pitch, True, th, X, Y, Z, 0)
    Param = {"samplingFrequency": fs, "demodulationFrequency": f0, "speedOfSound": C_SOUND,
             "startTime": -(2 * z0 / C_SOUND - 16 / fs), "fnumber": 1.5}
    Options = {"flagCompounding": True, "flagMaskTransmit": False, "interpolation": "lanczos", "lanczosOrder": 3}
    half = lat / 2
    scat = {"n": 200, "x": (-half, half), "y": (-half, half), "z": (z0, z0 + zs)}
    return Workload(f"c3-{probe}-{n_tx}tx-{nz}x{nx}x{ny}", ns, n_frame, probe, Param, Options, [g], (nz, nx, ny), 3,
                    storage="float32", scatter=scat)


@dataclass
class ServeRequest:
    probe: int
    n_tx: int
    grid: tuple
    n_frame: int
    storage: str          # "float32" | "float16"
    arrival_s: float      # Poisson arrival time from the start of the stream


def serving_mix(seed: int, n_requests: int, rate_hz: float, max_frames: int = 64) -> list:
    """Seeded request stream: probe 64+64 or 128+128, 1-32 transmits, 1-64
    frames, grids from 32x32x64 to 128x128x256, FP32 or FP16 storage,
    exponential inter-arrival times at ``rate_hz``."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n_requests))
    out = []
    for k in range(n_requests):
        out.append(ServeRequest(probe=int(rng.choice([64, 128])), n_tx=int(rng.choice(C3_TX)),
                                grid=C3_GRIDS[int(rng.integers(len(C3_GRIDS)))],
                                n_frame=int(rng.integers(1, max_frames + 1)),
                                storage=str(rng.choice(["float32", "float16"])), arrival_s=float(t[k])))
    return out


# ---------------------------------------------------------------------------
# Scatterers and channel data
# ---------------------------------------------------------------------------
def scatterers(w: Workload, seed: int):
    """Positions [F][S][3] and amplitudes [F][S] (float64 numpy)."""
    rng = np.random.default_rng(seed)
    sc = w.scatter
    nf = w.n_frame

    def uniform(k, box):
        return np.stack([rng.uniform(*box["x"], k), rng.uniform(*box["y"], k), rng.uniform(*box["z"], k)], -1)

    base = uniform(sc["n"], sc)
    amp = rng.rayleigh(1.0, sc["n"])
    pos = np.repeat(base[None], nf, 0)
    amps = np.repeat(amp[None], nf, 0)
    if "jitter" in sc:
        steps = rng.normal(0.0, sc["jitter"], (nf, sc["n"], 3))
        steps[0] = 0.0
        pos = pos + np.cumsum(steps, axis=0)
    if "layer" in sc:
        L = sc["layer"]
        lay = np.stack([rng.uniform(*sc["x"], L["n"]), rng.uniform(*sc["y"], L["n"]),
                        rng.uniform(*L["z"], L["n"])], -1)
        la = rng.rayleigh(1.0, L["n"]) * 10 ** (L["gain_db"] / 20)
        pos = np.concatenate([pos, np.repeat(lay[None], nf, 0)], 1)
        amps = np.concatenate([amps, np.repeat(la[None], nf, 0)], 1)
    if "vessel" in sc:
        V = sc["vessel"]
        r = V["radius"] * np.sqrt(rng.uniform(0, 1, V["n"]))
        ang = rng.uniform(0, 2 * np.pi, V["n"])
        x0 = rng.uniform(*sc["x"], V["n"])
        v = V["vmax"] * (1 - (r / V["radius"]) ** 2)          # parabolic profile, along x
        f = np.arange(nf)[:, None]
        span = sc["x"][1] - sc["x"][0]
        xs = (x0[None] + v[None] * f / V["prf"] - sc["x"][0]) % span + sc["x"][0]
        ys = np.broadcast_to(V["y"] + r * np.cos(ang), (nf, V["n"]))
        zs = np.broadcast_to(V["z"] + r * np.sin(ang), (nf, V["n"]))
        vp = np.stack([xs, ys, zs], -1)
        pos = np.concatenate([pos, vp], 1)
        amps = np.concatenate([amps, np.repeat(rng.rayleigh(1.0, V["n"])[None], nf, 0)], 1)
    return pos, amps


def _sources(group: Group):
    """Virtual sources and min distance exactly as the reference wrapper
    derives them (RCA.m:500-502, 527-558), in float64."""
    G, T = group.Geometry, group.Transmit
    ex = np.asarray(G["posEleX"], float).ravel()
    ey = np.asarray(G["posEleY"], float).ravel()
    ez = np.asarray(G["posEleZ"], float).ravel()
    ex, ey, ez = ex - ex.mean(), ey - ey.mean(), ez - ez.mean()
    tx_, ty_ = np.tan(np.asarray(T["thetaX"], float)), np.tan(np.asarray(T["thetaY"], float))
    vz = -10.0 / np.sqrt(1 + tx_ ** 2 + ty_ ** 2)
    vx, vy = vz * tx_, vz * ty_
    md = np.sqrt((ey[None] - vx[:, None]) ** 2 + (ex[None] - vy[:, None]) ** 2 + (ez[None] - vz[:, None]) ** 2).min(1)
    return ex, ey, ez, vx, vy, vz, md


def channel_data(w: Workload, seed: int = 0, device="cpu", noise_db: float = -30.0, frames=None):
    """Seeded channel data [frame][tx][element][sample] complex64 (torch).

    IQ(n) = sum_s A_s g(n/fs - t0 - tau_s) exp(-j 2 pi f0 (tau_s + t0)) + noise,
    tau_s = transmit delay (virtual-source model, RCA.cu:256-269) + receive
    delay (RCA.cu:308) evaluated in float64; g is a Gaussian envelope of
    2 cycles FWHM.
    """
    import torch

    pos, amp = scatterers(w, seed)
    if frames is not None:
        pos, amp = pos[frames], amp[frames]
    nf = pos.shape[0]
    fs, f0, c, t0 = (w.Param[k] for k in ("samplingFrequency", "demodulationFrequency", "speedOfSound", "startTime"))
    ns = w.n_sample
    sigma = 0.85 / f0
    K = int(math.ceil(4 * sigma * fs))
    dev = torch.device(device)
    out = torch.zeros((nf, w.n_tx, w.n_ele, ns), dtype=torch.complex64, device=dev)
    P = torch.as_tensor(pos, dtype=torch.float64, device=dev)
    A = torch.as_tensor(amp, dtype=torch.float64, device=dev)
    taps = torch.arange(-K, K + 1, device=dev, dtype=torch.float64)
    fchunk = max(1, int(2e7 // max(1, P.shape[1] * w.n_ele * (2 * K + 1))))
    for g in w.groups:
        ex, ey, ez, vx, vy, vz, md = (torch.as_tensor(a, dtype=torch.float64, device=dev) for a in _sources(g))
        rx = bool(g.Transmit["flagReceiveX"])
        eu = ex if rx else ey
        for t in range(g.n_tx):
            for f0i in range(0, nf, fchunk):
                p = P[f0i:f0i + fchunk]                                   # [f, S, 3]
                a = A[f0i:f0i + fchunk]
                su, sv, sz = (p[..., 0], p[..., 1], p[..., 2]) if rx else (p[..., 1], p[..., 0], p[..., 2])
                vv = vy[t] if rx else vx[t]
                ttx = (torch.sqrt((sv - vv) ** 2 + (sz - vz[t]) ** 2) - md[t]) / c   # [f, S]
                trx = torch.sqrt((su[..., None] - eu) ** 2 + (sz[..., None] - ez) ** 2) / c  # [f, S, E]
                tau = ttx[..., None] + trx
                idx = (tau + t0) * fs
                n0 = torch.round(idx)
                n = n0[..., None] + taps                                   # [f, S, E, taps]
                env = torch.exp(-0.5 * ((n - idx[..., None]) / (fs * sigma)) ** 2)
                ph = -2 * math.pi * f0 * (tau + t0)
                val = (a[..., None, None] * env) * torch.polar(torch.ones_like(ph), ph)[..., None]
                ok = (n >= 0) & (n < ns)
                ni = n.clamp(0, ns - 1).to(torch.int64)
                fi = torch.arange(p.shape[0], device=dev)[:, None, None, None]
                ei = torch.arange(w.n_ele, device=dev)[None, None, :, None]
                flat = ((fi + f0i) * w.n_tx + (g.tx0 + t)) * w.n_ele * ns + ei * ns + ni
                vals = torch.where(ok, val, torch.zeros_like(val)).to(torch.complex64)
                out.view(-1).index_add_(0, flat.reshape(-1), vals.reshape(-1))
    if noise_db is not None:
        gen = torch.Generator(device=dev)
        gen.manual_seed(int(seed) * 7919 + 17)
        rms = torch.sqrt(torch.mean(out.real.double() ** 2 + out.imag.double() ** 2)).item()
        s = rms * 10 ** (noise_db / 20) / math.sqrt(2)
        noise = torch.complex(torch.randn(out.shape, generator=gen, device=dev),
                              torch.randn(out.shape, generator=gen, device=dev)) * s
        out += noise.to(torch.complex64)
    return out


def group_data(w: Workload, data, gi: int):
    """Channel data of one receive orientation, [frame][tx][element][sample]."""
    g = w.groups[gi]
    return data[:, g.tx0:g.tx0 + g.n_tx]


def as_matlab(data_ftes):
    """[frame][tx][element][sample] -> the reference's [samples, channels, 1, events]
    indexing (a strided view for torch, a Fortran-ordered view for numpy)."""
    try:
        import torch
        if isinstance(data_ftes, torch.Tensor):
            F, T, E, S = data_ftes.shape
            return data_ftes.reshape(F * T, 1, E, S).permute(3, 2, 1, 0)
    except ImportError:  # pragma: no cover
        pass
    a = np.asarray(data_ftes)
    F, T, E, S = a.shape
    return a.reshape(F * T, 1, E, S).transpose(3, 2, 1, 0)
