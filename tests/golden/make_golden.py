"""Generates tests/golden/*.npz: inputs and outputs of the reference RCA
kernel (MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.cu, compiled
from its own source for the host by oracle/Makefile -> oracle/_ref/
librca_ref_cpu.so) on small seeded cases.

    make -C oracle && python tests/golden/make_golden.py

Each file holds the reference wrapper's inputs (data indexed [samples,
channels, 1, events], the Geometry / Transmit / Param / Options fields) and
the per-transmit kernel outputs before compounding (dataBf [frame][tx][pix]
complex64, mask [tx][pix]) plus the compounded outputs in the wrapper's
MATLAB shapes.  The cases cover both interpolation kernels, both receive
orientations, the transmit-cone mask, real (interleaved RF) input, a
non-meshgrid point list, and samples near both ends of the record.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import host as H  # noqa: E402

OUT = Path(__file__).resolve().parent


def case(seed: int, receive_x: bool, lanczos: bool, mask_tx: bool, real: bool = False,
         points: bool = False, n_ele=16, n_tx=4, n_frame=2, ns=96, grid=(24, 12, 10)):
    rng = np.random.default_rng(seed)
    pitch = 0.3e-3
    pos = (np.arange(n_ele) - (n_ele - 1) / 2) * pitch
    zeros = np.zeros(n_ele)
    nz, nx, ny = grid
    lat = (n_ele - 1) * pitch
    x = (np.arange(nx) - (nx - 1) / 2) * lat / nx * 1.2      # a little beyond the aperture
    y = (np.arange(ny) - (ny - 1) / 2) * lat / ny * 1.2
    z = 2e-3 + np.arange(nz) * 0.12e-3
    X, Z, Y = np.meshgrid(x, z, y)
    if points:
        k = nz * nx * ny // 4
        X = rng.uniform(x[0], x[-1], k)
        Y = rng.uniform(y[0], y[-1], k)
        Z = rng.uniform(z[0], z[-1], k)
    G = {"gridBfX": X, "gridBfY": Y, "gridBfZ": Z,
         "posEleX": pos if receive_x else zeros, "posEleY": zeros if receive_x else pos, "posEleZ": zeros,
         "apertureX": lat, "apertureY": lat, "apertureZ": 0.0}
    th = np.deg2rad(np.linspace(-8, 8, n_tx))
    T = {"thetaX": np.zeros(n_tx) if receive_x else th, "thetaY": th if receive_x else np.zeros(n_tx),
         "flagReceiveX": receive_x}
    fs, f0 = 15.6e6, 7.8e6
    P = {"samplingFrequency": fs, "demodulationFrequency": f0, "speedOfSound": 1540.0,
         "startTime": -(2 * 2e-3 / 1540 - 8 / fs), "fnumber": 1.2}
    O = {"flagInterpolationLanczos": lanczos, "flagCompounding": True, "flagMaskTransmit": mask_tx}
    if real:
        data = rng.normal(0, 100, (2 * ns, n_ele, 1, n_tx * n_frame)).astype(np.float32)
    else:
        data = (rng.normal(0, 100, (ns, n_ele, 1, n_tx * n_frame)) +
                1j * rng.normal(0, 100, (ns, n_ele, 1, n_tx * n_frame))).astype(np.complex64)
    return data, G, T, P, O


CASES = {
    "quad3_rx_x": dict(seed=1, receive_x=True, lanczos=False, mask_tx=False),
    "ref6_rx_x": dict(seed=2, receive_x=True, lanczos=True, mask_tx=False),
    "quad3_rx_y_mask": dict(seed=3, receive_x=False, lanczos=False, mask_tx=True),
    "ref6_rx_y_mask": dict(seed=4, receive_x=False, lanczos=True, mask_tx=True),
    "ref6_real_rf": dict(seed=5, receive_x=True, lanczos=True, mask_tx=False, real=True),
    "quad3_points": dict(seed=6, receive_x=True, lanczos=False, mask_tx=False, points=True),
}


# the reference's aberration-law and per-channel kernels (oracle/ref_variant.h):
# name -> (kernel variant, case arguments, aberration law: None / "ele" / "tx_ele")
VARIANT_CASES = {
    "ab1_ref6_rx_x": ("ab1", dict(seed=11, receive_x=True, lanczos=True, mask_tx=False), "ele"),
    "ab2_quad3_rx_y": ("ab2", dict(seed=12, receive_x=False, lanczos=False, mask_tx=False), "tx_ele"),
    "nosum_quad3_rx_x_mask": ("nosum", dict(seed=13, receive_x=True, lanczos=False, mask_tx=True,
                                            grid=(12, 6, 5)), None),
    "nosumab_ref6_rx_y": ("nosumab", dict(seed=14, receive_x=False, lanczos=True, mask_tx=False,
                                          grid=(12, 6, 5)), "ele"),
}


def variant_law(kind, n_tx, n_ch, seed):
    """Seeded receive aberration law (seconds): per element or per (tx, element)."""
    if kind is None:
        return None
    rng = np.random.default_rng(seed + 1000)
    return rng.uniform(-40e-9, 40e-9, (n_tx, n_ch) if kind == "tx_ele" else n_ch)


def main():
    if not H.have_ref_cpu():
        raise SystemExit("oracle/_ref/librca_ref_cpu.so missing: run `make -C oracle` with the reference present")
    for name, (kernel, kw, ab_kind) in VARIANT_CASES.items():
        data, G, T, P, O = case(**kw)
        r = H.prepare(data, G, T, P, O)
        ab = variant_law(ab_kind, r.n_tx, r.n_ch, kw["seed"])
        out, mask_tx = H.run_ref_cpu(r, kernel=kernel, ab_law=ab)
        extra = {} if ab is None else {"ab_law": ab}
        np.savez_compressed(
            OUT / f"{name}.npz", data=data, kernel=np.asarray(kernel),
            **{f"G_{k}": np.asarray(v) for k, v in G.items()},
            **{f"T_{k}": np.asarray(v) for k, v in T.items()},
            **{f"P_{k}": np.asarray(v) for k, v in P.items()},
            **{f"O_{k}": np.asarray(v) for k, v in O.items()},
            out=out.astype(np.complex64), mask_tx=mask_tx.astype(np.float32), **extra)
        print(name, out.shape, float(np.abs(out).max()))
    for name, kw in CASES.items():
        data, G, T, P, O = case(**kw)
        r = H.prepare(data, G, T, P, O)
        per_tx, mask_tx = H.run_ref_cpu(r)
        comp, mcomp = H.compound(per_tx, mask_tx, True)
        db, mk = H.matlab_shape(r, comp, mcomp)
        np.savez_compressed(
            OUT / f"{name}.npz", data=data,
            **{f"G_{k}": np.asarray(v) for k, v in G.items()},
            **{f"T_{k}": np.asarray(v) for k, v in T.items()},
            **{f"P_{k}": np.asarray(v) for k, v in P.items()},
            **{f"O_{k}": np.asarray(v) for k, v in O.items()},
            per_tx=per_tx.astype(np.complex64), mask_tx=mask_tx.astype(np.float32),
            dataBf=db.astype(np.complex64), mask=mk.astype(np.float32))
        print(name, per_tx.shape, float(np.abs(per_tx).max()))


def load(name: str):
    """(data, Geometry, Transmit, Param, Options, outputs) of a fixture."""
    z = np.load(OUT / f"{name}.npz")

    def grab(prefix):
        d = {}
        for k in z.files:
            if k.startswith(prefix):
                v = z[k]
                d[k[len(prefix):]] = bool(v) if v.dtype == bool else (v.item() if v.ndim == 0 else v)
        return d

    outs = {k: z[k] for k in ("per_tx", "mask_tx", "dataBf", "mask", "out", "ab_law", "kernel") if k in z.files}
    return z["data"], grab("G_"), grab("T_"), grab("P_"), grab("O_"), outs


if __name__ == "__main__":
    main()
