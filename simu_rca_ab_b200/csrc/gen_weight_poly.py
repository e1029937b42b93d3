"""Writes weight_poly.h: polynomial forms of the windowed-sinc interpolation
weights used by the fused kernel.

For a kernel K(x) = sinc(x) sinc(x / W) with taps x_j = d + LO - j,
j = 0 .. TAPS-1, d in [0, 1), K is even and the taps are symmetric, so
    w_{TAPS-1-j}(d) = w_j(1 - d).
Each of the TAPS/2 left-hand weights w_j is fitted on u = 2d - 1 in [-1, 1]
by a Chebyshev least-squares fit (FP64, 4001 points) and stored in
monomial form; the right-hand weights are the same polynomials at -u.
Two degrees are written:
  8: maximum weight error (FP64 evaluation) ~1e-6 for the 2-lobe window,
     ~5e-7 for the 3- and 4-lobe windows; FP32 Horner adds ~1e-7.  Used
     for complex64 (FP32) slabs.
  6: maximum weight error 3e-5 .. 8e-5 (RMS 6e-6 .. 1.5e-5), far below the
     ~5e-4 relative rounding of FP16 / BF16 sample storage.  Used for
     FP16 / BF16 slabs: two FMAs fewer per tap pair.

    python gen_weight_poly.py      # rewrites weight_poly.h next to this file
"""
from pathlib import Path

import numpy as np

DEGS = (8, 6)
# name: (LO, TAPS, W, zero outside |x| < W)
KINDS = {
    "K_REF6": (2, 6, 2.0, False),      # the reference's sinc(x) sinc(x/2) (RCA.cu:331-336)
    "K_LANCZOS2": (1, 4, 2.0, True),
    "K_LANCZOS3": (2, 6, 3.0, True),
    "K_LANCZOS4": (3, 8, 4.0, True),
}


def kernel(x, W, lanczos):
    s = np.sinc(x) * np.sinc(x / W)
    return np.where(lanczos & (np.abs(x) >= W), 0.0, s)


def fit(lo, taps, W, lanczos, deg):
    u = np.linspace(-1.0, 1.0, 4001)
    d = (u + 1.0) / 2.0
    coefs, err = [], 0.0
    for j in range(taps // 2):
        y = kernel(d + lo - j, W, lanczos)
        c = np.polynomial.chebyshev.chebfit(u, y, deg)
        mono = np.polynomial.chebyshev.cheb2poly(c)
        err = max(err, float(np.max(np.abs(np.polynomial.polynomial.polyval(u, mono) - y))))
        coefs.append(mono)
    return coefs, err


def main():
    out = ["// Generated by gen_weight_poly.py -- do not edit.",
           "// Polynomials in u = 2d - 1 of the left-hand interpolation weights",
           "// w_j(d), j < TAPS/2; w_{TAPS-1-j}(d) = w_j at -u.  Degree 8 for FP32",
           "// sample storage, degree 6 for FP16 / BF16 sample storage.",
           "// Coefficients live in constant memory (uniform operands of the FMAs).",
           "#pragma once", "", "namespace rcabf {", "",
           "template <int KIND, int DEG> struct WeightPoly;", ""]
    for deg in DEGS:
        for name, (lo, taps, W, lan) in KINDS.items():
            coefs, err = fit(lo, taps, W, lan, deg)
            rows = []
            for mono in coefs:
                rows.append("{" + ", ".join(f"{v:.9e}f" for v in mono) + "}")
            out.append(f"// {name}, degree {deg}: max fit error {err:.2e}")
            out.append(f"static __constant__ float WPOLY{deg}_{name}[{taps // 2}][{deg + 1}] = {{")
            out.append("    " + ",\n    ".join(rows) + "};")
            out.append(f"template <> struct WeightPoly<{name}, {deg}> {{")
            out.append(f"    static constexpr int HALF = {taps // 2};")
            out.append(f"    static __device__ __forceinline__ float c(int j, int m) {{ return WPOLY{deg}_{name}[j][m]; }}")
            out.append("};")
            out.append("")
    out.append("}  // namespace rcabf")
    (Path(__file__).resolve().parent / "weight_poly.h").write_text("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
