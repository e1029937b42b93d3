"""The interpolation-weight polynomials of the voxel-blocked kernel
(`csrc/weight_poly.h`, written by `csrc/gen_weight_poly.py`).

The header is parsed as text and checked three ways:
- it holds the tables the generator writes today (degrees 8 and 6, every
  kernel kind), to the printed precision;
- each table, evaluated as the kernel evaluates it (even and odd Horner
  chains in s = u^2 in FP32, w_{T-1-j}(u) = w_j(-u)), meets the windowed
  sinc it fits (the generator's own kernel function, FP64) within the
  bound stated for its degree: 2e-6 at degree 8 (complex64 slabs), 1e-4
  at degree 6 (FP16 / BF16 slabs, whose stored samples carry ~5e-4
  relative rounding), and within 1e-6 of the FP64 fit's own error;
- the degree-6 RMS weight error stays below 2e-5.
"""
import importlib.util
import re
from pathlib import Path

import numpy as np
import pytest

CSRC = Path(__file__).resolve().parents[1] / "simu_rca_ab_b200" / "csrc"
BOUND = {8: 2e-6, 6: 1e-4}


def _gen():
    spec = importlib.util.spec_from_file_location("gen_weight_poly", CSRC / "gen_weight_poly.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _tables():
    """{(kind, degree): float32 array [HALF][DEG + 1]} parsed from weight_poly.h."""
    text = (CSRC / "weight_poly.h").read_text()
    out = {}
    pat = re.compile(r"static __constant__ float WPOLY(\d+)_(\w+)\[(\d+)\]\[(\d+)\] = \{(.*?)\};", re.S)
    for deg, kind, half, ncoef, body in pat.findall(text):
        rows = re.findall(r"\{([^{}]*)\}", body)
        vals = [[float(v.strip().rstrip("f")) for v in r.split(",")] for r in rows]
        a = np.array(vals, dtype=np.float32)
        assert a.shape == (int(half), int(ncoef)) and int(ncoef) == int(deg) + 1, (kind, deg, a.shape)
        # every table has its template specialisation
        assert f"struct WeightPoly<{kind}, {deg}>" in text, (kind, deg)
        out[(kind, int(deg))] = a
    return out


def _eval_fp32(coef, u):
    """The kernel's evaluation: w_j = E_j(s) + u O_j(s), w_{T-1-j} = E_j - u O_j."""
    f = np.float32
    u = u.astype(f)
    s = (u * u).astype(f)
    deg = coef.shape[1] - 1
    half = coef.shape[0]
    w = np.zeros((2 * half, u.size), np.float32)
    for j in range(half):
        e = np.full_like(u, coef[j, deg])
        for m in range(deg - 2, -1, -2):
            e = (e * s + coef[j, m]).astype(f)
        o = np.full_like(u, coef[j, deg - 1])
        for m in range(deg - 3, 0, -2):
            o = (o * s + coef[j, m]).astype(f)
        w[j] = (u * o + e).astype(f)
        w[2 * half - 1 - j] = (-u * o + e).astype(f)
    return w


@pytest.fixture(scope="module")
def gen():
    return _gen()


@pytest.fixture(scope="module")
def tables():
    return _tables()


def test_header_holds_every_kind_at_both_degrees(gen, tables):
    assert set(gen.DEGS) == {8, 6}
    assert set(tables) == {(k, d) for k in gen.KINDS for d in gen.DEGS}


@pytest.mark.parametrize("deg", [8, 6])
def test_header_matches_the_generator(gen, tables, deg):
    for kind, (lo, taps, W, lan) in gen.KINDS.items():
        coefs, _ = gen.fit(lo, taps, W, lan, deg)
        # the header prints 10 significant digits; the kernel reads FP32
        want = np.array(coefs, dtype=np.float64).astype(np.float32)
        got = tables[(kind, deg)]
        assert np.allclose(got, want, rtol=2e-7, atol=0.0), kind


@pytest.mark.parametrize("deg", [8, 6])
def test_weights_meet_the_windowed_sinc(gen, tables, deg):
    u = np.linspace(-1.0, 1.0, 2001)
    d = (u + 1.0) / 2.0
    for kind, (lo, taps, W, lan) in gen.KINDS.items():
        w = _eval_fp32(tables[(kind, deg)], u)
        assert w.shape[0] == taps
        ref = np.stack([gen.kernel(d + lo - j, W, lan) for j in range(taps)])
        err = np.abs(w.astype(np.float64) - ref)
        _, fit_err = gen.fit(lo, taps, W, lan, deg)   # the FP64 fit's own maximum error
        print(f"{kind} degree {deg}: max {err.max():.2e} (FP64 fit {fit_err:.2e}), "
              f"rms {np.sqrt(np.mean(err ** 2)):.2e}")
        assert err.max() <= BOUND[deg], (kind, err.max())
        # FP32 coefficients and Horner steps add at most 1e-6 to the fit error
        assert err.max() <= fit_err + 1e-6, (kind, err.max(), fit_err)
        if deg == 6:
            assert np.sqrt(np.mean(err ** 2)) <= 2e-5, kind
