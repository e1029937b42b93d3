"""The tensor-core kernel's weight rows (fused_tc_kernel.cuh, the builders),
restated in numpy on the CPU: the barrel shifter that places a voxel's taps
at its row offset inside a 16-row record (and, for the two chunks of a
32-row window, clips them to each chunk), and the split of each weight into
a 16-bit value and its 16-bit remainder.

Checked against direct constructions: every tap lands in its row exactly
once across a window's records, nothing lands outside them, and the value +
remainder pair carries the FP32 weight to ~2^-22 (FP16) / ~2^-16 (BF16)
relative, the precision the kernel's documentation states."""
import numpy as np
import pytest


def barrel_place(w, o, n_pos):
    """tc_place<TAPS, NP>: taps at positions [o, o + TAPS) of NP, shifted by
    log2(NP) select stages (taps pushed past the end drop out)."""
    v = np.zeros(n_pos, np.float32)
    v[:len(w)] = w
    b = 1
    while b < n_pos:
        if o & b:
            v = np.concatenate([np.zeros(b, np.float32), v[:-b]])
        b <<= 1
    return v


def record_rows(w, o, nk, ch):
    """The 16 weights of record `ch` of a window of `nk` 16-row chunks, for
    a voxel whose taps start at row o of the window (the builders' two
    paths: a one-chunk window places at o; a two-chunk window places at
    o + 16 - 16 ch over 32 positions and keeps the upper 16, a start past
    the end leaving the chunk empty)."""
    if nk == 1:
        return barrel_place(w, o, 16)
    e = o + 16 - 16 * ch
    return barrel_place(w, e if e < 32 else 0, 32)[16:]


@pytest.mark.parametrize("taps", [3, 4, 6, 8])
def test_taps_land_once_in_their_rows(taps):
    rng = np.random.default_rng(taps)
    for nk in (1, 2):
        for o in range(0, 16 * nk - taps + 1):
            w = rng.uniform(-1, 1, taps).astype(np.float32)
            full = np.concatenate([record_rows(w, o, nk, ch) for ch in range(nk)])
            ref = np.zeros(16 * nk, np.float32)
            ref[o:o + taps] = w
            assert np.array_equal(full, ref), (taps, nk, o)


def _split(x, dtype):
    """value + remainder, each rounded to the 16-bit type (the builders'
    tc_pack / tc_pack_rem)."""
    if dtype == "f16":
        hi = x.astype(np.float16).astype(np.float32)
        lo = (x - hi).astype(np.float16).astype(np.float32)
    else:   # bf16: round to nearest even on the upper 16 bits
        def bf(a):
            u = a.astype(np.float32).view(np.uint32).astype(np.uint64)
            u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
            return u.astype(np.uint32).view(np.float32)
        hi = bf(x)
        lo = bf((x - hi).astype(np.float32))
    return hi, lo


@pytest.mark.parametrize("dtype,bits", [("f16", 21), ("bf16", 15)])
def test_value_and_remainder_carry_the_weight(dtype, bits):
    """Each weight of a voxel's row is 2^8 x tap weight x the real or
    imaginary part of P (apodisation in (0, 1] x a unit phasor), as the
    builders form it; the value + remainder pair carries it to 2^-bits of the
    row's scale 2^8 |P| (the remainder of a small tail tap may fall into
    FP16's subnormal range, far below that scale)."""
    rng = np.random.default_rng(1)
    n = 200_000
    p_abs = rng.uniform(0.05, 1.0, n)
    phase = rng.uniform(0, 2 * np.pi, n)
    tap = rng.uniform(-0.25, 1.0, n)
    for part in (np.cos(phase), np.sin(phase)):
        x = (256.0 * tap * p_abs * part).astype(np.float32)
        hi, lo = _split(x, dtype)
        err = np.abs((hi.astype(np.float64) + lo) - x.astype(np.float64))
        assert np.all(np.isfinite(hi)) and np.all(np.isfinite(lo))
        assert np.all(err <= 2.0 ** -bits * 256.0 * p_abs)
