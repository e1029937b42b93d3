"""Test helper: numpy emulation of the tensor-core Casorati Gram
(csrc/casorati_gram.cu), operation for operation, so that the GPU result can
be checked bit for bit.

The slices follow the kernel's float32 arithmetic (power-of-two scale per
(row, chunk), rint, exact remainders); the integer level sums are exact in
float64 BLAS (every partial sum is an integer below 2^53); levels, chunk
scales, chunks and the complex assembly combine in float64 in the kernel's
order.
"""
from __future__ import annotations

import numpy as np

N_SLICES = 4
N_LEVELS = 5


def chunk_exponents(y32: np.ndarray):
    """Largest-magnitude exponent e (max < 2^e) of each row of a block and
    the flag of rows treated as zero (max below 2^-100, or zero)."""
    m = np.abs(y32).max(axis=1).astype(np.float32)
    E = (m.view(np.uint32) >> 23) & 0xFF
    e = E.astype(np.int64) - 126
    zero = (E == 0) | (e < -100)
    return np.where(zero, 0, e), zero


def slices(y32: np.ndarray, cv: int):
    """y32: float32 [R][P] -> (d [4][R][P] float64 integers, e [R][n_chunks])."""
    R, P = y32.shape
    nch = -(-P // cv)
    d = np.zeros((N_SLICES, R, P))
    e = np.zeros((R, nch), np.int64)
    for c in range(nch):
        sl = slice(c * cv, min(P, (c + 1) * cv))
        blk = y32[:, sl]
        ex, zero = chunk_exponents(blk)
        scale = ((133 - ex).astype(np.uint32) << 23).view(np.float32)
        scale = np.where(zero, np.float32(0), scale).astype(np.float32)
        r = (blk * scale[:, None]).astype(np.float32)
        for s in range(N_SLICES):
            ds = np.rint(r)
            d[s][:, sl] = ds
            r = ((r - ds) * np.float32(128)).astype(np.float32)
        e[:, c] = ex
    return d, e


def real_gram(y32: np.ndarray, cv: int) -> np.ndarray:
    """Y = y y^T as the kernels form it."""
    R, P = y32.shape
    d, e = slices(y32, cv)
    Y = np.zeros((R, R))
    for c in range(e.shape[1]):
        sl = slice(c * cv, min(P, (c + 1) * cv))
        v = None
        for n in range(N_LEVELS):
            A = np.zeros((R, R))
            for s in range(max(0, n - N_SLICES + 1), min(n, N_SLICES - 1) + 1):
                A += d[s][:, sl] @ d[n - s][:, sl].T
            assert np.abs(A).max() < 2 ** 31
            v = A if v is None else v + A * 2.0 ** (-7 * n)
        Y = Y + v * np.ldexp(1.0, e[:, c][:, None] + e[:, c][None, :] - 12)
    return Y


def casorati_gram(x: np.ndarray, cv: int = 16384) -> np.ndarray:
    """x: complex64 [T][P] -> G [T][T] complex128, bit for bit as
    rcabf_casorati_gram (upper triangle of Y, Hermitian assembly)."""
    x = np.asarray(x, np.complex64)
    T, P = x.shape
    y = np.empty((2 * T, P), np.float32)
    y[0::2] = x.real
    y[1::2] = x.imag
    Y = real_gram(y, cv)
    Yu = np.triu(Y) + np.triu(Y, 1).T         # the kernels read the upper triangle only
    re = Yu[0::2, 0::2] + Yu[1::2, 1::2]
    im = Yu[0::2, 1::2] - Yu[1::2, 0::2]
    return re + 1j * im
