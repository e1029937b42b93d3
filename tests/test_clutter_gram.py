"""Tensor-core Casorati Gram (casorati_gram.cu, tcgen05.mma kind::i8), the
C' * C step of SVDClutterFilter.m:25.

CPU: the slice split is exact to 2^-27 of each chunk's largest value; the
emulation of the kernels' arithmetic (tests/gram_emulation.py) is within
1e-9 of max|G| of the FP64 Gram (oracle/clutter.py) on the clutter test
ensemble, and the filter built on it matches the FP64 filter; the tile walk
covers Y's upper triangle.  GPU: the kernels' G equals the emulation bit for
bit (one and several chunks, a partial last chunk, odd frame counts, strided
rows, zero and tiny rows, a 60 dB dynamic range) and the plan's figures."""
import numpy as np
import pytest

from oracle import clutter as OC
from tests import gram_emulation as GE
from tests.test_clutter import CASES, _ensemble


def _fp64_gram(x):
    x64 = np.asarray(x, np.complex128)
    return x64.conj() @ x64.T


def test_slices_reconstruct_each_value():
    rng = np.random.default_rng(0)
    y = (rng.normal(size=(6, 3000)) * np.logspace(-3, 3, 6)[:, None]).astype(np.float32)
    y[2, :100] *= 1e-6                     # small values under a large chunk maximum
    d, e = GE.slices(y, 1024)
    for c in range(e.shape[1]):
        sl = slice(1024 * c, min(3000, 1024 * (c + 1)))
        rec = sum(d[s][:, sl] * 2.0 ** (-7 * s) for s in range(4)) * np.ldexp(1.0, e[:, c] - 6)[:, None]
        bound = np.ldexp(1.0, e[:, c] - 28)[:, None]     # <= 2^-27 of the chunk maximum
        assert (np.abs(rec - y[:, sl].astype(np.float64)) <= bound).all()
        assert np.abs(d[:, :, sl]).max() <= 64


def test_emulated_gram_is_close_to_fp64_and_filters_alike():
    c = _ensemble()                       # [pix][t], 60 dB tissue / blood / noise
    x = np.ascontiguousarray(c.T)
    g = GE.casorati_gram(x, 4096)
    g64 = _fp64_gram(x)
    err = np.abs(g - g64).max() / np.abs(g64).max()
    print(f"emulated int8-slice Gram vs FP64: {err:.2e} of max|G|")
    assert err < 1e-9
    assert np.array_equal(g, g.conj().T)
    ev, vec = np.linalg.eigh(g)
    order = np.argsort(ev)[::-1]
    for w, kind in CASES:
        keep = OC.keep_matlab(64, w, kind)
        v = vec[:, order][:, keep]
        ref, _ = OC.svd_filter_fp64(c, None, keep)
        out = (c.astype(np.complex128) @ v) @ v.conj().T
        rel = np.linalg.norm(out - ref) / np.linalg.norm(ref)
        assert rel < 1e-5, (kind, rel)


def _tiles(rows, nb):
    n_i, n_j = -(-rows // 128), -(-rows // nb)
    out = []
    for J in range(n_j):
        for I in range(min(n_i - 1, (nb * J + nb - 1) // 128) + 1):
            out.append((I, J))
    return out


@pytest.mark.parametrize("nt", [1, 8, 37, 64, 100, 200, 333])
def test_tile_walk_covers_the_upper_triangle(nt):
    from simu_rca_ab_b200.clutter import gram_plan
    p = gram_plan(nt, 50000)
    rows, nb = 2 * nt, p["column_block"]
    tiles = _tiles(rows, nb)
    assert len(tiles) == p["n_tiles"]
    cover = np.zeros((rows, rows), bool)
    for I, J in tiles:
        cover[128 * I:128 * I + 128, nb * J:nb * J + nb] = True
    assert cover[np.triu_indices(rows)].all()
    assert p["n_chunks"] == -(-50000 // p["chunk_voxels"])


def test_plan_rejects_bad_chunks():
    from simu_rca_ab_b200 import _lib as L
    from simu_rca_ab_b200.clutter import gram_plan
    for cv in (100, 131072):
        with pytest.raises(L.RcabfError):
            gram_plan(10, 1000, cv)
    with pytest.raises(L.RcabfError):
        gram_plan(0, 1000)


def _run(x, cv=0, ld=None):
    import torch
    from simu_rca_ab_b200.clutter import casorati_gram
    t = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    if ld is not None:
        buf = torch.zeros((x.shape[0], ld), dtype=torch.complex64, device="cuda")
        buf[:, :x.shape[1]] = t
        t = buf[:, :x.shape[1]]
    g = casorati_gram(t, cv)
    torch.cuda.synchronize()
    return g.cpu().numpy()


def _errcount():
    import ctypes as C

    from simu_rca_ab_b200 import _lib as L
    n = C.c_int64()
    L.check(L.lib().rcabf_take_error_count(C.byref(n)))
    return n.value


def _signal(nt, npx, seed, spread=0.0):
    rng = np.random.default_rng(seed)
    x = (rng.normal(size=(nt, npx)) + 1j * rng.normal(size=(nt, npx)))
    if spread:
        x *= np.logspace(0, spread, npx)[None, :]
    return x.astype(np.complex64)


@pytest.mark.gpu
@pytest.mark.parametrize("nt,npx,cv,ld", [(64, 6000, 0, None), (200, 40000, 0, None), (37, 5000, 1024, None),
                                          (8, 100, 0, None), (1, 777, 64, None), (50, 3000, 512, 3100),
                                          (130, 2048, 2048, None)])
def test_gram_is_bit_exact_against_the_emulation(cuda, nt, npx, cv, ld):
    x = _signal(nt, npx, nt + npx, spread=3.0)
    g = _run(x, cv, ld)
    ref = GE.casorati_gram(x, cv or 16384)
    assert _errcount() == 0
    g64 = _fp64_gram(x)
    print(f"{nt} frames x {npx} pixels (chunk {cv or 16384}): max|G - G_fp64| / max|G| "
          f"{np.abs(g - g64).max() / np.abs(g64).max():.2e}")
    assert np.array_equal(g, ref)


@pytest.mark.gpu
def test_gram_of_the_clutter_ensemble(cuda):
    c = _ensemble()
    x = np.ascontiguousarray(c.T)
    g = _run(x)
    assert np.array_equal(g, GE.casorati_gram(x))
    g64 = _fp64_gram(x)
    assert np.abs(g - g64).max() / np.abs(g64).max() < 1e-9


@pytest.mark.gpu
def test_zero_tiny_and_huge_rows(cuda):
    x = _signal(12, 4000, 3)
    x[2] = 0                     # a zero frame
    x[5, :2000] *= 1e-35         # a chunk whose largest value is below 2^-100 (treated as zero)
    x[7] *= 1e30                 # a huge frame (G up to 1e61, FP64 holds it)
    x[9].imag = 0                # a real frame
    g = _run(x, 1024)
    assert np.array_equal(g, GE.casorati_gram(x, 1024))
    assert np.all(g[2] == 0) and np.all(g[:, 2] == 0)
    assert np.isfinite(g).all()


@pytest.mark.gpu
def test_the_filter_uses_the_tensor_core_gram(cuda):
    """The filter on the tensor-core Gram against the FP64 filter: as close
    as the same filter on an FP64 (ZGEMM) Gram is.  Both share the FP32
    projection, whose rounding (~1e-7 of the input, 60 dB above the blood
    the high-pass keeps) dominates either error."""
    import torch
    from simu_rca_ab_b200.clutter import svd_clutter_filter
    c = _ensemble()
    x = torch.from_numpy(np.ascontiguousarray(c.T)).cuda()
    for w, kind in CASES:
        ref, ev_ref = OC.svd_filter_fp64(c, None, OC.keep_matlab(64, w, kind))
        errs = {}
        for gram in ("tensor_core", "fp64"):
            out, ev = svd_clutter_filter(x, None, w, kind, time_axis=0, order="C", gram=gram)
            got = out.cpu().numpy().T
            errs[gram] = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert np.allclose(ev.cpu().numpy(), ev_ref, rtol=1e-6, atol=1e-8 * ev_ref[0])
        print(kind, w, "filtered vs FP64 filter: tensor-core Gram "
              f"{errs['tensor_core']:.2e}, FP64 ZGEMM Gram {errs['fp64']:.2e}")
        assert errs["tensor_core"] < 1e-4
        assert errs["tensor_core"] < 1.5 * errs["fp64"] + 1e-6
