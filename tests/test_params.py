"""Argument handling of the drop-in: the reference wrapper's validation
order, defaults and error identifiers (bfVirtualSourceGeneric_RCA.m:136-455),
and the grid classification.  Host logic only."""
import warnings

import numpy as np
import pytest

from simu_rca_ab_b200.params import RCAError, RCAWarning, grid_spec, normalize
from tests.golden.make_golden import case


def base():
    data, G, T, P, O = case(1, True, False, False)
    return data, dict(G), dict(T), dict(P), dict(O)


def ident(fn):
    with pytest.raises(RCAError) as e, warnings.catch_warnings():
        warnings.simplefilter("ignore", RCAWarning)
        fn()
    return e.value.identifier.split(":")[1]


def test_valid_input_normalizes():
    data, G, T, P, O = base()
    a = normalize(data, G, T, P, O)
    assert a.n_tx == 4 and a.n_ele == 16 and a.grid.kind == 0
    assert a.interp == 0 and a.compounding and not a.mask_transmit


@pytest.mark.parametrize("mutate,expected", [
    (lambda d, G, T, P, O: ("abc", G, T, P, O), "dataNotNumeric"),
    (lambda d, G, T, P, O: (d, G, T, P, 5), "OptionsNotStruct"),
    (lambda d, G, T, P, O: (d, G, T, P, {**O, "flagInterpolationLanczos": 1}), "flagInterpolationLanczosInvalid"),
    (lambda d, G, T, P, O: (d, G, T, P, {**O, "flagCompounding": "yes"}), "flagCompoundingInvalid"),
    (lambda d, G, T, P, O: (d, G, T, P, {**O, "flagMaskTransmit": 0}), "flagMaskTransmitInvalid"),
    (lambda d, G, T, P, O: (d, G, T, P, {**O, "decreaseFactorGPU": 1.5}), "decreaseFactorGPUInvalid"),
    (lambda d, G, T, P, O: (d, {k: v for k, v in G.items() if k != "gridBfY"}, T, P, O), "gridBfMissing"),
    (lambda d, G, T, P, O: (d, {**G, "gridBfY": G["gridBfY"][:2]}, T, P, O), "gridBfInvalid"),
    (lambda d, G, T, P, O: (d, {k: v for k, v in G.items() if k != "posEleZ"}, T, P, O), "posEleMissing"),
    (lambda d, G, T, P, O: (d, {**G, "posEleZ": np.zeros(3)}, T, P, O), "posEleInvalid"),
    (lambda d, G, T, P, O: (d, {**G, "apertureX": [1, 2]}, T, P, O), "apertureXInvalid"),
    (lambda d, G, T, P, O: (d, {**G, "apertureZ": "x"}, T, P, O), "apertureZInvalid"),
    (lambda d, G, T, P, O: (d, G, [1], P, O), "TransmitNotStruct"),
    (lambda d, G, T, P, O: (d, G, {"flagReceiveX": True}, P, O), "ThetaORVirtualSourceRequired"),
    (lambda d, G, T, P, O: (d, G, {**T, "virtualSourceX": [0]}, P, O), "ThetaORVirtualSourceRequired"),
    (lambda d, G, T, P, O: (d, G, {**T, "thetaY": T["thetaY"][:2]}, P, O), "tiltsNotSameLength"),
    (lambda d, G, T, P, O: (d, G, {"virtualSourceX": [0, 0], "virtualSourceY": [0], "virtualSourceZ": [0, 0]}, P, O),
     "virtualSourcesNotSameLength"),
    (lambda d, G, T, P, O: (d, G, {"thetaX": [0.0]}, P, O), "ThetaORVirtualSourceInvalid"),
    (lambda d, G, T, P, O: (d, G, {**T, "flagReceiveX": 1}, P, O), "flagReceiveXInvalid"),
    (lambda d, G, T, P, O: (d, G, T, [], O), "ParamNotStruct"),
    (lambda d, G, T, P, O: (d, G, T, {k: v for k, v in P.items() if k != "samplingFrequency"}, O), "samplingFrequencyMissing"),
    (lambda d, G, T, P, O: (d, G, T, {**P, "samplingFrequency": [1, 2]}, O), "samplingFrequencyInvalid"),
    (lambda d, G, T, P, O: (d, G, T, {k: v for k, v in P.items() if k != "demodulationFrequency"}, O),
     "demodulationFrequencyMissing"),
    (lambda d, G, T, P, O: (d, G, T, {**P, "demodulationFrequency": True}, O), "demodulationFrequencyInvalid"),
    (lambda d, G, T, P, O: (d, G, T, {**P, "speedOfSound": "c"}, O), "speedOfSoundInvalid"),
    (lambda d, G, T, P, O: (d, G, T, {**P, "startTime": [0, 1]}, O), "startTimeInvalid"),
    # the reference reports an invalid f-number with the start-time identifier (RCA.m:449-454)
    (lambda d, G, T, P, O: (d, G, T, {**P, "fnumber": [1, 2]}, O), "startTimeInvalid"),
])
def test_reference_error_identifiers(mutate, expected):
    args = mutate(*base())
    assert ident(lambda: normalize(*args)) == expected


def test_defaults_and_warnings():
    data, G, T, P, O = base()
    for k in ("apertureX", "apertureY", "apertureZ"):
        G.pop(k)
    for k in ("speedOfSound", "startTime", "fnumber"):
        P.pop(k)
    T.pop("flagReceiveX")
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        a = normalize(data, G, T, P, None)
    ids = {str(x.message).split("[")[-1].rstrip("]").split(":")[1] for x in w}
    assert {"apertureXDefault", "apertureYDefault", "apertureZDefault", "thetaToVirtualSource",
            "speedOfSoundDefault", "startTimeDefault", "fnumberDefault"} <= ids
    assert a.c == 1540.0 and a.t0 == 0.0 and a.fnumber == 1.0 and a.receive_x
    assert all(np.isnan(v) for v in a.aperture)
    assert a.interp == 0 and a.compounding and a.mask_transmit and a.decrease_factor == 1


def test_grid_meshgrid_xzy_is_rectilinear():
    x, y, z = np.linspace(-1, 1, 5), np.linspace(-2, 2, 3), np.linspace(1, 4, 7)
    X, Z, Y = np.meshgrid(x, z, y)
    g = grid_spec(X, Y, Z)
    assert g.kind == 0 and (g.n_z, g.n_x, g.n_y) == (7, 5, 3)
    assert (g.stride_z, g.stride_x, g.stride_y) == (1, 7, 35)
    assert np.array_equal(g.x, x) and np.array_equal(g.z, z) and np.array_equal(g.y, y)


def test_grid_other_axis_orders_and_2d():
    x, y, z = np.linspace(-1, 1, 5), np.linspace(-2, 2, 3), np.linspace(1, 4, 7)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    g = grid_spec(X, Y, Z)
    assert g.kind == 0 and (g.stride_x, g.stride_y, g.stride_z) == (1, 5, 15)
    X2, Z2 = np.meshgrid(x, z)
    g2 = grid_spec(X2, np.zeros_like(X2), Z2)
    assert g2.kind == 0 and (g2.n_z, g2.n_x, g2.n_y) == (7, 5, 1) and g2.stride_x == 7


def test_grid_scattered_points():
    rng = np.random.default_rng(0)
    g = grid_spec(rng.normal(size=20), rng.normal(size=20), rng.normal(size=20))
    assert g.kind == 1 and g.n_z == 20 and g.n_x == g.n_y == 1
