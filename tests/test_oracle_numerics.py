"""Known-answer tests of the oracle's numerics against the reference's unit tests:
ErfTest (modules/numerics/src/test/java/ffx/numerics/special/ErfTest.java, 1e-15),
UniformBSplineTest (.../spline/UniformBSplineTest.java, 1e-6) and the
Complex3DParallelTest round trip (.../fft/Complex3DParallelTest.java, 1e-14)."""
import numpy as np
import pytest

from oracle import binding as ob


def test_erfc_known_answers(fixtures):
    num = fixtures["numerics"]
    for x, erf in num["erf"]:
        assert abs(ob.erfc(x) - (1.0 - erf)) <= num["erf_tolerance"], x


def test_bspline_known_answers(fixtures):
    num = fixtures["numerics"]
    tol = num["bspline_tolerance"]
    for case in num["bspline"]:
        out = ob.bspline(case["x"], case["order"])
        assert np.allclose(out[:, 0], case["values"], atol=tol, rtol=0), case
        assert np.allclose(out[:, 1], case["derivs"], atol=tol, rtol=0), case


@pytest.mark.parametrize("shape", [(32, 32, 32), (21, 45, 32), (54, 54, 70)])
def test_fft_round_trip(shape):
    rng = np.random.default_rng(7)
    data = rng.random(shape) + 0j
    back = ob.fft3d(ob.fft3d(data, -1), +1) / data.size
    assert np.max(np.abs(back - data)) < 1e-14


@pytest.mark.parametrize("shape", [(20, 21, 28), (33, 26, 22), (13, 17, 11)])
def test_fft_matches_numpy(shape):
    """Including lengths with prime factors above 7 (the general pass)."""
    rng = np.random.default_rng(8)
    data = rng.random(shape) + 1j * rng.random(shape)
    assert np.allclose(ob.fft3d(data, -1), np.fft.fftn(data), atol=1e-11)
