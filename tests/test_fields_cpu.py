"""Field waveforms of the oracle against a plain restatement of the reference's
formulas (Fields/*.h), including the triangular, rectangular and sinc fields.

The reference defines the waveforms as follows (units: tesla, seconds).
  triangular (TriangularField.h:52-70): p = (t + t0) mod P (shifted into [0, P));
      B = (2p/(P/2) - 1) A + off if p > P/2, else (-2p/(P/2) + 3) A + off
  rectangular (RectangularField.h:30-63): with 1/tau, the alternating form doubles
      A, shifts t0 and the offset; rising half: A(1 - e^{-p/tau}) + off',
      falling half: A e^{-(p - P/2)/tau} + off' - (A - A_max)
  sinc (SincField.h:32-48): p = (t mod P) - P/2, B = A sinc^2(pi * (22/P) * p) + off
"""
import math

import numpy as np
import pytest

import oracle
from stochasticphysics_b200._abi import FieldSpec

A = np.array([1.0e-2, -4.0e-3, 2.5e-3])
OFF = np.array([1e-4, 0.0, -2e-4])
P = 4.0e-5


def tri(t, t0):
    nt = t + t0
    pos = P + math.fmod(nt, P) if nt < 0 else math.fmod(nt, P)
    w = 2 * pos / (P / 2) - 1 if pos > P / 2 else -2 * pos / (P / 2) + 3
    return w * A + OFF


def rect(t, t0, tau, alternating):
    half = P / 2
    inv = 1.0 / tau
    amp = 2 * A if alternating else A
    maxf = amp * (-math.expm1(-half * inv))
    toff = t0 - math.log(1 - np.linalg.norm(maxf) / (2 * np.linalg.norm(amp))) * tau if alternating else t0
    off = amp * math.expm1(-toff * inv) + OFF if alternating else OFF
    nt = t + toff
    pos = math.fmod(nt + P, P) if nt < 0 else math.fmod(nt, P)
    if pos <= half:
        return amp * (-math.expm1(-pos * inv)) + off
    return amp * math.exp(-(pos - half) * inv) + off - (amp - maxf)


def sinc(t):
    half = P / 2
    pos = (math.fmod(t + P, P) if t < 0 else math.fmod(t, P)) - half
    x = math.pi * (11.0 / half) * pos
    s = 1.0 if x == 0 else math.sin(x) / x
    return A * s * s + OFF


TIMES = np.concatenate([np.linspace(-3 * P, 5 * P, 997), [0.0, P / 2, P, -P / 2, 1e-15]])


@pytest.mark.parametrize("t0", [0.0, 3e-6, -7e-6])
def test_triangular(t0):
    got = oracle.field_eval(FieldSpec.triangular(A, P, t0, OFF), TIMES)
    want = np.array([tri(t, t0) for t in TIMES])
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-18)
    # the reference's waveform swings between A and 3A around the offset
    assert np.all(np.abs(got - OFF) <= 3 * np.abs(A) * (1 + 1e-12))


@pytest.mark.parametrize("alternating", [False, True])
@pytest.mark.parametrize("tau", [2e-6, 5e-5])
def test_rectangular(alternating, tau):
    got = oracle.field_eval(FieldSpec.rectangular(A, P, tau, 1e-6, alternating, OFF), TIMES)
    want = np.array([rect(t, 1e-6, tau, alternating) for t in TIMES])
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-18)


def test_sinc():
    got = oracle.field_eval(FieldSpec.sinc(A, P, OFF), TIMES)
    want = np.array([sinc(t) for t in TIMES])
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-18)
    # peak A + off at the middle of each period
    np.testing.assert_allclose(oracle.field_eval(FieldSpec.sinc(A, P, OFF), [P / 2, 1.5 * P]), [A + OFF] * 2, rtol=1e-15)


def test_sinusoidal_and_lissajous_unchanged():
    t = np.linspace(0, 1e-4, 101)
    s = oracle.field_eval(FieldSpec.sinusoidal(A, 2.5e4, 0.3, OFF), t)
    np.testing.assert_allclose(s, A * np.sin(2 * np.pi * 2.5e4 * t + 0.3)[:, None] + OFF, rtol=1e-12, atol=1e-18)
    lj = oracle.field_eval(FieldSpec.lissajous(A, (2.5e4, 2.6e4, 1e3), (0.0, 0.5, 1.0), OFF), t)
    w = 2 * np.pi * np.array([2.5e4, 2.6e4, 1e3])
    np.testing.assert_allclose(lj, OFF + A * np.sin(np.outer(t, w) + [0.0, 0.5, 1.0]), rtol=1e-12, atol=1e-18)
