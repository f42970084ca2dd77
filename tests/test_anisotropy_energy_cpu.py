"""The oracle's anisotropy fields against the energies they derive from.

No reference test pins the cubic anisotropy (its `Anisotropy_Test` is disabled), so its
restated field (Problems/Anisotropy/CubicAnisotropy.h:133-146) is checked against physics:
H = -(1 / (Ms V)) dE/dm for the cubic energy E = K1 V (c1^2 c2^2 + c2^2 c3^2 + c3^2 c1^2),
c_i = m . a_i, by central differences in m; the uniaxial field (UniaxialAnisotropy.h:143)
against E = K V (m . n)^2 the same way.  The reference's sign conventions hold throughout
(K < 0 is an easy axis for the uniaxial term, K1 is passed unchanged to the cubic one)."""
import math

import numpy as np
import pytest

import oracle

MS, R = 4.8e5, 10e-9
V = 4.0 / 3.0 * math.pi * R ** 3


def euler_axes(phi, theta, psi):
    """Columns of the ZXZ rotation (the body axes x, y, z), as the reference builds them."""
    sp, cp, st, ct, ss, cs = math.sin(phi), math.cos(phi), math.sin(theta), math.cos(theta), math.sin(psi), math.cos(psi)
    x = np.array([cp * cs - ct * sp * ss, ct * sp * cs + cp * ss, st * sp])
    y = np.array([-sp * cs - ct * cp * ss, ct * cp * cs - sp * ss, st * cp])
    z = np.array([st * ss, -st * cs, ct])
    return x, y, z, (sp, st, ss), (cp, ct, cs)


def grad(energy, m, h=1e-6):
    g = np.zeros(3)
    for i in range(3):
        e = np.zeros(3)
        e[i] = h
        g[i] = (energy(m + e) - energy(m - e)) / (2 * h)
    return g


@pytest.mark.parametrize("K1", [-1.1e4, 2.5e4])
def test_cubic_field_is_the_energy_gradient(K1):
    rng = np.random.default_rng(3)
    for _ in range(20):
        x, y, z, s, c = euler_axes(*rng.uniform(0.1, 3.0, 3))
        assert abs(np.dot(x, y)) < 1e-14 and abs(np.dot(y, z)) < 1e-14
        m = rng.normal(size=3)
        m /= np.linalg.norm(m)

        def energy(v):
            c1, c2, c3 = v @ x, v @ y, v @ z
            return K1 * V * (c1 ** 2 * c2 ** 2 + c2 ** 2 * c3 ** 2 + c3 ** 2 * c1 ** 2)

        f, _ = oracle.cubic(K1, MS, R, m, x, y, z, np.array(s), np.array(c))
        expect = -grad(energy, m) / (MS * V)
        np.testing.assert_allclose(f, expect, rtol=1e-6, atol=1e-9 * np.abs(expect).max())


@pytest.mark.parametrize("K", [-1e4, 5e3])
def test_uniaxial_field_is_the_energy_gradient(K):
    rng = np.random.default_rng(4)
    for _ in range(20):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        m = rng.normal(size=3)
        m /= np.linalg.norm(m)
        f, _ = oracle.uniaxial(K, MS, R, m, n)
        expect = -grad(lambda v: K * V * (v @ n) ** 2, m) / (MS * V)
        np.testing.assert_allclose(f, expect, rtol=1e-6, atol=1e-9 * np.abs(expect).max())


def test_cubic_easy_directions_minimise_the_energy():
    """K1 < 0 (magnetite): the <111> directions are the energy minima, so the field there
    is parallel to m (no torque on m), while a <100> direction is an equilibrium too."""
    x, y, z, s, c = euler_axes(0.4, 1.1, 2.0)
    for m in ((x + y + z) / math.sqrt(3), x):
        f, _ = oracle.cubic(-1.1e4, MS, R, m, x, y, z, np.array(s), np.array(c))
        assert np.linalg.norm(np.cross(m, f)) < 1e-9 * max(np.linalg.norm(f), 1.0)
