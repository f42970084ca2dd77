"""CPU checks of the oracle itself: Philox known answers, determinism, precision."""
import dataclasses

import numpy as np

import oracle
from stochasticphysics_b200 import provider
from stochasticphysics_b200._abi import Solver


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors published with Random123 (Salmon et al., SC'11)."""
    assert oracle.philox4x32_10([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert oracle.philox4x32_10([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert oracle.philox4x32_10([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_normals_are_standard():
    z = oracle.philox_normals(123, 0, 20000, 0, 3, 3).ravel()
    assert abs(z.mean()) < 0.02 and abs(z.std() - 1.0) < 0.02


def test_thread_count_does_not_change_results():
    spec = provider.neel_relaxation(n=200, steps=1000, oversampling=100)
    a = oracle.simulate(spec, threads=1)
    b = oracle.simulate(spec, threads=5)
    np.testing.assert_array_equal(a["mean"], b["mean"])


def test_sharded_particles_recombine():
    """Particles are independent: two shards with their global ids give the full ensemble."""
    spec = provider.neel_relaxation(n=300, steps=1000, oversampling=100)
    full = oracle.simulate(spec)
    parts = [oracle.simulate(spec.subset(0, 128)), oracle.simulate(spec.subset(128, 300))]
    w = sum(p["weight"] for p in parts)
    mean = sum(p["mean"] * p["weight"] for p in parts) / w
    np.testing.assert_allclose(mean, full["mean"], rtol=1e-12, atol=1e-14)


def test_long_double_agrees_with_double():
    spec = provider.with_injected_noise(provider.brown_neel_relaxation(n=16, steps=1000, oversampling=100), seed=2)
    a = oracle.simulate(spec, trajectories=True)
    b = oracle.simulate(spec, trajectories=True, long_double=True)
    assert np.max(np.abs(a["trajectories"] - b["trajectories"])) < 1e-10


def test_zero_temperature_is_deterministic():
    spec = dataclasses.replace(provider.neel_relaxation(n=8, steps=1000, oversampling=100), temperature=0.0,
                               solver=Solver.EulerMaruyama)
    a = oracle.simulate(spec)
    b = oracle.simulate(dataclasses.replace(spec, seed=999))
    np.testing.assert_array_equal(a["mean"], b["mean"])


def test_op_counts_are_positive():
    ops = oracle.count_ops(provider.neel_relaxation(n=1, steps=1000, oversampling=100))
    assert 80 < ops["flops"] < 400
    ops_bn = oracle.count_ops(provider.brown_neel_relaxation(n=1, steps=1000, oversampling=100))
    assert ops_bn["flops"] > ops["flops"] and ops_bn["transcendentals"] > 5


def test_euler_maruyama_normalized_keeps_unit_vectors():
    """EulerMaruyama_Normalized.inl:40-56 on the CPU: after every step |m| = 1 (and
    |n| = 1 for the coupled Cartesian problem), while plain EulerMaruyama drifts."""
    import dataclasses
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Problem, Solver
    base = provider.neel_relaxation(n=32, steps=500, oversampling=100)
    em = oracle.simulate(dataclasses.replace(base, solver=Solver.EulerMaruyama), final_state=True)
    emn = oracle.simulate(dataclasses.replace(base, solver=Solver.EulerMaruyama_Normalized), final_state=True)
    np.testing.assert_allclose(np.linalg.norm(emn["final_state"], axis=1), 1.0, rtol=1e-14)
    assert np.abs(np.linalg.norm(em["final_state"], axis=1) - 1).max() > 1e-9


def test_reference_millstein_does_not_keep_the_langevin_equilibrium():
    """The reference's Millstein step (Millstein.inl:35-44) adds the Ito-Stratonovich
    drift as D |dW|^2 summed over all noise components, where a consistent scheme adds
    D dt.  With zero anisotropy in a constant field the Heun step relaxes to the
    Langevin value coth(xi) - 1/xi; the Millstein step as written does not (the
    Cartesian magnetisation even shrinks).  The engine keeps the reference's formula;
    this test pins the behaviour so that it stays documented."""
    import dataclasses
    import math
    import stochasticphysics_b200 as sp
    from stochasticphysics_b200 import provider
    from stochasticphysics_b200._abi import Solver
    n, B = 512, 0.01
    rng = np.random.default_rng(21)
    v = rng.standard_normal((n, 3))
    m0 = v / np.linalg.norm(v, axis=1, keepdims=True)
    V = 4 / 3 * math.pi * (10e-9) ** 3
    xi = 4.8e5 * V * B / (1.3806485279e-23 * 295)
    langevin = 1 / math.tanh(xi) - 1 / xi
    out = {}
    for solver in (Solver.Heun_Strong, Solver.Millstein):
        spec = dataclasses.replace(provider.neel_relaxation(n=n, steps=20000, oversampling=1000, solver=solver),
                                   anisotropy_constant=np.zeros(n), magnetisation=m0,
                                   field=sp.FieldSpec.constant((0.0, 0.0, B)))
        out[solver] = oracle.simulate(spec)["mean"][10:, 2].mean()
    assert abs(out[Solver.Heun_Strong] - langevin) < 4 / math.sqrt(3 * n)
    assert out[Solver.Millstein] < 0.5 * langevin
