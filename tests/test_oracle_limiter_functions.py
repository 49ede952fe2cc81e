"""The oracle's WBAP-L2 limiter functions and its pressure compression ratio against the reference's own unit cases
for them (test/cpp/CFV/test_Limiters.cpp:244-286 FWBAP_L2_Biway and :315-343 FWBAP_L2_Multiway,
test/cpp/Euler/test_GasThermo.cpp:447-475 IdealGasGetCompressionRatioPressure), restated with seeded random arrays in
place of Eigen's setRandom (uniform on [-1, 1]); plus the exact values the formulas give."""
import numpy as np

import oracle


def _rand(rng, *shape):
    return rng.uniform(-1.0, 1.0, size=shape)


def test_biway_identical_inputs_pass_through():  # test_Limiters.cpp:244-257
    u1 = _rand(np.random.default_rng(1), 2, 3)
    out = oracle.wbap_l2_biway(u1, u1.copy(), 1.0)
    assert np.allclose(out, u1, rtol=1e-10, atol=0)


def test_biway_no_nan_for_random_inputs():  # :259-266
    rng = np.random.default_rng(2)
    out = oracle.wbap_l2_biway(_rand(rng, 3, 5), _rand(rng, 3, 5), 1.0)
    assert not np.isnan(out).any()


def test_biway_output_non_negative_for_same_sign():  # :268-286
    rng = np.random.default_rng(3)
    u1 = np.abs(_rand(rng, 1, 100)) + 0.1
    u2 = np.abs(_rand(rng, 1, 100)) + 0.1
    out = oracle.wbap_l2_biway(u1, u2, 1.0)
    assert (out >= -1e-10).all()


def test_biway_values():
    # th = u1 / |u2| sign(u2): u1 (n + th^3) / (n + th^4); opposite signs and a zero neighbour limit to 0 or u1 ...
    u1 = np.array([2.0, 2.0, -1.0, 3.0])
    u2 = np.array([1.0, -1.0, 2.0, 0.0])
    out = oracle.wbap_l2_biway(u1, u2, 1.0)
    th = np.array([2.0, -2.0, -0.5, 0.0])
    ref = u1 * (1 + th ** 3) / (1 + th ** 4) * np.abs(np.sign(u2))
    assert np.allclose(out, ref, rtol=1e-14, atol=1e-300)
    assert out[3] == 0.0  # a zero neighbour value cuts the slope


def test_multiway_identical_inputs_pass_through():  # :315-330
    u0 = _rand(np.random.default_rng(4), 2, 3)
    out = oracle.wbap_l2_multiway(np.stack([u0] * 4), 1.0)
    assert np.allclose(out, u0, rtol=1e-8, atol=0)


def test_multiway_no_nan_for_random_inputs():  # :332-343
    rng = np.random.default_rng(5)
    out = oracle.wbap_l2_multiway(np.stack([_rand(rng, 3, 4) for _ in range(5)]), 1.0)
    assert not np.isnan(out).any()


def test_multiway_equals_biway_for_two_inputs():
    rng = np.random.default_rng(6)
    a, b = _rand(rng, 50), _rand(rng, 50)
    assert np.allclose(oracle.wbap_l2_multiway(np.stack([a, b]), 1.0), oracle.wbap_l2_biway(a, b, 1.0), rtol=1e-14, atol=1e-300)


def _prim_to_cons(rho, vx, vy, vz, p, gamma=1.4):
    v = np.array([vx, vy, vz])
    return np.array([rho, *(rho * v), p / (gamma - 1) + 0.5 * rho * v @ v])


def test_compression_ratio_zero_increment():  # test/cpp/Euler/test_GasThermo.cpp:447-456
    U = _prim_to_cons(1.225, 100.0, -50.0, 25.0, 101325.0)
    alpha, bad = oracle.pp_compression_ratio(U, np.zeros(5), 0.0)
    assert abs(alpha) <= 1e-14 and not bad


def test_compression_ratio_in_unit_interval_and_keeps_internal_energy():  # test_GasThermo.cpp:458-475
    U = _prim_to_cons(1.0, 0.0, 0.0, 0.0, 1.0)
    dU = np.array([0.0, 0.0, 0.0, 0.0, -100.0])
    alpha, bad = oracle.pp_compression_ratio(U, dU, 0.0)
    assert 0.0 <= alpha <= 1.0
    Un = U + alpha * dU
    assert Un[4] - 0.5 * Un[0] * np.sum((Un[1:4] / Un[0]) ** 2) >= -1e-10


def test_characteristic_eigenvectors_invert_each_other():  # test/cpp/Euler/test_GasThermo.cpp:174-238
    for rho, v, p in ((1.0, (1.5, -0.3, 0.7), 1.0), (1.225, (300.0, -150.0, 75.0), 101325.0), (1.225, (100.0, -50.0, 25.0), 101325.0)):
        R, L = oracle.euler_eigen(_prim_to_cons(rho, *v, p))
        assert np.abs(L @ R - np.eye(5)).max() < 1e-10, (rho, v, p)
