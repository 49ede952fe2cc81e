"""The oracle's positivity-preserving increment limiting (EulerEvaluator.hxx:1938-2140,
EulerEvaluator.hpp:1645-1857, Gas.hpp:1750-1860): a hand-derived known answer and the
properties the reference's routines guarantee (no CPU fallback of the product is involved)."""
import numpy as np

import oracle

GAMMA = 1.4


def _state(rng, n):
    u = np.zeros((n, 5))
    u[:, 0] = 1 + 0.5 * rng.random(n)
    v = rng.normal(size=(n, 3)) * 0.5
    u[:, 1:4] = u[:, :1] * v
    u[:, 4] = (1 + rng.random(n)) / (GAMMA - 1) + 0.5 * u[:, 0] * (v ** 2).sum(1)
    return u


def _p(u):
    return (GAMMA - 1) * (u[:, 4] - 0.5 * (u[:, 1:4] ** 2).sum(1) / u[:, 0])


def test_density_only_known_answer():
    # rho 1, p 1 at rest; a density increment of -2 at relax 0.9: alphaRho = (1 - relaxedRho) / (2 + 2e-10)
    # with relaxedRho = 0.9 rhoEps + 0.1; the pressure stays 1, so alpha = alphaRho^2 (compress 2) * (1 - 1e-5)
    u = np.array([[1.0, 0, 0, 0, 1.0 / (GAMMA - 1)]])
    inc = np.array([[-2.0, 0, 0, 0, 0]])
    a, n, amin, bad = oracle.cell_rhs_alpha(u, inc, 1.0, 1.0, relax=0.9)
    rhoEps = 1e-10 * 1.0 * 1e-1
    aRho = (1 - (rhoEps * 0.9 + 0.1)) / (2 + 1e-10 * 2)
    assert not bad and n == 1
    assert abs(a[0] - aRho ** 2 * (1 - 1e-5)) < 1e-15 and amin == a[0]


def test_small_increments_are_untouched():
    rng = np.random.default_rng(1)
    u = _state(rng, 500)
    inc = rng.normal(size=u.shape) * 1e-3
    a, n, amin, bad = oracle.cell_rhs_alpha(u, inc, 1.0, 1.0)
    assert n == 0 and amin == 1.0 and not bad and np.all(a == 1.0)
    un, fix, bad = oracle.add_fixed_increment(u, inc, 1.0, 1.0, 1.0)
    assert fix == 1.0 and not bad and np.array_equal(un, u + inc)


def test_alpha_keeps_the_relaxed_floors_and_the_flags():
    rng = np.random.default_rng(2)
    u = _state(rng, 4000)
    inc = rng.normal(size=u.shape) * np.array([0.8, 0.8, 0.8, 0.8, 3.0])
    for relax in (0.9, 1.0):
        a, n, amin, bad = oracle.cell_rhs_alpha(u, inc, 1.0, 1.0, relax=relax)
        assert not bad and 0 < n < len(u) and 0 <= amin < 1
        assert np.all((a > 0) & (a <= 1)) and amin == a.min()
        un = u + a[:, None] * inc
        rhoEps = 1e-11
        # the density floor relaxed towards the old density, the pressure positive
        assert np.all(un[:, 0] >= rhoEps * relax + u[:, 0] * (1 - relax) - 1e-12)
        assert np.all(_p(un) > 0)
        a1, _, _, _ = oracle.cell_rhs_alpha(u, inc, 1.0, 1.0, relax=relax, flag=1)
        assert np.all(a1[a < 1] == amin) and np.all(a1[a == 1] == 1)
        a2, _, _, _ = oracle.cell_rhs_alpha(u, inc, 1.0, 1.0, relax=relax, flag=2)
        assert np.all(a2 == amin)
        ae = oracle.cell_rhs_alpha_expansion(u, inc, np.ones(len(u)), 1.0, 1.0, amin)
        bad_new = (_p(u + inc) < 1e-11) | ((u + inc)[:, 0] < 1e-11)
        assert np.all(ae[bad_new] == amin) and np.all(ae[~bad_new] == 1)


def test_add_fixed_increment_keeps_density_and_pressure_positive():
    rng = np.random.default_rng(3)
    u = _state(rng, 4000)
    inc = rng.normal(size=u.shape) * np.array([2.0, 2.0, 2.0, 2.0, 8.0])
    un, fix, bad = oracle.add_fixed_increment(u, inc, 1.0, 1.0, 1.0)
    assert not bad and 0 < fix < 1
    assert np.all(un[:, 0] > 0) and np.all(_p(un) > 0)
    ok = ((u + inc)[:, 0] > 1e-11) & (_p(u + inc) > 1e-11)
    assert np.array_equal(un[ok], (u + inc)[ok])
    # the SA variable (6th) stays non-negative
    u6 = np.concatenate([u, np.abs(rng.normal(size=(len(u), 1)))], 1)
    i6 = np.concatenate([inc, rng.normal(size=(len(u), 1)) * 3], 1)
    un6, _, bad6 = oracle.add_fixed_increment(u6, i6, 1.0, 1.0, 1.0)
    assert not bad6 and np.all(un6[:, 5] >= 0) and np.allclose(un6[:, :5], un)
