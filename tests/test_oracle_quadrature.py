"""The oracle's quadrature rules (QuadratureHub.hpp:39-380) against the reference's own quadrature unit cases
(test/cpp/Geom/test_Quadrature.cpp), restated with the same element kinds, orders, monomials and tolerances.

The reference elements are the line [-1, 1], the quadrilateral [-1, 1]^2, the hexahedron [-1, 1]^3, the triangle
(0,0)-(1,0)-(0,1) and the tetrahedron (0,0,0)-(1,0,0)-(0,1,0)-(0,0,1).  The weights sum to the element measure
(:296-418), and each rule integrates monomials exactly up to the degree the case lists (:420-609).  Comparisons
use doctest's Approx: |a - b| < eps (1 + max(|a|, |b|)).  The GPU's rules are checked against these through
the setup parity of the cell and face integrals."""
from math import factorial

import numpy as np

import oracle

VOLUME = dict(line=2.0, quad=4.0, hex=8.0, tri=0.5, tet=1.0 / 6.0)


def _approx(a, b, eps):
    return abs(a - b) < eps * (1 + max(abs(a), abs(b)))


def _exact(elem, a, b=0, c=0):
    if elem in ("line", "quad", "hex"):
        one = lambda k: 0.0 if k % 2 else 2.0 / (k + 1)
        return one(a) * (one(b) if elem != "line" else 1) * (one(c) if elem == "hex" else 1)
    if elem == "tri":
        return factorial(a) * factorial(b) / factorial(a + b + 2)
    return factorial(a) * factorial(b) * factorial(c) / factorial(a + b + c + 3)


def _numeric(elem, order, a, b=0, c=0):
    p, w = oracle.quad_rule(elem, order)
    return float(np.sum(w * p[:, 0] ** a * p[:, 1] ** b * p[:, 2] ** c))


def test_weight_sums_equal_the_element_measure():
    for elem, vol in VOLUME.items():
        for order in range(0, 7):
            p, w = oracle.quad_rule(elem, order)
            assert len(w) > 0
            assert _approx(float(w.sum()), vol, 1e-12), (elem, order)
    p, w = oracle.quad_rule("tri", 1)  # the one-point rule carries the whole area
    assert len(w) == 1 and _approx(float(w[0]), 0.5, 1e-10)


def test_line_rules():
    for order, deg in ((1, 1), (3, 3), (5, 5), (6, 7)):
        for a in range(0, min(deg, 6) + 1):
            assert _approx(_numeric("line", order, a), _exact("line", a), 1e-12), (order, a)


def test_quad_rules():
    for order, deg in ((1, 1), (3, 3), (5, 5), (6, 5)):
        for a in range(deg + 1):
            for b in range(deg + 1):
                if a + b > 2 * deg:
                    continue
                assert _approx(_numeric("quad", order, a, b), _exact("quad", a, b), 1e-12), (order, a, b)


def test_hex_rules():
    for order, deg in ((1, 1), (3, 3)):
        for a in range(deg + 1):
            for b in range(deg + 1):
                for c in range(deg + 1):
                    assert _approx(_numeric("hex", order, a, b, c), _exact("hex", a, b, c), 1e-12), (order, a, b, c)


def test_triangle_rules():
    for order, deg in ((1, 1), (2, 2), (4, 4), (5, 5), (6, 6)):
        for a in range(deg + 1):
            for b in range(deg + 1 - a):
                assert _approx(_numeric("tri", order, a, b), _exact("tri", a, b), 1e-10), (order, a, b)


def test_tetrahedron_rules():
    for order, deg in ((1, 1), (2, 2), (3, 3), (5, 5), (6, 6)):
        for a in range(deg + 1):
            for b in range(deg + 1 - a):
                for c in range(deg + 1 - a - b):
                    assert _approx(_numeric("tet", order, a, b, c), _exact("tet", a, b, c), 1e-10), (order, a, b, c)


def test_point_counts_of_the_rules_on_the_path():
    """The face and cell rules of the benchmark configurations: 9-point quadrilateral and 7-point triangle faces
    at integration order 5, 3-point line faces, 14-point tetrahedra."""
    assert len(oracle.quad_rule("quad", 5)[1]) == 9
    assert len(oracle.quad_rule("tri", 5)[1]) == 7
    assert len(oracle.quad_rule("line", 5)[1]) == 3
    assert len(oracle.quad_rule("tet", 5)[1]) == 14
    assert len(oracle.quad_rule("hex", 3)[1]) == 8
