"""The oracle's shape functions (Geom/Elements/{Line2,Tri3,Quad4,Tet4,Hex8}.hpp) against the reference's own shape
function unit cases (test/cpp/Geom/test_Elements.cpp:488-578): partition of unity at random interior points
(1e-12), nodal interpolation at the standard node coordinates of each element (Kronecker delta, 1e-10), and the
first derivatives against central differences with h = 1e-7 (1e-5), with doctest's Approx comparison."""
import numpy as np
import pytest

import oracle

# standard node coordinates (Geom/Elements/*.hpp standardCoords)
NODES = {
    "line": [(-1, 0, 0), (1, 0, 0)],
    "tri": [(0, 0, 0), (1, 0, 0), (0, 1, 0)],
    "quad": [(-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0)],
    "tet": [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)],
    "hex": [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1), (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)],
}
DIM = dict(line=1, tri=2, quad=2, tet=3, hex=3)


def _approx(a, b, eps):
    return np.all(np.abs(a - b) < eps * (1 + np.maximum(np.abs(a), np.abs(b))))


def _interior(elem, rng):
    d = DIM[elem]
    if elem in ("tri", "tet"):
        while True:
            x = rng.uniform(0.05, 0.9, size=d)
            if x.sum() < 0.95:
                break
    else:
        x = rng.uniform(-0.9, 0.9, size=d)
    return np.concatenate([x, np.zeros(3 - d)])


@pytest.mark.parametrize("elem", list(NODES))
def test_partition_of_unity(elem):
    rng = np.random.default_rng(42)
    for _ in range(10):
        N, _ = oracle.shape(elem, _interior(elem, rng))
        assert _approx(N.sum(), 1.0, 1e-12)


@pytest.mark.parametrize("elem", list(NODES))
def test_nodal_interpolation(elem):
    for j, p in enumerate(NODES[elem]):
        N, _ = oracle.shape(elem, p)
        assert _approx(N, np.eye(len(NODES[elem]))[j], 1e-10), (elem, j, N)


@pytest.mark.parametrize("elem", list(NODES))
def test_first_derivatives_against_central_differences(elem):
    rng = np.random.default_rng(123)
    h = 1e-7
    for _ in range(5):
        p = _interior(elem, rng)
        _, dN = oracle.shape(elem, p)
        for d in range(DIM[elem]):
            e = np.zeros(3)
            e[d] = h
            fd = (oracle.shape(elem, p + e)[0] - oracle.shape(elem, p - e)[0]) / (2 * h)
            assert _approx(dN[d], fd, 1e-5), (elem, d)
