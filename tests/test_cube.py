"""The field of a uniform cube (nlnhost.h nln_cubic_acc), the near-zone term
of background subtraction, against the reference's compiled cubic_acc
(nln/ewald_le2.c:773-1033), an FP64 quadrature and Gauss's law.  CPU only."""
import numpy as np
import pytest

from oracle import oracle as O


def _acc(r, a):
    from pgrav import host
    return host.cubic_acc(r, a)


def _points(rng, a, n):
    """Sinks inside, on the faces' planes and edges' lines, and outside."""
    pts = [(0.0, 0.0, 0.0), (a, 0.0, 0.0), (a, a, 0.0), (a, a, a), (-a, 0.3 * a, -a),
           (0.5 * a, 0.0, 0.0), (2 * a, 0.0, 0.0), (0.0, -3 * a, 0.0)]
    pts += list(rng.uniform(-1.2 * a, 1.2 * a, (n, 3)))
    pts += list(rng.uniform(-6 * a, 6 * a, (n, 3)))
    return np.array(pts)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_matches_reference_cubic_acc():
    rng = np.random.default_rng(3)
    a = 0.35
    compared = 0
    for r in _points(rng, a, 60):
        got = _acc(r, a)
        assert np.all(np.isfinite(got))
        want = O.ref_cubic_acc(r, a).astype(np.float64)
        if not np.all(np.isfinite(want)):
            # the reference's expression is 0/0 on the cube's face planes
            # and edge lines (it is NaN at (a, 0, 0)); the limit exists
            assert np.any(np.isclose(np.abs(r), a))
            continue
        # the reference evaluates a long float expression: float rounding
        scale = max(np.abs(want).max(), 1e-2 * a)
        assert np.abs(got - want).max() <= 2e-4 * scale, (r, got, want)
        compared += 1
    assert compared >= 120


def test_matches_fp64_quadrature_outside():
    """Gauss-Legendre product rule over the cube for sinks outside it."""
    a = 0.5
    x, w = np.polynomial.legendre.leggauss(48)
    x, w = a * x, a * w
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    W = w[:, None, None] * w[None, :, None] * w[None, None, :]
    rng = np.random.default_rng(5)
    for _ in range(12):
        d = rng.normal(size=3)
        r = d / np.linalg.norm(d) * rng.uniform(2.2, 5.0) * a
        ux, uy, uz = X - r[0], Y - r[1], Z - r[2]
        q = W / (ux * ux + uy * uy + uz * uz) ** 1.5
        want = np.array([(q * ux).sum(), (q * uy).sum(), (q * uz).sum()])
        assert np.abs(_acc(r, a) - want).max() <= 1e-9 * np.abs(want).max()


def test_symmetry_far_field_and_gauss_law():
    a = 0.25
    assert np.abs(_acc((0, 0, 0), a)).max() < 1e-14
    rng = np.random.default_rng(7)
    for r in rng.uniform(-0.6, 0.6, (20, 3)):
        assert np.allclose(_acc(-r, a), -_acc(r, a), rtol=1e-12, atol=1e-14)
        p = np.roll(r, 1)                         # cubic symmetry: axes permute
        assert np.allclose(_acc(p, a), np.roll(_acc(r, a), 1), rtol=1e-12, atol=1e-14)
    # far away: the monopole of mass (2a)^3
    r = np.array([40.0, -25.0, 13.0]) * a
    mono = -(2 * a) ** 3 * r / np.linalg.norm(r) ** 3
    assert np.allclose(_acc(r, a), mono, rtol=1e-5)
    # div acc = -4 pi rho inside the cube, 0 outside (central differences)
    h = 1e-4 * a

    def div(r):
        s = 0.0
        for k in range(3):
            e = np.zeros(3)
            e[k] = h
            s += (_acc(r + e, a)[k] - _acc(r - e, a)[k]) / (2 * h)
        return s
    for r in (np.array([0.1, -0.2, 0.3]) * a, np.array([0.9, 0.5, -0.7]) * a):
        assert div(r) == pytest.approx(-4 * np.pi, rel=1e-6)
    for r in (np.array([1.5, 0.2, 0.1]) * a, np.array([-2.0, 3.0, 0.5]) * a):
        assert abs(div(r)) < 1e-6
