"""The Ewald restatement (oracle/grav_oracle.c orc_ewald, after nln/ewald.c)
and the FP64 correction table (csrc/host/ewald_table.cpp), on the CPU."""
import ctypes
import itertools

import numpy as np
import pytest

from oracle import oracle as O

# The potential at a lattice site of a simple cubic lattice of unit masses
# in a neutralising background, self term removed: lim_{r->0} (phi + 1/r)
# = 2.8372974794806 / L  (the Ewald constant of the simple cubic lattice,
# e.g. Nijboer & De Wette, Physica 23 (1957) 309).
SC_CONSTANT = 2.837297479480620


@pytest.fixture(scope="module")
def host():
    from pgrav import host as H
    L = H.lib()
    L.nln_ewald_eval.argtypes = [ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    L.nln_ewald_table.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_void_p]
    L.nln_ewald_table.restype = ctypes.c_int
    return L


NQ = 56   # C, 3 first, 6 second, 10 third, 15 fourth, 21 fifth derivatives
IDX3 = [(0, 0, 0), (0, 0, 1), (0, 0, 2), (0, 1, 1), (0, 1, 2), (0, 2, 2), (1, 1, 1),
        (1, 1, 2), (1, 2, 2), (2, 2, 2)]
IDX4 = list(itertools.combinations_with_replacement(range(3), 4))
IDX5 = list(itertools.combinations_with_replacement(range(3), 5))


def full(vals, idx, rank):
    T = np.zeros((3,) * rank)
    for v, ijk in zip(vals, idx):
        for p in set(itertools.permutations(ijk)):
            T[p] = v
    return T


def ev(host, y, L=1.0):
    o = np.zeros(NQ)
    y = np.ascontiguousarray(y, np.float64)
    host.nln_ewald_eval(L, y.ctypes.data, o.ctypes.data)
    return o


def test_restatement_periodic_and_odd():
    rng = np.random.default_rng(0)
    x = rng.uniform(-0.5, 0.5, (20, 3))
    f, p = O.ewald(x, 1.0)
    for k in range(3):
        xs = x.copy()
        xs[:, k] += 1.0
        f2, p2 = O.ewald(xs, 1.0)
        assert np.abs(f2 - f).max() < 1e-9 and np.abs(p2 - p).max() < 1e-9
    fm, pm = O.ewald(-x, 1.0)
    assert np.abs(fm + f).max() < 1e-12 and np.abs(pm - p).max() < 1e-12


def test_restatement_x0_rule():
    f, p = O.ewald(np.zeros(3), 1.0)
    assert np.all(f == 0) and p[0] == pytest.approx(np.pi / 4)  # pi/(alpha^2 L^3), alpha = 2/L


def test_restatement_lattice_constant():
    # phi(x) + 1/|x| -> SC constant as x -> 0 (the quadratic term is -(2 pi/3) x^2)
    x = np.array([[1e-3, 0.0, 0.0]])
    f, p = O.ewald(x, 1.0)
    assert p[0] + 1e3 + 2 * np.pi / 3 * 1e-6 == pytest.approx(SC_CONSTANT, abs=1e-8)


def test_force_is_gradient_of_potential():
    y = np.array([[0.17, -0.22, 0.31]])
    h = 1e-6
    f, _ = O.ewald(y, 1.0)
    for k in range(3):
        e = np.zeros((1, 3))
        e[0, k] = h
        _, pp = O.ewald(y + e, 1.0)
        _, pm = O.ewald(y - e, 1.0)
        assert (pp[0] - pm[0]) / (2 * h) == pytest.approx(f[0, k], rel=1e-7)


def test_table_matches_restatement(host):
    rng = np.random.default_rng(1)
    for L in (1.0, 3.0):
        for y in rng.uniform(-0.6 * L, 0.6 * L, (40, 3)):
            o = ev(host, y, L)
            f, p = O.ewald(y, L)
            r = np.linalg.norm(y)
            assert o[0] == pytest.approx(p[0] + 1.0 / r, rel=1e-9, abs=1e-10 / L)
            assert np.abs(o[1:4] - (f[0] - y / r ** 3)).max() < 1e-10 / L ** 2


def test_table_constant_and_laplacian(host):
    o = ev(host, np.zeros(3))
    assert o[0] == pytest.approx(SC_CONSTANT, abs=1e-12)
    assert np.abs(o[1:4]).max() < 1e-14
    y = np.array([0.3, 0.1, -0.2])
    o = ev(host, y, 2.0)
    assert o[4] + o[7] + o[9] == pytest.approx(-4 * np.pi / 8.0, rel=1e-10)  # -4 pi / L^3


def test_table_derivatives_by_differences(host):
    y = np.array([0.21, -0.13, 0.33])
    h = 1e-5
    o = ev(host, y)
    H = np.array([[o[4], o[5], o[6]], [o[5], o[7], o[8]], [o[6], o[8], o[9]]])
    T = full(o[10:20], IDX3, 3)
    X = full(o[20:35], IDX4, 4)
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        op, om = ev(host, y + e), ev(host, y - e)
        assert np.abs((op[1:4] - om[1:4]) / (2 * h) - H[:, k]).max() < 1e-7
        Hp = np.array([[op[4], op[5], op[6]], [op[5], op[7], op[8]], [op[6], op[8], op[9]]])
        Hm = np.array([[om[4], om[5], om[6]], [om[5], om[7], om[8]], [om[6], om[8], om[9]]])
        assert np.abs((Hp - Hm) / (2 * h) - T[:, :, k]).max() < 1e-5
        Tp, Tm = full(op[10:20], IDX3, 3), full(om[10:20], IDX3, 3)
        assert np.abs((Tp - Tm) / (2 * h) - X[:, :, :, k]).max() < 1e-4 * np.abs(X).max()


def test_high_derivatives_by_differences_and_traceless(host):
    # both branches of the n = 0 term (series for alpha r < 1, closed form
    # beyond), and Laplace: the traces of the third to fifth derivatives
    # vanish because the Laplacian of C is the constant -4 pi / L^3
    for y in (np.array([0.01, -0.02, 0.005]), np.array([0.4, 0.35, -0.3]),
              np.array([0.55, -0.1, 0.6])):
        o = ev(host, y)
        T, X, F = full(o[10:20], IDX3, 3), full(o[20:35], IDX4, 4), full(o[35:56], IDX5, 5)
        assert np.abs(np.einsum('iik->k', T)).max() < 1e-9 * np.abs(T).max()
        assert np.abs(np.einsum('iikl->kl', X)).max() < 1e-9 * np.abs(X).max()
        assert np.abs(np.einsum('iiklm->klm', F)).max() < 1e-9 * np.abs(F).max()
        h = 1e-5
        for k in range(3):
            e = np.zeros(3)
            e[k] = h
            op, om = ev(host, y + e), ev(host, y - e)
            Tp, Tm = full(op[10:20], IDX3, 3), full(om[10:20], IDX3, 3)
            assert np.abs((Tp - Tm) / (2 * h) - X[..., k]).max() < 1e-4 * np.abs(X).max()
            Xp, Xm = full(op[20:35], IDX4, 4), full(om[20:35], IDX4, 4)
            assert np.abs((Xp - Xm) / (2 * h) - F[..., k]).max() < 1e-4 * np.abs(F).max()


def test_table_grid(host):
    n, L, reach = 5, 2.0, 0.625
    tab = np.zeros(n ** 3 * NQ)
    assert host.nln_ewald_table(L, n, reach, tab.ctypes.data) == 0
    tab = tab.reshape(n, n, n, NQ)
    h = reach * L / (n - 1)
    assert np.allclose(tab[1, 2, 3], ev(host, np.array([1, 2, 3]) * h, L), rtol=1e-13, atol=1e-13)


def test_direct_ewald_oracle_softening_limit():
    """With eps2 -> 0 the softened periodic oracle tends to the plain EwaldForces sum."""
    rng = np.random.default_rng(2)
    pos = rng.uniform(0, 1, (40, 3))
    m = rng.uniform(0.5, 1.5, 40) / 40
    a0, p0 = O.direct_ewald(pos, m, 1.0, 0.0, np.arange(5))
    a1, _ = O.direct_ewald(pos, m, 1.0, 1e-14, np.arange(5))
    assert np.abs(a1 - a0).max() < 1e-6 * np.abs(a0).max()
    # momentum: sum_i m_i a_i over all sinks vanishes
    a, _ = O.direct_ewald(pos, m, 1.0, 0.0, np.arange(40))
    assert np.abs((m[:, None] * a).sum(0)).max() < 1e-10


def test_restatement_matches_reference_golden(golden):
    """orc_ewald against the committed outputs of the reference's ewald()
    (tests/golden/make_golden.py; runs without the reference tree)."""
    for tag, L in (("1", 1.0), ("3", 3.0)):
        f, p = O.ewald(golden[f"ewald{tag}_x"], L)
        f0, p0 = golden[f"ewald{tag}_f"], golden[f"ewald{tag}_phi"]
        assert np.abs(f - f0).max() <= 1e-12 * np.abs(f0).max()
        assert np.abs(p - p0).max() <= 1e-12 * np.abs(p0).max()


# ---- pinned to the reference's own ewald() (nln/ewald.c:13-64, compiled
# unmodified into oracle/_ref by oracle/Makefile with stand-in 2hot headers)
needs_ref = pytest.mark.skipif(not O.ref_available(),
                               reason="oracle/_ref (the reference's compiled CPU code) is not built")


def _displacements(L, n=12000, seed=11):
    rng = np.random.default_rng(seed)
    x = np.concatenate([
        rng.uniform(-0.5 * L, 0.5 * L, (n - 2000, 3)),     # minimum-image cube
        rng.uniform(-2.0 * L, 2.0 * L, (1000, 3)),          # other images
        rng.normal(0.0, 1e-4 * L, (500, 3)),                # near the lattice site
        np.eye(3)[rng.integers(0, 3, 500)] * rng.uniform(-L, L, (500, 1))])  # on the axes
    x[0] = 0.0                                              # the x == 0 rule
    return x


@needs_ref
@pytest.mark.parametrize("L", [1.0, 3.0])
def test_restatement_matches_reference_ewald(L):
    """orc_ewald against the reference's ewald() at 12,000 displacements:
    relative agreement 1e-12 (the two evaluate the same sums in the same
    order, so they agree exactly)."""
    x = _displacements(L)
    f0, p0 = O.ref_ewald(x, L)
    f1, p1 = O.ewald(x, L)
    assert np.all(np.isfinite(f0)) and np.all(np.isfinite(p0))
    assert np.abs(f1 - f0).max() <= 1e-12 * np.abs(f0).max()
    assert np.abs(p1 - p0).max() <= 1e-12 * np.abs(p0).max()
    assert np.array_equal(f1, f0) and np.array_equal(p1, p0)


@needs_ref
@pytest.mark.parametrize("L", [1.0, 3.0])
def test_table_values_match_reference_ewald(host, L):
    """The FP64 table's C = phi + 1/r and gradient (csrc/host/ewald_table.cpp,
    analytic derivatives of the same Ewald sum) against the reference's
    ewald() at 10,000 displacements in the table's reach cube: C within
    1e-12 / L, gradient within 1e-11 / L^2 (the force itself is up to
    ~800 / L^2 there)."""
    rng = np.random.default_rng(3)
    y = rng.uniform(-0.625 * L, 0.625 * L, (10000, 3))
    f, p = O.ref_ewald(y, L)
    r = np.linalg.norm(y, axis=1)
    o = np.array([ev(host, yy, L)[:4] for yy in y])
    assert np.abs(o[:, 0] - (p + 1.0 / r)).max() < 1e-12 / L
    assert np.abs(o[:, 1:4] - (f - y / r[:, None] ** 3)).max() < 1e-11 / L ** 2


@needs_ref
def test_table_interpolation_bound_against_reference(host):
    """The device lookup (csrc/ewald.cuh ew_lookup: fourth-order Taylor
    expansion about the nearest node of the 32^3 table over [0, 0.625 L]^3),
    emulated here in FP64, against the reference's ewald() at 4,000 random
    displacements: C within 1e-7 / L and its gradient within 3e-5 / L^2
    (largest gradient 7 / L^2).  In FP32 on the device C's rounding adds
    about 1e-6 / L."""
    import math
    n, L, reach = 32, 1.0, 0.625
    tab = np.zeros(n ** 3 * NQ)
    assert host.nln_ewald_table(L, n, reach, tab.ctypes.data) == 0
    tab = tab.reshape(n, n, n, NQ)
    h = reach * L / (n - 1)

    def idx(a):  # multi-index offset of include/nlnlists.h
        s = sum(a)
        return s * (s + 1) * (s + 2) // 6 + (a[1] + a[2]) * (a[1] + a[2] + 1) // 2 + a[2]

    rng = np.random.default_rng(5)
    y = rng.uniform(-reach * L, reach * L, (4000, 3))
    sg = np.where(y < 0, -1.0, 1.0)
    a = np.abs(y)
    ijk = np.minimum(np.rint(a / h).astype(int), n - 1)
    d = a - ijk * h
    V = tab[ijk[:, 0], ijk[:, 1], ijk[:, 2]]
    terms = [b for b in itertools.product(range(5), repeat=3) if sum(b) <= 4]
    out = np.zeros((len(y), 4))
    for col, al in enumerate([(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)]):
        acc = np.zeros(len(y))
        for b in terms:
            if sum(al) + sum(b) <= 4:
                w = np.prod([d[:, k] ** b[k] / math.factorial(b[k]) for k in range(3)], axis=0)
                acc += V[:, idx(tuple(al[k] + b[k] for k in range(3)))] * w
        out[:, col] = acc * np.prod([sg[:, k] ** al[k] for k in range(3)], axis=0)
    f, p = O.ref_ewald(y, L)
    r = np.linalg.norm(y, axis=1)
    assert np.abs(out[:, 0] - (p + 1.0 / r)).max() < 1e-7 / L
    assert np.abs(out[:, 1:4] - (f - y / r[:, None] ** 3)).max() < 3e-5 / L ** 2


@needs_ref
def test_reference_periodic_scheme_matches_ewald_sum():
    """The reference's own periodic scheme -- every body in the 125 images of
    the box (SetGravOffset, nln/mac.c:91-111) plus FixCubeEwaldLE's order-8
    local expansion of the rest (nln/main.c:1811-1859, the compiled
    nln/ewald_le2.c) -- against the Ewald-summed direct sum (the oracle of
    nln/grav_n2.c) on a 16^3 clustered box: the same forces within the
    expansion's truncation, potentials up to one constant (the two schemes'
    conventions for the mean and the self images)."""
    from pgrav import ics
    pos, m = ics.grf_box(16, seed=7)
    eps2 = (1 / 16 / 50) ** 2
    pc = (pos.astype(np.float64) - 0.5).astype(np.float32)   # the reference centres its box
    samp = np.arange(0, len(m), 16)
    acc, phi = O.ref_periodic_le(pc, m, 1.0, eps2, samp)
    a2, p2 = O.direct_ewald(pc.astype(np.float64), m.astype(np.float64), 1.0, eps2, samp)
    e = np.linalg.norm(acc - a2, axis=1) / np.sqrt(np.mean((a2 ** 2).sum(1)))
    assert np.sqrt(np.mean(e ** 2)) < 3e-5 and e.max() < 1e-4, (np.sqrt(np.mean(e ** 2)), e.max())
    d = phi - p2
    assert d.std() < 1e-6 * np.sqrt(np.mean(p2 ** 2)), d.std()
