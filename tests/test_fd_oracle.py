"""The FP64 list checker of the adjoint (oracle ListsFP64): the full FP64
evaluation against the restatement's AoSoA evaluation of the same lists
(point, quadrupole and order-4 cells) and, for periodic trees with the
correction list, against the Ewald-summed direct sum; central differences
of the partial loss against those of the full loss; and the direct-sum
gradient against differences of the direct sum.  CPU only."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.fixture(scope="module")
def small():
    from pgrav import host, ics
    pos, m = ics.plummer(3000, seed=41)
    t = host.Tree(pos, m, leaf_max=8, group_max=32, p2cut=7, p4cut=0, tol=1e-3, emit_aosoa=True)
    return t


def test_full_eval_matches_aosoa_restatement(small):
    t = small
    eps2 = 1e-4
    chk = O.ListsFP64(t)
    got = chk.eval(t.sorted_pos, t.points[:t.n, 3], eps2)
    want = O.tree_eval(t, eps2)   # FP32 moments from the host, same lists
    e = np.linalg.norm(got[:, :3] - want[:, :3], axis=1) / np.linalg.norm(want[:, :3], axis=1)
    assert np.sqrt(np.mean(e ** 2)) < 1e-5
    assert np.abs(got[:, 3] - want[:, 3]).max() < 1e-5 * np.abs(want[:, 3]).max()


def test_partial_differences_equal_full_differences(small):
    t = small
    eps2 = 1e-4
    rng = np.random.default_rng(3)
    x = t.sorted_pos.astype(np.float64)
    m = t.points[:t.n, 3].astype(np.float64)
    w = rng.normal(size=(t.n, 3))
    u = rng.normal(size=t.n)
    chk = O.ListsFP64(t)
    sel = rng.choice(t.n, 5, replace=False)
    chk.select(sel)
    h = 1e-6

    def full(xx, mm):
        o = chk.eval(xx, mm, eps2)
        return float((w * o[:, :3]).sum() + (u * o[:, 3]).sum())

    coords = [(s, c) for s in range(5) for c in (0, 1, 2, 3)]
    part = chk.fd_grad(x, m, w, u, eps2, coords, h=h, mass_rel=True)
    for (s, c), p in zip(coords, part):
        j = sel[s]
        xp, xm, mp, mq = x.copy(), x.copy(), m.copy(), m.copy()
        if c < 3:
            xp[j, c] += h
            xm[j, c] -= h
            f = (full(xp, m) - full(xm, m)) / (2 * h)
        else:
            mp[j] += h * m[j]
            mq[j] -= h * m[j]
            f = (full(x, mp) - full(x, mq)) / (2 * h * m[j])
        assert abs(p - f) <= 1e-6 * max(1.0, abs(f)), (s, c, p, f)


@pytest.fixture(scope="module")
def small_hexa():
    from pgrav import host, ics
    pos, m = ics.plummer(3000, seed=42)
    return host.Tree(pos, m, leaf_max=8, group_max=32, p2cut=7, p4cut=20, tol=1e-3,
                     emit_aosoa=True)


def test_order4_eval_matches_aosoa_restatement(small_hexa):
    """Order-4 lists: the exact STF terms in FP64 against the restatement of
    do_gravph_avx8 on the host's FP32 tables (the same expansion)."""
    t = small_hexa
    assert len(t.hlist) > 0
    eps2 = 1e-4
    got = O.ListsFP64(t).eval(t.sorted_pos, t.points[:t.n, 3], eps2)
    want = O.tree_eval(t, eps2)
    e = np.linalg.norm(got[:, :3] - want[:, :3], axis=1) / np.linalg.norm(want[:, :3], axis=1)
    assert np.sqrt(np.mean(e ** 2)) < 1e-5, np.sqrt(np.mean(e ** 2))
    assert np.abs(got[:, 3] - want[:, 3]).max() < 1e-5 * np.abs(want[:, 3]).max()


@pytest.fixture(scope="module")
def small_box():
    from pgrav import host, ics
    pos, m = ics.grf_box(8, seed=5)
    return host.Tree(pos, m, leaf_max=8, group_max=32, p2cut=7, p4cut=20, tol=1e-6, box=1.0)


def test_periodic_eval_matches_ewald_direct_sum(small_box):
    """A periodic 8^3 box: shifts, order-4 cells and the correction list in
    FP64 against the Ewald-summed direct sum (softened nearest images)."""
    t = small_box
    assert len(t.clist) > 0
    eps2 = (1.0 / 8 / 50) ** 2
    x = t.sorted_pos.astype(np.float64)
    m = t.points[:t.n, 3].astype(np.float64)
    got = O.ListsFP64(t).eval(x, m, eps2)
    samp = np.arange(0, t.n, 4)
    acc, phi = O.direct_ewald(x, m, 1.0, eps2, samp)
    e = np.linalg.norm(got[samp, :3] - acc, axis=1)
    assert np.sqrt(np.mean(e ** 2) / np.mean((acc ** 2).sum(1))) < 1e-4
    assert np.sqrt(np.mean((got[samp, 3] - phi) ** 2) / np.mean(phi ** 2)) < 1e-5
    # without the correction list the same lists miss the periodic images
    bare = O.ListsFP64(t, ewald=False).eval(x, m, eps2)
    e0 = np.linalg.norm(bare[samp, :3] - acc, axis=1)
    assert np.sqrt(np.mean(e0 ** 2) / np.mean((acc ** 2).sum(1))) > 1e-2


def test_ewald_c0_is_the_limit():
    """C(0) against C(y) = Phi(y) + 1/|y| at small |y| (C is smooth and even)."""
    c0 = O.ewald_c0(1.0)
    for r in (1e-3, 2e-3):
        y = np.array([r, 0.0, 0.0])
        _, phi = O.ewald(y[None], 1.0)
        assert abs(float(phi[0]) + 1.0 / r - c0) < 5.0 * r * r, (r, float(phi[0]) + 1 / r, c0)


def _partial_vs_full(t, ewald, nsel, seed):
    eps2 = 1e-4
    rng = np.random.default_rng(seed)
    x = t.sorted_pos.astype(np.float64)
    m = t.points[:t.n, 3].astype(np.float64)
    w = rng.normal(size=(t.n, 3))
    u = rng.normal(size=t.n)
    chk = O.ListsFP64(t, ewald=ewald)
    sel = rng.choice(t.n, nsel, replace=False)
    chk.select(sel)
    h = 1e-6

    def full(xx, mm):
        o = chk.eval(xx, mm, eps2)
        return float((w * o[:, :3]).sum() + (u * o[:, 3]).sum())

    coords = [(s, c) for s in range(nsel) for c in (0, 1, 2, 3)]
    part = chk.fd_grad(x, m, w, u, eps2, coords, h=h, mass_rel=True)
    for (s, c), p in zip(coords, part):
        j = sel[s]
        xp, xm, mp, mq = x.copy(), x.copy(), m.copy(), m.copy()
        if c < 3:
            xp[j, c] += h
            xm[j, c] -= h
            f = (full(xp, m) - full(xm, m)) / (2 * h)
        else:
            mp[j] += h * m[j]
            mq[j] -= h * m[j]
            f = (full(x, mp) - full(x, mq)) / (2 * h * m[j])
        assert abs(p - f) <= 1e-6 * max(1.0, abs(f)), (s, c, p, f)


def test_partial_differences_periodic_order4():
    """Hit lists and partial loss with order-4 cells and image shifts: central
    differences of the partial loss equal those of the full loss."""
    from pgrav import host, ics
    pos, m0 = ics.grf_box(12, seed=6)
    t = host.Tree(pos, m0, leaf_max=4, group_max=16, p2cut=4, p4cut=8, tol=1e-3, box=1.0)
    assert len(t.hlist) > 0 and np.any((np.asarray(t.hlist) >> 27) != 13)
    _partial_vs_full(t, False, 4, 5)


def test_partial_differences_correction_list():
    """The same with the periodic correction list (a 6^3 box)."""
    from pgrav import host, ics
    pos, m0 = ics.grf_box(6, seed=6)
    t = host.Tree(pos, m0, leaf_max=4, group_max=16, p2cut=4, p4cut=8, tol=1e-3, box=1.0)
    assert len(t.clist) > 0
    _partial_vs_full(t, True, 3, 6)


def test_direct_grad_by_differences():
    rng = np.random.default_rng(4)
    n, eps2 = 300, 1e-3
    x = rng.normal(size=(n, 3))
    m = rng.uniform(0.5, 1.5, n) / n
    w = rng.normal(size=(n, 3))
    u = rng.normal(size=n)
    gx, gm = O.direct_grad(x, m, w, u, eps2)

    def L(xx, mm):
        d = xx[:, None, :] - xx[None]
        r2 = (d * d).sum(-1) + eps2     # the self pair: d = 0, phi_i gets -m_i / eps
        ri = 1 / np.sqrt(r2)
        a = -(mm[None, :, None] * d * (ri ** 3)[..., None]).sum(1)
        phi = -(mm[None] * ri).sum(1)
        return (w * a).sum() + (u * phi).sum()

    h = 1e-6
    for j, c in ((3, 0), (17, 2), (200, 1)):
        xp, xm = x.copy(), x.copy()
        xp[j, c] += h
        xm[j, c] -= h
        assert (L(xp, m) - L(xm, m)) / (2 * h) == pytest.approx(gx[j, c], rel=1e-6, abs=1e-9)
    mp, mq = m.copy(), m.copy()
    mp[5] += h
    mq[5] -= h
    assert (L(x, mp) - L(x, mq)) / (2 * h) == pytest.approx(gm[5], rel=1e-6, abs=1e-9)
