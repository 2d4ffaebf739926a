"""The FP64 list checker of the adjoint (oracle ListsFP64): the full FP64
evaluation against the restatement's AoSoA evaluation of the same lists,
central differences of the partial loss against those of the full loss,
and the direct-sum gradient against differences of the direct sum.  CPU only."""
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
