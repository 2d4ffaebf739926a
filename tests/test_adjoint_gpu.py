"""GPU: the hand-written adjoint (csrc/adjoint.cuh) against FP64 central
differences of an FP64 evaluation of the same interaction lists (point,
quadrupole and order-4 cells; periodic boxes with image shifts and the
Ewald correction), against the analytic FP64 direct-sum gradient, and
through checkpointed leapfrog steps (pgrav/autograd.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def fp64_lists_loss(t, pos_tree, mass_tree, eps2, w, u):
    """L = sum w.a + u phi of the tree's lists, every cell's moments taken in
    FP64 from the bodies (the kernels' formulas: Plummer monopole, the
    physical quadrupole potential 1/2 rho^-5 d.Q.d with Q = -3 (S2 - tr/3))."""
    x = np.asarray(pos_tree, np.float64)
    m = np.asarray(mass_tree, np.float64)
    n = len(x)
    first, count = t.cell_ranges()
    cm = np.concatenate([[0.0], np.cumsum(m)])
    cmx = np.concatenate([np.zeros((1, 3)), np.cumsum(m[:, None] * x, 0)])
    cmxx = np.concatenate([np.zeros((1, 3, 3)), np.cumsum(m[:, None, None] * x[:, :, None] * x[:, None, :], 0)])
    M = cm[first + count] - cm[first]
    X = (cmx[first + count] - cmx[first]) / M[:, None]
    S2 = (cmxx[first + count] - cmxx[first]) - M[:, None, None] * X[:, :, None] * X[:, None, :]
    Q = -3.0 * (S2 - np.trace(S2, axis1=1, axis2=2)[:, None, None] / 3.0 * np.eye(3))
    L = 0.0
    for g in range(t.ngroups):
        G = t.groups[g]
        s = x[G["first"]:G["first"] + G["count"]]
        ws, us = w[G["first"]:G["first"] + G["count"]], u[G["first"]:G["first"] + G["count"]]
        idx = (t.plist[t.ptr[0][g]:t.ptr[0][g + 1]] & ((1 << 27) - 1)).astype(np.int64)
        body = idx < n
        src = np.where(body[:, None], x[np.minimum(idx, n - 1)], X[np.maximum(idx - n, 0)])
        ms = np.where(body, m[np.minimum(idx, n - 1)], M[np.maximum(idx - n, 0)])
        d = s[:, None, :] - src[None]
        rho2 = (d * d).sum(-1) + eps2
        ri = 1.0 / np.sqrt(rho2)
        a = -(ms[None, :, None] * d * (ri ** 3)[..., None]).sum(1)
        phi = -(ms[None] * ri).sum(1)
        qi = t.qlist[t.ptr[1][g]:t.ptr[1][g + 1]].astype(np.int64) & ((1 << 27) - 1)
        if len(qi):
            d = s[:, None, :] - X[qi][None]
            rho2 = (d * d).sum(-1) + eps2
            ri = 1.0 / np.sqrt(rho2)
            a -= (M[qi][None, :, None] * d * (ri ** 3)[..., None]).sum(1)
            phi -= (M[qi][None] * ri).sum(1)
            Qd = np.einsum('kab,ikb->ika', Q[qi], d)
            P2 = (d * Qd).sum(-1)
            phi += (0.5 * ri ** 5 * P2).sum(1)
            a += (2.5 * (ri ** 7 * P2)[..., None] * d - (ri ** 5)[..., None] * Qd).sum(1)
        L += float((ws * a).sum() + (us * phi).sum())
    return L


def test_adjoint_matches_central_differences(monkeypatch):
    import torch
    from pgrav import autograd as AG, host, ics
    n, eps2 = 2000, 1e-4
    pos, m = ics.plummer(n, seed=31)
    rng = np.random.default_rng(7)
    w = rng.normal(size=(n, 3))
    u = rng.normal(size=n)
    tkw = dict(tol=1e-3, p2cut=7, p4cut=0, leaf_max=8)
    p = torch.tensor(pos, dtype=torch.float32, device="cuda", requires_grad=True)
    mm = torch.tensor(m, dtype=torch.float32, device="cuda", requires_grad=True)
    a, phi = AG.gravity(p, mm, eps2, **tkw)
    L = (torch.tensor(w, dtype=torch.float32, device="cuda") * a).sum() + \
        (torch.tensor(u, dtype=torch.float32, device="cuda") * phi).sum()
    L.backward()
    gx = p.grad.cpu().numpy().astype(np.float64)
    gm = mm.grad.cpu().numpy().astype(np.float64)
    # FP64 central differences of the same lists
    t = host.Tree(pos, m, **tkw)
    o = t.order
    xt = pos[o].astype(np.float64)
    mt = m[o].astype(np.float64)
    wt, ut = w[o], u[o]
    inv = np.empty(n, np.int64)
    inv[o] = np.arange(n)
    h = 1e-6
    picks = rng.choice(n * 3, 48, replace=False)
    fd = []
    for k in picks:
        b, c = divmod(int(k), 3)
        xp = xt.copy()
        xp[inv[b], c] += h
        xm = xt.copy()
        xm[inv[b], c] -= h
        fd.append((fp64_lists_loss(t, xp, mt, eps2, wt, ut) - fp64_lists_loss(t, xm, mt, eps2, wt, ut)) / (2 * h))
    fd = np.array(fd)
    ad = gx.ravel()[picks]
    scale = np.sqrt(np.mean(gx ** 2))
    assert np.abs(ad - fd).max() < 2e-4 * scale, (np.abs(ad - fd).max() / scale)
    mpicks = rng.choice(n, 16, replace=False)
    fdm = []
    for b in mpicks:
        mp = mt.copy()
        mp[inv[b]] += h * mt[inv[b]]
        mq = mt.copy()
        mq[inv[b]] -= h * mt[inv[b]]
        fdm.append((fp64_lists_loss(t, xt, mp, eps2, wt, ut) - fp64_lists_loss(t, xt, mq, eps2, wt, ut)) / (2 * h * mt[inv[b]]))
    fdm = np.array(fdm)
    mscale = np.sqrt(np.mean(gm ** 2))
    assert np.abs(gm[mpicks] - fdm).max() < 2e-4 * mscale, (np.abs(gm[mpicks] - fdm).max() / mscale)


def _adjoint_vs_oracle_fd(pos, m, eps2, tkw, nsel, seed, ewald=False, pool=None):
    """The GPU adjoint (through pgrav.autograd) at nsel bodies against FP64
    central differences of the oracle's evaluation of the same lists
    (ListsFP64, every cell's moments from the bodies).  Returns the largest
    position and mass errors, each over the rms of that gradient, and the
    FD values themselves.  pool: tree positions to draw the bodies from."""
    import torch
    from oracle import oracle as O
    from pgrav import autograd as AG, host
    n = len(pos)
    rng = np.random.default_rng(seed)
    w = rng.normal(size=(n, 3))
    u = rng.normal(size=n)
    kw = dict(tkw)
    if ewald:
        kw["ewald"] = True
    p = torch.tensor(pos, dtype=torch.float32, device="cuda", requires_grad=True)
    mm = torch.tensor(m, dtype=torch.float32, device="cuda", requires_grad=True)
    a, phi = AG.gravity(p, mm, eps2, **kw)
    L = (torch.tensor(w, dtype=torch.float32, device="cuda") * a).sum() + \
        (torch.tensor(u, dtype=torch.float32, device="cuda") * phi).sum()
    L.backward()
    gx = p.grad.cpu().numpy().astype(np.float64)
    gm = mm.grad.cpu().numpy().astype(np.float64)
    t = host.Tree(pos, m, **tkw)
    o = np.asarray(t.order)
    chk = O.ListsFP64(t, ewald=ewald)
    sel = rng.choice(n if pool is None else pool, nsel, replace=False)     # tree positions
    chk.select(sel)
    xt = np.asarray(t.sorted_pos, np.float64)
    mt = np.asarray(t.points[:n, 3], np.float64)
    coords = [(s, c) for s in range(nsel) for c in (0, 1, 2, 3)]
    fd = chk.fd_grad(xt, mt, w[o], u[o], eps2, coords, h=1e-6, mass_rel=True).reshape(nsel, 4)
    ad = np.concatenate([gx[o[sel]], gm[o[sel]][:, None]], 1)
    scale = np.array([np.sqrt(np.mean(gx ** 2))] * 3 + [np.sqrt(np.mean(gm ** 2))])
    ex = np.abs(ad[:, :3] - fd[:, :3]).max() / scale[0]
    em = np.abs(ad[:, 3] - fd[:, 3]).max() / scale[3]
    return ex, em, dict(fd=fd, ad=ad, scale=scale, tree=t, sel=sel, w=w[o], u=u[o], x=xt, m=mt,
                        coords=coords)


def test_adjoint_order4_matches_central_differences():
    """Order-4 cells (p4cut = 20): the trace-free moment duals, their chain
    through the centre of mass, and the pair terms of orders 2..4."""
    from pgrav import host, ics
    pos, m = ics.plummer(4000, seed=34)
    tkw = dict(tol=1e-3, p2cut=4, p4cut=8, leaf_max=8)
    t = host.Tree(pos, m, **tkw)
    # bodies of cells on order-4 lists, whose moments' chain the check covers
    hc = np.unique(np.asarray(t.hlist) & ((1 << 27) - 1))
    first, count = t.cell_ranges()
    pool = np.unique(np.concatenate([np.arange(first[c], first[c] + count[c]) for c in hc]))
    assert len(hc) > 50 and len(pool) > 500
    ex, em, _ = _adjoint_vs_oracle_fd(pos, m, 1e-4, tkw, 16, 35, pool=pool)
    assert ex < 2e-4 and em < 2e-4, (ex, em)


def test_adjoint_periodic_matches_central_differences():
    """A periodic 16^3 box with order-4 cells, image shifts and the Ewald
    correction.  The oracle sums the correction exactly over each entry's
    bodies; the kernels use cell moments and each group's Taylor series of
    it, so the bar is that truncation (the correction itself moves the
    gradient by far more)."""
    from pgrav import ics
    n1 = 16
    pos, m = ics.grf_box(n1, seed=36)
    eps2 = (1.0 / n1 / 50) ** 2
    tkw = dict(tol=1e-4, p2cut=4, p4cut=8, leaf_max=8, group_max=16, box=1.0)
    # without the correction the same periodic lists (image shifts, order-4
    # cells) match the oracle's differences to FP32 accuracy
    ex0, em0, _ = _adjoint_vs_oracle_fd(pos, m, eps2, tkw, 8, 37, ewald=False)
    assert ex0 < 2e-5 and em0 < 2e-5, (ex0, em0)
    ex, em, r = _adjoint_vs_oracle_fd(pos, m, eps2, tkw, 8, 37, ewald=True)
    assert ex < 3e-3 and em < 3e-3, (ex, em)
    # the correction's share of the gradient is far above that bar
    from oracle import oracle as O
    chk0 = O.ListsFP64(r["tree"], ewald=False)
    chk0.select(r["sel"])
    fd0 = chk0.fd_grad(r["x"], r["m"], r["w"], r["u"], eps2, r["coords"], h=1e-6,
                       mass_rel=True).reshape(-1, 4)
    share = np.abs(r["fd"] - fd0).max(0) / r["scale"]
    assert share[:3].max() > 10 * ex and share[3] > 10 * em, (share, ex, em)


def direct_grad(x, m, eps2, w, u, block=512):
    n = len(x)
    gx = np.zeros((n, 3))
    gm = np.zeros(n)
    for i0 in range(0, n, block):
        xi, wi, ui = x[i0:i0 + block], w[i0:i0 + block], u[i0:i0 + block]
        d = xi[:, None, :] - x[None]
        rho2 = (d * d).sum(-1) + eps2
        ri = 1.0 / np.sqrt(rho2)
        ri3 = ri ** 3
        wd = (wi[:, None, :] * d).sum(-1)
        t = m[None, :, None] * (ri3[..., None] * wi[:, None, :] - (3 * ri ** 5 * wd)[..., None] * d
                                - (ui[:, None] * ri3)[..., None] * d)
        gx[i0:i0 + block] -= t.sum(1)
        gx += t.sum(0)
        gm += -(ri3 * wd + ui[:, None] * ri).sum(0)
    return gx, gm


def test_adjoint_against_direct_sum_gradient():
    import torch
    from pgrav import autograd as AG, ics
    n, eps2 = 8192, 1e-4
    pos, m = ics.plummer(n, seed=32)
    rng = np.random.default_rng(8)
    w = rng.normal(size=(n, 3)).astype(np.float32)
    u = rng.normal(size=n).astype(np.float32)
    p = torch.tensor(pos, dtype=torch.float32, device="cuda", requires_grad=True)
    mm = torch.tensor(m, dtype=torch.float32, device="cuda", requires_grad=True)
    a, phi = AG.gravity(p, mm, eps2, tol=1e-6, p2cut=7, p4cut=0)
    ((torch.tensor(w, device="cuda") * a).sum() + (torch.tensor(u, device="cuda") * phi).sum()).backward()
    gx, gm = direct_grad(pos.astype(np.float64), m.astype(np.float64), eps2, w.astype(np.float64), u.astype(np.float64))
    ex = np.linalg.norm(p.grad.cpu().numpy() - gx, axis=1) / np.sqrt(np.mean((gx ** 2).sum(1)))
    em = np.abs(mm.grad.cpu().numpy() - gm) / np.sqrt(np.mean(gm ** 2))
    assert np.sqrt(np.mean(ex ** 2)) < 1e-3 and np.sqrt(np.mean(em ** 2)) < 1e-3, (np.sqrt(np.mean(ex ** 2)), np.sqrt(np.mean(em ** 2)))


def test_leapfrog_checkpointing_gives_the_same_gradient():
    import torch
    from pgrav import autograd as AG, ics
    n, eps2 = 4096, 1e-3
    pos, m = ics.plummer(n, seed=33)
    rng = np.random.default_rng(9)
    vel = rng.normal(0, 0.2, (n, 3)).astype(np.float32)
    target = torch.tensor(rng.normal(size=(n, 3)), dtype=torch.float32, device="cuda")
    grads = []
    for ck in (0, 4):
        x0 = torch.tensor(pos, dtype=torch.float32, device="cuda", requires_grad=True)
        v0 = torch.tensor(vel, device="cuda", requires_grad=True)
        mm = torch.tensor(m, dtype=torch.float32, device="cuda", requires_grad=True)
        x, v = AG.leapfrog(x0, v0, mm, eps2, 1e-3, 8, checkpoint_every=ck, tol=1e-4, p2cut=7)
        ((x * target).sum() + (v * target).sum()).backward()
        grads.append((x0.grad.cpu().numpy(), v0.grad.cpu().numpy(), mm.grad.cpu().numpy()))
    for a, b in zip(grads[0], grads[1]):
        np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6 * np.abs(a).max())
