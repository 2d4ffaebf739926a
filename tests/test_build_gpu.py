"""GPU: the tree, moments, critical radii, sink groups and lists built on the
device (grav_plan_build_CUDA) against the host builder (nln_tree_build +
nln_tree_walk, the product's own host walk) on the same bodies: every table
and list bit for bit, and the forces of the two plans bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(kind, seed=3):
    from pgrav import ics
    if kind == "plummer":
        return ics.plummer(20000, seed=seed) + (0.0,)
    if kind == "hernquist":
        return ics.hernquist(12000, seed=seed) + (0.0,)
    if kind == "box":
        return ics.grf_box(24, seed=seed, rms_disp=0.5) + (1.0,)
    if kind == "clumps":
        # coincident and near-coincident bodies: leaves that cannot split
        rng = np.random.default_rng(seed)
        pos = np.concatenate([rng.normal(0, 1, (5000, 3)), np.zeros((300, 3)),
                              np.full((200, 3), 0.25) + rng.normal(0, 1e-7, (200, 3))])
        return pos.astype(np.float32), np.full(len(pos), 1.0 / len(pos), np.float32), 0.0
    raise ValueError(kind)


PARAMS = [
    ("plummer", dict(leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)),
    ("plummer", dict(leaf_max=8, group_max=16, p2cut=7, p4cut=0, tol=1e-3, rel_tol=1e-3)),
    ("hernquist", dict(leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-5, ptol_boost=2.0)),
    ("box", dict(leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-5)),
    ("clumps", dict(leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4, rel_tol0=1e-4)),
]


@pytest.mark.parametrize("kind,kw", PARAMS, ids=[f"{k}-{i}" for i, (k, _) in enumerate(PARAMS)])
def test_device_build_equals_host_build(kind, kw):
    from pgrav import gravcuda as gc, host
    pos, m, box = _case(kind)
    eps2 = 1e-4
    t = host.Tree(pos, m, box=box, **kw)
    ewald = box > 0
    gp = gc.Plan.build(pos, m, eps2, box=box, ewald=ewald, **kw)
    assert np.array_equal(gp.order(), t.order)
    pr = gp.problem()
    assert pr["ncells"] == t.ncells
    assert np.array_equal(pr["points"].view(np.uint32), t.points.view(np.uint32))
    assert np.array_equal(pr["groups"].view(np.uint8), t.groups.view(np.uint8))
    for k, name in enumerate(("P", "Q", "H", "correction")):
        if k == 3 and not ewald:
            continue
        assert np.array_equal(pr["ptr"][k], t.ptr[k]), name
        host_list = (t.plist, t.qlist, t.hlist, t.clist)[k]
        assert np.array_equal(pr["lists"][k], host_list), name
    if pr["hcells"] is not None:
        assert np.array_equal(pr["hcells"].view(np.uint8), t.hcells.view(np.uint8))
    if pr["qcells"] is not None:
        assert np.array_equal(pr["qcells"].view(np.uint8), t.qcells.view(np.uint8))
    assert np.array_equal(gp.counts(), t.counts)
    # the same tables evaluate to the same forces
    hp = gc.Plan(t, eps2, ewald=ewald)
    hp.eval()
    gp.eval()
    a, b = hp.download(), gp.download()
    hp.free()
    gp.free()
    assert np.array_equal(a, b)


def test_device_build_refuses_bad_bodies():
    from pgrav import gravcuda as gc
    pos = np.random.default_rng(0).uniform(0, 1, (1000, 3)).astype(np.float32)
    m = np.full(1000, 1e-3, np.float32)
    pos[7, 1] = 1.5   # outside the periodic box
    with pytest.raises(gc.GravError, match="outside"):
        gc.Plan.build(pos, m, 1e-4, box=1.0)
    pos[7, 1] = np.nan
    with pytest.raises(gc.GravError, match="non-finite"):
        gc.Plan.build(pos, m, 1e-4)


def test_build_eval_returns_input_order():
    """grav_build_eval_CUDA (positions in, forces out, one call) equals the
    host-built plan's evaluation, reordered to the input order, bit for bit;
    twice in a row (the pool's reused memory carries nothing over)."""
    from pgrav import gravcuda as gc, host, ics
    pos, m = ics.grf_box(20, seed=4, rms_disp=0.5)
    eps2 = (1 / 20 / 50) ** 2
    kw = dict(leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-5)
    t = host.Tree(pos, m, box=1.0, **kw)
    plan = gc.Plan(t, eps2, ewald=True)
    plan.eval()
    want = plan.download()
    plan.free()
    b = np.concatenate([pos, m[:, None]], 1).astype(np.float32)
    for _ in range(2):
        got = gc.build_eval(b, eps2, box=1.0, ewald=True, **kw)
        assert np.array_equal(got[t.order], want)
    gc.lib().grav_groups_release_CUDA()


def test_stepper_gpu_rebuilds_match_host_rebuilds():
    """KDK steps with the tree rebuilt on the GPU every 2 steps give the same
    trajectory as with the host rebuilds (the builders agree bit for bit)."""
    from pgrav import ics, step as S
    pos, m = ics.plummer(4000, seed=6)
    vel = np.random.default_rng(1).normal(0, 0.1, pos.shape).astype(np.float32)
    kw = dict(leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
    runs = []
    for gpu in (True, False):
        st = S.Stepper(pos, vel, m, 1e-4, rebuild=2, graph=False, tree_kw=kw, gpu_build=gpu)
        st.run(5, 1e-3)
        runs.append(st.state())
        st.free()
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
