"""GPU: the device time step (csrc/step.cuh) -- refit of the cell tables
against the host refit (nln_tree_refit), the integrator against
nln/integrate.c's formulas, graph replay against eager launches, and energy
conservation over KDK steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    import torch
    from pgrav import gravcuda, host, ics, step
    return torch, gravcuda, host, ics, step


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


def test_refit_in_place_keeps_forces(mods):
    torch, gc, host, ics, _ = mods
    pos, m = ics.plummer(20000, seed=21)
    t = host.Tree(pos, m, tol=1e-4, p2cut=7, p4cut=20)
    plan = gc.Plan(t, 1e-4)
    plan.set_tree(t)
    plan.eval()
    f0 = plan.download()
    plan.refit()
    plan.eval()
    f1 = plan.download()
    plan.free()
    # R differs (a parent's bmax is a bound) but kernels see R^l q_l
    assert _rel(f1[:, :3], f0[:, :3]).max() < 2e-6
    assert np.abs(f1[:, 3] - f0[:, 3]).max() < 2e-6 * np.abs(f0[:, 3]).max()


@pytest.mark.parametrize("box", [0.0, 1.0])
def test_device_refit_matches_host_refit(mods, box):
    torch, gc, host, ics, step = mods
    if box:
        pos, m = ics.grf_box(24, seed=22, rms_disp=0.3)
        eps2 = (1.0 / 24 / 50) ** 2
    else:
        pos, m = ics.plummer(20000, seed=22)
        eps2 = 1e-4
    t = host.Tree(pos, m, tol=1e-4, p2cut=7, p4cut=20, box=box)
    plan = gc.Plan(t, eps2, ewald=box > 0)
    plan.set_tree(t)
    # move every body a little, on the device and in the host tree
    rng = np.random.default_rng(3)
    moved = t.sorted_pos + rng.normal(0, 1e-3, t.sorted_pos.shape).astype(np.float32)
    body = np.concatenate([moved, t.points[:t.n, 3:4]], 1).astype(np.float32)
    step.memcpy_h2d(plan.bodies_ptr(), body)
    plan.refit()
    plan.eval()
    got = plan.download()
    plan.free()
    t.refit(moved)
    ref_plan = gc.Plan(t, eps2, ewald=box > 0)
    ref_plan.eval()
    ref = ref_plan.download()
    ref_plan.free()
    e = _rel(got[:, :3], ref[:, :3])
    assert np.sqrt(np.mean(e * e)) < 1e-6 and e.max() < 2e-5, (np.sqrt(np.mean(e * e)), e.max())
    assert np.abs(got[:, 3] - ref[:, 3]).max() < 1e-5 * np.abs(ref[:, 3]).max()


def test_integrate_matches_formula(mods):
    torch, gc, host, ics, step = mods
    pos, m = ics.plummer(5000, seed=23)
    t = host.Tree(pos, m, tol=1e-4)
    plan = gc.Plan(t, 1e-4)
    plan.set_tree(t)
    plan.eval()
    f = plan.download()
    rng = np.random.default_rng(4)
    v = rng.normal(0, 0.3, (t.n, 4)).astype(np.float32)
    v[:, 3] = 0
    dvel = torch.from_numpy(v.copy()).cuda()
    dt, dtv, dtsync = 1e-3, 1e-3, 5e-4
    params = torch.tensor([dt, dtv, dtsync], dtype=torch.float64, device="cuda")
    energy = torch.zeros(2, dtype=torch.float64, device="cuda")
    plan.integrate(dvel.data_ptr(), params.data_ptr(), energy.data_ptr())
    torch.cuda.synchronize()
    body = step.memcpy_d2h(np.empty((t.n, 4), np.float32), plan.bodies_ptr())
    plan.free()
    x0 = t.points[:t.n, :3].astype(np.float64)
    mm = t.points[:t.n, 3].astype(np.float64)
    a = f[:, :3].astype(np.float64)
    vc = v[:, :3] + dtsync * a
    v1 = (v[:, :3] + dtv * a).astype(np.float32)
    x1 = (x0 + dt * v1.astype(np.float64)).astype(np.float32)
    # FP64 arithmetic rounded to FP32 (a fused multiply-add may round once less)
    np.testing.assert_allclose(dvel.cpu().numpy()[:, :3], v1, rtol=2e-7, atol=1e-9)
    np.testing.assert_allclose(body[:, :3], x1, rtol=2e-7, atol=1e-9)
    ke, pe = energy.cpu().numpy()
    assert ke == pytest.approx(float((mm[:, None] * vc * vc).sum()), rel=1e-10)
    assert pe == pytest.approx(float((mm * f[:, 3]).sum()), rel=1e-9)


def test_graph_replay_equals_eager(mods):
    torch, gc, host, ics, step = mods
    pos, m = ics.plummer(8000, seed=24)
    vel = np.zeros_like(pos)
    runs = []
    for graph in (False, True):
        s = step.Stepper(pos, vel, m, 1e-4, rebuild=100, graph=graph, tree_kw=dict(tol=1e-4))
        s.run(3, 1e-3)
        p, v = s.state()
        runs.append((p, v, [h["e"] for h in s.history]))
        s.free()
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
    # energies are FP64 atomic sums: equal up to summation order
    np.testing.assert_allclose(runs[0][2], runs[1][2], rtol=1e-12)


def test_kdk_energy_conservation_plummer(mods):
    torch, gc, host, ics, step = mods
    n = 16384
    pos, m = ics.plummer(n, seed=25)
    # isotropic velocities at half the local circular speed: a bound, moving system
    r = np.linalg.norm(pos, axis=1)
    vc = np.sqrt(r * r / (1 + r * r) ** 1.5)
    rng = np.random.default_rng(5)
    d = rng.normal(size=pos.shape)
    vel = (0.5 * vc / np.linalg.norm(d, axis=1))[:, None] * d
    s = step.Stepper(pos, vel, m, 0.01 ** 2, rebuild=10, graph=True,
                     tree_kw=dict(tol=1e-5, p2cut=7, p4cut=20))
    s.run(40, 2e-3)
    e = np.array([h["e"] for h in s.history])
    s.free()
    assert np.all(np.isfinite(e))
    assert np.abs(e - e[0]).max() < 2e-4 * abs(e[0]), (e[0], np.abs(e - e[0]).max())


def test_kdk_periodic_box_runs_and_wraps(mods):
    torch, gc, host, ics, step = mods
    n1 = 16
    pos, m = ics.grf_box(n1, seed=26, rms_disp=0.3)
    rng = np.random.default_rng(6)
    vel = rng.normal(0, 0.05, pos.shape)
    s = step.Stepper(pos, vel, m, (1.0 / n1 / 50) ** 2, box=1.0, rebuild=3, graph=True,
                     tree_kw=dict(tol=1e-5, p2cut=7, p4cut=20))
    s.run(7, 1e-2)
    p, v = s.state()
    e = np.array([h["e"] for h in s.history])
    s.free()
    assert np.all(np.isfinite(e)) and np.all(np.isfinite(p))
    # rebuilds wrapped every body back into the box; since the last rebuild
    # bodies moved by at most a few v dt
    assert p.min() > -0.05 and p.max() < 1.05


def test_checkpoint_and_resume_continue_the_run(tmp_path):
    """8 KDK steps straight through against 4 steps, an SDF checkpoint
    (Stepper.save) at that rebuild boundary, a resumed stepper
    (Stepper.load, which builds its tree from the saved bodies as the
    straight run rebuilds from the same bodies) and 4 more steps: the same
    positions and velocities bit for bit."""
    from pgrav import ics, step as S
    pos, m = ics.plummer(3000, seed=21)
    vel = np.random.default_rng(2).normal(0, 0.1, pos.shape).astype(np.float32)
    kw = dict(leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
    a = S.Stepper(pos, vel, m, 1e-4, rebuild=4, graph=True, tree_kw=kw)
    a.run(8, 1e-3)
    want = a.state()
    a.free()
    b = S.Stepper(pos, vel, m, 1e-4, rebuild=4, graph=True, tree_kw=kw)
    b.run(4, 1e-3)
    path = tmp_path / "ck.sdf"
    b.save(path)
    b.free()
    c = S.Stepper.load(path, graph=True, tree_kw=kw)
    assert c.nsteps == 4
    c.run(4, 1e-3)
    got = c.state()
    c.free()
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


def test_cosmo_integrate_matches_reference_restatement(mods):
    """CosmoIntegrate on the device (grav_plan_set_integrator_CUDA kind 1)
    against the oracle's restatement of nln/integrate.c:82-135 on the same
    bodies, forces and factors: positions and velocities bit for bit."""
    torch, gc, host, ics, step = mods
    from oracle import oracle as O
    from pgrav.cosmo import Cosmology
    pos, m = ics.plummer(6000, seed=25)
    t = host.Tree(pos, m, tol=1e-4)
    plan = gc.Plan(t, 1e-4)
    plan.eval()
    f = plan.download()
    x0 = step.memcpy_d2h(np.empty((t.n, 4), np.float32), plan.bodies_ptr())
    rng = np.random.default_rng(6)
    v = rng.normal(0, 0.3, (t.n, 4)).astype(np.float32)
    v[:, 3] = 0
    c = Cosmology(H0=0.0511365, Omega_m=0.3, Omega_lambda=0.7)
    tpos, dt = c.t_at_a(0.25), 0.05 * c.t_at_a(0.25)
    tvel = tpos - 0.5 * dt
    fac = c.kdk(tpos, tvel, dt, tpos + 0.5 * dt - tvel)
    dvel = torch.from_numpy(v.copy()).cuda()
    params = torch.tensor(fac, dtype=torch.float64, device="cuda")
    energy = torch.zeros(2, dtype=torch.float64, device="cuda")
    plan.set_integrator(1)
    plan.integrate(dvel.data_ptr(), params.data_ptr(), energy.data_ptr())
    torch.cuda.synchronize()
    x1 = step.memcpy_d2h(np.empty((t.n, 4), np.float32), plan.bodies_ptr())
    plan.free()
    rx, rv, ke, pe = O.cosmo_integrate(x0, v, f.astype(np.float32), fac)
    np.testing.assert_array_equal(x1[:, :3], rx[:, :3])
    np.testing.assert_array_equal(dvel.cpu().numpy()[:, :3], rv[:, :3])
    got = energy.cpu().numpy()
    assert got[0] == pytest.approx(ke, rel=1e-12) and got[1] == pytest.approx(pe, rel=1e-12)


def test_zeldovich_plane_wave_grows_linearly(mods):
    """A comoving run (Stepper with a Cosmology) of an Einstein-de Sitter box:
    sheets displaced by a plane wave follow the Zel'dovich solution, exact in
    one dimension before shell crossing -- the displacement grows as a from
    a = 0.1 to 0.2 (periodic forces with the Ewald correction, kicks and
    drifts of the cosmological leapfrog).  16 sheets of 48 x 48 bodies: the
    in-sheet spacing stays well below the closest sheets' separation, where
    a sheet's field is uniform to 1e-5."""
    torch, gc, host, ics, step = mods
    from pgrav.cosmo import Cosmology
    ns, nt = 16, 48
    gs, gt = (np.arange(ns) + 0.5) / ns, (np.arange(nt) + 0.5) / nt
    q = np.stack(np.meshgrid(gs, gt, gt, indexing="ij"), -1).reshape(-1, 3)
    n = len(q)
    m = np.full(n, 1.0 / n)
    c = Cosmology(H0=np.sqrt(8 * np.pi / 3), Omega_m=1.0)   # G rho_bar = 1 in a unit box
    a0, a1 = 0.1, 0.2
    A = 0.4 / (2 * np.pi * a1)                               # k A a1 = 0.4: no shell crossing
    psi = np.zeros_like(q)
    psi[:, 0] = A * np.sin(2 * np.pi * q[:, 0])
    x = np.mod(q + a0 * psi, 1.0)
    u = a0 * a0 * c.hubble(a0) * psi                         # a dx/dt of the growing mode
    t0, t1 = c.t_at_a(a0), c.t_at_a(a1)
    st = step.Stepper(x, u, m, (0.05 / nt) ** 2, box=1.0, rebuild=4, graph=True,
                      tree_kw=dict(tol=1e-6, p2cut=7, p4cut=20), cosmo=c, tstart=t0)
    nst = 40
    st.run(nst, (t1 - t0) / nst)
    assert st.tpos == pytest.approx(t1, rel=1e-12)
    xe, ue = st.state()
    st.free()
    d = np.mod(xe - q + 0.5, 1.0) - 0.5
    s = np.sin(2 * np.pi * q[:, 0])
    amp = 2 * np.mean(d[:, 0] * s)
    assert amp == pytest.approx(a1 * A, rel=1e-3), (amp, a1 * A)
    assert np.abs(d[:, 0] - a1 * A * s).max() < 2e-3 * a1 * A
    assert np.abs(d[:, 1:]).max() < 1e-3 * a1 * A
    # peculiar velocities at tvel (half a step behind) follow a^2 H psi
    at = c.a_at_t(st.tvel)
    want = at * at * c.hubble(at) * psi[:, 0]
    assert np.abs(ue[:, 0] - want).max() < 2e-3 * np.abs(want).max()


def test_cosmological_checkpoint_and_resume(tmp_path):
    """A comoving run checkpointed at a rebuild boundary (Stepper.save keeps
    the cosmology and the step times in the SDF header) and resumed
    (Stepper.load) continues the straight run: the peculiar velocities are
    stored as a dx/dt, so the canonical momenta come back to FP32 rounding."""
    from pgrav import ics, step as S
    from pgrav.cosmo import Cosmology
    pos, m = ics.grf_box(16, seed=22)
    c = Cosmology(H0=np.sqrt(8 * np.pi / 3), Omega_m=0.3, Omega_lambda=0.7)
    t0 = c.t_at_a(0.2)
    dt = 0.02 * t0
    vel = np.random.default_rng(3).normal(0, 0.01, pos.shape).astype(np.float32)
    kw = dict(leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-5)
    mk = lambda: S.Stepper(pos, vel, m, (1 / 16 / 50) ** 2, box=1.0, rebuild=4, graph=True,
                           tree_kw=kw, cosmo=c, tstart=t0)
    a = mk()
    a.run(8, dt)
    want = a.state()
    a.free()
    b = mk()
    b.run(4, dt)
    path = tmp_path / "cosmo.sdf"
    b.save(path)
    b.free()
    r = S.Stepper.load(path, graph=True, tree_kw=kw)
    assert r.cosmo is not None and r.nsteps == 4
    assert r.cosmo.params.Omega_lambda == pytest.approx(0.7)
    r.run(4, dt)
    got = r.state()
    r.free()
    dx = np.abs(np.mod(got[0] - want[0] + 0.5, 1.0) - 0.5)
    assert dx.max() < 1e-6, dx.max()
    assert np.abs(got[1] - want[1]).max() < 1e-5 * np.abs(want[1]).max()
