"""GPU: work-queue retuning (grav_plan_retune_CUDA), the autotuner, and a
merged batch of independent systems against each member alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


def test_retune_keeps_results_and_autotune_picks_a_shape():
    from pgrav import autotune as AT, gravcuda as gc, host, ics
    pos, m = ics.plummer(30000, seed=51)
    t = host.Tree(pos, m, tol=1e-4, p2cut=7, p4cut=20)
    plan = gc.Plan(t, 1e-4)
    plan.eval()
    ref = plan.download()
    for shape in ((4, 64, 64, 32, 0, 0), (8, 32, 32, 32, 1, 0), (8, 1 << 20, 1 << 20, 1 << 20, 2, 0)):
        plan.retune(shape)
        plan.eval()
        got = plan.download()
        assert _rel(got[:, :3], ref[:, :3]).max() < 1e-6
        tu = plan.tuning()
        assert (tu.warps_per_block, tu.chunk_p, tu.blocks_per_sm) == (shape[0], shape[1], shape[4])
    best, trials = AT.autotune(plan, reps=1)
    assert len(trials) >= 6 and best.warps_per_block in (4, 8)
    plan.eval()
    assert _rel(plan.download()[:, :3], ref[:, :3]).max() < 1e-6
    plan.free()


def test_autotune_places_the_ewald_moments_of_a_periodic_plan():
    """For a periodic plan the autotuner also tries the Ewald moments on the
    side stream and on the evaluation's stream; whatever it picks, the
    forces are those of the default shape."""
    from pgrav import autotune as AT, gravcuda as gc, host, ics
    pos, m = ics.grf_box(20, seed=52, rms_disp=0.3)
    t = host.Tree(pos, m, tol=1e-4, box=1.0, p2cut=7, p4cut=20)
    plan = gc.Plan(t, (1.0 / 20 / 50) ** 2, ewald=True)
    plan.eval()
    ref = plan.download()
    best, trials = AT.autotune(plan, reps=1, shapes=((8, 0), (4, 0)), scales=(0.5, 1.0))
    tried = {tr["ewald_side"] for tr in trials}
    assert 0 in tried and any(x < 0 for x in tried) and any(x > 0 for x in tried), tried
    assert best.ewald_side in tried
    plan.eval()
    e = _rel(plan.download()[:, :3], ref[:, :3])
    assert e.max() < 1e-6, e.max()
    plan.free()


def test_merged_batch_equals_members():
    from pgrav import gravcuda as gc, host, ics
    members, outs = [], []
    for k, n in enumerate((3000, 700, 12000, 1500)):
        pos, m = (ics.plummer if k % 2 == 0 else ics.hernquist)(n, seed=60 + k)
        t = host.Tree(pos, m, tol=1e-4, p2cut=7, p4cut=20)
        p = gc.Plan(t, 1e-4)
        p.eval()
        outs.append(p.download())
        p.free()
        members.append(t)
    b = host.Tree.merge(members)
    plan = gc.Plan(b, 1e-4)
    plan.eval()
    got = plan.download()
    plan.free()
    want = np.concatenate(outs)
    assert _rel(got[:, :3], want[:, :3]).max() < 1e-6
    assert np.abs(got[:, 3] - want[:, 3]).max() < 1e-6 * np.abs(want[:, 3]).max()
