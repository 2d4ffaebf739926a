"""GPU: the FP64 direct-sum reference against the CPU oracle, and the
batched periodic evaluation (tree + Ewald correction) against both."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gc():
    from pgrav import gravcuda
    return gravcuda


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    e = np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
    return np.sqrt(np.mean(e ** 2))


def test_direct_fp64_isolated_matches_oracle(gc):
    from pgrav import ics
    pos, m = ics.plummer(3000, seed=4)
    pts = np.concatenate([pos, m[:, None]], 1)
    sinks = np.arange(0, 3000, 37)
    got = gc.direct_fp64(pts, sinks, 1e-4)
    acc, phi = O.direct(pos, m, 1e-4, sinks)
    assert np.abs(got[:, :3] - acc).max() <= 1e-12 * np.abs(acc).max()
    assert np.abs(got[:, 3] - phi).max() <= 1e-12 * np.abs(phi).max()


@pytest.mark.parametrize("eps2", [0.0, (1 / 8 / 50) ** 2])
def test_direct_fp64_ewald_matches_oracle(gc, eps2):
    from pgrav import ics
    pos, m = ics.grf_box(8, seed=5)   # 512 bodies
    pts = np.concatenate([pos, m[:, None]], 1)
    sinks = np.arange(0, 512, 23)
    got = gc.direct_fp64(pts, sinks, eps2, box=1.0)
    acc, phi = O.direct_ewald(pos, m, 1.0, eps2, sinks)
    assert rel_rms(got[:, :3], acc) < 1e-6
    assert np.abs(got[:, 3] - phi).max() < 1e-6 * np.abs(phi).max()


def test_direct_fp64_ewald_many_sinks_match_oracle(gc):
    """The GPU FP64 Ewald direct sum (k_direct64: FP64 table, fifth-order
    Taylor) against the CPU oracle's per-pair ewald() (restated from
    nln/ewald.c and pinned to it) on 64 sinks of a 16^3 clustered box."""
    from pgrav import ics
    pos, m = ics.grf_box(16, seed=9, rms_disp=0.5)
    eps2 = (1.0 / 16 / 50) ** 2
    pts = np.concatenate([pos, m[:, None]], 1)
    sinks = np.random.default_rng(2).choice(len(pos), 64, replace=False)
    got = gc.direct_fp64(pts, sinks, eps2, box=1.0)
    acc, phi = O.direct_ewald(pos, m, 1.0, eps2, sinks)
    assert rel_rms(got[:, :3], acc) < 1e-7
    assert np.abs(got[:, 3] - phi).max() < 1e-7 * np.abs(phi).max()


def test_batched_ewald_accuracy(gc):
    """Periodic 64^3 clustered box (GRF, P(k) ~ k^-2.5, rms displacement 0.25
    spacing), order 4 + Ewald, MAC tolerance 2e-6: rms relative force error
    <= 1e-4 against the FP64 Ewald direct sum on 512 sinks (the accuracy bar
    of the periodic configurations)."""
    from pgrav import host, ics
    n1 = 64
    pos, m = ics.grf_box(n1, seed=7)
    eps2 = (1.0 / n1 / 50) ** 2
    t = host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=2e-6, box=1.0)
    plan = gc.Plan(t, eps2, ewald=True)
    plan.eval()
    got = plan.download()
    samp = np.random.default_rng(1).choice(t.n, 512, replace=False)
    ref = gc.direct_fp64(t.points[:t.n], samp, eps2, box=1.0)
    err = rel_rms(got[samp, :3], ref[:, :3])
    assert err <= 1e-4, err
    # the correction matters: without it the error is far larger
    plan0 = gc.Plan(t, eps2, ewald=False)
    plan0.eval()
    assert rel_rms(plan0.download()[samp, :3], ref[:, :3]) > 100 * err
    plan.free()
    plan0.free()
    perr = np.sqrt(np.mean((got[samp, 3] - ref[:, 3]) ** 2) / np.mean(ref[:, 3] ** 2))
    assert perr < 1e-4, perr


def test_batched_ewald_small_box_large_groups(gc):
    """32^3 box: groups are large against the box (radius ~0.05 L), where the
    group Taylor expansion of the correction bounds the error near 1e-3."""
    from pgrav import host, ics
    n1 = 32
    pos, m = ics.grf_box(n1, seed=7)
    eps2 = (1.0 / n1 / 50) ** 2
    t = host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-5, box=1.0)
    plan = gc.Plan(t, eps2, ewald=True)
    plan.eval()
    got = plan.download()
    plan.free()
    samp = np.random.default_rng(1).choice(t.n, 256, replace=False)
    ref = gc.direct_fp64(t.points[:t.n], samp, eps2, box=1.0)
    assert rel_rms(got[samp, :3], ref[:, :3]) < 2e-3


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["x"]).ref_available(),
                    reason="oracle/_ref (the reference's compiled CPU code) is not built")
def test_batched_matches_reference_periodic_scheme(gc):
    """The periodic evaluation (each source in the image nearest the group,
    the rest of the lattice from the Ewald table) against the reference's own
    periodic scheme on the same bodies: every body in the 125 images of the
    box plus FixCubeEwaldLE's order-8 local expansion (nln/mac.c:91-111,
    nln/main.c:1811-1859, the compiled nln/ewald_le2.c).  64^3 clustered box,
    order 4, MAC 2e-6: forces within the 1e-4 bar, potentials up to one
    constant (the schemes' conventions for the mean and the self images)."""
    from oracle import oracle as O
    from pgrav import host, ics
    n1 = 64
    pos, m = ics.grf_box(n1, seed=9)
    eps2 = (1.0 / n1 / 50) ** 2
    t = host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=2e-6, box=1.0)
    plan = gc.Plan(t, eps2, ewald=True)
    plan.eval()
    got = plan.download()
    plan.free()
    samp = np.sort(np.random.default_rng(2).choice(t.n, 256, replace=False))
    xt = (t.points[:t.n, :3].astype(np.float64) - 0.5).astype(np.float32)  # centred, as there
    acc, phi = O.ref_periodic_le(xt, t.points[:t.n, 3], 1.0, eps2, samp)
    assert rel_rms(got[samp, :3], acc) <= 1e-4, rel_rms(got[samp, :3], acc)
    d = got[samp, 3] - phi
    assert d.std() < 1e-4 * np.sqrt(np.mean(phi ** 2)), d.std()
