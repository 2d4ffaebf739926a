"""GPU parity of the drop-in entry points (grav_mn_CUDA and friends) against
the oracle and the reference kernels' fixtures, through the C ABI."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# routine -> oracle kind with the same semantics
ROUTINES = {
    "pMp": O.MONO_PLUMMER, "pQp": O.QUAD_PLUMMER, "pHp": O.HEXA_PLUMMER, "pMs": O.MONO_MASKED,
    "pM_sK1": O.MONO_K1, "pQ": O.QUAD_COM, "pH": O.HEXA_COM, "pM": O.MONO_BARE,
}
GOLDEN_KIND = {"pMp": 0, "pQp": 1, "pHp": 2, "pMs": 3, "pM_sK1": 4, "pQ": 5, "pH": 6, "pM": 0}
RMS_TOL = 1e-5  # relative rms acceleration, the drop-in parity bar


def rms_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.sqrt(np.mean(np.sum((a - b) ** 2, axis=-1)) / np.mean(np.sum(b * b, axis=-1)))


@pytest.fixture(scope="module")
def gc():
    from pgrav import gravcuda
    return gravcuda


@pytest.mark.parametrize("routine", list(ROUTINES))
def test_grav_mn_matches_oracle(gc, golden, routine):
    kind = ROUTINES[routine]
    gk = GOLDEN_KIND[routine]
    rec = golden[f"k{gk}_records"]
    e = float(golden[f"k{gk}_e"]) if routine != "pM" else 0.0
    sz = O.KIND_SZ[kind]
    f, nblk = O.pack_aosoa(rec)
    rng = np.random.default_rng(7)
    nsink = 300
    sinks = rng.normal(0.0, 0.3, (nsink, 3)).astype(np.float32)
    bt = gc.body_table(sinks, 1.0)
    d = gc.DropIn(bt)
    # two calls on overlapping sink ranges, as mac.c issues per node
    d.mn(routine, 0, 200, f, nblk * 8, sz, e)
    d.mn(routine, 100, 200, f, nblk * 8, sz, e)
    got = d.terminate()
    mult = np.ones(nsink)
    mult[100:200] = 2.0
    want = np.array([O.list_eval(kind, f, nblk, s, e) for s in sinks]) * mult[:, None]
    assert rms_rel(got[:, :3], want[:, :3]) < RMS_TOL
    assert rms_rel(got[:, 3:], want[:, 3:]) < RMS_TOL


@pytest.mark.parametrize("routine", ["pMp", "pQp", "pHp", "pM_sK1", "pQ", "pH", "pMs"])
def test_grav_mn_matches_reference_fixture(gc, golden, routine):
    gk = GOLDEN_KIND[routine]
    rec = golden[f"k{gk}_records"]
    e = float(golden[f"k{gk}_e"])
    f, nblk = O.pack_aosoa(rec)
    sinks = golden[f"k{gk}_sinks"]
    d = gc.DropIn(gc.body_table(sinks, 1.0))
    d.mn(routine, 0, len(sinks), f, nblk * 8, O.KIND_SZ[ROUTINES[routine]], e)
    got = d.terminate()
    ref = golden[f"k{gk}_ref"]
    assert rms_rel(got[:, :3], ref[:, :3]) < RMS_TOL
    assert rms_rel(got[:, 3:], ref[:, 3:]) < RMS_TOL


def test_plummer_tree_lists_match_reference(gc):
    """Config-1 style: Plummer sphere, order-2 lists from the host walk, every
    group's M and Q list through grav_mn_CUDA, against the reference's
    do_gravp/do_gravpq (compiled, when present) or the restatement."""
    from pgrav import host, ics
    pos, m = ics.plummer(8192, seed=5)
    t = host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=7, p4cut=0, tol=1e-3, emit_aosoa=True)
    eps2 = 0.01 ** 2
    bt = gc.body_table(t.sorted_pos, t.points[:t.n, 3])
    d = gc.DropIn(bt)
    for k, (routine, sz) in enumerate((("pMp", 4), ("pQp", 13))):
        ptr, data = t.aosoa[k]
        for g in range(t.ngroups):
            b0, b1 = ptr[g], ptr[g + 1]
            if b1 > b0:
                d.mn(routine, int(t.groups["first"][g]), int(t.groups["count"][g]),
                     data[b0 * sz * 8:b1 * sz * 8], int(b1 - b0) * 8, sz, eps2)
    got = d.terminate()
    use_ref = O.ref_available()
    want = O.tree_eval(t, eps2, quad_kind=O.QUAD_PLUMMER, reference=use_ref)
    assert rms_rel(got[:, :3], want[:, :3]) < RMS_TOL
    assert rms_rel(got[:, 3:], want[:, 3:]) < RMS_TOL


def test_body_runs_k1(gc, golden):
    xyz = golden["mm_xyz"]
    seg = golden["mm_seg"]
    sinks = golden["mm_sinks"]
    # sinks and sources in one table: sources first, then the sinks
    allpos = np.concatenate([xyz, sinks]).astype(np.float32)
    d = gc.DropIn(gc.body_table(allpos, float(golden["mm_mass"])))
    ns = len(sinks)
    d.mnss(len(xyz), ns, np.zeros(ns), [[0, len(seg)]], seg, 0, [int(seg[:, 1].sum())],
           float(golden["mm_mass"]), float(golden["mm_e"]))
    got = d.terminate()[len(xyz):]
    assert rms_rel(got[:, :3], golden["mm_ref"][:, :3]) < RMS_TOL
    assert rms_rel(got[:, 3:], golden["mm_ref"][:, 3:]) < RMS_TOL


def test_error_paths_return_status(gc):
    L = gc.lib()
    bt = gc.body_table(np.zeros((8, 3), np.float32), 1.0)
    d = gc.DropIn(bt)
    f = np.zeros(8 * 4, np.float32)
    with pytest.raises(gc.GravError):
        d.mn("pNope", 0, 8, f, 8, 4, 0.0)
    with pytest.raises(gc.GravError):
        d.mn("pMp", 4, 8, f, 8, 4, 0.0)   # sinks past the table
    with pytest.raises(gc.GravError):
        d.mn("pMp", 0, 8, f, 7, 4, 0.0)   # source_n not a multiple of 8
    d.terminate()
    assert L.gravcuda_status() == 0
