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


def _qsz_records(golden):
    rec = golden[f"k{O.QUAD_DIPOLE}_records"]    # m x y z R qx qy qz qxx qxy qyy qxz qyz
    assert np.abs(rec[:, 5:8]).max() > 0           # the dipole fields are exercised
    return rec


def test_grav_qnss_matches_reference_fixture(gc, golden):
    """grav_qnss_CUDA ("pQ1_qnss", live at nln/mac.c:467; reference kernel
    nln/pgrav.cu:293-368) on the committed outputs of do_gravdq_avx8, the
    same arithmetic: every sink against the whole buffer."""
    rec = _qsz_records(golden)
    f, nblk = O.pack_aosoa(rec)
    sinks = golden[f"k{O.QUAD_DIPOLE}_sinks"]
    d = gc.DropIn(gc.body_table(sinks, 1.0))
    seg = np.tile(np.array([[0, nblk * 8]], np.uint32), (len(sinks), 1))
    d.qnss(0, len(sinks), seg, f, nblk * 8)
    got = d.terminate()
    ref = golden[f"k{O.QUAD_DIPOLE}_ref"]
    assert rms_rel(got[:, :3], ref[:, :3]) < RMS_TOL
    assert rms_rel(got[:, 3:], ref[:, 3:]) < RMS_TOL


def test_grav_qnss_runs_match_oracle(gc, golden):
    """Per-sink runs as nln/mac.c:395-425 queues them (each sink its own run
    of 8-record blocks of one shared buffer, empty runs included), at a
    nonzero sink base, against the oracle's do_gravdq restatement and, when
    built, the compiled reference on the same runs."""
    rng = np.random.default_rng(3)
    rec = _qsz_records(golden)
    f, nblk = O.pack_aosoa(rec)
    nsink, base = 40, 7
    sinks = rng.normal(0.0, 0.3, (base + nsink, 3)).astype(np.float32)
    b0 = rng.integers(0, nblk, nsink)
    nb = np.minimum(rng.integers(0, 8, nsink), nblk - b0)
    nb[3] = 0
    seg = np.stack([b0 * 8, nb * 8], 1).astype(np.uint32)
    d = gc.DropIn(gc.body_table(sinks, 1.0))
    d.qnss(base, nsink, seg, f, nblk * 8)
    got = d.terminate()[base:]
    for i in range(nsink):
        sub = O.aligned_f32(int(nb[i]) * 8 * 13)
        sub[:] = f[b0[i] * 8 * 13:(b0[i] + nb[i]) * 8 * 13]
        want = O.list_eval(O.QUAD_DIPOLE, sub, int(nb[i]), sinks[base + i], 0.0)
        if nb[i] == 0:
            assert np.all(got[i] == 0)
            continue
        assert np.linalg.norm(got[i, :3] - want[:3]) <= 1e-5 * np.linalg.norm(want[:3])
        assert abs(got[i, 3] - want[3]) <= 1e-5 * abs(want[3])
        if O.ref_available():
            r = O.ref_list_eval(O.QUAD_DIPOLE, sub, int(nb[i]), sinks[base + i], 0.0)
            assert np.linalg.norm(got[i, :3] - r[:3]) <= 2e-5 * np.linalg.norm(r[:3])


def test_grav_qns_matches_oracle(gc, golden):
    """grav_qns_CUDA ("pQQ1", nln/pgrav.cu:1149-1200) on a hexacell table
    registered by WalkInitSrcCUDA (nln/physics.h:140-157 with DIPOLE: 40
    floats per cell, mass 0, pos 1..3, bmax 5, dipole 12..14, quadrupole
    15..19) and index lists with repeats, against do_gravdq's restatement on
    the same cells packed as a QSZ list."""
    rng = np.random.default_rng(5)
    rec = _qsz_records(golden)
    nc = len(rec)
    qtab = np.zeros((nc, 40), np.float32)
    qtab[:, 0] = rec[:, 0]
    qtab[:, 1:4] = rec[:, 1:4]
    qtab[:, 4] = 9.0      # rcrit_m: not read
    qtab[:, 5] = rec[:, 4]
    qtab[:, 12:15] = rec[:, 5:8]
    qtab[:, 15:20] = rec[:, 8:13]
    qtab[:, 20:] = 7.0    # higher moments and bookkeeping: not read
    nsink = 50
    sinks = rng.normal(0.0, 0.3, (nsink, 3)).astype(np.float32)
    d = gc.DropIn(gc.body_table(sinks, 1.0))
    d.init_src(qtab)
    lists = [rng.integers(0, nc, int(k)) for k in (100, 37, 1)]
    spans = [(0, 20), (20, 25), (45, 5)]
    for (b, m), sl in zip(spans, lists):
        d.qns(b, m, sl)
    got = d.terminate()
    d.terminate_src()
    for (b, m), sl in zip(spans, lists):
        f, nblk = O.pack_aosoa(rec[sl])
        for i in range(b, b + m):
            want = O.list_eval(O.QUAD_DIPOLE, f, nblk, sinks[i], 0.0)
            assert np.linalg.norm(got[i, :3] - want[:3]) <= 1e-5 * np.linalg.norm(want[:3])
            assert abs(got[i, 3] - want[3]) <= 1e-5 * abs(want[3])


def test_grav_qns_rejects_bad_indices(gc, golden):
    rec = _qsz_records(golden)
    qtab = np.zeros((len(rec), 40), np.float32)
    qtab[:, 0] = rec[:, 0]
    qtab[:, 1:4] = rec[:, 1:4]
    qtab[:, 5] = rec[:, 4]
    d = gc.DropIn(gc.body_table(np.zeros((4, 3), np.float32), 1.0))
    d.init_src(qtab)
    d.qns(0, 4, np.array([0, len(rec) + 5], np.int32))   # one entry past the table
    with pytest.raises(gc.GravError):
        d.terminate()
    d.terminate_src()


def test_dropin_phases_are_counted():
    """gravcuda_dropin_phases after a walk of drop-in calls: every call
    counted, the staging copies and the submitter's CUDA calls timed."""
    import numpy as np
    from pgrav import gravcuda as gc, host, ics
    pos, m = ics.plummer(4000, seed=5)
    t = host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4,
                  emit_aosoa=True)
    gids = np.arange(min(64, t.ngroups))
    packs = []
    ncalls = 0
    for kind, routine, sz in ((0, "pMp", 4), (1, "pQp", 13), (2, "pHp", 29)):
        bp, data = t.aosoa_subset(gids, kind)
        packs.append((routine, sz, bp, data))
        ncalls += int((np.diff(bp) > 0).sum())
    first = t.groups["first"][gids].astype(np.int64)
    count = t.groups["count"][gids].astype(np.int32)
    bt = gc.body_table(t.sorted_pos, t.points[:t.n, 3])
    d = gc.DropIn(bt)
    secs = gc.drive_mn(d, first, count, packs, 1e-4)
    ph = gc.dropin_phases()
    assert secs > 0 and ph["calls"] == ncalls, (ph, ncalls)
    assert ph["staging_copy_s"] > 0 and ph["submitter_s"] > 0


def test_c_driven_calls_with_split_copies_match_oracle():
    """The mac.c call sequence issued from C (lib/libmacdrive.so) on lists
    long enough that the staging copy is split between the calling thread
    and the copy workers (>= 64 KB parts), calls of every kind and size
    back to back: every group's sinks against the oracle on the same AoSoA
    lists.  A copy that returned before all of its parts were written would
    hand a stale list to the device."""
    from pgrav import gravcuda as gc, host, ics
    pos, m = ics.grf_box(32, seed=11, rms_disp=0.3)
    t = host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-5, box=1.0)
    lens = sum(np.diff(t.ptr[k]) for k in range(3))
    gids = np.sort(np.argsort(lens)[-40:])
    eps2 = (1.0 / 32 / 50) ** 2
    packs = []
    for kind, routine, sz in ((0, "pMp", 4), (1, "pQp", 13), (2, "pHp", 29)):
        bp, data = t.aosoa_subset(gids, kind)
        packs.append((routine, sz, bp, data))
    big = max(int(np.diff(bp).max()) * sz * 8 * 4 for _, sz, bp, _ in packs)
    assert big >= 2 * (64 << 10), big          # the copy is split
    first = t.groups["first"][gids].astype(np.int64)
    count = t.groups["count"][gids].astype(np.int32)
    bt = gc.body_table(t.sorted_pos, t.points[:t.n, 3])
    gots = []
    for _ in range(3):                           # later passes reuse the staging buffers
        d = gc.DropIn(bt.copy())
        gc.drive_mn(d, first, count, packs, eps2)   # ends with WalkTerminateSinkCUDA
        gots.append(d.btab[:, 7:11].copy())
    kinds = {"pMp": O.MONO_PLUMMER, "pQp": O.QUAD_PLUMMER, "pHp": O.HEXA_PLUMMER}
    want = np.zeros((t.n, 4))
    for routine, sz, bp, data in packs:
        for j, g in enumerate(gids):
            nblk = int(bp[j + 1] - bp[j])
            if nblk == 0:
                continue
            f = O.aligned_f32(nblk * sz * 8)
            f[:] = data[bp[j] * sz * 8:bp[j + 1] * sz * 8]
            f0, c = int(first[j]), int(count[j])
            for s in range(f0, f0 + c):
                want[s] += O.list_eval(kinds[routine], f, nblk, t.sorted_pos[s], eps2)
    rows = np.concatenate([np.arange(f0, f0 + c) for f0, c in zip(first, count)])
    for got in gots:
        assert rms_rel(got[rows, :3], want[rows, :3]) < RMS_TOL
        assert rms_rel(got[rows, 3:], want[rows, 3:]) < RMS_TOL


def test_background_subtracted_monopoles(gc, golden):
    """A background-subtracting walk (nln/mac.c DLRcritMACsb) hands the
    drop-in ordinary pMp lists whose extra entries are negative-mass
    monopoles: the uniform cubes of opened cells and of single bodies
    (mac.c:1662-1690, 1695-1708).  grav_mn_CUDA evaluates them as it does
    every entry; against the oracle and, on the real-mass part, the
    reference fixture."""
    rec = np.asarray(golden["k0_records"], np.float32)
    sinks = golden["k0_sinks"]
    e = float(golden["k0_e"])
    rng = np.random.default_rng(9)
    anti = np.zeros((57, 4), np.float32)
    anti[:, :3] = rng.uniform(-1.5, 1.5, (57, 3))
    anti[:, 3] = -float(rec[:, 3].mean()) * rng.uniform(0.2, 1.0, 57)   # -rho0 x cube volume
    both = np.concatenate([rec, anti])
    f, nblk = O.pack_aosoa(both)
    d = gc.DropIn(gc.body_table(sinks, 1.0))
    d.mn("pMp", 0, len(sinks), f, nblk * 8, 4, e)
    got = d.terminate()
    want = np.array([O.list_eval(O.MONO_PLUMMER, f, nblk, s, e) for s in sinks])
    assert rms_rel(got[:, :3], want[:, :3]) < RMS_TOL
    assert rms_rel(got[:, 3:], want[:, 3:]) < RMS_TOL
    # the anti-masses alone are what separates it from the reference fixture
    fa, na = O.pack_aosoa(anti)
    wanta = np.array([O.list_eval(O.MONO_PLUMMER, fa, na, s, e) for s in sinks])
    assert rms_rel(got - wanta, golden["k0_ref"]) < RMS_TOL
