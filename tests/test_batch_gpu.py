"""GPU parity of the batched index-list path (grav_groups_*) against the
oracle on identical lists, and its accuracy against the FP64 direct sum."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
RMS_TOL = 1e-5


def rms_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.sqrt(np.mean(np.sum((a - b) ** 2, axis=-1)) / np.mean(np.sum(b * b, axis=-1)))


@pytest.fixture(scope="module")
def gc():
    from pgrav import gravcuda
    return gravcuda


def make_tree(kind, n, **kw):
    from pgrav import host, ics
    if kind == "plummer":
        pos, m = ics.plummer(n, seed=11)
        return host.Tree(pos, m, emit_aosoa=True, **kw)
    n1 = int(round(n ** (1 / 3)))
    pos, m = ics.grf_box(n1, seed=11)
    return host.Tree(pos, m, box=1.0, emit_aosoa=True, **kw)


@pytest.mark.parametrize("order", [2, 4])
def test_batched_plummer_matches_oracle(gc, order):
    t = make_tree("plummer", 20000, leaf_max=16, group_max=32, p2cut=7,
                  p4cut=20 if order == 4 else 0, tol=1e-3)
    eps2 = 0.01 ** 2
    plan = gc.Plan(t, eps2, quad_phi_sign=1.0)
    plan.eval()
    got = plan.download()
    want = O.tree_eval(t, eps2)
    assert rms_rel(got[:, :3], want[:, :3]) < RMS_TOL
    assert rms_rel(got[:, 3:], want[:, 3:]) < RMS_TOL
    assert (plan.counts() == t.counts).all()


def test_batched_reference_sign(gc):
    """quad_phi_sign = -1 reproduces do_gravpq's potential exactly."""
    t = make_tree("plummer", 6000, leaf_max=16, group_max=32, p2cut=7, p4cut=0, tol=1e-3)
    eps2 = 0.01 ** 2
    plan = gc.Plan(t, eps2, quad_phi_sign=-1.0)
    plan.eval()
    got = plan.download()
    want = O.tree_eval(t, eps2, quad_kind=O.QUAD_PLUMMER)
    assert rms_rel(got, want) < RMS_TOL


def test_batched_periodic_images_match_oracle(gc):
    """Periodic box: every list entry carries its image shift; the Newtonian
    part must match the oracle on the same shifted lists."""
    t = make_tree("box", 32 ** 3, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-3)
    assert ((t.plist >> 27) != 13).any()
    eps2 = (1.0 / 32 / 50) ** 2
    plan = gc.Plan(t, eps2)
    plan.eval()
    got = plan.download()
    want = O.tree_eval(t, eps2)
    assert rms_rel(got[:, :3], want[:, :3]) < RMS_TOL


def test_batched_accuracy_vs_direct(gc):
    t = make_tree("plummer", 20000, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-5)
    eps2 = 0.01 ** 2
    plan = gc.Plan(t, eps2)
    plan.eval()
    got = plan.download()
    rng = np.random.default_rng(3)
    samp = rng.choice(t.n, 1000, replace=False)
    acc, phi = O.direct(t.sorted_pos, t.points[:t.n, 3], eps2, samp)
    err = np.linalg.norm(got[samp, :3] - acc, axis=1) / np.linalg.norm(acc, axis=1)
    assert np.sqrt(np.mean(err ** 2)) < 1e-4
    perr = np.abs(got[samp, 3] - phi) / np.abs(phi)
    assert np.sqrt(np.mean(perr ** 2)) < 1e-4


def test_batched_repeatable(gc):
    t = make_tree("plummer", 5000, leaf_max=8, group_max=32, p2cut=7, p4cut=20, tol=1e-3)
    plan = gc.Plan(t, 1e-4)
    plan.eval()
    a = plan.download()
    plan.eval()
    b = plan.download()
    assert np.array_equal(a, b)  # deterministic: fixed per-group summation order


def test_upload_refuses_bad_entries(gc):
    """Every list entry is checked on the device at upload: an index past its
    table, or an image code past 26, fails the upload with a status."""
    t = make_tree("plummer", 5000, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
    for kind, bad in ((0, t.n + t.ncells + 5), (2, t.ncells + 1), (0, 5 | (27 << 27))):
        lst = {0: t.plist, 1: t.qlist, 2: t.hlist}[kind]
        keep = int(lst[3])
        lst[3] = bad
        try:
            with pytest.raises(gc.GravError, match="outside its table|image code"):
                gc.Plan(t, 1e-4)
        finally:
            lst[3] = keep
    p = gc.Plan(t, 1e-4)   # intact lists still upload
    p.free()


def test_lists_read_in_place_from_host_memory(gc):
    """lists_in_host: the kernels read page-locked lists over PCIe; the
    results are those of the copied lists, bit for bit."""
    t = make_tree("box", 24 ** 3, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
    eps2 = (1.0 / 24 / 50) ** 2
    outs = []
    for in_host in (False, True):
        pp = gc.pinned_problem(t, lists_in_host=in_host)
        outs.append(gc.groups_eval_problem(pp, eps2, 1.0, ewald=True).copy())
    assert np.array_equal(outs[0], outs[1])
    # pageable lists are refused in that mode
    prob = gc.pinned_problem(t, lists_in_host=True).problem
    prob.plist = t.plist.ctypes.data
    with pytest.raises(gc.GravError, match="page-locked"):
        gc.check(gc.lib().grav_groups_CUDA(__import__("ctypes").byref(prob),
                                           np.empty((t.n, 4), np.float32).ctypes.data))


@pytest.mark.parametrize("chunks", ["1", "3", "7"])
def test_pipelined_end_to_end_matches_plan(gc, chunks, monkeypatch):
    """grav_groups_CUDA copies the lists group range by group range on a copy
    stream while the kernels evaluate the ranges already copied: the results
    are those of a plan that uploaded everything first, bit for bit."""
    t = make_tree("box", 24 ** 3, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
    eps2 = (1.0 / 24 / 50) ** 2
    plan = gc.Plan(t, eps2, ewald=True)
    plan.eval()
    ref = plan.download()
    plan.free()
    monkeypatch.setenv("GRAV_E2E_CHUNKS", chunks)
    pp = gc.pinned_problem(t, lists_in_host=False)
    got = gc.groups_eval_problem(pp, eps2, 1.0, ewald=True).copy()
    assert np.array_equal(got, ref)


def test_pipelined_end_to_end_reports_bad_entries(gc, monkeypatch):
    """Without an upload-time list check, the kernels' own index checks flag
    an entry past its table and the call fails with a status."""
    t = make_tree("plummer", 5000, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
    monkeypatch.setenv("GRAV_E2E_CHUNKS", "3")
    for kind, bad in ((0, t.n + t.ncells + 5), (2, t.ncells + 1), (1, 7 | (27 << 27))):
        pp = gc.pinned_problem(t, lists_in_host=False)
        lst = pp.lists[kind]
        lst[len(lst) // 2] = bad
        with pytest.raises(gc.GravError, match="device error word"):
            gc.groups_eval_problem(pp, 1e-4, 0.0)
        gc.lib().gravcuda_clear_status()
    pp = gc.pinned_problem(t, lists_in_host=False)
    gc.groups_eval_problem(pp, 1e-4, 0.0)   # intact lists still evaluate


def test_end_to_end_list_buffer_grows_and_releases(gc, monkeypatch):
    """The memory kept between end-to-end calls serves a smaller problem,
    grows for a larger one, and is allocated again after
    grav_groups_release_CUDA."""
    monkeypatch.setenv("GRAV_E2E_CHUNKS", "2")
    small = make_tree("plummer", 3000, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
    large = make_tree("plummer", 12000, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
    refs = {}
    for t in (small, large):
        plan = gc.Plan(t, 1e-4)
        plan.eval()
        refs[id(t)] = plan.download()
        plan.free()
    for t in (small, large, small):
        got = gc.groups_eval_problem(gc.pinned_problem(t), 1e-4, 0.0)
        assert np.array_equal(got, refs[id(t)])
    gc.lib().grav_groups_release_CUDA()
    got = gc.groups_eval_problem(gc.pinned_problem(large), 1e-4, 0.0)
    assert np.array_equal(got, refs[id(large)])
    gc.lib().grav_groups_release_CUDA()


@pytest.mark.parametrize("chunks", ["1", "3", "7"])
@pytest.mark.parametrize("kind", ["box", "plummer"])
def test_run_packed_end_to_end_matches_plan(gc, chunks, kind, monkeypatch):
    """grav_groups_CUDA given run-packed lists (nln_tree_pack) copies the
    packed words and unpacks them on the device (k_unpack) before each
    range's kernels: the results are the plain-list plan's, bit for bit."""
    if kind == "box":
        t = make_tree("box", 24 ** 3, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
        eps2, box, ewald = (1.0 / 24 / 50) ** 2, 1.0, True
    else:
        t = make_tree("plummer", 8000, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
        eps2, box, ewald = 1e-4, 0.0, False
    plan = gc.Plan(t, eps2, ewald=ewald)
    plan.eval()
    ref = plan.download()
    plan.free()
    monkeypatch.setenv("GRAV_E2E_CHUNKS", chunks)
    pp = gc.pinned_problem(t, packed=True)
    assert pp.problem.plist is None
    assert pp.h2d_bytes < t.plist.nbytes + t.qlist.nbytes + t.hlist.nbytes + t.clist.nbytes
    got = gc.groups_eval_problem(pp, eps2, box, ewald=ewald).copy()
    assert np.array_equal(got, ref)
    gc.lib().grav_groups_release_CUDA()


def test_run_packed_end_to_end_reports_malformed_runs(gc, monkeypatch):
    """A packed group that unpacks longer or shorter than its plain range, a
    run word at a group's start and a run word after a run word each fail
    the call with the device error word; the device writes stay inside each
    group's range."""
    t = make_tree("plummer", 6000, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
    t.pack()
    monkeypatch.setenv("GRAV_E2E_CHUNKS", "2")
    z, zp = t.zlist[0], t.zptr[0]
    runs = np.nonzero((z >> 27) == 31)[0]
    r = int(runs[len(runs) // 2])
    g = int(np.searchsorted(zp, r, side="right") - 1)
    edits = [
        (r, z[r] + 1),                      # one entry too many
        (r, z[r] - 1 if (z[r] & 0x7FFFFFF) > 1 else z[r] + 2),   # too few / too many
        (int(zp[g]), (31 << 27) | 1),       # run word starts the group
        (r + 1 if r + 1 < zp[g + 1] else r - 1, (31 << 27) | 1),  # run next to a run
    ]
    for pos, val in edits:
        pp = gc.pinned_problem(t, packed=True)
        pp.lists[0][pos] = val
        with pytest.raises(gc.GravError, match="device error word"):
            gc.groups_eval_problem(pp, 1e-4, 0.0)
        gc.lib().gravcuda_clear_status()
    gc.groups_eval_problem(gc.pinned_problem(t, packed=True), 1e-4, 0.0)
    gc.lib().grav_groups_release_CUDA()


def test_ewald_moments_on_side_stream_match_finish_pass(gc):
    """The periodic correction's moments computed by k_ewald_side on a side
    stream, beside the list kernels (the default), give the results of the
    moments computed inside the finish pass, bit for bit.  (The periodic
    KDK test of test_step_gpu.py runs the fork and join inside a captured
    CUDA graph.)"""
    t = make_tree("box", 20 ** 3, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
    eps2 = (1.0 / 20 / 50) ** 2
    outs = []
    for side in (-1, 0, 3):
        plan = gc.Plan(t, eps2, ewald=True, tuning=gc.Tuning(8, 0, 0, 0, 0, 0, side))
        plan.eval()
        outs.append(plan.download())
        plan.free()
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])


@pytest.mark.parametrize("order", [2, 4])
def test_plain_fp32_kernels_match_oracle(gc, order):
    """precision = 1 (plain FP32: absolute coordinates, plain sums) on the same
    lists: a Plummer sphere about the origin, where absolute FP32
    coordinates lose nothing, matches the oracle like the mixed form."""
    t = make_tree("plummer", 20000, leaf_max=16, group_max=32, p2cut=7,
                  p4cut=20 if order == 4 else 0, tol=1e-3)
    eps2 = 0.01 ** 2
    plan = gc.Plan(t, eps2, plain=True)
    plan.eval()
    got = plan.download()
    plan.free()
    want = O.tree_eval(t, eps2)
    assert rms_rel(got[:, :3], want[:, :3]) < RMS_TOL
    assert rms_rel(got[:, 3:], want[:, 3:]) < RMS_TOL


def test_plain_fp32_loses_accuracy_far_from_the_origin(gc):
    """The same sphere moved to (1e4, 1e4, 1e4), order 2: plain FP32 rounds
    every cell centre to an absolute FP32 coordinate (ulp 1e-3 there), the
    mixed form keeps FP32 offsets from FP64 group centres.  Reference: the
    FP64 evaluation of the same lists from the same (FP32) bodies."""
    from pgrav import host, ics
    pos, m = ics.plummer(20000, seed=11)
    pos = pos + np.float32(1.0e4)
    t = host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=7, p4cut=0, tol=1e-3)
    eps2 = 0.01 ** 2
    want = O.ListsFP64(t).eval(t.sorted_pos, t.points[:t.n, 3], eps2)
    errs = {}
    for plain in (False, True):
        plan = gc.Plan(t, eps2, plain=plain)
        plan.eval()
        errs[plain] = rms_rel(plan.download()[:, :3], want[:, :3])
        plan.free()
    assert errs[False] < 1e-5, errs
    assert errs[True] > 10 * errs[False], errs
