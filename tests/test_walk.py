"""Host walk invariants (csrc/host/nlnhost.cpp): the chunked list assembly
equals the single-chunk one, and every group's correction list covers each
body exactly once, in the image its Newtonian entries use."""
import numpy as np


def _decode(e, n):
    idx = e & ((1 << 27) - 1)
    sc = e >> 27
    return idx, np.stack([sc // 9 - 1, (sc // 3) % 3 - 1, sc % 3 - 1], -1)


def test_chunked_walk_equals_single_chunk():
    from pgrav import host, ics
    pos, m = ics.grf_box(64, seed=3, rms_disp=0.3)
    # 64^3 bodies in groups of <= 32 gives more than one 16384-group chunk;
    # emit_aosoa forces a single chunk
    a = host.Tree(pos, m, tol=3e-4, box=1.0, group_max=16)
    b = host.Tree(pos, m, tol=3e-4, box=1.0, group_max=16, emit_aosoa=True)
    assert a.ngroups > 16384
    for k in range(4):
        assert np.array_equal(a.ptr[k], b.ptr[k])
    for x, y in ((a.plist, b.plist), (a.qlist, b.qlist), (a.hlist, b.hlist), (a.clist, b.clist)):
        assert np.array_equal(x, y)
    assert np.array_equal(a.counts, b.counts)


def test_correction_list_covers_bodies_once_in_newtonian_image():
    from pgrav import host, ics
    pos, m = ics.grf_box(24, seed=5, rms_disp=0.3)
    t = host.Tree(pos, m, tol=1e-4, box=1.0, ewald_theta=0.2)
    cf, cc = t.cell_ranges()
    n = t.n

    def bodies_with_shift(lst, ptr, g, kind):
        out = np.full((n, 3), 99, np.int64)
        hit = np.zeros(n, np.int64)
        idx, sh = _decode(lst[ptr[g]:ptr[g + 1]].astype(np.int64), n)
        for i, s in zip(idx, sh):
            if kind in (0, 3) and i < n:
                rng = np.array([i])
            else:
                c = i - n if kind in (0, 3) else i
                rng = np.arange(cf[c], cf[c] + cc[c])
            hit[rng] += 1
            out[rng] = s
        return hit, out

    rng = np.random.default_rng(0)
    for g in rng.choice(t.ngroups, 12, replace=False):
        hits_n = np.zeros(n, np.int64)
        img_n = np.full((n, 3), 99, np.int64)
        for kind, lst in ((0, t.plist), (1, t.qlist), (2, t.hlist)):
            h, o = bodies_with_shift(lst, t.ptr[kind], g, kind)
            hits_n += h
            img_n[h > 0] = o[h > 0]
        hc, img_c = bodies_with_shift(t.clist, t.ptr[3], g, 3)
        assert np.all(hits_n == 1) and np.all(hc == 1)
        assert np.array_equal(img_n, img_c)
        # coarse cells make the correction list shorter than the Newtonian lists
        assert t.ptr[3][g + 1] - t.ptr[3][g] <= sum(t.ptr[k][g + 1] - t.ptr[k][g] for k in range(3))


def test_merge_renumbers_members():
    from pgrav import host, ics
    trees = []
    for k, n in enumerate((700, 1500, 333)):
        pos, m = (ics.plummer if k % 2 == 0 else ics.hernquist)(n, seed=40 + k)
        trees.append(host.Tree(pos, m, tol=1e-3, p2cut=7, p4cut=20))
    b = host.Tree.merge(trees)
    assert b.n == sum(t.n for t in trees) and b.ncells == sum(t.ncells for t in trees)
    assert b.ngroups == sum(t.ngroups for t in trees)
    assert list(b.body_offsets) == [0, 700, 2200, 2533]
    assert (b.counts == sum(t.counts for t in trees)).all()
    bo = co = go = 0
    for t in trees:
        assert np.array_equal(b.points[bo:bo + t.n], t.points[:t.n])
        assert np.array_equal(b.points[b.n + co:b.n + co + t.ncells], t.points[t.n:])
        assert np.array_equal(b.order[bo:bo + t.n], bo + t.order)
        assert np.array_equal(b.groups["first"][go:go + t.ngroups], bo + t.groups["first"])
        for g in range(t.ngroups):
            e = t.plist[t.ptr[0][g]:t.ptr[0][g + 1]] & ((1 << 27) - 1)
            want = np.where(e < t.n, bo + e, b.n + co + (e - t.n))
            got = b.plist[b.ptr[0][go + g]:b.ptr[0][go + g + 1]] & ((1 << 27) - 1)
            assert np.array_equal(got, want)
            for k, lst, blst in ((1, t.qlist, b.qlist), (2, t.hlist, b.hlist)):
                e = lst[t.ptr[k][g]:t.ptr[k][g + 1]] & ((1 << 27) - 1)
                got = blst[b.ptr[k][go + g]:b.ptr[k][go + g + 1]] & ((1 << 27) - 1)
                assert np.array_equal(got, co + e)
        ch, nc, lv = t.cell_links()
        bch, bnc, blv = b.cell_links()
        assert np.array_equal(bch[co:co + t.ncells], np.where(ch >= 0, ch + co, -1))
        assert np.array_equal(blv[co:co + t.ncells], lv)
        bo += t.n
        co += t.ncells
        go += t.ngroups


def test_run_packed_lists_unpack_to_the_plain_lists():
    """nln_tree_pack: every kind of list (points, quadrupole, order 4,
    correction) of an isolated and a periodic tree unpacks, with the CPU
    decoder, to exactly the plain list and offsets; runs never cross a group
    or an image-code change, and the point list packs several-fold."""
    from pgrav import host, ics
    from oracle import oracle as O
    pos, m = ics.plummer(6000, seed=8)
    iso = host.Tree(pos, m, tol=1e-4, p2cut=7, p4cut=20).pack()
    pos, m = ics.grf_box(20, seed=9, rms_disp=0.3)
    per = host.Tree(pos, m, tol=1e-4, box=1.0, p2cut=7, p4cut=20).pack()
    for t in (iso, per):
        plain = (t.plist, t.qlist, t.hlist, t.clist)
        for k in range(4):
            if len(t.ptr[k]) == 0:
                assert len(t.zlist[k]) == 0
                continue
            ptr, lst = O.unpack_runs(t.zptr[k], t.zlist[k])
            assert np.array_equal(ptr, t.ptr[k]), k
            assert np.array_equal(lst, plain[k]), k
            assert len(t.zlist[k]) <= len(plain[k])
        assert len(t.zlist[0]) * 3 < len(t.plist)
    # groups with empty lists of a kind keep zero words
    q = np.diff(per.ptr[1]) == 0
    assert np.array_equal(np.diff(per.zptr[1])[q], np.zeros(q.sum(), np.int64))


def test_unpack_rejects_malformed_runs():
    """The CPU decoder (the device unpacker's checker) refuses a run word at
    a group's start and a run word after a run word."""
    import pytest
    from oracle import oracle as O
    run = lambda n: (31 << 27) | n
    e = (13 << 27) | 100
    ptr, lst = O.unpack_runs([0, 3], np.array([e, run(4), e + 20], np.uint32))
    assert ptr.tolist() == [0, 6]
    assert lst.tolist() == [e, e + 1, e + 2, e + 3, e + 4, e + 20]
    with pytest.raises(AssertionError, match="starts a group"):
        O.unpack_runs([0, 1, 3], np.array([e, run(2), e], np.uint32))
    with pytest.raises(AssertionError, match="follows a run word"):
        O.unpack_runs([0, 3], np.array([e, run(2), run(1)], np.uint32))


def test_coincident_bodies_split_into_small_groups():
    """A leaf of coincident bodies cannot split: its run becomes consecutive
    groups of at most group_max sinks, and the walk still covers every body."""
    from pgrav import host
    rng = np.random.default_rng(5)
    pos = np.concatenate([rng.normal(0, 1, (3000, 3)), np.zeros((300, 3))]).astype(np.float32)
    m = np.full(len(pos), 1.0 / len(pos), np.float32)
    t = host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)
    assert t.groups["count"].max() <= 32
    assert t.groups["count"].sum() == t.n
    first = t.groups["first"]
    assert np.array_equal(first[1:], first[:-1] + t.groups["count"][:-1])
