"""Pin the CPU restatement (oracle/grav_oracle.c) to the reference's own
kernels: the committed fixtures from the compiled reference AVX kernels
(tests/golden/make_golden.py) always, and the compiled reference itself on
fresh random lists when oracle/_ref is present."""
import numpy as np
import pytest

from oracle import oracle as O

KINDS = [O.MONO_PLUMMER, O.QUAD_PLUMMER, O.HEXA_PLUMMER, O.MONO_MASKED, O.MONO_K1, O.QUAD_COM,
         O.HEXA_COM, O.QUAD_DIPOLE]


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("kind", KINDS)
def test_restatement_matches_golden(golden, kind):
    rec = golden[f"k{kind}_records"]
    f, nblk = O.pack_aosoa(rec)
    e = float(golden[f"k{kind}_e"])
    ref = golden[f"k{kind}_ref"]
    for i, s in enumerate(golden[f"k{kind}_sinks"]):
        got = O.list_eval(kind, f, nblk, s, e)
        # the reference is FP32 with an 11-bit rsqrt + one Newton step
        assert rel(got[:3], ref[i, :3]) < 2e-5, (kind, i)
        assert abs(got[3] - ref[i, 3]) <= 2e-5 * abs(ref[i, 3]) + 1e-7, (kind, i)


def test_k1_fixture_has_inside_lanes(golden):
    rec = golden[f"k{O.MONO_K1}_records"]
    eps = 1.0 / float(golden[f"k{O.MONO_K1}_e"])
    s = golden[f"k{O.MONO_K1}_sinks"]
    d = np.linalg.norm(s[:, None, :] - rec[None, :, 1:4], axis=2)
    assert (d < eps).sum() > 10  # the K1 polynomial branch is exercised


def test_segments_k1_golden(golden):
    xyz = golden["mm_xyz"]
    seg = golden["mm_seg"]
    for i, s in enumerate(golden["mm_sinks"]):
        out = np.zeros(4)
        n = O.orc().orc_segments_k1(xyz.ravel(), 3, float(golden["mm_mass"]), seg.ravel(),
                                    len(seg), s, float(golden["mm_e"]), out)
        assert n == seg[:, 1].sum()
        assert rel(out, golden["mm_ref"][i]) < 2e-5


def test_reference_pgrav_fixture(golden):
    """The reference's only test input (nln/py_pgrav/test_pgrav.py): seed 123,
    16 sources of mass 1/16, sink at (1,0,0), unsoftened monopole."""
    src = golden["pgrav_src"]
    f, nblk = O.pack_aosoa(src)
    got = O.list_eval(O.MONO_BARE, f, nblk, golden["pgrav_sink"][1:4], 0.0)
    assert rel(got, golden["pgrav_ref"]) < 2e-5
    # and the FP64 direct sum agrees (the fixture is a plain 16-body sum)
    x = src[:, 1:4].astype(np.float64) - golden["pgrav_sink"][1:4]
    r = np.linalg.norm(x, axis=1)
    a = (src[:, 0] / r ** 3) @ x
    assert rel(got[:3], a) < 1e-6


def test_mxn_restatement_matches_pinteract(golden):
    for kind, pk in ((O.MONO_PLUMMER, 0), (O.QUAD_COM, 1), (O.HEXA_COM, 2)):
        rec = golden[f"k{kind}_records"]
        f, nblk = O.pack_aosoa(rec)
        m = 16
        p = np.zeros((m, 4), np.float32)
        p[:, 1:4] = golden[f"k{kind}_sinks"]
        accp = np.zeros((m, 4), np.float32)
        # pMinteract is unsoftened; pQinteract/pHinteract are the COM kernels
        okind = {0: O.MONO_BARE, 1: O.QUAD_COM, 2: O.HEXA_COM}[pk]
        O.orc().orc_mxn_eval(okind, p.ravel(), accp.ravel(), m, 4, f, nblk, O.KIND_SZ[okind], 0.0)
        ref = golden[f"pinteract{pk}_ref"]
        assert rel(accp[:, :3], ref[:, :3]) < 2e-5
        if pk == 1:
            # pQinteract adds the quadrupole potential with + (nln/pgrav_vec.c), do_gravq with -
            continue
        assert rel(accp[:, 3], ref[:, 3]) < 2e-5


@pytest.mark.skipif(not O.ref_available(), reason="reference kernels not built here")
@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("seed", [1, 2])
def test_restatement_matches_compiled_reference(kind, seed):
    rng = np.random.default_rng(seed * 100 + kind)
    sz = O.KIND_SZ[kind]
    n = int(rng.integers(1, 400))
    rec = rng.normal(0.0, 0.05, (n, sz)).astype(np.float32)
    rec[:, 0] = rng.uniform(0.1, 1.0, n)
    rec[:, 1:4] = rng.uniform(-2.0, 2.0, (n, 3))
    if sz > 4:
        rec[:, 1:4] += np.sign(rec[:, 1:4]) * 1.0
        rec[:, 4] = rng.uniform(0.01, 0.2, n)
        # dipole fields: zero about the centre of mass, except for do_gravdq's records
        rec[:, 5:8] = 0.0 if kind != O.QUAD_DIPOLE else rng.normal(0.0, 0.1, (n, 3)) * rec[:, :1]
    f, nblk = O.pack_aosoa(rec)
    e = {O.MONO_PLUMMER: 1e-3, O.QUAD_PLUMMER: 1e-3, O.HEXA_PLUMMER: 1e-3, O.MONO_MASKED: 0.3,
         O.MONO_K1: 2.0, O.QUAD_COM: 0.0, O.HEXA_COM: 0.0, O.QUAD_DIPOLE: 0.0}[kind]
    for s in rng.uniform(-0.5, 0.5, (8, 3)).astype(np.float32):
        a = O.list_eval(kind, f, nblk, s, e)
        b = O.ref_list_eval(kind, f, nblk, s, e)
        assert rel(a[:3], b[:3]) < 2e-5
        assert abs(a[3] - b[3]) <= 2e-5 * abs(b[3]) + 1e-6


def test_direct_sum_symmetry():
    rng = np.random.default_rng(0)
    pos = rng.normal(size=(200, 3))
    m = rng.uniform(0.5, 1.5, 200)
    acc, phi = O.direct(pos, m, 1e-4)
    # momentum conservation: sum m a = 0; potential energy symmetric
    assert np.abs((m[:, None] * acc).sum(0)).max() < 1e-10 * np.abs(m[:, None] * acc).sum()
    assert np.all(phi < 0)
