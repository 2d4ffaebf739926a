"""Generate tests/golden/ref_kernels.npz: outputs of the reference's own CPU
code (the AVX kernels of nln/do_grav_avx8.c and nln/pgrav_vec.c, and ewald()
of nln/ewald.c, compiled unmodified into oracle/_ref by oracle/Makefile) on
seeded inputs.

Run here, where the reference tree is present:  python tests/golden/make_golden.py
The fixture travels with the repository; tests compare both the CPU
restatement (oracle/grav_oracle.c) and the GPU kernels against it.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402

# kind -> (e value, description)
CASES = {
    O.MONO_PLUMMER: 1e-4,
    O.QUAD_PLUMMER: 1e-4,
    O.HEXA_PLUMMER: 1e-4,
    O.MONO_MASKED: 0.05,
    O.MONO_K1: 5.0,        # 1/eps = 5: eps = 0.2, so some lanes fall inside
    O.QUAD_COM: 0.0,
    O.HEXA_COM: 0.0,
}


def make_records(rng, kind, n):
    sz = O.KIND_SZ[kind]
    rec = np.zeros((n, sz), np.float32)
    rec[:, 0] = rng.uniform(0.5, 1.5, n) / n
    if sz == 4:
        rec[:, 1:4] = rng.normal(0.0, 0.6, (n, 3))
    else:
        # cells 1..3 units away, moments of plausible size
        d = rng.normal(size=(n, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        rec[:, 1:4] = d * rng.uniform(1.0, 3.0, (n, 1))
        rec[:, 4] = rng.uniform(0.05, 0.3, n)
        rec[:, 8:] = rng.normal(0.0, 0.05, (n, sz - 8)) * rec[:, :1]
    return rec


def main():
    O.build()
    assert O.ref_available(), "reference kernels not built (needs the reference tree)"
    rng = np.random.default_rng(20261203)
    out = {}
    for kind, e in CASES.items():
        n = 203  # not a multiple of 8: exercises the zero-mass padding lanes
        rec = make_records(rng, kind, n)
        f, nblk = O.pack_aosoa(rec)
        sinks = rng.normal(0.0, 0.3, (16, 3)).astype(np.float32)
        res = np.zeros((16, 4), np.float32)
        for i, s in enumerate(sinks):
            res[i] = O.ref_list_eval(kind, f, nblk, s, e)
        out[f"k{kind}_records"] = rec
        out[f"k{kind}_sinks"] = sinks
        out[f"k{kind}_e"] = np.float32(e)
        out[f"k{kind}_ref"] = res
    # MxN kernels of nln/pgrav_vec.c on one monopole / quadrupole / order-4 list
    for kind, pk in ((O.MONO_PLUMMER, 0), (O.QUAD_COM, 1), (O.HEXA_COM, 2)):
        rec = out[f"k{kind}_records"]
        f, nblk = O.pack_aosoa(rec)
        m = 16
        p = np.zeros((m, 4), np.float32)
        p[:, 1:4] = out[f"k{kind}_sinks"]
        accp = np.zeros((m, 4), np.float32)
        O.ref().ref_pinteract(pk, p.ravel(), accp.ravel(), m, 4, f, nblk)
        out[f"pinteract{pk}_ref"] = accp
    # body-run K1 kernel (do_gravmm_sK1_avx8)
    xyz = rng.normal(0.0, 0.5, (300, 3)).astype(np.float32)
    seg = np.array([[0, 40], [57, 13], [100, 150], [260, 39]], np.uint32)
    sinks = rng.normal(0.0, 0.5, (8, 3)).astype(np.float32)
    res = np.zeros((8, 4), np.float32)
    for i, s in enumerate(sinks):
        O.ref().ref_segments_k1(xyz.ravel(), 3, np.float32(1.0 / 300), seg.ravel(), len(seg),
                                int(seg[:, 1].sum()), s, 5.0, res[i])
    out.update(mm_xyz=xyz, mm_seg=seg, mm_sinks=sinks, mm_mass=np.float32(1.0 / 300),
               mm_e=np.float32(5.0), mm_ref=res)
    # the reference's one test fixture (nln/py_pgrav/test_pgrav.py:6-27): seed 123,
    # 16 sources of mass 1/16, a sink at (1,0,0); values from pMinteract
    rs = np.random.RandomState(123)
    src = np.empty((16, 4), np.float32)
    src[:, 0] = 1.0 / 16
    src[:, 1] = rs.uniform(0.0, 1.0, 16)
    src[:, 2] = rs.uniform(-0.5, 0.5, 16)
    src[:, 3] = rs.uniform(-0.5, 0.5, 16)
    f, nblk = O.pack_aosoa(src)
    p = np.array([1.0, 0.0, 0.0, 0.0], np.float32)
    accp = np.zeros(4, np.float32)
    O.ref().ref_pinteract(0, p, accp, 1, 4, f, nblk)
    out.update(pgrav_src=src, pgrav_sink=p, pgrav_ref=accp)
    # (added after the cases above, from their own seeds, so earlier arrays keep their values)
    # do_gravdq_avx8: quadrupole plus the dipole fields, the arithmetic of the CUDA
    # pQ1_mnss / pQQ1 kernels behind grav_qnss_CUDA / grav_qns_CUDA
    rng = np.random.default_rng(20261204)
    rec = make_records(rng, O.QUAD_COM, 203)
    rec[:, 5:8] = rng.normal(0.0, 0.1, (203, 3)) * rec[:, :1]
    f, nblk = O.pack_aosoa(rec)
    sinks = rng.normal(0.0, 0.3, (16, 3)).astype(np.float32)
    res = np.zeros((16, 4), np.float32)
    for i, s in enumerate(sinks):
        res[i] = O.ref_list_eval(O.QUAD_DIPOLE, f, nblk, s, 0.0)
    k = O.QUAD_DIPOLE
    out.update({f"k{k}_records": rec, f"k{k}_sinks": sinks, f"k{k}_e": np.float32(0.0),
                f"k{k}_ref": res})
    # ewald() of nln/ewald.c (compiled unmodified with the stand-in 2hot headers of
    # oracle/ref_stubs) at seeded displacements, box sides 1 and 3
    rng = np.random.default_rng(20261205)
    for tag, L in (("1", 1.0), ("3", 3.0)):
        x = np.concatenate([rng.uniform(-0.5 * L, 0.5 * L, (200, 3)),
                            rng.uniform(-2.0 * L, 2.0 * L, (50, 3)),
                            rng.normal(0.0, 1e-3 * L, (6, 3))])
        fe, pe = O.ref_ewald(x, L)
        out.update({f"ewald{tag}_x": x, f"ewald{tag}_f": fe, f"ewald{tag}_phi": pe})
    np.savez_compressed(os.path.join(HERE, "ref_kernels.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_kernels.npz"))


if __name__ == "__main__":
    main()
