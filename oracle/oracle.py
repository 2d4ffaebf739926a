"""TEST INFRASTRUCTURE ONLY: ctypes access to the parity checkers.

* ``liboracle``   -- this repository's CPU restatement (oracle/grav_oracle.c)
* ``libnlnref``   -- the reference's own AVX kernels compiled unmodified from
                     nln/do_grav_avx8.c and nln/pgrav_vec.c (oracle/Makefile)

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, as the checker; the product path never does.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libnlnref.so")

# list kinds (shared numbering with grav_oracle.c / ref_harness.c)
MONO_PLUMMER, QUAD_PLUMMER, HEXA_PLUMMER = 0, 1, 2
MONO_MASKED, MONO_K1, QUAD_COM, HEXA_COM, MONO_BARE = 3, 4, 5, 6, 7
QUAD_PLUMMER_P = 8
QUAD_DIPOLE = 9      # do_gravdq_avx8: unsoftened quadrupole plus the dipole fields
KIND_SZ = {0: 4, 1: 13, 2: 29, 3: 4, 4: 4, 5: 13, 6: 29, 7: 4, 8: 13, 9: 13}

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")

_orc = None
_ref = None


def unpack_runs(zptr, zlist):
    """Plain list offsets and entries of a run-packed list (format of
    include/nlnlists.h), decoded on the CPU: an entry word is itself, a run
    word (image code 31, count n) stands for the n entries after the entry
    word before it, index + 1 .. + n, same image code."""
    w = np.asarray(zlist, np.uint32)
    zptr = np.asarray(zptr, np.int64)
    is_run = (w >> np.uint32(27)) == 31
    cnt = np.where(is_run, w & np.uint32((1 << 27) - 1), 1).astype(np.int64)
    first = np.zeros(len(w), bool)
    first[zptr[:-1][zptr[:-1] < len(w)]] = True
    assert not np.any(is_run & first), "a run word starts a group"
    assert not np.any(is_run[1:] & is_run[:-1]), "a run word follows a run word"
    end = np.cumsum(cnt)
    start = end - cnt
    out = np.empty(int(end[-1]) if len(w) else 0, np.uint32)
    out[start[~is_run]] = w[~is_run]
    ri = np.nonzero(is_run)[0]
    if len(ri):
        rc = cnt[ri]
        off = np.arange(rc.sum()) - np.repeat(np.cumsum(rc) - rc, rc) + 1
        out[np.repeat(start[ri], rc) + off - 1] = np.repeat(w[ri - 1], rc) + off.astype(np.uint32)
    ptr = np.concatenate([[0], end])[zptr]
    return ptr, out


# The reference's nln/ directory, where oracle/Makefile compiles the
# reference's own CPU code from (NLN_REF_DIR overrides); absent on a machine
# without the reference tree, where only the restatement is built.
REF_NLN = os.environ.get("NLN_REF_DIR", "/root/reference/nln")


def build():
    """Compile the restatement (and the reference's CPU code when the reference tree is present)."""
    cmd = ["make", "-s", "-C", HERE]
    if os.path.exists(os.path.join(REF_NLN, "do_grav_avx8.c")):
        cmd.append(f"REF_NLN={REF_NLN}")
    subprocess.run(cmd, check=True)


def orc():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = ctypes.CDLL(ORACLE_SO)
        lib.orc_list_eval.argtypes = [ctypes.c_int, _f32p, ctypes.c_long, ctypes.c_int, _f32p,
                                      ctypes.c_float, _f64p]
        lib.orc_list_eval.restype = ctypes.c_int
        lib.orc_mxn_eval.argtypes = [ctypes.c_int, _f32p, _f32p, ctypes.c_int, ctypes.c_int, _f32p,
                                     ctypes.c_long, ctypes.c_int, ctypes.c_float]
        lib.orc_segments_k1.argtypes = [_f32p, ctypes.c_int, ctypes.c_float, _u32p, ctypes.c_int,
                                        _f32p, ctypes.c_float, _f64p]
        lib.orc_segments_k1.restype = ctypes.c_long
        lib.orc_direct.argtypes = [_f64p, _f64p, ctypes.c_long, ctypes.c_double, _i64p,
                                   ctypes.c_long, _f64p, _f64p]
        lib.orc_ewald.argtypes = [_f64p, ctypes.c_double, _f64p, _f64p]
        lib.orc_ewald_batch.argtypes = [_f64p, ctypes.c_long, ctypes.c_double, _f64p, _f64p]
        lib.orc_direct_ewald.argtypes = [_f64p, _f64p, ctypes.c_long, ctypes.c_double,
                                         ctypes.c_double, _i64p, ctypes.c_long, _f64p, _f64p]
        lib.orc_groups_eval.argtypes = [ctypes.c_int, _f32p, ctypes.c_int, _i64p, _i64p, _i64p,
                                        _i32p, ctypes.c_long, _f32p, ctypes.c_float, _f64p]
        L_, vp = ctypes.c_long, ctypes.c_void_p
        pp = ctypes.POINTER(ctypes.c_void_p)
        lib.orc_lists_eval64x.argtypes = [L_, _f64p, _f64p, L_, _i64p, _i32p, L_, _i64p, _i32p,
                                          pp, pp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                          _f64p]
        lib.orc_fd_hits_x.argtypes = [L_, L_, _i32p, L_, pp, pp, ctypes.c_int, _i64p, _i64p, L_,
                                      vp, vp]
        lib.orc_fd_hits_x.restype = L_
        lib.orc_fd_partial_loss_x.argtypes = [
            ctypes.c_int, L_, L_, _f64p, _f64p, L_, _i64p, _i32p, L_, _i64p, _i32p, _i64p, pp,
            pp, L_, _i64p, np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS"), _f64p, _f64p,
            ctypes.c_double, ctypes.c_double, ctypes.c_int]
        lib.orc_fd_partial_loss_x.restype = ctypes.c_double
        lib.orc_cosmo_integrate.argtypes = [L_, _f32p, _f32p, _f32p, _f64p, ctypes.c_void_p,
                                             ctypes.c_void_p]
        lib.orc_ewald_c0.argtypes = [ctypes.c_double]
        lib.orc_ewald_c0.restype = ctypes.c_double
        lib.orc_direct_grad.argtypes = [L_, _f64p, _f64p, _f64p, _f64p, ctypes.c_double, _f64p,
                                        _f64p]
        _orc = lib
    return _orc


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(REF_SO)
        lib.ref_list_eval.argtypes = [ctypes.c_int, _f32p, ctypes.c_long, ctypes.c_int, _f32p,
                                      ctypes.c_float, _f32p]
        lib.ref_list_eval.restype = ctypes.c_int
        lib.ref_groups_eval.argtypes = [ctypes.c_int, _f32p, ctypes.c_int, _i64p, _i64p, _i64p,
                                        _i32p, ctypes.c_long, _f32p, ctypes.c_float, _f32p,
                                        ctypes.c_int]
        lib.ref_pinteract.argtypes = [ctypes.c_int, _f32p, _f32p, ctypes.c_int, ctypes.c_int,
                                      _f32p, ctypes.c_long]
        lib.ref_segments_k1.argtypes = [_f32p, ctypes.c_int, ctypes.c_float, _u32p, ctypes.c_int,
                                        ctypes.c_long, _f32p, ctypes.c_float, _f32p]
        lib.ref_segments_k1.restype = ctypes.c_long
        lib.ref_ewald_batch.argtypes = [_f64p, ctypes.c_long, ctypes.c_double, _f64p, _f64p]
        if hasattr(lib, "cubic_acc"):
            lib.cubic_acc.argtypes = [_f32p, ctypes.c_float, _f32p]
        if hasattr(lib, "ref_periodic_le"):
            lib.ref_periodic_le.argtypes = [ctypes.c_long, _f32p, _f32p, ctypes.c_double,
                                            ctypes.c_int, ctypes.c_double, _i64p, ctypes.c_long,
                                            _f64p, _f64p]
        _ref = lib
    return _ref


def ref_periodic_le(pos, mass, L, eps2, sinks, nimage=2):
    """The reference's periodic scheme (ref_harness.c ref_periodic_le): the
    direct sum over the (2 nimage + 1)^3 images of the box plus the compiled
    FixCubeEwaldLE far field (nln/ewald_le2.c), for a box of side L centred
    on the origin; (acc (nsink, 3), phi (nsink,)) in FP64, G = 1."""
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    mass = np.ascontiguousarray(mass, np.float32)
    sinks = np.ascontiguousarray(sinks, np.int64)
    acc = np.zeros((len(sinks), 3))
    phi = np.zeros(len(sinks))
    ref().ref_periodic_le(len(mass), pos.ravel(), mass, float(L), int(nimage), float(eps2), sinks,
                          len(sinks), acc.ravel(), phi)
    return acc, phi


def ref_cubic_acc(r, a):
    """The reference's cubic_acc (nln/ewald_le2.c:773-1033, compiled
    unmodified): acceleration at r from the cube of half-side a and unit
    density centred on the origin (float)."""
    rr = np.ascontiguousarray(r, np.float32).reshape(3)
    out = np.zeros(3, np.float32)
    ref().cubic_acc(rr, float(a), out)
    return out


def aligned_f32(n, align=64):
    """A zeroed float32 array whose data pointer is `align`-byte aligned (the
    reference AVX kernels load 32-byte vectors)."""
    buf = np.zeros(n + align // 4, dtype=np.float32)
    off = (-buf.ctypes.data % align) // 4
    return buf[off:off + n]


def pack_aosoa(fields):
    """(nsrc, sz) records -> the reference 8-lane AoSoA layout, zero-padded
    to a multiple of 8 sources (mac.c:606-612 pads with zero-mass lanes)."""
    fields = np.asarray(fields, dtype=np.float32)
    n, sz = fields.shape
    nblk = (n + 7) // 8
    pad = np.zeros((nblk * 8, sz), dtype=np.float32)
    pad[:n] = fields
    out = aligned_f32(nblk * 8 * sz)
    out[:] = pad.reshape(nblk, 8, sz).transpose(0, 2, 1).ravel()
    return out, nblk


def list_eval(kind, f, nblk, pos0, e):
    out = np.zeros(4, dtype=np.float64)
    orc().orc_list_eval(kind, f, nblk, KIND_SZ[kind], np.ascontiguousarray(pos0, np.float32),
                        float(e), out)
    return out


def ref_list_eval(kind, f, nblk, pos0, e):
    out = np.zeros(4, dtype=np.float32)
    ref().ref_list_eval(kind, f, nblk, KIND_SZ[kind], np.ascontiguousarray(pos0, np.float32),
                        float(e), out)
    return out


def direct(pos, mass, eps2, sinks=None):
    """FP64 direct sum (self included, Plummer eps2); returns (acc[nsink,3], phi[nsink])."""
    pos = np.ascontiguousarray(pos, np.float64)
    mass = np.ascontiguousarray(mass, np.float64)
    n = len(mass)
    sinks = np.arange(n, dtype=np.int64) if sinks is None else np.ascontiguousarray(sinks, np.int64)
    acc = np.zeros((len(sinks), 3))
    phi = np.zeros(len(sinks))
    orc().orc_direct(pos, mass, n, float(eps2), sinks, len(sinks), acc, phi)
    return acc, phi


def ewald(x, L):
    x = np.ascontiguousarray(np.atleast_2d(x), np.float64)
    f = np.zeros_like(x)
    phi = np.zeros(len(x))
    orc().orc_ewald_batch(x, len(x), float(L), f, phi)
    return f, phi


def ref_ewald(x, L):
    """ewald() of nln/ewald.c, compiled unmodified into oracle/_ref: (f, phi)
    at displacements x (n, 3) = source - sink."""
    x = np.ascontiguousarray(np.atleast_2d(x), np.float64)
    f = np.zeros_like(x)
    phi = np.zeros(len(x))
    ref().ref_ewald_batch(x, len(x), float(L), f, phi)
    return f, phi


def direct_ewald(pos, mass, L, eps2, sinks):
    pos = np.ascontiguousarray(pos, np.float64)
    mass = np.ascontiguousarray(mass, np.float64)
    sinks = np.ascontiguousarray(sinks, np.int64)
    acc = np.zeros((len(sinks), 3))
    phi = np.zeros(len(sinks))
    orc().orc_direct_ewald(pos, mass, len(mass), float(L), float(eps2), sinks, len(sinks), acc, phi)
    return acc, phi


def tree_eval(tree, eps2, quad_kind=QUAD_PLUMMER_P, hexa_kind=HEXA_PLUMMER, mono_kind=MONO_PLUMMER,
              reference=False):
    """Evaluate a host tree's AoSoA lists (built with emit_aosoa) for every
    sink: (n, 4) (ax, ay, az, phi) in tree order.  reference=True runs the
    compiled reference AVX kernels (FP32) instead of the restatement."""
    n = tree.n
    sf = np.ascontiguousarray(tree.groups["first"]).astype(np.int64)
    sc = np.ascontiguousarray(tree.groups["count"]).astype(np.int32)
    pos = np.ascontiguousarray(tree.sorted_pos.ravel(), np.float32)
    out = np.zeros((n, 4), np.float32 if reference else np.float64)
    if reference and quad_kind == QUAD_PLUMMER_P:
        raise ValueError("the reference quadrupole kernels use the -1 potential sign")
    for k, kind in ((0, mono_kind), (1, quad_kind), (2, hexa_kind)):
        ptr, data = tree.aosoa[k]
        if ptr[-1] == 0:
            continue
        d = aligned_f32(len(data))
        d[:] = data
        bf = np.ascontiguousarray(ptr[:-1])
        bc = np.ascontiguousarray(np.diff(ptr))
        if reference:
            ref().ref_groups_eval(kind, d, KIND_SZ[kind], bf, bc, sf, sc, len(sf), pos, eps2,
                                  out.ravel(), 0 or os.cpu_count())
        else:
            orc().orc_groups_eval(kind, d, KIND_SZ[kind], bf, bc, sf, sc, len(sf), pos, eps2,
                                  out.ravel())
    return out


# ---------------------------------------------------------------- FP64 list checks
class ListsFP64:
    """FP64 evaluation of a walked tree's batched index lists of every kind
    (points, quadrupole and order-4 cells, the periodic correction list,
    image shifts) with every cell's moments recomputed from the bodies
    (orc_lists_eval64x), and central differences of L = sum w.a + u phi
    restricted to the terms that depend on one body (orc_fd_hits_x /
    orc_fd_partial_loss_x): the checker of the hand-written adjoint.
    ewald: apply the correction list (periodic trees that carry one)."""

    def __init__(self, tree, ewald=True):
        self.t = t = tree
        self.n, self.nc, self.ng = int(t.n), int(t.ncells), int(t.ngroups)
        self.box = float(getattr(t, "box", 0.0) or 0.0)
        first, count = t.cell_ranges()
        child, nchild, _ = t.cell_links()
        self.cfirst = np.ascontiguousarray(first, np.int64)
        self.ccount = np.ascontiguousarray(count, np.int32)
        parent = np.full(self.nc, -1, np.int32)
        inner = np.nonzero(child >= 0)[0]
        parent[np.concatenate([np.arange(child[c], child[c] + nchild[c]) for c in inner])
               if len(inner) else np.zeros(0, np.int64)] = np.repeat(inner, nchild[inner])
        self.parent = parent
        leaves = np.nonzero(child < 0)[0]
        leaf = np.full(self.n, -1, np.int64)
        for c in leaves:
            leaf[first[c]:first[c] + count[c]] = c
        self.leaf = leaf
        self.gfirst = np.ascontiguousarray(t.groups["first"], np.int64)
        self.gcount = np.ascontiguousarray(t.groups["count"], np.int32)
        self.bgroup = np.repeat(np.arange(self.ng, dtype=np.int64), self.gcount)
        lists = [t.plist, t.qlist, t.hlist, getattr(t, "clist", np.zeros(0, np.uint32))]
        self._keep = []
        ptrs, datas = [], []
        for k in range(4):
            has = len(lists[k]) > 0 and (k < 3 or (ewald and self.box > 0))
            if has:
                pk = np.ascontiguousarray(t.ptr[k], np.int64)
                lk = np.ascontiguousarray(lists[k], np.uint32)
                self._keep += [pk, lk]
                ptrs.append(pk.ctypes.data)
                datas.append(lk.ctypes.data)
            else:
                ptrs.append(None)
                datas.append(None)
        self.ewald = int(ptrs[3] is not None)
        self.ptrs = (ctypes.c_void_p * 4)(*ptrs)
        self.lists = (ctypes.c_void_p * 4)(*datas)

    def eval(self, x, m, eps2):
        """(n, 4) FP64 (ax, ay, az, phi), tree order, positions x (n, 3) and masses m."""
        x = np.ascontiguousarray(x, np.float64)
        m = np.ascontiguousarray(m, np.float64)
        out = np.zeros((self.n, 4))
        orc().orc_lists_eval64x(self.n, x.ravel(), m, self.nc, self.cfirst, self.ccount, self.ng,
                                self.gfirst, self.gcount, self.ptrs, self.lists, float(eps2),
                                self.box, self.ewald, out.ravel())
        return out

    def select(self, bodies):
        """Prepare central differences for up to 64 bodies (tree order)."""
        self.sel = np.ascontiguousarray(bodies, np.int64)
        args = (self.n, self.nc, self.parent, self.ng, self.ptrs, self.lists, len(self.sel),
                self.sel, self.leaf)
        nh = orc().orc_fd_hits_x(*args, 0, None, None)
        if nh < 0:
            raise ValueError("at most 64 selected bodies")
        self.hits = np.zeros(3 * max(nh, 1), np.int64)
        self.hmask = np.zeros(max(nh, 1), np.uint64)
        orc().orc_fd_hits_x(*args, nh, self.hits.ctypes.data, self.hmask.ctypes.data)
        self.nhits = nh

    def partial_loss(self, s, x, m, w, u, eps2):
        """The part of L that depends on selected body s (index into select()'s list)."""
        return orc().orc_fd_partial_loss_x(
            int(s), int(self.sel[s]), self.n, np.ascontiguousarray(x, np.float64).ravel(),
            np.ascontiguousarray(m, np.float64), self.nc, self.cfirst, self.ccount, self.ng,
            self.gfirst, self.gcount, self.bgroup, self.ptrs, self.lists, self.nhits, self.hits,
            self.hmask, np.ascontiguousarray(w, np.float64).ravel(),
            np.ascontiguousarray(u, np.float64), float(eps2), self.box, self.ewald)

    def fd_grad(self, x, m, w, u, eps2, coords, h=1e-6, mass_rel=False):
        """Central differences of L for (selected body s, component c) pairs;
        c = 3 means the mass (relative step h m when mass_rel)."""
        x = np.array(x, np.float64)
        m = np.array(m, np.float64)
        out = []
        for s, c in coords:
            j = int(self.sel[s])
            if c < 3:
                x0 = x[j, c]
                x[j, c] = x0 + h
                lp = self.partial_loss(s, x, m, w, u, eps2)
                x[j, c] = x0 - h
                lm = self.partial_loss(s, x, m, w, u, eps2)
                x[j, c] = x0
                out.append((lp - lm) / (2 * h))
            else:
                m0 = m[j]
                hh = h * m0 if mass_rel else h
                m[j] = m0 + hh
                lp = self.partial_loss(s, x, m, w, u, eps2)
                m[j] = m0 - hh
                lm = self.partial_loss(s, x, m, w, u, eps2)
                m[j] = m0
                out.append((lp - lm) / (2 * hh))
        return np.array(out)


def cosmo_integrate(pos4, vel4, acc4, factors):
    """CosmoIntegrate (orc_cosmo_integrate) on copies of float32 (n, 4)
    arrays: returns (pos4, vel4, ke, pe)."""
    pos = np.ascontiguousarray(pos4, np.float32).copy()
    vel = np.ascontiguousarray(vel4, np.float32).copy()
    acc = np.ascontiguousarray(acc4, np.float32)
    ke, pe = ctypes.c_double(), ctypes.c_double()
    orc().orc_cosmo_integrate(len(pos), pos.ravel(), vel.ravel(), acc.ravel(),
                              np.ascontiguousarray(factors, np.float64), ctypes.byref(ke),
                              ctypes.byref(pe))
    return pos, vel, ke.value, pe.value


def ewald_c0(L):
    """C(0) = lim Phi(y) + 1/|y| of the Ewald sum in a cube of side L."""
    return orc().orc_ewald_c0(float(L))


def direct_grad(x, m, w, u, eps2):
    """FP64 dL/dx (n, 3) and dL/dm (n,) of L = sum w.a + u phi for the
    Plummer-softened direct sum (orc_direct_grad)."""
    x = np.ascontiguousarray(x, np.float64)
    m = np.ascontiguousarray(m, np.float64)
    gx = np.zeros_like(x)
    gm = np.zeros(len(m))
    orc().orc_direct_grad(len(m), x.ravel(), m, np.ascontiguousarray(w, np.float64).ravel(),
                          np.ascontiguousarray(u, np.float64), float(eps2), gx.ravel(), gm)
    return gx, gm
