"""ctypes binding of libnlnhost.so (include/nlnhost.h): the host tree build,
FP64 moments, AREL critical radii, group MAC walk and list packing."""
import ctypes
import os

import numpy as np

from . import _build

_lib = None

QCELL_DTYPE = np.dtype([("cen", "<f8", 3), ("mass", "<f4"), ("R", "<f4"), ("q2", "<f4", 5),
                        ("B2", "<f4"), ("pad", "<f4", 2)])
HCELL_DTYPE = np.dtype([("cen", "<f8", 3), ("mass", "<f4"), ("R", "<f4"), ("q2", "<f4", 5),
                        ("q3", "<f4", 7), ("q4", "<f4", 9), ("B2", "<f4"), ("pad", "<f4", 2)])
GROUP_DTYPE = np.dtype([("cen", "<f8", 3), ("first", "<i8"), ("count", "<i4"), ("radius", "<f4")])
assert QCELL_DTYPE.itemsize == 64 and HCELL_DTYPE.itemsize == 128
assert GROUP_DTYPE.itemsize == 40

SHIFT_NONE = 13
IDX_BITS = 27
IDX_MASK = (1 << IDX_BITS) - 1


class Params(ctypes.Structure):
    _fields_ = [("leaf_max", ctypes.c_int), ("group_max", ctypes.c_int),
                ("p2cut", ctypes.c_int), ("p4cut", ctypes.c_int),
                ("tol", ctypes.c_double), ("rel_tol", ctypes.c_double),
                ("rel_tol0", ctypes.c_double), ("box", ctypes.c_double),
                ("nthreads", ctypes.c_int), ("emit_aosoa", ctypes.c_int),
                ("ewald_theta", ctypes.c_double), ("ptol_boost", ctypes.c_double)]


def lib():
    global _lib
    if _lib is None:
        path = _build.HOST_SO
        if not os.path.exists(path):
            _build.build_host()
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.nln_tree_build.argtypes = [vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int64,
                                     ctypes.POINTER(Params)]
        L.nln_tree_build.restype = vp
        L.nln_tree_free.argtypes = [vp]
        L.nln_last_error.restype = ctypes.c_char_p
        L.nln_tree_walk.argtypes = [vp]
        L.nln_tree_walk.restype = ctypes.c_int
        for name in ("nln_nbodies", "nln_ncells", "nln_ngroups"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = ctypes.c_int64
        for name in ("nln_order", "nln_points", "nln_qcells", "nln_hcells", "nln_groups",
                     "nln_sorted_pos"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = vp
        for name in ("nln_list_ptr", "nln_list_data", "nln_aosoa_ptr", "nln_aosoa_data"):
            getattr(L, name).argtypes = [vp, ctypes.c_int]
            getattr(L, name).restype = vp
        L.nln_list_len.argtypes = [vp, ctypes.c_int]
        L.nln_list_len.restype = ctypes.c_int64
        L.nln_counts.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.nln_aosoa_subset.argtypes = [vp, vp, ctypes.c_int64, ctypes.c_int, vp, vp]
        L.nln_aosoa_subset.restype = ctypes.c_int64
        L.nln_cell_ranges.argtypes = [vp, vp, vp]
        L.nln_cell_links.argtypes = [vp, vp, vp, vp]
        L.nln_tree_refit.argtypes = [vp, vp]
        L.nln_tree_merge.argtypes = [vp, ctypes.c_int]
        L.nln_tree_merge.restype = vp
        L.nln_tree_refit.restype = ctypes.c_int
        L.nln_tree_pack.argtypes = [vp]
        L.nln_tree_pack.restype = ctypes.c_int
        for name in ("nln_packed_ptr", "nln_packed_data"):
            getattr(L, name).argtypes = [vp, ctypes.c_int]
            getattr(L, name).restype = vp
        L.nln_packed_len.argtypes = [vp, ctypes.c_int]
        L.nln_packed_len.restype = ctypes.c_int64
        _lib = L
    return _lib


class _Handle:
    """Owns one nln_tree; freed when the last array viewing its memory goes."""

    def __init__(self, h):
        self.h = h

    def __del__(self):
        try:
            if self.h:
                lib().nln_tree_free(self.h)
                self.h = None
        except Exception:
            pass


def cubic_acc(r, a):
    """Acceleration at r (3,) from the uniform cube of half-side a and unit
    density centred on the origin, G = 1 (nln_cubic_acc): the near-zone field
    a background-subtracting walk adds back per sink, scaled by -rho0."""
    rr = (ctypes.c_double * 3)(*[float(v) for v in np.asarray(r, np.float64).reshape(3)])
    out = (ctypes.c_double * 3)()
    lib().nln_cubic_acc(rr, ctypes.c_double(float(a)), out)
    return np.array(out[:])


def _view(ptr, dtype, count, owner=None):
    """A zero-copy array over library memory; the buffer keeps `owner` (the
    tree's handle) alive as long as the array exists."""
    if count == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    dt = np.dtype(dtype)
    buf = (ctypes.c_char * (dt.itemsize * count)).from_address(ptr)
    buf._owner = owner
    return np.frombuffer(buf, dtype=dt, count=count)


class Tree:
    """An oct-tree with its sink groups and interaction lists.

    Bodies are stored in key (tree) order; ``order[i]`` is the original
    index of tree body ``i``.  Lists are index lists into ``points`` (float4
    bodies then cell monopoles), ``qcells`` and ``hcells``.  Periodic trees
    (box > 0) also carry ``clist``/``ptr[3]``, the Ewald correction list:
    ``ewald_theta`` is its opening angle (a cell wholly inside a group's
    minimum-image cube stands for its subtree once bmax + group radius <=
    ewald_theta x its distance to the group's nearest lattice image; 0 makes
    the list repeat the Newtonian entries).
    """

    def __init__(self, pos, mass, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-3,
                 rel_tol=0.0, rel_tol0=0.0, box=0.0, nthreads=0, emit_aosoa=False, walk=True,
                 ewald_theta=0.2, ptol_boost=0.0):
        pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        mass = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, np.float32), (len(pos),)))
        self.params = Params(leaf_max, group_max, p2cut, p4cut, tol, rel_tol, rel_tol0, box,
                             nthreads, int(bool(emit_aosoa)), ewald_theta, ptol_boost)
        L = lib()
        h = L.nln_tree_build(pos.ctypes.data, 3, mass.ctypes.data, 1, len(pos),
                             ctypes.byref(self.params))
        if not h:
            raise ValueError(L.nln_last_error().decode())
        self._attach(h, box)
        if walk:
            self.walk()

    def _attach(self, h, box):
        L = lib()
        self._h = h
        self._owner = _Handle(h)
        self.n = L.nln_nbodies(h)
        self.ncells = L.nln_ncells(h)
        self.box = float(box)
        self.order = _view(L.nln_order(h), np.int64, self.n, self._owner)
        self.sorted_pos = _view(L.nln_sorted_pos(h), np.float32, 3 * self.n, self._owner).reshape(-1, 3)
        self.points = _view(L.nln_points(h), np.float32, 4 * (self.n + self.ncells), self._owner).reshape(-1, 4)
        self.qcells = _view(L.nln_qcells(h), QCELL_DTYPE, self.ncells, self._owner)
        self.hcells = _view(L.nln_hcells(h), HCELL_DTYPE, self.ncells, self._owner)
        self.ngroups = L.nln_ngroups(h)
        self.groups = _view(L.nln_groups(h), GROUP_DTYPE, self.ngroups, self._owner)

    @classmethod
    def merge(cls, trees):
        """A batch of independent isolated trees as one (nln_tree_merge): the
        members' bodies one after another, then their cells; lists renumbered
        so each still refers only to its own member."""
        L = lib()
        hs = (ctypes.c_void_p * len(trees))(*[t._h for t in trees])
        h = L.nln_tree_merge(hs, len(trees))
        if not h:
            raise ValueError(L.nln_last_error().decode())
        self = cls.__new__(cls)
        self.params = trees[0].params
        self._merged = True
        self._attach(h, 0.0)
        self._views()
        self.body_offsets = np.concatenate([[0], np.cumsum([t.n for t in trees])])
        return self

    def walk(self):
        L = lib()
        if L.nln_tree_walk(self._h) != 0:
            raise RuntimeError("walk failed")
        self._views()

    def _views(self):
        L = lib()
        ng = self.ngroups
        self.ptr = [_view(L.nln_list_ptr(self._h, k), np.int64, ng + 1, self._owner) for k in range(4)]
        self.plist = _view(L.nln_list_data(self._h, 0), np.uint32, L.nln_list_len(self._h, 0), self._owner)
        self.qlist = _view(L.nln_list_data(self._h, 1), np.uint32, L.nln_list_len(self._h, 1), self._owner)
        self.hlist = _view(L.nln_list_data(self._h, 2), np.uint32, L.nln_list_len(self._h, 2), self._owner)
        # periodic correction list (bodies and cells as n + cell index); empty when isolated
        self.clist = _view(L.nln_list_data(self._h, 3), np.uint32, L.nln_list_len(self._h, 3), self._owner)
        c = (ctypes.c_int64 * 4)()
        L.nln_counts(self._h, c)
        self.counts = np.array(list(c), dtype=np.int64)
        self.aosoa = None
        if self.params.emit_aosoa and not getattr(self, "_merged", False):
            self.aosoa = []
            for k, sz in enumerate((4, 13, 29)):
                ptr = _view(L.nln_aosoa_ptr(self._h, k), np.int64, ng + 1, self._owner)
                data = _view(L.nln_aosoa_data(self._h, k), np.float32, int(ptr[-1]) * sz * 8, self._owner)
                self.aosoa.append((ptr, data))

    def pack(self):
        """Run-pack the lists (nln_tree_pack; format in nlnlists.h).  Sets
        zptr[k] (ngroups + 1 word offsets) and zlist[k] (the words) for
        k = 0 P, 1 Q, 2 H, 3 correction (empty arrays for a kind without
        lists) and returns self."""
        L = lib()
        if L.nln_tree_pack(self._h) != 0:
            raise RuntimeError(L.nln_last_error().decode())
        ng = self.ngroups
        self.zptr, self.zlist = [], []
        for k in range(4):
            n = L.nln_packed_len(self._h, k)
            if n < 0:
                self.zptr.append(np.zeros(0, np.int64))
                self.zlist.append(np.zeros(0, np.uint32))
                continue
            self.zptr.append(_view(L.nln_packed_ptr(self._h, k), np.int64, ng + 1, self._owner))
            self.zlist.append(_view(L.nln_packed_data(self._h, k), np.uint32, n, self._owner))
        return self

    def cell_ranges(self):
        """(first, count) body range of every cell, tree order."""
        first = np.zeros(self.ncells, np.int64)
        count = np.zeros(self.ncells, np.int32)
        lib().nln_cell_ranges(self._h, first.ctypes.data, count.ctypes.data)
        return first, count

    def cell_links(self):
        """(child, nchild, level) of every cell: first child (-1 for a leaf),
        child count (children are consecutive) and depth (root 0)."""
        child = np.zeros(self.ncells, np.int32)
        nchild = np.zeros(self.ncells, np.int32)
        level = np.zeros(self.ncells, np.int32)
        lib().nln_cell_links(self._h, child.ctypes.data, nchild.ctypes.data, level.ctypes.data)
        return child, nchild, level

    def refit(self, pos_tree_order):
        """Recompute every cell's moments (and the point, quadrupole and
        order-4 tables, in place) for new body positions in tree order; the
        tree, the critical radii and the lists are kept."""
        p = np.ascontiguousarray(pos_tree_order, np.float32).reshape(-1, 3)
        if len(p) != self.n:
            raise ValueError("refit needs one position per body")
        if lib().nln_tree_refit(self._h, p.ctypes.data) != 0:
            raise RuntimeError("refit failed")

    def aosoa_subset(self, gids, kind):
        """Reference AoSoA blocks (kind 0 = M, 1 = Q, 2 = H) for groups gids:
        (blk_ptr[len(gids)+1], data) with data 64-byte aligned."""
        sz = (4, 13, 29)[kind]
        gids = np.ascontiguousarray(gids, np.int64)
        ptr = np.zeros(len(gids) + 1, np.int64)
        L = lib()
        nblk = L.nln_aosoa_subset(self._h, gids.ctypes.data, len(gids), kind, ptr.ctypes.data, None)
        if nblk < 0:
            raise ValueError("no lists of that kind")
        buf = np.zeros(nblk * sz * 8 + 16, np.float32)
        off = (-buf.ctypes.data % 64) // 4
        data = buf[off:off + nblk * sz * 8]
        L.nln_aosoa_subset(self._h, gids.ctypes.data, len(gids), kind, ptr.ctypes.data,
                           data.ctypes.data)
        return ptr, data

    @property
    def interactions(self):
        """Sink-source interactions by type: body-body, monopole, quadrupole, order-4."""
        return self.counts

    def close(self):
        """Drop this object's reference; the library memory is freed once no
        array viewing it remains."""
        self._owner = None
