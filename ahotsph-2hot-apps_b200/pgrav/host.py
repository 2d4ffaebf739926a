"""ctypes binding of libnlnhost.so (include/nlnhost.h): the host tree build,
FP64 moments, AREL critical radii, group MAC walk and list packing."""
import ctypes
import os

import numpy as np

from . import _build

_lib = None

QCELL_DTYPE = np.dtype([("cen", "<f8", 3), ("mass", "<f4"), ("R", "<f4"), ("q2", "<f4", 5),
                        ("pad", "<f4", 3)])
HCELL_DTYPE = np.dtype([("cen", "<f8", 3), ("mass", "<f4"), ("R", "<f4"), ("q2", "<f4", 5),
                        ("q3", "<f4", 7), ("q4", "<f4", 9), ("pad", "<f4", 3)])
PSEG_DTYPE = np.dtype([("base", "<u4"), ("len", "<u2"), ("shift", "<u2")])
GROUP_DTYPE = np.dtype([("cen", "<f8", 3), ("first", "<i8"), ("count", "<i4"), ("radius", "<f4")])
assert QCELL_DTYPE.itemsize == 64 and HCELL_DTYPE.itemsize == 128
assert PSEG_DTYPE.itemsize == 8 and GROUP_DTYPE.itemsize == 40

SHIFT_NONE = 13
IDX_BITS = 27
IDX_MASK = (1 << IDX_BITS) - 1


class Params(ctypes.Structure):
    _fields_ = [("leaf_max", ctypes.c_int), ("group_max", ctypes.c_int),
                ("p2cut", ctypes.c_int), ("p4cut", ctypes.c_int),
                ("tol", ctypes.c_double), ("rel_tol", ctypes.c_double),
                ("rel_tol0", ctypes.c_double), ("box", ctypes.c_double),
                ("nthreads", ctypes.c_int), ("emit_aosoa", ctypes.c_int)]


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
        _lib = L
    return _lib


def _view(ptr, dtype, count):
    if count == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    dt = np.dtype(dtype)
    buf = (ctypes.c_char * (dt.itemsize * count)).from_address(ptr)
    return np.frombuffer(buf, dtype=dt, count=count).copy()


class Tree:
    """An oct-tree with its sink groups and interaction lists.

    Bodies are stored in key (tree) order; ``order[i]`` is the original
    index of tree body ``i``.  Lists are index lists into ``points`` (float4
    bodies then cell monopoles), ``qcells`` and ``hcells``.
    """

    def __init__(self, pos, mass, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-3,
                 rel_tol=0.0, rel_tol0=0.0, box=0.0, nthreads=0, emit_aosoa=False, walk=True):
        pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        mass = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, np.float32), (len(pos),)))
        self.params = Params(leaf_max, group_max, p2cut, p4cut, tol, rel_tol, rel_tol0, box,
                             nthreads, int(bool(emit_aosoa)))
        L = lib()
        h = L.nln_tree_build(pos.ctypes.data, 3, mass.ctypes.data, 1, len(pos),
                             ctypes.byref(self.params))
        if not h:
            raise ValueError(L.nln_last_error().decode())
        self._h = h
        self.n = L.nln_nbodies(h)
        self.ncells = L.nln_ncells(h)
        self.box = float(box)
        self.order = _view(L.nln_order(h), np.int64, self.n)
        self.sorted_pos = _view(L.nln_sorted_pos(h), np.float32, 3 * self.n).reshape(-1, 3)
        self.points = _view(L.nln_points(h), np.float32, 4 * (self.n + self.ncells)).reshape(-1, 4)
        self.qcells = _view(L.nln_qcells(h), QCELL_DTYPE, self.ncells)
        self.hcells = _view(L.nln_hcells(h), HCELL_DTYPE, self.ncells)
        self.ngroups = L.nln_ngroups(h)
        self.groups = _view(L.nln_groups(h), GROUP_DTYPE, self.ngroups)
        if walk:
            self.walk()

    def walk(self):
        L = lib()
        if L.nln_tree_walk(self._h) != 0:
            raise RuntimeError("walk failed")
        ng = self.ngroups
        self.ptr = [_view(L.nln_list_ptr(self._h, k), np.int64, ng + 1) for k in range(3)]
        self.plist = _view(L.nln_list_data(self._h, 0), PSEG_DTYPE, L.nln_list_len(self._h, 0))
        self.qlist = _view(L.nln_list_data(self._h, 1), np.uint32, L.nln_list_len(self._h, 1))
        self.hlist = _view(L.nln_list_data(self._h, 2), np.uint32, L.nln_list_len(self._h, 2))
        c = (ctypes.c_int64 * 4)()
        L.nln_counts(self._h, c)
        self.counts = np.array(list(c), dtype=np.int64)
        self.aosoa = None
        if self.params.emit_aosoa:
            self.aosoa = []
            for k, sz in enumerate((4, 13, 29)):
                ptr = _view(L.nln_aosoa_ptr(self._h, k), np.int64, ng + 1)
                data = _view(L.nln_aosoa_data(self._h, k), np.float32, int(ptr[-1]) * sz * 8)
                self.aosoa.append((ptr, data))

    @property
    def interactions(self):
        """Sink-source interactions by type: body-body, monopole, quadrupole, order-4."""
        return self.counts

    def close(self):
        if getattr(self, "_h", None):
            lib().nln_tree_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
