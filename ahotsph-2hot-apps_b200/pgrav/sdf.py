"""Snapshots and checkpoints in the reference's SDF format (nlnhost.h
nln_sdf_*): outbody records (mass, x y z, vx vy vz, optionally ax ay az
phi, int64 ident; nln/physics.h:49-110) behind an ASCII header of scalar
declarations (nln/output.c:217-330)."""
import ctypes

import numpy as np

from . import host

INT, INT64, FLOAT, DOUBLE = 0, 1, 2, 3
_TYPES = {int: INT64, float: DOUBLE}
_ready = False


def _lib():
    global _ready
    L = host.lib()
    if not _ready:
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        L.nln_sdf_write.argtypes = [ctypes.c_char_p, i64, vp, vp, vp, vp, vp, ctypes.c_int, vp,
                                    vp, vp]
        L.nln_sdf_write.restype = ctypes.c_int
        L.nln_sdf_read.argtypes = [ctypes.c_char_p]
        L.nln_sdf_read.restype = vp
        L.nln_sdf_count.argtypes = [vp]
        L.nln_sdf_count.restype = i64
        L.nln_sdf_has_acc.argtypes = [vp]
        L.nln_sdf_has_acc.restype = ctypes.c_int
        L.nln_sdf_nkeys.argtypes = [vp]
        L.nln_sdf_nkeys.restype = ctypes.c_int
        L.nln_sdf_key.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_double)]
        L.nln_sdf_key.restype = ctypes.c_char_p
        L.nln_sdf_bodies.argtypes = [vp, vp, vp, vp, vp, vp]
        L.nln_sdf_bodies.restype = ctypes.c_int
        L.nln_sdf_free.argtypes = [vp]
        L.nln_sdf_error.restype = ctypes.c_char_p
        _ready = True
    return L


def write(path, pos, vel, mass, ident=None, acc_phi=None, header=None):
    """Write bodies (n, 3) positions and velocities, (n,) masses, optional
    int64 idents (default 0..n-1) and (n, 4) (ax, ay, az, phi) to an SDF file.
    header: {key: value} or {key: (type, value)} with type INT, INT64, FLOAT,
    DOUBLE (Python ints are written as int64_t, floats as double)."""
    L = _lib()
    pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    n = len(pos)
    vel = np.ascontiguousarray(vel, np.float32).reshape(n, 3)
    mass = np.ascontiguousarray(np.broadcast_to(np.asarray(mass, np.float32), (n,)))
    ident = np.arange(n, dtype=np.int64) if ident is None else np.ascontiguousarray(ident, np.int64)
    ap = None if acc_phi is None else np.ascontiguousarray(acc_phi, np.float32).reshape(n, 4)
    keys, types, values = [], [], []
    for k, v in (header or {}).items():
        t, val = v if isinstance(v, tuple) else (_TYPES[type(v)], v)
        keys.append(k.encode())
        types.append(t)
        values.append(float(val))
    kk = (ctypes.c_char_p * max(1, len(keys)))(*keys)
    tt = np.asarray(types or [0], np.int32)
    vv = np.asarray(values or [0.0], np.float64)
    rc = L.nln_sdf_write(str(path).encode(), n, mass.ctypes.data, pos.ctypes.data, vel.ctypes.data,
                         None if ap is None else ap.ctypes.data, ident.ctypes.data, len(keys), kk,
                         tt.ctypes.data, vv.ctypes.data)
    if rc != 0:
        raise IOError(L.nln_sdf_error().decode())


def read(path):
    """(header, bodies): header {key: value} (ints for int types), bodies a
    dict of pos (n, 3), vel (n, 3), mass (n,), ident (n,) and, when the file
    has them, acc_phi (n, 4)."""
    L = _lib()
    h = L.nln_sdf_read(str(path).encode())
    if not h:
        raise IOError(L.nln_sdf_error().decode())
    try:
        n = L.nln_sdf_count(h)
        header = {}
        for k in range(L.nln_sdf_nkeys(h)):
            t, v = ctypes.c_int(), ctypes.c_double()
            name = L.nln_sdf_key(h, k, ctypes.byref(t), ctypes.byref(v)).decode()
            header[name] = int(v.value) if t.value in (INT, INT64) else v.value
        out = {"pos": np.empty((n, 3), np.float32), "vel": np.empty((n, 3), np.float32),
               "mass": np.empty(n, np.float32), "ident": np.empty(n, np.int64)}
        acc = np.empty((n, 4), np.float32) if L.nln_sdf_has_acc(h) else None
        L.nln_sdf_bodies(h, out["mass"].ctypes.data, out["pos"].ctypes.data,
                         out["vel"].ctypes.data, None if acc is None else acc.ctypes.data,
                         out["ident"].ctypes.data)
        if acc is not None:
            out["acc_phi"] = acc
        return header, out
    finally:
        L.nln_sdf_free(h)
