"""ctypes binding of libgravcuda.so (include/gravcuda.h).

The library is the product's only compute path: nothing here falls back to
the CPU.  Loading it on a machine without a GPU works (tests check the
exported symbols there); calling a compute entry point needs a CUDA device.
"""
import ctypes
import os

import numpy as np

from . import _build
from .host import GROUP_DTYPE, HCELL_DTYPE, QCELL_DTYPE  # noqa: F401

_lib = None

# every entry point declared in include/gravcuda.h
EXPORTS = [
    "CUDA_Init", "CUDA_Finalize", "vecwidthCUDA", "qallocCUDA", "WalkInitSrcCUDA",
    "WalkTerminateSrcCUDA", "WalkInitSinkCUDA", "WalkTerminateSinkCUDA", "grav_mn_CUDA",
    "grav_mns_CUDA", "grav_mnss_CUDA", "grav_qns_CUDA", "grav_qnss_CUDA",
    "gravcuda_set_error_mode", "gravcuda_status", "gravcuda_status_string",
    "gravcuda_clear_status", "grav_mn_status_CUDA", "gravcuda_peek_accumulators",
    "grav_groups_upload_CUDA", "grav_groups_eval_CUDA", "grav_groups_download_CUDA",
    "grav_plan_output", "grav_plan_counts", "grav_plan_launches", "grav_plan_free",
    "grav_groups_CUDA", "grav_direct_fp64_CUDA", "grav_plan_set_timing", "grav_plan_kernel_ms",
    "grav_groups_eval_dev_CUDA", "grav_plan_set_tree_CUDA", "grav_plan_refit_CUDA",
    "grav_plan_bodies", "grav_plan_integrate_CUDA", "grav_plan_step_CUDA",
    "grav_plan_set_integrator_CUDA", "gravcuda_dropin_phases",
    "grav_plan_adjoint_CUDA", "grav_plan_retune_CUDA", "grav_plan_get_tuning",
    "grav_groups_CUDA_phases", "grav_groups_release_CUDA", "grav_fp32_peak_CUDA",
    "grav_plan_build_CUDA", "grav_plan_order", "grav_plan_build_phases", "grav_plan_problem",
    "grav_build_eval_CUDA", "grav_build_eval_phases",
]


class GravError(RuntimeError):
    pass


class Segment(ctypes.Structure):
    _fields_ = [("base", ctypes.c_uint), ("length", ctypes.c_uint)]


class Problem(ctypes.Structure):
    _fields_ = [("nbodies", ctypes.c_int64), ("ncells", ctypes.c_int64),
                ("ngroups", ctypes.c_int64), ("points", ctypes.c_void_p),
                ("qcells", ctypes.c_void_p), ("hcells", ctypes.c_void_p),
                ("groups", ctypes.c_void_p), ("pptr", ctypes.c_void_p),
                ("qptr", ctypes.c_void_p), ("hptr", ctypes.c_void_p),
                ("plist", ctypes.c_void_p), ("qlist", ctypes.c_void_p),
                ("hlist", ctypes.c_void_p), ("eps2", ctypes.c_double), ("box", ctypes.c_double),
                ("quad_phi_sign", ctypes.c_float), ("ewald", ctypes.c_int),
                ("cptr", ctypes.c_void_p), ("clist", ctypes.c_void_p),
                ("lists_in_host", ctypes.c_int),
                ("zptr", ctypes.c_void_p * 4), ("zlist", ctypes.c_void_p * 4),
                ("precision", ctypes.c_int)]


class Tuning(ctypes.Structure):
    _fields_ = [("warps_per_block", ctypes.c_int), ("chunk_p", ctypes.c_int),
                ("chunk_q", ctypes.c_int), ("chunk_h", ctypes.c_int),
                ("blocks_per_sm", ctypes.c_int), ("ewald_n", ctypes.c_int),
                ("ewald_side", ctypes.c_int)]


def lib(record_errors=True):
    """Load libgravcuda.so (building it when absent).  With record_errors the
    library returns error codes instead of aborting (gravcuda_set_error_mode(1))."""
    global _lib
    if _lib is None:
        path = _build.CUDA_SO
        if not os.path.exists(path):
            _build.build_cuda()
        L = ctypes.CDLL(path)
        vp, i32, i64, f32, f64 = (ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float,
                                  ctypes.c_double)
        cs = ctypes.c_char_p
        sig = {
            "CUDA_Init": ([vp], None), "CUDA_Finalize": ([], None), "vecwidthCUDA": ([], i32),
            "qallocCUDA": ([vp], i32), "WalkInitSrcCUDA": ([vp, i32, i64], None),
            "WalkTerminateSrcCUDA": ([], None), "WalkInitSinkCUDA": ([vp, i32, i64], None),
            "WalkTerminateSinkCUDA": ([vp, i32, i64], None),
            "grav_mn_CUDA": ([cs, vp, vp, i32, i32, vp, i32, i32, f32, vp, i32], None),
            "grav_mns_CUDA": ([cs, i32, i32, vp, i32, i32, f32, f32, vp, i32], None),
            "grav_mnss_CUDA": ([cs, i32, i32, vp, vp, i32, vp, i32, i32, vp, f32, f32, vp, i32],
                               None),
            "grav_qns_CUDA": ([cs, i32, i32, vp, i32, i32], None),
            "grav_qnss_CUDA": ([cs, i32, i32, vp, vp, i32, i32], None),
            "gravcuda_set_error_mode": ([i32], None), "gravcuda_status": ([], i32),
            "gravcuda_status_string": ([], cs), "gravcuda_clear_status": ([], None),
            "grav_mn_status_CUDA": ([cs, vp, i32, i32, vp, i32, i32, f32, i32], i32),
            "gravcuda_peek_accumulators": ([vp, i64, i64], i32),
            "grav_groups_upload_CUDA": ([vp, vp, vp], i32),
            "grav_groups_eval_CUDA": ([vp, vp], i32),
            "grav_groups_download_CUDA": ([vp, vp], i32),
            "grav_plan_output": ([vp], vp), "grav_plan_counts": ([vp, vp], None),
            "grav_plan_launches": ([vp], i32), "grav_plan_free": ([vp], None),
            "grav_groups_CUDA": ([vp, vp], i32), "grav_groups_CUDA_phases": ([vp], None),
            "grav_groups_release_CUDA": ([], None),
            "grav_direct_fp64_CUDA": ([vp, i64, vp, i64, f64, f64, vp], i32),
            "grav_plan_set_timing": ([vp, i32], i32), "grav_plan_kernel_ms": ([vp, vp], i32),
            "grav_groups_eval_dev_CUDA": ([vp, vp, vp], i32),
            "grav_plan_set_tree_CUDA": ([vp, vp, vp, vp, vp, vp], i32),
            "grav_plan_refit_CUDA": ([vp, vp], i32), "grav_plan_bodies": ([vp], vp),
            "grav_plan_integrate_CUDA": ([vp, vp, vp, vp, vp], i32),
            "grav_plan_set_integrator_CUDA": ([vp, i32], i32),
            "gravcuda_dropin_phases": ([vp], None),
            "grav_plan_step_CUDA": ([vp, vp, vp, vp, vp, i32], i32),
            "grav_plan_adjoint_CUDA": ([vp, vp, vp, vp], i32),
            "grav_plan_retune_CUDA": ([vp, vp], i32), "grav_plan_get_tuning": ([vp, vp], i32),
            "grav_fp32_peak_CUDA": ([vp], i32),
            "grav_plan_build_CUDA": ([vp, vp, i64, f64, f32, i32, vp, vp], i32),
            "grav_plan_order": ([vp], vp), "grav_plan_build_phases": ([vp], None),
            "grav_plan_problem": ([vp, vp], i32),
            "grav_build_eval_CUDA": ([vp, vp, i64, f64, f32, i32, vp], i32),
            "grav_build_eval_phases": ([vp], None),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    if record_errors:
        _lib.gravcuda_set_error_mode(1)
    return _lib


def check(rc=None):
    """Raise GravError when the library recorded an error."""
    L = lib()
    st = L.gravcuda_status() if rc is None else rc
    if st:
        msg = L.gravcuda_status_string().decode()
        L.gravcuda_clear_status()
        raise GravError(f"gravcuda status {st}: {msg}")


def _p(a):
    return None if a is None else a.ctypes.data


def d2h(ptr, dtype, count):
    """A host copy of `count` items of `dtype` at device pointer `ptr`."""
    from cuda.bindings import runtime as rt
    out = np.empty(count, dtype=dtype)
    if count:
        err, = rt.cudaMemcpy(out.ctypes.data, ptr, out.nbytes,
                             rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        if int(err) != 0:
            raise GravError(f"cudaMemcpy D2H failed: {err}")
    return out


def _host_array(ptr, dtype, count):
    if not ptr or count == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array((ctypes.c_char * (np.dtype(dtype).itemsize * count)).from_address(
        ptr)).view(dtype).copy()


class Plan:
    """A device-resident batched problem (grav_groups_upload_CUDA, or built on
    the GPU by Plan.build)."""

    @classmethod
    def build(cls, pos, mass, eps2, box=0.0, ewald=False, quad_phi_sign=1.0, tuning=None,
              leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-3, rel_tol=0.0, rel_tol0=0.0,
              ewald_theta=0.2, ptol_boost=0.0, bodies=None):
        """The tree, moments, critical radii, sink groups and lists built on
        the GPU (grav_plan_build_CUDA) from positions (n, 3) and masses (n,),
        or from `bodies`, a CUDA float32 tensor (n, 4) of (x, y, z, m); the
        parameters are host.Tree's, and the result is bit-identical to a plan
        uploaded from host.Tree on the same bodies.  Results come in tree
        order: plan.order() maps tree positions to input indices."""
        import torch
        from .host import Params
        if bodies is None:
            pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
            n = len(pos)
            b = np.empty((n, 4), np.float32)
            b[:, :3] = pos
            b[:, 3] = np.broadcast_to(np.asarray(mass, np.float32), (n,))
            bodies = torch.from_numpy(b).cuda()
        n = int(bodies.shape[0])
        params = Params(leaf_max, group_max, p2cut, p4cut, tol, rel_tol, rel_tol0, float(box), 0, 0,
                        ewald_theta, ptol_boost)
        tun = None
        if tuning is not None:
            tun = Tuning(*tuning) if not isinstance(tuning, Tuning) else tuning
        h = ctypes.c_void_p()
        check(lib().grav_plan_build_CUDA(ctypes.byref(params), bodies.data_ptr(), n, float(eps2),
                                         float(quad_phi_sign), int(bool(ewald)),
                                         ctypes.byref(tun) if tun is not None else None,
                                         ctypes.byref(h)))
        self = cls.__new__(cls)
        self.tree = None
        self.ewald = bool(ewald)
        self._keep = [params]
        self._h = h
        self.n = n
        return self

    def order(self):
        """Tree position -> input index (device-built plans), numpy int64."""
        return d2h(self.order_ptr(), np.int64, self.n)

    def order_ptr(self):
        """Device pointer to the plan's int64 tree position -> input index
        (device-built plans)."""
        ptr = lib().grav_plan_order(self._h)
        if not ptr:
            raise GravError("the plan was not built on the device")
        return ptr

    def problem(self):
        """Host copies of the plan's tables and lists (grav_plan_problem):
        dict with points, qcells, hcells, groups, ptr (4 offset arrays) and
        lists (P, Q, H, correction)."""
        p = Problem()
        check(lib().grav_plan_problem(self._h, ctypes.byref(p)))
        n, nc, ng = p.nbodies, p.ncells, p.ngroups
        ptr = [_host_array(x, np.int64, ng + 1) for x in (p.pptr, p.qptr, p.hptr, p.cptr)]
        lists = [d2h(x, np.uint32, int(q[-1]) if len(q) else 0) if x else np.zeros(0, np.uint32)
                 for x, q in zip((p.plist, p.qlist, p.hlist, p.clist), ptr)]
        return {"points": d2h(p.points, np.float32, 4 * (n + nc)).reshape(-1, 4),
                "qcells": d2h(p.qcells, QCELL_DTYPE, nc) if p.qcells else None,
                "hcells": d2h(p.hcells, HCELL_DTYPE, nc) if p.hcells else None,
                "groups": d2h(p.groups, GROUP_DTYPE, ng), "ptr": ptr, "lists": lists,
                "ncells": nc}

    def __init__(self, tree, eps2, quad_phi_sign=1.0, ewald=False, tuning=None, plain=False):
        """plain: the plain FP32 kernels (absolute coordinates, plain sums)
        instead of the mixed-precision ones (grav_problem.precision = 1)."""
        self.tree = tree
        self.ewald = bool(ewald)
        self._keep = []

        def keep(a, dtype=None):
            a = np.ascontiguousarray(a if dtype is None else a.astype(dtype, copy=False))
            self._keep.append(a)
            return a

        t = tree
        pts = keep(t.points, np.float32)
        groups = keep(t.groups)
        has_q = len(t.qlist) > 0
        has_h = len(t.hlist) > 0
        prob = Problem()
        prob.nbodies, prob.ncells, prob.ngroups = t.n, t.ncells, t.ngroups
        prob.points = pts.ctypes.data
        prob.qcells = keep(t.qcells).ctypes.data if len(t.qcells) else None
        prob.hcells = keep(t.hcells).ctypes.data if (has_h or ewald) and len(t.hcells) else None
        prob.groups = groups.ctypes.data
        prob.pptr = keep(t.ptr[0]).ctypes.data
        prob.qptr = keep(t.ptr[1]).ctypes.data
        prob.hptr = keep(t.ptr[2]).ctypes.data
        prob.plist = keep(t.plist).ctypes.data if len(t.plist) else keep(np.zeros(1, np.uint32)).ctypes.data
        prob.qlist = keep(t.qlist).ctypes.data if has_q else keep(np.zeros(1, np.uint32)).ctypes.data
        prob.hlist = keep(t.hlist).ctypes.data if has_h else keep(np.zeros(1, np.uint32)).ctypes.data
        prob.eps2 = float(eps2)
        prob.box = float(t.box)
        prob.quad_phi_sign = float(quad_phi_sign)
        prob.ewald = int(bool(ewald))
        prob.precision = 1 if plain else 0
        if ewald:
            prob.cptr = keep(t.ptr[3]).ctypes.data
            prob.clist = keep(t.clist).ctypes.data if len(t.clist) else keep(np.zeros(1, np.uint32)).ctypes.data
        self.problem = prob
        h = ctypes.c_void_p()
        tun = None
        if tuning is not None:
            tun = Tuning(*tuning) if not isinstance(tuning, Tuning) else tuning
        L = lib()
        check(L.grav_groups_upload_CUDA(ctypes.byref(prob),
                                        ctypes.byref(tun) if tun is not None else None,
                                        ctypes.byref(h)))
        self._h = h
        self.n = t.n

    def eval(self, stream=None):
        check(lib().grav_groups_eval_CUDA(self._h, stream))

    def download(self):
        out = np.empty((self.n, 4), dtype=np.float32)
        check(lib().grav_groups_download_CUDA(self._h, out.ctypes.data))
        return out

    def output_ptr(self):
        return lib().grav_plan_output(self._h)

    def bodies_ptr(self):
        """Device pointer of the body table (x, y, z, m float4, tree order)."""
        return lib().grav_plan_bodies(self._h)

    def set_tree(self, tree=None):
        """Give the plan its tree's links so that it can refit on the device."""
        t = tree or self.tree
        first, count = t.cell_ranges()
        child, nchild, level = t.cell_links()
        self._links = (first, count, child, nchild, level)
        check(lib().grav_plan_set_tree_CUDA(self._h, first.ctypes.data, count.ctypes.data,
                                            child.ctypes.data, nchild.ctypes.data,
                                            level.ctypes.data))

    def refit(self, stream=None):
        check(lib().grav_plan_refit_CUDA(self._h, stream))

    def integrate(self, vel_ptr, params_ptr, energy_ptr, stream=None):
        check(lib().grav_plan_integrate_CUDA(self._h, vel_ptr, params_ptr, energy_ptr, stream))

    def set_integrator(self, kind):
        """0: Integrate (params {dt, dtv, dtsync}); 1: CosmoIntegrate (params of
        nln_cosmo_kdk, 6 doubles) for later integrate and step calls."""
        check(lib().grav_plan_set_integrator_CUDA(self._h, int(kind)))

    def retune(self, tuning):
        """New tile shapes (a Tuning or a tuple of its fields); rebuilds the queue only."""
        tun = Tuning(*tuning) if not isinstance(tuning, Tuning) else tuning
        check(lib().grav_plan_retune_CUDA(self._h, ctypes.byref(tun)))

    def tuning(self):
        t = Tuning()
        check(lib().grav_plan_get_tuning(self._h, ctypes.byref(t)))
        return t

    def adjoint(self, wu_ptr, grad_ptr, stream=None):
        """dL/d(x, m) per body (device float4, tree order) for L = sum w.a + u phi
        (wu: device float4 (w, u) per body, tree order)."""
        check(lib().grav_plan_adjoint_CUDA(self._h, wu_ptr, grad_ptr, stream))

    def step(self, vel_ptr, params_ptr, energy_ptr, stream=None, graph=False):
        check(lib().grav_plan_step_CUDA(self._h, vel_ptr, params_ptr, energy_ptr, stream,
                                        int(bool(graph))))

    def counts(self):
        c = (ctypes.c_int64 * 4)()
        lib().grav_plan_counts(self._h, c)
        return np.array(list(c), dtype=np.int64)

    def launches(self):
        return lib().grav_plan_launches(self._h)

    def set_timing(self, on=True):
        check(lib().grav_plan_set_timing(self._h, int(bool(on))))

    def kernel_ms(self):
        """Per-kernel milliseconds of the last evaluation: order-4, quadrupole, point, finish."""
        ms = (ctypes.c_float * 4)()
        check(lib().grav_plan_kernel_ms(self._h, ms))
        return dict(zip(("hexa", "quad", "point", "finish"), list(ms)))

    def free(self):
        if getattr(self, "_h", None):
            lib().grav_plan_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def groups_eval(tree, eps2, quad_phi_sign=1.0):
    """One-call end-to-end form (grav_groups_CUDA): returns (n, 4) float32
    (ax, ay, az, phi) in tree order."""
    plan = Plan(tree, eps2, quad_phi_sign)
    plan.eval()
    out = plan.download()
    plan.free()
    return out


# ---------------------------------------------------------------- drop-in API
BODY_STRIDE = 14  # floats per reference body record (nln/physics.h:33-44)


def body_table(pos, mass):
    """A reference-layout body table (mass, pos[3], vel[3], acc[3], phi, nterms, ident)."""
    n = len(pos)
    bt = np.zeros((n, BODY_STRIDE), dtype=np.float32)
    bt[:, 0] = mass
    bt[:, 1:4] = pos
    return bt


class DropIn:
    """The reference call sequence of nln/mac.c on the drop-in entry points:
    WalkInitSinkCUDA, any number of grav_*_CUDA calls, WalkTerminateSinkCUDA."""

    def __init__(self, btab):
        self.btab = np.ascontiguousarray(btab, dtype=np.float32)
        assert self.btab.shape[1] == BODY_STRIDE
        L = lib()
        L.CUDA_Init(None)
        check()
        L.WalkInitSinkCUDA(self.btab.ctypes.data, BODY_STRIDE, len(self.btab))
        check()

    def slot(self):
        L = lib()
        inuse = ctypes.c_int()
        while True:
            q = L.qallocCUDA(ctypes.byref(inuse))
            check()
            if q >= 0:
                return q

    def mn(self, routine, first, count, f, source_n, sz, e):
        """grav_mn_CUDA on sinks [first, first+count) with list f."""
        L = lib()
        p = self.btab.ctypes.data + 4 * BODY_STRIDE * first
        f = np.ascontiguousarray(f, dtype=np.float32)
        L.grav_mn_CUDA(routine.encode(), p, None, count, BODY_STRIDE, f.ctypes.data, source_n, sz,
                       float(e), None, self.slot())
        check()

    def mnss(self, sink_base, m, ss_index, ss_seg, seg, source_base, source_n, mmass, e):
        L = lib()
        ss_index = np.ascontiguousarray(ss_index, np.uint16)
        ss_seg = np.ascontiguousarray(ss_seg, np.uint32).reshape(-1, 2)
        seg = np.ascontiguousarray(seg, np.uint32).reshape(-1, 2)
        source_n = np.ascontiguousarray(source_n, np.int32)
        L.grav_mnss_CUDA(b"pMM_mnss_sK1", sink_base, m, ss_index.ctypes.data, ss_seg.ctypes.data,
                         len(ss_seg), seg.ctypes.data, len(seg), source_base, source_n.ctypes.data,
                         float(mmass), float(e), None, self.slot())
        check()

    def qnss(self, base, m, seg, source, source_n):
        """grav_qnss_CUDA ("pQ1_qnss"): sink base+i against the run seg[i]
        (base, length records) of the QSZ AoSoA buffer `source`."""
        seg = np.ascontiguousarray(seg, np.uint32).reshape(-1, 2)
        source = np.ascontiguousarray(source, np.float32)
        lib().grav_qnss_CUDA(b"pQ1_qnss", base, m, seg.ctypes.data, source.ctypes.data,
                             int(source_n), self.slot())
        check()

    def init_src(self, qtab):
        """WalkInitSrcCUDA: the cell table (ncells x stride floats, hexacell layout)."""
        self._qtab = np.ascontiguousarray(qtab, np.float32)
        lib().WalkInitSrcCUDA(self._qtab.ctypes.data, self._qtab.shape[1], len(self._qtab))
        check()

    def qns(self, base, m, source_list):
        """grav_qns_CUDA ("pQQ1"): sinks [base, base+m) against cells source_list."""
        sl = np.ascontiguousarray(source_list, np.int32)
        lib().grav_qns_CUDA(b"pQQ1", base, m, sl.ctypes.data, len(sl), self.slot())
        check()

    def terminate_src(self):
        lib().WalkTerminateSrcCUDA()
        check()

    def peek(self):
        out = np.empty((len(self.btab), 4), dtype=np.float32)
        check(lib().gravcuda_peek_accumulators(out.ctypes.data, 0, len(self.btab)))
        return out

    def terminate(self):
        L = lib()
        L.WalkTerminateSinkCUDA(self.btab.ctypes.data, BODY_STRIDE, len(self.btab))
        check()
        return self.btab[:, 7:11].copy()


def fp32_peak():
    """Measured FP32 CUDA-core peak of the current device, TFLOP/s (grav_fp32_peak_CUDA)."""
    out = ctypes.c_double()
    check(lib().grav_fp32_peak_CUDA(ctypes.byref(out)))
    return out.value


_drive = None


def drive_mn(dropin, first, count, packs, e):
    """Time the drop-in call sequence of nln/mac.c from C (lib/libmacdrive.so):
    for every group g and list kind, one grav_mn_CUDA on a slot from
    qallocCUDA, then WalkTerminateSinkCUDA; returns the wall-clock seconds.
    dropin: a DropIn (its body table is registered); first, count: sinks of
    each group in that table; packs: (routine, sz, blk_ptr, data) per kind,
    blk_ptr with one entry per group plus one."""
    global _drive
    if _drive is None:
        lib()
        _drive = ctypes.CDLL(_build.build_drive())
        _drive.mac_drive_mn.restype = ctypes.c_double
        _drive.mac_drive_mn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
                                        ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float]
    first = np.ascontiguousarray(first, np.int64)
    count = np.ascontiguousarray(count, np.int32)
    k = len(packs)
    names = (ctypes.c_char_p * k)(*[r.encode() for r, _, _, _ in packs])
    sz = (ctypes.c_int * k)(*[int(z) for _, z, _, _ in packs])
    datas = [np.ascontiguousarray(d, np.float32) for _, _, _, d in packs]
    ptrs = [np.ascontiguousarray(b, np.int64) for _, _, b, _ in packs]
    data_p = (ctypes.c_void_p * k)(*[d.ctypes.data for d in datas])
    ptr_p = (ctypes.c_void_p * k)(*[b.ctypes.data for b in ptrs])
    secs = _drive.mac_drive_mn(dropin.btab.ctypes.data, BODY_STRIDE, len(dropin.btab), len(first),
                               first.ctypes.data, count.ctypes.data, k, names, sz, data_p, ptr_p,
                               float(e))
    check()
    return secs


def dropin_phases():
    """gravcuda_dropin_phases: seconds of staging copies, staging waits, queue
    waits, the submitter's CUDA calls and the final drain, and the call count."""
    out = (ctypes.c_double * 6)()
    lib().gravcuda_dropin_phases(out)
    return {"staging_copy_s": out[0], "staging_wait_s": out[1], "queue_wait_s": out[2],
            "submitter_s": out[3], "drain_s": out[4], "calls": int(out[5])}


def direct_fp64(points, sinks, eps2, box=0.0):
    """FP64 direct sum on the GPU at sample sinks (grav_direct_fp64_CUDA):
    (nsink, 4) doubles (ax, ay, az, phi); Ewald-summed when box > 0."""
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
    sinks = np.ascontiguousarray(sinks, np.int64)
    out = np.zeros((len(sinks), 4), np.float64)
    check(lib().grav_direct_fp64_CUDA(pts.ctypes.data, len(pts), sinks.ctypes.data, len(sinks),
                                      float(eps2), float(box), out.ctypes.data))
    return out


class PinnedProblem:
    """A tree's tables and lists copied into page-locked host memory, as the
    host side of an end-to-end grav_groups_CUDA call reads them.  With
    packed, the run-packed lists (tree.pack()) stand in for the plain ones;
    `lists` holds the pinned point, quadrupole and order-4 lists (packed
    words when packed)."""

    def __init__(self, tree, lists_in_host=False, packed=False):
        import torch
        self._keep = []
        self.h2d_bytes = 0

        def pin(a):
            a = np.ascontiguousarray(a)
            buf = torch.empty(max(1, a.nbytes), dtype=torch.uint8, pin_memory=True)
            v = buf.numpy()[:a.nbytes].view(a.dtype).reshape(a.shape)
            v[...] = a
            self._keep.append(buf)
            self.h2d_bytes += a.nbytes
            return v

        t = tree
        p = Problem()
        p.nbodies, p.ncells, p.ngroups = t.n, t.ncells, t.ngroups
        p.points = pin(t.points).ctypes.data
        has_q, has_h = len(t.qlist) > 0, len(t.hlist) > 0
        periodic = t.box > 0
        p.qcells = pin(t.qcells).ctypes.data if has_q else None
        p.hcells = pin(t.hcells).ctypes.data if (has_h or periodic) and len(t.hcells) else None
        p.groups = pin(t.groups).ctypes.data
        p.pptr = pin(t.ptr[0]).ctypes.data
        p.qptr = pin(t.ptr[1]).ctypes.data
        p.hptr = pin(t.ptr[2]).ctypes.data
        if periodic:
            p.cptr = pin(t.ptr[3]).ctypes.data
        if packed:
            if lists_in_host:
                raise ValueError("packed lists are for the copied form")
            if not hasattr(t, "zlist"):
                t.pack()
            self.lists = []
            for k in range(4):
                if len(t.zlist[k]) == 0:
                    self.lists.append(None)
                    continue
                p.zptr[k] = pin(t.zptr[k]).ctypes.data
                self.lists.append(pin(t.zlist[k]))
                p.zlist[k] = self.lists[-1].ctypes.data
            self.lists = self.lists[:3]
        else:
            self.lists = [pin(t.plist if len(t.plist) else np.zeros(1, np.uint32)),
                          pin(t.qlist if has_q else np.zeros(1, np.uint32)),
                          pin(t.hlist if has_h else np.zeros(1, np.uint32))]
            p.plist, p.qlist, p.hlist = (a.ctypes.data for a in self.lists)
            if periodic:
                p.clist = pin(t.clist if len(t.clist) else np.zeros(1, np.uint32)).ctypes.data
        p.quad_phi_sign = 1.0
        p.lists_in_host = int(bool(lists_in_host))
        self.problem = p
        buf = torch.empty(t.n * 16, dtype=torch.uint8, pin_memory=True)
        self._keep.append(buf)
        self.out = buf.numpy().view(np.float32).reshape(t.n, 4)


def pinned_problem(tree, lists_in_host=False, packed=False):
    return PinnedProblem(tree, lists_in_host, packed)


def groups_eval_problem(pp, eps2, box, ewald=False):
    """grav_groups_CUDA on a PinnedProblem: upload, evaluate, download, free."""
    pp.problem.eps2 = float(eps2)
    pp.problem.box = float(box)
    pp.problem.ewald = int(bool(ewald))
    check(lib().grav_groups_CUDA(ctypes.byref(pp.problem), pp.out.ctypes.data))
    return pp.out


def build_eval(bodies, eps2, box=0.0, ewald=False, quad_phi_sign=1.0, out=None, leaf_max=16,
               group_max=32, p2cut=7, p4cut=20, tol=1e-3, rel_tol=0.0, rel_tol0=0.0,
               ewald_theta=0.2, ptol_boost=0.0):
    """grav_build_eval_CUDA: host bodies (n, 4) float32 (x, y, z, m) to host
    (ax, ay, az, phi) (n, 4) in the same order: copy, GPU tree build,
    evaluation and copy back in one call.  out: an (n, 4) float32 array to
    fill (page-locked memory copies fastest)."""
    from .host import Params
    b = np.ascontiguousarray(bodies, np.float32).reshape(-1, 4)
    n = len(b)
    out = np.empty((n, 4), np.float32) if out is None else out
    params = Params(leaf_max, group_max, p2cut, p4cut, tol, rel_tol, rel_tol0, float(box), 0, 0,
                    ewald_theta, ptol_boost)
    check(lib().grav_build_eval_CUDA(ctypes.byref(params), b.ctypes.data, n, float(eps2),
                                     float(quad_phi_sign), int(bool(ewald)), out.ctypes.data))
    return out


def build_eval_phases():
    out = np.zeros(4, np.float64)
    lib().grav_build_eval_phases(out.ctypes.data)
    return dict(zip(("h2d", "build", "eval_d2h", "release"), out.tolist()))


def build_phases():
    """Seconds of this thread's last GPU tree build: sort, cells, moments and
    tables, sink groups, the two walk passes (count and fill), the list
    offsets and allocations between them, and the whole
    grav_plan_build_CUDA call."""
    out = np.zeros(7, np.float64)
    lib().grav_plan_build_phases(out.ctypes.data)
    return dict(zip(("sort", "cells", "moments", "groups", "walk", "lists", "total"),
                    out.tolist()))


def groups_phases():
    """Seconds of the phases of this thread's last grav_groups_CUDA call:
    host checks and queue, allocation and table upload, list copies with
    the overlapped evaluation, download, release."""
    out = np.zeros(5, np.float64)
    lib().grav_groups_CUDA_phases(out.ctypes.data)
    return dict(zip(("host", "upload", "copy_eval", "download", "release"), out.tolist()))
