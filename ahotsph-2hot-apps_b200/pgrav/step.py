"""Time stepping on the device: the KDK integrator of nln/integrate.c:16-59
(Integrate) around the batched force evaluation.

The tree and the interaction lists are rebuilt every ``rebuild`` steps,
on the GPU from the bodies already there (grav_plan_build_CUDA; gpu_build,
the default) or on the host (nlnhost.h, bit-identical lists).  Between
rebuilds every step runs on the GPU as evaluate, integrate (kick by dtv,
drift by dt) and refit of the cell tables, optionally replayed from one
captured CUDA graph (grav_plan_step_CUDA).  Velocities lag the
positions by half a step after the first kick (dtv = dt/2 once, then dt),
and the energies of each step are those of Integrate: KE of the velocity
synchronised to the positions' time, PE = 1/2 sum m phi (G = 1).
"""
import numpy as np

from . import gravcuda as gc
from . import host


def _rt():
    from cuda.bindings import runtime as rt
    return rt


def memcpy_d2h(dst_array, src_ptr):
    rt = _rt()
    err, = rt.cudaMemcpy(dst_array.ctypes.data, src_ptr, dst_array.nbytes,
                         rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    if int(err) != 0:
        raise gc.GravError(f"cudaMemcpy D2H failed: {err}")
    return dst_array


def memcpy_d2d(dst_ptr, src_ptr, nbytes):
    rt = _rt()
    err, = rt.cudaMemcpy(dst_ptr, src_ptr, nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
    if int(err) != 0:
        raise gc.GravError(f"cudaMemcpy D2D failed: {err}")


def memcpy_h2d(dst_ptr, src_array):
    rt = _rt()
    src = np.ascontiguousarray(src_array)
    err, = rt.cudaMemcpy(dst_ptr, src.ctypes.data, src.nbytes,
                         rt.cudaMemcpyKind.cudaMemcpyHostToDevice)
    if int(err) != 0:
        raise gc.GravError(f"cudaMemcpy H2D failed: {err}")


class Stepper:
    """KDK steps of a particle set with the batched evaluation.

    pos, vel: (n, 3); mass: (n,); eps2 Plummer softening; box > 0 makes the
    run periodic (with the Ewald correction unless ewald=False).  tree_kw
    goes to host.Tree (tol, leaf_max, ...).  graph=True replays each step
    from a CUDA graph captured on the first step after every rebuild.

    cosmo (a pgrav.cosmo.Cosmology) makes the run comoving: pos are
    comoving positions (box the comoving side), vel the peculiar velocities
    a dx/dt, eps2 the comoving softening, tstart the cosmic time of the
    initial conditions, G = 1.  Steps use CosmoIntegrate's factors
    (nln/integrate.c:82-135) on comoving coordinates: the canonical momentum
    p = a^2 dx/dt takes kick(t0, t1) = int dt/a times the comoving
    acceleration and the positions drift by int dt/a^2 (the reference applies
    the same factors to physical positions, scaled by a0 and a1).  The energy
    record is the physical peculiar kinetic energy and the physical potential
    energy (phi / a).
    """

    def __init__(self, pos, vel, mass, eps2, box=0.0, ewald=None, rebuild=8, graph=True,
                 tree_kw=None, gpu_build=True, cosmo=None, tstart=0.0):
        import torch
        self.torch = torch
        self.pos = np.array(pos, np.float32).reshape(-1, 3)
        self.vel = np.array(vel, np.float32).reshape(-1, 3)
        self.mass = np.asarray(mass, np.float32)
        self.n = len(self.pos)
        self.eps2 = float(eps2)
        self.box = float(box)
        self.ewald = (self.box > 0) if ewald is None else bool(ewald)
        self.rebuild = max(1, int(rebuild))
        self.graph = bool(graph)
        self.tree_kw = dict(tree_kw or {})
        self.gpu_build = bool(gpu_build)
        self.orig = None  # GPU rebuilds: tree position -> original body index (device int64)
        self.build_s = []  # seconds of every rebuild
        self.build_phases = []  # GPU rebuilds: gravcuda.build_phases() of each
        self.cosmo = cosmo
        self.tpos = float(tstart)
        self.tvel = float(tstart)
        if cosmo is not None:
            self.vel = (self.vel * np.float32(cosmo.a_at_t(tstart))).astype(np.float32)  # p = a u
        self.nsteps = 0
        self.history = []
        self.stream = torch.cuda.Stream()
        dev = torch.device("cuda")
        self.params = torch.zeros(6 if cosmo is not None else 3, dtype=torch.float64, device=dev)
        self.energy = torch.zeros(2, dtype=torch.float64, device=dev)
        self.dvel = None
        self.plan = None
        self.tree = None
        self._build()

    # -- rebuild: tree and lists from the current positions
    def _build(self):
        import time
        t0 = time.perf_counter()
        if self.gpu_build:
            self._build_gpu()
        else:
            self._build_host()
        if self.cosmo is not None:
            self.plan.set_integrator(1)
        self.torch.cuda.synchronize()
        self.build_s.append(time.perf_counter() - t0)
        if self.gpu_build:
            from . import gravcuda
            self.build_phases.append(gravcuda.build_phases())

    # On the GPU: the bodies and velocities stay on the device.  They go to
    # the builder in the original order, as the host rebuild hands them over
    # (the key sort breaks ties by input index), so both rebuilds make the
    # same tree; then into the new tree's order.
    def _build_gpu(self):
        torch = self.torch
        n = self.n
        if self.plan is None:
            bodies = torch.empty((n, 4), dtype=torch.float32, device="cuda")
            bodies[:, :3] = torch.from_numpy(self.pos).cuda()
            bodies[:, 3] = torch.from_numpy(self.mass).cuda()
            vel = torch.from_numpy(self.vel).cuda()
        else:
            torch.cuda.synchronize()
            tree_bodies = torch.empty((n, 4), dtype=torch.float32, device="cuda")
            memcpy_d2d(tree_bodies.data_ptr(), self.plan.bodies_ptr(), n * 16)
            bodies = torch.empty_like(tree_bodies)
            bodies[self.orig] = tree_bodies
            vel = torch.empty((n, 3), dtype=torch.float32, device="cuda")
            vel[self.orig] = self.dvel[:, :3]
            self.plan.free()
            self.plan = None
        if self.box > 0:
            x = torch.remainder(bodies[:, :3], self.box)
            x[x >= self.box] = 0.0
            bodies[:, :3] = x
        self.plan = gc.Plan.build(None, None, self.eps2, box=self.box, ewald=self.ewald,
                                  bodies=bodies, **self.tree_kw)
        order = torch.empty(n, dtype=torch.int64, device="cuda")
        memcpy_d2d(order.data_ptr(), self.plan.order_ptr(), n * 8)
        self.dvel = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        self.dvel[:, :3] = vel[order]
        self.orig = order

    # On the host: tree and lists from the host copy of the positions.
    def _build_host(self):
        torch = self.torch
        if self.plan is not None:
            self._pull()
            self.plan.free()
            self.plan = None
            self.tree = None  # release the old lists before the new walk
        if self.box > 0:
            self.pos = np.mod(self.pos, np.float32(self.box)).astype(np.float32)
            self.pos[self.pos >= self.box] = 0.0
        self.tree = host.Tree(self.pos, self.mass, box=self.box, **self.tree_kw)
        self.plan = gc.Plan(self.tree, self.eps2, ewald=self.ewald)
        self.plan.set_tree(self.tree)
        v = np.zeros((self.n, 4), np.float32)
        v[:, :3] = self.vel[self.tree.order]
        self.dvel = torch.from_numpy(v).to("cuda")

    # -- device state back to host arrays in the original body order
    def _pull(self):
        self.torch.cuda.synchronize()
        body = memcpy_d2h(np.empty((self.n, 4), np.float32), self.plan.bodies_ptr())
        order = self.orig.cpu().numpy() if self.gpu_build else self.tree.order
        self.pos[order] = body[:, :3]
        self.vel[order] = self.dvel.cpu().numpy()[:, :3]

    def state(self):
        """(pos, vel) in the original order, current (comoving runs: comoving
        positions and the peculiar velocities a dx/dt at tvel)."""
        self._pull()
        if self.cosmo is not None:
            return self.pos.copy(), (self.vel / np.float32(self.cosmo.a_at_t(self.tvel))).astype(np.float32)
        return self.pos.copy(), self.vel.copy()

    def step(self, dt):
        torch = self.torch
        if self.nsteps > 0 and self.nsteps % self.rebuild == 0:
            self._build()
        dtv = 0.5 * dt if self.nsteps == 0 else dt
        dtsync = self.tpos - self.tvel
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        if self.cosmo is not None:
            f = self.cosmo.kdk(self.tpos, self.tvel, dt, dtv)
            # comoving form: the acceleration is a0^2 times the physical one
            coef = [f[0] * f[5], f[1] * f[5], f[2], 1.0, 1.0, f[5]]
        else:
            coef = [dt, dtv, dtsync]
        with torch.cuda.stream(self.stream):
            self.params.copy_(torch.tensor(coef, dtype=torch.float64))
            e0.record(self.stream)
            self.plan.step(self.dvel.data_ptr(), self.params.data_ptr(), self.energy.data_ptr(),
                           self.stream.cuda_stream, graph=self.graph)
            e1.record(self.stream)
        self.stream.synchronize()
        ke, pe = self.energy.cpu().numpy()
        pscale = 1.0 / self.cosmo.a_at_t(self.tpos) if self.cosmo is not None else 1.0
        rec = {"t": self.tpos, "ke": 0.5 * float(ke), "pe": 0.5 * float(pe) * pscale,
               "ms": e0.elapsed_time(e1), "graph": self.graph}
        if self.cosmo is not None:
            rec["a"] = self.cosmo.a_at_t(self.tpos)
        rec["e"] = rec["ke"] + rec["pe"]
        self.history.append(rec)
        self.tpos += dt
        self.tvel += dtv
        self.nsteps += 1
        return rec

    def run(self, nsteps, dt):
        return [self.step(dt) for _ in range(nsteps)]

    def save(self, path):
        """A checkpoint: the bodies (original order, ident = original index)
        and the step state in an SDF file with the reference's header keys
        (nln/output.c:217-330) plus this run's parameters."""
        from . import sdf
        pos, vel = self.state()
        sdf.write(path, pos, vel, self.mass, header={
            "version": (sdf.INT, 2), "version_2HOT": (sdf.INT, 2), "npart": (sdf.INT64, self.n),
            "iter": (sdf.INT, self.nsteps), "do_periodic": (sdf.INT, int(self.box > 0)),
            "tpos": (sdf.DOUBLE, self.tpos), "tvel": (sdf.DOUBLE, self.tvel),
            "tacc": (sdf.DOUBLE, self.tpos), "R0": (sdf.FLOAT, 0.5 * self.box),
            "L0": (sdf.FLOAT, self.box), "Gnewt": (sdf.DOUBLE, 1.0),
            "eps2": (sdf.DOUBLE, self.eps2), "ewald": (sdf.INT, int(self.ewald)),
            "rebuild": (sdf.INT, self.rebuild), **self._cosmo_header()})

    def _cosmo_header(self):
        from . import sdf
        if self.cosmo is None:
            return {}
        p = self.cosmo.params
        h = {"cosmology": (sdf.INT, 1)}
        for k in ("H0", "Omega_m", "Omega_r", "Omega_lambda", "Omega_de", "w0", "wa"):
            h[k] = (sdf.DOUBLE, float(getattr(p, k)))
        return h

    @classmethod
    def load(cls, path, graph=True, tree_kw=None, gpu_build=True):
        """Resume from a checkpoint written by save(): the same bodies, step
        count and times.  The tree is built from the saved bodies, so a
        checkpoint taken on a rebuild step (a multiple of `rebuild`) continues
        exactly as the saved run would have."""
        from . import sdf
        h, b = sdf.read(path)
        order = np.argsort(b["ident"], kind="stable")
        cosmo = None
        if h.get("cosmology"):
            from .cosmo import Cosmology
            cosmo = Cosmology(**{k: float(h[k]) for k in ("H0", "Omega_m", "Omega_r",
                                                          "Omega_lambda", "Omega_de", "w0", "wa")})
        st = cls(b["pos"][order], b["vel"][order], b["mass"][order], h["eps2"],
                 box=float(h.get("L0", 0.0)) if h.get("do_periodic") else 0.0,
                 ewald=bool(h.get("ewald", 0)), rebuild=h.get("rebuild", 8), graph=graph,
                 tree_kw=tree_kw, gpu_build=gpu_build, cosmo=cosmo,
                 tstart=float(h["tvel"]) if cosmo is not None else 0.0)
        st.nsteps = int(h["iter"])
        st.tpos = float(h["tpos"])
        st.tvel = float(h["tvel"])
        return st

    def free(self):
        if self.plan is not None:
            self.plan.free()
            self.plan = None
