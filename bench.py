#!/usr/bin/env python
"""Benchmark of the 2HOT tree-gravity force evaluation on B200.

One step = one force evaluation (every sink group of the step through the
batched kernels) of a seeded synthetic particle set.  The default workload
is the periodic 256^3 box: N = 2^24 particles on a grid displaced by a
Gaussian random field with P(k) ~ k^-2.5 (rms 0.5 grid spacing), Plummer
softening 1/50 of the spacing, order-4 moments plus the Ewald correction,
force error measured against an FP64 Ewald-summed direct sum on 8192 sinks.

After the timed region the same run measures, untimed, one block per
configuration of the benchmark set (--configs; all by default):
  plummer64k  Plummer N = 65,536, order 2: batched and drop-in GPU results
              against the reference's own AVX kernels on the full lists, and
              against the FP64 direct sum on every sink
  box128      periodic 128^3, order 4 + Ewald: mixed-precision against plain
              FP32 kernels, accuracy on 4096 sinks and time
  batch1024   1024 isolated systems of uneven N in one launch per list kind,
              autotuned tile shapes, graph-captured KDK step
  adjoint     Plummer N = 2^20: adjoint/forward time, FP64 central
              differences at 64 coordinates and 16 masses, the FP64
              direct-sum gradient on an N = 8192 system, and 16 leapfrog KDK
              steps checkpointed every 4, checked against FP64 differences
  kdk256      32 graph-captured KDK steps of the 256^3 box with energy drift

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload box256|box128|plummer64k|batch1024] [--configs all|none|a,b]

Under torchrun (N > 1) every rank evaluates its own replica of the workload
(the force evaluation does not shard across GPUs here): value is the sum of
interactions over ranks divided by the slowest rank's time.  The
configuration blocks run on rank 0 only.

The CPU legs (cpu_baseline, and the per-configuration checks against the
reference's own kernels and the FP64 checkers) call oracle/, the parity
checker; nothing measured on the GPU goes through it.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
for _p in (REPO, os.path.join(REPO, "ahotsph-2hot-apps_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "tree-gravity interactions/s (one force evaluation per step)"
UNIT = "interactions/s"
# algorithmic flops per interaction: 23 for body-body and monopole cells
# (reference count 26-27, nln/grav.c:56-75), 66 quadrupole
# (nln/do_grav_avx8.c:378), 217 order 4 (nln/do_grav_avx8.c:45)
FLOPS = np.array([23, 23, 66, 217], np.float64)
# DRAM bytes (read + write) per interaction of each list kernel, from one ncu
# capture of the kernels on the periodic 128^3 box (MAC 1e-4); a launch's
# traffic is this times its interactions (traffic grows with list entries)
DRAM_BYTES_PER_INTERACTION = {"hexa": 0.2007, "quad": 0.193, "point": 0.164}
ALL_CONFIGS = ("plummer64k", "box128", "batch1024", "adjoint", "kdk256")
# blocks that run only when named: the periodic adjoint alone (--adjoint-workload)
EXTRA_CONFIGS = ("adjoint_periodic",)

WORKLOADS = {
    # N = 2^24 periodic box, order 4 + Ewald (the metric's N)
    # (MAC tolerance chosen for <= 1e-4 rms relative force error)
    "box256": dict(kind="box", n1d=256, rms_disp=0.5, p2cut=7, p4cut=20, ewald=True,
                   tol=1.5e-6, sample=8192),
    # 32^3 and 64^3 periodic boxes, order 4 + Ewald (small cases: the
    # periodic adjoint's check, profiling)
    "box32": dict(kind="box", n1d=32, rms_disp=0.25, p2cut=7, p4cut=20, ewald=True,
                  tol=2.5e-6, sample=1024),
    "box64": dict(kind="box", n1d=64, rms_disp=0.25, p2cut=7, p4cut=20, ewald=True,
                  tol=2.5e-6, sample=2048),
    # 128^3 periodic box, order 4 + Ewald
    "box128": dict(kind="box", n1d=128, rms_disp=0.25, p2cut=7, p4cut=20, ewald=True,
                   tol=2.5e-6, sample=4096),
    # Plummer sphere N = 65536, order 2
    "plummer64k": dict(kind="plummer", n=65536, eps=0.01, p2cut=7, p4cut=0, ewald=False,
                       tol=2e-5, sample=8192),
    # 1024 independent isolated systems, N log-uniform in [512, 65536],
    # half Plummer half Hernquist (a = 1), eps = 0.01 a, order 4, one launch per kind
    "batch1024": dict(kind="batch", nsys=1024, nmin=512, nmax=65536, eps=0.01, p2cut=7,
                      p4cut=20, ewald=False, tol=1e-5, sample=2048),
}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    e = np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)
    return float(np.sqrt(np.mean(e * e))), float(e.max())


def time_evals(plan, stream, reps):
    """Mean device milliseconds of `reps` evaluations (CUDA events on the stream)."""
    import torch
    plan.eval(stream.cuda_stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        plan.eval(stream.cuda_stream)
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_problem(w, seed=123):
    from pgrav import ics
    if w["kind"] == "batch":
        rng = np.random.default_rng(seed)
        ns = np.floor(np.exp(rng.uniform(np.log(w["nmin"]), np.log(w["nmax"]), w["nsys"])))
        systems = []
        for k, n in enumerate(ns.astype(int)):
            gen = ics.plummer if k % 2 == 0 else ics.hernquist
            systems.append(gen(int(n), seed=seed + 1 + k))
        return systems, None, w["eps"] ** 2, 0.0
    if w["kind"] == "box":
        pos, m = ics.grf_box(w["n1d"], seed=seed, slope=-2.5, rms_disp=w["rms_disp"])
        eps = 1.0 / w["n1d"] / 50.0
        return pos, m, eps * eps, 1.0
    pos, m = ics.plummer(w["n"], seed=seed)
    return pos, m, w["eps"] ** 2, 0.0


def build_tree(w, pos, m, box, tol, nthreads=0):
    from pgrav import host
    if w["kind"] == "batch":
        # members built in parallel (one host thread each), then merged
        from concurrent.futures import ThreadPoolExecutor
        kw = dict(leaf_max=16, group_max=32, p2cut=w["p2cut"], p4cut=w["p4cut"], tol=tol,
                  nthreads=1)
        with ThreadPoolExecutor(max_workers=os.cpu_count()) as ex:
            members = list(ex.map(lambda s: host.Tree(s[0], s[1], **kw), pos))
        t = host.Tree.merge(members)
        del members
        return t
    return host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=w["p2cut"], p4cut=w["p4cut"],
                     tol=tol, box=box, nthreads=nthreads)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5], f[6], f[7], f[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        sm = [r[0] for r in rows]
        reasons = set()
        for r in rows:
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                "sw_power_cap"), r[2:]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": rows[0][1],
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path)), "measured"
    return {"hbm_gbs": 6650.0, "sm_max_mhz": 1965.0}, "fallback"


def cpu_reference_rate(tree, eps2, seconds=15.0, nthreads=None, seed=0, max_groups=4096,
                       max_bytes=1 << 30):
    """The reference's own AVX kernels (nln/do_grav_avx8.c compiled from the
    reference source into oracle/_ref) over the same lists, for a random
    sample of groups (at most max_groups, and at most max_bytes of packed
    AoSoA lists), all host threads: (interactions/s, seconds, threads, sample)."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    nthreads = nthreads or os.cpu_count()
    rng = np.random.default_rng(seed)
    per_group = sum(float(tree.ptr[k][-1]) / tree.ngroups * sz * 4 for k, sz in ((0, 4), (1, 13), (2, 29)))
    max_groups = int(max(16, min(max_groups, max_bytes / max(per_group, 1.0))))
    gids = np.sort(rng.choice(tree.ngroups, min(max_groups, tree.ngroups), replace=False))
    sf = np.ascontiguousarray(tree.groups["first"][gids]).astype(np.int64)
    sc = np.ascontiguousarray(tree.groups["count"][gids]).astype(np.int32)
    pos = np.ascontiguousarray(tree.sorted_pos.ravel(), np.float32)
    out = np.zeros((tree.n, 4), np.float32)
    lists = []
    inter = 0
    for kind, refkind in ((0, O.MONO_PLUMMER), (1, O.QUAD_PLUMMER), (2, O.HEXA_PLUMMER)):
        ptr = tree.ptr[kind]
        if ptr[-1] == 0:
            continue
        bp, data = tree.aosoa_subset(gids, kind)
        lists.append((refkind, O.KIND_SZ[refkind], data, np.ascontiguousarray(bp[:-1]),
                      np.ascontiguousarray(np.diff(bp))))
        inter += int(((ptr[gids + 1] - ptr[gids]) * tree.groups["count"][gids]).sum())
    reps, t0 = 0, time.perf_counter()
    while True:
        for refkind, sz, data, bf, bc in lists:
            O.ref().ref_groups_eval(refkind, data, sz, bf, bc, sf, sc, len(gids), pos, eps2,
                                    out.ravel(), nthreads)
        reps += 1
        el = time.perf_counter() - t0
        if el > seconds or reps >= 1000:
            break
    return (inter * reps / el, el, nthreads,
            f"{len(gids)} random sink groups ({int(sc.sum())} sinks, {inter} interactions) "
            f"x {reps} passes; Newtonian list terms only (the reference applies its periodic "
            f"correction separately)")


def dropin_rate(tree, eps2, max_groups=2048, seed=1, max_bytes=1 << 30):
    """The plain FP32 drop-in path (gravcuda.h Part 1 as nln/mac.c drives it:
    WalkInitSinkCUDA, one grav_mn_CUDA per group and list kind on the
    reference AoSoA lists with absolute FP32 coordinates, then
    WalkTerminateSinkCUDA) over a random sample of the same groups, the
    calls issued from C (lib/libmacdrive.so), the sampled groups' sinks in a
    body table of their own; wall clock from the first call to the results,
    Newtonian list terms: (interactions/s, seconds, sample)."""
    from pgrav import gravcuda as gc
    rng = np.random.default_rng(seed)
    per_group = sum(float(tree.ptr[k][-1]) / tree.ngroups * sz * 4 for k, sz in ((0, 4), (1, 13), (2, 29)))
    ng = int(max(16, min(max_groups, tree.ngroups, max_bytes / max(per_group, 1.0))))
    gids = np.sort(rng.choice(tree.ngroups, ng, replace=False))
    packs = []
    inter = 0
    for kind, routine, sz in ((0, "pMp", 4), (1, "pQp", 13), (2, "pHp", 29)):
        ptr = tree.ptr[kind]
        if ptr[-1] == 0:
            continue
        bp, data = tree.aosoa_subset(gids, kind)
        packs.append((routine, sz, bp, data))
        inter += int(((ptr[gids + 1] - ptr[gids]) * tree.groups["count"][gids]).sum())
    first = tree.groups["first"][gids].astype(np.int64)
    count = tree.groups["count"][gids].astype(np.int32)
    idx = np.concatenate([np.arange(f, f + c) for f, c in zip(first, count)])
    local_first = np.concatenate([[0], np.cumsum(count)[:-1]]).astype(np.int64)
    bt = gc.body_table(tree.sorted_pos[idx], tree.points[idx, 3])
    secs = []
    for _ in range(3):  # the first pass sizes the slots' buffers
        d = gc.DropIn(bt.copy())
        secs.append(gc.drive_mn(d, local_first, count, packs, eps2))
    el = min(secs[1:])
    return (inter / el, el, f"{ng} random sink groups ({int(count.sum())} sinks, {inter} "
            f"interactions), one grav_mn_CUDA per group and kind (pMp/pQp/pHp) issued from C "
            f"(best of 2 passes after one)")


def kdk_run(w, pos, m, eps2, box, tol, nsteps, dt, rebuild):
    """The large periodic box's time-stepping leg: nsteps KDK steps
    (Integrate of nln/integrate.c) from rest, graph-captured device steps
    between host rebuilds; energies per step."""
    from pgrav import step as S
    st = S.Stepper(pos, np.zeros_like(pos), m, eps2, box=box, ewald=w["ewald"] and box > 0,
                   rebuild=rebuild, graph=True,
                   tree_kw=dict(leaf_max=16, group_max=32, p2cut=w["p2cut"], p4cut=w["p4cut"],
                                tol=tol))
    t0 = time.perf_counter()
    st.run(nsteps, dt)
    wall = time.perf_counter() - t0
    h = st.history
    builds = list(st.build_s)
    build_phases = [{k: round(v, 4) for k, v in ph.items()} for ph in st.build_phases]
    st.free()
    e = np.array([r["e"] for r in h])
    pe = np.array([r["pe"] for r in h])
    ms = np.array([r["ms"] for r in h])
    steady = ms[[k for k in range(len(ms)) if k % rebuild != 0]] if len(ms) > 1 else ms
    return {"steps": nsteps, "dt": dt, "rebuild_every": rebuild, "graph": True,
            "rebuilds": "tree, moments, critical radii, groups and lists rebuilt on the GPU "
                        "from the bodies on the device (grav_plan_build_CUDA)",
            "rebuild_s": builds,
            "rebuild_phases_s": build_phases,
            "device_ms_per_step_median": float(np.median(steady)),
            "device_ms_first_step_after_rebuild_median": float(np.median(ms[::rebuild])),
            "wall_s": wall, "energy_first": float(e[0]), "energy_last": float(e[-1]),
            "max_abs_energy_change_over_abs_pe0": float(np.abs(e - e[0]).max() / abs(pe[0])),
            "ke_last": float(h[-1]["ke"]), "pe_first": float(pe[0]), "pe_last": float(pe[-1])}


# ---------------------------------------------------------------- configuration legs
def config_plummer64k(args, stream):
    """Plummer N = 65,536, G = 1, M = 1, a = 1, eps = 0.01, order 2 (p4cut 0),
    MAC tol 2e-5.  GPU: the batched kernels and the drop-in (grav_mn_CUDA
    per group, pMp/pQp) on the host walk's lists.  CPU leg: the reference's
    own do_gravp_avx8/do_gravpq_avx8 over the same full lists (the parity
    check, bar 1e-5 relative rms), and the FP64 direct sum on every sink."""
    import torch
    from oracle import oracle as O
    from pgrav import gravcuda as gc, host, ics
    w = WORKLOADS["plummer64k"]
    pos, m = ics.plummer(w["n"], seed=123)
    eps2 = w["eps"] ** 2
    t = host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=w["p2cut"], p4cut=0, tol=w["tol"],
                  emit_aosoa=True)
    res = {"workload": "Plummer N=65536, eps 0.01, order 2, MAC tol 2e-5", "n_bodies": int(t.n),
           "groups": int(t.ngroups),
           "interactions_per_sink": [round(float(x) / t.n, 1) for x in t.counts]}
    inter = float(t.counts.sum())
    # the reference quadrupole kernels' potential sign (-1) for the parity check
    plan_r = gc.Plan(t, eps2, quad_phi_sign=-1.0)
    ms = time_evals(plan_r, stream, 20)
    got_r = plan_r.download()
    plan_r.free()
    plan = gc.Plan(t, eps2)
    plan.eval()
    got = plan.download()
    plan.free()
    res["batched"] = {"ms": ms, "value": inter / (ms * 1e-3), "unit": UNIT}
    # drop-in: one grav_mn_CUDA per group and kind, as nln/mac.c issues them (from C)
    bt = gc.body_table(t.sorted_pos, t.points[:t.n, 3])
    packs = [(routine, sz, t.aosoa[k][0], t.aosoa[k][1])
             for k, (routine, sz) in enumerate((("pMp", 4), ("pQp", 13)))]
    first = np.ascontiguousarray(t.groups["first"], np.int64)
    count = np.ascontiguousarray(t.groups["count"], np.int32)
    secs = []
    for _ in range(3):  # the first pass sizes the slots' buffers
        d = gc.DropIn(bt.copy())
        secs.append(gc.drive_mn(d, first, count, packs, eps2))
    got_d = d.btab[:, 7:11].copy()
    el = min(secs[1:])
    res["dropin"] = {"s": el, "value": inter / el, "unit": UNIT,
                     "timing": "wall clock of the calls issued from C (lib/libmacdrive.so), first "
                               "grav_mn_CUDA to the end of WalkTerminateSinkCUDA, best of 2 "
                               "passes after one"}
    # CPU leg: the reference's own kernels over the full lists, all host threads
    if O.ref_available():
        t0 = time.perf_counter()
        ref = O.tree_eval(t, eps2, quad_kind=O.QUAD_PLUMMER, reference=True)
        el = time.perf_counter() - t0
        b_rms, b_max = rel_rms(got_r[:, :3], ref[:, :3])
        d_rms, d_max = rel_rms(got_d[:, :3], ref[:, :3])
        pb = float(np.sqrt(np.mean((got_r[:, 3] - ref[:, 3]) ** 2) / np.mean(ref[:, 3] ** 2)))
        pd = float(np.sqrt(np.mean((got_d[:, 3] - ref[:, 3]) ** 2) / np.mean(ref[:, 3] ** 2)))
        res["vs_reference_kernels"] = {
            "kernels": "do_gravp_avx8 + do_gravpq_avx8 (nln/do_grav_avx8.c, compiled unmodified)",
            "cpu_s": el, "cpu_value": inter / el, "cores": os.cpu_count(), "cpu_model": cpu_model(),
            "batched_rms_rel_acc": b_rms, "batched_max_rel_acc": b_max, "batched_rms_phi": pb,
            "dropin_rms_rel_acc": d_rms, "dropin_max_rel_acc": d_max, "dropin_rms_phi": pd,
            "bar_rms": 1e-5, "meets_target": bool(b_rms <= 1e-5 and d_rms <= 1e-5 and
                                                  pb <= 1e-5 and pd <= 1e-5)}
    ref64 = gc.direct_fp64(t.points[:t.n], np.arange(t.n), eps2)
    a_rms, a_max = rel_rms(got[:, :3], ref64[:, :3])
    res["vs_fp64_direct"] = {"sinks": int(t.n), "rms_rel_force_err": a_rms,
                             "max_rel_force_err": a_max,
                             "rms_phi_err": float(np.sqrt(np.mean((got[:, 3] - ref64[:, 3]) ** 2) /
                                                          np.mean(ref64[:, 3] ** 2)))}
    return res


def config_box128(args, stream):
    """Periodic 128^3 box (GRF, P(k) ~ k^-2.5, rms displacement 0.25
    spacing), eps = spacing/50, order 4 + Ewald (FP64-built table): the
    mixed-precision kernels (FP32 offsets from FP64 group centres,
    compensated sums) against the plain FP32 kernels (absolute FP32
    coordinates, plain sums) on the same lists; errors against the FP64
    Ewald-summed direct sum on 4096 random sinks."""
    from pgrav import gravcuda as gc, host, ics
    w = WORKLOADS["box128"]
    pos, m = ics.grf_box(w["n1d"], seed=123, slope=-2.5, rms_disp=w["rms_disp"])
    eps2 = (1.0 / w["n1d"] / 50.0) ** 2
    t = host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=w["tol"], box=1.0)
    inter = float(t.counts.sum())
    samp = np.sort(np.random.default_rng(7).choice(t.n, 4096, replace=False))
    ref = gc.direct_fp64(t.points[:t.n], samp, eps2, box=1.0)
    res = {"workload": f"periodic 128^3, order 4 + Ewald, MAC tol {w['tol']}",
           "n_bodies": int(t.n), "groups": int(t.ngroups),
           "interactions_per_sink": [round(float(x) / t.n, 1) for x in t.counts], "sinks": 4096}
    for name, plain in (("mixed", False), ("plain_fp32", True)):
        plan = gc.Plan(t, eps2, ewald=True, plain=plain)
        ms = time_evals(plan, stream, 10)
        out = plan.download()
        plan.free()
        e_rms, e_max = rel_rms(out[samp, :3], ref[:, :3])
        pe = float(np.sqrt(np.mean((out[samp, 3] - ref[:, 3]) ** 2) / np.mean(ref[:, 3] ** 2)))
        res[name] = {"ms": ms, "value": inter / (ms * 1e-3), "unit": UNIT,
                     "rms_rel_force_err": e_rms, "max_rel_force_err": e_max, "rms_phi_err": pe,
                     "meets_target": bool(e_rms <= 1e-4)}
        if name == "mixed":
            out_mixed = out
    res["plain_over_mixed_time"] = res["plain_fp32"]["ms"] / res["mixed"]["ms"]
    res["plain_over_mixed_rms_err"] = (res["plain_fp32"]["rms_rel_force_err"] /
                                       res["mixed"]["rms_rel_force_err"])
    # the reference's own periodic scheme on 32 of those sinks: every body in
    # the 125 images of the box plus FixCubeEwaldLE's order-8 local expansion
    # (the compiled nln/ewald_le2.c), where the reference library is built
    from oracle import oracle as O
    if O.ref_available():
        t0 = time.perf_counter()
        s32 = samp[::128]
        xt = (t.points[:t.n, :3].astype(np.float64) - 0.5).astype(np.float32)
        racc, rphi = O.ref_periodic_le(xt, t.points[:t.n, 3], 1.0, eps2, s32)
        e_rms, e_max = rel_rms(out_mixed[s32, :3], racc)
        d = out_mixed[s32, 3] - rphi
        sel = np.searchsorted(samp, s32)
        e_ew, _ = rel_rms(racc, ref[sel, :3])
        res["vs_reference_periodic_scheme"] = {
            "scheme": "125 images direct (FP64) + FixCubeEwaldLE order-8 local expansion "
                      "(nln/ewald_le2.c compiled unmodified), subtract_background 0",
            "sinks": int(len(s32)), "rms_rel_force_err": e_rms, "max_rel_force_err": e_max,
            "phi_offset": float(d.mean()),
            "phi_spread_over_rms_phi": float(d.std() / np.sqrt(np.mean(rphi ** 2))),
            "reference_scheme_vs_ewald_sum_rms": e_ew, "cpu_s": time.perf_counter() - t0,
            "bar": 1e-4, "meets_target": bool(e_rms <= 1e-4)}
    return res


def config_batch1024(args, stream):
    """1024 isolated systems, N log-uniform in [512, 65536], half Plummer half
    Hernquist (a = 1), eps = 0.01 a, order 4, FP32: one persistent launch per
    list kind from one length-sorted queue, tile shapes from the autotuner,
    and the graph-captured KDK step (evaluate, integrate, refit)."""
    import torch
    from pgrav import autotune as AT, gravcuda as gc
    w = WORKLOADS["batch1024"]
    t0 = time.perf_counter()
    systems, _, eps2, _ = make_problem(w)
    tree = build_tree(w, systems, None, 0.0, w["tol"])
    setup = time.perf_counter() - t0
    plan = gc.Plan(tree, eps2)
    ta = time.perf_counter()
    best, trials = AT.autotune(plan)
    search = time.perf_counter() - ta
    ms = time_evals(plan, stream, 10)
    inter = float(plan.counts().sum())
    out = plan.download()
    rng = np.random.default_rng(7)
    offs = tree.body_offsets
    pick = rng.choice(len(offs) - 1, 8, replace=False)
    got, refs = [], []
    for sidx in pick:
        lo, hi = int(offs[sidx]), int(offs[sidx + 1])
        ss = np.sort(rng.choice(hi - lo, min(hi - lo, w["sample"] // 8), replace=False))
        refs.append(gc.direct_fp64(tree.points[lo:hi], ss, eps2))
        got.append(out[lo + ss])
    e_rms, e_max = rel_rms(np.concatenate(got)[:, :3], np.concatenate(refs)[:, :3])
    plan.set_tree(tree)
    vel = torch.zeros((tree.n, 4), dtype=torch.float32, device="cuda")
    prm = torch.tensor([1e-3, 5e-4, 0.0], dtype=torch.float64, device="cuda")
    en = torch.zeros(2, dtype=torch.float64, device="cuda")
    with torch.cuda.stream(stream):
        plan.step(vel.data_ptr(), prm.data_ptr(), en.data_ptr(), stream.cuda_stream, graph=True)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(10):
            plan.step(vel.data_ptr(), prm.data_ptr(), en.data_ptr(), stream.cuda_stream,
                      graph=True)
        b.record(stream)
    torch.cuda.synchronize()
    res = {"workload": "1024 isolated systems, N log-uniform in [512, 65536], Plummer/Hernquist, "
                       "order 4, MAC tol 1e-5",
           "systems": int(len(offs) - 1), "n_bodies": int(tree.n), "groups": int(tree.ngroups),
           "host_build_s": setup, "ms": ms, "value": inter / (ms * 1e-3), "unit": UNIT,
           "launches_per_eval": plan.launches(),
           "tuning": {"chosen": {"warps_per_block": best.warps_per_block,
                                 "blocks_per_sm": best.blocks_per_sm,
                                 "chunks": [best.chunk_p, best.chunk_q, best.chunk_h]},
                      "trials": len(trials), "search_s": search,
                      "auto_ms": trials[0]["ms"], "best_ms": min(x["ms"] for x in trials)},
           "graph_kdk_step_ms": a.elapsed_time(b) / 10,
           "rms_rel_force_err": e_rms, "max_rel_force_err": e_max,
           "accuracy_sinks": int(sum(len(r) for r in refs)),
           "oracle": "each system's own FP64 direct sum (8 random systems)",
           "meets_target": bool(e_rms <= 1e-4)}
    plan.free()
    return res


def _fp64_leapfrog_loss(x0, v0, m, eps2, dt, nsteps, trees, checkers, target):
    """L = sum (x_final + v_final) . target of FP64 KDK steps (kick dt/2,
    drift dt, kick dt/2, two force evaluations per step as the autograd
    leapfrog takes them) on the lists of `trees` (one per force evaluation),
    every cell's moments recomputed in FP64 from the current bodies."""
    x, v = x0.copy(), v0.copy()
    k = 0

    def acc(xx):
        nonlocal k
        t, chk = trees[k], checkers[k]
        k += 1
        o = chk.eval(xx[t.order], m[t.order], eps2)
        a = np.empty_like(xx)
        a[t.order] = o[:, :3]
        return a

    for _ in range(nsteps):
        v = v + 0.5 * dt * acc(x)
        x = x + dt * v
        v = v + 0.5 * dt * acc(x)
    return float((x * target).sum() + (v * target).sum())


def config_adjoint(args, stream):
    """Plummer N = 2^20, order 2, eps 0.01, MAC tol 1e-5; L = sum_i w_i.a_i +
    u_i phi_i with w, u ~ N(0, 1) (seed 0).  GPU: forward and adjoint times
    (CUDA events, same lists).  CPU checks: FP64 central differences (h =
    1e-6) of an FP64 evaluation of the same lists at 64 position
    coordinates and 16 masses (only the terms that depend on the perturbed
    body are re-evaluated; the rest cancel), the FP64 direct-sum gradient on
    a separate N = 8192 Plummer system, and 16 leapfrog KDK steps (dt = 1e-3)
    checkpointed every 4 against the unsegmented backward and against FP64
    differences through the same steps."""
    import torch
    from oracle import oracle as O
    from pgrav import autograd as AG, gravcuda as gc, host, ics
    n, eps2, tol = 1 << 20, 1e-4, 1e-5
    pos, m = ics.plummer(n, seed=123)
    t = host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=7, p4cut=0, tol=tol)
    plan = gc.Plan(t, eps2)
    plan.set_tree(t)
    rng = np.random.default_rng(0)
    wu_h = rng.normal(size=(n, 4)).astype(np.float32)
    wu = torch.from_numpy(wu_h).cuda()
    grad = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    for _ in range(3):
        plan.eval(stream.cuda_stream)
        plan.adjoint(wu.data_ptr(), grad.data_ptr(), stream.cuda_stream)
    tm = {}
    for name, fn in (("forward", lambda: plan.eval(stream.cuda_stream)),
                     ("adjoint", lambda: plan.adjoint(wu.data_ptr(), grad.data_ptr(),
                                                      stream.cuda_stream))):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(5):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        tm[name] = a.elapsed_time(b) / 5
    plan.eval(stream.cuda_stream)
    plan.adjoint(wu.data_ptr(), grad.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    g = grad.cpu().numpy().astype(np.float64)
    counts = plan.counts()
    plan.free()
    res = {"workload": "Plummer N=2^20, order 2, eps 0.01, MAC tol 1e-5", "n_bodies": n,
           "interactions_per_sink": [round(float(x) / n, 1) for x in counts],
           "forward_ms": tm["forward"], "adjoint_ms": tm["adjoint"],
           "adjoint_over_forward": tm["adjoint"] / tm["forward"], "target_ratio": 2.5,
           "meets_target": bool(tm["adjoint"] / tm["forward"] <= 2.5)}
    # FP64 central differences at 64 coordinates and 16 masses
    t0 = time.perf_counter()
    chk = O.ListsFP64(t)
    sel = rng.choice(n, 64, replace=False)
    chk.select(sel)
    x = t.sorted_pos.astype(np.float64)
    mm = t.points[:n, 3].astype(np.float64)
    wv, uv = wu_h[:, :3].astype(np.float64), wu_h[:, 3].astype(np.float64)
    coords = [(s, int(rng.integers(3))) for s in range(64)]
    fdx = chk.fd_grad(x, mm, wv, uv, eps2, coords, h=1e-6)
    fdm = chk.fd_grad(x, mm, wv, uv, eps2, [(s, 3) for s in range(16)], h=1e-6, mass_rel=True)
    adx = np.array([g[sel[s], c] for s, c in coords])
    adm = g[sel[:16], 3]
    sx, sm = float(np.sqrt(np.mean(g[:, :3] ** 2))), float(np.sqrt(np.mean(g[:, 3] ** 2)))
    ex, em = float(np.abs(adx - fdx).max() / sx), float(np.abs(adm - fdm).max() / sm)
    res["fd"] = {"h": 1e-6, "coordinates": 64, "masses": 16, "cpu_s": time.perf_counter() - t0,
                 "max_err_over_grad_rms_x": ex, "max_err_over_grad_rms_m": em,
                 "rms_rel_err_x": float(np.sqrt(np.mean((adx - fdx) ** 2) / np.mean(fdx ** 2))),
                 "bar": 1e-3, "meets_target": bool(ex <= 1e-3 and em <= 1e-3),
                 "oracle": "FP64 evaluation of the same lists, cell moments from the bodies"}
    del chk, t
    # FP64 direct-sum gradient on an N = 8192 Plummer system
    n2 = 8192
    p2, m2 = ics.plummer(n2, seed=32)
    w2 = rng.normal(size=(n2, 3)).astype(np.float32)
    u2 = rng.normal(size=n2).astype(np.float32)
    pt = torch.tensor(p2, device="cuda", requires_grad=True)
    mt = torch.tensor(m2, device="cuda", requires_grad=True)
    a2, f2 = AG.gravity(pt, mt, eps2, tol=1e-6, p2cut=7, p4cut=0)
    ((torch.tensor(w2, device="cuda") * a2).sum() +
     (torch.tensor(u2, device="cuda") * f2).sum()).backward()
    gx, gm = O.direct_grad(p2, m2, w2, u2, eps2)
    exd = np.linalg.norm(pt.grad.cpu().numpy() - gx, axis=1) / np.sqrt(np.mean((gx ** 2).sum(1)))
    emd = np.abs(mt.grad.cpu().numpy() - gm) / np.sqrt(np.mean(gm ** 2))
    res["vs_direct_gradient"] = {"n_bodies": n2, "mac_tol": 1e-6,
                                 "rms_rel_err_x": float(np.sqrt(np.mean(exd ** 2))),
                                 "rms_rel_err_m": float(np.sqrt(np.mean(emd ** 2))),
                                 "bar": 1e-3,
                                 "meets_target": bool(np.sqrt(np.mean(exd ** 2)) <= 1e-3 and
                                                      np.sqrt(np.mean(emd ** 2)) <= 1e-3)}
    res["leapfrog"] = leapfrog_check(args)
    res["leapfrog_2p20"] = leapfrog_time(n, eps2, tol)
    res["headline_adjoint"] = headline_adjoint(stream, args.adjoint_workload)
    res["periodic_32"] = periodic_adjoint_check(stream)
    return res


def periodic_adjoint_check(stream, nsel=3, seed=37):
    """The adjoint of the periodic 32^3 box (order 4 + Ewald, lists built on
    the GPU): its time against the evaluation's, and FP64 central
    differences (h = 1e-6) of the oracle's evaluation of the same lists at
    nsel bodies (positions and masses), the correction summed exactly over
    each entry's bodies.  The bar is the correction's truncation (the
    kernels use cell moments and each group's Taylor series of it)."""
    import torch
    from oracle import oracle as O
    from pgrav import gravcuda as gc, host
    w = WORKLOADS["box32"]
    pos, m, eps2, box = make_problem(w)
    n = len(m)
    kw = dict(leaf_max=16, group_max=32, p2cut=w["p2cut"], p4cut=w["p4cut"], tol=w["tol"])
    res = headline_adjoint(stream, "box32")
    rng = np.random.default_rng(seed)
    wu_h = rng.normal(size=(n, 4)).astype(np.float32)
    b = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    b[:, :3] = torch.from_numpy(np.asarray(pos, np.float32)).cuda()
    b[:, 3] = torch.from_numpy(np.asarray(m, np.float32)).cuda()
    plan = gc.Plan.build(None, None, eps2, bodies=b, box=box, ewald=True, **kw)
    order = plan.order()
    wu = torch.from_numpy(wu_h[order]).cuda()
    grad = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    plan.eval(stream.cuda_stream)
    plan.adjoint(wu.data_ptr(), grad.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    g = grad.cpu().numpy().astype(np.float64)   # tree order
    plan.free()
    t0 = time.perf_counter()
    t = host.Tree(pos, m, box=box, **kw)
    assert np.array_equal(np.asarray(t.order), order)
    chk = O.ListsFP64(t, ewald=True)
    sel = rng.choice(n, nsel, replace=False)
    chk.select(sel)
    x = np.asarray(t.sorted_pos, np.float64)
    mm = np.asarray(t.points[:n, 3], np.float64)
    wt = wu_h[order].astype(np.float64)
    coords = [(s, c) for s in range(nsel) for c in (0, 1, 2, 3)]
    fd = chk.fd_grad(x, mm, wt[:, :3], wt[:, 3], eps2, coords, h=1e-6,
                     mass_rel=True).reshape(nsel, 4)
    ad = g[sel]
    sx, sm = float(np.sqrt(np.mean(g[:, :3] ** 2))), float(np.sqrt(np.mean(g[:, 3] ** 2)))
    ex = float(np.abs(ad[:, :3] - fd[:, :3]).max() / sx)
    em = float(np.abs(ad[:, 3] - fd[:, 3]).max() / sm)
    res["fd"] = {"h": 1e-6, "bodies": nsel, "coordinates": 4 * nsel, "cpu_s": time.perf_counter() - t0,
                 "max_err_over_grad_rms_x": ex, "max_err_over_grad_rms_m": em, "bar": 5e-3,
                 "meets_target": bool(ex <= 5e-3 and em <= 5e-3),
                 "oracle": "FP64 evaluation of the same lists (image shifts, order-4 cells), the "
                           "correction summed exactly over each entry's bodies"}
    res["target_ratio"] = 2.5
    res["meets_target"] = bool(res["adjoint_over_forward"] <= 2.5 and res["fd"]["meets_target"])
    return res


def headline_adjoint(stream, workload="box256", reps=2):
    """The adjoint of a periodic workload (the headline 256^3 box by default,
    order 4 + Ewald, tree and lists built on the GPU): forward and adjoint
    times with CUDA events on the same plan (the adjoint reads the
    evaluation's correction moments).  Its correctness is pinned in
    tests/test_adjoint_gpu.py against FP64 differences of the oracle on
    periodic order-4 lists with the correction."""
    import torch
    from pgrav import gravcuda as gc
    w = WORKLOADS[workload]
    pos, m, eps2, box = make_problem(w)
    n = len(m)
    bodies = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    bodies[:, :3] = torch.from_numpy(np.asarray(pos, np.float32)).cuda()
    bodies[:, 3] = torch.from_numpy(np.asarray(m, np.float32)).cuda()
    del pos
    plan = gc.Plan.build(None, None, eps2, bodies=bodies, box=box, ewald=True, leaf_max=16,
                         group_max=32, p2cut=w["p2cut"], p4cut=w["p4cut"], tol=w["tol"])
    del bodies
    g = torch.Generator(device="cuda").manual_seed(0)
    wu = torch.randn((n, 4), device="cuda", generator=g)
    grad = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    plan.eval(stream.cuda_stream)
    plan.adjoint(wu.data_ptr(), grad.data_ptr(), stream.cuda_stream)
    tm = {}
    for name, fn in (("forward", lambda: plan.eval(stream.cuda_stream)),
                     ("adjoint", lambda: plan.adjoint(wu.data_ptr(), grad.data_ptr(),
                                                      stream.cuda_stream))):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        tm[name] = a.elapsed_time(b) / reps
    finite = bool(torch.isfinite(grad).all().item())
    plan.free()
    return {"workload": f"periodic {w['n1d']}^3 box, order 4 + Ewald, lists built on the GPU",
            "n_bodies": n, "forward_ms": tm["forward"], "adjoint_ms": tm["adjoint"],
            "adjoint_over_forward": tm["adjoint"] / tm["forward"], "grad_finite": finite}


def leapfrog_time(n, eps2, tol, nsteps=16, every=4, dt=1e-3):
    """Forward and backward through 16 leapfrog KDK steps (dt = 1e-3) of the
    Plummer N = n system, checkpointed every 4 steps; every force
    evaluation builds its tree on the GPU (as the autograd function does)."""
    import torch
    from pgrav import autograd as AG, ics
    pos, m = ics.plummer(n, seed=123)
    rng = np.random.default_rng(11)
    vel = rng.normal(0, 0.2, (n, 3)).astype(np.float32)
    tgt = torch.tensor(rng.normal(size=(n, 3)), dtype=torch.float32, device="cuda")
    kw = dict(tol=tol, p2cut=7, p4cut=0, leaf_max=16, group_max=32)
    x0 = torch.tensor(pos, device="cuda", requires_grad=True)
    v0 = torch.tensor(vel, device="cuda", requires_grad=True)
    mm = torch.tensor(m, device="cuda", requires_grad=True)
    torch.cuda.reset_peak_memory_stats()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x, v = AG.leapfrog(x0, v0, mm, eps2, dt, nsteps, checkpoint_every=every, **kw)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    ((x * tgt).sum() + (v * tgt).sum()).backward()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    g = x0.grad
    return {"n_bodies": n, "steps": nsteps, "dt": dt, "checkpoint_every": every, "mac_tol": tol,
            "forward_s": t1 - t0, "backward_s": t2 - t1,
            "force_evaluations": 2 * nsteps * 3,
            "peak_torch_memory_gb": torch.cuda.max_memory_allocated() / 1e9,
            "grad_finite": bool(torch.isfinite(g).all().item()),
            "note": "wall clock; each force evaluation (forward, recomputation, backward) builds "
                    "its tree and lists on the GPU"}


def leapfrog_check(args, n=4096, nsteps=16, every=4, dt=1e-3, ncoords=4):
    """16 KDK steps through the autograd leapfrog, checkpointed every 4,
    against the unsegmented backward and against FP64 central differences
    through the same steps on the same lists (one tree per force
    evaluation, built from the base trajectory)."""
    import torch
    from oracle import oracle as O
    from pgrav import autograd as AG, host, ics
    eps2, kw = 1e-4, dict(tol=1e-4, p2cut=7, p4cut=0, leaf_max=16, group_max=32)
    pos, m = ics.plummer(n, seed=33)
    rng = np.random.default_rng(9)
    vel = rng.normal(0, 0.2, (n, 3)).astype(np.float32)
    target = rng.normal(size=(n, 3))
    tgt = torch.tensor(target, dtype=torch.float32, device="cuda")
    grads, walls = [], []
    for ck in (every, 0):
        x0 = torch.tensor(pos, device="cuda", requires_grad=True)
        v0 = torch.tensor(vel, device="cuda", requires_grad=True)
        mm = torch.tensor(m, device="cuda", requires_grad=True)
        t0 = time.perf_counter()
        x, v = AG.leapfrog(x0, v0, mm, eps2, dt, nsteps, checkpoint_every=ck, **kw)
        ((x * tgt).sum() + (v * tgt).sum()).backward()
        torch.cuda.synchronize()
        walls.append(time.perf_counter() - t0)
        grads.append(x0.grad.cpu().numpy().astype(np.float64))
    same = float(np.abs(grads[0] - grads[1]).max() / np.abs(grads[1]).max())
    # FP64 differences: the base trajectory's trees, then +-h trajectories on them
    x, v = pos.astype(np.float64), vel.astype(np.float64)
    m64 = m.astype(np.float64)
    trees, checkers = [], []

    def acc(xx):
        t = host.Tree(xx.astype(np.float32), m, **kw)
        c = O.ListsFP64(t)
        trees.append(t)
        checkers.append(c)
        o = c.eval(xx[t.order], m64[t.order], eps2)
        a = np.empty_like(xx)
        a[t.order] = o[:, :3]
        return a

    for _ in range(nsteps):
        v = v + 0.5 * dt * acc(x)
        x = x + dt * v
        v = v + 0.5 * dt * acc(x)
    h = 1e-6
    picks = [(int(b), int(c)) for b, c in zip(rng.choice(n, ncoords, replace=False),
                                                rng.integers(0, 3, ncoords))]
    fd, ad = [], []
    for b, c in picks:
        xp, xm = pos.astype(np.float64), pos.astype(np.float64)
        xp[b, c] += h
        xm[b, c] -= h
        lp = _fp64_leapfrog_loss(xp, vel.astype(np.float64), m64, eps2, dt, nsteps, trees,
                                 checkers, target)
        lm = _fp64_leapfrog_loss(xm, vel.astype(np.float64), m64, eps2, dt, nsteps, trees,
                                 checkers, target)
        fd.append((lp - lm) / (2 * h))
        ad.append(grads[0][b, c])
    fd, ad = np.array(fd), np.array(ad)
    err = float(np.abs(ad - fd).max() / np.abs(fd).max())
    return {"n_bodies": n, "steps": nsteps, "dt": dt, "checkpoint_every": every,
            "mac_tol": kw["tol"], "loss": "sum (x_final + v_final) . T, T ~ N(0, 1)",
            "wall_s_checkpointed": walls[0], "wall_s_plain": walls[1],
            "checkpointed_vs_plain_max_rel": same, "fd_coordinates": ncoords, "fd_h": h,
            "fd_max_rel_err": err, "bar": 1e-3,
            "meets_target": bool(same <= 1e-5 and err <= 1e-3),
            "note": "the FP64 differences rebuild the base trajectory's trees on the host "
                    "(nlnhost.h, bit-identical to the GPU builder's the autograd function uses)"}


def job_rate(ms_local, inter_local, world, device="cpu"):
    """Whole-job figures of `world` replicas, one per GPU, each evaluating the
    same workload: the step time is the slowest rank's (an all-reduce MAX
    over the process group when world > 1) and the interactions are every
    rank's.  Returns (ms_max, interactions per second)."""
    import torch
    ms_t = torch.tensor([float(ms_local)], dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    return ms_max, inter_local * world / (ms_max * 1e-3)


def run_reference(args, w, rank, world):
    """--impl reference: the reference's CPU kernels on the host cores."""
    if rank != 0:
        return 0
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libnlnref.so (the reference AVX kernels) is not built"}))
        return 0
    pos, m, eps2, box = make_problem(w)
    tree = build_tree(w, pos, m, box, args.tol or w["tol"])
    rates, secs = [], []
    for _ in range(args.warmup):
        cpu_reference_rate(tree, eps2, seconds=1.0)
    per_step = max(2.0, 60.0 / max(1, args.steps))
    info = None
    for _ in range(args.steps):
        info = cpu_reference_rate(tree, eps2, seconds=per_step)
        rates.append(info[0])
        secs.append(info[1])
    value = float(np.mean(rates))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            # each step is a bounded sample of the evaluation (see cpu_baseline.sample):
            # the wall time of that sample, not of a whole evaluation
            "ms_per_step": float(np.mean(secs) * 1e3),
            "full_evaluation_ms_at_this_rate": float(tree.counts.sum() / value * 1e3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": config_of(args, w, tree, box),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": info[2],
                             "cpu_model": cpu_model(), "kind": "reference", "sample": info[3]},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def tree_input_bytes(tree):
    """Bytes one evaluation reads: point and cell tables plus the index lists."""
    return (tree.points.nbytes + tree.qcells.nbytes + tree.hcells.nbytes + tree.plist.nbytes +
            tree.qlist.nbytes + tree.hlist.nbytes + tree.clist.nbytes)


def config_of(args, w, tree, box):
    c = {"workload": args.workload, "n_bodies": int(tree.n), "groups": int(tree.ngroups),
         **({"systems": int(len(tree.body_offsets) - 1)} if hasattr(tree, "body_offsets") else {}),
         "mac_tol": args.tol or w["tol"], "order": 4 if w["p4cut"] else 2,
         "periodic": bool(box > 0), "ewald": bool(w["ewald"]),
         "interactions_per_sink": [round(float(x) / tree.n, 1) for x in tree.counts],
         "l2": "inputs larger than L2 (no flush)" if tree_input_bytes(tree) >= 126e6 else
               "L2 flushed between steps (256 MB overwrite outside the step events)"}
    return c


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="box256", choices=list(WORKLOADS))
    ap.add_argument("--tol", type=float, default=0.0)
    ap.add_argument("--e2e-steps", type=int, default=3,
                    help="end-to-end calls from lists built on the host (grav_groups_CUDA)")
    ap.add_argument("--e2e-pos-steps", type=int, default=3,
                    help="end-to-end calls from positions (GPU tree build + evaluation)")
    ap.add_argument("--e2e-plain-lists", action="store_true",
                    help="end-to-end leg: copy the plain lists instead of the run-packed ones")
    ap.add_argument("--e2e-lists-in-host", action="store_true",
                    help="end-to-end leg: the kernels read the lists in place from page-locked "
                         "host memory instead of the pipelined copy")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--dropin-groups", type=int, default=2048,
                    help="also time the plain FP32 drop-in path on this many sample groups "
                         "(0: skip)")
    ap.add_argument("--kdk-steps", type=int, default=32,
                    help="graph-captured KDK steps of the kdk256 configuration (energy drift)")
    ap.add_argument("--kdk-dt", type=float, default=0.01)
    ap.add_argument("--kdk-rebuild", type=int, default=8)
    ap.add_argument("--autotune", action="store_true",
                    help="pick the tile shapes with the autotuner first (always for batch1024)")
    ap.add_argument("--configs", default="all",
                    help="configuration blocks measured after the timed region: all, none, or a "
                         "comma list of " + ",".join(ALL_CONFIGS + EXTRA_CONFIGS))
    ap.add_argument("--adjoint-workload", default="box256",
                    choices=[k for k, v in WORKLOADS.items() if v["kind"] == "box"],
                    help="the periodic workload of the adjoint blocks' forward/adjoint timing")
    args = ap.parse_args()
    configs = (list(ALL_CONFIGS) if args.configs == "all" else
               [] if args.configs == "none" else [c for c in args.configs.split(",") if c])
    unknown = [c for c in configs if c not in ALL_CONFIGS + EXTRA_CONFIGS]
    if unknown:
        ap.error(f"unknown configuration(s) {unknown}")
    w = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, w, rank, world)

    import torch
    import torch.distributed as dist
    from datetime import timedelta
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
    from pgrav import gravcuda as gc

    # ---- setup (untimed): ICs, host tree + walk, device plan
    t0 = time.perf_counter()
    pos, m, eps2, box = make_problem(w)
    t1 = time.perf_counter()
    tree = build_tree(w, pos, m, box, args.tol or w["tol"])
    t2 = time.perf_counter()
    plan = gc.Plan(tree, eps2, ewald=w["ewald"] and box > 0)
    plan.set_timing(True)
    t3 = time.perf_counter()
    log(f"[bench] ics {t1 - t0:.1f}s tree+walk {t2 - t1:.1f}s upload {t3 - t2:.1f}s "
        f"groups {tree.ngroups} counts/sink {np.round(tree.counts / tree.n, 1)}")
    tuning = None
    if args.autotune or w["kind"] == "batch":
        from pgrav import autotune as AT
        ta = time.perf_counter()
        best, trials = AT.autotune(plan)
        tuning = {"chosen": {"warps_per_block": best.warps_per_block,
                             "blocks_per_sm": best.blocks_per_sm,
                             "chunks": [best.chunk_p, best.chunk_q, best.chunk_h],
                             "ewald_side": best.ewald_side},
                  "trials": len(trials), "search_s": time.perf_counter() - ta,
                  "best_ms": min(t["ms"] for t in trials),
                  "auto_ms": trials[0]["ms"]}
        plan.set_timing(True)
    stream = torch.cuda.Stream()
    for _ in range(max(3, args.warmup)):
        plan.eval(stream.cuda_stream)
    torch.cuda.synchronize()

    # ---- timed region: one event pair per step; when the step's inputs fit
    # in L2 (126 MB), a 256 MB buffer is overwritten between steps, outside
    # the events, so every step starts cold
    flush = tree_input_bytes(tree) < 126e6
    scratch = torch.empty(64 << 20, dtype=torch.float32, device="cuda") if flush else None
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for a, b in evs:
                if flush:
                    scratch.zero_()
                a.record(stream)
                plan.eval(stream.cuda_stream)
                b.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
    kms = plan.kernel_ms()
    clocks = clk.summary()
    counts = plan.counts().astype(np.float64)
    inter = float(counts.sum())
    ms_max, value = job_rate(ms, inter, world, "cuda")

    # ---- roofline of the dominant kernel (FP32 CUDA-core pipe): the peak is
    # measured here (FMA microkernel, grav_fp32_peak_CUDA), after the timed region
    peaks, peak_src = measured_peaks()
    sm_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    derived = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12  # TFLOP/s at the nominal clock
    with ClockSampler(local) as pclk:
        fp32_peak = gc.fp32_peak()
    peak_clocks = pclk.summary()
    kflops = {"hexa": counts[3] * FLOPS[3], "quad": counts[2] * FLOPS[2],
              "point": (counts[0] + counts[1]) * FLOPS[0]}
    dom = max(("hexa", "quad", "point"), key=lambda k: kms[k])
    achieved = kflops[dom] / (kms[dom] * 1e-3) / 1e12
    total_tflops = float((counts * FLOPS).sum() / (ms * 1e-3) / 1e12)
    roofline = {"bound": "fp32", "kernel": f"k_batch<{dom}>", "achieved": achieved,
                "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                "traffic": float(DRAM_BYTES_PER_INTERACTION[dom] * (
                    counts[3] if dom == "hexa" else counts[2] if dom == "quad" else counts[0] + counts[1])),
                "traffic_note": "bytes per launch: DRAM bytes per interaction of one ncu capture "
                                "of this kernel on the periodic 128^3 box times this launch's "
                                "interactions",
                "peak_source": ("measured in this run: FP32 FMA microkernel "
                                "(grav_fp32_peak_CUDA, 8 independent chains per thread, 2048 "
                                "threads per SM, scalar and paired f32x2 FMAs, the larger of "
                                "their best of 5 launches, CUDA events)"),
                "peak_clocks": peak_clocks,
                "peak_derived": derived,
                "peak_derived_source": (f"148 SMs x 128 FP32 lanes x 2 x {sm_mhz:.0f} MHz "
                                        f"(sm_max_mhz of {peak_src} MEASURED_PEAKS.json)"),
                "frac_of_derived": achieved / derived,
                "kernel_ms": {k: round(v, 4) for k, v in kms.items()},
                "step_tflops": total_tflops, "step_frac": total_tflops / fp32_peak}

    # ---- accuracy against the FP64 direct sum (untimed; run after the end-to-end
    # leg from positions so that leg starts on a quiet device)
    def measure_accuracy(out):
        acc = None
        if not args.no_accuracy and rank == 0:
            rng = np.random.default_rng(7)
            if w["kind"] == "batch":
                # each system's own FP64 direct sum, on sinks of 8 random systems
                offs = tree.body_offsets
                pick = rng.choice(len(offs) - 1, 8, replace=False)
                got, refs = [], []
                for sidx in pick:
                    lo, hi = int(offs[sidx]), int(offs[sidx + 1])
                    ss = np.sort(rng.choice(hi - lo, min(hi - lo, w["sample"] // 8), replace=False))
                    refs.append(gc.direct_fp64(tree.points[lo:hi], ss, eps2))
                    got.append(out[lo + ss])
                ref = np.concatenate(refs)
                gotv = np.concatenate(got)
                samp = None
            else:
                samp = np.sort(rng.choice(tree.n, min(w["sample"], tree.n), replace=False))
                ref = gc.direct_fp64(tree.points[:tree.n], samp, eps2, box=box)
                gotv = out[samp]
            e = np.linalg.norm(gotv[:, :3] - ref[:, :3], axis=1) / np.linalg.norm(ref[:, :3], axis=1)
            # potential: rms error over rms potential (a periodic potential can pass through zero)
            pe = np.sqrt(np.mean((gotv[:, 3] - ref[:, 3]) ** 2) / np.mean(ref[:, 3] ** 2))
            acc = {"rms_rel_force_err": float(np.sqrt(np.mean(e * e))),
                   "max_rel_force_err": float(e.max()),
                   "p99_rel_force_err": float(np.quantile(e, 0.99)),
                   "rms_phi_err_over_rms_phi": float(pe),
                   "sinks": int(len(ref)),
                   "target_rms": 1e-4, "meets_target": bool(np.sqrt(np.mean(e * e)) <= 1e-4),
                   "oracle": "FP64 direct sum" + (" with Ewald images" if box > 0 else "")}
        return acc

    launches = plan.launches()
    out_plan = plan.download() if rank == 0 else None
    batch_kdk = None
    if w["kind"] == "batch" and rank == 0:
        # the graph-captured KDK step of the batch (evaluate, integrate, refit)
        plan.set_tree(tree)
        vel = torch.zeros((tree.n, 4), dtype=torch.float32, device="cuda")
        prm = torch.tensor([1e-3, 5e-4, 0.0], dtype=torch.float64, device="cuda")
        en = torch.zeros(2, dtype=torch.float64, device="cuda")
        with torch.cuda.stream(stream):
            plan.step(vel.data_ptr(), prm.data_ptr(), en.data_ptr(), stream.cuda_stream, graph=True)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(args.steps):
                plan.step(vel.data_ptr(), prm.data_ptr(), en.data_ptr(), stream.cuda_stream,
                          graph=True)
            b.record(stream)
        torch.cuda.synchronize()
        batch_kdk = {"graph_step_ms": a.elapsed_time(b) / args.steps, "steps": args.steps,
                     "step": "evaluate + integrate + refit, one CUDA graph launch",
                     "systems": int(len(tree.body_offsets) - 1)}
    plan.free()   # the end-to-end leg uploads its own copy

    # ---- end to end from positions: positions in host memory to forces in host
    # memory in one call (grav_build_eval_CUDA): bodies to the device, tree,
    # moments, critical radii, sink groups and lists built there, evaluation,
    # results back in the bodies' order.  The reference arm has no comparable
    # leg: it times its kernels on lists its host walk built.
    e2e_pos = None
    if args.e2e_pos_steps > 0 and w["kind"] != "batch":
        import torch as _t
        nb = len(pos)
        bbuf = _t.empty((nb, 4), dtype=_t.float32, pin_memory=True).numpy()
        bbuf[:, :3] = pos
        bbuf[:, 3] = m
        obuf = _t.empty((nb, 4), dtype=_t.float32, pin_memory=True).numpy()
        kw = dict(leaf_max=16, group_max=32, p2cut=w["p2cut"], p4cut=w["p4cut"],
                  tol=args.tol or w["tol"])
        ew = w["ewald"] and box > 0
        gc.build_eval(bbuf, eps2, box=box, ewald=ew, out=obuf, **kw)  # warm-up
        walls, phases = [], []
        for _ in range(args.e2e_pos_steps):
            ta = time.perf_counter()
            gc.build_eval(bbuf, eps2, box=box, ewald=ew, out=obuf, **kw)
            walls.append(time.perf_counter() - ta)
            phases.append(gc.build_eval_phases())
        e2e_s = float(np.median(walls))
        mid = int(np.argsort(walls)[len(walls) // 2])
        same = bool(out_plan is not None and np.array_equal(obuf[tree.order], out_plan))
        e2e_pos = {"value": inter * world / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(bbuf.nbytes), "d2h_bytes_per_step": int(obuf.nbytes),
               "ms_per_step": e2e_s * 1e3, "steps": args.e2e_pos_steps,
               "timing": "wall clock around grav_build_eval_CUDA: bodies (page-locked) to the "
                         "device, tree + moments + critical radii + groups + MAC walk on the GPU, "
                         "evaluation, (ax, ay, az, phi) back in the input order",
               "walls_s": walls, "phases_s": phases[mid],
               "equals_plan_output": same}
        gc.lib().grav_groups_release_CUDA()

    acc = measure_accuracy(out_plan)

    # ---- end to end through the drop-in boundary: lists built by the host walk
    # (as the reference's walk builds them) in page-locked host memory, forces
    # back in host memory, one grav_groups_CUDA call per step
    e2e = None
    host = out = None
    pack_s = None
    if args.e2e_steps > 0:
        packed = not (args.e2e_plain_lists or args.e2e_lists_in_host)
        if packed:
            tp = time.perf_counter()
            tree.pack()   # list building: the walk's lists in run-packed form
            pack_s = time.perf_counter() - tp
        host = gc.pinned_problem(tree, lists_in_host=args.e2e_lists_in_host, packed=packed)
        out = host.out
        torch.cuda.synchronize()
        gc.groups_eval_problem(host, eps2, box, ewald=w["ewald"] and box > 0)  # warm-up
        walls, phases = [], []
        for _ in range(args.e2e_steps):
            ta = time.perf_counter()
            gc.groups_eval_problem(host, eps2, box, ewald=w["ewald"] and box > 0)
            torch.cuda.synchronize()
            walls.append(time.perf_counter() - ta)
            phases.append(gc.groups_phases())
        e2e_s = float(np.median(walls))
        mid = int(np.argsort(walls)[len(walls) // 2])
        e2e = {"value": inter * world / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(host.h2d_bytes), "d2h_bytes_per_step": int(out.nbytes),
               "ms_per_step": e2e_s * 1e3, "steps": args.e2e_steps,
               "timing": "wall clock around grav_groups_CUDA (upload, evaluate, download)",
               "walls_s": walls, "phases_s": phases[mid],
               "lists": ("read by the kernels in place from page-locked host memory over PCIe "
                         "(every step; tables copied at upload)" if args.e2e_lists_in_host else
                         ("run-packed (nln_tree_pack), " if packed else "plain, ") +
                         "copied from page-locked host memory group range by group range on a "
                         "copy stream, overlapped with the evaluation of the ranges already "
                         "copied (every step)" + ("; unpacked on the device" if packed else "")),
               "host_pack_s": pack_s}
        gc.lib().grav_groups_release_CUDA()  # the end-to-end call's kept list buffer

    dropin = None
    if rank == 0 and args.dropin_groups > 0 and w["kind"] != "batch":
        rate, el, sample = dropin_rate(tree, eps2, max_groups=args.dropin_groups)
        newt_ms = kms["hexa"] + kms["quad"] + kms["point"]
        batched = inter / (newt_ms * 1e-3)
        dropin = {"value": rate, "unit": UNIT, "seconds": el, "sample": sample,
                  "batched_newtonian_value": batched,
                  "batched_over_dropin": batched / rate,
                  "note": "batched: the three list kernels' event time (no Ewald) over all groups"}

    cpu = None
    if rank == 0 and args.cpu_seconds > 0:
        info = cpu_reference_rate(tree, eps2, seconds=args.cpu_seconds)
        if info:
            cpu = {"value": info[0], "unit": UNIT, "cores": info[2], "cpu_model": cpu_model(),
                   "kind": "reference", "sample": info[3]}

    cfg = config_of(args, w, tree, box)
    # the configuration legs build their own trees: release this step's host
    # lists and pinned copies (and torch's cache of pinned blocks) first
    host = out = tree = None
    import gc as pygc
    pygc.collect()
    empty_host = getattr(torch._C, "_host_emptyCache", None)
    if empty_host:
        empty_host()
    blocks = {}
    if rank == 0:
        for name in configs:
            log(f"[bench] configuration {name}")
            tc = time.perf_counter()
            try:
                if name == "kdk256":
                    if w["kind"] != "box":
                        continue
                    blocks[name] = kdk_run(w, pos, m, eps2, box, args.tol or w["tol"],
                                           args.kdk_steps, args.kdk_dt, args.kdk_rebuild)
                else:
                    fn = {"plummer64k": config_plummer64k, "box128": config_box128,
                          "batch1024": config_batch1024, "adjoint": config_adjoint,
                          "adjoint_periodic": lambda a, st: headline_adjoint(
                              st, a.adjoint_workload)}[name]
                    blocks[name] = fn(args, stream)
            except Exception as exc:  # one failing leg must not hide the others
                blocks[name] = {"error": f"{type(exc).__name__}: {exc}"}
            blocks.setdefault(name, {})["leg_wall_s"] = time.perf_counter() - tc
            pygc.collect()
            torch.cuda.empty_cache()

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms_max,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 (FP64 centres, compensated sums)", "data": "synthetic (seeded)",
                "config": cfg, "gpu_launches": launches * args.steps,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "e2e_from_positions": e2e_pos,
                "clocks": clocks,
                "accuracy": acc,
                "host_setup_s": {"ics": t1 - t0, "tree_walk": t2 - t1, "upload": t3 - t2}}
        if dropin:
            line["dropin"] = dropin
        if tuning:
            line["tuning"] = tuning
        if batch_kdk:
            line["batch_kdk"] = batch_kdk
        if blocks:
            line["configs"] = blocks
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
