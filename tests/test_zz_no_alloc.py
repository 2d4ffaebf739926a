"""grav_groups_eval_dev_CUDA, the entry point that allocates no device
memory (its scratch is a static device array), against the plan path
(grav_groups_upload_CUDA + grav_groups_eval_CUDA) on the same problem.

With lists left unsplit the plan path also runs one work item per group
and list kind and sums the partials in the same order; its order-4 kernel
evaluates records in pairs with the terms in another order, so the two
agree to FP32 rounding (relative force differences below 1e-5), and the
two calls in a row agree bit for bit, which checks that nothing carries
over in the scratch between calls.  This file sorts last so that the GPU
case also runs after every other GPU test in one process."""
import ctypes

import numpy as np
import pytest


def _tree():
    from pgrav import host, ics
    pos, m = ics.plummer(20000, seed=11)
    return host.Tree(pos, m, leaf_max=16, group_max=32, p2cut=7, p4cut=20, tol=1e-4)


def test_dev_entry_rejects_problems_beyond_the_scratch():
    """The size check comes before any CUDA call, so this runs without a GPU."""
    from pgrav import gravcuda as gc
    L = gc.lib()
    p = gc.Problem()
    p.nbodies, p.ncells, p.ngroups = 10 ** 7, 10 ** 6, 10 ** 6
    fake = 1 << 20  # aligned, never dereferenced: the call must refuse first
    p.points = p.groups = p.pptr = p.plist = fake
    rc = L.grav_groups_eval_dev_CUDA(ctypes.byref(p), fake, None)
    assert rc == -1
    msg = L.gravcuda_status_string().decode()
    L.gravcuda_clear_status()
    assert "static scratch" in msg and "at most" in msg, msg
    # and the Ewald correction is refused
    p.ngroups, p.box, p.ewald = 10, 1.0, 1
    assert L.grav_groups_eval_dev_CUDA(ctypes.byref(p), fake, None) == -1
    assert "Ewald" in L.gravcuda_status_string().decode()
    L.gravcuda_clear_status()


@pytest.mark.gpu
def test_dev_entry_matches_plan_on_two_calls():
    import torch
    from pgrav import gravcuda as gc
    t = _tree()
    assert len(t.plist) and len(t.qlist) and len(t.hlist)
    eps2 = 1e-4
    whole = 1 << 24   # no list splitting in the plan path
    plan = gc.Plan(t, eps2, tuning=gc.Tuning(8, whole, whole, whole, 0, 0))
    plan.eval()
    ref = plan.download()
    plan.free()

    dev = torch.device("cuda:0")
    keep = []

    def on_device(a):
        x = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)).to(dev)
        keep.append(x)
        return x.data_ptr()

    p = gc.Problem()
    p.nbodies, p.ncells, p.ngroups = t.n, t.ncells, t.ngroups
    p.points, p.qcells, p.hcells = on_device(t.points), on_device(t.qcells), on_device(t.hcells)
    p.groups = on_device(t.groups)
    p.pptr, p.qptr, p.hptr = on_device(t.ptr[0]), on_device(t.ptr[1]), on_device(t.ptr[2])
    p.plist, p.qlist, p.hlist = on_device(t.plist), on_device(t.qlist), on_device(t.hlist)
    p.eps2, p.box, p.quad_phi_sign, p.ewald = eps2, 0.0, 1.0, 0
    out = torch.empty((t.n, 4), dtype=torch.float32, device=dev)
    first = None
    for call in range(2):
        out.fill_(float("nan"))
        gc.check(gc.lib().grav_groups_eval_dev_CUDA(ctypes.byref(p), out.data_ptr(), None))
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), f"call {call}"
        ra = np.linalg.norm(got[:, :3] - ref[:, :3], axis=1) / np.linalg.norm(ref[:, :3], axis=1)
        rp = np.abs(got[:, 3] - ref[:, 3]) / np.abs(ref[:, 3])
        assert ra.max() < 1e-5 and np.sqrt(np.mean(ra * ra)) < 2e-6, (call, ra.max())
        assert rp.max() < 1e-5, (call, rp.max())
        if first is None:
            first = got.copy()
        else:
            assert np.array_equal(got, first), "the second call differs from the first"
