"""torch.autograd.Function over the tree-gravity evaluation and its
hand-written adjoint (grav_plan_adjoint_CUDA), and a leapfrog integrator
that backpropagates through KDK steps with step-level checkpointing.

The forward builds the tree and the interaction lists on the host from the
current positions and evaluates them on the GPU; the backward rebuilds the
same (deterministic) tree from the saved inputs, holds those lists fixed
(the tree is piecewise constant in the positions) and returns dL/dx and
dL/dm for any loss whose gradient with respect to the outputs
(accelerations, potentials) autograd supplies.  Only the inputs are saved,
so checkpointed segments keep no device tables alive.  Isolated systems
with monopole and quadrupole cells (p4cut = 0).
"""
import numpy as np
import torch

from . import gravcuda as gc
from . import host


class TreeGravity(torch.autograd.Function):
    """(acc (n, 3), phi (n,)) of bodies at pos (n, 3) with masses mass (n,)."""

    @staticmethod
    def _plan(pos, mass, eps2, kw):
        p = pos.detach().to("cpu", torch.float32).numpy()
        m = mass.detach().to("cpu", torch.float32).numpy()
        tree = host.Tree(p, m, **kw)
        plan = gc.Plan(tree, float(eps2))
        plan.set_tree(tree)
        return tree, plan

    @staticmethod
    def forward(ctx, pos, mass, eps2, tree_kw):
        kw = dict(tree_kw or {})
        kw.setdefault("p4cut", 0)
        if kw["p4cut"]:
            raise ValueError("the adjoint covers monopole and quadrupole cells (p4cut = 0)")
        tree, plan = TreeGravity._plan(pos, mass, eps2, kw)
        plan.eval()
        out_t = torch.from_numpy(plan.download())
        plan.free()
        order = torch.from_numpy(tree.order)
        out = torch.empty_like(out_t)
        out[order] = out_t
        ctx.save_for_backward(pos, mass)
        ctx.eps2, ctx.kw = eps2, kw
        dev = pos.device
        return out[:, :3].to(dev), out[:, 3].to(dev)

    @staticmethod
    def backward(ctx, gacc, gphi):
        pos, mass = ctx.saved_tensors
        tree, plan = TreeGravity._plan(pos, mass, ctx.eps2, ctx.kw)
        n = tree.n
        order = torch.from_numpy(tree.order)
        wu = torch.zeros((n, 4), dtype=torch.float32)
        if gacc is not None:
            wu[:, :3] = gacc.detach().to("cpu", torch.float32)[order]
        if gphi is not None:
            wu[:, 3] = gphi.detach().to("cpu", torch.float32)[order]
        wu = wu.cuda()
        grad_t = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        plan.adjoint(wu.data_ptr(), grad_t.data_ptr(), torch.cuda.current_stream().cuda_stream)
        grad = torch.empty_like(grad_t)
        grad[order.cuda()] = grad_t
        torch.cuda.current_stream().synchronize()
        plan.free()
        dev = gacc.device if gacc is not None else gphi.device
        return grad[:, :3].to(dev), grad[:, 3].to(dev), None, None


def gravity(pos, mass, eps2, **tree_kw):
    """Accelerations and potentials (G = 1), differentiable in pos and mass."""
    return TreeGravity.apply(pos, mass, eps2, tree_kw)


def leapfrog(pos, vel, mass, eps2, dt, nsteps, checkpoint_every=0, **tree_kw):
    """KDK leapfrog (kick dt/2, drift dt, kick dt/2 per step) through the
    differentiable force; with checkpoint_every = k the steps run in segments
    of k under torch.utils.checkpoint, so only segment boundaries are stored
    and each segment's forces are recomputed in the backward pass."""
    from torch.utils.checkpoint import checkpoint

    def one(x, v):
        a, _ = gravity(x, mass, eps2, **tree_kw)
        v = v + 0.5 * dt * a
        x = x + dt * v
        a, _ = gravity(x, mass, eps2, **tree_kw)
        v = v + 0.5 * dt * a
        return x, v

    def segment(x, v, k):
        for _ in range(k):
            x, v = one(x, v)
        return x, v

    x, v = pos, vel
    done = 0
    while done < nsteps:
        k = min(checkpoint_every or nsteps, nsteps - done)
        if checkpoint_every:
            x, v = checkpoint(segment, x, v, k, use_reentrant=False)
        else:
            x, v = segment(x, v, k)
        done += k
    return x, v
