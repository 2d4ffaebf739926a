"""torch.autograd.Function over the tree-gravity evaluation and its
hand-written adjoint (grav_plan_adjoint_CUDA), and a leapfrog integrator
that backpropagates through KDK steps with step-level checkpointing.

The forward builds the tree and the interaction lists on the GPU from the
current positions (grav_plan_build_CUDA) and evaluates them; the backward
rebuilds the same (deterministic) tree from the saved inputs, holds those lists fixed
(the tree is piecewise constant in the positions) and returns dL/dx and
dL/dm for any loss whose gradient with respect to the outputs
(accelerations, potentials) autograd supplies.  Only the inputs are saved,
so checkpointed segments keep no device tables alive.  Every list kind is
covered: bodies, monopole, quadrupole and order-4 cells, and in periodic
boxes (box > 0, ewald=True) the image shifts and the Ewald correction.
"""
import torch

from . import gravcuda as gc
from .step import memcpy_d2d


class TreeGravity(torch.autograd.Function):
    """(acc (n, 3), phi (n,)) of bodies at pos (n, 3) with masses mass (n,)."""

    @staticmethod
    def _plan(pos, mass, eps2, kw):
        """The plan built on the GPU and tree position -> input index (device)."""
        n = pos.shape[0]
        bodies = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        bodies[:, :3] = pos.detach().to("cuda", torch.float32)
        bodies[:, 3] = mass.detach().to("cuda", torch.float32)
        torch.cuda.synchronize()
        plan = gc.Plan.build(None, None, float(eps2), bodies=bodies, **kw)
        order = torch.from_numpy(plan.order()).cuda()
        return order, plan

    @staticmethod
    def forward(ctx, pos, mass, eps2, tree_kw):
        kw = dict(tree_kw or {})
        order, plan = TreeGravity._plan(pos, mass, eps2, kw)
        plan.eval()
        n = pos.shape[0]
        out_t = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        memcpy_d2d(out_t.data_ptr(), plan.output_ptr(), n * 16)
        plan.free()
        out = torch.empty_like(out_t)
        out[order] = out_t
        ctx.save_for_backward(pos, mass)
        ctx.eps2, ctx.kw = eps2, kw
        dev = pos.device
        return out[:, :3].to(dev), out[:, 3].to(dev)

    @staticmethod
    def backward(ctx, gacc, gphi):
        pos, mass = ctx.saved_tensors
        order, plan = TreeGravity._plan(pos, mass, ctx.eps2, ctx.kw)
        if ctx.kw.get("ewald"):
            plan.eval()   # the correction's adjoint reads the evaluation's group moments
        n = pos.shape[0]
        wu = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        if gacc is not None:
            wu[:, :3] = gacc.detach().to("cuda", torch.float32)[order]
        if gphi is not None:
            wu[:, 3] = gphi.detach().to("cuda", torch.float32)[order]
        grad_t = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        plan.adjoint(wu.data_ptr(), grad_t.data_ptr(), torch.cuda.current_stream().cuda_stream)
        grad = torch.empty_like(grad_t)
        grad[order] = grad_t
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
    and each segment's forces are recomputed in the backward pass.  In a
    periodic box (tree_kw box > 0) drifted positions wrap into [0, box)."""
    from torch.utils.checkpoint import checkpoint
    box = float(tree_kw.get("box", 0.0) or 0.0)

    def one(x, v):
        a, _ = gravity(x, mass, eps2, **tree_kw)
        v = v + 0.5 * dt * a
        x = x + dt * v
        if box > 0:
            x = torch.remainder(x, box)
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
