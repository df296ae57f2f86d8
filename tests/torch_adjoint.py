"""Test-only torch.autograd.Function bindings of the CUDA adjoint (cvr_adj_*).

`TrajectoryLoss.apply(pos0, vel0, eps, sigma, charge, engine)` returns
J = (1/M) sum_{t=1..M} U(r_t) as a 0-d float64 tensor; its backward hands
back the adjoint kernel's gradient (computed in the same call) scaled by the
incoming cotangent.  `Forces.apply(pos, eps, sigma, charge, engine)` returns
F(pos); its backward is the hand-written VJP kernel.

The tensors live on the host (the engine copies them to its own device
buffers): this is a test harness, not a training API.

eps and sigma must be symmetric.  The C ABI reports, for an off-diagonal
entry, the derivative with respect to the shared value; torch treats the two
entries as separate inputs, so the backward hands each entry half of it
(summed back by any symmetric construction such as `sym2`).
"""
import numpy as np
import torch

from caviar_b200 import _abi


def sym2(v):
    """[v0, v1, v2] -> [[v0, v1], [v1, v2]] (differentiable)."""
    return torch.stack([torch.stack([v[0], v[1]]), torch.stack([v[1], v[2]])])


def _entrywise(g):
    g = np.array(g, copy=True)
    off = ~np.eye(g.shape[0], dtype=bool)
    g[off] *= 0.5
    return torch.from_numpy(g)


class Engine:
    """A cvr_adj context plus the fixed part of the system (types, cutoffs)."""

    def __init__(self, system, precision=_abi.PREC_MIXED, nsteps=10, checkpoint_every=5):
        self.s = system
        self.a = _abi.Adjoint.from_system(system, precision)
        self.nsteps = nsteps
        self.K = checkpoint_every

    def load(self, pos, vel, eps, sigma, charge):
        s = self.s
        self.a.set_params(charge.detach().numpy(), eps.detach().numpy(), sigma.detach().numpy(), s.rc_lj, s.alpha,
                          s.rc_r, s.kmax, s.k_e, s.dt)
        self.a.set_state(pos.detach().numpy(), vel.detach().numpy() if vel is not None else np.zeros_like(s.pos),
                         s.type)


class TrajectoryLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos0, vel0, eps, sigma, charge, engine):
        engine.load(pos0, vel0, eps, sigma, charge)
        J, g = engine.a.loss_grad(engine.nsteps, engine.K)
        ctx.save_for_backward(torch.from_numpy(g["pos"]), torch.from_numpy(g["vel"]), _entrywise(g["eps"]),
                              _entrywise(g["sigma"]), torch.from_numpy(g["charge"].copy()))
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        gp, gv, ge, gs, gq = ctx.saved_tensors
        return gJ * gp, gJ * gv, gJ * ge, gJ * gs, gJ * gq, None


class Forces(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, eps, sigma, charge, engine):
        engine.load(pos, None, eps, sigma, charge)
        f, _, _ = engine.a.forces()
        ctx.engine = engine
        ctx.save_for_backward(pos, eps, sigma, charge)
        return torch.from_numpy(f)

    @staticmethod
    def backward(ctx, gF):
        pos, eps, sigma, charge = ctx.saved_tensors
        engine = ctx.engine
        engine.load(pos, None, eps, sigma, charge)
        w, g = engine.a.force_vjp(gF.detach().contiguous().numpy())
        return torch.from_numpy(w), _entrywise(g["eps"]), _entrywise(g["sigma"]), \
            torch.from_numpy(g["charge"].copy()), None
