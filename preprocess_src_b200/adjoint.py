"""Gradients of the final cell shape through the step, as a torch.autograd.Function.

``ShapeRun`` is a thin wrapper over the adjoint entry points of the C ABI
(``rbc_adjoint_record`` / ``rbc_adjoint_backward``): its forward restores a
saved initial state, sets the coefficients from ``theta = (Gs, C, g)``, runs
``nsteps`` steps with a checkpoint every ``ckpt_every`` steps and returns the
final vertex positions as a ``[3, nv]`` float64 tensor (x, y, z rows of the
reference's cel->x/y/z).  Its backward takes any upstream gradient of those
positions and returns dL/dtheta from one reverse sweep (and dL/dx0 when the
initial positions are an input).

The coefficient map is the one of ``configs.base_params``: P = g / 2 and
B = Gs / 2 in lattice units (dx = dt = 1), so dL/dg = dL/dP / 2 and
dL/dGs = dL/dB / 2.
"""
from __future__ import annotations

import numpy as np
import torch

from .step import Simulation


class InitialState:
    """Snapshot of a simulation's state (lattice, cells, iteration) that a
    run starts from."""

    def __init__(self, sim: Simulation):
        self.fn = sim.export_lattice(fn=True, macro=False)["fn"]
        c = sim.export_cells()
        self.x, self.y, self.z, self.xd, self.gx = c["x"], c["y"], c["z"], c["xd"], c["gx"]
        self.iter = sim.iter

    def restore(self, sim: Simulation, x0: np.ndarray | None = None):
        """x0: optional [3, nv] initial positions replacing the saved ones
        (cel->x and fem->xd both)."""
        sim.import_lattice(self.fn)
        if x0 is None:
            sim.import_cells(self.x, self.y, self.z, xd=self.xd, gx=self.gx)
        else:
            x0 = np.asarray(x0, dtype=np.float64)
            sim.import_cells(x0[0], x0[1], x0[2], xd=x0.T.reshape(-1), gx=self.gx)
        sim.iter = self.iter


class ShapeRun(torch.autograd.Function):
    """final_positions = ShapeRun.apply(theta, x0, sim, init, nsteps, ckpt_every, binomial)

    theta: float64 tensor [3] = (Gs, C, g); x0: float64 tensor [3, nv] of
    initial positions, or None for the saved ones.  binomial: None for a
    checkpoint every ckpt_every steps, or (unit, snapshots) for binomial
    checkpointing over units of that many steps with that many snapshot slots
    (memory independent of nsteps).  The simulation must not be stepped
    between this forward and its backward (the backward reads the checkpoints
    the forward recorded)."""

    @staticmethod
    def forward(ctx, theta, x0, sim: Simulation, init: InitialState, nsteps: int, ckpt_every: int = 100,
                binomial=None):
        Gs, C_, g = (float(v) for v in theta.detach().cpu().tolist())
        sim.set_coefficients(P=g / 2.0, B=Gs / 2.0, C_=C_)
        init.restore(sim, None if x0 is None else x0.detach().cpu().numpy())
        if binomial is None:
            sim.adjoint_record(nsteps, ckpt_every)
        else:
            sim.adjoint_record_binomial(nsteps, *binomial)
        c = sim.export_cells()
        ctx.sim = sim
        ctx.x0_given = x0 is not None
        ctx.token = (id(sim), sim.iter)
        return torch.from_numpy(np.stack([c["x"], c["y"], c["z"]])).to(theta.device)

    @staticmethod
    def backward(ctx, grad_out):
        sim = ctx.sim
        if (id(sim), sim.iter) != ctx.token:
            raise RuntimeError("the simulation was stepped after the forward of this ShapeRun")
        go = grad_out.detach().to(torch.float64).cpu().numpy()
        r = sim.adjoint_backward(go[0], go[1], go[2], want_x0=ctx.x0_given)
        dP, dB, dC = r["grad"]
        dtheta = torch.tensor([dB / 2.0, dC, dP / 2.0], dtype=torch.float64, device=grad_out.device)
        dx0 = torch.from_numpy(r["dx0"]).to(grad_out.device) if ctx.x0_given else None
        return dtheta, dx0, None, None, None, None, None


def shape_loss(final: torch.Tensor, target: torch.Tensor, LX: float, LZ: float) -> torch.Tensor:
    """Mean over vertices of the squared distance to the target, with the
    minimum image in the periodic x and z."""
    d = final - target
    L = torch.tensor([LX, 0.0, LZ], dtype=d.dtype, device=d.device)[:, None]
    per = torch.tensor([1.0, 0.0, 1.0], dtype=d.dtype, device=d.device)[:, None]
    d = d - per * L * torch.round(d / torch.where(L > 0, L, torch.ones_like(L)))
    return (d * d).sum(dim=0).mean()
