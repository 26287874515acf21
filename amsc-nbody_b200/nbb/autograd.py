"""torch.autograd wrapper of the hand-written rollout adjoint.

``rollout(mass, positions, velocities, config, steps, checkpoint_every)``
returns the final positions and velocities of a leapfrog rollout and
differentiates through libnbb's own reverse pass (nbb_sim_rollout /
nbb_sim_backward); torch records nothing of the step itself.  Tensors are
FP64, shaped (n,) for masses and (3, n) for positions and velocities, on the
CPU or on the GPU (copied through host memory).  The wrapper exists to check
the adjoint against finite differences and the direct-sum adjoint.
"""
from __future__ import annotations

import numpy as np
import torch

from .api import Simulation, SimulationConfig
from .ics import ParticleData


class RolloutFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mass, positions, velocities, config: SimulationConfig, steps: int, checkpoint_every: int):
        m = mass.detach().cpu().numpy()
        p = positions.detach().cpu().numpy()
        v = velocities.detach().cpu().numpy()
        sim = Simulation(ParticleData(m, p[0], p[1], p[2], v[0], v[1], v[2]), config)
        sim.initialize()
        sim.rollout(int(steps), int(checkpoint_every))
        fx, fy, fz, fvx, fvy, fvz = sim.download()
        ctx.sim = sim
        dev = positions.device
        return (torch.from_numpy(np.stack([fx, fy, fz])).to(dev),
                torch.from_numpy(np.stack([fvx, fvy, fvz])).to(dev))

    @staticmethod
    def backward(ctx, grad_positions, grad_velocities):
        sim = ctx.sim
        gp = grad_positions.detach().cpu().numpy() if grad_positions is not None else np.zeros((3, sim._n))
        gv = grad_velocities.detach().cpu().numpy() if grad_velocities is not None else None
        gm, gx0, gv0 = sim.backward(gp, gv)
        ctx.sim = None
        sim.close()
        dev = (grad_positions if grad_positions is not None else grad_velocities).device
        return (torch.from_numpy(gm).to(dev), torch.from_numpy(gx0).to(dev), torch.from_numpy(gv0).to(dev),
                None, None, None)


def rollout(mass, positions, velocities, config: SimulationConfig, steps: int, checkpoint_every: int = 32):
    return RolloutFunction.apply(mass, positions, velocities, config, steps, checkpoint_every)
