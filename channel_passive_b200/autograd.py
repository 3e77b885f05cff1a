"""torch.autograd over the discrete adjoint of the RK3 step (kmm_adjoint_* in include/kmm.h).

``control_objective(amp, gains, channel, U0, nsteps, dt, w_tau, w_q)`` returns the time-averaged
objective J = w_tau <tau_w> + w_q <q_w> of ``nsteps`` RK3 steps from the initial fields U0 under the
opposition control v_wall = amp * gains * v(y_d) (kmm_set_control), as a 0-d float64 tensor that
``backward`` differentiates with respect to ``amp`` (0-d) and ``gains`` ((nz, nxh)) through the
hand-written discrete adjoint on the GPU.  The channel must be an FP64 handle with a fixed time
step; its state after the call is the end of the trajectory.  The reference has no adjoint; this
is the differentiable form of its (commented) opposition-control hook.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import Channel


class ControlObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, amp, gains, channel: Channel, U0: np.ndarray, nsteps: int, dt: float, w_tau: float,
                w_q: float):
        g = gains.detach().to("cpu", torch.float32).numpy()
        channel.set_control(float(amp.detach().cpu()), g)
        channel.set_initial_data_uvw(U0, dt)
        J = channel.adjoint_forward(int(nsteps), w_tau, w_q)
        ctx.channel = channel
        ctx.gshape, ctx.gdtype, ctx.gdevice = gains.shape, gains.dtype, gains.device
        ctx.adtype, ctx.adevice = amp.dtype, amp.device
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        dA, dg = ctx.channel.adjoint_backward()
        s = float(gJ)
        ga = torch.tensor(s * dA, dtype=ctx.adtype, device=ctx.adevice)
        gg = torch.from_numpy(s * dg).to(device=ctx.gdevice, dtype=ctx.gdtype).reshape(ctx.gshape)
        return ga, gg, None, None, None, None, None, None


def control_objective(amp, gains, channel: Channel, U0: np.ndarray, nsteps: int, dt: float = 0.01,
                      w_tau: float = 1.0, w_q: float = 0.0):
    return ControlObjective.apply(amp, gains, channel, U0, nsteps, dt, w_tau, w_q)
