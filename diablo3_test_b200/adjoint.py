"""torch.autograd.Function over libdiablo_gpu's step and its hand-written
discrete adjoint (diablo_adjoint_record / diablo_adjoint_run).

    u1, u2, u3, p, *th = ChannelSteps.apply(channel, nsteps, every, u1, u2, u3, p, *th)

takes and returns the Fourier state in the reference layout (float64 CUDA
tensors of shape (Ny+2, Nz+2, Nx+2), each complex coefficient stored as two
reals, the layout of ``vv(0:Nxp, 0:Nz+1, 0:Nyp+1)``), one tensor per scalar
after p.  The forward advances `channel` by nsteps steps keeping checkpoints
every `every` steps; backward recomputes each segment from its checkpoint and
runs the adjoint substeps backwards (no autograd graph of the step is built).
DNS in FP64 with velocities and scalars, the scalar filter of
filter_scalars and the 'Front' thermal-wind advection included
(for/channel.f90:rk_chan_1 without LES).
"""
from __future__ import annotations

import torch

from . import _lib


class ChannelSteps(torch.autograd.Function):
    @staticmethod
    def forward(ctx, channel, nsteps: int, every: int, *state):
        fids = [_lib.U1, _lib.U2, _lib.U3, _lib.P] + [_lib.TH + n for n in range(channel.params.n_th)]
        if len(state) != len(fids):
            raise ValueError(f"{len(fids)} state tensors: u1, u2, u3, p and one per scalar")
        for fid, t in zip(fids, state):
            channel.upload(fid, t.detach().contiguous(), _lib.LAYOUT_FOURIER)
        channel.adjoint_record(nsteps, every)
        outs = []
        for fid in fids:
            o = torch.zeros_like(state[0])
            channel.download(fid, _lib.LAYOUT_FOURIER, out=o)
            outs.append(o)
        channel.synchronize()
        ctx.channel = channel
        return tuple(outs)

    @staticmethod
    def backward(ctx, *grads):
        lam = [g.detach().clone().contiguous() if g is not None else None for g in grads]
        ref = next(t for t in lam if t is not None)
        lam = [t if t is not None else torch.zeros_like(ref) for t in lam]
        ctx.channel.adjoint_run(lam)
        return (None, None, None) + tuple(lam)
