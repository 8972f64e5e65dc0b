"""Differentiable transport: ring-detector signals as a torch autograd Function of the
regions' absorption and scattering coefficients.

The forward pass traces photons with the adjoint sums on (``lp_forward``): every photon
keeps its path length L_r and interaction count k_r in each region, and a photon scored
with weight s in ring d adds s * (-L_r / factor) to dS_d/dmua_r and
s * (k_r / mus_r - L_r / factor) to dS_d/dmus_r (perturbation Monte Carlo, Hayakawa et
al., Opt. Lett. 26, 2001).  The Jacobians come out of the same launch, so a gradient
costs one forward pass plus the per-photon bookkeeping.  backward() is the
vector-Jacobian product with the saved Jacobians.  No reference counterpart.
"""
from __future__ import annotations

import numpy as np

from .propagation import Simulation


class TransportFunction:
    """Factory of the torch.autograd.Function (torch is imported lazily)."""

    _fn = None

    @classmethod
    def get(cls):
        if cls._fn is None:
            import torch

            class _Transport(torch.autograd.Function):
                @staticmethod
                def forward(ctx, mua, mus, sim, base_nmuasg, n, first):
                    table = np.array(base_nmuasg, np.float32, copy=True)
                    table[:, 1] = mua.detach().cpu().numpy().astype(np.float32)
                    table[:, 2] = mus.detach().cpu().numpy().astype(np.float32)
                    sim.set_media(table)
                    signal = sim.forward(int(n), int(first))
                    g = sim.gradient()
                    ctx.jmua = torch.from_numpy(g["d_mua"])
                    ctx.jmus = torch.from_numpy(g["d_mus"])
                    ctx.dtype = mua.dtype
                    return torch.from_numpy(signal).to(mua.device)

                @staticmethod
                def backward(ctx, grad_signal):
                    g = grad_signal.detach().cpu().to(torch.float64)
                    gm = (g @ ctx.jmua).to(ctx.dtype).to(grad_signal.device)
                    gs = (g @ ctx.jmus).to(ctx.dtype).to(grad_signal.device)
                    return gm, gs, None, None, None, None

            cls._fn = _Transport
        return cls._fn


def ring_signals(sim: Simulation, base_nmuasg, mua, mus, n: int, first: int = 0):
    """S_d (float64 tensor, one value per ring) for photons [first, first + n), with
    mua/mus (tensors, one value per region) replacing the coefficients of base_nmuasg.
    Differentiable with respect to mua and mus."""
    return TransportFunction.get().apply(mua, mus, sim, base_nmuasg, n, first)
