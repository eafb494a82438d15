"""Reverse-mode gradient of a gauge loss over a rollout (``hb_adjoint_*``).

    L(n, ZBC) = sum over steps t = obs_every, 2 obs_every, ... and gauge cells g
                of (H_t[g] - Hobs_t[g])^2

for a rollout of ``nsteps`` steps from an initial water level and velocities,
with per-cell Manning coefficients n (FNC = 9.81 n^2, mesh.cpp:364) and bed
elevations ZBC.  The gradient is the library's hand-written adjoint of the
fp64 step (variant H), with checkpoints every ``checkpoint_every`` steps.
``gauge_loss_function()`` puts it behind ``torch.autograd.Function``.
"""
import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check, lib
from .solver import Deck, Solver, _stream_handle


def _dp(a):
    return a.ctypes.data_as(_lib._dp) if a is not None else None


class Adjoint:
    """The rollout, its loss and gradient on one fp64 variant-H handle."""

    def __init__(self, deck: Deck, gauges: Sequence[int], obs_every: int, nsteps: int, checkpoint_every: int = 10,
                 device: int = 0):
        self.deck = deck
        self.solver = Solver(deck, variant="H", precision="fp64", device=device, init_state=False)
        self.gauges = np.ascontiguousarray(gauges, dtype=np.int32)
        self.obs_every, self.nsteps, self.k = int(obs_every), int(nsteps), int(checkpoint_every)
        self.nobs = self.nsteps // self.obs_every
        self.cells = deck.cells
        self._h = C.c_void_p()
        check(lib().hb_adjoint_create(self.solver._h, self.gauges.ctypes.data_as(_lib._ip), len(self.gauges),
                                      self.obs_every, self.nsteps, self.k, C.byref(self._h)))
        st = deck.state()
        self.set_initial(st["Z"], st["U"], st["V"])
        self.n = np.sqrt(deck.array("fnc") / 9.81).copy()
        self.zbc = deck.array("zbc").copy()

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().hb_adjoint_destroy(self._h)
            self._h = C.c_void_p()
        if getattr(self, "solver", None) is not None:
            self.solver.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_initial(self, Z0, U0, V0):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (Z0, U0, V0)]
        check(lib().hb_adjoint_set_initial(self._h, *[_dp(a) for a in arrs]))

    def set_parameters(self, n: Optional[np.ndarray] = None, zbc: Optional[np.ndarray] = None):
        n = None if n is None else np.ascontiguousarray(n, dtype=np.float64)
        zbc = None if zbc is None else np.ascontiguousarray(zbc, dtype=np.float64)
        check(lib().hb_adjoint_set_parameters(self._h, _dp(n), _dp(zbc)))
        if n is not None:
            self.n = n.copy()
        if zbc is not None:
            self.zbc = zbc.copy()

    def set_observations(self, obs: np.ndarray):
        obs = np.ascontiguousarray(obs, dtype=np.float64).reshape(self.nobs, len(self.gauges))
        check(lib().hb_adjoint_set_observations(self._h, _dp(obs)))

    def forward(self, stream=None):
        """Runs the rollout; returns (loss, gauge depths [nobs][ngauges])."""
        loss = C.c_double()
        gd = np.empty((self.nobs, len(self.gauges)))
        check(lib().hb_adjoint_forward(self._h, C.byref(loss), _dp(gd), _stream_handle(stream)))
        return loss.value, gd

    def backward(self, stream=None):
        """dL/dn and dL/dZBC of the last forward (reference order)."""
        gn, gz = np.empty(self.cells), np.empty(self.cells)
        check(lib().hb_adjoint_backward(self._h, _dp(gn), _dp(gz), _stream_handle(stream)))
        return gn, gz

    def loss(self, n=None, zbc=None):
        self.set_parameters(n, zbc)
        return self.forward()[0]


def gauge_loss_function():
    """torch.autograd.Function: loss = GaugeLoss.apply(n, zbc, adjoint), with
    n and ZBC float64 tensors of [cells] (reference order)."""
    import torch

    class GaugeLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, n, zbc, adj: Adjoint):
            adj.set_parameters(n.detach().cpu().numpy(), zbc.detach().cpu().numpy())
            loss, _ = adj.forward()
            ctx.adj = adj
            ctx.device = n.device
            return torch.tensor(loss, dtype=torch.float64, device=n.device)

        @staticmethod
        def backward(ctx, grad_out):
            gn, gz = ctx.adj.backward()
            scale = grad_out.detach().cpu().item()
            return (torch.from_numpy(gn * scale).to(ctx.device), torch.from_numpy(gz * scale).to(ctx.device), None)

    return GaugeLoss
