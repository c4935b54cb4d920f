"""Differentiable time loop: ``torch.autograd.Function`` over fv_record / fv_adjoint.

    from schemi_b200 import adjoint, cases, fv
    case, _ = cases.rayleigh_taylor_2d(64, 192)
    g = fv.FVCase(case)
    a = torch.randn(64, dtype=torch.float64, device="cuda").mul_(1e-3).requires_grad_()
    prim = adjoint.rayleigh_taylor_primitive(a, 64, 192)
    J, U_T = adjoint.TimeLoop.apply(prim, g, 5.0, 50, 0)
    J.backward()                                   # a.grad = dJ/da

Forward: the restart set (c_1..c_N, v_x, v_y, v_z, p; shape (N+4, n_cells), FP64, CUDA) is
uploaded with fv_upload_device, and fv_record runs main's time loop to t_end on the GPU, storing a
checkpoint every `checkpoint_every` steps and accumulating the mixing-width objective
J = sum_n dt_{n-1} W(U^n) (W = 4/L_x sum X_h (1 - X_h) dA, X_h the mole fraction of species
`heavy`).  Returns J and the final conserved state U^N ((N+5, n_cells)).
Backward: fv_adjoint sweeps the trajectory backwards (recomputing between checkpoints) with the
hand-written adjoint kernels and returns dJtot/dU^0; the restart-set-to-conserved conversion
(phaseInitialization.cpp:1827-1885 for an ideal mixture) is differentiated here in torch.
The step sizes are frozen at their recorded values (the CFL reduction is not differentiated).
A handle holds one trajectory: a second forward on the same FVCase replaces it, and the first
forward's backward then raises instead of sweeping the wrong trajectory.
"""

from __future__ import annotations

import math
from typing import Optional

import torch

from . import fv as fvmod


def conserved_from_primitive(prim: torch.Tensor, case) -> torch.Tensor:
    """Ideal-mixture conversion of the restart set to the conserved state (both (F, n_cells))."""
    ns = case.n_species
    dev, dt = prim.device, prim.dtype
    M = torch.tensor([s.M for s in case.species], dtype=dt, device=dev)[:, None]
    Cv = torch.tensor([s.Cv for s in case.species], dtype=dt, device=dev)[:, None]
    c = prim[:ns]
    v = prim[ns:ns + 3]
    p = prim[ns + 3]
    rho_k = c * M
    rho = rho_k.sum(0)
    X = c / c.sum(0)
    Uv = p * (X * Cv).sum(0) / case.R
    m = rho * v
    E = Uv + 0.5 * rho * (v * v).sum(0)
    return torch.cat([rho_k, rho[None], m, E[None]], 0)


class TimeLoop(torch.autograd.Function):
    """(J, U_T) = TimeLoop.apply(prim, fvcase, t_end, checkpoint_every, heavy)."""

    @staticmethod
    def forward(ctx, prim: torch.Tensor, g, t_end: float, checkpoint_every: int = 50, heavy: int = 0):
        if prim.dtype != torch.float64 or not prim.is_cuda:
            raise TypeError("prim must be a float64 CUDA tensor of shape (n_species + 4, n_cells)")
        prim = prim.detach().contiguous()
        torch.cuda.current_stream().synchronize()  # the library works on its own stream
        g.upload_device([prim[i].data_ptr() for i in range(prim.shape[0])])
        st = g.record(t_end, checkpoint_every, fvmod.OBJ_MIXING_WIDTH, heavy)
        UT = torch.empty((g.n_conserved, g.n_cells), dtype=torch.float64, device=prim.device)
        g.state_copy(UT.data_ptr())
        ctx.g = g
        ctx.record_id = g.records
        ctx.record_stats = st
        ctx.save_for_backward(prim)
        J = torch.tensor(st.objective, dtype=torch.float64, device=prim.device)
        return J, UT

    @staticmethod
    def backward(ctx, gJ: Optional[torch.Tensor], gUT: Optional[torch.Tensor]):
        (prim,) = ctx.saved_tensors
        g = ctx.g
        if g.records != ctx.record_id:
            # fv_record keeps one trajectory per handle; sweeping a later one would return the
            # gradient of another forward without any error
            raise RuntimeError("the handle's trajectory was recorded again by a later TimeLoop.apply "
                               "before this backward; use one FVCase per forward that is still to be "
                               "differentiated")
        lam0 = torch.empty((g.n_conserved, g.n_cells), dtype=torch.float64, device=prim.device)
        gain = float(gJ) if gJ is not None else 0.0
        gUT_ptr = None
        if gUT is not None:
            gUT = gUT.detach().to(torch.float64).contiguous()
            gUT_ptr = gUT.data_ptr()
        torch.cuda.current_stream().synchronize()
        ctx.adjoint_stats = g.adjoint(gUT_ptr, gain, lam0.data_ptr())
        with torch.enable_grad():
            p = prim.detach().requires_grad_(True)
            U0 = conserved_from_primitive(p, g.case)
            (gp,) = torch.autograd.grad(U0, p, lam0)
        return gp, None, None, None, None


def rayleigh_taylor_primitive(a: torch.Tensor, nx: int, ny: int) -> torch.Tensor:
    """Restart set of the Rayleigh-Taylor case as a differentiable function of the interface
    mode amplitudes a (the torch form of cases.rt_fields): heavy fraction per cell from the
    exact interface height eta(x) = 1.5 + sum_m a_m cos(2 pi m x) at the cell-centre x."""
    dev, dt = a.device, torch.float64
    dy = 3.0 / ny
    xc = (torch.arange(nx, dtype=dt, device=dev) + 0.5) * (1.0 / nx)
    m = torch.arange(1, a.numel() + 1, dtype=dt, device=dev)
    eta = 1.5 + torch.cos(2 * math.pi * torch.outer(xc, m)) @ a.to(dt)
    y_lo = torch.arange(ny, dtype=dt, device=dev)[:, None] * dy
    frac = torch.clamp((y_lo + dy - eta[None, :]) / dy, 0.0, 1.0)
    yc = (torch.arange(ny, dtype=dt, device=dev)[:, None] + 0.5) * dy
    p = (2.5 - 0.1 * torch.where(yc > 1.5, 3.0 * (yc - 1.5), 1.0 * (yc - 1.5))) * torch.ones((1, nx), dtype=dt,
                                                                                             device=dev)
    cA = 3.0 * frac / 3.0  # c = rho_fraction / M, as cases.rt_fields writes it
    cB = 1.0 * (1 - frac) / 1.0
    z = torch.zeros((ny, nx), dtype=dt, device=dev)
    return torch.stack([cA, cB, z, z, z, p]).reshape(6, nx * ny)
