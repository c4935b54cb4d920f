"""TEST INFRASTRUCTURE: FP64 CPU restatement of the zero-slope step in torch, for tangent runs.

The CUDA adjoint (schemi_b200/csrc/fv_adjoint.cuh) is checked against the forward-mode
derivative (``torch.func.jvp``) of this independent FP64 CPU restatement of the same discrete map:
the multi-dimensional MUSCL-Hancock step of the reference with a limiter whose multi-dimensional
slopes are zero, i.e. for every cell the face state equals the cell state --

* the closure of an ideal-gas mixture (Schemi/src/thermodynamics/mixtureIdeal.cpp): c_k = rho_k / M_k,
  p = R sum_k c_k T, Uv = sum_k c_k Cv_k T, sound speed^2 = g1 (Uv + p) / rho, g1 = R / sum_k X_k Cv_k;
* the HLLC / HLL face flux (Schemi/src/flowSolvers/HLLCSolver.cpp:52-403, HLLSolver.cpp:52-300);
* the ghost state of a boundary face (Schemi/src/solverStages/HancockStage.cpp:324-446):
  fixedValueCell values, the slip reflection of the normal velocity, otherwise the owner's value;
* the conservative update with the gravity source (Schemi/src/Advections/Advection.cpp:414-431);
* main's CFL step (Schemi/main/Schemi.cpp:802-835) with the end-time clamp (:933-935) and the first
  step min_timestep (:664-670) -- the step sizes are taken from a plain forward pass and then
  frozen for the tangent pass, as the adjoint freezes them.

Only the tests import this module; nothing in the package does.  Its forward pass is checked
against the C restatement (fv_oracle.cpp) on the same inputs.
"""

from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

VERY_BIG = 1e300  # Schemi/headers/globalConstants.hpp veryBig


class TangentCase:
    """A zero-slope ideal-gas case on a uniform 2D/3D mesh, state as torch FP64 tensors."""

    def __init__(self, case):
        if case.dims not in (2, 3):
            raise ValueError("2D or 3D cases only")
        if case.eos != "ideal":
            raise ValueError("ideal-gas mixtures only")
        self.case = case
        self.dims = case.dims
        self.ns = case.n_species
        self.R = case.R
        self.M = torch.tensor([s.M for s in case.species], dtype=torch.float64)
        self.Cv = torch.tensor([s.Cv for s in case.species], dtype=torch.float64)
        self.flux = case.flux
        cfg = case.fv_config()
        self.cfg = cfg
        # array shape (z, y, x) of the used axes; h per axis from the node coordinates 0 + d i
        self.shape = tuple(reversed([int(case.n[a]) for a in range(self.dims)]))
        self.h = []
        for a in range(3):
            if a < self.dims:
                n = int(case.n[a])
                d = float(case.L[a]) / n
                nodes = 0.0 + d * np.arange(n + 1, dtype=np.float64)
                self.h.append(torch.from_numpy(np.abs(nodes[1:] - nodes[:-1])))
            else:
                self.h.append(torch.tensor([float(case.L[a])], dtype=torch.float64))
        self.periodic = [a in case.periodic_axes() for a in range(3)]
        self.gravity = bool(cfg.gravity)
        self.g = [float(cfg.g[d]) for d in range(3)]
        self.courant = float(cfg.courant)
        self.min_dt = float(cfg.min_timestep)
        self.courant_only = bool(cfg.courant_only)
        # broadcastable per-axis cell sizes, volume and face areas
        hx = self._axis(self.h[0], 0)
        hy = self._axis(self.h[1], 1) if self.dims >= 2 else self.h[1]
        hz = self._axis(self.h[2], 2) if self.dims >= 3 else self.h[2]
        self.hs = [hx, hy, hz]
        self.V = hx * hy * hz
        self.S = [hy * hz, hx * hz, hx * hy]
        self.area = hx * hy if self.dims == 2 else hx * hy * hz
        minedge = torch.minimum(torch.minimum(hx, hy), hz) if self.dims == 3 else torch.minimum(
            torch.minimum(hx, hy), hz * torch.ones_like(hx))
        self.minedge = minedge
        self.nmom = self.dims

    def _axis(self, h: torch.Tensor, a: int) -> torch.Tensor:
        """Reshape per-axis sizes to broadcast over the (z, y, x) array."""
        shp = [1] * self.dims
        shp[self.dims - 1 - a] = -1
        return h.reshape(shp)

    # ---- state conversions
    def conserved_from_primitive(self, prim: Sequence[torch.Tensor]) -> torch.Tensor:
        """prim: c_1..c_N, v_x, v_y, v_z, p (arrays of the mesh shape) -> U (N+5, *shape)."""
        ns = self.ns
        c = torch.stack([prim[k] for k in range(ns)])
        v = torch.stack([prim[ns + d] for d in range(3)])
        p = prim[ns + 3]
        M = self.M.reshape([-1] + [1] * self.dims)
        Cv = self.Cv.reshape([-1] + [1] * self.dims)
        rho_k = c * M
        rho = rho_k.sum(0)
        X = c / c.sum(0)
        Cvm = (X * Cv).sum(0)
        Uv = p * Cvm / self.R
        m = rho * v
        E = Uv + 0.5 * rho * (v * v).sum(0)
        return torch.cat([rho_k, rho[None], m, E[None]], 0)

    def face_state(self, U: torch.Tensor) -> dict:
        ns = self.ns
        rho_k = U[:ns]
        rho = U[ns]
        m = [U[ns + 1 + d] if d < self.nmom else torch.zeros_like(rho) for d in range(3)]
        E = U[ns + 4]
        v = [m[d] / rho for d in range(3)]
        Uv = E - 0.5 * rho * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
        c = rho_k / self.M.reshape([-1] + [1] * self.dims)
        return self._close(rho_k, rho, m, v, c, Uv=Uv, E=E)

    def _close(self, rho_k, rho, m, v, c, Uv=None, E=None, p=None):
        Cv = self.Cv.reshape([-1] + [1] * (c.dim() - 1))
        X = c / c.sum(0)
        g1 = self.R / (X * Cv).sum(0)
        if p is None:
            p = g1 * Uv
        else:
            Uv = p / g1
            E = Uv + 0.5 * rho * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
        cs = torch.sqrt(g1 * (Uv + p) / rho)
        return {"rho_k": rho_k, "rho": rho, "m": m, "v": v, "E": E, "p": p, "cs": cs, "c": c}

    def ghost(self, W: dict, patch: int, axis: int) -> dict:
        cfg = self.cfg
        ns = self.ns
        cs = []
        for k in range(ns):
            if cfg.bc_conc[patch][k] == 3:
                cs.append(torch.full_like(W["rho"], float(cfg.bc_conc_value[patch][k])))
            else:
                cs.append(W["c"][k])
        c = torch.stack(cs)
        rho_k = c * self.M.reshape([-1] + [1] * (c.dim() - 1))
        rho = rho_k.sum(0)
        vt = cfg.bc_vel[patch]
        if vt == 3:
            v = [torch.full_like(rho, float(cfg.bc_vel_value[patch][d])) for d in range(3)]
        elif vt == 2:
            v = [-W["v"][d] if d == axis else W["v"][d] for d in range(3)]
        else:
            v = list(W["v"])
        m = [v[d] * rho for d in range(3)]
        p = torch.full_like(rho, float(cfg.bc_p_value[patch])) if cfg.bc_p[patch] == 3 else W["p"]
        return self._close(rho_k, rho, m, v, c, p=p)

    def riemann(self, L: dict, R: dict, axis: int) -> List[torch.Tensor]:
        """Flux along +e_axis in FaceFlux order: rho, rho_1..rho_N, m_x, m_y, m_z, E."""
        uL, uR = L["v"][axis], R["v"][axis]
        SL = torch.where((uR - R["cs"]) < (uL - L["cs"]), uR - R["cs"], uL - L["cs"])
        SR = torch.where((uL + L["cs"]) < (uR + R["cs"]), uR + R["cs"], uL + L["cs"])
        qL = [L["rho"]] + [L["rho_k"][k] for k in range(self.ns)] + L["m"] + [L["E"]]
        qR = [R["rho"]] + [R["rho_k"][k] for k in range(self.ns)] + R["m"] + [R["E"]]
        nd = [1.0 if d == axis else 0.0 for d in range(3)]

        def phys(q, u, p, E):
            f = [q[k] * u for k in range(self.ns + 1)]
            f += [q[self.ns + 1 + d] * u + nd[d] * p for d in range(3)]
            f += [(E + p) * u]
            return f

        fL = phys(qL, uL, L["p"], L["E"])
        fR = phys(qR, uR, R["p"], R["E"])
        if self.flux == "HLLC":
            rL, rR = L["rho"], R["rho"]
            Sc = (R["p"] - L["p"] + rL * uL * (SL - uL) - rR * uR * (SR - uR)) / (rL * (SL - uL) - rR * (SR - uR))
            P = 0.5 * (L["p"] + R["p"] + rL * (SL - uL) * (Sc - uL) + rR * (SR - uR) * (Sc - uR))

            def star(q, f, u, S, p, E):
                fac = S - u
                den = 1.0 / (S - Sc)
                out = [f[k] + S * (q[k] * fac * den - q[k]) for k in range(self.ns + 1)]
                for d in range(3):
                    ms = (q[self.ns + 1 + d] * fac - nd[d] * (p - P)) * den
                    out.append(f[self.ns + 1 + d] + S * (ms - q[self.ns + 1 + d]))
                Es = (E * fac - p * u + P * Sc) * den
                out.append(f[-1] + S * (Es - E))
                return out

            sL = star(qL, fL, uL, SL, L["p"], L["E"])
            sR = star(qR, fR, uR, SR, R["p"], R["E"])
            out = []
            for i in range(len(fL)):
                x = torch.where(SR > 0, sR[i], fR[i])
                x = torch.where(Sc >= 0, sL[i], x)
                x = torch.where(SL >= 0, fL[i], x)
                out.append(x)
            return out
        den = 1.0 / (SR - SL)
        out = []
        for i in range(len(fL)):
            mid = (SR * fL[i] - SL * fR[i] + SR * SL * (qR[i] - qL[i])) * den
            x = torch.where(SR > 0, mid, fR[i])
            x = torch.where(SL >= 0, fL[i], x)
            out.append(x)
        return out

    def _take(self, W: dict, sl) -> dict:
        out = {}
        for key, val in W.items():
            if isinstance(val, list):
                out[key] = [x[sl] for x in val]
            elif key in ("rho_k", "c"):
                out[key] = val[(slice(None),) + sl]
            else:
                out[key] = val[sl]
        return out

    def _cat(self, parts: List[dict], dim: int) -> dict:
        out = {}
        for key in parts[0]:
            if isinstance(parts[0][key], list):
                out[key] = [torch.cat([p[key][i] for p in parts], dim) for i in range(len(parts[0][key]))]
            elif key in ("rho_k", "c"):
                out[key] = torch.cat([p[key] for p in parts], dim + 1)
            else:
                out[key] = torch.cat([p[key] for p in parts], dim)
        return out

    # patches: tail = x-, point = x+, right = y-, left = y+, bottom = z-, top = z+
    _LOW = {0: 0, 1: 3, 2: 2}
    _HIGH = {0: 1, 1: 4, 2: 5}

    def divergence(self, W: dict) -> List[torch.Tensor]:
        """sum over faces of F.n S / V per conserved component, FaceFlux order."""
        nF = self.ns + 5
        div = [torch.zeros(self.shape, dtype=torch.float64) for _ in range(nF)]
        for a in range(self.dims):
            ax = self.dims - 1 - a  # array axis
            n = self.shape[ax]

            def sl(i0, i1):
                s = [slice(None)] * self.dims
                s[ax] = slice(i0, i1)
                return tuple(s)

            # left / right states of all faces 1/2 .. n-1/2 (+ wrap / walls)
            L = self._take(W, sl(0, n - 1))
            R = self._take(W, sl(1, n))
            if self.periodic[a]:
                Lw = self._take(W, sl(n - 1, n))
                Rw = self._take(W, sl(0, 1))
                Lall = self._cat([Lw, L, Lw], ax)
                Rall = self._cat([Rw, R, Rw], ax)
            else:
                first = self._take(W, sl(0, 1))
                last = self._take(W, sl(n - 1, n))
                gLo = self.ghost(first, self._LOW[a], a)
                gHi = self.ghost(last, self._HIGH[a], a)
                Lall = self._cat([gLo, L, last], ax)
                Rall = self._cat([first, R, gHi], ax)
            F = self.riemann(Lall, Rall, a)  # faces -1/2 .. n-1/2 (n + 1 of them)
            S = self.S[a]
            for i in range(nF):
                Fi = F[i]
                hi = Fi.narrow(ax, 1, n)
                lo = Fi.narrow(ax, 0, n)
                div[i] = div[i] + (hi - lo) * S / self.V
        return div

    def step(self, U: torch.Tensor, dt: float, g: Optional[Sequence[float]] = None) -> torch.Tensor:
        ns = self.ns
        W = self.face_state(U)
        div = self.divergence(W)
        g = self.g if g is None else g
        out = [None] * (ns + 5)
        out[ns] = U[ns] - dt * div[0]
        for k in range(ns):
            out[k] = U[k] - dt * div[k + 1]
        for d in range(3):
            if d < self.nmom:
                md = U[ns + 1 + d] - dt * div[ns + 1 + d]
                if self.gravity:
                    md = md + dt * g[d] * U[ns]
                out[ns + 1 + d] = md
            else:
                out[ns + 1 + d] = U[ns + 1 + d]
        E = U[ns + 4] - dt * div[ns + 4]
        if self.gravity:
            E = E + dt * sum(g[d] * W["m"][d] for d in range(3))
        out[ns + 4] = E
        return torch.stack(out)

    def cfl(self, U: torch.Tensor) -> float:
        W = self.face_state(U)
        v = W["v"]
        speed = torch.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
        sig = float(((speed + W["cs"]) / self.minedge).max())
        dt = self.courant / sig
        if not self.courant_only:
            dt = min(dt, VERY_BIG)
        return max(dt, self.min_dt)

    def width(self, U: torch.Tensor, heavy: int) -> torch.Tensor:
        c = U[: self.ns] / self.M.reshape([-1] + [1] * self.dims)
        X = c[heavy] / c.sum(0)
        area = float(self.case.L[0]) * (float(self.case.L[2]) if self.dims == 3 else 1.0)
        return 4.0 / area * (X * (1 - X) * self.area).sum()

    # ---- trajectories
    def schedule(self, U0: torch.Tensor, t_end: float, max_steps: int = 1 << 60) -> List[float]:
        """Step sizes of main's loop from U0 to t_end (first step min_timestep)."""
        dts = []
        t = 0.0
        dt_free = self.min_dt
        U = U0
        with torch.no_grad():
            while t < t_end and len(dts) < max_steps:
                dt = min(dt_free, t_end - t)
                U = self.step(U, dt)
                dts.append(dt)
                t += dt
                dt_free = self.cfl(U)
        return dts

    def objective(self, U0: torch.Tensor, dts: Sequence[float], heavy: int) -> torch.Tensor:
        """J = sum_{n=1..N} dt_{n-1} W(U^n) with the step sizes frozen."""
        U = U0
        J = torch.zeros((), dtype=torch.float64)
        for dt in dts:
            U = self.step(U, dt)
            J = J + dt * self.width(U, heavy)
        return J

    def final_state(self, U0: torch.Tensor, dts: Sequence[float]) -> torch.Tensor:
        U = U0
        for dt in dts:
            U = self.step(U, dt)
        return U


def tangent(f, x: torch.Tensor, dx: torch.Tensor) -> Tuple[torch.Tensor, torch.Tensor]:
    """Forward-mode directional derivative (value, J'(x) dx)."""
    return torch.func.jvp(f, (x,), (dx,))
