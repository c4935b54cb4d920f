"""Regenerates the golden fixtures in this directory by running the reference solver.

The reference (Eicosane-2/Schemi) is compiled from its own sources by ``oracle/Makefile``
(``make -C oracle ref``) into ``oracle/_ref/schemi_patched``; each case below is written as a
task deck by ``schemi_b200.deck`` and fed to it through its restart reader.  The fixtures hold
the reference's per-step outputs, so the parity tests need neither the reference sources nor
the binary at run time.

    python tests/golden/make_golden.py [fixture names]
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from schemi_b200 import cases  # noqa: E402
from schemi_b200.case import BC, Case, PatchBC  # noqa: E402
import oracle as O  # noqa: E402

FIELDS = {"T": "temperature", "c1": "concentration_1", "c2": "concentration_2", "c3": "concentration_3", "vx": "velocity_x",
          "vy": "velocity_y", "vz": "velocity_z", "p": "pressure", "rho": "density", "E": "total_energy",
          "mx": "momentum_x", "my": "momentum_y"}


def golden_cases():
    """(name, case, prim, n_steps or None for a run to t_end, steps to keep)."""
    out = []
    c, p = cases.shock_tube_1d()
    out.append(("shock_tube_1d_full", c, p, None, [1, 2, 10, 100, 500, "last"]))
    c, p = cases.kelvin_helmholtz_2d(n=24, periodic=False)
    out.append(("kh_slip_24_vanleer", c, p, 12, [1, 12]))
    c, p = cases.kelvin_helmholtz_2d(n=24, periodic=False, limiter="Koren2")
    out.append(("kh_slip_24_koren2", c, p, 10, [1, 10]))
    c, p = cases.kelvin_helmholtz_2d(n=24, periodic=False, limiter="linear")
    out.append(("kh_slip_24_linear", c, p, 10, [1, 10]))
    c, p = cases.kelvin_helmholtz_2d(n=24, periodic=False)
    c.flux = "HLL"
    out.append(("kh_slip_24_hll", c, p, 10, [10]))
    c, p = cases.rayleigh_taylor_2d(nx=16, ny=48, modes=4)
    out.append(("rt_16x48_gravity", c, p, 10, [1, 10]))
    c, p, _ = cases.richtmyer_meshkov(0, n=32)
    c.precision = "f64"
    out.append(("rm_32_superbee", c, p, 10, [1, 10]))
    c3, p3 = cases.reacting_shear_3d(n=12, periodic=False)
    n = 12
    c = Case(dims=2, n=(n, n, 1), L=(1.0, 1.0, 1.0), species=c3.species, t_end=1.0, R_units="SI",
             eos="vanDerWaals", limiter="vanLeer", name="vdw2d")
    for k in ("tail", "point", "right", "left"):
        c.bc[k] = PatchBC.uniform("slip", 3)
    out.append(("vdw_2d_12", c, [a.reshape(n, n, n)[0].ravel() for a in p3], 10, [1, 10]))
    c, p = cases.shock_tube_1d(n=100)
    c.bc["tail"] = PatchBC([BC("fixedValueCell", 1.0), BC("fixedValueCell", 0.0)],
                           BC("fixedValueCell", (0.2, 0.0, 0.0)), BC("fixedValueCell", 1.0))
    c.bc["point"] = PatchBC([BC("slip"), BC("slip")], BC("slip"), BC("slip"))
    out.append(("tube_fixedvalue_slip_100", c, p, 20, [1, 20]))
    c, p = cases.shock_tube_1d(n=200)
    c.flux, c.limiter = "HLL", "superbee"
    out.append(("tube_hll_superbee_200", c, p, 30, [30]))
    # every limiter whose phi acts in 1D MUSCL-Hancock (r > 0 happens only in 1D), on the 200-cell
    # two-species tube; minmod and superbee are pinned above, UTCDFS and the unlimited linear
    # reconstruction end in the reference's Riemann failure (step 2 and step 4)
    for lim in ("vanAlbada", "vanAlbada2", "vanLeer", "vanLeer2", "minmod2", "HQUICK", "Koren", "Koren2",
                "Sweby", "Schmidtmann"):
        c, p = cases.shock_tube_1d(n=200)
        c.limiter = lim
        out.append((f"tube_{lim.lower()}_200", c, p, 40, [1, 2, 40]))
    # the equations of state beyond ideal and van der Waals (abstractMixtureThermodynamics.cpp:39-43)
    for eos in ("stiffened", "RedlichKwong", "Kataoka"):
        c, p = cases.real_gas_tube(eos)
        out.append((f"tube_{eos.lower()}_200", c, p, 40, [1, 2, 40]))
    # Cl2 <-> 2Cl chemistry (the ClorumTest mechanism and solver, hot mixture)
    c, p = cases.chlorine_dissociation_2d(4)
    out.append(("cl2_4x4_vdw_gs", c, p, 10, [1, 2, 10]))
    c, p = cases.chlorine_dissociation_2d(4, eos="ideal")
    out.append(("cl2_4x4_ideal_gs", c, p, 10, [1, 10]))
    c, p = cases.chlorine_dissociation_2d(4)
    c.const_timestep = 2e-5  # #Constant_timestep: main skips its CFL block
    out.append(("cl2_4x4_vdw_const_dt", c, p, 8, [1, 8]))
    for solver, tag in (("Jacobi", "jacobi"), ("GaussElimination", "ge"), ("conjugateGradient", "cg")):
        c, p = cases.chlorine_dissociation_2d(4, solver=solver)
        out.append((f"cl2_4x4_vdw_{tag}", c, p, 6, [1, 6]))
    # SecondOrderRK: two stages without the Hancock predictor, then the 0.5 average
    c, p = cases.kelvin_helmholtz_2d(n=24, periodic=False)
    c.order = "SecondOrderRK"
    out.append(("kh_slip_24_rk2", c, p, 10, [1, 2, 10]))
    c, p = cases.kelvin_helmholtz_2d(n=24, periodic=False, limiter="linear")
    c.order = "SecondOrderRK"
    out.append(("kh_slip_24_rk2_linear", c, p, 8, [1, 8]))
    c, p = cases.shock_tube_1d(n=200)
    c.order = "SecondOrderRK"
    out.append(("tube_rk2_minmod_200", c, p, 30, [1, 2, 30]))
    c, p = cases.rayleigh_taylor_2d(nx=16, ny=48, modes=4)
    c.order = "SecondOrderRK"
    c.g_delta = (0.0, -0.02, 0.0)
    out.append(("rt_16x48_rk2_gravity", c, p, 10, [1, 10]))
    # ThirdOrder: SSP-RK3 with the directional limiter of thirdOrderLimiter.hpp
    c, p = cases.kelvin_helmholtz_2d(n=24, periodic=False)
    c.order = "ThirdOrder"
    out.append(("kh_slip_24_rk3", c, p, 8, [1, 2, 8]))
    c, p = cases.kelvin_helmholtz_2d(n=20, periodic=False, limiter="Sweby")
    c.order = "ThirdOrder"
    out.append(("kh_slip_20_rk3_sweby", c, p, 6, [1, 6]))
    c, p = cases.kelvin_helmholtz_2d(n=20, periodic=False, limiter="Schmidtmann")
    c.order = "ThirdOrder"
    out.append(("kh_slip_20_rk3_schmidtmann", c, p, 6, [1, 6]))
    c, p = cases.shock_tube_1d(n=200)
    c.order = "ThirdOrder"
    out.append(("tube_rk3_minmod_200", c, p, 30, [1, 2, 30]))
    c, p = cases.rayleigh_taylor_2d(nx=16, ny=48, modes=4)
    c.order = "ThirdOrder"
    out.append(("rt_16x48_rk3_gravity", c, p, 8, [1, 8]))
    c, p = cases.shock_tube_1d(n=100)
    c.bc["tail"] = PatchBC([BC("fixedValueCell", 1.0), BC("fixedValueCell", 0.0)],
                           BC("fixedValueCell", (0.2, 0.0, 0.0)), BC("fixedValueCell", 1.0))
    c.bc["point"] = PatchBC([BC("slip"), BC("slip")], BC("slip"), BC("slip"))
    c.order = "ThirdOrder"
    c.limiter = "vanAlbada"
    out.append(("tube_rk3_fixedvalue_slip_100", c, p, 20, [1, 20]))
    # ThirdOrderCada: the same stages with the smoothness switch of thirdOrderLimiterCada.hpp
    # (the tube's jumps are limited, its rarefaction and the shear layers are not)
    c, p = cases.shock_tube_1d(n=200)
    c.order = "ThirdOrderCada"
    out.append(("tube_cada_minmod_200", c, p, 30, [1, 2, 30]))
    c, p = cases.kelvin_helmholtz_2d(n=24, periodic=False)
    c.order = "ThirdOrderCada"
    out.append(("kh_slip_24_cada", c, p, 8, [1, 2, 8]))
    c, p = cases.rayleigh_taylor_2d(nx=16, ny=48, modes=4)
    c.order = "ThirdOrderCada"
    c.limiter = "superbee"
    out.append(("rt_16x48_cada_superbee_gravity", c, p, 8, [1, 8]))
    out.append(("tube_cada_blend_50", *cada_blend_tube(), 3, [1, 3]))
    # chemistry after the multi-stage average (secondOrderStepSolverRK.cpp:114-118,
    # thirdOrderStepSolver.cpp:125-129)
    c, p = cases.chlorine_dissociation_2d(4)
    c.order = "SecondOrderRK"
    out.append(("cl2_4x4_vdw_gs_rk2", c, p, 8, [1, 2, 8]))
    c, p = cases.chlorine_dissociation_2d(4, eos="ideal")
    c.order = "ThirdOrder"
    out.append(("cl2_4x4_ideal_gs_rk3", c, p, 6, [1, 6]))
    # 3D: the shear layer of the reacting benchmark (3 species, van der Waals) in a slip-walled
    # 8^3 box without its reaction (the reference has no periodic patch and no A+B->2C), with the
    # zero-slope limiter (fused march) and with the linear one (generic path)
    for lim, tag in (("vanLeer", "vanleer"), ("linear", "linear")):
        c, p = cases.reacting_shear_3d(n=8, precision="f64", periodic=False)
        c.chemistry = "no"
        c.limiter = lim
        out.append((f"shear3d_8_vdw_{tag}", c, p, 6, [1, 6]))
    for order, tag in (("SecondOrderRK", "rk2"), ("ThirdOrderCada", "cada")):
        c, p = cases.reacting_shear_3d(n=8, precision="f64", periodic=False)
        c.chemistry = "no"
        c.order = order
        out.append((f"shear3d_8_vdw_{tag}", c, p, 4, [1, 4]))
    return out


def cada_blend_tube():
    """A 1D tube whose cell 20 sits inside the blend window of thirdOrderLimiterCada.hpp at the
    first stage: its face pressure gradients are 15 and sqrt(T - 15^2), T = sqrt(5/2) (8 pi)^2,
    so eta = 1 up to rounding (1e-15, the window is 1e-6); a jump of 1 at cell 35 (gradient 50,
    eta 2.5) is limited and the uniform regions are not."""
    import math

    c, _ = cases.shock_tube_1d(n=50)
    c.order = "ThirdOrderCada"
    n, h = 50, 1.0 / 50
    T = math.sqrt(5.0 / 2.0) * (8 * math.pi) ** 2
    g2 = math.sqrt(T - 15.0 ** 2)
    pr = np.ones(n)
    pr[20] = 1.0 + 15.0 * h
    pr[21:] = pr[20] + g2 * h
    pr[35:] += 1.0
    prim = [np.full(n, 0.5), np.full(n, 0.3), np.zeros(n), np.zeros(n), np.zeros(n), pr]
    return c, prim


def main(only=None):
    for name, case, prim, nsteps, keep in golden_cases():
        if only and name not in only:
            continue
        if nsteps is not None:
            oc = O.OracleCase(case)
            oc.upload(prim)
            for _ in range(nsteps):
                oc.step()
            case.t_end = oc.time()[0]
        outs, times, wall = O.run_reference(case, prim, frequency_of_output=1)
        idx = sorted(i for i in outs if i >= 2)
        last = idx[-1]
        data = {"n_steps": np.int64(len(idx)), "t_end": np.float64(case.t_end)}
        for k in keep:
            i = last if k == "last" else k + 1       # output_<s+1> holds the state after step s
            step = len(idx) if k == "last" else k
            r = outs[i]
            data[f"time_{step}"] = np.float64(times[i])
            for short, col in FIELDS.items():
                if col in r:
                    data[f"{short}_{step}"] = np.asarray(r[col], dtype=np.float64)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
        print(f"{name}: {len(idx)} steps, reference wall {wall:.2f} s")


if __name__ == "__main__":
    main(sys.argv[1:] or None)
