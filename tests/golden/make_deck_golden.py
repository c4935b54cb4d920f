"""Regenerates the task-deck fixtures ``deck_<name>.npz`` by running the reference solver.

Each fixture holds a complete task directory as the reference reads it (``set/*.txt`` and, for
restart decks, ``fieldsOutput/output_000001`` + ``result/Time.tsv``), the ``set/main.txt`` of
every run made in that directory (a second run restarts from an output of the first), and every
file the reference left behind: ``result/output_<NNNNNN>.tsv``, ``result/Time.tsv``,
``fieldsOutput/output_<NNNNNN>/*.dat`` and ``timeOfCalculation.tsv``.  The GPU driver test
replays the same runs with ``schemi_b200/lib/fvrun`` and compares the files byte for byte
(numerically for the chemistry deck).

The reference is compiled from its own sources by ``oracle/Makefile`` (``make -C oracle ref``);
the decks are written by ``schemi_b200.deck``.

    python tests/golden/make_deck_golden.py [fixture names without the deck_ prefix]
"""

import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from schemi_b200 import cases  # noqa: E402
from schemi_b200.case import BC, Case, PatchBC, Species  # noqa: E402
from schemi_b200.deck import write_deck  # noqa: E402
import oracle as O  # noqa: E402

START_KEY = "#Start_From_Time-Step"
END_KEY = "#Time_of_calculation"


def _t_after(case, prim, steps, frac):
    """End time that the oracle reaches after ``steps`` steps plus ``frac`` of the next step."""
    oc = O.OracleCase(case)
    oc.upload(prim)
    for _ in range(steps):
        oc.step()
    t, dt = oc.time()
    return t + frac * dt


def _set_main(text, **values):
    lines = text.split("\n")
    keys = {"start": START_KEY, "t_end": END_KEY}
    for name, v in values.items():
        i = lines.index(keys[name])
        lines[i + 1] = v
    return "\n".join(lines)


def deck_cases():
    """(name, case, prim, frequency, restart, [main.txt edits per run], tolerance[, write_deck
    keyword arguments])."""
    out = []
    # Kelvin-Helmholtz 8x8, slip walls: restart deck, then a second run from output 2
    c, p = cases.kelvin_helmholtz_2d(n=8, periodic=False)
    c.t_end = _t_after(c, p, 10, 0.37)
    out.append(("kh8_restart", c, p, 4, True, [{}, {"start": "2", "t_end": repr(c.t_end * 1.6)}], 0.0))
    # two-species tube from the uniform outer zone, driven through a fixed-value inflow
    c, p = cases.shock_tube_1d(n=40)
    p = [np.full_like(a, float(np.mean(a))) for a in p]
    c.bc["tail"] = PatchBC([BC("fixedValueCell", 0.7), BC("fixedValueCell", 0.3)],
                           BC("fixedValueCell", (0.3, 0.0, 0.0)), BC("fixedValueCell", 0.9))
    c.bc["point"] = PatchBC([BC("freeBoundary"), BC("freeBoundary")], BC("freeBoundary"), BC("freeBoundary"))
    c.t_end = _t_after(c, p, 14, 0.61)
    out.append(("tube40_fresh", c, p, 5, False, [{}], 0.0))
    out.append(("tube40_initialisation", c, p, 5, False, [{"start": "initialisation"}], 0.0))
    # Rayleigh-Taylor 8x16 with growing gravity
    c, p = cases.rayleigh_taylor_2d(nx=8, ny=16, modes=2)
    c.g_delta = (0.0, -0.05, 0.0)
    c.t_end = _t_after(c, p, 12, 0.5)
    out.append(("rt8x16_gravity", c, p, 5, True, [{}], 0.0))
    # three-species van der Waals mixture, 6x6 slip box
    c3, p3 = cases.reacting_shear_3d(n=6, periodic=False)
    c = Case(dims=2, n=(6, 6, 1), L=(1.0, 1.0, 1.0), species=c3.species, t_end=1.0, R_units="SI",
             eos="vanDerWaals", limiter="vanLeer", name="vdw2d")
    for k in ("tail", "point", "right", "left"):
        c.bc[k] = PatchBC.uniform("slip", 3)
    p = [a.reshape(6, 6, 6)[0].ravel() for a in p3]
    c.t_end = _t_after(c, p, 7, 0.8)
    out.append(("vdw3_6x6", c, p, 3, True, [{}], 0.0))
    # constant time step: no CFL block, sonic speeds stay those of the initial state
    c, p = cases.kelvin_helmholtz_2d(n=8, periodic=False, limiter="superbee")
    oc = O.OracleCase(c)
    oc.upload(p)
    oc.step()
    c.const_timestep = 0.5 * oc.time()[1]
    c.t_end = 4.5 * c.const_timestep
    out.append(("kh8_const_dt", c, p, 2, True, [{}], 0.0))
    # Cl2 dissociation (chemistry pass): compared to a relative tolerance
    c, p = cases.chlorine_dissociation_2d(4)
    c.t_end = _t_after(c, p, 6, 0.5)
    out.append(("cl2_4x4", c, p, 2, True, [{}], 1e-10))
    # multi-stage step solvers: ThirdOrderCada with a restart from output 2 (the averaged
    # concentrations go through the output files), SecondOrderRK with growing gravity
    c, p = cases.kelvin_helmholtz_2d(n=8, periodic=False)
    c.order = "ThirdOrderCada"
    c.t_end = _t_after(c, p, 6, 0.45)
    out.append(("kh8_cada_restart", c, p, 3, True, [{}, {"start": "2", "t_end": repr(c.t_end * 1.5)}], 0.0))
    c, p = cases.rayleigh_taylor_2d(nx=8, ny=16, modes=2)
    c.order = "SecondOrderRK"
    c.g_delta = (0.0, -0.05, 0.0)
    c.t_end = _t_after(c, p, 9, 0.5)
    out.append(("rt8x16_rk2_gravity", c, p, 4, True, [{}], 0.0))
    # initial fields from zones (a fresh run): a plane, a sphere, a slab of two planes and a
    # cylinder before the outer zone (first match wins), and a gaussian modifier of species 1
    c, p = cases.kelvin_helmholtz_2d(n=16, periodic=False)
    zones = [
        ("plane 0 1 0 point: 0 0.25 0", [0.05, 0.02], (0.3, 0.0, 0.0), 2.6),
        ("sphere 0.5 0.6 0.5 0.15", [0.01, 0.2], (-0.2, 0.05, 0.0), 2.4),
        ("planes 2 1 0 0 point: 0.8 0 0 -1 0 0 point: 0.7 0 0", [0.03, 0.1], (0.0, -0.1, 0.0), 2.55),
        ("cylinder 0 0 1 top: 0.2 0.8 1 bottom: 0.2 0.8 0 0.12", [0.06, 0.05], (0.1, 0.1, 0.0), 2.7),
    ]
    c.t_end = _t_after(c, p, 6, 0.3)
    out.append(("kh16_zones_fresh", c, p, 3, False, [{}], 0.0,
                {"zones": zones, "modifiers": {1: (1.0, 0.5, 0.5, 0.2)}}))
    # 1D mixing-zone width (output::mixedZoneWidth1D): a fresh run, then a restart from output 2
    # that appends to result/timeWidth.tsv
    c, p = cases.shock_tube_1d(n=60)
    c.t_end = _t_after(c, p, 9, 0.4)
    out.append(("tube60_width", c, p, 3, False, [{}, {"start": "2", "t_end": repr(c.t_end * 1.5)}], 0.0,
                {"mixing_width": True}))
    # the same with a finite mixing zone: mole fraction 1 for x <= 0.4, 0.83 up to 0.6, 0 beyond
    # (zones; the outer zone takes the means of the restart set below)
    c, _ = cases.shock_tube_1d(n=60)
    p = [np.zeros(60), np.full(60, 0.125), np.zeros(60), np.zeros(60), np.zeros(60), np.full(60, 0.1)]
    zones = [("plane 1 0 0 point: 0.4 0 0", [1.0, 0.0], (0.0, 0.0, 0.0), 1.0),
             ("plane 1 0 0 point: 0.6 0 0", [0.3, 0.06], (0.0, 0.0, 0.0), 0.5)]
    c.t_end = 0.03
    out.append(("tube60_zones_width", c, p, 4, False, [{}, {"start": "2", "t_end": "0.05"}], 0.0,
                {"mixing_width": True, "zones": zones}))
    # the equations of state beyond ideal and van der Waals, with their data files
    # (set/stiffenedFluidData.txt, set/KataokaVanDerWaalsFluidData.txt) and the Helmholtz energy and
    # entropy of each mixture in the outputs
    for eos in ("stiffened", "RedlichKwong", "Kataoka"):
        c, p = cases.real_gas_tube(eos, n=60)
        c.t_end = _t_after(c, p, 10, 0.4)
        out.append((f"tube60_{eos.lower()}", c, p, 4, True, [{}], 0.0,
                    {} if eos == "stiffened" else {"gpu_tolerance": 1e-11}))
    # the diffusion stage (explicit solver, constant coefficients): a tube with the explicit
    # enthalpy flow, the molar-mass correction and the diffusion time-step limit; a tube with the
    # "linear" reconstruction and neither; a three-species van der Waals box; a Rayleigh-Taylor
    # box under growing gravity (the interpolated face velocities); a 3D van der Waals box
    c, p = cases.shock_tube_1d(n=60)
    c.diffusion, c.mu, c.D, c.kappa = True, 1e-4, 1e-3, 1e-4
    c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", True, True
    c.t_end = _t_after(c, p, 20, 0.4)
    out.append(("tube60_diffusion", c, p, 6, True, [{}], 0.0))
    c, p = cases.shock_tube_1d(n=60)
    c.diffusion, c.mu, c.D, c.kappa = True, 2e-4, 5e-4, 2e-4
    c.enthalpy_flow, c.molmass_diffusion, c.reconstruction = "no", False, "linear"
    c.t_end = _t_after(c, p, 20, 0.4)
    out.append(("tube60_diffusion_linear", c, p, 6, True, [{}], 0.0))
    c3, p3 = cases.reacting_shear_3d(n=6, periodic=False)
    c = Case(dims=2, n=(6, 6, 1), L=(1.0, 1.0, 1.0), species=c3.species, t_end=1.0, R_units="SI",
             eos="vanDerWaals", limiter="vanLeer", name="vdw2d")
    for k in ("tail", "point", "right", "left"):
        c.bc[k] = PatchBC.uniform("slip", 3)
    p = [a.reshape(6, 6, 6)[0].ravel() for a in p3]
    c.diffusion, c.mu, c.D, c.kappa = True, 1e-5, 1e-5, 1e-3
    c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", False, True
    c.t_end = _t_after(c, p, 8, 0.5)
    out.append(("vdw3_6x6_diffusion", c, p, 3, True, [{}], 0.0))
    c, p = cases.rayleigh_taylor_2d(nx=8, ny=16, modes=2)
    c.g_delta = (0.0, -0.05, 0.0)
    c.diffusion, c.mu, c.D, c.kappa = True, 1e-3, 1e-3, 1e-3
    c.enthalpy_flow, c.molmass_diffusion = "explicit", True
    c.t_end = _t_after(c, p, 12, 0.5)
    out.append(("rt8x16_gravity_diffusion", c, p, 5, True, [{}], 0.0))
    c, p = cases.reacting_shear_3d(n=6, periodic=False, precision="f64")
    c.chemistry = "no"
    for k in list(c.bc):
        c.bc[k] = PatchBC.uniform("slip", 3)
    c.diffusion, c.mu, c.D, c.kappa = True, 1e-5, 1e-5, 1e-3
    c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", False, True
    c.t_end = _t_after(c, p, 6, 0.5)
    out.append(("vdw3_6x6x6_diffusion", c, p, 3, True, [{}], 0.0))
    # the same stage with the Gauss-Seidel solver (implicit matrices, the averaged enthalpy flow)
    c, p = cases.shock_tube_1d(n=60)
    c.diffusion, c.mu, c.D, c.kappa, c.sle_solver = True, 1e-4, 1e-3, 1e-4, "GaussSeidel"
    c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", True, True
    c.t_end = _t_after(c, p, 20, 0.4)
    out.append(("tube60_diffusion_gs", c, p, 6, True, [{}], 0.0))
    c3, p3 = cases.reacting_shear_3d(n=6, periodic=False)
    c = Case(dims=2, n=(6, 6, 1), L=(1.0, 1.0, 1.0), species=c3.species, t_end=1.0, R_units="SI",
             eos="vanDerWaals", limiter="vanLeer", name="vdw2d")
    for k in ("tail", "point", "right", "left"):
        c.bc[k] = PatchBC.uniform("slip", 3)
    p = [a.reshape(6, 6, 6)[0].ravel() for a in p3]
    c.diffusion, c.mu, c.D, c.kappa, c.sle_solver = True, 1e-5, 1e-5, 1e-3, "GaussSeidel"
    c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", False, True
    c.t_end = _t_after(c, p, 8, 0.5)
    out.append(("vdw3_6x6_diffusion_gs", c, p, 3, True, [{}], 0.0))
    c, p = cases.rayleigh_taylor_2d(nx=8, ny=16, modes=2)
    c.g_delta = (0.0, -0.05, 0.0)
    c.diffusion, c.mu, c.D, c.kappa, c.sle_solver = True, 1e-3, 1e-3, 1e-3, "GaussSeidel"
    c.enthalpy_flow, c.molmass_diffusion = "explicit", True
    c.t_end = _t_after(c, p, 12, 0.5)
    out.append(("rt8x16_gravity_diffusion_gs", c, p, 5, True, [{}], 0.0))
    c, p = cases.reacting_shear_3d(n=6, periodic=False, precision="f64")
    c.chemistry = "no"
    for k in list(c.bc):
        c.bc[k] = PatchBC.uniform("slip", 3)
    c.diffusion, c.mu, c.D, c.kappa, c.sle_solver = True, 1e-5, 1e-5, 1e-3, "GaussSeidel"
    c.enthalpy_flow, c.molmass_diffusion = "no", True
    c.t_end = _t_after(c, p, 6, 0.5)
    out.append(("vdw3_6x6x6_diffusion_gs", c, p, 3, True, [{}], 0.0))
    # the other matrix solvers of the stage: Jacobi (1D, 2D under gravity, 3D), Thomas (the 1D
    # tridiagonal sweep), noSolver (the implicit branch, its solves returning the start field) and
    # the conjugate-gradient three (on the GPU their dot products are block sums: compared there to
    # a tolerance)
    for solver, tag in (("Jacobi", "jacobi"), ("Thomas", "thomas"), ("noSolver", "nosolver"), ("conjugateGradient", "cg"),
                        ("JacobiConjugateGradient", "jcg"), ("biConjugateGradient", "bicg")):
        c, p = cases.shock_tube_1d(n=60)
        c.diffusion, c.mu, c.D, c.kappa, c.sle_solver = True, 1e-4, 1e-3, 1e-4, solver
        # (the conjugate-gradient decks without the molar-mass correction: with it the tube is ill
        # conditioned, a one-ulp change of the input moving the state by 1e-5 within six steps)
        c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", "Gradient" not in solver, True
        c.t_end = _t_after(c, p, 20, 0.4)
        out.append((f"tube60_diffusion_{tag}", c, p, 6, True, [{}], 0.0,
                    {"gpu_tolerance": 1e-10} if "Gradient" in solver else {}))
    c, p = cases.rayleigh_taylor_2d(nx=8, ny=16, modes=2)
    c.g_delta = (0.0, -0.05, 0.0)
    c.diffusion, c.mu, c.D, c.kappa, c.sle_solver = True, 1e-3, 1e-3, 1e-3, "Jacobi"
    c.enthalpy_flow, c.molmass_diffusion = "explicit", True
    c.t_end = _t_after(c, p, 12, 0.5)
    out.append(("rt8x16_gravity_diffusion_jacobi", c, p, 5, True, [{}], 0.0))
    c, p = cases.reacting_shear_3d(n=6, periodic=False, precision="f64")
    c.chemistry = "no"
    for k in list(c.bc):
        c.bc[k] = PatchBC.uniform("slip", 3)
    c.diffusion, c.mu, c.D, c.kappa, c.sle_solver = True, 1e-5, 1e-5, 1e-3, "Jacobi"
    c.enthalpy_flow, c.molmass_diffusion = "explicit", False
    c.t_end = _t_after(c, p, 6, 0.5)
    out.append(("vdw3_6x6x6_diffusion_jacobi", c, p, 3, True, [{}], 0.0))
    # the implicit enthalpy flow (the upwind term of SLEMatrix::addNabla in the temperature matrix;
    # with the explicit solver the temperature keeps its value, the factory's second solver being a
    # noMatrixSolver): a tube with Gauss-Seidel, with Jacobi and with the explicit solver, and a
    # three-species van der Waals box with Gauss-Seidel
    for solver, tag in (("GaussSeidel", "gs"), ("Jacobi", "jacobi"), ("explicit", "explicit")):
        c, p = cases.shock_tube_1d(n=60)
        c.diffusion, c.mu, c.D, c.kappa, c.sle_solver = True, 1e-4, 1e-3, 1e-4, solver
        c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "implicit", True, True
        c.t_end = _t_after(c, p, 20, 0.4)
        out.append((f"tube60_enthalpy_implicit_{tag}", c, p, 6, True, [{}], 0.0))
    c3, p3 = cases.reacting_shear_3d(n=6, periodic=False)
    c = Case(dims=2, n=(6, 6, 1), L=(1.0, 1.0, 1.0), species=[Species(**vars(s)) for s in c3.species], t_end=1.0,
             R_units="SI", eos="vanDerWaals", limiter="vanLeer", name="vdw2d")
    for k in ("tail", "point", "right", "left"):
        c.bc[k] = PatchBC.uniform("slip", 3)
    p = [a.reshape(6, 6, 6)[0].ravel() for a in p3]
    c.diffusion, c.mu, c.D, c.kappa, c.sle_solver = True, 1e-5, 1e-5, 1e-3, "GaussSeidel"
    c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "implicit", False, True
    c.t_end = _t_after(c, p, 8, 0.5)
    out.append(("vdw3_6x6_enthalpy_implicit_gs", c, p, 3, True, [{}], 0.0))
    # the transport models: hard spheres (kinetic diameters) and Lennard-Jones (eps / k_B, sigma)
    # with both solvers; their face coefficients read the interpolated temperature and
    # concentrations and the Riemann star pressure, the viscous heating the cells' viscosity.  The
    # Lennard-Jones collision integrals call pow and exp, whose last bit the GPU's libm may set
    # otherwise than the host's.
    for solver, tag in (("explicit", ""), ("GaussSeidel", "_gs")):
        c, p = cases.shock_tube_1d(n=60)
        c.diffusion, c.transport, c.sle_solver = True, "hardSpheres", solver
        c.mu, c.D, c.kappa = 1e-6, 0.0, 1e-6
        c.species[0].diameter, c.species[1].diameter = 1.0, 1.3
        # (the explicit solver with the molar-mass correction: see the van der Waals box below)
        c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", solver != "explicit", True
        c.t_end = _t_after(c, p, 20, 0.4)
        out.append((f"tube60_hardspheres{tag}", c, p, 6, True, [{}], 0.0))
    c3, p3 = cases.reacting_shear_3d(n=6, periodic=False)
    for model, solver, name in (("hardSpheres", "GaussSeidel", "vdw3_6x6_hardspheres_gs"),
                                ("LennardJones", "explicit", "vdw3_6x6_lennardjones")):
        c = Case(dims=2, n=(6, 6, 1), L=(1.0, 1.0, 1.0), species=[Species(**vars(s)) for s in c3.species],
                 t_end=1.0, R_units="SI", eos="vanDerWaals", limiter="vanLeer", name="vdw2d")
        for k in ("tail", "point", "right", "left"):
            c.bc[k] = PatchBC.uniform("slip", 3)
        p = [a.reshape(6, 6, 6)[0].ravel() for a in p3]
        c.diffusion, c.transport, c.sle_solver = True, model, solver
        c.mu, c.D, c.kappa = 0.0, 0.0, 0.0
        for sp, d, e, sg in zip(c.species, (3.64, 3.46, 3.80), (98.0, 107.0, 71.4), (3.68, 3.43, 3.80)):
            sp.diameter, sp.tr_eps, sp.tr_sigma = d, e, sg
        # (the explicit solver takes the enthalpy flow's negative source into its diagonal without
        # the time step, SLEMatrix.cpp:2166-2175: with the molar-mass correction the first 1e-15 s
        # step cools this box to 15 K; the explicit deck runs without that correction)
        c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", solver != "explicit", True
        c.t_end = _t_after(c, p, 8, 0.5)
        out.append((name, c, p, 3, True, [{}], 0.0, {} if model == "hardSpheres" else {"gpu_tolerance": 1e-11}))
    c, p = cases.shock_tube_1d(n=60)
    c.diffusion, c.transport, c.sle_solver = True, "LennardJones", "GaussSeidel"
    c.mu, c.D, c.kappa = 0.0, 1e-6, 0.0
    for sp, e, sg in zip(c.species, (0.8, 1.1), (1.0, 1.2)):
        sp.tr_eps, sp.tr_sigma = e, sg
    # (without the molar-mass correction: with it this tube is ill conditioned, a one-ulp change of
    # its input moving the state by 1e-4 within six steps, and the GPU's collision integrals may
    # differ from the host's in the last bit)
    c.enthalpy_flow, c.molmass_diffusion = "explicit", False
    c.t_end = _t_after(c, p, 20, 0.4)
    out.append(("tube60_lennardjones_gs", c, p, 6, True, [{}], 0.0, {"gpu_tolerance": 1e-11}))
    # the Cl2 mechanism after a Gauss-Seidel hard-sphere diffusion stage (secondOrderStepSolver.cpp:
    # 69-91) on a hot, non-uniform mixture, with the ClorumTest deck's transport data
    c, p = cases.chlorine_dissociation_2d(n=4)
    c.diffusion, c.transport, c.sle_solver = True, "hardSpheres", "GaussSeidel"
    c.mu, c.D, c.kappa = 2e-8, 2e-8, 2e-5
    c.species[0].diameter, c.species[1].diameter = 3.2, 1.6
    c.enthalpy_flow, c.molmass_diffusion = "explicit", True
    c.t_end = _t_after(c, p, 12, 0.5)
    out.append(("cl2_4x4_diffusion_gs", c, p, 4, True, [{}], 0.0, {"gpu_tolerance": 1e-11}))
    return out


# Task decks shipped with the reference (its tests/TestsTasks directory) whose every stage is in
# this step: 1D, HLLC, the vanAlbada limiter, ideal gas, turbulence off; diffusion off, or (the
# Diffusion deck) explicit with constant coefficients.  Their set/
# directories are stored unchanged.  Noh_CGS is refused by the reference itself (a parenthesised
# fixed velocity that its stream reader cannot parse): exit code 1, "Unknown type of boundary
# condition", and only the empty result/Time.tsv left behind.
SHIPPED = [
    ("sod_cgs_1000", "TestsTasks/Sod_CGS/Sod_CGS_1000"),
    ("blastwaves_cgs_3000", "TestsTasks/BlastWaves/BlastWaves_CGS_3000"),
    ("gaussconcentration_cgs_1000", "TestsTasks/GaussConcentration_CGS/GaussConcentration_CGS_1000"),
    ("noh_1_1000", "TestsTasks/Noh_1/Noh_1_1000"),
    ("noh_2_1000", "TestsTasks/Noh_2/Noh_2_1000"),
    ("rarefactions_100_cgs", "TestsTasks/Rarefactions_CGS/Rarefactions_100_CGS"),
    ("noh_cgs_1000", "TestsTasks/Noh_CGS/Noh_CGS_1000"),
    ("diffusion_1000", "TestsTasks/Diffusion/Diffusion_1000"),
    # Gauss-Seidel diffusion of a van der Waals mixture between fixed walls, 100 x 100; to
    # t = 2e-3 (320 steps) instead of 2.0 (about 330,000)
    ("poiseuille_100x100_short", "TestsTasks/PoiseuilleFlow/PoiseuilleFlow_SI_100x100", "2E-3"),
    # the chemistry integrator's deck: Cl2 dissociation after a Gauss-Seidel hard-sphere diffusion
    # stage, van der Waals, 2 x 2 at a constant 1e-8 s step (the GPU's exp may differ in the
    # last bit: compared numerically there)
    ("chlorum_2x2", "Chemical Reactions/ClorumTest/Chlorum"),
]
SHIPPED_ROOT = "/root/reference/tests"
# decks whose GPU replay is compared numerically (relative to each column's scale)
SHIPPED_GPU_TOLERANCE = {"chlorum_2x2": 1e-11}


def _files(d):
    found = {}
    for root, _, names in os.walk(d):
        for n in names:
            full = os.path.join(root, n)
            found[os.path.relpath(full, d)] = open(full, "rb").read()
    return found


def _key(prefix, rel):
    return prefix + ":" + rel.replace(os.sep, "|")


def _save(name, d, inputs, runs_main, rcs, tol, logs, gpu_tol=None):
    data = {_key("in", rel): np.frombuffer(b, dtype=np.uint8) for rel, b in inputs.items()}
    for r, main_txt in enumerate(runs_main):
        data[f"run{r}:main.txt"] = np.frombuffer(main_txt.encode(), dtype=np.uint8)
    for rel, b in _files(d).items():
        if rel.startswith("set" + os.sep):
            continue
        data[_key("out", rel)] = np.frombuffer(b, dtype=np.uint8)
    data["runs"] = np.int64(len(runs_main))
    data["rc"] = np.asarray(rcs, dtype=np.int64)
    data["tolerance"] = np.float64(tol)
    if gpu_tol is not None:
        data["gpu_tolerance"] = np.float64(gpu_tol)
    # the end of what the reference printed (a failed run's error message is among its last lines)
    data["log_tails"] = np.asarray([lg[-600:] for lg in logs])
    np.savez_compressed(os.path.join(HERE, f"deck_{name}.npz"), **data)
    outs = sorted(k for k in data if k.startswith("out:result|output_"))
    print(f"deck_{name}: {len(runs_main)} run(s), exit {rcs}, outputs {[k.split('_')[-1] for k in outs]}")


def _shorten(main_txt: str, t_end: str) -> str:
    """main.txt with #Time_of_calculation replaced, line endings kept."""
    i = main_txt.index(END_KEY)
    j = main_txt.index("\n", i)
    k = main_txt.index("\n", j + 1)
    cr = "\r" if main_txt[k - 1] == "\r" else ""
    return main_txt[:j + 1] + t_end + cr + main_txt[k:]


def shipped(binary, only=None):
    """Fixtures of the reference's own task decks, their set/ directories unchanged (a long deck
    with only its #Time_of_calculation shortened)."""
    for name, rel, *t_end in SHIPPED:
        if only and name not in only:
            continue
        d = tempfile.mkdtemp(prefix="schemi_deck_")
        try:
            shutil.copytree(os.path.join(SHIPPED_ROOT, rel, "set"), os.path.join(d, "set"))
            if t_end:
                path = os.path.join(d, "set", "main.txt")
                with open(path, newline="") as f:
                    txt = f.read()
                with open(path, "w", newline="") as f:
                    f.write(_shorten(txt, t_end[0]))
            inputs = _files(d)
            main_txt = inputs[os.path.join("set", "main.txt")].decode()
            res = subprocess.run([binary], cwd=d, stdin=subprocess.DEVNULL, stdout=subprocess.PIPE,
                                 stderr=subprocess.STDOUT, timeout=1800)
            _save(name, d, inputs, [main_txt], [res.returncode], 0.0, [res.stdout.decode(errors="replace")],
                  SHIPPED_GPU_TOLERANCE.get(name))
        finally:
            shutil.rmtree(d, ignore_errors=True)


def main(only=None):
    binary = O.REF_BIN_PATCHED
    if not os.path.exists(binary):
        raise SystemExit(f"{binary} missing: run make -C oracle ref")
    shipped(binary, only)
    for name, case, prim, freq, restart, runs, tol, *extra in deck_cases():
        if only and name not in only:
            continue
        d = tempfile.mkdtemp(prefix="schemi_deck_")
        extra = dict(extra[0]) if extra else {}
        gpu_tol = extra.pop("gpu_tolerance", None)
        try:
            write_deck(case, d, prim, frequency_of_output=freq, restart=restart, **extra)
            inputs = _files(d)
            base = inputs[os.path.join("set", "main.txt")].decode()
            data = {_key("in", rel): np.frombuffer(b, dtype=np.uint8) for rel, b in inputs.items()}
            rcs = []
            for r, edits in enumerate(runs):
                main_txt = _set_main(base, **edits)
                with open(os.path.join(d, "set", "main.txt"), "w") as f:
                    f.write(main_txt)
                data[f"run{r}:main.txt"] = np.frombuffer(main_txt.encode(), dtype=np.uint8)
                res = subprocess.run([binary], cwd=d, stdin=subprocess.DEVNULL, stdout=subprocess.PIPE,
                                     stderr=subprocess.STDOUT, timeout=600)
                rcs.append(res.returncode)
                if res.returncode != 0:
                    raise RuntimeError(f"{name} run {r}: reference failed\n" +
                                       res.stdout.decode(errors="replace")[-2000:])
            for rel, b in _files(d).items():
                if rel.startswith("set" + os.sep):
                    continue
                data[_key("out", rel)] = np.frombuffer(b, dtype=np.uint8)
            data["runs"] = np.int64(len(runs))
            data["rc"] = np.asarray(rcs, dtype=np.int64)
            data["tolerance"] = np.float64(tol)
            if gpu_tol is not None:
                data["gpu_tolerance"] = np.float64(gpu_tol)
            np.savez_compressed(os.path.join(HERE, f"deck_{name}.npz"), **data)
            outs = sorted(k for k in data if k.startswith("out:result|output_"))
            print(f"deck_{name}: {len(runs)} run(s), outputs {[k.split('_')[-1] for k in outs]}")
        finally:
            shutil.rmtree(d, ignore_errors=True)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
