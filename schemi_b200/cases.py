"""Seeded synthetic cases with the shapes of the benchmark configurations.

No dataset is involved: every initial field is generated here from a seed (PCG64 through
``numpy.random.default_rng``).  Each builder returns ``(Case, prim)`` where ``prim`` is the
restart set c_1..c_N, v_x, v_y, v_z, p in cell order (x fastest).  ``scale`` shrinks the mesh
for tests (cells per axis divided by ``scale``) while keeping the physics of the workload.

  shock_tube_1d        1D two-species shock tube, 1000 cells, HLLC + minmod, CFL 0.5, t = 0.2
  kelvin_helmholtz_2d  2D mixing layer 1024^2, periodic x / slip y, HLLC + vanLeer, t = 1
  reacting_shear_3d    3D reacting shear layer 256^3, vdW EOS, A+B->2C, periodic x and z
  chlorine_dissociation_2d  hot Cl2/Cl mixture with the reference's Cl2 mechanism (chemistry pin)
  richtmyer_meshkov    one 2D shock-tube case of the 512-case ensemble (sizes 128^2..512^2)
  rayleigh_taylor_2d   2D RT 512x1536 with gravity and a 64-mode interface perturbation
"""

from __future__ import annotations

import math
from typing import List, Sequence, Tuple

import numpy as np

from .case import BC, R_SI, Case, PatchBC, Species


def _centres(n: int, L: float) -> np.ndarray:
    return (np.arange(n) + 0.5) * (L / n)


def shock_tube_1d(n: int = 1000, limiter: str = "minmod", flux: str = "HLLC", precision: str = "f64",
                  t_end: float = 0.2) -> Tuple[Case, list]:
    """Two-component shock tube: left rho=1,u=0,p=1 species A (gamma 1.4), right rho=0.125,
    p=0.1 species B (gamma 1.67), transmissive ends, R = 1 units (M = 1, Cv = R/(gamma-1))."""
    sp = [Species(M=1.0, Cv=1.0 / 0.4), Species(M=1.0, Cv=1.0 / 0.67)]
    case = Case(dims=1, n=(n, 1, 1), L=(1.0, 1.0, 1.0), species=sp, t_end=t_end, limiter=limiter, flux=flux,
                courant=0.5, min_timestep=1e-15, precision=precision, name="shock_tube_1d")
    x = _centres(n, 1.0)
    left = x < 0.5
    cA = np.where(left, 1.0, 0.0)
    cB = np.where(left, 0.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    z = np.zeros(n)
    return case, [cA, cB, z, z.copy(), z.copy(), p]


def diffusion_tube_1d(n: int = 1000, t_end: float = 0.3) -> Tuple[Case, list]:
    """Interdiffusion of two ideal gases of equal molar mass at rest: c_1 = 0.05 mol/m^3 for
    x < 0.5, c_2 = 0.05 beyond, p = 100 Pa, slip ends, SI units (M = 28.8, Cv = 20.78615655),
    vanAlbada, HLLC, Courant 0.47; the diffusion stage with the explicit solver, mu = 2e-7,
    D = 2e-2, kappa = 2e-4, the explicit enthalpy flow, the molar-mass correction and the
    Courant-Source-Diffusion=0.25,0.5 limit -- the parameters of the reference's
    tests/TestsTasks/Diffusion/Diffusion_1000 deck."""
    sp = [Species(M=28.8, Cv=20.78615655, Tc=1.0, Pc=1.0) for _ in range(2)]
    case = Case(dims=1, n=(n, 1, 1), L=(1.0, 1.0, 1.0), species=sp, t_end=t_end, R_units="SI",
                limiter="vanAlbada", courant=0.47, min_timestep=1e-15, name="diffusion_tube_1d")
    case.bc["tail"] = PatchBC.uniform("slip", 2)
    case.bc["point"] = PatchBC.uniform("slip", 2)
    case.diffusion, case.mu, case.D, case.kappa = True, 2e-7, 2e-2, 2e-4
    case.enthalpy_flow, case.molmass_diffusion, case.diffusion_timestep = "explicit", True, True
    x = _centres(n, 1.0)
    left = x < 0.5
    z = np.zeros(n)
    return case, [np.where(left, 0.05, 0.0), np.where(left, 0.0, 0.05), z, z.copy(), z.copy(), np.full(n, 100.0)]


def poiseuille_2d(n: int = 100, t_end: float = 2e-3) -> Tuple[Case, list]:
    """A van der Waals gas (M = 0.0288, Cv = 20.8572, Tc = 131.523 K, Pc = 4.108e6 Pa) at rest in
    a channel [0, 1] x [0, 0.5] m, c = 37.615 mol/m^3, p = 101317 Pa, driven by p = 101325 Pa held
    at the inlet (fixedValueCell) and a free outlet, walls with v = 0 (fixedValueCell) and slip
    concentration and pressure, SI units, vanAlbada, HLLC, Courant 0.47; the diffusion stage with
    the Gauss-Seidel solver (2000 iterations), mu = D = 2e-3, kappa = 2, the explicit enthalpy
    flow and the molar-mass correction, Courant-Source=0.25,0.5 -- the parameters of the
    reference's tests/TestsTasks/PoiseuilleFlow/PoiseuilleFlow_SI_100x100 deck (whose 2.0 s this
    shortens to t_end)."""
    sp = [Species(M=0.0288, Cv=20.8572, Tc=131.523, Pc=4.108e6)]
    case = Case(dims=2, n=(n, n, 1), L=(1.0, 0.5, 1.0), species=sp, t_end=t_end, R_units="SI",
                eos="vanDerWaals", limiter="vanAlbada", courant=0.47, min_timestep=1e-15, name="poiseuille_2d")
    case.bc["tail"] = PatchBC([BC("freeBoundary")], BC("freeBoundary"), BC("fixedValueCell", 101325.0))
    case.bc["point"] = PatchBC.uniform("freeBoundary", 1)
    for wall in ("right", "left"):
        case.bc[wall] = PatchBC([BC("slip")], BC("fixedValueCell", (0.0, 0.0, 0.0)), BC("slip"))
    case.diffusion, case.sle_solver, case.sle_max_iter = True, "GaussSeidel", 2000
    case.mu, case.D, case.kappa = 2e-3, 2e-3, 2.0
    case.enthalpy_flow, case.molmass_diffusion, case.diffusion_timestep = "explicit", True, False
    z = np.zeros(n * n)
    return case, [np.full(n * n, 37.615), z, z.copy(), z.copy(), np.full(n * n, 101317.0)]


def real_gas_tube(eos: str, n: int = 200, limiter: str = "minmod") -> Tuple[Case, list]:
    """Two-component shock tube for the equations of state beyond ideal and van der Waals
    (transmissive ends, HLLC).
    stiffened: R = 1 units, left a stiffened liquid-like species (gamma 2, p0 0.5; rho 1, p 1),
    right a gas (gamma 1.4, p0 0; rho 0.125, p 0.1).
    RedlichKwong / Kataoka: SI units on a 1 m tube, nitrogen- and argon-like species (critical
    points 126.2 K / 3.39 MPa and 150.9 K / 4.9 MPa; Kataoka: Lennard-Jones eps 95 R and 120 R
    J/mol, sigma 3.7e-10 and 3.4e-10 m, b from the critical point), left 1 MPa at 400 mol/m^3,
    right 0.1 MPa at 40 mol/m^3."""
    x = _centres(n, 1.0)
    left = x < 0.5
    z = np.zeros(n)
    if eos == "stiffened":
        sp = [Species(M=1.0, Cv=1.0, p0=0.5, gamma=2.0), Species(M=1.0, Cv=1.0 / 0.4, p0=0.0, gamma=1.4)]
        case = Case(dims=1, n=(n, 1, 1), L=(1.0, 1.0, 1.0), species=sp, t_end=0.2, limiter=limiter, eos=eos,
                    courant=0.5, min_timestep=1e-15, name="stiffened_tube")
        cA = np.where(left, 1.0, 0.0)
        cB = np.where(left, 0.0, 0.125)
        p = np.where(left, 1.0, 0.1)
        return case, [cA, cB, z, z.copy(), z.copy(), p]
    R = R_SI
    sp = [Species(M=0.028, Cv=20.8, Tc=126.2, Pc=3.39e6, lj_eps=95.0 * R, lj_sigma=3.7e-10),
          Species(M=0.040, Cv=12.5, Tc=150.9, Pc=4.9e6, lj_eps=120.0 * R, lj_sigma=3.4e-10)]
    case = Case(dims=1, n=(n, 1, 1), L=(1.0, 1.0, 1.0), species=sp, t_end=1e-3, limiter=limiter, eos=eos,
                R_units="SI", courant=0.5, min_timestep=1e-15, name=f"{eos}_tube")
    cA = np.where(left, 400.0, 0.0)
    cB = np.where(left, 0.0, 40.0)
    p = np.where(left, 1.0e6, 1.0e5)
    return case, [cA, cB, z, z.copy(), z.copy(), p]


def kelvin_helmholtz_2d(n: int = 1024, precision: str = "f64", seed: int = 2026, t_end: float = 1.0,
                        periodic: bool = True, limiter: str = "vanLeer") -> Tuple[Case, list]:
    """KH mixing layer on [0,1]^2: band |y-0.5|<0.25 is species A (M=29) with rho=2, u=+0.5;
    outside species B (M=4) with rho=1, u=-0.5; p=2.5; gamma 1.4 for both;
    v = 0.01 sin(4 pi x) + U(-1e-3, 1e-3).  Periodic in x (slip when ``periodic`` is False,
    which makes the case expressible in the reference), slip in y."""
    sp = [Species(M=29.0, Cv=1.0 / 0.4), Species(M=4.0, Cv=1.0 / 0.4)]
    xk = "periodic" if periodic else "slip"
    bc = {"tail": PatchBC.uniform(xk, 2), "point": PatchBC.uniform(xk, 2),
          "right": PatchBC.uniform("slip", 2), "left": PatchBC.uniform("slip", 2)}
    case = Case(dims=2, n=(n, n, 1), L=(1.0, 1.0, 1.0), species=sp, t_end=t_end, limiter=limiter, flux="HLLC",
                courant=0.5, bc=bc, precision=precision, name="kelvin_helmholtz_2d")
    x = _centres(n, 1.0)[None, :]
    y = _centres(n, 1.0)[:, None]
    band = np.abs(y - 0.5) < 0.25
    rng = np.random.default_rng(seed)
    cA = np.where(band, 2.0 / 29.0, 0.0) * np.ones((n, n))
    cB = np.where(band, 0.0, 1.0 / 4.0) * np.ones((n, n))
    u = np.where(band, 0.5, -0.5) * np.ones((n, n))
    v = 0.01 * np.sin(4 * np.pi * x) + rng.uniform(-1e-3, 1e-3, size=(n, n))
    p = np.full((n, n), 2.5)
    z = np.zeros((n, n))
    return case, [cA.ravel(), cB.ravel(), u.ravel(), v.ravel(), z.ravel(), p.ravel()]


def richtmyer_meshkov_draws(index: int, base_seed: int = 2028) -> Tuple[int, float, float, float]:
    """Seeded draws of ensemble case ``index``: cells per axis n ~ U{128..512}, interface
    amplitude a ~ U(0.01, 0.05), wavelength lam ~ U(0.25, 1), end time in shock transits ~ U(2, 4)."""
    rng = np.random.default_rng(base_seed + index)
    n = int(rng.integers(128, 513))
    a = float(rng.uniform(0.01, 0.05))
    lam = float(rng.uniform(0.25, 1.0))
    transits = float(rng.uniform(2.0, 4.0))
    return n, a, lam, transits


def richtmyer_meshkov(index: int, n: int = 0, precision: str = "f32flux", limiter: str = "superbee",
                      base_seed: int = 2028) -> Tuple[Case, list, float]:
    """Case ``index`` of the RM ensemble: light gas (gamma 1.4, rho 1) left of the interface
    x = 0.5 + a cos(2 pi y / lam), heavy gas (gamma 1.09, rho 5) right of it, p = 1; a Mach 1.2
    shock in the light gas starts at x = 0.3 (post-shock state from Rankine-Hugoniot).
    n ~ U{128..512} (seed base_seed + index) unless given; free at x=0, slip elsewhere.
    Returns (case, prim, t_end) with t_end ~ U(2, 4) shock transit times of the unit box."""
    n_draw, a, lam, transits = richtmyer_meshkov_draws(index, base_seed)
    n = n or n_draw
    g1, g2 = 1.4, 1.09
    sp = [Species(M=1.0, Cv=1.0 / (g1 - 1.0)), Species(M=5.0, Cv=1.0 / (g2 - 1.0))]
    bc = {"tail": PatchBC.uniform("freeBoundary", 2), "point": PatchBC.uniform("slip", 2),
          "right": PatchBC.uniform("slip", 2), "left": PatchBC.uniform("slip", 2)}
    # Rankine-Hugoniot, light gas at rest: rho=1, p=1, c=sqrt(g p / rho)
    Ms = 1.2
    c0 = math.sqrt(g1 * 1.0 / 1.0)
    p2 = 1.0 * (1 + 2 * g1 / (g1 + 1) * (Ms * Ms - 1))
    rho2 = 1.0 * ((g1 + 1) * Ms * Ms) / ((g1 - 1) * Ms * Ms + 2)
    Ws = Ms * c0
    u2 = Ws * (1 - 1.0 / rho2)
    t_end = transits / Ws
    case = Case(dims=2, n=(n, n, 1), L=(1.0, 1.0, 1.0), species=sp, t_end=t_end, limiter=limiter, flux="HLLC",
                courant=0.5, bc=bc, precision=precision, name=f"richtmyer_meshkov_{index}")
    x = _centres(n, 1.0)[None, :] * np.ones((n, 1))
    y = _centres(n, 1.0)[:, None] * np.ones((1, n))
    heavy = x > 0.5 + a * np.cos(2 * np.pi * y / lam)
    shocked = x < 0.3
    cA = np.where(heavy, 0.0, np.where(shocked, rho2, 1.0) / 1.0)
    cB = np.where(heavy, 5.0 / 5.0, 0.0)
    u = np.where(shocked, u2, 0.0)
    p = np.where(shocked, p2, 1.0)
    z = np.zeros((n, n))
    return case, [cA.ravel(), cB.ravel(), u.ravel(), z.ravel(), z.ravel(), p.ravel()], t_end


def rayleigh_taylor_2d(nx: int = 512, ny: int = 1536, modes: int = 64, seed: int = 2029,
                       amplitudes: Sequence[float] = None, precision: str = "f64", t_end: float = 5.0,
                       limiter: str = "vanLeer") -> Tuple[Case, list]:
    """RT on [0,1]x[0,3]: heavy (rho=3) over light (rho=1), gamma 1.4 both, g = (0, -0.1),
    hydrostatic p with p = 2.5 at y = 1.5; interface eta(x) = sum_m a_m cos(2 pi m x) with
    a_m ~ N(0, 1e-3); cells initialised with the exact heavy volume fraction per column.
    Slip on all walls."""
    rng = np.random.default_rng(seed)
    a = np.asarray(amplitudes if amplitudes is not None else rng.normal(0.0, 1e-3, size=modes), dtype=np.float64)
    sp = [Species(M=3.0, Cv=1.0 / 0.4), Species(M=1.0, Cv=1.0 / 0.4)]
    bc = {p: PatchBC.uniform("slip", 2) for p in ("tail", "point", "right", "left")}
    case = Case(dims=2, n=(nx, ny, 1), L=(1.0, 3.0, 1.0), species=sp, t_end=t_end, limiter=limiter, flux="HLLC",
                courant=0.5, gravity=(0.0, -0.1, 0.0), bc=bc, precision=precision, name="rayleigh_taylor_2d")
    prim = rt_fields(nx, ny, a)
    return case, prim


def rt_interface(x: np.ndarray, a: np.ndarray) -> np.ndarray:
    m = np.arange(1, a.size + 1)
    return 1.5 + np.cos(2 * np.pi * np.outer(x, m)) @ a


def rt_fields(nx: int, ny: int, a: np.ndarray) -> list:
    dy = 3.0 / ny
    xc = _centres(nx, 1.0)
    eta = rt_interface(xc, a)                    # (nx,)
    y_lo = np.arange(ny)[:, None] * dy           # (ny, 1)
    # heavy fraction: part of the cell above the interface
    frac = np.clip((y_lo + dy - eta[None, :]) / dy, 0.0, 1.0)
    yc = (np.arange(ny)[:, None] + 0.5) * dy
    g = 0.1
    # hydrostatic pressure integrated from the interface: dp/dy = -rho g
    rho_mix = 3.0 * frac + 1.0 * (1 - frac)
    p = 2.5 - g * np.where(yc > 1.5, 3.0 * (yc - 1.5), 1.0 * (yc - 1.5)) * np.ones((1, nx))
    cA = 3.0 * frac / 3.0
    cB = 1.0 * (1 - frac) / 1.0
    z = np.zeros((ny, nx))
    del rho_mix
    return [cA.ravel(), cB.ravel(), z.ravel(), z.ravel(), z.ravel(), p.ravel()]


def chlorine_dissociation_2d(n: int = 4, T0: float = 1500.0, p0: float = 1e5, seed: int = 2030,
                             eos: str = "vanDerWaals", precision: str = "f64",
                             solver: str = "Gauss-Seidel") -> Tuple[Case, list]:
    """Hot Cl2 / Cl mixture on [0,1]^2 m (SI) with the species, Arrhenius parameters and solver of
    the reference's ClorumTest deck (tests/Chemical Reactions/ClorumTest/Chlorum/set: Cl2 M=0.0709,
    Cv=25.635, Tc=416.9 K, Pc=7.9773e6 Pa; Cl M=0.03545, Cv=12.471; dissociation A=5.74e9, n=0,
    E=232613.66 J/mol; recombination A=2.3e7, n=-1.5, E=0; Gauss-Seidel, 200 iterations), slip
    walls, at rest, with seeded cell-to-cell variations of temperature (T0 +- 10%) and of the
    Cl fraction (0..20%) so that every cell reacts at its own rate."""
    from .case import R_SI

    R = R_SI
    sp = [Species(M=0.0709, Cv=25.635, Tc=416.9, Pc=7.9773e6), Species(M=0.03545, Cv=12.471, Tc=0.0, Pc=1.0)]
    bc = {p: PatchBC.uniform("slip", 2) for p in ("tail", "point", "right", "left")}
    case = Case(dims=2, n=(n, n, 1), L=(1.0, 1.0, 1.0), species=sp, t_end=1.0, R_units="SI", eos=eos,
                limiter="vanAlbada", flux="HLLC", courant=0.47, bc=bc, precision=precision, chemistry="Cl2",
                chem_forward=(5.74e9, 0.0, 232613.66), chem_backward=(2.3e7, -1.5, 0.0), chem_solver=solver,
                chem_max_iter=200, name="chlorine_dissociation_2d")
    rng = np.random.default_rng(seed)
    T = T0 * (1 + 0.1 * rng.uniform(-1, 1, size=n * n))
    xCl = 0.2 * rng.uniform(0, 1, size=n * n)
    # total concentration from p0 at T (vdW with mole-fraction mixing of a and b)
    a = np.array([27 * R * R * s.Tc ** 2 / (64 * s.Pc) for s in sp])
    b = np.array([R * s.Tc / (8 * s.Pc) for s in sp])
    X = np.stack([1 - xCl, xCl])
    am = sum(X[k] * X[l] * np.sqrt(a[k] * a[l]) for k in range(2) for l in range(2))
    bm = sum(X[k] * X[l] * 0.5 * (b[k] + b[l]) for k in range(2) for l in range(2))
    c = p0 / (R * T)
    if eos == "vanDerWaals":
        for _ in range(50):
            f = R * T * c / (1 - c * bm) - am * c * c - p0
            df = R * T / (1 - c * bm) ** 2 - 2 * am * c
            c = c - f / df
    z = np.zeros(n * n)
    return case, [c * X[0], c * X[1], z, z, z, np.full(n * n, p0)]


def reacting_shear_3d(n: int = 256, seed: int = 2027, precision: str = "f32flux", t_end: float = 1e-3,
                      periodic: bool = True) -> Tuple[Case, list]:
    """3D reacting shear layer on [0,1]^3 m (SI units): species A, B, C with M = 0.029 kg/mol,
    molar Cv = 1005*0.029 - R; van der Waals a = 0.1370 Pa m^6/mol^2, b = 3.87e-5 m^3/mol entered
    as Tc = 8a/(27Rb), Pc = a/(27b^2); A above y = 0.5 at +50 m/s, B below at -50 m/s with a
    tanh profile of thickness 0.05; T0 = 300 K, p = 101325 Pa; 1% (0.5 m/s) uniform velocity
    noise; A + B -> 2C with rate A c_A c_B exp(-8000/T), A = 1e9, heat release
    2e6 J/kg * 0.058 kg per mol of reaction.  Periodic x and z, slip y."""
    from .case import R_SI

    R = R_SI
    a_vdw, b_vdw = 0.1370, 3.87e-5
    Tc = 8 * a_vdw / (27 * R * b_vdw)
    Pc = a_vdw / (27 * b_vdw * b_vdw)
    Cv = 1005.0 * 0.029 - R
    sp = [Species(M=0.029, Cv=Cv, Tc=Tc, Pc=Pc) for _ in range(3)]
    xk = "periodic" if periodic else "slip"
    bc = {"tail": PatchBC.uniform(xk, 3), "point": PatchBC.uniform(xk, 3),
          "bottom": PatchBC.uniform(xk, 3), "top": PatchBC.uniform(xk, 3),
          "right": PatchBC.uniform("slip", 3), "left": PatchBC.uniform("slip", 3)}
    case = Case(dims=3, n=(n, n, n), L=(1.0, 1.0, 1.0), species=sp, t_end=t_end, R_units="SI",
                eos="vanDerWaals", limiter="vanLeer", flux="HLLC", courant=0.5, bc=bc, precision=precision,
                chemistry="A+B->2C", chem_forward=(1e9, 0.0, 8000.0 * R), chem_q=2e6 * 0.058,
                name="reacting_shear_3d")
    rng = np.random.default_rng(seed)
    yc = _centres(n, 1.0)[None, :, None] * np.ones((n, n, n))
    s = 0.5 * (1 + np.tanh((yc - 0.5) / 0.05))          # 1 above, 0 below
    T0, p0 = 300.0, 101325.0
    # total molar concentration from the vdW equation of state at (p0, T0): solve by Newton
    c = p0 / (R * T0)
    for _ in range(50):
        f = R * T0 * c / (1 - c * b_vdw) - a_vdw * c * c - p0
        df = R * T0 / (1 - c * b_vdw) ** 2 - 2 * a_vdw * c
        c -= f / df
    cA = c * s
    cB = c * (1 - s)
    cC = np.zeros_like(cA)
    u = 50.0 * (2 * s - 1) + rng.uniform(-0.5, 0.5, size=cA.shape)
    v = rng.uniform(-0.5, 0.5, size=cA.shape)
    w = rng.uniform(-0.5, 0.5, size=cA.shape)
    p = np.full(cA.shape, p0)
    return case, [cA.ravel(), cB.ravel(), cC.ravel(), u.ravel(), v.ravel(), w.ravel(), p.ravel()]
