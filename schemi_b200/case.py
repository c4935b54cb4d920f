"""Case description shared by the task-file writer, the C-ABI binding and the tests.

A :class:`Case` holds what the reference reads from its task files (``set/main.txt``,
``set/sub_k.txt``, ``set/velocity.txt``, ``set/pressure.txt``, ``set/g.txt``): mesh, species,
equation of state, flux solver, limiter, boundary conditions and time-step controls.
:meth:`Case.fv_config` turns it into the ``fv_config`` struct of ``include/fvstep.h``.

Name strings are the reference's factory names:
  flux solvers   Schemi/src/interfaces/abstractFlowSolver.cpp:29-35 ("HLLC", "HLL")
  limiters       Schemi/src/interfaces/abstractLimiter.cpp:39-53
  EOS            Schemi/src/interfaces/abstractMixtureThermodynamics.cpp:39-43 ("ideal", "vanDerWaals")
  BC types       Schemi/src/boundary/boundaryConditionFromString.cpp:12-32
  gas constant   Schemi/src/thermodynamics/phaseInitialization.cpp:418-435 ("SI", "1", "CGS", "CGmS")
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

MAX_SPECIES = 4
R_SI = 8.31446261815324  # Schemi/headers/globalConstants.hpp:28

GAS_CONSTANT = {"SI": R_SI, "1": 1.0, "CGS": R_SI * 1e7, "CGmS": R_SI * 1e1}

EOS = {"ideal": 0, "vanDerWaals": 1, "RedlichKwong": 2, "stiffened": 3, "Kataoka": 4}
FLUX = {"HLLC": 0, "HLL": 1}
LIMITERS = ["zero", "minmod", "vanLeer", "linear", "vanAlbada", "HQUICK", "vanLeer2", "superbee",
            "vanAlbada2", "minmod2", "Sweby", "Koren", "Koren2", "UTCDFS", "Schmidtmann"]
LIMITER = {name: i for i, name in enumerate(LIMITERS)}
BC_TYPES = {"freeBoundary": 1, "slip": 2, "fixedValueCell": 3, "fixedValueSurface": 4, "periodic": 100}
PRECISION = {"f64": 0, "f32flux": 1}
CHEMISTRY = {"no": 0, "A+B->2C": 1, "Cl2": 2}
# set/chemicalKinetics.txt #Iterative_solver names (abstractChemicalKinetics.cpp:21-29)
CHEM_SOLVERS = {"Gauss-Seidel": 0, "Jacobi": 1, "GaussElimination": 2, "conjugateGradient": 3,
                "JacobiConjugateGradient": 4}
# #Approximation_order values with a GPU step (abstractStepSolver.cpp:56-146)
ORDERS = {"SecondOrder": 0, "SecondOrderRK": 1, "ThirdOrder": 2, "ThirdOrderCada": 3}
SLE_SOLVERS = {"explicit": 0, "GaussSeidel": 1, "Jacobi": 2, "Thomas": 3, "noSolver": 4, "conjugateGradient": 5,
               "JacobiConjugateGradient": 6, "biConjugateGradient": 7}
TRANSPORT_MODELS = {"constant": 0, "hardSpheres": 1, "LennardJones": 2}
ENTHALPY_FLOWS = {"no": 0, "explicit": 1, "implicit": 2}

# patch order of the task files: #Tail, #Point, #Bottom, #Right, #Left, #Top
PATCHES = ["tail", "point", "bottom", "right", "left", "top"]
# which patches a task of dimension D uses (the others are "blank" in the task files)
PATCHES_USED = {1: ["tail", "point"], 2: ["tail", "point", "right", "left"],
                3: ["tail", "point", "bottom", "right", "left", "top"]}


class fv_arrhenius_t(ctypes.Structure):
    """Mirror of ``fv_arrhenius``: k = A T^n exp(-E / (R T))."""

    _fields_ = [("A", ctypes.c_double), ("n", ctypes.c_double), ("E", ctypes.c_double)]


class fv_config_t(ctypes.Structure):
    """Mirror of ``fv_config`` in include/fvstep.h."""

    _fields_ = [
        ("dims", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("L", ctypes.c_double * 3),
        ("n_species", ctypes.c_int),
        ("R", ctypes.c_double),
        ("M", ctypes.c_double * MAX_SPECIES),
        ("Cv", ctypes.c_double * MAX_SPECIES),
        ("Tc", ctypes.c_double * MAX_SPECIES),
        ("Pc", ctypes.c_double * MAX_SPECIES),
        ("eos", ctypes.c_int),
        ("flux", ctypes.c_int),
        ("limiter", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("courant", ctypes.c_double),
        ("min_timestep", ctypes.c_double),
        ("courant_only", ctypes.c_int),
        ("gravity", ctypes.c_int),
        ("g", ctypes.c_double * 3),
        ("g_delta", ctypes.c_double * 3),
        ("bc_conc", (ctypes.c_int * MAX_SPECIES) * 6),
        ("bc_conc_value", (ctypes.c_double * MAX_SPECIES) * 6),
        ("bc_vel", ctypes.c_int * 6),
        ("bc_vel_value", (ctypes.c_double * 3) * 6),
        ("bc_p", ctypes.c_int * 6),
        ("bc_p_value", ctypes.c_double * 6),
        ("chemistry", ctypes.c_int),
        ("chem_forward", fv_arrhenius_t),
        ("chem_backward", fv_arrhenius_t),
        ("chem_q", ctypes.c_double),
        ("chem_solver", ctypes.c_int),
        ("chem_max_iter", ctypes.c_int),
        ("const_timestep", ctypes.c_double),
        ("order", ctypes.c_int),
        ("stiff_p0", ctypes.c_double * MAX_SPECIES),
        ("stiff_gamma", ctypes.c_double * MAX_SPECIES),
        ("lj_eps", ctypes.c_double * MAX_SPECIES),
        ("lj_sigma", ctypes.c_double * MAX_SPECIES),
        ("kataoka_b_critical", ctypes.c_int),
        ("kataoka_b_coeff", ctypes.c_double),
        ("diffusion", ctypes.c_int),
        ("sle_solver", ctypes.c_int),
        ("sle_max_iter", ctypes.c_int),
        ("transport", ctypes.c_int),
        ("mu_const", ctypes.c_double),
        ("D_const", ctypes.c_double),
        ("kappa_const", ctypes.c_double),
        ("enthalpy_flow", ctypes.c_int),
        ("molmass_diffusion", ctypes.c_int),
        ("linear_reconstruction", ctypes.c_int),
        ("diffusion_timestep", ctypes.c_int),
        ("dt_coeff_source", ctypes.c_double),
        ("dt_coeff_diffusion", ctypes.c_double),
        ("transport_diameter", ctypes.c_double * MAX_SPECIES),
        ("transport_lj_eps", ctypes.c_double * MAX_SPECIES),
        ("transport_lj_sigma", ctypes.c_double * MAX_SPECIES),
    ]


@dataclass
class Species:
    """One ``set/sub_k.txt``: molar mass, molar Cv and the van der Waals critical point."""

    M: float
    Cv: float
    Tc: float = 1.0
    Pc: float = 1.0
    p0: float = 0.0      # stiffened gas (set/stiffenedFluidData.txt)
    gamma: float = 1.4
    lj_eps: float = 0.0  # Kataoka (set/KataokaVanDerWaalsFluidData.txt)
    lj_sigma: float = 0.0
    # transport models (sub_k.txt #Kinetic_diameter_(A), #Lennard_Jones_eps/kB_(K),
    # #Lennard_Jones_sigma_(A))
    diameter: float = 1.0
    tr_eps: float = 1.0
    tr_sigma: float = 1.0


@dataclass
class BC:
    """Boundary condition of one field on one patch: a type name and, for fixedValue*, a value."""

    kind: str = "freeBoundary"
    value: object = 0.0

    def task_string(self, vector: bool) -> str:
        if self.kind in ("fixedValueCell", "fixedValueSurface"):
            if vector:
                return f"{self.kind} " + " ".join(repr(float(x)) for x in self.value)
            return f"{self.kind} {float(self.value)!r}"
        return self.kind


@dataclass
class PatchBC:
    """Boundary conditions of all fields on one patch."""

    conc: List[BC]
    vel: BC
    p: BC

    @staticmethod
    def uniform(kind: str, n_species: int) -> "PatchBC":
        return PatchBC([BC(kind) for _ in range(n_species)], BC(kind), BC(kind))


@dataclass
class Case:
    dims: int
    n: Tuple[int, int, int]
    L: Tuple[float, float, float]
    species: List[Species]
    t_end: float
    R_units: str = "1"
    eos: str = "ideal"
    flux: str = "HLLC"
    limiter: str = "minmod"
    courant: float = 0.5
    min_timestep: float = 1e-15
    courant_only: bool = False
    gravity: Optional[Tuple[float, float, float]] = None
    g_delta: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    bc: Dict[str, PatchBC] = field(default_factory=dict)
    precision: str = "f64"
    chemistry: str = "no"
    chem_forward: Tuple[float, float, float] = (0.0, 0.0, 0.0)   # Arrhenius A, n, E (J/mol)
    chem_backward: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    chem_q: float = 0.0
    chem_solver: str = "Gauss-Seidel"
    chem_max_iter: int = 200
    const_timestep: float = 0.0   # > 0: every step takes this dt (#Constant_timestep)
    order: str = "SecondOrder"    # #Approximation_order: a key of ORDERS
    name: str = "case"
    # Kataoka-van der Waals b rule (set/KataokaVanDerWaalsFluidData.txt): "critical" (b = coeff R Tc
    # / (8 Pc)) or "Kataoka" (b = coeff sigma^3 N_A), and its coefficient
    kataoka_b: Tuple[str, float] = ("critical", 1.0)
    # diffusion stage (#Diffusion_flag, #Type_of_SLE_solver_flag, set/transportCoefficients.txt,
    # #Reconstruction, #Source_timestep_correction "Courant-Source-Diffusion=<source>,<diffusion>")
    diffusion: bool = False
    sle_solver: str = "explicit"          # a key of SLE_SOLVERS
    sle_max_iter: int = 2000
    transport: str = "constant"           # a key of TRANSPORT_MODELS
    mu: float = 0.0                       # #Viscosity_coefficient
    D: float = 0.0                        # #Diffusion_coefficient
    kappa: float = 0.0                    # #Heat_conduction_coefficient
    enthalpy_flow: str = "explicit"       # a key of ENTHALPY_FLOWS
    molmass_diffusion: bool = True
    reconstruction: str = "star"          # "star" or "linear"
    diffusion_timestep: bool = False
    dt_coeffs: Tuple[float, float] = (0.25, 0.5)

    def __post_init__(self):
        for p in PATCHES_USED[self.dims]:
            if p not in self.bc:
                self.bc[p] = PatchBC.uniform("freeBoundary", len(self.species))

    @property
    def n_species(self) -> int:
        return len(self.species)

    @property
    def n_cells(self) -> int:
        nx, ny, nz = self.n
        return nx * (ny if self.dims >= 2 else 1) * (nz if self.dims >= 3 else 1)

    @property
    def shape(self) -> Tuple[int, ...]:
        """Array shape in C order (z, y, x) of the dimensions used."""
        return tuple(reversed(self.n[: self.dims]))

    @property
    def n_conserved(self) -> int:
        """rho_1..rho_N, rho, m_x, m_y, m_z, E."""
        return self.n_species + 5

    @property
    def R(self) -> float:
        return GAS_CONSTANT[self.R_units]

    def periodic_axes(self) -> List[int]:
        axes = []
        for ax, (lo, hi) in enumerate([("tail", "point"), ("right", "left"), ("bottom", "top")]):
            if lo in self.bc and self.bc[lo].vel.kind == "periodic":
                axes.append(ax)
        return axes

    def expressible_in_reference(self) -> bool:
        """The reference has no periodic patch and no A+B->2C mechanism."""
        return not self.periodic_axes() and self.chemistry in ("no", "Cl2")

    def fv_config(self) -> fv_config_t:
        c = fv_config_t()
        c.dims = self.dims
        for d in range(3):
            c.n[d] = int(self.n[d])
            c.L[d] = float(self.L[d])
        if len(self.species) > MAX_SPECIES:
            raise ValueError(f"at most {MAX_SPECIES} species")
        c.n_species = len(self.species)
        c.R = self.R
        for k, s in enumerate(self.species):
            c.M[k], c.Cv[k], c.Tc[k], c.Pc[k] = s.M, s.Cv, s.Tc, s.Pc
            c.stiff_p0[k], c.stiff_gamma[k] = s.p0, s.gamma
            c.lj_eps[k], c.lj_sigma[k] = s.lj_eps, s.lj_sigma
            c.transport_diameter[k] = s.diameter
            c.transport_lj_eps[k], c.transport_lj_sigma[k] = s.tr_eps, s.tr_sigma
        c.kataoka_b_critical = int(self.kataoka_b[0] == "critical")
        c.kataoka_b_coeff = float(self.kataoka_b[1])
        c.diffusion = int(self.diffusion)
        c.sle_solver = SLE_SOLVERS[self.sle_solver]
        c.sle_max_iter = int(self.sle_max_iter)
        c.transport = TRANSPORT_MODELS[self.transport]
        c.mu_const, c.D_const, c.kappa_const = float(self.mu), float(self.D), float(self.kappa)
        c.enthalpy_flow = ENTHALPY_FLOWS[self.enthalpy_flow]
        c.molmass_diffusion = int(self.molmass_diffusion)
        c.linear_reconstruction = int(self.reconstruction == "linear")
        c.diffusion_timestep = int(self.diffusion_timestep)
        c.dt_coeff_source, c.dt_coeff_diffusion = float(self.dt_coeffs[0]), float(self.dt_coeffs[1])
        c.eos = EOS[self.eos]
        c.flux = FLUX[self.flux]
        c.limiter = LIMITER[self.limiter]
        c.precision = PRECISION[self.precision]
        c.courant = self.courant
        c.min_timestep = self.min_timestep
        c.courant_only = int(self.courant_only)
        c.gravity = int(self.gravity is not None)
        g = self.gravity or (0.0, 0.0, 0.0)
        for d in range(3):
            c.g[d] = g[d]
            c.g_delta[d] = self.g_delta[d]
        for pi, pname in enumerate(PATCHES):
            pb = self.bc.get(pname)
            if pb is None:
                continue
            for k in range(self.n_species):
                c.bc_conc[pi][k] = BC_TYPES[pb.conc[k].kind]
                c.bc_conc_value[pi][k] = float(pb.conc[k].value) if pb.conc[k].kind.startswith("fixed") else 0.0
            c.bc_vel[pi] = BC_TYPES[pb.vel.kind]
            if pb.vel.kind.startswith("fixed"):
                for d in range(3):
                    c.bc_vel_value[pi][d] = float(pb.vel.value[d])
            c.bc_p[pi] = BC_TYPES[pb.p.kind]
            c.bc_p_value[pi] = float(pb.p.value) if pb.p.kind.startswith("fixed") else 0.0
        c.chemistry = CHEMISTRY[self.chemistry]
        c.chem_forward.A, c.chem_forward.n, c.chem_forward.E = self.chem_forward
        c.chem_backward.A, c.chem_backward.n, c.chem_backward.E = self.chem_backward
        c.chem_q = self.chem_q
        c.chem_solver = CHEM_SOLVERS[self.chem_solver]
        c.chem_max_iter = self.chem_max_iter
        c.const_timestep = self.const_timestep
        c.order = ORDERS[self.order]
        return c


def primitive_arrays(case: Case, conc: Sequence, vel: Sequence, p) -> list:
    """Restart set in upload order: c_1..c_N, v_x, v_y, v_z, p (flattened, x fastest)."""
    import numpy as np

    out = [np.ascontiguousarray(np.asarray(c, dtype=np.float64).reshape(-1)) for c in conc]
    out += [np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1)) for v in vel]
    out.append(np.ascontiguousarray(np.asarray(p, dtype=np.float64).reshape(-1)))
    for a in out:
        if a.size != case.n_cells:
            raise ValueError("field size does not match the mesh")
    return out
