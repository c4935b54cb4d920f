"""Task-file (deck) writer and result reader in the reference's formats.

``write_deck`` produces a ``set/`` directory the reference solver accepts, plus a restart
point (``fieldsOutput/output_000001/<field>.dat`` and a two-line ``result/Time.tsv``) so that
arbitrary initial fields enter through the reference's restart reader
(Schemi/main/Schemi.cpp:342-573, Schemi/src/thermodynamics/phaseInitialization.cpp:1382-1746).

File layouts follow the reference readers:
  main.txt        Schemi/main/Schemi.cpp:101-163 (24 positional "#label value" pairs)
  g.txt           Schemi/main/Schemi.cpp:83-99
  sub_k.txt       Schemi/src/thermodynamics/phaseInitialization.cpp:256-330
  velocity.txt, pressure.txt, k/epsilon/a/b.txt: 6 patch BCs then #Values_in_zones
  zonesDescription.txt   Schemi/src/service/zone.cpp:24-126
  output_NNNNNN.tsv / .dat      Schemi/src/service/output.cpp:14-308 (20 significant digits)
Labels are skipped by the reference readers; values are positional.
"""

from __future__ import annotations

import os
from typing import Dict, Optional, Sequence

import numpy as np

from .case import PATCHES, PATCHES_USED, Case

_PATCH_LABELS = ["#Tail_boundary_condition", "#Point_boundary_condition", "#Bottom_boundary_condition",
                 "#Right_boundary_condition", "#Left_boundary_condition", "#Top_boundary_condition"]

# Inert model files the reference parses even when diffusion and turbulence are off.
_TRANSPORT = """#Transport_coefficient_model
constant
#Viscosity_coefficient
2E-5
#Diffusion_coefficient
2E-5
#Heat_conduction_coefficient
2E-2
#Flag_for_enthalpy_flow_solution
explicit
#Flag_for_molar_mass_diffusion_correction
on"""

def _transport_block(case):
    """set/transportCoefficients.txt of a diffusion deck (phaseInitialization.cpp:193-243)."""
    return "\n".join([
        "#Transport_coefficient_model", case.transport,
        "#Viscosity_coefficient", _f(case.mu),
        "#Diffusion_coefficient", _f(case.D),
        "#Heat_conduction_coefficient", _f(case.kappa),
        "#Flag_for_enthalpy_flow_solution", case.enthalpy_flow,
        "#Flag_for_molar_mass_diffusion_correction", "on" if case.molmass_diffusion else "off",
    ])


_TURB_PARAMS = """#Cmu
0.09
#Turbulent_Schmidt
0.7
#Turbulent_Prandtl_T
0.7
#Turbulent_Prandtl_e
1E6
#sigma_k
0.7
#sigma_epsilon
0.6
#sigma_a
1.4
#sigma_b
0.7
#CMS_R
1E-1
#CMS_D
1E0
#Minimal_k
1E-15
#Minimal_epsilon
1E-15
#Minimal_b
1E-15
#C0
0.92
#C1
1.44
#C2
1.92
#C3
2.0
#C4
1.1
#Ca
2.5
#Cb1
2.0
#Cb2
5.0
#alpha_2
0.15
#alpha_3
0.2
#alpha_4
0.1
#CMS_M
1.0"""

_TURB_PEAK = """#Type_of_peak
no
#Maximum_k
1
#Maximum_epsilon
1000
#Center_coordinate
1.0
#Left_width
0.005
#Right_width
0.005"""

_GONCHAROV = """off
#Number_of_particles
1
#Initialisation_check_type
viaRe
#Initial_data
0.51 0.2 0.2 1 2 2 7E-4 1E-2 1E15"""


def _f(x: float) -> str:
    return repr(float(x))


def _bc_block(case: Case, getter, vector: bool) -> str:
    used = PATCHES_USED[case.dims]
    lines = []
    for label, pname in zip(_PATCH_LABELS, PATCHES):
        lines.append(label)
        if pname in used:
            lines.append(getter(case.bc[pname]).task_string(vector))
        else:
            lines.append("blank")
    return "\n".join(lines)


def _chemistry_block(case: Case) -> str:
    """set/chemicalKinetics.txt: the mechanism name, then the Arrhenius parameters, solver and
    iteration count in the order ChlorumDissociation's constructor reads them
    (chemicalKineticsChlorumDissociation.cpp:275-308)."""
    if case.chemistry == "no":
        return "#Type_of_chemical_reaction\nno"
    if case.chemistry != "Cl2":
        raise ValueError(f"the reference has no {case.chemistry} mechanism")
    (af, nf, ef), (ab, nb, eb) = case.chem_forward, case.chem_backward
    lines = ["#Type_of_chemical_reaction", "Cl2",
             "#A_forw", _f(af), "#n_forw", _f(nf), "#E_forw", _f(ef),
             "#A_backw", _f(ab), "#n_backw", _f(nb), "#E_backw", _f(eb),
             "#Iterative_solver", case.chem_solver,
             "#Number_of_chemical_solver_iterations", str(case.chem_max_iter)]
    return "\n".join(lines)


def write_deck(case: Case, directory: str, prim: Sequence[np.ndarray], frequency_of_output: int = 1,
               restart: bool = True, zones=None, modifiers=None, mixing_width: bool = False) -> None:
    """Write ``directory/set`` and the restart point for the reference solver.

    ``prim`` is the restart set c_1..c_N, v_x, v_y, v_z, p (flattened in cell order, x fastest);
    the outer zone of the initial fields takes its means.  ``zones``: zones before the outer one,
    each ``(description, [c_1..c_N], (v_x, v_y, v_z), p)`` with the description in the syntax of
    zonesDescription.txt (zone.cpp:25-125), e.g. ``"sphere 0.5 0.5 0.5 0.2"`` or
    ``"plane 0 1 0 point: 0 0.5 0"``.  ``modifiers``: ``{k: (A, B, x0, c)}`` written as
    ``set/sub_<k>_modifFunction.txt`` (gaussian, phaseInitialization.cpp:1197-1228).
    ``mixing_width``: ``#Calculation_of_mixing_zone_width on`` (a 1D task then writes
    ``result/timeWidth.tsv``).
    """
    zones = list(zones or [])
    if not case.expressible_in_reference():
        raise ValueError("the reference has no periodic patch or A+B->2C mechanism")
    N = case.n_species
    sdir = os.path.join(directory, "set")
    os.makedirs(sdir, exist_ok=True)
    nx, ny, nz = case.n
    dims_name = {1: "1D", 2: "2D", 3: "3D"}[case.dims]
    ncell = [nx, ny if case.dims >= 2 else 1, nz if case.dims >= 3 else 1]
    # "<type>=<source coefficient>,<diffusion coefficient>" (Schemi.cpp:180-243)
    src_ts = ("Courant" if case.courant_only else
              "Courant-Source-Diffusion" if case.diffusion_timestep else "Courant-Source") + \
        f"={_f(case.dt_coeffs[0])},{_f(case.dt_coeffs[1])}"
    main = [
        ("#Radius-vector_of_system's_parallelepiped", " ".join(_f(x) for x in case.L)),
        ("#Number_of_cells_in_direction", " ".join(str(x) for x in ncell)),
        ("#Time_of_calculation", _f(case.t_end)),
        ("#Courant_number", _f(case.courant)),
        ("#Frequency_of_output", str(frequency_of_output)),
        ("#Minimal_timestep", _f(case.min_timestep)),
        ("#Number_of_components", str(N)),
        ("#Defines_universal_gas_constant", case.R_units),
        ("#Equation_of_state", case.eos),
        ("#TVD_limiter_type", case.limiter),
        ("#Number_of_iterations_of_SLE_matrix_solver", str(case.sle_max_iter)),
        ("#Diffusion_flag", "on" if case.diffusion else "off"),
        ("#Turbulence_flag", "off"),
        ("#Type_of_SLE_solver_flag", case.sle_solver if case.diffusion else "GaussSeidel"),
        ("#Type_of_source_flag", "BHR"),
        ("#Type_of_flow_solver", case.flux),
        ("#Dimensions_of_the_task", dims_name),
        ("#Constant_timestep", _f(case.const_timestep) if case.const_timestep > 0 else "-1E-8"),
        ("#Source_timestep_correction", src_ts),
        ("#Reconstruction", case.reconstruction),
        ("#Approximation_order", case.order),
        ("#Start_From_Time-Step", "1" if restart else "no"),
        ("#Calculation_of_mixing_zone_width", "on" if mixing_width else "off"),
        ("#Nonlinearity_iterations", "off"),
    ]
    _write(sdir, "main.txt", "\n".join(f"{k}\n{v}" for k, v in main))
    g = case.gravity or (0.0, 0.0, 0.0)
    _write(sdir, "g.txt", "#Free_fall_acceleration_flag\n" + ("on" if case.gravity is not None else "off") +
           "\n#Free_fall_acceleration_vector_components\n" + " ".join(_f(x) for x in g) +
           "\n#Acceleration_growth\n" + " ".join(_f(x) for x in case.g_delta))
    # the zones, then the outer zone (a restart takes the fields from the restart point instead)
    _write(sdir, "zonesDescription.txt", f"#Number_of_zones\n{len(zones)}\n#Outer_zone: yes\n#Zones_description" +
           "".join("\n" + z[0] for z in zones))
    mean = [float(np.mean(a)) for a in prim]
    zone_c = [[_f(z[1][k]) for z in zones] + [_f(mean[k])] for k in range(N)]
    zone_v = " ".join(_f(x) for z in zones for x in z[2]) + (" " if zones else "") + " ".join(_f(x) for x in mean[N:N + 3])
    zone_p = " ".join([_f(z[3]) for z in zones] + [_f(mean[N + 3])])
    nzv = len(zones) + 1
    for k, sp in enumerate(case.species):
        body = [
            "#Molar_mass_(kg/mol)", _f(sp.M),
            "#Molar_isohoric_heat_capacity_(J/T/mol)", _f(sp.Cv),
            "#Critical_temperature_(K)", _f(sp.Tc),
            "#Critical_pressure_(Pa)", _f(sp.Pc),
            "#Kinetic_diameter_(A)", _f(sp.diameter),
            "#Lennard_Jones_eps/kB_(K)", _f(sp.tr_eps),
            "#Lennard_Jones_sigma_(A)", _f(sp.tr_sigma),
            _bc_block(case, lambda pb, k=k: pb.conc[k], False),
            "#Values_in_zones", " ".join(zone_c[k]),
        ]
        _write(sdir, f"sub_{k + 1}.txt", "\n".join(body))
    for k, (A, B, x0, w) in (modifiers or {}).items():
        _write(sdir, f"sub_{k}_modifFunction.txt",
               f"#Function\ngaussian\n#A\n{_f(A)}\n#B\n{_f(B)}\n#x0\n{_f(x0)}\n#c\n{_f(w)}")
    _write(sdir, "velocity.txt", _bc_block(case, lambda pb: pb.vel, True) + "\n#Values_in_zones\n" + zone_v)
    _write(sdir, "pressure.txt", _bc_block(case, lambda pb: pb.p, False) + "\n#Values_in_zones\n" + zone_p)
    free = "\n".join(f"{lab}\n{'freeBoundary' if p in PATCHES_USED[case.dims] else 'blank'}"
                     for lab, p in zip(_PATCH_LABELS, PATCHES))
    _write(sdir, "k.txt", free + "\n#Values_in_zones\n" + " ".join(["0.0"] * nzv))
    _write(sdir, "epsilon.txt", free + "\n#Values_in_zones\n" + " ".join(["0.0"] * nzv))
    _write(sdir, "a.txt", free + "\n#Values_in_zones\n" + " ".join(["0.0 0.0 0.0"] * nzv))
    _write(sdir, "b.txt", free + "\n#Values_in_zones\n" + " ".join(["0"] * nzv))
    if case.eos == "stiffened":
        # abstractMixtureThermodynamics.cpp:71-95: "<label> p0 gamma" per species
        _write(sdir, "stiffenedFluidData.txt",
               "\n".join(f"#sub_{k + 1} {_f(sp.p0)} {_f(sp.gamma)}" for k, sp in enumerate(case.species)))
    elif case.eos == "Kataoka":
        # abstractMixtureThermodynamics.cpp:96-143: "<label> eps sigma" per species, then the b rule
        _write(sdir, "KataokaVanDerWaalsFluidData.txt",
               "\n".join(f"#sub_{k + 1} {_f(sp.lj_eps)} {_f(sp.lj_sigma)}" for k, sp in enumerate(case.species))
               + f"\n#b_calculation {case.kataoka_b[0]} {_f(case.kataoka_b[1])}")
    _write(sdir, "chemicalKinetics.txt", _chemistry_block(case))
    _write(sdir, "transportCoefficients.txt", _transport_block(case) if case.diffusion else _TRANSPORT)
    _write(sdir, "turbulentParameters.txt", _TURB_PARAMS)
    _write(sdir, "turbPeak.txt", _TURB_PEAK)
    _write(sdir, "GoncharovModel.txt", _GONCHAROV)
    _write(sdir, "MPIRanks.txt", "#MPI_nodes_in_directions\n1 1 1")
    if restart:
        rdir = os.path.join(directory, "fieldsOutput", "output_000001")
        os.makedirs(rdir, exist_ok=True)
        os.makedirs(os.path.join(directory, "result"), exist_ok=True)
        for k in range(N):
            _write_column(os.path.join(rdir, f"sub_{k + 1}.dat"), [prim[k]])
        _write_column(os.path.join(rdir, "velocity.dat"), prim[N:N + 3])
        _write_column(os.path.join(rdir, "pressure.dat"), [prim[N + 3]])
        z = np.zeros(case.n_cells)
        for name in ("k", "epsilon", "b"):
            _write_column(os.path.join(rdir, f"{name}.dat"), [z])
        _write_column(os.path.join(rdir, "a.dat"), [z, z, z])
        with open(os.path.join(directory, "result", "Time.tsv"), "w") as f:
            f.write("0\t0\n1\t0\n")


def _write(d: str, name: str, text: str) -> None:
    with open(os.path.join(d, name), "w") as f:
        f.write(text)


def _write_column(path: str, cols: Sequence[np.ndarray]) -> None:
    arr = np.stack([np.asarray(c, dtype=np.float64).reshape(-1) for c in cols], axis=1)
    np.savetxt(path, arr, fmt="%.20g", delimiter="\t")


def read_output(directory: str, index: int) -> Dict[str, np.ndarray]:
    """Columns of ``result/output_<index>.tsv`` as float64 arrays (cell order as written)."""
    path = os.path.join(directory, "result", f"output_{index:06d}.tsv")
    with open(path) as f:
        header = f.readline().rstrip("\n").split("\t")
    data = np.loadtxt(path, skiprows=1, dtype=np.float64, ndmin=2)
    return {name: data[:, i] for i, name in enumerate(header) if name}


def read_times(directory: str) -> Dict[int, float]:
    out = {}
    with open(os.path.join(directory, "result", "Time.tsv")) as f:
        for line in f:
            parts = line.split("\t")
            if len(parts) == 2:
                out[int(parts[0])] = float(parts[1])
    return out


def read_restart(directory: str, index: int, n_species: int) -> list:
    """Restart set c_1..c_N, v_x, v_y, v_z, p of ``fieldsOutput/output_<index>`` (cell order)."""
    rdir = os.path.join(directory, "fieldsOutput", f"output_{index:06d}")
    out = [np.loadtxt(os.path.join(rdir, f"sub_{k + 1}.dat"), dtype=np.float64, ndmin=1) for k in range(n_species)]
    v = np.loadtxt(os.path.join(rdir, "velocity.dat"), dtype=np.float64, ndmin=2)
    out += [v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy()]
    out.append(np.loadtxt(os.path.join(rdir, "pressure.dat"), dtype=np.float64, ndmin=1))
    return out
