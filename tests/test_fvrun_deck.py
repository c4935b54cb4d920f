"""Task-deck driver (schemi_b200/lib/fvrun): deck parsing on the CPU.

``fvrun --print-config`` reads a deck the way the reference's main and phaseInitialization do
(Schemi/main/Schemi.cpp:83-310, Schemi/src/thermodynamics/phaseInitialization.cpp:256-446) and
prints the fv_config it maps to; these tests write decks with ``schemi_b200.deck`` and check that
the driver recovers the case, and that decks outside the step (diffusion, zones, unknown names)
are refused with the reference's messages or the driver's own.  The same driver source linked
against the CPU oracle (oracle/lib/fvrun_oracle) replays the reference's deck fixtures, so the
host side -- time loop, output schedule, restart, file writer -- is checked without a GPU.
"""

import json
import os
import subprocess

import pytest

from deck_replay import fixtures, load, replay, unpack_inputs
from schemi_b200 import cases
from schemi_b200.build import DRIVER
from schemi_b200.case import BC, PatchBC
from schemi_b200.deck import write_deck


def _driver():
    if not os.path.exists(DRIVER):
        pytest.fail(f"{DRIVER} is not built (python -m schemi_b200.build)")
    return DRIVER


def _print_config(d):
    res = subprocess.run([_driver(), "--print-config", d], capture_output=True, text=True, timeout=60)
    return res


def _deck_cases():
    out = []
    c, p = cases.kelvin_helmholtz_2d(n=8, periodic=False)
    out.append(("kh", c, p))
    c, p = cases.rayleigh_taylor_2d(nx=8, ny=16, modes=2)
    c.g_delta = (0.0, -0.05, 0.0)
    out.append(("rt", c, p))
    c, p = cases.chlorine_dissociation_2d(4)
    out.append(("cl2", c, p))
    c, p = cases.shock_tube_1d(n=40)
    c.bc["tail"] = PatchBC([BC("fixedValueCell", 0.7), BC("fixedValueCell", 0.3)],
                           BC("fixedValueCell", (0.3, 0.0, 0.0)), BC("fixedValueCell", 0.9))
    c.flux, c.limiter, c.courant_only, c.const_timestep = "HLL", "Schmidtmann", True, 1e-4
    out.append(("tube", c, p))
    c, p = cases.kelvin_helmholtz_2d(n=8, periodic=False)
    c.order = "SecondOrderRK"
    out.append(("kh_rk2", c, p))
    c, p = cases.shock_tube_1d(n=40)
    c.order = "ThirdOrderCada"
    out.append(("tube_cada", c, p))
    return out


@pytest.mark.parametrize("name,case,prim", _deck_cases(), ids=[c[0] for c in _deck_cases()])
def test_print_config_matches_case(tmp_path, name, case, prim):
    write_deck(case, str(tmp_path), prim, frequency_of_output=3, restart=True)
    res = _print_config(str(tmp_path))
    assert res.returncode == 0, res.stderr
    got = json.loads(res.stdout.strip().splitlines()[-1])
    want = case.fv_config()
    N = case.n_species
    assert got["dims"] == want.dims
    assert got["n"] == list(want.n)
    assert got["L"] == list(want.L)
    assert got["n_species"] == N
    assert got["R"] == want.R
    assert got["M"] == list(want.M)[:N]
    assert got["Cv"] == list(want.Cv)[:N]
    for key in ("eos", "flux", "limiter", "courant_only", "gravity", "chemistry"):
        assert got[key] == getattr(want, key), key
    assert got["courant"] == want.courant
    assert got["min_timestep"] == want.min_timestep
    # a case without a constant step is written with a negative #Constant_timestep
    if want.const_timestep > 0:
        assert got["const_timestep"] == want.const_timestep
    else:
        assert got["const_timestep"] <= 0
    assert got["g"] == list(want.g)
    assert got["bc_vel"] == list(want.bc_vel)
    assert got["bc_p"] == list(want.bc_p)
    assert got["order"] == want.order
    assert got["t_end"] == case.t_end
    assert got["frequency"] == 3
    assert got["start"] == "1"


def _edit(path, key, value):
    lines = open(path).read().split("\n")
    lines[lines.index(key) + 1] = value
    open(path, "w").write("\n".join(lines))


@pytest.mark.parametrize("file,key,value,message", [
    ("main.txt", "#Turbulence_flag", "yes", "Turbulence"),
    ("main.txt", "#Approximation_order", "FourthOrder", "Unknown gas dynamics approximation order."),
    ("main.txt", "#TVD_limiter_type", "vanLeer3", "limiter"),
    ("main.txt", "#Type_of_flow_solver", "KT", "HLLC"),
    ("main.txt", "#Source_timestep_correction", "Courant", "Wrong format of time-step parameters settings"),
    ("main.txt", "#Source_timestep_correction", "Implicit=0.25,0.5", "Unknown source time-step flag."),
    ("main.txt", "#Defines_universal_gas_constant", "Planck", "Unknown type of universal gas constant."),
    ("main.txt", "#Reconstruction", "cubic", "Unknown reconstruction flag."),
    ("main.txt", "#Equation_of_state", "BenedictWebbRubin", "Unknown type of equation of state."),
    ("main.txt", "#Equation_of_state", "stiffened", "stiffenedFluidData.txt not found."),
    ("main.txt", "#Equation_of_state", "Kataoka", "KataokaVanDerWaalsFluidData.txt not found."),
    ("zonesDescription.txt", "#Number_of_zones", "1", "end of file"),
    ("g.txt", "#Free_fall_acceleration_flag", "maybe", "Unknown gravitation flag."),
    ("chemicalKinetics.txt", "#Type_of_chemical_reaction", "H2Cl2Combustion", "not implemented"),
    # the Thomas solver is a 1D one (abstractMatrixSolver.cpp:57-58): on this 2D deck the name is
    # unknown to the factory
    ("main.txt", "#Type_of_SLE_solver_flag", "Thomas", "Unknown or inappropriate matrix solver flag."),
])
def test_unsupported_deck_refused(tmp_path, file, key, value, message):
    c, p = cases.kelvin_helmholtz_2d(n=8, periodic=False)
    write_deck(c, str(tmp_path), p, restart=True)
    _edit(os.path.join(tmp_path, "set", file), key, value)
    res = _print_config(str(tmp_path))
    assert res.returncode != 0
    assert message in res.stderr


def _diffusion_case():
    c, p = cases.shock_tube_1d(n=40)
    c.diffusion, c.mu, c.D, c.kappa = True, 1e-4, 1e-3, 1e-4
    c.enthalpy_flow, c.molmass_diffusion, c.diffusion_timestep = "explicit", True, True
    return c, p


def test_print_config_diffusion(tmp_path):
    """A diffusion deck: the stage's settings from main.txt and set/transportCoefficients.txt."""
    c, p = _diffusion_case()
    c.dt_coeffs = (0.3, 0.45)
    c.reconstruction = "linear"
    write_deck(c, str(tmp_path), p, restart=True)
    res = _print_config(str(tmp_path))
    assert res.returncode == 0, res.stderr
    got = json.loads(res.stdout.strip().splitlines()[-1])
    want = c.fv_config()
    for key in ("diffusion", "sle_solver", "transport", "enthalpy_flow", "molmass_diffusion",
                "linear_reconstruction", "diffusion_timestep"):
        assert got[key] == getattr(want, key), key
    for key in ("mu_const", "D_const", "kappa_const", "dt_coeff_source", "dt_coeff_diffusion"):
        assert got[key] == getattr(want, key), key


@pytest.mark.parametrize("model", ["hardSpheres", "LennardJones"])
def test_print_config_transport_models(tmp_path, model):
    """The transport model of set/transportCoefficients.txt and its species data from sub_k.txt
    (#Kinetic_diameter_(A), #Lennard_Jones_eps/kB_(K), #Lennard_Jones_sigma_(A)); the data a
    model does not read is left at zero."""
    c, p = _diffusion_case()
    c.transport = model
    for sp, d, e, sg in zip(c.species, (3.2, 1.6), (316.0, 130.0), (4.217, 3.0)):
        sp.diameter, sp.tr_eps, sp.tr_sigma = d, e, sg
    write_deck(c, str(tmp_path), p, restart=True)
    res = _print_config(str(tmp_path))
    assert res.returncode == 0, res.stderr
    got = json.loads(res.stdout.strip().splitlines()[-1])
    assert got["transport"] == {"hardSpheres": 1, "LennardJones": 2}[model]
    hs = model == "hardSpheres"
    assert got["transport_diameter"] == ([3.2, 1.6] if hs else [0, 0])
    assert got["transport_lj_eps"] == ([0, 0] if hs else [316.0, 130.0])
    assert got["transport_lj_sigma"] == ([0, 0] if hs else [4.217, 3.0])


@pytest.mark.parametrize("file,key,value,message", [
    ("main.txt", "#Type_of_SLE_solver_flag", "LU", "Unknown or inappropriate matrix solver flag."),
    ("main.txt", "#Type_of_flow_solver", "HLL", "the diffusion stage runs with HLLC"),
    ("main.txt", "#Approximation_order", "SecondOrderRK", "the diffusion stage runs with SecondOrder"),
    ("sub_1.txt", "#Kinetic_diameter_(A)", "wide", "not a number for kinetic diameter"),
    ("transportCoefficients.txt", "#Transport_coefficient_model", "Sutherland", "Unknown flag for transport model."),
    ("transportCoefficients.txt", "#Flag_for_enthalpy_flow_solution", "maybe",
     "Unknown flag for enthalpy flow calculation."),
    ("transportCoefficients.txt", "#Flag_for_molar_mass_diffusion_correction", "maybe",
     "Unknown flag for molar mass diffusion correction."),
])
def test_unsupported_diffusion_deck_refused(tmp_path, file, key, value, message):
    c, p = _diffusion_case()
    c.transport = "hardSpheres"
    write_deck(c, str(tmp_path), p, restart=True)
    _edit(os.path.join(tmp_path, "set", file), key, value)
    res = _print_config(str(tmp_path))
    assert res.returncode != 0
    assert message in res.stderr


def test_missing_deck_file(tmp_path):
    res = _print_config(str(tmp_path))
    assert res.returncode != 0
    assert "g.txt not found." in res.stderr


def test_deck_fixtures_parse(tmp_path):
    """Every committed deck fixture parses (its inputs written out, then --print-config), except
    the reference's refused deck, which fails to parse with the reference's message."""
    names = fixtures()
    assert len(names) >= 6
    for name in names:
        z = load(name)
        d = tmp_path / name
        unpack_inputs(z, str(d))
        for r in range(int(z["runs"])):
            (d / "set" / "main.txt").write_bytes(z[f"run{r}:main.txt"].tobytes())
            res = _print_config(str(d))
            if int(z["rc"][r]) == 0:
                assert res.returncode == 0, (name, res.stderr)
            else:
                assert res.returncode != 0, name
                assert res.stderr.strip().split("\n")[-1] in str(z["log_tails"][r]), (name, res.stderr)


SHIPPED = ["sod_cgs_1000", "blastwaves_cgs_3000", "gaussconcentration_cgs_1000", "noh_1_1000", "noh_2_1000",
           "rarefactions_100_cgs", "noh_cgs_1000"]


def test_shipped_decks_are_fixtures():
    """The reference's own in-scope task decks (1D, HLLC, vanAlbada, ideal gas, no diffusion or
    turbulence) are among the replayed fixtures, and its refused Noh_CGS deck with them."""
    assert set(SHIPPED) <= set(fixtures())
    z = load("noh_cgs_1000")
    assert int(z["rc"][0]) == 1
    assert "Unknown type of boundary condition" in str(z["log_tails"][0])


ORACLE_DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "lib",
                             "fvrun_oracle")


@pytest.mark.parametrize("name", fixtures())
def test_host_io_on_oracle_matches_reference_files(tmp_path, name):
    """The driver's deck reader, time loop, output schedule, restart and file writer, linked
    against the CPU oracle through the same C-ABI calls, reproduce the reference's files."""
    if not os.path.exists(ORACLE_DRIVER):
        subprocess.run(["make", "-s", "-C", os.path.dirname(os.path.dirname(ORACLE_DRIVER))], check=True)
    problems = replay(ORACLE_DRIVER, name, str(tmp_path))
    assert not problems, "\n".join(problems)


def _replace(path, old, new):
    text = open(path).read()
    assert old in text
    open(path, "w").write(text.replace(old, new))


def test_unknown_outer_zone_flag_refused(tmp_path):
    c, p = cases.kelvin_helmholtz_2d(n=8, periodic=False)
    write_deck(c, str(tmp_path), p, restart=False)
    _replace(os.path.join(tmp_path, "set", "zonesDescription.txt"), "#Outer_zone: yes", "#Outer_zone: maybe")
    res = _print_config(str(tmp_path))
    assert res.returncode != 0
    assert "Unknown flag for outer zone description." in res.stderr


@pytest.mark.parametrize("description,message", [
    ("cube 0 0 0 1", "Unknown zone type."),
    ("sphere 0.5 0.5 0.5 0", "Radius cannot be less or equal zero."),
])
def test_bad_zone_refused(tmp_path, description, message):
    c, p = cases.kelvin_helmholtz_2d(n=8, periodic=False)
    write_deck(c, str(tmp_path), p, restart=False,
               zones=[(description, [0.05, 0.02], (0.0, 0.0, 0.0), 2.5)])
    res = _print_config(str(tmp_path))
    assert res.returncode != 0
    assert message in res.stderr


def test_cells_outside_every_zone_refused(tmp_path):
    """Without the outer zone a cell outside every zone stops the fresh run with the reference's
    message (phaseInitialization.cpp:1188-1193)."""
    c, p = cases.kelvin_helmholtz_2d(n=8, periodic=False)
    write_deck(c, str(tmp_path), p, restart=False,
               zones=[("sphere 0.5 0.5 0.5 0.1", [0.05, 0.02], (0.0, 0.0, 0.0), 2.5)])
    _replace(os.path.join(tmp_path, "set", "zonesDescription.txt"), "#Outer_zone: yes", "#Outer_zone: no")
    res = subprocess.run([ORACLE_DRIVER, str(tmp_path)], capture_output=True, text=True, timeout=60)
    assert res.returncode != 0
    assert "Cell 0 of 1 component concentration dropped out of all zones." in res.stderr
